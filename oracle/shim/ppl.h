/* Oracle build shim (test infrastructure only).
 *
 * source/Image_Type.cpp:1 defines ENABLE_PPL, which makes include/Image_Type.hpp:30
 * include the MSVC Parallel Patterns Library. This stand-in runs
 * concurrency::parallel_for serially, so the oracle stays single-threaded like
 * the BM3D path itself (source/BM3D.cpp never enables PPL). */
#ifndef ORACLE_SHIM_PPL_H_
#define ORACLE_SHIM_PPL_H_

namespace concurrency {

template <typename Index, typename Func>
void parallel_for(Index first, Index last, const Func &func)
{
    for (Index i = first; i < last; ++i) func(i);
}

template <typename Index, typename Func>
void parallel_for(Index first, Index last, Index step, const Func &func)
{
    for (Index i = first; i < last; i += step) func(i);
}

}  // namespace concurrency

#endif
