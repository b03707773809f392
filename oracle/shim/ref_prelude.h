/* Oracle build shim (test infrastructure only), force-included with
 * `-include` before every reference translation unit.
 *
 * Two reference headers hold in-class explicit template specialisations
 * (include/Args.h:61-166, include/Histogram.h:28-30 and 59-61), which MSVC
 * accepts and GCC rejects. Neither is on the BM3D path: Args parses CLI flags
 * (BM3D_IO, include/BM3D.h:374-505) and Histogram is used only by
 * Conversion.hpp's ValidRange (auto-levels), which BM3D never reaches.
 * This prelude defines their include guards first and supplies minimal
 * stand-ins with the same names, so the reference's own headers and
 * source/BM3D.cpp + source/Image_Type.cpp compile unmodified, in place. */
#ifndef ORACLE_REF_PRELUDE_H_
#define ORACLE_REF_PRELUDE_H_

#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#define MW_ARGS_H_
#define HISTOGRAM_H_

/* Stand-in for include/Args.h (CLI only; never constructed by the oracle). */
class Args
{
public:
    Args(const int, const std::vector<std::string> &) {}
    void Check() const {}
    template <typename T> void GetPara(int &i, T &, int = 0) { ++i; }
};

/* Stand-in for include/Histogram.h (off the BM3D path). Any instantiation
 * aborts, so an accidental use cannot silently change results. */
template <typename _Ty = int>
class Histogram
{
public:
    template <typename... A> explicit Histogram(const A &...) { std::abort(); }
    template <typename P> void Add(const P &) { std::abort(); }
    _Ty Min(double = 0) const { std::abort(); }
    _Ty Max(double = 0) const { std::abort(); }
};

#endif
