/* Oracle build shim (test infrastructure only): stand-in for FFTW 3's <fftw3.h>.
 *
 * FFTW 3 (version unpinned by the reference: msvc FFTW3.x64.props links the
 * Windows prebuilt libfftw3-3 / libfftw3f-3 / libfftw3l-3) is not vendored with
 * the reference and is not installed here. The reference's BM3D path only ever
 * calls three FFTW entry points through include/fftw3_helper.hpp:
 *   fftw{,f,l}_plan_r2r_3d    (fftw3_helper.hpp:337-342 double, 837-842 float)
 *   fftw{,f,l}_execute_r2r    (fftw3_helper.hpp:346-349 double, 853-856 float)
 *   fftw{,f,l}_destroy_plan   (plan destructor)
 * with kinds FFTW_REDFT10 (forward) and FFTW_REDFT01 (backward)
 * (source/BM3D.cpp:13-23). Those three get real prototypes here and are
 * implemented in oracle/fftw_shim.cpp from FFTW's documented definitions.
 * Every other FFTW name that fftw3_helper.hpp mentions is declared as an
 * undefined variadic template so the helper compiles; none is ever called. */
#ifndef ORACLE_SHIM_FFTW3_H_
#define ORACLE_SHIM_FFTW3_H_

#include <cstddef>
#include <cstdio>

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED (1U << 1)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

enum oracle_fftw_r2r_kind {
    FFTW_R2HC = 0, FFTW_HC2R = 1, FFTW_DHT = 2,
    FFTW_REDFT00 = 3, FFTW_REDFT01 = 4, FFTW_REDFT10 = 5, FFTW_REDFT11 = 6,
    FFTW_RODFT00 = 7, FFTW_RODFT01 = 8, FFTW_RODFT10 = 9, FFTW_RODFT11 = 10
};

/* Value returned by the never-called stand-ins: converts to whatever the
 * helper assigns it to. */
struct oracle_fftw_any {
    template <typename T> operator T() const { return T(); }
};

/* One separable 3-D real-to-real plan (opaque to the reference). */
struct oracle_r2r_plan;

#define ORACLE_FFTW_TYPES(P, R)                                                   \
    typedef R P##_complex[2];                                                     \
    typedef oracle_r2r_plan P##_plan_s;                                           \
    typedef oracle_r2r_plan *P##_plan;                                            \
    typedef enum oracle_fftw_r2r_kind P##_r2r_kind;                               \
    struct P##_iodim64 { std::ptrdiff_t n, is, os; };                             \
    typedef void (*P##_write_char_func)(char c, void *);                          \
    typedef int (*P##_read_char_func)(void *);                                    \
    P##_plan_s *P##_plan_r2r_3d(int n0, int n1, int n2, R *in, R *out,           \
        P##_r2r_kind kind0, P##_r2r_kind kind1, P##_r2r_kind kind2, unsigned flags); \
    void P##_execute_r2r(const P##_plan_s *p, R *in, R *out);                     \
    void P##_destroy_plan(P##_plan_s *p);

ORACLE_FFTW_TYPES(fftw, double)
ORACLE_FFTW_TYPES(fftwf, float)
ORACLE_FFTW_TYPES(fftwl, long double)

#define ORACLE_FFTW_UNUSED(name) \
    template <typename... A> oracle_fftw_any name(A &&...);

ORACLE_FFTW_UNUSED(fftw_alignment_of)
ORACLE_FFTW_UNUSED(fftw_alloc_complex)
ORACLE_FFTW_UNUSED(fftw_alloc_real)
ORACLE_FFTW_UNUSED(fftw_cleanup)
ORACLE_FFTW_UNUSED(fftw_cleanup_threads)
ORACLE_FFTW_UNUSED(fftw_cost)
ORACLE_FFTW_UNUSED(fftw_estimate_cost)
ORACLE_FFTW_UNUSED(fftw_execute)
ORACLE_FFTW_UNUSED(fftw_execute_dft)
ORACLE_FFTW_UNUSED(fftw_execute_dft_c2r)
ORACLE_FFTW_UNUSED(fftw_execute_dft_r2c)
ORACLE_FFTW_UNUSED(fftw_execute_split_dft)
ORACLE_FFTW_UNUSED(fftw_execute_split_dft_c2r)
ORACLE_FFTW_UNUSED(fftw_execute_split_dft_r2c)
ORACLE_FFTW_UNUSED(fftw_export_wisdom)
ORACLE_FFTW_UNUSED(fftw_export_wisdom_to_file)
ORACLE_FFTW_UNUSED(fftw_export_wisdom_to_filename)
ORACLE_FFTW_UNUSED(fftw_export_wisdom_to_string)
ORACLE_FFTW_UNUSED(fftw_flops)
ORACLE_FFTW_UNUSED(fftw_forget_wisdom)
ORACLE_FFTW_UNUSED(fftw_fprint_plan)
ORACLE_FFTW_UNUSED(fftw_free)
ORACLE_FFTW_UNUSED(fftw_import_system_wisdom)
ORACLE_FFTW_UNUSED(fftw_import_wisdom)
ORACLE_FFTW_UNUSED(fftw_import_wisdom_from_file)
ORACLE_FFTW_UNUSED(fftw_import_wisdom_from_filename)
ORACLE_FFTW_UNUSED(fftw_import_wisdom_from_string)
ORACLE_FFTW_UNUSED(fftw_init_threads)
ORACLE_FFTW_UNUSED(fftw_malloc)
ORACLE_FFTW_UNUSED(fftw_plan_dft)
ORACLE_FFTW_UNUSED(fftw_plan_dft_1d)
ORACLE_FFTW_UNUSED(fftw_plan_dft_2d)
ORACLE_FFTW_UNUSED(fftw_plan_dft_3d)
ORACLE_FFTW_UNUSED(fftw_plan_dft_c2r)
ORACLE_FFTW_UNUSED(fftw_plan_dft_c2r_1d)
ORACLE_FFTW_UNUSED(fftw_plan_dft_c2r_2d)
ORACLE_FFTW_UNUSED(fftw_plan_dft_c2r_3d)
ORACLE_FFTW_UNUSED(fftw_plan_dft_r2c)
ORACLE_FFTW_UNUSED(fftw_plan_dft_r2c_1d)
ORACLE_FFTW_UNUSED(fftw_plan_dft_r2c_2d)
ORACLE_FFTW_UNUSED(fftw_plan_dft_r2c_3d)
ORACLE_FFTW_UNUSED(fftw_plan_guru64_dft)
ORACLE_FFTW_UNUSED(fftw_plan_guru64_dft_c2r)
ORACLE_FFTW_UNUSED(fftw_plan_guru64_dft_r2c)
ORACLE_FFTW_UNUSED(fftw_plan_guru64_r2r)
ORACLE_FFTW_UNUSED(fftw_plan_guru64_split_dft)
ORACLE_FFTW_UNUSED(fftw_plan_guru64_split_dft_c2r)
ORACLE_FFTW_UNUSED(fftw_plan_guru64_split_dft_r2c)
ORACLE_FFTW_UNUSED(fftw_plan_many_dft)
ORACLE_FFTW_UNUSED(fftw_plan_many_dft_c2r)
ORACLE_FFTW_UNUSED(fftw_plan_many_dft_r2c)
ORACLE_FFTW_UNUSED(fftw_plan_many_r2r)
ORACLE_FFTW_UNUSED(fftw_plan_r2r)
ORACLE_FFTW_UNUSED(fftw_plan_r2r_1d)
ORACLE_FFTW_UNUSED(fftw_plan_r2r_2d)
ORACLE_FFTW_UNUSED(fftw_plan_with_nthreads)
ORACLE_FFTW_UNUSED(fftw_print_plan)
ORACLE_FFTW_UNUSED(fftw_set_timelimit)
ORACLE_FFTW_UNUSED(fftw_sprint_plan)
ORACLE_FFTW_UNUSED(fftwf_alignment_of)
ORACLE_FFTW_UNUSED(fftwf_alloc_complex)
ORACLE_FFTW_UNUSED(fftwf_alloc_real)
ORACLE_FFTW_UNUSED(fftwf_cleanup)
ORACLE_FFTW_UNUSED(fftwf_cleanup_threads)
ORACLE_FFTW_UNUSED(fftwf_cost)
ORACLE_FFTW_UNUSED(fftwf_estimate_cost)
ORACLE_FFTW_UNUSED(fftwf_execute)
ORACLE_FFTW_UNUSED(fftwf_execute_dft)
ORACLE_FFTW_UNUSED(fftwf_execute_dft_c2r)
ORACLE_FFTW_UNUSED(fftwf_execute_dft_r2c)
ORACLE_FFTW_UNUSED(fftwf_execute_split_dft)
ORACLE_FFTW_UNUSED(fftwf_execute_split_dft_c2r)
ORACLE_FFTW_UNUSED(fftwf_execute_split_dft_r2c)
ORACLE_FFTW_UNUSED(fftwf_export_wisdom)
ORACLE_FFTW_UNUSED(fftwf_export_wisdom_to_file)
ORACLE_FFTW_UNUSED(fftwf_export_wisdom_to_filename)
ORACLE_FFTW_UNUSED(fftwf_export_wisdom_to_string)
ORACLE_FFTW_UNUSED(fftwf_flops)
ORACLE_FFTW_UNUSED(fftwf_forget_wisdom)
ORACLE_FFTW_UNUSED(fftwf_fprint_plan)
ORACLE_FFTW_UNUSED(fftwf_free)
ORACLE_FFTW_UNUSED(fftwf_import_system_wisdom)
ORACLE_FFTW_UNUSED(fftwf_import_wisdom)
ORACLE_FFTW_UNUSED(fftwf_import_wisdom_from_file)
ORACLE_FFTW_UNUSED(fftwf_import_wisdom_from_filename)
ORACLE_FFTW_UNUSED(fftwf_import_wisdom_from_string)
ORACLE_FFTW_UNUSED(fftwf_init_threads)
ORACLE_FFTW_UNUSED(fftwf_malloc)
ORACLE_FFTW_UNUSED(fftwf_plan_dft)
ORACLE_FFTW_UNUSED(fftwf_plan_dft_1d)
ORACLE_FFTW_UNUSED(fftwf_plan_dft_2d)
ORACLE_FFTW_UNUSED(fftwf_plan_dft_3d)
ORACLE_FFTW_UNUSED(fftwf_plan_dft_c2r)
ORACLE_FFTW_UNUSED(fftwf_plan_dft_c2r_1d)
ORACLE_FFTW_UNUSED(fftwf_plan_dft_c2r_2d)
ORACLE_FFTW_UNUSED(fftwf_plan_dft_c2r_3d)
ORACLE_FFTW_UNUSED(fftwf_plan_dft_r2c)
ORACLE_FFTW_UNUSED(fftwf_plan_dft_r2c_1d)
ORACLE_FFTW_UNUSED(fftwf_plan_dft_r2c_2d)
ORACLE_FFTW_UNUSED(fftwf_plan_dft_r2c_3d)
ORACLE_FFTW_UNUSED(fftwf_plan_guru64_dft)
ORACLE_FFTW_UNUSED(fftwf_plan_guru64_dft_c2r)
ORACLE_FFTW_UNUSED(fftwf_plan_guru64_dft_r2c)
ORACLE_FFTW_UNUSED(fftwf_plan_guru64_r2r)
ORACLE_FFTW_UNUSED(fftwf_plan_guru64_split_dft)
ORACLE_FFTW_UNUSED(fftwf_plan_guru64_split_dft_c2r)
ORACLE_FFTW_UNUSED(fftwf_plan_guru64_split_dft_r2c)
ORACLE_FFTW_UNUSED(fftwf_plan_many_dft)
ORACLE_FFTW_UNUSED(fftwf_plan_many_dft_c2r)
ORACLE_FFTW_UNUSED(fftwf_plan_many_dft_r2c)
ORACLE_FFTW_UNUSED(fftwf_plan_many_r2r)
ORACLE_FFTW_UNUSED(fftwf_plan_r2r)
ORACLE_FFTW_UNUSED(fftwf_plan_r2r_1d)
ORACLE_FFTW_UNUSED(fftwf_plan_r2r_2d)
ORACLE_FFTW_UNUSED(fftwf_plan_with_nthreads)
ORACLE_FFTW_UNUSED(fftwf_print_plan)
ORACLE_FFTW_UNUSED(fftwf_set_timelimit)
ORACLE_FFTW_UNUSED(fftwf_sprint_plan)
ORACLE_FFTW_UNUSED(fftwl_alignment_of)
ORACLE_FFTW_UNUSED(fftwl_alloc_complex)
ORACLE_FFTW_UNUSED(fftwl_alloc_real)
ORACLE_FFTW_UNUSED(fftwl_cleanup)
ORACLE_FFTW_UNUSED(fftwl_cleanup_threads)
ORACLE_FFTW_UNUSED(fftwl_cost)
ORACLE_FFTW_UNUSED(fftwl_estimate_cost)
ORACLE_FFTW_UNUSED(fftwl_execute)
ORACLE_FFTW_UNUSED(fftwl_execute_dft)
ORACLE_FFTW_UNUSED(fftwl_execute_dft_c2r)
ORACLE_FFTW_UNUSED(fftwl_execute_dft_r2c)
ORACLE_FFTW_UNUSED(fftwl_execute_split_dft)
ORACLE_FFTW_UNUSED(fftwl_execute_split_dft_c2r)
ORACLE_FFTW_UNUSED(fftwl_execute_split_dft_r2c)
ORACLE_FFTW_UNUSED(fftwl_export_wisdom)
ORACLE_FFTW_UNUSED(fftwl_export_wisdom_to_file)
ORACLE_FFTW_UNUSED(fftwl_export_wisdom_to_filename)
ORACLE_FFTW_UNUSED(fftwl_export_wisdom_to_string)
ORACLE_FFTW_UNUSED(fftwl_flops)
ORACLE_FFTW_UNUSED(fftwl_forget_wisdom)
ORACLE_FFTW_UNUSED(fftwl_fprint_plan)
ORACLE_FFTW_UNUSED(fftwl_free)
ORACLE_FFTW_UNUSED(fftwl_import_system_wisdom)
ORACLE_FFTW_UNUSED(fftwl_import_wisdom)
ORACLE_FFTW_UNUSED(fftwl_import_wisdom_from_file)
ORACLE_FFTW_UNUSED(fftwl_import_wisdom_from_filename)
ORACLE_FFTW_UNUSED(fftwl_import_wisdom_from_string)
ORACLE_FFTW_UNUSED(fftwl_init_threads)
ORACLE_FFTW_UNUSED(fftwl_malloc)
ORACLE_FFTW_UNUSED(fftwl_plan_dft)
ORACLE_FFTW_UNUSED(fftwl_plan_dft_1d)
ORACLE_FFTW_UNUSED(fftwl_plan_dft_2d)
ORACLE_FFTW_UNUSED(fftwl_plan_dft_3d)
ORACLE_FFTW_UNUSED(fftwl_plan_dft_c2r)
ORACLE_FFTW_UNUSED(fftwl_plan_dft_c2r_1d)
ORACLE_FFTW_UNUSED(fftwl_plan_dft_c2r_2d)
ORACLE_FFTW_UNUSED(fftwl_plan_dft_c2r_3d)
ORACLE_FFTW_UNUSED(fftwl_plan_dft_r2c)
ORACLE_FFTW_UNUSED(fftwl_plan_dft_r2c_1d)
ORACLE_FFTW_UNUSED(fftwl_plan_dft_r2c_2d)
ORACLE_FFTW_UNUSED(fftwl_plan_dft_r2c_3d)
ORACLE_FFTW_UNUSED(fftwl_plan_guru64_dft)
ORACLE_FFTW_UNUSED(fftwl_plan_guru64_dft_c2r)
ORACLE_FFTW_UNUSED(fftwl_plan_guru64_dft_r2c)
ORACLE_FFTW_UNUSED(fftwl_plan_guru64_r2r)
ORACLE_FFTW_UNUSED(fftwl_plan_guru64_split_dft)
ORACLE_FFTW_UNUSED(fftwl_plan_guru64_split_dft_c2r)
ORACLE_FFTW_UNUSED(fftwl_plan_guru64_split_dft_r2c)
ORACLE_FFTW_UNUSED(fftwl_plan_many_dft)
ORACLE_FFTW_UNUSED(fftwl_plan_many_dft_c2r)
ORACLE_FFTW_UNUSED(fftwl_plan_many_dft_r2c)
ORACLE_FFTW_UNUSED(fftwl_plan_many_r2r)
ORACLE_FFTW_UNUSED(fftwl_plan_r2r)
ORACLE_FFTW_UNUSED(fftwl_plan_r2r_1d)
ORACLE_FFTW_UNUSED(fftwl_plan_r2r_2d)
ORACLE_FFTW_UNUSED(fftwl_plan_with_nthreads)
ORACLE_FFTW_UNUSED(fftwl_print_plan)
ORACLE_FFTW_UNUSED(fftwl_set_timelimit)
ORACLE_FFTW_UNUSED(fftwl_sprint_plan)

#endif
