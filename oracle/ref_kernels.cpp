/*
 * ref_kernels.cpp -- the reference's own OpenCL kernels (IAC/kernel.cl),
 * compiled unchanged for the host CPU.  TEST INFRASTRUCTURE ONLY.
 *
 * kernel.cl is not copied into this repository: the Makefile passes the path
 * of the file inside the reference checkout as IAC_KERNEL_CL and this unit
 * #includes it after a handful of macros that map the OpenCL C dialect onto
 * C++ (address-space qualifiers removed, get_global_id() read from a
 * thread-local work-item id, atomic_add/atomic_cmpxchg mapped to the GCC
 * __atomic builtins).  Each exported iacref_* function runs one NDRange launch:
 * every work item of the global range, spread over OpenMP threads.
 *
 * Output goes to oracle/_ref/libiacref.so, which is git-ignored; it is the
 * reference's arithmetic compiled with -ffp-contract=off and IEEE sqrtf.
 * The kernels' debug printf calls are compiled out.
 */
#include <cmath>
#include <cstdint>
#include <cstdio>

using std::cos;
using std::floor;
using std::round;
using std::sin;
using std::sqrt;

typedef unsigned long ulong;

static thread_local unsigned int iacref_gid;

#define __kernel static
#define __global
#define __constant static const
#define get_global_id(dim) (iacref_gid)
#define printf(...) ((void)0)

template <class T, class V>
static inline void atomic_add(volatile T *p, V v)
{
    __atomic_fetch_add(p, (T)v, __ATOMIC_RELAXED);
}
template <class T, class V>
static inline T atomic_cmpxchg(volatile T *p, V cmp, V val)
{
    T expected = (T)cmp;
    __atomic_compare_exchange_n(p, &expected, (T)val, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
    return expected;
}

#include IAC_KERNEL_CL

#undef printf

#define IACREF_LAUNCH(global, call)                                  \
    do {                                                             \
        _Pragma("omp parallel for schedule(dynamic, 8)")             \
        for (unsigned long g_ = 0; g_ < (unsigned long)(global); g_++) { \
            iacref_gid = (unsigned int)g_;                           \
            call;                                                    \
        }                                                            \
    } while (0)

extern "C" {

void iacref_AutoCorr_CQ_small(const float *I, const float *K, const double *P, unsigned long *out,
                              unsigned long global)
{
    IACREF_LAUNCH(global, AutoCorr_CQ_small(I, K, P, out));
}

/* first work item and count for row-sampled checks of the dense kernels */
void iacref_AutoCorr_CQ_small_rows(const float *I, const float *K, const double *P,
                                   unsigned long *out, unsigned long first, unsigned long count)
{
    _Pragma("omp parallel for schedule(dynamic, 8)")
    for (unsigned long g = first; g < first + count; g++) {
        iacref_gid = (unsigned int)g;
        AutoCorr_CQ_small(I, K, P, out);
    }
}

void iacref_Merge_CQ(const double *small, const float *RW, const double *P, unsigned long *out,
                     unsigned long global)
{
    IACREF_LAUNCH(global, Merge_CQ(small, RW, P, out));
}

void iacref_Autocor_sparseHL(const float *HL, const double *P, const float *R, unsigned long *out,
                             unsigned long global)
{
    IACREF_LAUNCH(global, Autocor_sparseHL(HL, P, R, out));
}

void iacref_AutoCorr_CQ_AV(const float *I, const float *K, const double *P, unsigned long *out,
                           unsigned long global)
{
    IACREF_LAUNCH(global, AutoCorr_CQ_AV(I, K, P, out));
}

void iacref_AutoCorr_CQ_AV_rows(const float *I, const float *K, const double *P,
                                unsigned long *out, unsigned long first, unsigned long count)
{
    _Pragma("omp parallel for schedule(dynamic, 8)")
    for (unsigned long g = first; g < first + count; g++) {
        iacref_gid = (unsigned int)g;
        AutoCorr_CQ_AV(I, K, P, out);
    }
}

void iacref_SimulateCrystal(const float *PM, const float *EM, const double *P, float *out,
                            unsigned long global)
{
    IACREF_LAUNCH(global, SimulateCrystal(PM, EM, P, out));
}

void iacref_AutoCorr_sparseHL_AAV(const float *HL, const double *P, unsigned long *out,
                                  unsigned long global)
{
    IACREF_LAUNCH(global, AutoCorr_sparseHL_AAV(HL, P, out));
}

} /* extern "C" */
