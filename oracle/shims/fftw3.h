/*
 * Minimal single-precision FFTW3 interface, project-written, so that the
 * reference's CPU renderer (meshless_vis/meshless_vis_cpu.cpp) compiles and
 * runs without FFTW being installed.  Only the calls that file makes are
 * declared; oracle/shims/fftw_shim.c implements them with an FP64 direct DFT
 * (unnormalised, FFTW's sign convention for the backward transform).
 *
 * Test infrastructure only: this header and its implementation are linked into
 * oracle/_ref/libmeshless_vis_ref.so and never into the product library.
 */
#ifndef MV_SHIM_FFTW3_H
#define MV_SHIM_FFTW3_H

#include <stddef.h>
#include <string.h> /* the reference file calls memset/memcpy without <cstring> */

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct mv_shim_fftwf_plan_s* fftwf_plan;

#define FFTW_ESTIMATE (1U << 6)

void* fftwf_malloc(size_t n);
void fftwf_free(void* p);
int fftwf_init_threads(void);
void fftwf_plan_with_nthreads(int nthreads);
void fftwf_cleanup_threads(void);
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex* in, float* out, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);

#ifdef __cplusplus
}
#endif

#endif
