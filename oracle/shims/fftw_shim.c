/*
 * Project-written implementation of the FFTW3 subset declared in
 * oracle/shims/fftw3.h.  It exists so that the reference's own CPU renderer
 * (meshless_vis/meshless_vis_cpu.cpp, which calls fftwf_plan_dft_c2r_2d at
 * :64 and fftwf_execute at :261) can be built and run here, where FFTW is not
 * installed.  It is also the C2R used by the FP64 oracle (oracle.c).
 *
 * Semantics follow FFTW's documented unnormalised backward c2r transform:
 *   out[x][y] = sum_{kx, ky} X[kx][ky] exp(+2 pi i (kx x / n0 + ky y / n1))
 * over the full Hermitian extension of the [n0][n1/2+1] input.  It is computed
 * as a complex inverse DFT along axis 0 for each of the n1/2+1 columns, then a
 * real inverse along axis 1 that uses only the real part of the DC and (n1
 * even) Nyquist columns.  All arithmetic is double precision; power-of-two
 * lengths use an iterative radix-2 FFT, other lengths a direct DFT.
 *
 * Test infrastructure only.
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct mv_shim_fftwf_plan_s {
    int n0, n1;
    fftwf_complex* in;
    float* out;
};

void* fftwf_malloc(size_t n) {
    void* p = NULL;
    if (posix_memalign(&p, 64, n ? n : 64) != 0) return NULL;
    return p;
}
void fftwf_free(void* p) { free(p); }
int fftwf_init_threads(void) { return 1; }
void fftwf_plan_with_nthreads(int nthreads) { (void)nthreads; }
void fftwf_cleanup_threads(void) {}

fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex* in, float* out, unsigned flags) {
    (void)flags;
    fftwf_plan p = (fftwf_plan)malloc(sizeof(*p));
    p->n0 = n0;
    p->n1 = n1;
    p->in = in;
    p->out = out;
    return p;
}
void fftwf_destroy_plan(fftwf_plan p) { free(p); }

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* In-place inverse (sign +) complex transform of length n on re/im arrays. */
static void mv_inverse_dft(double* re, double* im, int n, double* wre, double* wim) {
    if (is_pow2(n)) {
        for (int i = 1, j = 0; i < n; i++) {
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) {
                double t = re[i]; re[i] = re[j]; re[j] = t;
                t = im[i]; im[i] = im[j]; im[j] = t;
            }
        }
        for (int len = 2; len <= n; len <<= 1) {
            double ang = 2.0 * M_PI / (double)len;
            for (int i = 0; i < n; i += len) {
                for (int k = 0; k < len / 2; k++) {
                    double c = cos(ang * k), s = sin(ang * k);
                    double ur = re[i + k], ui = im[i + k];
                    double vr = re[i + k + len / 2] * c - im[i + k + len / 2] * s;
                    double vi = re[i + k + len / 2] * s + im[i + k + len / 2] * c;
                    re[i + k] = ur + vr; im[i + k] = ui + vi;
                    re[i + k + len / 2] = ur - vr; im[i + k + len / 2] = ui - vi;
                }
            }
        }
        return;
    }
    for (int x = 0; x < n; x++) {
        double sr = 0.0, si = 0.0;
        for (int k = 0; k < n; k++) {
            double a = 2.0 * M_PI * (double)(((long long)k * x) % n) / (double)n;
            double c = cos(a), s = sin(a);
            sr += re[k] * c - im[k] * s;
            si += re[k] * s + im[k] * c;
        }
        wre[x] = sr;
        wim[x] = si;
    }
    memcpy(re, wre, sizeof(double) * n);
    memcpy(im, wim, sizeof(double) * n);
}

/* Exported for the oracle: FP64 C2R of a [n0][n1/2+1] complex array (re/im
 * interleaved doubles) into a [n0][n1] double image. */
void mvo_c2r_2d(const double* in, int n0, int n1, double* out) {
    int h = n1 / 2 + 1;
    int nmax = n0 > n1 ? n0 : n1;
    double* t = (double*)malloc(sizeof(double) * 2 * (size_t)n0 * h);
    double* re = (double*)malloc(sizeof(double) * nmax);
    double* im = (double*)malloc(sizeof(double) * nmax);
    double* wre = (double*)malloc(sizeof(double) * nmax);
    double* wim = (double*)malloc(sizeof(double) * nmax);
    for (int ky = 0; ky < h; ky++) {
        for (int kx = 0; kx < n0; kx++) {
            re[kx] = in[2 * ((size_t)kx * h + ky)];
            im[kx] = in[2 * ((size_t)kx * h + ky) + 1];
        }
        mv_inverse_dft(re, im, n0, wre, wim);
        for (int x = 0; x < n0; x++) {
            t[2 * ((size_t)x * h + ky)] = re[x];
            t[2 * ((size_t)x * h + ky) + 1] = im[x];
        }
    }
    for (int x = 0; x < n0; x++) {
        /* full Hermitian row of length n1, then a complex inverse transform */
        for (int ky = 0; ky < n1; ky++) {
            if (ky < h) {
                re[ky] = t[2 * ((size_t)x * h + ky)];
                im[ky] = t[2 * ((size_t)x * h + ky) + 1];
            } else {
                re[ky] = t[2 * ((size_t)x * h + (n1 - ky))];
                im[ky] = -t[2 * ((size_t)x * h + (n1 - ky)) + 1];
            }
        }
        im[0] = 0.0;
        if ((n1 & 1) == 0) im[n1 / 2] = 0.0;
        mv_inverse_dft(re, im, n1, wre, wim);
        for (int y = 0; y < n1; y++) out[(size_t)x * n1 + y] = re[y];
    }
    free(t); free(re); free(im); free(wre); free(wim);
}

void fftwf_execute(const fftwf_plan p) {
    int h = p->n1 / 2 + 1;
    size_t nin = (size_t)p->n0 * h, nout = (size_t)p->n0 * p->n1;
    double* in = (double*)malloc(sizeof(double) * 2 * nin);
    double* out = (double*)malloc(sizeof(double) * nout);
    for (size_t i = 0; i < nin; i++) {
        in[2 * i] = p->in[i][0];
        in[2 * i + 1] = p->in[i][1];
    }
    mvo_c2r_2d(in, p->n0, p->n1, out);
    for (size_t i = 0; i < nout; i++) p->out[i] = (float)out[i];
    free(in);
    free(out);
}
