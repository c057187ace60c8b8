/*
 * FP64 oracle for the libMeshlessVis hot path.  TEST INFRASTRUCTURE ONLY:
 * tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py may load
 * it as a checker; the product library never links, loads or calls it.
 *
 * It restates, in double precision, the reference's algorithm for:
 *   - the basis-function transforms Phi^(r)
 *       meshless_vis/fourier_transform_cpu.cpp:37-66 (same branch points at
 *       0.06f / 0.24f, same closed forms and quadratic coefficients);
 *     plus GAUSSIAN_DECAYING = exp(-pi r^2), an appended basis with no
 *     reference twin (the reference Gaussian exp(+pi r^2) grows);
 *   - the direct slice sum  meshless_vis/fourier_transform_cpu.cpp:73-134
 *       (frequency index mapping :88-90, f = fu u + fv v :93-96,
 *        r = sqrt(fu^2+fv^2) :99, stored value (Re*scale, -Im*scale) :126-130,
 *        first group assigns / later groups accumulate :124-131);
 *   - arrange_samples  meshless_vis/meshless_vis_cpu.cpp:209-234;
 *   - the scale step.x*step.y  meshless_vis/meshless_vis_cpu.cpp:139-143;
 * and the new 3D-half-spectrum path, which has no reference twin:
 *   F(i,j,l) = sum_k w_k Phi^(s3 |(i,j,l)| h_k) exp(-2 pi i s3 (i,j,l).x_k)
 *   for i in [-Kx/2,Kx/2), j in [-Ky/2,Ky/2), l in [0,Kz/2], stored
 *   [i+Kx/2][j+Ky/2][l]; and the Fourier-slice extraction from it (trilinear
 *   interpolation, Hermitian fold for k_z < 0, zero outside the grid), the
 *   same scheme the CUDA slice kernel uses.
 *
 * Parity pin: this restatement is checked against the reference's own CPU code
 * (built verbatim from its sources into oracle/_ref by oracle/Makefile) and
 * against the golden vectors in tests/golden/ that the reference produced.
 *
 * Particles are passed as the reference's Constraint layout, 4 floats per
 * particle (x, y, z, weight), plus an optional float radius per particle
 * (NULL = "no radii": Phi^(r) is evaluated at r itself,
 * fourier_transform_cpu.cpp:113-118).
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

enum { MVO_SPH = 0, MVO_GAUSSIAN = 1, MVO_WENDLAND_D3_C2 = 2, MVO_GAUSSIAN_DECAYING = 3 };

void mvo_c2r_2d(const double* in, int n0, int n1, double* out); /* fftw_shim.c */

double mvo_phi(int basis, double r) {
    switch (basis) {
    case MVO_SPH:
        /* fourier_transform_cpu.cpp:37-47 */
        if (r >= (double)0.06f) {
            double m = M_PI * r, c = cos(2.0 * m), s = sin(2.0 * m);
            return (2.3561944901923448 / (m * m * m * m * m * m)) * (c - 1.0) * (c + m * s - 1.0);
        }
        return M_PI + r * (-0.007968913156311 + r * (-18.293608272337678));
    case MVO_GAUSSIAN:
        /* fourier_transform_cpu.cpp:49-52 (growing exponential, as written) */
        return exp(M_PI * r * r);
    case MVO_WENDLAND_D3_C2:
        /* fourier_transform_cpu.cpp:54-66 */
        if (r >= (double)0.24f) {
            double m = M_PI * r, c = cos(2.0 * m), s = sin(2.0 * m);
            double m2 = m * m, m4 = m2 * m2;
            return ((M_PI * 7.5) / (m4 * m4)) * (4.0 * m2 - 6.0 + (6.0 - m2) * c + 4.5 * m * s);
        }
        return 0.299199300341890 + r * (-0.002379178586124 + r * (-0.370530218163545));
    case MVO_GAUSSIAN_DECAYING:
        return exp(-M_PI * r * r);
    default:
        return 0.0;
    }
}

void mvo_phi_array(int basis, const double* r, int n, double* out) {
    for (int i = 0; i < n; i++) out[i] = mvo_phi(basis, r[i]);
}

/* Reference index -> signed u frequency, fourier_transform_cpu.cpp:88-90. */
static void slice_index(int index, int cx, int* x, int* y) {
    int xx = index % (2 * cx);
    if (xx > cx) xx -= 2 * cx;
    *x = xx;
    *y = index / (2 * cx);
}

/*
 * Direct slice sum of one group, reference semantics.  out has 2*cx*cy complex
 * values (re, im interleaved) in the reference's index order; accumulate != 0
 * adds to out (later groups), else assigns (first group).
 */
void mvo_slice_sum(const float* xyzw, const float* radii, int n, int basis, float step_x, float step_y,
                   int cx, int cy, const float* u, const float* v, int accumulate, double* out) {
    int size = 2 * cx * cy;
    double scale = (double)step_x * (double)step_y;
#pragma omp parallel for schedule(dynamic, 16)
    for (int index = 0; index < size; index++) {
        int x, y;
        slice_index(index, cx, &x, &y);
        double fu = (double)step_x * x, fv = (double)step_y * y;
        double f0 = fu * u[0] + fv * v[0], f1 = fu * u[1] + fv * v[1], f2 = fu * u[2] + fv * v[2];
        double r = sqrt(fu * fu + fv * fv);
        double sr = 0.0, si = 0.0;
        for (int k = 0; k < n; k++) {
            double t = mvo_phi(basis, radii ? r * (double)radii[k] : r);
            double ph = 2.0 * M_PI * (f0 * xyzw[4 * k] + f1 * xyzw[4 * k + 1] + f2 * xyzw[4 * k + 2]);
            double a = (double)xyzw[4 * k + 3] * t;
            sr += a * cos(ph);
            si += a * sin(ph);
        }
        if (accumulate) {
            out[2 * index] += sr * scale;
            out[2 * index + 1] += -si * scale;
        } else {
            out[2 * index] = sr * scale;
            out[2 * index + 1] = -si * scale;
        }
    }
}

/* arrange_samples, meshless_vis_cpu.cpp:209-234, into a zeroed [nx][ny/2+1]. */
void mvo_arrange(const double* slice, int cx, int cy, int nx, int ny, double* arranged) {
    int h = ny / 2 + 1;
    for (size_t i = 0; i < 2 * (size_t)nx * h; i++) arranged[i] = 0.0;
    for (int index = 0; index < 2 * cx * cy; index++) {
        int x = index % (2 * cx), y = index / (2 * cx), ix = x;
        if (x > cx) {
            x -= 2 * cx;
            ix = x + nx;
        }
        if (x == cx) continue;
        arranged[2 * ((size_t)ix * h + y)] = slice[2 * index];
        arranged[2 * ((size_t)ix * h + y) + 1] = slice[2 * index + 1];
    }
}

void mvo_c2r(const double* arranged, int nx, int ny, double* image) { mvo_c2r_2d(arranged, nx, ny, image); }

/*
 * 3D half-spectrum at an explicit list of integer wavenumber triples
 * (ijk[3*p..3*p+2]); out gets npts complex values.
 */
void mvo_spectrum_points(const float* xyzw, const float* radii, int n, int basis, double s3, const int* ijk,
                         int npts, double* out) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int p = 0; p < npts; p++) {
        double k0 = s3 * ijk[3 * p], k1 = s3 * ijk[3 * p + 1], k2 = s3 * ijk[3 * p + 2];
        double r = sqrt(k0 * k0 + k1 * k1 + k2 * k2);
        double sr = 0.0, si = 0.0;
        for (int k = 0; k < n; k++) {
            double t = mvo_phi(basis, radii ? r * (double)radii[k] : r);
            double ph = 2.0 * M_PI * (k0 * xyzw[4 * k] + k1 * xyzw[4 * k + 1] + k2 * xyzw[4 * k + 2]);
            double a = (double)xyzw[4 * k + 3] * t;
            sr += a * cos(ph);
            si -= a * sin(ph);
        }
        out[2 * p] = sr;
        out[2 * p + 1] = si;
    }
}

/* Full 3D half-spectrum, layout [i+Kx/2][j+Ky/2][l], l in [0,Kz/2]. */
void mvo_spectrum_grid(const float* xyzw, const float* radii, int n, int basis, double s3, int kx, int ky, int kz,
                       int accumulate, double* out) {
    int lz = kz / 2 + 1;
    long long total = (long long)kx * ky * lz;
#pragma omp parallel for schedule(dynamic, 64)
    for (long long q = 0; q < total; q++) {
        int l = (int)(q % lz);
        int j = (int)((q / lz) % ky) - ky / 2;
        int i = (int)(q / ((long long)lz * ky)) - kx / 2;
        double k0 = s3 * i, k1 = s3 * j, k2 = s3 * l;
        double r = sqrt(k0 * k0 + k1 * k1 + k2 * k2);
        double sr = 0.0, si = 0.0;
        for (int k = 0; k < n; k++) {
            double t = mvo_phi(basis, radii ? r * (double)radii[k] : r);
            double ph = 2.0 * M_PI * (k0 * xyzw[4 * k] + k1 * xyzw[4 * k + 1] + k2 * xyzw[4 * k + 2]);
            double a = (double)xyzw[4 * k + 3] * t;
            sr += a * cos(ph);
            si -= a * sin(ph);
        }
        if (accumulate) {
            out[2 * q] += sr;
            out[2 * q + 1] += si;
        } else {
            out[2 * q] = sr;
            out[2 * q + 1] = si;
        }
    }
}

static void spec_at(const double* spec, int kx, int ky, int kz, int i, int j, int l, double* re, double* im) {
    int lz = kz / 2 + 1;
    if (i < -kx / 2 || i >= kx - kx / 2 || j < -ky / 2 || j >= ky - ky / 2 || l < 0 || l >= lz) {
        *re = 0.0;
        *im = 0.0;
        return;
    }
    size_t q = ((size_t)(i + kx / 2) * ky + (size_t)(j + ky / 2)) * lz + l;
    *re = spec[2 * q];
    *im = spec[2 * q + 1];
}

/*
 * Fourier-slice extraction of one view from a 3D half-spectrum, written
 * straight into the C2R layout [nx][ny/2+1] (every element written; samples
 * that arrange_samples leaves out are zero).  Slice sample (x, y),
 * x in (-cx, cx), y in [0, cy): k = step.x x u + step.y y v, grid coordinate
 * p = k / s3; if p_z < 0 the sample is conj(F(-p)); F(p) is the trilinear
 * interpolation of the 8 surrounding grid values, zero outside the grid; the
 * value is multiplied by scale = step.x * step.y.
 */
void mvo_extract_slice(const double* spec, int kx, int ky, int kz, double s3, float step_x, float step_y, int cx,
                       int cy, const float* u, const float* v, int nx, int ny, double* arranged) {
    int h = ny / 2 + 1;
    double scale = (double)step_x * (double)step_y;
    for (int ix = 0; ix < nx; ix++) {
        int x;
        int valid_x = 1;
        if (ix < cx) x = ix;
        else if (ix > nx - cx) x = ix - nx;
        else { x = 0; valid_x = 0; }
        for (int y = 0; y < h; y++) {
            double vr = 0.0, vi = 0.0;
            if (valid_x && y < cy) {
                double fu = (double)step_x * x, fv = (double)step_y * y;
                double p0 = (fu * u[0] + fv * v[0]) / s3;
                double p1 = (fu * u[1] + fv * v[1]) / s3;
                double p2 = (fu * u[2] + fv * v[2]) / s3;
                int conj = 0;
                if (p2 < 0.0) {
                    p0 = -p0; p1 = -p1; p2 = -p2;
                    conj = 1;
                }
                double f0 = floor(p0), f1 = floor(p1), f2 = floor(p2);
                double t0 = p0 - f0, t1 = p1 - f1, t2 = p2 - f2;
                int i0 = (int)f0, j0 = (int)f1, l0 = (int)f2;
                for (int c = 0; c < 8; c++) {
                    int di = c & 1, dj = (c >> 1) & 1, dl = (c >> 2) & 1;
                    double wgt = (di ? t0 : 1.0 - t0) * (dj ? t1 : 1.0 - t1) * (dl ? t2 : 1.0 - t2);
                    double sr, si;
                    spec_at(spec, kx, ky, kz, i0 + di, j0 + dj, l0 + dl, &sr, &si);
                    vr += wgt * sr;
                    vi += wgt * si;
                }
                if (conj) vi = -vi;
                vr *= scale;
                vi *= scale;
            }
            arranged[2 * ((size_t)ix * h + y)] = vr;
            arranged[2 * ((size_t)ix * h + y) + 1] = vi;
        }
    }
}
