// Plain FP32 form of the Fourier sum (the reference's
// sample_fourier_transform_over_grid, meshless_vis/fourier_transform.cu:67-141,
// generalised to any integer lattice of wavenumbers: the reference's 2D
// slice, or the 3D half-spectrum).
//
// Work decomposition.  Thread = one lattice row segment: L consecutive x for
// one (y, z).  Block = 256 such threads.  Grid.y = split of the particle range
// (split-K, the reference's "partial sums", meshless_vis/fourier_transform.cu:
// 80-83), each split writing FP32 partial sums to a workspace that the
// finalize kernel reduces in FP64.
//
// Phase.  Per particle tile (256 particles staged in shared memory by the
// block) the loader converts each position to fixed-point turns per lattice
// axis, Q_a = round(2^32 (M p)_a) mod 2^32, in FP64, and the x-step rotation
// R = exp(2 pi i Qx / 2^32) with an FP64 sincospi.  A thread forms the exact
// integer phase of its first term, x0 Qx + y Qy + z Qz mod 2^32 (wrapping
// 32-bit multiply-add), takes one SFU sincos of it, and reaches its other L-1
// terms by complex multiplication with R.  The reference instead forms
// 2 pi f.x in FP32 and calls __sincosf per term on an unreduced argument
// (fourier_transform.cu:125), whose error grows with |f.x|.
//
// Amplitude w_j Phi^(|k| h_j):
//   - groups without radii: Phi^(|k|) is applied per frequency in FP64 by the
//     finalize kernel (it does not depend on the particle);
//   - SPH / Wendland with radii: Phi^ is read from a shared-memory table of
//     cubic pieces on node-centred cells of width ds (a branch point of the
//     reference's piecewise definition falls on a cell boundary), built per
//     launch in FP64 by phi_table_kernel; max error ~1.1e-7 of Phi^(0); terms
//     beyond the table (s > 63 for Wendland, > 60 for SPH, where |Phi^| <
//     1e-11) and terms of negative radii read its last, all-zero cell;
//   - Gaussians with radii: exp2 per term.
//
// Accumulation: each tile's terms are summed in FP32 registers; the tile sums
// go into FP64 running sums in global scratch (folded kernel) or are added
// with Kahan compensation in registers (unfolded kernel); splits are reduced
// in FP64.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "meshless.h"
#include "mv_device.cuh"
#include "mv_internal.h"

namespace mv {

namespace {

constexpr int kThreads = 256;  // threads per block == particles per tile
constexpr int kMaxTable = 4096;  // cubic cells held in shared memory (64 KB)

// kAmpGaussRec: decaying Gaussian exp(-pi h^2 |k|^2) factored as
// exp(-pi h^2 (y^2+z^2)) (one exp2 per particle and thread) times the x factor
// g(x) = exp(-pi h^2 x^2), advanced along the thread's L terms by
// g(x+1) = g(x) q(x), q(x+1) = q(x) exp(-2 pi h^2).  An x factor that
// underflows FP32 stays below 1e-28 over 8 steps, so nothing significant is
// lost.
// kAmpShell: the branch part of an h-binned group (fold kernel only): the
// table holds Phi^ minus its smooth closed form (zero from the branch point
// on), particles come sorted by h-bin, and a term counts only when the
// particle's bin is the one holding r0 / |k| (see fold_sum_kernel).
enum Amp : int { kAmpFactored = 0, kAmpTable = 1, kAmpExp2 = 2, kAmpGaussRec = 3, kAmpShell = 4 };

struct SumKernelArgs {
    const float4* particles;
    const float* radii;
    int n;
    int chunk;  // particles per split (multiple of kThreads)
    Lattice lat;
    int nxc;     // number of x chunks of L
    int n_rest;  // ny * nz
    float2* partial;  // [split][nxc * L][n_rest]
    const float4* table;  // cubic cells (kAmpTable); cell table_n is all zero
    int table_n;
    float inv_ds;  // 1 / cell width (kAmpTable)
    float amp_scale;  // kAmpExp2: +-pi log2(e)
};

template <int L, int BASIS, int AMP>
__global__ void __launch_bounds__(kThreads, 2) plain_sum_kernel(SumKernelArgs a) {
    extern __shared__ float4 s_tab[];  // table cells (kAmpTable only)
    __shared__ uint4 s_q[kThreads];    // Qx, Qy, Qz, weight bits
    __shared__ float2 s_rot[kThreads];  // exp(2 pi i Qx / 2^32)
    __shared__ float s_h[kThreads];    // per-particle amplitude parameter

    const int tid = threadIdx.x;
    if constexpr (AMP == kAmpTable) {
        for (int i = tid; i <= a.table_n; i += kThreads) s_tab[i] = a.table[i];
    }

    const long long t = (long long)blockIdx.x * kThreads + tid;
    const bool active = t < (long long)a.nxc * a.n_rest;
    const int xc = active ? (int)(t / a.n_rest) : 0;
    const int rest = active ? (int)(t % a.n_rest) : 0;
    const int y = a.lat.y0 + rest / a.lat.nz;
    const int z = a.lat.z0 + rest % a.lat.nz;
    const int xb = a.lat.x0 + xc * L;

    // |k| (kAmpTable) or |k|^2 (kAmpExp2) of the thread's L terms.
    float r[L];
    float ryz2 = 0.f;  // kAmpGaussRec: (ky y)^2 + (kz z)^2
    if constexpr (AMP == kAmpGaussRec) {
        const double ry = a.lat.ky * y, rz = a.lat.kz * z;
        ryz2 = (float)(ry * ry + rz * rz);
        const double rx = a.lat.kx * xb;
        r[0] = (float)(rx * rx);                            // (kx x0)^2
        r[1] = (float)(a.lat.kx * a.lat.kx * (2.0 * xb + 1));  // exponent of q(x0), per unit -pi h^2
        r[2] = (float)(2.0 * a.lat.kx * a.lat.kx);             // exponent of q's ratio
    } else if constexpr (AMP != kAmpFactored) {
        const double ry = a.lat.ky * y, rz = a.lat.kz * z;
#pragma unroll
        for (int m = 0; m < L; ++m) {
            const double rx = a.lat.kx * (xb + m);
            const double r2 = rx * rx + ry * ry + rz * rz;
            r[m] = AMP == kAmpTable ? (float)sqrt(r2) : (float)r2;
        }
    }

    float2 tot[L], comp[L];
#pragma unroll
    for (int m = 0; m < L; ++m) {
        tot[m] = make_float2(0.f, 0.f);
        comp[m] = make_float2(0.f, 0.f);
    }

    const int beg = blockIdx.y * a.chunk;
    const int end = min(a.n, beg + a.chunk);
    const uint32_t ux = (uint32_t)xb, uy = (uint32_t)y, uz = (uint32_t)z;

    for (int t0 = beg; t0 < end; t0 += kThreads) {
        __syncthreads();
        const int idx = t0 + tid;
        if (idx < end) {
            const float4 p = a.particles[idx];
            const double px = p.x, py = p.y, pz = p.z;
            const double* m = a.lat.m;
            const uint32_t qx = fixed_turns(m[0] * px + m[1] * py + m[2] * pz);
            s_q[tid] = make_uint4(qx, fixed_turns(m[3] * px + m[4] * py + m[5] * pz),
                                  fixed_turns(m[6] * px + m[7] * py + m[8] * pz), __float_as_uint(p.w));
            double sn, cs;
            sincospi((double)(int32_t)qx * (1.0 / 2147483648.0), &sn, &cs);
            s_rot[tid] = make_float2((float)cs, (float)sn);
            if constexpr (AMP == kAmpTable) s_h[tid] = a.radii[idx] * a.inv_ds;
            else if constexpr (AMP == kAmpExp2 || AMP == kAmpGaussRec) {
                const float h = a.radii[idx];
                s_h[tid] = a.amp_scale * h * h;
            }
        }
        __syncthreads();
        const int cnt = min(kThreads, end - t0);

        float2 acc[L];
#pragma unroll
        for (int m = 0; m < L; ++m) acc[m] = make_float2(0.f, 0.f);

#pragma unroll 2
        for (int j = 0; j < cnt; ++j) {
            const uint4 q = s_q[j];
            const float2 R = s_rot[j];
            float hv = 0.f;
            if constexpr (AMP != kAmpFactored) hv = s_h[j];
            const uint32_t ph = ux * q.x + uy * q.y + uz * q.z;
            float sn, cs;
            __sincosf(turns_to_radians(ph), &sn, &cs);
            float w = __uint_as_float(q.w);
            float Rx = R.x, Ry = R.y, qc = 1.f;
            if constexpr (AMP == kAmpGaussRec) {
                // hv = -pi log2(e) h^2
                w *= exp2f(hv * (ryz2 + r[0]));
                const float q0 = exp2f(hv * r[1]);
                qc = exp2f(hv * r[2]);
                Rx *= q0;
                Ry *= q0;
            }
            float zr = w * cs, zi = w * sn;
#pragma unroll
            for (int m = 0; m < L; ++m) {
                if constexpr (AMP == kAmpFactored || AMP == kAmpGaussRec) {
                    acc[m].x += zr;
                    acc[m].y += zi;
                } else {
                    float amp;
                    if constexpr (AMP == kAmpTable) {
                        const float u = r[m] * hv;  // s / ds
                        const float tt = u + 12582912.0f;  // round to nearest cell (1.5 * 2^23)
                        // beyond the table (and for negative radii) the last,
                        // all-zero cell is used
                        const unsigned k = min((unsigned)(__float_as_int(tt) - 0x4B400000), (unsigned)a.table_n);
                        const float fr = u - (tt - 12582912.0f);
                        const float4 c = s_tab[k];
                        amp = fmaf(fmaf(fmaf(c.w, fr, c.z), fr, c.y), fr, c.x);
                    } else {
                        amp = exp2f(hv * r[m]);
                    }
                    acc[m].x = fmaf(amp, zr, acc[m].x);
                    acc[m].y = fmaf(amp, zi, acc[m].y);
                }
                if (m + 1 < L) {
                    const float nr = fmaf(zr, Rx, -zi * Ry);
                    const float ni = fmaf(zr, Ry, zi * Rx);
                    zr = nr;
                    zi = ni;
                    if constexpr (AMP == kAmpGaussRec) {
                        Rx *= qc;
                        Ry *= qc;
                    }
                }
            }
        }
        // Kahan: add this tile's sums to the running totals.
#pragma unroll
        for (int m = 0; m < L; ++m) {
            float yv = acc[m].x - comp[m].x;
            float tv = tot[m].x + yv;
            comp[m].x = (tv - tot[m].x) - yv;
            tot[m].x = tv;
            yv = acc[m].y - comp[m].y;
            tv = tot[m].y + yv;
            comp[m].y = (tv - tot[m].y) - yv;
            tot[m].y = tv;
        }
    }

    if (!active) return;
    const size_t plane = (size_t)a.nxc * L * a.n_rest;
    float2* out = a.partial + blockIdx.y * plane + (size_t)(xc * L) * a.n_rest + rest;
#pragma unroll
    for (int m = 0; m < L; ++m) out[(size_t)m * a.n_rest] = make_float2(tot[m].x - comp[m].x, tot[m].y - comp[m].y);
}

// Folded form: the lattice's x range holds 0 (and, with FY == 2, so does its
// y range).  |k| and every Phi^ factor are even in x and in y, and the phase
// at (-x, y, z) is that at (x, y, z) with the x part conjugated:
//   e^{i n.Q} at (sx xp, sy yp, z) = c^{sx} d_{sy},  c = e^{i xp Qx},
//   d_{+-} = w e^{i (+-yp Qy + z Qz)}.
// A thread owns L representatives xp = xc L + m >= 0, one yp >= 0 (FY == 2;
// FY == 1: one y of the lattice) and one z, and sums the terms at (+-xp, yp)
// (and (+-xp, -yp)) together: one amplitude evaluation and one x rotation
// serve up to four lattice points.  With u = amp c, the four real sums
//   A0 = sum ur dr, A1 = sum ui di, A2 = sum ur di, A3 = sum ui dr
// give T(+xp) = (A0 - A1, A2 + A3) and T(-xp) = (A0 + A1, A2 - A3); they are
// kept as the pairs (A0, A3) += u (dr, dr) and (A2, A1) += u (di, di), one
// packed FP32 FMA (sm_100 FFMA2) each.
// Terms outside the lattice and the mirrors of xp = 0 / yp = 0 are computed
// but not stored.  The partial-sum layout is the plain kernel's.
// Each 256-particle tile is summed in FP32 registers and added to the
// thread's running sums in FP64, which live in global scratch (read and
// written once per tile, coalesced across the warp), so L is bounded by the
// tile accumulators alone.
struct FoldKernelArgs {
    SumKernelArgs s;
    int xpc;       // x chunks of L representatives: ceil(XP / L)
    int yrows;     // FY == 2: YP representatives yp; FY == 1: lat.ny
    size_t plane;  // partial sums per split: lat.nx * n_rest
    double2* sums;  // [split][L * 2 FY][gridDim.x * kThreads] running FP64 sums
    // kAmpShell: particles sorted into shell_nbins h-bins (classification
    // edges, first particle of each bin) and the branch point r0
    int shell_nbins;
    const float* shell_edges;
    const int* shell_first;
    float shell_r0;
    const uint32_t* shell_reps;  // representatives sorted by |k|: x | y << 10 | z << 20
    int shell_count;
    const float* shell_radii;    // the particles' radii, ascending within each bin
};

template <int L, int FY, int AMP>
__global__ void __launch_bounds__(kThreads, 2) fold_sum_kernel(FoldKernelArgs fa) {
    const SumKernelArgs& a = fa.s;
    constexpr bool kShell = AMP == kAmpShell;
    constexpr bool kTab = AMP == kAmpTable || kShell;
    extern __shared__ float4 s_tab[];  // table cells (kAmpTable, kAmpShell)
    __shared__ uint4 s_q[kThreads];    // Qx, Qy, Qz, weight bits
    __shared__ float2 s_rot[kThreads];  // exp(2 pi i Qx / 2^32)
    __shared__ float s_h[kThreads];    // per-particle amplitude parameter
    __shared__ int s_bin[kShell ? kThreads : 1];  // kAmpShell: the particle's h-bin

    const int tid = threadIdx.x;
    if constexpr (kTab) {
        for (int i = tid; i <= a.table_n; i += kThreads) s_tab[i] = a.table[i];
    }

    const int nz = a.lat.nz;
    const long long n_rest_f = (long long)fa.yrows * nz;
    const long long t = (long long)blockIdx.x * kThreads + tid;
    bool active;
    int xc, yr, zr;
    if constexpr (kShell) {
        // one representative per thread (L == 1), from the list sorted by |k|:
        // a warp's 32 have nearly the same |k|, hence the same h-bin or two
        active = t < fa.shell_count;
        const uint32_t e = active ? fa.shell_reps[t] : 0u;
        xc = (int)(e & 1023u);
        yr = (int)((e >> 10) & 1023u);
        zr = (int)(e >> 20);
    } else {
        active = t < (long long)fa.xpc * n_rest_f;
        xc = active ? (int)(t / n_rest_f) : 0;
        const int rf = active ? (int)(t % n_rest_f) : 0;
        yr = rf / nz;
        zr = rf % nz;
    }
    const int yp = FY == 2 ? yr : a.lat.y0 + yr;
    const int z = a.lat.z0 + zr;
    const int xb = xc * L;

    // |k| (table kinds) or |k|^2 (kAmpExp2) of the thread's L representatives.
    float r[L];
    if constexpr (AMP != kAmpFactored) {
        const double ry = a.lat.ky * yp, rz = a.lat.kz * z;
#pragma unroll
        for (int m = 0; m < L; ++m) {
            const double rx = a.lat.kx * (xb + m);
            const double r2 = rx * rx + ry * ry + rz * rz;
            r[m] = kTab ? (float)sqrt(r2) : (float)r2;
        }
    }

    constexpr int NP = 2 * FY;  // packed pairs of real sums per representative
    const size_t tstride = (size_t)gridDim.x * kThreads;
    double2* sums = fa.sums + (size_t)blockIdx.y * (L * NP) * tstride + t;  // this thread's, stride tstride

    // kAmpShell: at frequency k only the particles of the h-bin holding
    // r0 / |k| count (the tensor form takes the closed form for that bin and
    // the reference's piecewise Phi^ for the others); rb[m] is that bin for
    // each representative, and a warp reads the particles of the bins between
    // its representatives' extremes, a block those of its warps
    int rb[kShell ? L : 1];
    int beg = blockIdx.y * a.chunk, end = min(a.n, beg + a.chunk), w_lo = 0, w_hi = a.n;
    if constexpr (kShell) {
        int bmin = fa.shell_nbins, bmax = -1, cut = 0;
#pragma unroll
        for (int m = 0; m < L; ++m) {
            const float hstar = r[m] > 0.f ? fa.shell_r0 / r[m] : INFINITY;
            rb[m] = hbin_of(fa.shell_edges, fa.shell_nbins, hstar);
            bmin = min(bmin, rb[m]);
            bmax = max(bmax, rb[m]);
            // the bin's particles are sorted by radius, and Phi^ - C is zero
            // from the branch point on (h |k| >= r0): only the run below
            // h* = r0 / |k| counts (with a margin of 1e-5 of h* for rounding)
            int lo = fa.shell_first[rb[m]], hi = fa.shell_first[rb[m] + 1];
            const float hcut = hstar * 1.00001f;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (fa.shell_radii[mid] < hcut) lo = mid + 1;
                else hi = mid;
            }
            cut = max(cut, lo);
        }
        if (!active) {
            bmin = fa.shell_nbins;
            bmax = -1;
            cut = 0;
        }
        bmin = __reduce_min_sync(0xffffffffu, bmin);
        bmax = __reduce_max_sync(0xffffffffu, bmax);
        cut = __reduce_max_sync(0xffffffffu, cut);
        w_lo = bmax < 0 ? 0 : fa.shell_first[bmin];
        w_hi = bmax < 0 ? 0 : cut;
        __shared__ int s_lo, s_hi;
        if (tid == 0) {
            s_lo = a.n;
            s_hi = 0;
        }
        __syncthreads();
        if ((tid & 31) == 0 && w_hi > w_lo) {
            atomicMin(&s_lo, w_lo);
            atomicMax(&s_hi, w_hi);
        }
        __syncthreads();
        beg = s_lo;
        end = s_hi;  // one split: the launcher runs the shell part unsplit
    }
    const uint32_t uxb = (uint32_t)xb, uy = (uint32_t)yp, uz = (uint32_t)z;

    for (int t0 = beg; t0 < end; t0 += kThreads) {
        __syncthreads();
        const int idx = t0 + tid;
        if (idx < end) {
            const float4 p = a.particles[idx];
            const double px = p.x, py = p.y, pz = p.z;
            const double* mm = a.lat.m;
            const uint32_t qx = fixed_turns(mm[0] * px + mm[1] * py + mm[2] * pz);
            s_q[tid] = make_uint4(qx, fixed_turns(mm[3] * px + mm[4] * py + mm[5] * pz),
                                  fixed_turns(mm[6] * px + mm[7] * py + mm[8] * pz), __float_as_uint(p.w));
            double sn, cs;
            sincospi((double)(int32_t)qx * (1.0 / 2147483648.0), &sn, &cs);
            s_rot[tid] = make_float2((float)cs, (float)sn);
            if constexpr (kTab) s_h[tid] = a.radii[idx] * a.inv_ds;
            else if constexpr (AMP == kAmpExp2) {
                const float h = a.radii[idx];
                s_h[tid] = a.amp_scale * h * h;
            }
            if constexpr (kShell) {
                // the bin of sorted particle idx: the last b with first[b] <= idx
                int lo = 0, hi = fa.shell_nbins;
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (fa.shell_first[mid] <= idx) lo = mid;
                    else hi = mid;
                }
                s_bin[tid] = lo;
            }
        }
        __syncthreads();
        // this warp's particles of the tile (warp-uniform)
        const int j0 = kShell ? max(0, w_lo - t0) : 0;
        const int cnt = kShell ? min(min(kThreads, end - t0), w_hi - t0) : min(kThreads, end - t0);

        float2 acc[L][NP];
#pragma unroll
        for (int m = 0; m < L; ++m)
#pragma unroll
            for (int i = 0; i < NP; ++i) acc[m][i] = make_float2(0.f, 0.f);

#pragma unroll 2
        for (int j = j0; j < cnt; ++j) {
            const uint4 q = s_q[j];
            const float2 R = s_rot[j];
            float hv = 0.f;
            if constexpr (AMP != kAmpFactored) hv = s_h[j];
            int pbin = 0;
            if constexpr (kShell) pbin = s_bin[j];
            const float w = __uint_as_float(q.w);
            const uint32_t pyz = uy * q.y + uz * q.z;
            float sn, cs;
            __sincosf(turns_to_radians(pyz), &sn, &cs);
            const float2 dpr = make_float2(w * cs, w * cs), dpi = make_float2(w * sn, w * sn);
            float2 dmr = make_float2(0.f, 0.f), dmi = make_float2(0.f, 0.f);
            if constexpr (FY == 2) {
                __sincosf(turns_to_radians(pyz - 2u * uy * q.y), &sn, &cs);
                dmr = make_float2(w * cs, w * cs);
                dmi = make_float2(w * sn, w * sn);
            }
            __sincosf(turns_to_radians(uxb * q.x), &sn, &cs);
            float cr = cs, ci = sn;
#pragma unroll
            for (int m = 0; m < L; ++m) {
                float ur = cr, ui = ci;
                if constexpr (AMP != kAmpFactored) {
                    float amp;
                    if constexpr (kTab) {
                        // s / ds = r hv: nearest cell and offset (1.5 * 2^23 rounds)
                        const float tt = fmaf(r[m], hv, 12582912.0f);
                        const float fr = fmaf(r[m], hv, -(tt - 12582912.0f));
                        // beyond the table (and for negative radii) the last,
                        // all-zero cell is used
                        const unsigned k = min((unsigned)(__float_as_int(tt) - 0x4B400000), (unsigned)a.table_n);
                        const float4 c = s_tab[k];
                        amp = fmaf(fmaf(fmaf(c.w, fr, c.z), fr, c.y), fr, c.x);
                        if constexpr (kShell) amp = pbin == rb[m] ? amp : 0.f;
                    } else {
                        amp = exp2f(hv * r[m]);
                    }
                    ur *= amp;
                    ui *= amp;
                }
                const float2 u = make_float2(ur, ui);
                acc[m][0] = __ffma2_rn(u, dpr, acc[m][0]);  // (A0, A3)
                acc[m][1] = __ffma2_rn(u, dpi, acc[m][1]);  // (A2, A1)
                if constexpr (FY == 2) {
                    acc[m][2] = __ffma2_rn(u, dmr, acc[m][2]);
                    acc[m][3] = __ffma2_rn(u, dmi, acc[m][3]);
                }
                if (m + 1 < L) {
                    const float nr = fmaf(cr, R.x, -ci * R.y);
                    const float ni = fmaf(cr, R.y, ci * R.x);
                    cr = nr;
                    ci = ni;
                }
            }
        }
        // add this tile's sums to the running FP64 sums
        const bool first = t0 == beg;
#pragma unroll
        for (int m = 0; m < L; ++m)
#pragma unroll
            for (int i = 0; i < NP; ++i) {
                double2* p = sums + (size_t)(m * NP + i) * tstride;
                const double2 o = first ? make_double2(0.0, 0.0) : *p;
                *p = make_double2(o.x + (double)acc[m][i].x, o.y + (double)acc[m][i].y);
            }
    }

    if (!active) return;
    const bool any = beg < end;
    float2* out = a.partial + blockIdx.y * fa.plane;
    const int x_lo = a.lat.x0, x_hi = a.lat.x0 + a.lat.nx - 1;
    const int y_lo = a.lat.y0, y_hi = a.lat.y0 + a.lat.ny - 1;
#pragma unroll
    for (int m = 0; m < L; ++m) {
        const int xp = xb + m;
#pragma unroll
        for (int sy = 0; sy < FY; ++sy) {
            const int y = sy == 0 ? yp : -yp;
            if (sy == 1 && yp == 0) continue;
            if (y < y_lo || y > y_hi) continue;
            // (A0, A3) and (A2, A1) of this y sign
            const double2 z2 = make_double2(0.0, 0.0);
            const double2 p0 = any ? sums[(size_t)(m * NP + 2 * sy) * tstride] : z2;
            const double2 p1 = any ? sums[(size_t)(m * NP + 2 * sy + 1) * tstride] : z2;
            const size_t rest = (size_t)(y - y_lo) * nz + (z - a.lat.z0);
            if (xp <= x_hi)
                out[(size_t)(xp - x_lo) * a.n_rest + rest] = make_float2((float)(p0.x - p1.y), (float)(p1.x + p0.y));
            if (xp > 0 && -xp >= x_lo)
                out[(size_t)(-xp - x_lo) * a.n_rest + rest] = make_float2((float)(p0.x + p1.y), (float)(p1.x - p0.y));
        }
    }
}

// Cubic pieces of Phi^ on cells [(k - 1/2) ds, (k + 1/2) ds]: the polynomial in
// fr = s/ds - k interpolating Phi^ (FP64, reference branch points) at the four
// Chebyshev points of the cell.  Cells never straddle a branch point because
// ds is chosen so that each branch point is a half-integer multiple of ds.
__global__ void phi_table_kernel(int basis, double ds, int n, float4* out, int kink) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > n) return;
    if (k == n) {
        out[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    double x[4], f[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        x[i] = 0.5 * cospi((2 * i + 1) / 8.0);
        f[i] = kink ? phi_kink_fp64(basis, (k + x[i]) * ds) : phi_fp64(basis, (k + x[i]) * ds);
    }
    // Newton divided differences, then expansion to monomials in fr.
    double d[4] = {f[0], f[1], f[2], f[3]};
    for (int lvl = 1; lvl < 4; ++lvl)
        for (int i = 3; i >= lvl; --i) d[i] = (d[i] - d[i - 1]) / (x[i] - x[i - lvl]);
    double c[4] = {d[3], 0.0, 0.0, 0.0};  // Horner-style expansion of the Newton form
    int deg = 0;
    for (int i = 2; i >= 0; --i) {
        // c(x) = c(x) * (x - x[i]) + d[i]
        double nc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int p = 0; p <= deg; ++p) {
            nc[p + 1] += c[p];
            nc[p] -= x[i] * c[p];
        }
        ++deg;
        nc[0] += d[i];
        for (int p = 0; p < 4; ++p) c[p] = nc[p];
    }
    out[k] = make_float4((float)c[0], (float)c[1], (float)c[2], (float)c[3]);
}

struct FinalizeArgs {
    const float2* partial;
    int splits;
    size_t plane;  // elements per split
    int n_rest;
    Lattice lat;
    int basis;
    bool factored;
    double scale;
    float2* out;
    long long out_base, out_sx, out_sy, out_sz;
    int wrap;
    int row;
    bool accumulate;
};

// Reduces the split partial sums in FP64, applies Phi^(|k|) for groups without
// radii (FP64) and the scale, conjugates (the kernel summed w e^{+i theta}),
// and writes or accumulates into the output layout.
__global__ void finalize_kernel(FinalizeArgs f) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long count = (long long)f.lat.nx * f.n_rest;
    if (q >= count) return;
    const int xi = (int)(q / f.n_rest);
    const int rest = (int)(q % f.n_rest);
    double sr = 0.0, si = 0.0;
    for (int s = 0; s < f.splits; ++s) {
        const float2 v = f.partial[s * f.plane + q];
        sr += v.x;
        si += v.y;
    }
    const int x = f.lat.x0 + xi;
    const int y = f.lat.y0 + rest / f.lat.nz;
    const int z = f.lat.z0 + rest % f.lat.nz;
    double factor = f.scale;
    if (f.factored) {
        const double rx = f.lat.kx * x, ry = f.lat.ky * y, rz = f.lat.kz * z;
        factor *= phi_fp64(f.basis, sqrt(rx * rx + ry * ry + rz * rz));
    }
    const float re = (float)(sr * factor), im = (float)(-si * factor);
    size_t idx;
    if (f.wrap > 0) idx = (size_t)(x < 0 ? x + f.wrap : x) * f.row + rest;
    else idx = (size_t)(f.out_base + xi * f.out_sx + (rest / f.lat.nz) * f.out_sy + (rest % f.lat.nz) * f.out_sz);
    if (f.accumulate) {
        float2 o = f.out[idx];
        f.out[idx] = make_float2(o.x + re, o.y + im);
    } else {
        f.out[idx] = make_float2(re, im);
    }
}

using SumKernel = void (*)(SumKernelArgs);

template <int L, int BASIS>
SumKernel pick_amp(int amp) {
    if (amp == kAmpFactored) return plain_sum_kernel<L, BASIS, kAmpFactored>;
    if constexpr (BASIS == kSph || BASIS == kWendland) return plain_sum_kernel<L, BASIS, kAmpTable>;
    else if constexpr (BASIS == kGaussianDecaying && L > 1) return plain_sum_kernel<L, BASIS, kAmpGaussRec>;
    else return plain_sum_kernel<L, BASIS, kAmpExp2>;
}

using FoldKernel = void (*)(FoldKernelArgs);

template <int L, int FY>
FoldKernel pick_fold(int amp) {
    if (amp == kAmpFactored) return fold_sum_kernel<L, FY, kAmpFactored>;
    if (amp == kAmpTable) return fold_sum_kernel<L, FY, kAmpTable>;
    return fold_sum_kernel<L, FY, kAmpExp2>;
}

template <int L>
SumKernel pick(int basis, int amp) {
    switch (basis) {
    case kSph: return pick_amp<L, kSph>(amp);
    case kGaussian: return pick_amp<L, kGaussian>(amp);
    case kWendland: return pick_amp<L, kWendland>(amp);
    default: return pick_amp<L, kGaussianDecaying>(amp);
    }
}

// Table cell width: a branch point of the reference's piecewise Phi^ (0.06f
// for SPH, 0.24f for Wendland) sits at (K + 1/2) ds.
double table_cell(int basis) { return basis == kSph ? (double)0.06f / 3.5 : (double)0.24f / 15.5; }

// The folded lattice's representatives (xp, yp, z), xp < XP, yp < YP, z of
// the lattice, sorted by |k|^2 and packed x | y << 10 | z << 20, in device
// memory: built once per lattice shape and device and kept for the process.
std::mutex g_reps_mu;
std::map<std::tuple<int, int, int, int, double, double, double>, std::pair<uint32_t*, long long>> g_reps;

int shell_representatives(const Lattice& lat, int xp_count, int yrows, const uint32_t** out, long long* count) {
    if (xp_count > 1024 || yrows > 1024 || lat.z0 != 0 || lat.nz > 4096)
        return set_error(kInvalidValue, "branch part: lattice too large for its representative list");
    int dev = 0;
    int st = check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (st != kOk) return st;
    const auto key = std::make_tuple(dev, xp_count, yrows, lat.nz, lat.kx, lat.ky, lat.kz);
    std::lock_guard<std::mutex> lock(g_reps_mu);
    auto it = g_reps.find(key);
    if (it == g_reps.end()) {
        std::vector<std::pair<double, uint32_t>> v;
        v.reserve((size_t)xp_count * yrows * lat.nz);
        for (int x = 0; x < xp_count; ++x)
            for (int y = 0; y < yrows; ++y)
                for (int z = 0; z < lat.nz; ++z) {
                    const double kx = lat.kx * x, ky = lat.ky * y, kz = lat.kz * z;
                    v.push_back({kx * kx + ky * ky + kz * kz, (uint32_t)x | ((uint32_t)y << 10) | ((uint32_t)z << 20)});
                }
        std::sort(v.begin(), v.end());
        std::vector<uint32_t> packed(v.size());
        for (size_t i = 0; i < v.size(); ++i) packed[i] = v[i].second;
        uint32_t* d = nullptr;
        st = check_cuda(cudaMalloc(&d, packed.size() * sizeof(uint32_t)), "cudaMalloc(representatives)");
        if (st != kOk) return st;
        st = check_cuda(cudaMemcpy(d, packed.data(), packed.size() * sizeof(uint32_t), cudaMemcpyHostToDevice),
                        "representatives H2D");
        if (st != kOk) {
            cudaFree(d);
            return st;
        }
        it = g_reps.emplace(key, std::make_pair(d, (long long)packed.size())).first;
    }
    *out = it->second.first;
    *count = it->second.second;
    return kOk;
}

}  // namespace

int launch_plain_sum(const SumRequest& req, Workspace& ws, KernelTimer* timer) {
    const Lattice& lat = req.lat;
    if (lat.nx <= 0 || lat.ny <= 0 || lat.nz <= 0) return kOk;
    if (req.basis < 0 || req.basis >= kBasisCount) return set_error(kInvalidValue, "unknown basis function id");
    if (req.n < 0) return set_error(kInvalidValue, "negative number of terms");
    if (req.n > 0 && req.particles == nullptr) return set_error(kInvalidValue, "dataset group has no device particles");

    const bool factored = req.radii == nullptr;
    int amp = factored ? kAmpFactored
              : (req.basis == kSph || req.basis == kWendland) ? kAmpTable
                                                                : kAmpExp2;
    if (req.kink) {
        if (amp != kAmpTable || req.shell_nbins <= 0)
            return set_error(kInvalidValue, "branch part needs SPH or Wendland with radii and h-bins");
        amp = kAmpShell;
    }
    const int L = lat.nx >= 8 ? 8 : 1;
    const int nxc = (lat.nx + L - 1) / L;
    const long long n_rest = (long long)lat.ny * lat.nz;
    // Folded form when x = 0 is on the lattice (and y folds too when the y
    // range holds both signs).  x representatives per thread: 8 without the y
    // fold; with it the L of {4, 5, 6} (more spill at 128 registers) that
    // minimises the chunks' work, ceil(XP / L) (30 + 20 L) instructions per
    // particle (a particle's phases and constants, then one Phi^ evaluation
    // and x rotation per representative): 65 representatives (C2's 128^3) and
    // 33 (64^3) take 6.
    const bool fold = lat.x0 <= 0 && lat.x0 + lat.nx - 1 >= 0;
    const bool fold_y = fold && lat.y0 < 0 && lat.y0 + lat.ny - 1 > 0;
    const int xp_count = std::max(-lat.x0, lat.x0 + lat.nx - 1) + 1;
    int fold_l = 8;
    if (fold_y) {
        long long best = -1;
        for (int l : {4, 5, 6}) {
            const long long cost = (long long)((xp_count + l - 1) / l) * (30 + 20 * l);
            if (best < 0 || cost < best) {
                best = cost;
                fold_l = l;
            }
        }
    }
    if (amp == kAmpShell && !fold_y) return set_error(kInvalidValue, "branch part needs a lattice holding x = 0, y = 0");
    if (amp == kAmpShell) fold_l = 1;  // one representative per thread, sorted by |k|
    const int yrows = fold_y ? std::max(-lat.y0, lat.y0 + lat.ny - 1) + 1 : lat.ny;
    const int xpc = (xp_count + fold_l - 1) / fold_l;
    const uint32_t* shell_reps = nullptr;
    long long threads = fold ? (long long)xpc * yrows * lat.nz : (long long)nxc * n_rest;
    if (amp == kAmpShell) {
        int st_reps = shell_representatives(lat, xp_count, yrows, &shell_reps, &threads);
        if (st_reps != kOk) return st_reps;
    }
    if (threads > (1LL << 31) - 1) return set_error(kInvalidValue, "lattice too large");
    const long long blocks_f = (threads + kThreads - 1) / kThreads;

    // Split the particle range until the grid holds ~plain_waves blocks per SM
    // (default 6: three waves of the 2 resident blocks; the autotuner may pick
    // another), keeping at least 4 tiles per split.
    const long long target = (long long)device_sm_count() * active_tune().plain_waves;
    long long max_splits = std::max<long long>(1, (req.n + 4 * kThreads - 1) / (4 * kThreads));
    long long splits = std::min<long long>(std::max<long long>(1, (target + blocks_f - 1) / blocks_f), max_splits);
    splits = std::min<long long>(splits, 65535);
    // Within a factor of two of that, the split count whose grid fills its
    // last wave of resident blocks (2 per SM) best; more splits only for a
    // fill at least 1% better.  C2 (215 blocks per split): 4 splits fill 2.9
    // waves (0.97), where 5 fill 3.6 (0.91).
    {
        const double resident = 2.0 * device_sm_count();
        const long long lo = std::max<long long>(1, splits / 2);
        const long long hi = std::min<long long>(std::min<long long>(2 * splits, max_splits), 65535);
        long long best = splits;
        double best_fill = -1.0;
        for (long long sp = lo; sp <= hi; ++sp) {
            const double waves = (double)(blocks_f * sp) / resident;
            const double fill = waves / std::ceil(waves);
            if (fill > best_fill + 0.01) {
                best_fill = fill;
                best = sp;
            }
        }
        splits = best;
    }
    if (amp == kAmpShell) splits = 1;  // each block reads a few h-bins only
    long long chunk = req.n > 0 ? ((req.n + splits - 1) / splits + kThreads - 1) / kThreads * kThreads : kThreads;
    splits = req.n > 0 ? (req.n + chunk - 1) / chunk : 1;

    // Table size: cells up to the largest s = |k|max * hmax (when known).
    int table_n = 0;
    double ds = 0.0;
    if (amp == kAmpTable || amp == kAmpShell) {
        ds = table_cell(req.basis);
        const double kx = std::fabs(lat.kx) * std::max(std::abs(lat.x0), std::abs(lat.x0 + lat.nx - 1));
        const double ky = std::fabs(lat.ky) * std::max(std::abs(lat.y0), std::abs(lat.y0 + lat.ny - 1));
        const double kz = std::fabs(lat.kz) * std::max(std::abs(lat.z0), std::abs(lat.z0 + lat.nz - 1));
        const double rmax = std::sqrt(kx * kx + ky * ky + kz * kz);
        const double smax = req.radius_max >= 0.f ? rmax * req.radius_max : 1e30;
        // Beyond kMaxTable cells (s > 63 for Wendland, > 60 for SPH) |Phi^| < 1e-11
        // and the zero cell stands in for it.
        table_n = (int)std::min<double>(kMaxTable, std::ceil(smax / ds) + 2.0);
        table_n = std::max(table_n, 1);
        // the branch part ends at the branch point, (K + 1/2) ds: cells 0 .. K
        if (req.kink) table_n = std::min(table_n, (int)std::llround(phi_branch_point(req.basis) / ds - 0.5) + 1);
    }

    const size_t plane = fold ? (size_t)lat.nx * n_rest : (size_t)nxc * L * n_rest;
    const size_t part_bytes = (plane * splits * sizeof(float2) + 255) / 256 * 256;
    const size_t table_cells = (amp == kAmpTable || amp == kAmpShell) ? (size_t)table_n + 1 : 0;
    const size_t table_bytes = (table_cells * sizeof(float4) + 255) / 256 * 256;
    // folded form: the running FP64 sums, 2 FY pairs per representative
    const size_t sums_bytes =
        fold ? (size_t)splits * fold_l * (fold_y ? 4 : 2) * (size_t)blocks_f * kThreads * sizeof(double2) : 0;
    int st = ws.reserve(part_bytes + table_bytes + sums_bytes);
    if (st != kOk) return st;

    SumKernelArgs a;
    a.particles = req.particles;
    a.radii = req.radii;
    a.n = req.n;
    a.chunk = (int)chunk;
    a.lat = lat;
    a.nxc = nxc;
    a.n_rest = (int)n_rest;
    a.partial = static_cast<float2*>(ws.ptr);
    a.table = reinterpret_cast<const float4*>(static_cast<char*>(ws.ptr) + part_bytes);
    a.table_n = table_n;
    a.inv_ds = ds > 0 ? (float)(1.0 / ds) : 0.f;
    a.amp_scale = req.basis == kGaussian ? kPiLog2e : -kPiLog2e;

    if (amp == kAmpTable || amp == kAmpShell) {
        phi_table_kernel<<<(table_n + 128) / 128, 128, 0, req.stream>>>(req.basis, ds, table_n,
                                                                         const_cast<float4*>(a.table), req.kink);
        count_launch();
    }

    const size_t dyn_smem = table_cells * sizeof(float4);
    if (fold) {
        FoldKernelArgs fa;
        fa.s = a;
        fa.xpc = xpc;
        fa.yrows = yrows;
        fa.plane = plane;
        fa.sums = reinterpret_cast<double2*>(static_cast<char*>(ws.ptr) + part_bytes + table_bytes);
        fa.shell_nbins = req.kink ? req.shell_nbins : 0;
        fa.shell_edges = req.shell_edges;
        fa.shell_first = req.shell_first;
        fa.shell_r0 = (float)phi_branch_point(req.basis);
        fa.shell_reps = shell_reps;
        fa.shell_radii = req.kink ? req.radii : nullptr;
        fa.shell_count = (int)threads;
        FoldKernel k = amp == kAmpShell ? fold_sum_kernel<1, 2, kAmpShell>
                       : !fold_y      ? pick_fold<8, 1>(amp)
                       : fold_l == 4  ? pick_fold<4, 2>(amp)
                       : fold_l == 5  ? pick_fold<5, 2>(amp)
                                      : pick_fold<6, 2>(amp);
        if (dyn_smem > 48 * 1024) {
            st = check_cuda(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_smem),
                            "cudaFuncSetAttribute");
            if (st != kOk) return st;
        }
        timer_begin(timer, 0, req.stream);
        k<<<dim3((unsigned)blocks_f, (unsigned)splits), kThreads, dyn_smem, req.stream>>>(fa);
        count_launch();
        timer_end(timer, 0, req.stream);
        st = check_cuda(cudaGetLastError(), "fold_sum_kernel launch");
    } else {
        SumKernel k = (L == 8) ? pick<8>(req.basis, amp) : pick<1>(req.basis, amp);
        if (dyn_smem > 48 * 1024) {
            st = check_cuda(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_smem),
                            "cudaFuncSetAttribute");
            if (st != kOk) return st;
        }
        timer_begin(timer, 0, req.stream);
        k<<<dim3((unsigned)blocks_f, (unsigned)splits), kThreads, dyn_smem, req.stream>>>(a);
        count_launch();
        timer_end(timer, 0, req.stream);
        st = check_cuda(cudaGetLastError(), "plain_sum_kernel launch");
    }
    if (st != kOk) return st;

    FinalizeArgs f;
    f.partial = a.partial;
    f.splits = (int)splits;
    f.plane = plane;
    f.n_rest = (int)n_rest;
    f.lat = lat;
    f.basis = req.basis;
    f.factored = factored;
    f.scale = req.scale;
    f.out = req.out;
    f.out_base = req.out_base;
    f.out_sx = req.out_sx;
    f.out_sy = req.out_sy;
    f.out_sz = req.out_sz;
    f.wrap = req.wrap;
    f.row = req.row;
    f.accumulate = req.accumulate;
    const long long count = (long long)lat.nx * n_rest;
    finalize_kernel<<<(unsigned)((count + 255) / 256), 256, 0, req.stream>>>(f);
    count_launch();
    return check_cuda(cudaGetLastError(), "finalize_kernel launch");
}

}  // namespace mv

// ===================================================================== no-alloc
// vis_fourier_slice_sum_noalloc: the direct slice sum of one group (the work
// vis_fourier_volume_rendering does per group, including the C2R arrangement)
// for callers that cannot allocate device memory: code that must keep a fixed
// device-memory footprint, renders inside a frame loop where a cudaMalloc (and
// the device-wide synchronisation a cudaFree implies) is not acceptable, or
// runs under another framework's memory pool.  The caller passes every input
// and output buffer; the split-K partial sums and the Phi^ table this kernel
// needs live in the file-scope array below instead of a workspace.
namespace mv {
namespace {

// Scratch of the no-alloc entry point: 8 MiB, held by every GPU that loads the
// library until the process exits.  Its size bounds the slice:
// (number of slice samples, rounded up to 8 in x) <= ~1.04 M.
constexpr size_t kNoAllocScratchBytes = (size_t)8 << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
std::map<int, void*> g_noalloc_address;  // device -> device address of g_noalloc_scratch

// Device address of the scratch array on the current device.  In host code the
// array's name is only a host-side stand-in, so the address is looked up once
// per device with cudaGetSymbolAddress (the first call on a device does this).
int noalloc_scratch(void** out) {
    int dev = 0;
    int st = check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (st != kOk) return st;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    auto it = g_noalloc_address.find(dev);
    if (it == g_noalloc_address.end()) {
        void* p = nullptr;
        st = check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(no-alloc scratch)");
        if (st != kOk) return st;
        it = g_noalloc_address.emplace(dev, p).first;
    }
    *out = it->second;
    return kOk;
}

}  // namespace
}  // namespace mv

extern "C" int vis_fourier_slice_sum_noalloc(const Constraint* d_constraints, const float* d_radii,
                                             int number_of_terms, BasisFunctionId basis_function_id,
                                             float2 step_size, int2 cutoff_frequency, float3 u_axis, float3 v_axis,
                                             int2 number_of_samples, float2* d_arranged, int accumulate,
                                             cudaStream_t stream) {
    using namespace mv;
    const int cx = cutoff_frequency.x, cy = cutoff_frequency.y;
    const int nx = number_of_samples.x, ny = number_of_samples.y;
    const int basis = (int)basis_function_id;
    if (number_of_terms < 0 || (number_of_terms > 0 && !d_constraints) || !d_arranged)
        return set_error(kInvalidValue, "vis_fourier_slice_sum_noalloc: NULL buffer or negative number of terms");
    if (basis < 0 || basis >= kBasisCount) return set_error(kInvalidValue, "vis_fourier_slice_sum_noalloc: unknown basis");
    if (cx < 0 || cy < 0 || nx < 1 || ny < 2 || 2 * cx > nx || 2 * cy > ny)
        return set_error(kInvalidConfig, "vis_fourier_slice_sum_noalloc: cutoff_frequency does not fit number_of_samples");

    // The lattice of vis_fourier_volume_rendering: x in (-cx, cx), y in [0, cy).
    Lattice lat{};
    lat.x0 = -cx + 1;
    lat.nx = cx > 0 ? 2 * cx - 1 : 0;
    lat.y0 = 0;
    lat.ny = cy;
    lat.z0 = 0;
    lat.nz = 1;
    lat.kx = step_size.x;
    lat.ky = step_size.y;
    lat.kz = 0.0;
    const double sx = step_size.x, sy = step_size.y;
    const double m[9] = {sx * u_axis.x, sx * u_axis.y, sx * u_axis.z, sy * v_axis.x, sy * v_axis.y, sy * v_axis.z,
                         0.0, 0.0, 0.0};
    for (int i = 0; i < 9; ++i) lat.m[i] = m[i];
    if (lat.nx == 0 || lat.ny == 0) return kOk;

    void* scratch = nullptr;
    int st = noalloc_scratch(&scratch);
    if (st != kOk) return st;

    const bool factored = d_radii == nullptr;
    const int amp = factored ? kAmpFactored : (basis == kSph || basis == kWendland) ? kAmpTable : kAmpExp2;
    const int L = lat.nx >= 8 ? 8 : 1;
    const int nxc = (lat.nx + L - 1) / L;
    const long long n_rest = (long long)lat.ny;
    const size_t plane = (size_t)nxc * L * n_rest;
    // Without a radius maximum the table covers the full kMaxTable cells.
    const int table_n = amp == kAmpTable ? kMaxTable : 0;
    const double ds = amp == kAmpTable ? table_cell(basis) : 0.0;
    const size_t table_bytes = amp == kAmpTable ? ((size_t)(table_n + 1) * sizeof(float4) + 255) / 256 * 256 : 0;
    if (table_bytes + plane * sizeof(float2) > kNoAllocScratchBytes)
        return set_error(kInvalidValue, "vis_fourier_slice_sum_noalloc: slice of " + std::to_string(plane) +
                                            " samples exceeds the no-alloc scratch (" +
                                            std::to_string((kNoAllocScratchBytes - table_bytes) / sizeof(float2)) +
                                            " samples at most)");
    const long long max_by_scratch = (long long)((kNoAllocScratchBytes - table_bytes) / (plane * sizeof(float2)));

    const long long threads = (long long)nxc * n_rest;
    const long long blocks_f = (threads + kThreads - 1) / kThreads;
    const long long target = (long long)device_sm_count() * 6;
    const long long max_splits = std::max<long long>(1, (number_of_terms + 4 * kThreads - 1) / (4 * kThreads));
    long long splits = std::min<long long>(std::max<long long>(1, (target + blocks_f - 1) / blocks_f), max_splits);
    splits = std::min<long long>(std::min<long long>(splits, max_by_scratch), 65535);
    const long long chunk =
        number_of_terms > 0 ? ((number_of_terms + splits - 1) / splits + kThreads - 1) / kThreads * kThreads : kThreads;
    splits = number_of_terms > 0 ? (number_of_terms + chunk - 1) / chunk : 1;

    // Scratch layout: [Phi^ table | split-K partials].  Every element the
    // kernels read is written earlier in the same call, so the previous
    // call's contents never matter and nothing needs clearing.
    SumKernelArgs a;
    a.particles = reinterpret_cast<const float4*>(d_constraints);
    a.radii = d_radii;
    a.n = number_of_terms;
    a.chunk = (int)chunk;
    a.lat = lat;
    a.nxc = nxc;
    a.n_rest = (int)n_rest;
    a.table = reinterpret_cast<const float4*>(scratch);
    a.table_n = table_n;
    a.partial = reinterpret_cast<float2*>(static_cast<unsigned char*>(scratch) + table_bytes);
    a.inv_ds = ds > 0 ? (float)(1.0 / ds) : 0.f;
    a.amp_scale = basis == kGaussian ? kPiLog2e : -kPiLog2e;

    if (amp == kAmpTable) {
        phi_table_kernel<<<(table_n + 128) / 128, 128, 0, stream>>>(basis, ds, table_n, const_cast<float4*>(a.table), 0);
        count_launch();
    }
    SumKernel k = (L == 8) ? pick<8>(basis, amp) : pick<1>(basis, amp);
    const size_t dyn_smem = amp == kAmpTable ? (size_t)(table_n + 1) * sizeof(float4) : 0;
    if (dyn_smem > 48 * 1024) {
        st = check_cuda(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_smem),
                        "cudaFuncSetAttribute");
        if (st != kOk) return st;
    }
    k<<<dim3((unsigned)blocks_f, (unsigned)splits), kThreads, dyn_smem, stream>>>(a);
    count_launch();
    st = check_cuda(cudaGetLastError(), "plain_sum_kernel launch (no-alloc)");
    if (st != kOk) return st;

    FinalizeArgs f;
    f.partial = a.partial;
    f.splits = (int)splits;
    f.plane = plane;
    f.n_rest = (int)n_rest;
    f.lat = lat;
    f.basis = basis;
    f.factored = factored;
    f.scale = (double)step_size.x * (double)step_size.y;
    f.out = d_arranged;
    f.out_base = 0;
    f.out_sx = f.out_sy = f.out_sz = 0;
    f.wrap = nx;
    f.row = ny / 2 + 1;
    f.accumulate = accumulate != 0;
    const long long count = (long long)lat.nx * n_rest;
    finalize_kernel<<<(unsigned)((count + 255) / 256), 256, 0, stream>>>(f);
    count_launch();
    return check_cuda(cudaGetLastError(), "finalize_kernel launch (no-alloc)");
}
