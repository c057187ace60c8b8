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
// Per particle tile (256 particles staged in shared memory by the block), the
// loader converts each position to fixed-point turns per lattice axis,
// Q_a = round(2^32 (M p)_a) mod 2^32, in FP64.  The phase of a term is then the
// exact integer x Qx + y Qy + z Qz mod 2^32 (wrapping 32-bit multiply-add),
// converted to radians in [-pi, pi) and passed to the SFU sincos.  The
// reference instead forms 2 pi f.x in FP32 and calls __sincosf on an
// unreduced argument (fourier_transform.cu:125), whose error grows with |f.x|.
//
// Accumulation: each tile's 256 terms are summed in FP32 registers and the
// tile sums are added with Kahan compensation; splits are reduced in FP64.
#include <algorithm>
#include <cstdio>

#include "mv_device.cuh"
#include "mv_internal.h"

namespace mv {

namespace {

constexpr int kThreads = 256;  // threads per block == particles per tile

struct SumKernelArgs {
    const float4* particles;
    const float* radii;
    int n;
    int chunk;  // particles per split (multiple of kThreads)
    Lattice lat;
    int nxc;     // number of x chunks of L
    int n_rest;  // ny * nz
    float2* partial;  // [split][nxc * L][n_rest]
};

template <int L, int BASIS, bool FACTORED>
__global__ void __launch_bounds__(kThreads) plain_sum_kernel(SumKernelArgs a) {
    __shared__ uint4 s_q[kThreads];  // Qx, Qy, Qz, weight bits
    __shared__ float s_h[kThreads];

    const int tid = threadIdx.x;
    const long long t = (long long)blockIdx.x * kThreads + tid;
    const bool active = t < (long long)a.nxc * a.n_rest;
    const int xc = active ? (int)(t / a.n_rest) : 0;
    const int rest = active ? (int)(t % a.n_rest) : 0;
    const int y = a.lat.y0 + rest / a.lat.nz;
    const int z = a.lat.z0 + rest % a.lat.nz;
    const int xb = a.lat.x0 + xc * L;

    float r[L];
    if constexpr (!FACTORED) {
        const double ry = a.lat.ky * y, rz = a.lat.kz * z;
#pragma unroll
        for (int m = 0; m < L; ++m) {
            const double rx = a.lat.kx * (xb + m);
            r[m] = (float)sqrt(rx * rx + ry * ry + rz * rz);
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
            s_q[tid] = make_uint4(fixed_turns(m[0] * px + m[1] * py + m[2] * pz),
                                  fixed_turns(m[3] * px + m[4] * py + m[5] * pz),
                                  fixed_turns(m[6] * px + m[7] * py + m[8] * pz), __float_as_uint(p.w));
            s_h[tid] = FACTORED ? 0.f : a.radii[idx];
        }
        __syncthreads();
        const int cnt = min(kThreads, end - t0);

        float2 acc[L];
#pragma unroll
        for (int m = 0; m < L; ++m) acc[m] = make_float2(0.f, 0.f);

        for (int j = 0; j < cnt; ++j) {
            const uint4 q = s_q[j];
            const float w = __uint_as_float(q.w);
            uint32_t ph = ux * q.x + uy * q.y + uz * q.z;
            float h = 0.f;
            if constexpr (!FACTORED) h = s_h[j];
#pragma unroll
            for (int m = 0; m < L; ++m) {
                float sn, cs;
                __sincosf(turns_to_radians(ph), &sn, &cs);
                float amp = w;
                if constexpr (!FACTORED) amp *= phi<BASIS>(r[m] * h);
                acc[m].x = fmaf(amp, cs, acc[m].x);
                acc[m].y = fmaf(amp, sn, acc[m].y);
                ph += q.x;
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
    else idx = (size_t)q;
    if (f.accumulate) {
        float2 o = f.out[idx];
        f.out[idx] = make_float2(o.x + re, o.y + im);
    } else {
        f.out[idx] = make_float2(re, im);
    }
}

using SumKernel = void (*)(SumKernelArgs);

template <int L>
SumKernel pick(int basis, bool factored) {
    switch (basis) {
    case kSph: return factored ? plain_sum_kernel<L, kSph, true> : plain_sum_kernel<L, kSph, false>;
    case kGaussian: return factored ? plain_sum_kernel<L, kGaussian, true> : plain_sum_kernel<L, kGaussian, false>;
    case kWendland: return factored ? plain_sum_kernel<L, kWendland, true> : plain_sum_kernel<L, kWendland, false>;
    default:
        return factored ? plain_sum_kernel<L, kGaussianDecaying, true> : plain_sum_kernel<L, kGaussianDecaying, false>;
    }
}

}  // namespace

int launch_plain_sum(const SumRequest& req, Workspace& ws, KernelTimer* timer) {
    const Lattice& lat = req.lat;
    if (lat.nx <= 0 || lat.ny <= 0 || lat.nz <= 0) return kOk;
    if (req.basis < 0 || req.basis >= kBasisCount) return set_error(kInvalidValue, "unknown basis function id");
    if (req.n < 0) return set_error(kInvalidValue, "negative number of terms");
    if (req.n > 0 && req.particles == nullptr) return set_error(kInvalidValue, "dataset group has no device particles");

    const bool factored = req.radii == nullptr;
    const int L = lat.nx >= 16 ? 4 : 1;
    const int nxc = (lat.nx + L - 1) / L;
    const long long n_rest = (long long)lat.ny * lat.nz;
    const long long threads = (long long)nxc * n_rest;
    if (threads > (1LL << 31) - 1) return set_error(kInvalidValue, "lattice too large");
    const long long blocks_f = (threads + kThreads - 1) / kThreads;

    // Split the particle range until the grid holds ~8 blocks per SM, keeping
    // at least 4 tiles of particles per split.
    const long long target = (long long)device_sm_count() * 8;
    long long max_splits = std::max<long long>(1, (req.n + 4 * kThreads - 1) / (4 * kThreads));
    long long splits = std::min<long long>(std::max<long long>(1, (target + blocks_f - 1) / blocks_f), max_splits);
    splits = std::min<long long>(splits, 65535);
    long long chunk = req.n > 0 ? ((req.n + splits - 1) / splits + kThreads - 1) / kThreads * kThreads : kThreads;
    splits = req.n > 0 ? (req.n + chunk - 1) / chunk : 1;

    const size_t plane = (size_t)nxc * L * n_rest;
    int st = ws.reserve(plane * splits * sizeof(float2));
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

    SumKernel k = (L == 4) ? pick<4>(req.basis, factored) : pick<1>(req.basis, factored);
    timer_begin(timer, 0, req.stream);
    k<<<dim3((unsigned)blocks_f, (unsigned)splits), kThreads, 0, req.stream>>>(a);
    count_launch();
    timer_end(timer, 0, req.stream);
    st = check_cuda(cudaGetLastError(), "plain_sum_kernel launch");
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
    f.wrap = req.wrap;
    f.row = req.row;
    f.accumulate = req.accumulate;
    const long long count = (long long)lat.nx * n_rest;
    finalize_kernel<<<(unsigned)((count + 255) / 256), 256, 0, req.stream>>>(f);
    count_launch();
    return check_cuda(cudaGetLastError(), "finalize_kernel launch");
}

}  // namespace mv
