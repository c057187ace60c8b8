// Tensor-core form of the 3D half-spectrum Fourier sum (sm_100a, tcgen05).
//
// For a group whose amplitude separates per axis -- a group without radii or
// with one radius for all particles (Phi^(|k| h) then factors out of the sum
// and is applied per frequency in FP64), or GAUSSIAN_DECAYING with per-particle
// radii (exp(-pi h^2 |k|^2) = gx gy gz) -- the sum is a complex GEMM:
//
//   F(a, b, c) = sum_j A[(a,b), j] B[j, c],
//   A[(a,b), j] = (w_j / W) gx(a,h_j) gy(b,h_j) exp(-2 pi i (a Qx_j + b Qy_j) / 2^32)
//   B[j, c]     = gz(c,h_j) exp(-2 pi i c Qz_j / 2^32)
//
// with exact 32-bit fixed-point positions Q (as in the plain form), W the
// group's largest |weight| (so |A|, |B| <= 1).  The reference evaluates every
// term separately (meshless_vis/fourier_transform.cu:100-130); no reference
// code has this factorisation.
//
// Real embedding with re/im interleaved along K (k = 2j + {0,1}):
//   A'[m, 2j..2j+1] = (Re A, Im A),  B'_re[2j..2j+1, n] = (Re B, -Im B),
//   B'_im[2j..2j+1, n] = (Im B, Re B);  C = A' [B'_re | B'_im] = [Re F | Im F].
// Split precision: operands are scaled by 2^12 (exact) and split as
// x 2^12 = hi + lo with hi, lo FP16; the scale keeps lo a normal FP16 number
// for every |x| >= 2^-15 (below that the absolute error is < 2^-36).  The three
// products hi*hi + hi*lo + lo*hi (error ~2^-22 relative) accumulate into ONE
// TMEM accumulator (FP32, units of 2^24).  Two accumulators alternate: while the
// MMAs fill one, the flush warps fold the other into a Kahan-compensated FP32
// running total also kept in TMEM.  This bounds every tensor-core accumulation
// chain to flush_stages x 12 MMAs (the tensor core's FP32 accumulation loses
// accuracy with chain length: 1.2e-6 rel-L2 at 4 stages, 5.2e-6 at 64).  At
// the end of the particle range the total is added to an FP64 accumulator in
// global memory (one RED.ADD.F64 per frequency and work item), which a
// finalize kernel converts to the float2 spectrum.
//
// CTA tile: M = 128 rows (a, b) (8-row chunks of constant a), N = 64 c values
// (128 real columns), K = 32 particles (64 real) per pipeline stage, 3 stages.
// Warp roles:
//   warp 0       allocates TMEM, one thread issues tcgen05.mma / commit;
//   warps 1-4    flush TMEM (warp w reads lanes 32 (w % 4) .. +31);
//   warps 5-16   generate operands straight into shared memory in the
//                canonical no-swizzle K-major layout (8x16-byte core matrices;
//                16 bytes of padding between K columns of core matrices keep
//                the stores free of bank conflicts), by recurrences along b and
//                c (8 steps from an exact fixed-point start, moving away from
//                the axis origin so Gaussian factors only shrink along a chain);
//   warp 17      streams the per-particle constants of each stage into shared
//                memory with cp.async.bulk (global -> own CTA, no multicast),
//                three stages ahead.
// Per-particle constants (fixed-point positions, unit rotations, Gaussian
// ratios) are computed once per launch by tc_prep_kernel.
//
// Every mbarrier wait is bounded (2 s of %globaltimer); a wait that runs out
// sets *error_flag, raises the CTA's abort flag, and all roles leave their
// loops; warp 0 drains its MMAs (bounded) before releasing TMEM.  The host
// reports a non-zero flag at the next synchronising call.  No TMA tensor maps,
// no clusters, no multicast.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>

#include "mv_device.cuh"
#include "mv_internal.h"

namespace mv {

namespace {

constexpr int kM = 128;
constexpr int kNc = 64;
constexpr int kN = 2 * kNc;
constexpr int kKp = 32;
constexpr int kKr = 2 * kKp;
constexpr int kStages = 3;
constexpr int kCoreBytes = 128;
constexpr int kLbo = 16 * kCoreBytes + 16;          // bytes between K-adjacent core matrices
constexpr int kOperandBytes = (kKr / 8) * kLbo;     // 8 K-columns of 16 core matrices
constexpr int kStageBytes = 4 * kOperandBytes;      // A_hi, A_lo, B_hi, B_lo
constexpr int kParticleBytes = 48;                  // sizeof(TcParticle)
constexpr int kSlotBytes = kKp * kParticleBytes;    // particle constants of one stage
constexpr int kProducerWarps = 12;  // 8 warps of A units + 4 warps of B units, 2 chains each
constexpr int kFlushWarps = 4;
constexpr int kLoaderWarp = 1 + kFlushWarps + kProducerWarps;
constexpr int kThreads = 32 * (kLoaderWarp + 1);
constexpr int kProducerThreads = 32 * kProducerWarps;
constexpr int kFlushThreads = 32 * kFlushWarps;
constexpr uint32_t kTmemCols = 512;  // accumulator 0 | accumulator 1 | total | compensation
constexpr uint32_t kColTotal = 2 * kN, kColComp = 3 * kN;
constexpr float kOperandScale = 4096.f;                     // 2^12 per operand
constexpr float kInvProductScale = 1.f / (4096.f * 4096.f);  // 2^-24
constexpr unsigned long long kWaitLimitNs = 2000000000ull;
constexpr size_t kBarrierOffset = (size_t)kStages * (kStageBytes + kSlotBytes);
constexpr size_t kSmemBytes = kBarrierOffset + 256;

// idesc of tcgen05.mma kind::f16: D F32, A/B F16, both K-major, N = 128, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | ((uint32_t)(kN >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);

// Per-particle constants of one group, computed once per launch by
// tc_prep_kernel (48 bytes, three float4 loads).
struct __align__(16) TcParticle {
    uint32_t qx, qy, qz;  // fixed-point turns of step * position
    float amp;            // 2^12 w / W
    float gam;            // -pi log2(e) step^2 h^2 (GAUSSIAN_DECAYING), else 0
    float rho2;           // exp2(2 gam): ratio of successive Gaussian step factors
    float2 ry, rz;        // exp(-2 pi i Qy / 2^32), exp(-2 pi i Qz / 2^32), accurate
    float pad[2];
};
static_assert(sizeof(TcParticle) == kParticleBytes, "TcParticle layout");

struct TcArgs {
    const TcParticle* tp;
    int k_begin, k_end;  // particle range of the group
    int kx, ky, lz_tc;   // lattice extents; c planes [0, lz_tc) are summed here
    int n_mtiles, n_ntiles;
    int k_chunk;  // particles per work item (multiple of kKp)
    int flush_stages;  // stages per TMEM accumulation chain (4 MMA K-steps each)
    double wmax;
    double* acc;  // [(a_idx * ky + b_idx) * lz_tc + c][2]
    int* error_flag;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: returns false (after flagging) if the phase does not complete
// within kWaitLimitNs or the CTA is already aborting.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag, int* error_flag,
                                          int code) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (true) {
        if (*abort_flag) return false;
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > kWaitLimitNs) {
            *abort_flag = 1;
            atomicOr(error_flag, code);
            return false;
        }
    }
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Plain bulk copy global -> this CTA's shared memory, completing on an mbarrier.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((kLbo >> 4) & 0x3FFF) << 16;        // leading (K) byte offset
    d |= (uint64_t)((kCoreBytes >> 4) & 0x3FFF) << 32;  // stride (M/N) byte offset
    d |= (uint64_t)1 << 46;                              // descriptor version (sm_100)
    return d;                                            // base offset 0, no swizzle
}

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float* v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};" ::"r"(taddr),
        "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "f"(v[8]),
        "f"(v[9]), "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15])
        : "memory");
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// exp(-2 pi i q / 2^32) for a fixed-point turn count q, accurate to ~1 ulp:
// q = hi + lo with hi a multiple of 2^16 (exact in FP32) and |lo| < 2^16.
__device__ __forceinline__ float2 unit_phase(uint32_t q) {
    const int32_t qi = (int32_t)q;
    const int32_t hi = qi & (int32_t)0xFFFF0000;
    const int32_t lo = qi - hi;  // in [0, 65536)
    float sh, ch;
    sincospif((float)hi * (1.0f / 2147483648.0f), &sh, &ch);
    const float th = (float)lo * (kPiF / 2147483648.0f);  // |th| < pi 2^-15
    const float th2 = th * th;
    const float sl = th * fmaf(th2, -1.0f / 6.0f, 1.0f);
    const float cl = fmaf(th2, -0.5f, 1.0f);
    const float s = fmaf(sh, cl, ch * sl);
    const float c = fmaf(ch, cl, -sh * sl);
    return make_float2(c, -s);
}

// Two complex values (already scaled by 2^12) -> FP16 hi and lo pairs.
__device__ __forceinline__ uint2 pack_hi_lo(float2 z0, float2 z1, uint2* lo_out) {
    const __half2 h0 = __floats2half2_rn(z0.x, z0.y);
    const __half2 h1 = __floats2half2_rn(z1.x, z1.y);
    const float2 f0 = __half22float2(h0), f1 = __half22float2(h1);
    const __half2 l0 = __floats2half2_rn(z0.x - f0.x, z0.y - f0.y);
    const __half2 l1 = __floats2half2_rn(z1.x - f1.x, z1.y - f1.y);
    lo_out->x = *reinterpret_cast<const uint32_t*>(&l0);
    lo_out->y = *reinterpret_cast<const uint32_t*>(&l1);
    return make_uint2(*reinterpret_cast<const uint32_t*>(&h0), *reinterpret_cast<const uint32_t*>(&h1));
}

__device__ __forceinline__ uint32_t h2_swap_negate(uint32_t h, bool negate_second) {
    // (re, im) -> (re, -im) when negate_second, else (im, re)
    if (negate_second) return h ^ 0x80000000u;
    return (h >> 16) | (h << 16);
}

template <bool GAUSS>
__global__ void __launch_bounds__(kThreads, 1) tc_sum_kernel(TcArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* slots = smem + kStages * kStageBytes;  // [kStages][kSlotBytes]
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kBarrierOffset);
    uint64_t* full = bars;                   // [kStages] producers -> MMA
    uint64_t* empty = bars + kStages;        // [kStages] MMA -> producers
    uint64_t* pdata = bars + 2 * kStages;    // [kStages] loader -> producers
    uint64_t* acc_full = bars + 3 * kStages;   // [2] MMA -> flush
    uint64_t* acc_empty = acc_full + 2;         // [2] flush -> MMA
    uint64_t* drain = acc_full + 4;
    volatile uint32_t* tmem_slot = reinterpret_cast<volatile uint32_t*>(acc_full + 5);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(acc_full + 5) + 1;

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;

    const int items_per_split = a.n_mtiles * a.n_ntiles;
    const int ks = blockIdx.x / items_per_split;
    const int ft = blockIdx.x % items_per_split;
    const int m_tile = ft / a.n_ntiles;
    const int n_tile = ft % a.n_ntiles;
    const int kb = a.k_begin + ks * a.k_chunk;
    const int ke = min(a.k_end, kb + a.k_chunk);
    const int n_stages = max(0, (ke - kb + kKp - 1) / kKp);
    const int flush_stages = a.flush_stages;
    const int n_chunks = (n_stages + flush_stages - 1) / flush_stages;

    if (tid == 0) {
        for (int i = 0; i < kStages; ++i) {
            mbar_init(&full[i], kProducerThreads);
            mbar_init(&empty[i], 1);
            mbar_init(&pdata[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&acc_full[i], 1);
            mbar_init(&acc_empty[i], kFlushThreads);
        }
        mbar_init(drain, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32((const void*)tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ------------------------------------------------------------- MMA
        if (lane == 0) {
            for (int s = 0; s < n_stages; ++s) {
                const int buf = s % kStages;
                const int k = s / flush_stages;
                const int b = k & 1;
                const bool first = (s % flush_stages) == 0;
                if (first && k >= 2 && !mbar_wait(&acc_empty[b], ((k >> 1) - 1) & 1, abort_flag, a.error_flag, 1))
                    break;
                if (!mbar_wait(&full[buf], (s / kStages) & 1, abort_flag, a.error_flag, 2)) break;
                tc_fence_after();
                const uint32_t base = smem_u32(smem + buf * kStageBytes);
                const uint32_t a_hi = base, a_lo = base + kOperandBytes;
                const uint32_t b_hi = base + 2 * kOperandBytes, b_lo = base + 3 * kOperandBytes;
                const uint32_t d = tmem + (uint32_t)(b * kN);
#pragma unroll
                for (int t = 0; t < kKr / 16; ++t) {
                    const uint32_t off = (uint32_t)(2 * t * kLbo);
                    mma_f16(d, smem_desc(a_hi + off), smem_desc(b_hi + off), (first && t == 0) ? 0u : 1u);
                    mma_f16(d, smem_desc(a_hi + off), smem_desc(b_lo + off), 1u);
                    mma_f16(d, smem_desc(a_lo + off), smem_desc(b_hi + off), 1u);
                }
                mma_commit(&empty[buf]);
                if ((s % flush_stages) == flush_stages - 1 || s == n_stages - 1) mma_commit(&acc_full[b]);
            }
            mma_commit(drain);
        }
        __syncwarp();
    } else if (warp <= kFlushWarps) {
        // ----------------------------------------------------------- flush
        const int quarter = warp & 3;
        const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16);
        const int row = quarter * 32 + lane;  // M row owned by this thread
        for (int k = 0; k < n_chunks; ++k) {
            const int b = k & 1;
            if (!mbar_wait(&acc_full[b], (k >> 1) & 1, abort_flag, a.error_flag, 4)) break;
            tc_fence_after();
            const bool last = k == n_chunks - 1;
#pragma unroll 1
            for (int cc = 0; cc < kN / 16; ++cc) {
                float dv[16], tt[16], cp[16];
                tmem_ld16(lane_base + b * kN + cc * 16, dv);
                if (k > 0) {
                    tmem_ld16(lane_base + kColTotal + cc * 16, tt);
                    tmem_ld16(lane_base + kColComp + cc * 16, cp);
                }
                tmem_wait_ld();
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const float v = dv[i] * kInvProductScale;
                    if (k == 0) {
                        tt[i] = v;
                        cp[i] = 0.f;
                    } else {
                        const float y = v - cp[i];
                        const float t = tt[i] + y;
                        cp[i] = (t - tt[i]) - y;
                        tt[i] = t;
                    }
                }
                if (!last) {
                    tmem_st16(lane_base + kColTotal + cc * 16, tt);
                    tmem_st16(lane_base + kColComp + cc * 16, cp);
                } else {
                    // add the item's total to the FP64 accumulator
                    const int rho = m_tile * kM + row;
                    const int c0 = n_tile * kNc;
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        const int n = cc * 16 + i;
                        const int c = c0 + (n % kNc);
                        if (c < a.lz_tc) {
                            const double v = ((double)tt[i] - (double)cp[i]) * a.wmax;
                            atomicAdd(a.acc + ((size_t)rho * a.lz_tc + c) * 2 + (n / kNc), v);
                        }
                    }
                }
            }
            tmem_wait_st();
            tc_fence_before();
            mbar_arrive(&acc_empty[b]);
        }
    } else if (warp == kLoaderWarp) {
        // ---------------------------------------------------------- loader
        if (lane == 0) {
            for (int s = 0; s < n_stages; ++s) {
                const int buf = s % kStages;
                // the producers are done with this slot once stage s - kStages is full
                if (s >= kStages && !mbar_wait(&full[buf], ((s / kStages) - 1) & 1, abort_flag, a.error_flag, 32))
                    break;
                const int j0 = kb + s * kKp;
                const uint32_t bytes = (uint32_t)(min(kKp, ke - j0) * kParticleBytes);
                mbar_arrive_expect_tx(&pdata[buf], bytes);
                bulk_copy_g2s(slots + buf * kSlotBytes, a.tp + j0, bytes, &pdata[buf]);
            }
        }
        __syncwarp();
    } else {
        // -------------------------------------------------------- producers
        const int p = tid - 32 * (1 + kFlushWarps);
        const int pp = p & 15;  // particle pair within the stage
        // A unit (p < 256): 8-row chunk rc of the M tile
        const bool has_a = p < 256;
        const int rc = (p >> 4) & 15;
        const int rho0 = m_tile * kM + rc * 8;
        const int a_x = rho0 / a.ky - a.kx / 2;
        const int b0 = rho0 % a.ky - a.ky / 2;
        const bool a_up = b0 >= 0;
        const int b_s = a_up ? b0 : b0 + 7;
        // B unit (p >= 256): 8-column chunk cb of the N tile
        const int cb = (p >> 4) & 7;
        const int c_s = n_tile * kNc + cb * 8;

        for (int s = 0; s < n_stages; ++s) {
            const int buf = s % kStages;
            if (!mbar_wait(&pdata[buf], (s / kStages) & 1, abort_flag, a.error_flag, 64)) break;
            uint32_t pqx[2], pqy[2], pqz[2];
            float pamp[2], pgam[2], prho2[2];
            float2 pry[2], prz[2];
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int jj = 2 * pp + e;
                if (kb + s * kKp + jj < ke) {
                    const float4* src = reinterpret_cast<const float4*>(slots + buf * kSlotBytes + jj * kParticleBytes);
                    const float4 v0 = src[0], v1 = src[1], v2 = src[2];
                    pqx[e] = __float_as_uint(v0.x);
                    pqy[e] = __float_as_uint(v0.y);
                    pqz[e] = __float_as_uint(v0.z);
                    pamp[e] = v0.w;
                    pgam[e] = v1.x;
                    prho2[e] = v1.y;
                    pry[e] = make_float2(v1.z, v1.w);
                    prz[e] = make_float2(v2.x, v2.y);
                } else {
                    pqx[e] = pqy[e] = pqz[e] = 0u;
                    pamp[e] = 0.f;
                    pgam[e] = 0.f;
                    prho2[e] = 1.f;
                    pry[e] = prz[e] = make_float2(1.f, 0.f);
                }
            }
            if (!mbar_wait(&empty[buf], ((s / kStages) & 1) ^ 1, abort_flag, a.error_flag, 8)) break;
            uint8_t* st = smem + buf * kStageBytes;
            float2 z[2], R[2];
            float q[2], rq[2];
            if (has_a) {
                // ---- A: rows rc*8 .. rc*8+7, particles 2pp, 2pp+1 (amp includes 2^12)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    float sn, cs;
                    __sincosf(turns_to_radians((uint32_t)a_x * pqx[e] + (uint32_t)b_s * pqy[e]), &sn, &cs);
                    float g = pamp[e];
                    if constexpr (GAUSS) g *= exp2f(pgam[e] * (float)(a_x * a_x + b_s * b_s));
                    z[e] = make_float2(g * cs, -g * sn);
                    R[e] = a_up ? pry[e] : make_float2(pry[e].x, -pry[e].y);
                    if constexpr (GAUSS) {
                        q[e] = exp2f(pgam[e] * (float)(2 * (a_up ? b_s : -b_s) + 1));
                        rq[e] = prho2[e];
                    } else {
                        q[e] = 1.f;
                        rq[e] = 1.f;
                    }
                }
                uint8_t* ahi = st;
                uint8_t* alo = st + kOperandBytes;
                const int col = (pp >> 1) * kLbo + rc * kCoreBytes + (pp & 1) * 8;
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int r = a_up ? i : 7 - i;
                    uint2 lo;
                    const uint2 hi = pack_hi_lo(z[0], z[1], &lo);
                    *reinterpret_cast<uint2*>(ahi + col + r * 16) = hi;
                    *reinterpret_cast<uint2*>(alo + col + r * 16) = lo;
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const float rx = R[e].x * q[e], ry = R[e].y * q[e];
                        const float nx = fmaf(z[e].x, rx, -z[e].y * ry);
                        const float ny = fmaf(z[e].x, ry, z[e].y * rx);
                        z[e] = make_float2(nx, ny);
                        if constexpr (GAUSS) q[e] *= rq[e];
                    }
                }
            } else {
                // ---- B: columns cb*8 .. cb*8+7 (Re) and 64 + ... (Im), scaled by 2^12
                const bool live = c_s < a.lz_tc;
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    float sn, cs;
                    __sincosf(turns_to_radians((uint32_t)c_s * pqz[e]), &sn, &cs);
                    float g = live ? kOperandScale : 0.f;
                    if constexpr (GAUSS) g *= exp2f(pgam[e] * (float)(c_s * c_s));
                    z[e] = make_float2(g * cs, -g * sn);
                    R[e] = prz[e];
                    if constexpr (GAUSS) {
                        q[e] = exp2f(pgam[e] * (float)(2 * c_s + 1));
                        rq[e] = prho2[e];
                    } else {
                        q[e] = 1.f;
                        rq[e] = 1.f;
                    }
                }
                uint8_t* bhi = st + 2 * kOperandBytes;
                uint8_t* blo = st + 3 * kOperandBytes;
                const int kcol = (pp >> 1) * kLbo + (pp & 1) * 8;
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    uint2 lo;
                    const uint2 hi = pack_hi_lo(z[0], z[1], &lo);
                    const int re_off = kcol + cb * kCoreBytes + i * 16;
                    const int im_off = kcol + (8 + cb) * kCoreBytes + i * 16;
                    *reinterpret_cast<uint2*>(bhi + re_off) =
                        make_uint2(h2_swap_negate(hi.x, true), h2_swap_negate(hi.y, true));
                    *reinterpret_cast<uint2*>(blo + re_off) =
                        make_uint2(h2_swap_negate(lo.x, true), h2_swap_negate(lo.y, true));
                    *reinterpret_cast<uint2*>(bhi + im_off) =
                        make_uint2(h2_swap_negate(hi.x, false), h2_swap_negate(hi.y, false));
                    *reinterpret_cast<uint2*>(blo + im_off) =
                        make_uint2(h2_swap_negate(lo.x, false), h2_swap_negate(lo.y, false));
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const float rx = R[e].x * q[e], ry = R[e].y * q[e];
                        const float nx = fmaf(z[e].x, rx, -z[e].y * ry);
                        const float ny = fmaf(z[e].x, ry, z[e].y * rx);
                        z[e] = make_float2(nx, ny);
                        if constexpr (GAUSS) q[e] *= rq[e];
                    }
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive(&full[buf]);
        }
    }

    // ------------------------------------------------------------- teardown
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) {
        // all MMAs this CTA issued are complete before TMEM is released (this
        // wait ignores the abort flag; it is bounded on its own)
        {
            const unsigned long long t0 = global_ns();
            while (!mbar_try_wait(drain, 0)) {
                if (global_ns() - t0 > kWaitLimitNs) {
                    atomicOr(a.error_flag, 16);
                    break;
                }
            }
        }
        __syncwarp();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

struct TcPrepArgs {
    const float4* particles;
    const float* radii;
    int n;
    double step;
    float gamma_scale;
    float inv_wmax;
    bool gauss;
    TcParticle* out;
};

__global__ void tc_prep_kernel(TcPrepArgs p) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= p.n) return;
    const float4 q = p.particles[j];
    TcParticle t;
    t.qx = fixed_turns(p.step * (double)q.x);
    t.qy = fixed_turns(p.step * (double)q.y);
    t.qz = fixed_turns(p.step * (double)q.z);
    t.amp = q.w * p.inv_wmax * kOperandScale;
    if (p.gauss) {
        const float h = p.radii[j];
        t.gam = p.gamma_scale * h * h;
    } else {
        t.gam = 0.f;
    }
    t.rho2 = exp2f(2.f * t.gam);
    t.ry = unit_phase(t.qy);
    t.rz = unit_phase(t.qz);
    t.pad[0] = t.pad[1] = 0.f;
    p.out[j] = t;
}

// acc (FP64) -> float2 spectrum planes c in [0, lz_tc): times the per-frequency
// Phi^ factor (groups whose Phi^ factors out) and the scale, written or added.
struct TcFinalizeArgs {
    const double* acc;
    int kx, ky, lz_tc, lz_out;
    double step;
    int basis;
    double h;  // radius of the factored Phi^(|k| h); 1 without radii
    bool factored;
    double scale;
    float2* out;
    bool accumulate;
};

__global__ void tc_finalize_kernel(TcFinalizeArgs f) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long count = (long long)f.kx * f.ky * f.lz_tc;
    if (q >= count) return;
    const int c = (int)(q % f.lz_tc);
    const long long rho = q / f.lz_tc;
    const int b = (int)(rho % f.ky) - f.ky / 2;
    const int a = (int)(rho / f.ky) - f.kx / 2;
    double factor = f.scale;
    if (f.factored) {
        const double k = f.step * sqrt((double)a * a + (double)b * b + (double)c * c);
        factor *= phi_fp64(f.basis, k * f.h);
    }
    const float re = (float)(f.acc[2 * q] * factor), im = (float)(f.acc[2 * q + 1] * factor);
    const size_t idx = (size_t)rho * f.lz_out + c;
    if (f.accumulate) {
        const float2 o = f.out[idx];
        f.out[idx] = make_float2(o.x + re, o.y + im);
    } else {
        f.out[idx] = make_float2(re, im);
    }
}

bool is_spectrum_lattice(const Lattice& L) {
    if (L.nx < 2 || L.ny < 2 || L.nz < 2) return false;
    if (L.x0 != -L.nx / 2 || L.y0 != -L.ny / 2 || L.z0 != 0) return false;
    const double s = L.kx;
    if (!(s > 0) || L.ky != s || L.kz != s) return false;
    return L.m[0] == s && L.m[4] == s && L.m[8] == s && L.m[1] == 0 && L.m[2] == 0 && L.m[3] == 0 && L.m[5] == 0 &&
           L.m[6] == 0 && L.m[7] == 0;
}

// Stages per TMEM accumulation chain before the flush into the compensated
// total: MV_TC_FLUSH_STAGES (1..1024) overrides the default.
int tc_flush_stages() {
    static const int v = [] {
        const char* e = std::getenv("MV_TC_FLUSH_STAGES");
        const int x = e ? std::atoi(e) : 0;
        return (x >= 1 && x <= 1024) ? x : 8;
    }();
    return v;
}

}  // namespace

int tensor_sum_available(const SumRequest& r) {
    const Lattice& L = r.lat;
    if (!is_spectrum_lattice(L) || r.wrap != 0) return 0;
    const int lz_tc = L.nz - 1;  // planes [0, Kz/2); the Nyquist plane goes to the plain form
    if (L.ny % 16 || ((long long)L.nx * L.ny) % kM || lz_tc % 8 || lz_tc < 8) return 0;
    if ((long long)L.nx * L.ny * lz_tc * 2 > (1LL << 31)) return 0;
    if (r.weight_max < 0.f) return 0;  // needs the registered |weight| maximum
    const bool uniform = r.radii && r.radius_min >= 0.f && r.radius_min == r.radius_max;
    const bool separable = !r.radii || uniform || r.basis == kGaussianDecaying;
    return separable ? 1 : 0;
}

int launch_tensor_sum(const SumRequest& req, Workspace& ws, Workspace& acc, KernelTimer* timer) {
    const Lattice& L = req.lat;
    const int kx = L.nx, ky = L.ny, lz_out = L.nz, lz_tc = L.nz - 1;
    const bool uniform = req.radii && req.radius_min >= 0.f && req.radius_min == req.radius_max;
    const bool gauss = req.radii && !uniform && req.basis == kGaussianDecaying;
    const bool factored = !gauss;
    const size_t acc_count = (size_t)kx * ky * lz_tc;
    int st = acc.reserve(acc_count * 2 * sizeof(double));
    if (st != kOk) return st;
    st = check_cuda(cudaMemsetAsync(acc.ptr, 0, acc_count * 2 * sizeof(double), req.stream), "cudaMemsetAsync");
    if (st != kOk) return st;

    if (req.n > 0 && req.weight_max > 0.f) {
        st = ws.reserve((size_t)req.n * sizeof(TcParticle));
        if (st != kOk) return st;
        TcPrepArgs pa;
        pa.particles = req.particles;
        pa.radii = req.radii;
        pa.n = req.n;
        pa.step = L.kx;
        pa.gamma_scale = gauss ? (float)(-(double)kPiLog2e * L.kx * L.kx) : 0.f;
        pa.inv_wmax = 1.0f / req.weight_max;
        pa.gauss = gauss;
        pa.out = static_cast<TcParticle*>(ws.ptr);
        tc_prep_kernel<<<(req.n + 255) / 256, 256, 0, req.stream>>>(pa);
        count_launch();
        st = check_cuda(cudaGetLastError(), "tc_prep_kernel launch");
        if (st != kOk) return st;

        TcArgs a;
        a.tp = pa.out;
        a.k_begin = 0;
        a.k_end = req.n;
        a.kx = kx;
        a.ky = ky;
        a.lz_tc = lz_tc;
        a.n_mtiles = (int)((long long)kx * ky / kM);
        a.n_ntiles = (lz_tc + kNc - 1) / kNc;
        const long long ftiles = (long long)a.n_mtiles * a.n_ntiles;
        // particle splits: enough items for ~4 waves, at least 64 stages each
        const long long target = (long long)device_sm_count() * 4;
        long long splits = std::max<long long>(1, (target + ftiles - 1) / ftiles);
        splits = std::min<long long>(splits, std::max<long long>(1, (req.n + 64 * kKp - 1) / (64 * kKp)));
        long long chunk = ((req.n + splits - 1) / splits + kKp - 1) / kKp * kKp;
        splits = (req.n + chunk - 1) / chunk;
        if (ftiles * splits > (1LL << 31) - 1) return set_error(kInvalidValue, "tensor sum: too many work items");
        a.k_chunk = (int)chunk;
        a.flush_stages = tc_flush_stages();
        a.wmax = req.weight_max;
        a.acc = static_cast<double*>(acc.ptr);
        a.error_flag = req.error_flag;
        auto kern = gauss ? tc_sum_kernel<true> : tc_sum_kernel<false>;
        st = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes),
                        "cudaFuncSetAttribute");
        if (st != kOk) return st;
        timer_begin(timer, 3, req.stream);
        kern<<<(unsigned)(ftiles * splits), kThreads, kSmemBytes, req.stream>>>(a);
        count_launch();
        timer_end(timer, 3, req.stream);
        st = check_cuda(cudaGetLastError(), "tc_sum_kernel launch");
        if (st != kOk) return st;
    }

    TcFinalizeArgs f;
    f.acc = static_cast<const double*>(acc.ptr);
    f.kx = kx;
    f.ky = ky;
    f.lz_tc = lz_tc;
    f.lz_out = lz_out;
    f.step = L.kx;
    f.basis = req.basis;
    f.h = uniform ? (double)req.radius_max : 1.0;
    f.factored = factored;
    f.scale = req.scale;
    f.out = req.out;
    f.accumulate = req.accumulate;
    const long long count = (long long)acc_count;
    tc_finalize_kernel<<<(unsigned)((count + 255) / 256), 256, 0, req.stream>>>(f);
    count_launch();
    st = check_cuda(cudaGetLastError(), "tc_finalize_kernel launch");
    if (st != kOk) return st;

    // The Nyquist plane l = Kz/2 with the plain form.
    SumRequest nyq = req;
    nyq.lat.z0 = lz_tc;
    nyq.lat.nz = 1;
    nyq.out_base = lz_tc;
    nyq.out_sx = (long long)ky * lz_out;
    nyq.out_sy = lz_out;
    nyq.out_sz = 1;
    return launch_plain_sum(nyq, ws, nullptr);
}

}  // namespace mv
