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
// A CTA-pair MMA of K = 16 costs about the same whatever its N up to 256, so
// jobs are shaped for N = 256 (128 frequency columns per n-tile): groups of
// pure phases fold F rows of b into the columns (rows (a, bh), columns (b mod
// F, c); TcJob::fold), and groups with per-particle Gaussian factors on
// lattices with more b values than planes exchange the axes (rows (a, c),
// columns b; TcJob::exch).
//
// Real embedding with re/im interleaved along K (k = 2j + {0,1}):
//   A'[m, 2j..2j+1] = (Re A, Im A),  B'_re[2j..2j+1, n] = (Re B, -Im B),
//   B'_im[2j..2j+1, n] = (Im B, Re B);  C = A' [B'_re | B'_im] = [Re F | Im F].
// Split precision: operands are scaled by 2^12 (exact) and split as
// x 2^12 = hi + lo with hi, lo FP16; the scale keeps lo a normal FP16 number
// for every |x| >= 2^-15 (below that the absolute error is < 2^-36).  The three
// products hi*hi + hi*lo + lo*hi (error ~2^-22 relative) accumulate into ONE
// TMEM accumulator (FP32, units of 2^24; 256 columns).  Every flush_stages
// stages (a chain of flush_stages x 12 MMAs; the tensor core's FP32
// accumulation loses accuracy with chain length: 1.6e-6 rel-L2 at 4 stages,
// 2.4e-6 at 8, 4.1e-6 at 16) the MMA pauses while the flush warps add the
// accumulator into an FP32 total in the other 256 TMEM columns.  A work item
// (one particle range of one tile) owns a slot of global memory: at its end
// an item of at most kMaxItemChains chains stores its FP32 total there once,
// and a longer item adds its FP32 total of every kMaxItemChains chains into
// FP64 totals there, with coalesced loads and stores (a warp's rows are
// contiguous).  No atomics: tc_reduce_kernel
// then sums every element's slots over particle chunks and jobs (groups,
// h-bins) in FP64, in a fixed order, and adds the result to the float2
// spectrum, so results are bitwise reproducible.
//
// The Nyquist plane c = Kz/2 is the same kind of GEMM with the axes
// exchanged: rows b with the fixed frequency Kz/2 on z, columns a on x (two
// jobs, a >= 0 and, by F(-a, b, c) = conj F(a, -b, -c), a < 0; see TcJob), so
// it runs as 1/Kx of the other planes' tiles in the same launch instead of a
// plain-form pass.
//
// CTA tile: M = 128 rows (a, b) (8-row chunks of constant a), N = up to 128 c
// values (256 real columns), K = 32 particles (64 real) per pipeline stage;
// CTA pairs run M = 256 over both CTAs (tile kinds and operand rings at
// TileMode and Shape below).
// Warp roles:
//   warp 0       allocates TMEM, one thread issues tcgen05.mma / commit;
//   warps 1-4    flush TMEM (warp w reads lanes 32 (w % 4) .. +31);
//   warps 5-16   generate operands straight into shared memory (8 warps of A
//                row chunks, 4 of B c chunks, two chunks per thread) in the
//                128-byte swizzled K-major layout (one 128-byte row of 64 FP16
//                per operand row and stage; the swizzle lets the tensor core
//                read at full rate and keeps the stores free of bank
//                conflicts), by recurrences along b and
//                c (8 steps from an exact fixed-point start, moving away from
//                the axis origin so Gaussian factors only shrink along a chain);
//   warp 17      lane 0 streams the per-particle constants of each stage into
//                shared memory with cp.async.bulk (global -> own CTA, no
//                multicast), up to the pipeline depth ahead; lane 1, once the
//                MMA has read a stage buffer, arrives on its full barrier, for
//                jobs with B-operand images together with the bulk copy of the
//                stage's B image (the B warps then idle).
// Per-particle constants (fixed-point positions, unit rotations, Gaussian
// ratios) are computed once per launch by tc_prep_kernel into 32-particle
// field-by-field blocks.  B-operand images (the B stages of a job whose m-tiles
// all read the same ones) are computed once per launch by tc_bimg_kernel, with
// the producers' own arithmetic, and read from L2 by every m-tile.
//
// Every mbarrier wait is bounded (2 s of %globaltimer); a wait that runs out
// sets *error_flag, raises the CTA's abort flag, and all roles leave their
// loops; warp 0 drains its MMAs (bounded) before releasing TMEM.  The host
// reports a non-zero flag at the next synchronising call.  No TMA tensor maps
// and no multicast loads (only tcgen05.commit signals both CTAs of a pair);
// clusters of 2 only for the CTA-pair tiles.
#include <cuda_fp16.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include <cub/device/device_radix_sort.cuh>

#include "meshless_vis_b200.h"
#include "mv_device.cuh"
#include "mv_internal.h"

namespace mv {

// Per-particle constants of one group, computed once per launch by
// tc_prep_kernel, in blocks of 32 particles laid out field by field (1280
// bytes per block) so that a producer reads the constants of its particle
// pair with conflict-free 64-bit shared-memory loads, and the loader moves one
// whole block per pipeline stage:
//   qx[32], qy[32], qz[32]  u32 fixed-point turns of step * position
//   amp[32]                 2^12 w / W
//   gam[32]                 -pi log2(e) step^2 h^2 (GAUSSIAN_DECAYING), else 0
//   rho2[32]                exp2(2 gam): ratio of successive Gaussian step factors
//   ry[32], rz[32]          float2 exp(-2 pi i Q / 2^32), accurate
// Particles past the group's end (up to the block boundary) have amp = 0.
constexpr int kBlockParticles = 32;
constexpr int kBlockBytes = 6 * 4 * kBlockParticles + 2 * 8 * kBlockParticles;  // 1280
constexpr int kOffQx = 0, kOffQy = 128, kOffQz = 256, kOffAmp = 384, kOffGam = 512, kOffRho2 = 640, kOffRy = 768,
              kOffRz = 1024;

namespace {

constexpr int kM = 128;
constexpr int kKp = 32;
constexpr int kKr = 2 * kKp;
constexpr int kRowBytes = 2 * kKr;                 // one operand row: 64 FP16 along K = one 128-byte swizzle row
constexpr int kAtomBytes = 8 * kRowBytes;           // 8-row swizzle atom
constexpr int kABytes = kM * kRowBytes;             // A operand: 128 rows
constexpr int kSlotBytes = kBlockBytes;            // particle constants of one stage
constexpr int kProducerWarps = 12;  // 8 warps of A units + 4 warps of B units
constexpr int kFlushWarps = 4;
constexpr int kLoaderWarp = 1 + kFlushWarps + kProducerWarps;
constexpr int kThreads = 32 * (kLoaderWarp + 1);
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kColTotal = 256;  // FP32 total: columns [256, 256 + accumulator columns)
constexpr float kOperandScale = 4096.f;                     // 2^12 per operand
constexpr double kInvProductScale = 1.0 / (4096.0 * 4096.0);  // 2^-24
// An FP32 total in TMEM sums at most this many accumulation chains (random-walk
// rounding of about 2^-24 sqrt(64) of the total) before it goes to the item's
// slot.
constexpr int kMaxItemChains = 64;
constexpr unsigned long long kWaitLimitNs = 2000000000ull;
// After a wait has run out, a CTA idles this long before it releases TMEM and
// exits, so bulk copies it issued (which complete within microseconds) have
// landed in its shared memory.
constexpr unsigned long long kAbortGraceNs = 200000ull;

// Tile kinds (template parameter MODE):
//   kNarrow (lattices with at most 64 tensor planes): 128x128 MMA, two
//       alternating 128-column TMEM accumulators (the MMAs never wait for a
//       flush), 3 stages of 64 KB;
//   kWide: 128x256 MMA, one 256-column accumulator (the MMA waits while a
//       flush reads it), 2 stages of 96 KB;
//   kPair: a CTA pair (cluster of 2) runs one 256x256 MMA (tcgen05
//       cta_group::2): each CTA holds 128 rows of A and the B rows of half the
//       n-tile's c values, and its 128 accumulator rows of all 256 columns in
//       its own TMEM.  Each CTA produces the operands of a narrow tile per
//       stage for twice its work, and the MMA reads 64 B/clk of shared memory
//       per CTA.  Used where the tensor planes are a multiple of 16 and the
//       rows a multiple of 256.
//   kPairNarrow: the CTA pair for lattices with at most 64 tensor planes
//       (planes a multiple of 16, rows of 256): one 256x128 MMA, two
//       alternating 128-column accumulators per CTA as in kNarrow.  Each CTA
//       reads A and half of B, 96 B/clk at the tensor core's rate, where a
//       128x128 MMA needs the port's full 128 B/clk; B work per CTA halves.
//   kPairDB: kPair for jobs of short items (at most kDBMaxChains chains): two
//       alternating 256-column accumulators fill all of TMEM, so the MMAs go
//       on while a flush reads the finished one, and the flush adds it into
//       the item's FP32 slot directly (a read-modify-write in L2; the item's
//       few chains keep its slot there).  Long items keep kPair, whose
//       per-chain slot traffic would no longer stay in L2.
enum TileMode : int { kNarrow = 0, kWide = 1, kPair = 2, kPairNarrow = 3, kPairDB = 4 };
constexpr int kDBMaxChains = 8;

constexpr bool pair_mode(int mode) { return mode == kPair || mode == kPairNarrow || mode == kPairDB; }
constexpr bool narrow_mode(int mode) { return mode == kNarrow || mode == kPairNarrow; }

template <int MODE>
struct Shape {
    static constexpr int kCtas = pair_mode(MODE) ? 2 : 1;
    static constexpr int kN = narrow_mode(MODE) ? 128 : 256;  // accumulator columns: the MMA's N at most
    static constexpr int kNc = kN / 2;                       // c values per n-tile (at most)
    static constexpr int kBRows = kN / kCtas;                // B operand rows held by one CTA
    static constexpr int kMTile = kM * kCtas;                // lattice rows per m-tile
    // Rings: A operands (kAStages), B operands (kBStages: deeper where B may
    // come as a copied image, whose copy starts only once the MMA has read
    // the B buffer it overwrites), particle constants (kSlots).  One full
    // barrier per stage, in a ring as deep as the deeper operand ring (an
    // arrival for stage S + kFull then waits for the MMA to be past stage S).
    static constexpr int kAStages = 3;
    static constexpr int kBStages = MODE == kWide ? 2 : 4;
    static constexpr int kSlots = 2;
    static constexpr int kFull = kAStages > kBStages ? kAStages : kBStages;
    static constexpr bool kDB = MODE == kPairDB;              // totals in the slot, no TMEM total
    static constexpr int kBufs = narrow_mode(MODE) || kDB ? 2 : 1;  // TMEM accumulators, kN columns each
    static constexpr int kBBytes = kBRows * kRowBytes;
    static constexpr int kAStageBytes = 2 * kABytes;  // A_hi, A_lo
    static constexpr int kBStageBytes = 2 * kBBytes;  // B_hi, B_lo (2 bnc rows each, packed)
    static constexpr int kChunksPerThread = kBRows > 128 ? kBRows / 128 : 1;  // 8-c chunks per B producer thread
    static constexpr size_t kBOffset = (size_t)kAStages * kAStageBytes;
    static constexpr size_t kSlotOffset = kBOffset + (size_t)kBStages * kBStageBytes;
    static constexpr size_t kBarrierOffset = kSlotOffset + (size_t)kSlots * kSlotBytes;
    static constexpr size_t kSmemBytes = kBarrierOffset + 256;
};
static_assert(Shape<kNarrow>::kSmemBytes <= 227 * 1024 && Shape<kWide>::kSmemBytes <= 227 * 1024 &&
                  Shape<kPair>::kSmemBytes <= 227 * 1024 && Shape<kPairNarrow>::kSmemBytes <= 227 * 1024,
              "shared memory");

// idesc of tcgen05.mma kind::f16: D F32, A/B F16, both K-major, M = m, N = n.
__host__ __device__ constexpr uint32_t mma_idesc(int m, int n) {
    return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}


struct TcArgs {
    const TcJob* jobs;
    const int2* items;  // (job, local item), longest first
    int n_items;
    int flush_stages;  // stages per TMEM accumulation chain (12 MMAs each)
    int* error_flag;
    unsigned long long wait_limit_ns;  // bound of every mbarrier wait (kWaitLimitNs unless a test shortens it)
    int withhold_first_arrival;        // test hook: CTA 0's loader skips its arrival on the first full barrier
};

// Work of one item as every role sees it.
struct TcItem {
    const TcJob* job;
    int m_tile, n_tile;
    int kb, ke;
    int n_stages, n_chunks;
    int c0, nc;    // the n-tile's first c and c values (a multiple of 8); the MMA's N is 2 nc
    int bc0, bnc;  // the c values whose B rows this CTA produces: all of them, or one half (kPair)
    int row0;      // this CTA's first lattice row
    int a_base, b_base, c_base;  // the job's frequency offsets, in registers for the stage loops
    int period;                  // h-binned or row-folded job: frequency columns per column block (else 0)
    int fold;                    // row-folded job: b steps per row (TcJob::fold), else 1
    const unsigned char* bimg;   // this CTA's B-operand images of the item's n-tile (one per block), or null
    int img_stride, img_bytes;   // bytes between images; bytes of one image (512 bnc)
    void* slot;                  // this CTA's part of the item's slot (TcJob::slots)
    int slot_fp64;               // FP64 totals ([column / 2][128 rows][column % 2]), else FP32 quads
};

template <int MODE>
__device__ __forceinline__ TcItem tc_item(const TcArgs& a, int it, int rank) {
    const int2 v = a.items[it];
    TcItem r;
    r.job = a.jobs + v.x;
    const int tiles = r.job->n_mtiles * r.job->n_ntiles;
    const int ks = v.y / tiles;
    const int ft = v.y % tiles;
    r.m_tile = ft / r.job->n_ntiles;
    r.n_tile = ft % r.job->n_ntiles;
    r.kb = ks * r.job->k_chunk;
    r.ke = min(r.job->n, r.kb + r.job->k_chunk);
    r.n_stages = max(0, (r.ke - r.kb + kKp - 1) / kKp);
    r.n_chunks = (r.n_stages + a.flush_stages - 1) / a.flush_stages;
    r.c0 = r.n_tile * r.job->nc_tile;
    r.nc = min(r.job->nc_tile, r.job->lz_tc - r.c0);
    r.bnc = r.nc / Shape<MODE>::kCtas;
    r.bc0 = r.c0 + rank * r.bnc;
    r.row0 = r.m_tile * Shape<MODE>::kMTile + rank * kM;
    r.a_base = r.job->a_base;
    r.b_base = r.job->b_base;
    r.c_base = r.job->c_base;
    r.period = r.job->period;
    r.fold = r.job->fold > 1 ? r.job->fold : 1;
    r.img_stride = r.job->img_stride;
    r.img_bytes = 4 * r.bnc * kRowBytes;
    r.bimg = r.job->bimg ? r.job->bimg + (size_t)(r.n_tile * Shape<MODE>::kCtas + rank) * r.job->n_blocks *
                                             (size_t)r.img_stride
                         : nullptr;
    r.slot_fp64 = r.job->slot_fp64;
    r.slot = static_cast<char*>(r.job->slots) +
             ((size_t)v.y * r.job->slot_stride + (size_t)rank * kM * 2 * r.job->nc_tile) * (r.slot_fp64 ? 8 : 4);
    return r;
}

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

// Arrive on the barrier at the same shared-memory offset in the pair's CTA 0
// (the leader, which issues the pair's MMAs); release at cluster scope.
__device__ __forceinline__ void mbar_arrive_leader(uint64_t* bar) {
    asm volatile(
        "{\n\t.reg .b32 ra;\n\t"
        "mapa.shared::cluster.u32 ra, %0, 0;\n\t"
        "mbarrier.arrive.release.cluster.shared::cluster.b64 _, [ra];\n\t}" ::"r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// Every thread of both CTAs of the cluster (aligned: the whole warp).
__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: returns false (after flagging) if the phase does not complete
// within kWaitLimitNs or the CTA is already aborting.
// As mbar_try_wait, but a thread that finds the phase incomplete is suspended
// until the phase completes or hint_ns nanoseconds pass, so waiting warps take
// no issue slots from the producers.
__device__ __forceinline__ bool mbar_try_wait_suspend(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}
constexpr uint32_t kSuspendHintNs = 100000;  // 0.1 ms per suspension; the phase's completion wakes the thread first

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag, int* error_flag,
                                          unsigned long long limit_ns, int code) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (true) {
        if (*abort_flag) return false;
        if (mbar_try_wait_suspend(bar, parity, kSuspendHintNs)) return true;
        if (global_ns() - t0 > limit_ns) {
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

// Shared-memory descriptor of a K-major operand in the 128-byte swizzle layout:
// row r of the operand is 128 bytes at (r / 8) * 1024 + (r % 8) * 128, its
// 16-byte chunk j stored at chunk position j ^ (r % 8).  The operand starts on
// a 1024-byte boundary; an MMA's K offset (32 bytes per 16 FP16) is added to the
// start address, and the hardware applies the swizzle on the address bits.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;                              // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)((kAtomBytes >> 4) & 0x3FFF) << 32;  // stride byte offset: between 8-row atoms
    d |= (uint64_t)1 << 46;                              // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;                              // 128-byte swizzle; base offset 0
    return d;
}

// CTAS = 2: the pair's MMA (cta_group::2), issued by one thread of CTA 0; the
// descriptors name this CTA's shared-memory offsets, which hold the operands
// in both CTAs (no output lanes disabled).
template <int CTAS>
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
    if constexpr (CTAS == 1) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
            : "memory");
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8, %9, %10, %11, %12}, p;\n\t}" ::"r"(
                d_tmem),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u), "r"(0u), "r"(0u),
            "r"(0u), "r"(0u)
            : "memory");
    }
}

// Arrives on bar once the MMAs issued so far are complete; CTAS = 2: on the
// barrier at the same offset in both CTAs of the pair.
template <int CTAS>
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    if constexpr (CTAS == 1) {
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(bar))
                     : "memory");
    } else {
        asm volatile(
            "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
                smem_u32(bar)),
            "h"((unsigned short)3)
            : "memory");
    }
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const float* v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};" ::"r"(taddr),
        "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "f"(v[8]),
        "f"(v[9]), "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15]), "f"(v[16]), "f"(v[17]),
        "f"(v[18]), "f"(v[19]), "f"(v[20]), "f"(v[21]), "f"(v[22]), "f"(v[23]), "f"(v[24]), "f"(v[25]), "f"(v[26]),
        "f"(v[27]), "f"(v[28]), "f"(v[29]), "f"(v[30]), "f"(v[31])
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

__device__ __forceinline__ uint32_t h2_bits(__half2 h) { return *reinterpret_cast<const uint32_t*>(&h); }

// A producer's two particles as packed pairs: X = (Re z0, Re z1), Y = (Im z0,
// Im z1), already scaled by 2^12.  split_pair: FP16 hi and lo of (Re, Im) for
// each particle (x: particle 0, y: particle 1); the residuals are packed FMAs.
__device__ __forceinline__ void split_pair(float2 X, float2 Y, uint2& hi, uint2& lo) {
    const __half2 h0 = __floats2half2_rn(X.x, Y.x), h1 = __floats2half2_rn(X.y, Y.y);
    const float2 f0 = __half22float2(h0), f1 = __half22float2(h1);
    const float2 m1 = make_float2(-1.f, -1.f);
    const float2 dx = __ffma2_rn(make_float2(f0.x, f1.x), m1, X);
    const float2 dy = __ffma2_rn(make_float2(f0.y, f1.y), m1, Y);
    hi = make_uint2(h2_bits(h0), h2_bits(h1));
    lo = make_uint2(h2_bits(__floats2half2_rn(dx.x, dy.x)), h2_bits(__floats2half2_rn(dx.y, dy.y)));
}

// One step of both particles' chains: z <- z R, with R = (RX, RY) (NRY =
// -RY) already scaled by this step's Gaussian ratio; then (GAUSS) R <- R rho
// for the next step (without GAUSS the ratio is 1).  Packed: X' = X Rx - Y Ry,
// Y' = X Ry + Y Rx.
template <bool GAUSS>
__device__ __forceinline__ void rotate_pair(float2& X, float2& Y, float2& RX, float2& RY, float2& NRY, float2 RHO) {
    const float2 nx = __ffma2_rn(X, RX, __fmul2_rn(Y, NRY));
    const float2 ny = __ffma2_rn(X, RY, __fmul2_rn(Y, RX));
    X = nx;
    Y = ny;
    if constexpr (GAUSS) {
        RX = __fmul2_rn(RX, RHO);
        RY = __fmul2_rn(RY, RHO);
        NRY = __fmul2_rn(NRY, RHO);
    }
}

__device__ __forceinline__ uint32_t h2_swap_negate(uint32_t h, bool negate_second) {
    // (re, im) -> (re, -im) when negate_second, else (im, re)
    if (negate_second) return h ^ 0x80000000u;
    return (h >> 16) | (h << 16);
}

// Swizzled offsets: row r (a multiple of 8 plus K, K < 8) of an operand,
// pair column col = 8 pp: r * 128 + ((col >> 4) ^ K) * 16 + (col & 15).  With
// base = 128 * (r - K) + (col & 15) and c16 = col & ~15 fixed per thread, a
// chain's step K adds K * 128 + (c16 ^ 16 K): one XOR and one add per step.
__device__ __forceinline__ int sw_step(int c16, int K) { return K * kRowBytes + (c16 ^ (K << 4)); }

// An A unit's 8 rows for its two particles (b moving away from 0: K = i when
// UP, 7 - i otherwise), from the chain start (X, Y); lo goes kABytes after hi.
template <bool GAUSS, bool UP>
__device__ __forceinline__ void a_chain(uint8_t* base, int c16, float2 X, float2 Y, float2 RX, float2 RY, float2 NRY,
                                        float2 Q, float2 RHO) {
    if constexpr (GAUSS) {  // the first step's ratio q0 = Q
        RX = __fmul2_rn(RX, Q);
        RY = __fmul2_rn(RY, Q);
        NRY = __fmul2_rn(NRY, Q);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        uint8_t* p = base + sw_step(c16, UP ? i : 7 - i);
        uint2 hi, lo;
        split_pair(X, Y, hi, lo);
        *reinterpret_cast<uint2*>(p) = hi;
        *reinterpret_cast<uint2*>(p + kABytes) = lo;
        if (i < 7) rotate_pair<GAUSS>(X, Y, RX, RY, NRY, RHO);
    }
}

// A B unit's 8 c values for its two particles: (Re B, -Im B) at re_base (a
// Re F row), (Im B, Re B) at im_base (the Im F row); lo goes lo_gap after hi.
// UP: the chain starts at the unit's first column and rises; otherwise it
// starts at the last and falls (negative frequencies, moving away from 0).
template <bool GAUSS, bool UP>
__device__ __forceinline__ void b_chain(uint8_t* re_base, uint8_t* im_base, int lo_gap, int c16, float2 X, float2 Y,
                                        float2 RX, float2 RY, float2 NRY, float2 Q, float2 RHO) {
    if constexpr (GAUSS) {  // the first step's ratio q0 = Q
        RX = __fmul2_rn(RX, Q);
        RY = __fmul2_rn(RY, Q);
        NRY = __fmul2_rn(NRY, Q);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int off = sw_step(c16, UP ? i : 7 - i);
        uint2 hi, lo;
        split_pair(X, Y, hi, lo);
        *reinterpret_cast<uint2*>(re_base + off) = make_uint2(h2_swap_negate(hi.x, true), h2_swap_negate(hi.y, true));
        *reinterpret_cast<uint2*>(re_base + off + lo_gap) =
            make_uint2(h2_swap_negate(lo.x, true), h2_swap_negate(lo.y, true));
        *reinterpret_cast<uint2*>(im_base + off) = make_uint2(h2_swap_negate(hi.x, false), h2_swap_negate(hi.y, false));
        *reinterpret_cast<uint2*>(im_base + off + lo_gap) =
            make_uint2(h2_swap_negate(lo.x, false), h2_swap_negate(lo.y, false));
        if (i < 7) rotate_pair<GAUSS>(X, Y, RX, RY, NRY, RHO);
    }
}

// Chebyshev polynomial T_q(t) by the three-term recurrence.
__device__ __forceinline__ float chebyshev_t(int q, float t) {
    float t0 = 1.f, t1 = t;
    if (q == 0) return 1.f;
    for (int i = 1; i < q; ++i) {
        const float t2 = fmaf(2.f * t, t1, -t0);
        t0 = t1;
        t1 = t2;
    }
    return t1;
}

// One B unit: the job's columns c_col .. c_col + 7 of a particle pair
// (fixed-point z turns pqz, Gaussian exponents pgam -- for h-binned jobs the
// particles' normalised radii t in their bin; unit rotations RX, RY, NRY = -RY
// and Gaussian ratios RHO as in rotate_pair), into a B operand of bnc c values
// at bhi: rows chunk*8 .. +7 of its Re F half and of its Im F half, hi rows
// then lo rows 2 bnc rows later.  Column c_col is frequency c_col + c_base; in
// an h-binned job (period > 0) it is frequency c_col % period + c_base of
// column block k = c_col / period: in a row-folded job (fold = F > 1) the b
// offset bl = k mod F, whose phase bl Qy (fixed-point y turns pqy) joins the
// chain's start; in an h-binned job (cheb_blocks) Chebyshev block q = k / F,
// weighted by T_q(t).  The chain's 8
// frequencies c_s .. c_s + 7 rise from c_s >= 0 and never cross a block (the
// period is a multiple of 8).  The producer warps run it into the stage
// buffer and tc_bimg_kernel into global memory: one arithmetic for both.
__device__ __forceinline__ void b_unit(uint8_t* bhi, int bnc, int chunk, int col, int c_col, int c_base, int period,
                                       int fold, bool cheb_blocks, const uint32_t* pqz, const uint32_t* pqy,
                                       const float* pgam, bool gauss, float2 RX, float2 RY, float2 NRY, float2 RHO) {
    int c_s = c_col + c_base, cheb = -1;
    uint32_t bl = 0u;
    if (period > 0) {
        const int blk = c_col / period;
        c_s = c_col - blk * period + c_base;
        bl = (uint32_t)(blk % fold);
        if (cheb_blocks) cheb = blk / fold;
    }
    // a unit of negative frequencies (the axis-exchanged jobs' b columns)
    // starts at its top and falls
    const bool down = c_s < 0;
    const int c_t = down ? c_s + 7 : c_s;
    float v[2][3];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        float sn, cs;
        __sincosf(turns_to_radians((uint32_t)c_t * pqz[e] + bl * pqy[e]), &sn, &cs);
        float g = kOperandScale, q = 1.f;
        if (gauss) {
            g *= exp2f(pgam[e] * (float)(c_t * c_t));
            q = exp2f(pgam[e] * (float)(down ? 1 - 2 * c_t : 2 * c_t + 1));
        } else if (cheb >= 0) {
            g *= chebyshev_t(cheb, pgam[e]);
        }
        v[e][0] = g * cs;
        v[e][1] = -g * sn;
        v[e][2] = q;
    }
    const float2 X = make_float2(v[0][0], v[1][0]);
    const float2 Y = make_float2(v[0][1], v[1][1]);
    // bnc and chunk * 8 are multiples of 8: row K of the chain is K within its atom
    uint8_t* re_base = bhi + chunk * 8 * kRowBytes + (col & 15);
    uint8_t* im_base = bhi + (bnc + chunk * 8) * kRowBytes + (col & 15);
    const int c16 = col & ~15;
    const float2 Q = gauss ? make_float2(v[0][2], v[1][2]) : make_float2(1.f, 1.f);
    // falling: the conjugate rotation
    if (down) {
        if (gauss) b_chain<true, false>(re_base, im_base, 2 * bnc * kRowBytes, c16, X, Y, RX, NRY, RY, Q, RHO);
        else b_chain<false, false>(re_base, im_base, 2 * bnc * kRowBytes, c16, X, Y, RX, NRY, RY, Q, RHO);
    } else {
        if (gauss) b_chain<true, true>(re_base, im_base, 2 * bnc * kRowBytes, c16, X, Y, RX, RY, NRY, Q, RHO);
        else b_chain<false, true>(re_base, im_base, 2 * bnc * kRowBytes, c16, X, Y, RX, RY, NRY, Q, RHO);
    }
}

// Persistent: CTA (or CTA pair) b walks items b, b + grid, ... of the
// longest-first item list.  Every role walks the same items in the same
// order, and the pipeline's stage and chain counters (hence mbarrier phases
// and the TMEM accumulator parity) run on across items; TMEM and the barriers
// are set up once per CTA.
//
// kPair: the barriers that gate the pair's MMAs (full, acc_empty) live in CTA
// 0 and count the arrivals of both CTAs; the MMA's completion (a_empty, b_empty,
// acc_full, drain) is signalled to both CTAs by multicast commits; each CTA's
// loader, producers and flush warps otherwise work on their own shared memory
// and TMEM.  Cluster barriers after set-up and before exit keep each CTA's
// shared memory alive while the other may still signal it.
template <int MODE>
__global__ void __launch_bounds__(kThreads, 1) tc_sum_kernel(TcArgs a) {
    using SH = Shape<MODE>;
    constexpr int kAStages = SH::kAStages, kBStages = SH::kBStages, kSlots = SH::kSlots, kFull = SH::kFull;
    constexpr int kBufs = SH::kBufs, kCtas = SH::kCtas;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* a_ring = smem;                   // [kAStages][kAStageBytes]
    uint8_t* b_ring = smem + SH::kBOffset;    // [kBStages][kBStageBytes]
    uint8_t* slots = smem + SH::kSlotOffset;  // [kSlots][kSlotBytes]
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + SH::kBarrierOffset);
    uint64_t* full = bars;                        // [kFull] producers, loader -> MMA (CTA 0's)
    uint64_t* pfull = full + kFull;               // [kFull] kPair, CTA 1: its producers, loader -> its forwarder
    uint64_t* a_empty = pfull + kFull;            // [kAStages] MMA -> A producers
    uint64_t* b_empty = a_empty + kAStages;       // [kBStages] MMA -> B producers, loader
    uint64_t* pdata = b_empty + kBStages;         // [kSlots] loader -> producers
    uint64_t* sfree = pdata + kSlots;             // [kSlots] producers -> loader: the slot has been read
    uint64_t* acc_full = sfree + kSlots;          // [kBufs] MMA -> flush: a chain is complete
    uint64_t* acc_empty = acc_full + 2;         // [kBufs] flush -> MMA (CTA 0's): the accumulator has been read
    uint64_t* drain = acc_full + 4;
    volatile uint32_t* tmem_slot = reinterpret_cast<volatile uint32_t*>(acc_full + 5);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(acc_full + 5) + 1;

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int flush_stages = a.flush_stages;
    const int rank = kCtas == 2 ? (int)cluster_rank() : 0;
    const int unit = blockIdx.x / kCtas, n_units = gridDim.x / kCtas;  // CTA or CTA pair

    // the swizzled operands need a 1024-byte aligned shared-memory window
    if (smem_u32(smem) & 1023u) {
        if (tid == 0) atomicOr(a.error_flag, 128);
        return;
    }

    if (tid == 0) {
        for (int i = 0; i < kFull; ++i) {
            // one arrival per producer warp and one from the loader (with the
            // B image's bytes, if any), plus (kPair) one from CTA 1's forwarder
            mbar_init(&full[i], kProducerWarps + 1 + (kCtas - 1));
            mbar_init(&pfull[i], kProducerWarps + 1);
        }
        for (int i = 0; i < kAStages; ++i) mbar_init(&a_empty[i], 1);
        for (int i = 0; i < kBStages; ++i) mbar_init(&b_empty[i], 1);
        for (int i = 0; i < kSlots; ++i) {
            mbar_init(&pdata[i], 1);
            mbar_init(&sfree[i], kProducerWarps);
        }
        for (int i = 0; i < kBufs; ++i) {
            mbar_init(&acc_full[i], 1);
            mbar_init(&acc_empty[i], kFlushWarps * kCtas);  // one arrival per flush warp of the pair
        }
        mbar_init(drain, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        // kPair: warp 0 of both CTAs allocates the same columns of both TMEMs
        if constexpr (kCtas == 1) {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                             smem_u32((const void*)tmem_slot)),
                         "r"(kTmemCols)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        } else {
            asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                             smem_u32((const void*)tmem_slot)),
                         "r"(kTmemCols)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
        }
    }
    tc_fence_before();
    if constexpr (kCtas == 1) __syncthreads();
    else cluster_sync();  // both CTAs' barriers and TMEM are ready before any cross-CTA signal
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ------------------------------------------------------------- MMA
        // (kPair: CTA 0 issues the pair's MMAs; warp 0 of CTA 1 only
        // allocates and releases TMEM)
        if (lane == 0 && rank == 0) {
            int S = 0, C = 0;  // stages and chains issued so far by this CTA
            for (int it = unit; it < a.n_items && !*abort_flag; it += n_units) {
                const TcItem I = tc_item<MODE>(a, it, 0);
                const uint32_t idesc = mma_idesc(kM * kCtas, 2 * I.nc);
                for (int s = 0; s < I.n_stages; ++s, ++S) {
                    const int fb = S % kFull, ab = S % kAStages, bb = S % kBStages;
                    const int k = C + s / flush_stages;  // chain index
                    const int b = k % kBufs, u = k / kBufs;  // accumulator and its use count
                    const bool first = (s % flush_stages) == 0;
                    // a chain starts once the flush of the accumulator's previous chain has read it
                    if (first && u >= 1 && !mbar_wait(&acc_empty[b], (u - 1) & 1, abort_flag, a.error_flag, a.wait_limit_ns, 1)) break;
                    if (!mbar_wait(&full[fb], (S / kFull) & 1, abort_flag, a.error_flag, a.wait_limit_ns, 2)) break;
                    tc_fence_after();
                    const uint32_t a_hi = smem_u32(a_ring + ab * SH::kAStageBytes), a_lo = a_hi + kABytes;
                    // B: hi rows, then lo rows (2 bnc rows each)
                    const uint32_t b_hi = smem_u32(b_ring + bb * SH::kBStageBytes);
                    const uint32_t b_lo = b_hi + (uint32_t)(2 * I.bnc * kRowBytes);
                    const uint32_t d = tmem + (uint32_t)(b * SH::kN);
#pragma unroll
                    for (int t = 0; t < kKr / 16; ++t) {
                        const uint32_t off = (uint32_t)(32 * t);
                        mma_f16<kCtas>(d, smem_desc(a_hi + off), smem_desc(b_hi + off), idesc,
                                       (first && t == 0) ? 0u : 1u);
                        mma_f16<kCtas>(d, smem_desc(a_hi + off), smem_desc(b_lo + off), idesc, 1u);
                        mma_f16<kCtas>(d, smem_desc(a_lo + off), smem_desc(b_hi + off), idesc, 1u);
                    }
                    mma_commit<kCtas>(&a_empty[ab]);
                    mma_commit<kCtas>(&b_empty[bb]);
                    if ((s % flush_stages) == flush_stages - 1 || s == I.n_stages - 1) mma_commit<kCtas>(&acc_full[b]);
                }
                C += I.n_chunks;
            }
            mma_commit<kCtas>(drain);
        }
        if constexpr (kCtas == 2) {
            // CTA 1's forwarder: once all of this CTA's producer warps have
            // filled a stage (local barrier), one cluster-scope arrival tells
            // CTA 0, whose thread issues the pair's MMAs (one remote release per
            // stage instead of one per producer warp)
            if (lane == 0 && rank == 1) {
                int S = 0;
                for (int it = unit; it < a.n_items && !*abort_flag; it += n_units) {
                    const TcItem I = tc_item<MODE>(a, it, 1);
                    int s = 0;
                    for (; s < I.n_stages; ++s, ++S) {
                        const int fb = S % kFull;
                        if (!mbar_wait(&pfull[fb], (S / kFull) & 1, abort_flag, a.error_flag, a.wait_limit_ns, 256)) break;
                        mbar_arrive_leader(&full[fb]);
                    }
                    if (s < I.n_stages) break;
                }
            }
        }
        __syncwarp();
    } else if (warp <= kFlushWarps) {
        // ----------------------------------------------------------- flush
        const int quarter = warp & 3;
        const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16);
        const int row = quarter * 32 + lane;  // M row owned by this thread
        int C = 0;
        for (int it = unit; it < a.n_items && !__any_sync(0xffffffffu, *abort_flag != 0); it += n_units) {
            const TcItem I = tc_item<MODE>(a, it, rank);
            const int ncols = 2 * I.nc;
            // FP32 slot: columns n..n+3 (n % 4 == 0) at [(n / 4) * 512 + row * 4];
            // FP64 slot: columns n, n + 1 (n even) at [(n / 2) * 256 + row * 2]
            float* slot32 = static_cast<float*>(I.slot) + row * 4;
            double* slot64 = static_cast<double*>(I.slot) + row * 2;
            for (int kk = 0; kk < I.n_chunks; ++kk) {
                const int k = C + kk;
                const int b = k % kBufs, u = k / kBufs;
                const uint32_t acc_col = lane_base + (uint32_t)(b * SH::kN);
                // warp-uniform outcome: the warp arrives as one below
                if (!__all_sync(0xffffffffu, mbar_wait(&acc_full[b], u & 1, abort_flag, a.error_flag, a.wait_limit_ns, 4))) break;
                tc_fence_after();
                if constexpr (SH::kDB) {
                    // the item's FP32 total is its slot: the first chain stores
                    // it, later ones add to it (the slot's loads are issued
                    // before the TMEM reads so their latency overlaps them);
                    // 16 columns per round trip
#pragma unroll 1
                    for (int cc = 0; cc < ncols; cc += 16) {
                        float4 sv[4];
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                            sv[i] = kk == 0 ? make_float4(0.f, 0.f, 0.f, 0.f)
                                            : __ldcg(reinterpret_cast<const float4*>(slot32 + (size_t)(cc + 4 * i) * kM));
                        float dv[16];
                        tmem_ld8(acc_col + cc, dv);
                        tmem_ld8(acc_col + cc + 8, dv + 8);
                        tmem_wait_ld();
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                            __stcg(reinterpret_cast<float4*>(slot32 + (size_t)(cc + 4 * i) * kM),
                                   make_float4(sv[i].x + dv[4 * i], sv[i].y + dv[4 * i + 1], sv[i].z + dv[4 * i + 2],
                                               sv[i].w + dv[4 * i + 3]));
                    }
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) {
                        if (rank == 0) mbar_arrive(&acc_empty[b]);
                        else mbar_arrive_leader(&acc_empty[b]);
                    }
                    continue;
                }
                tmem_wait_st();  // the previous flush's stores of the total
                // the chain partials are summed into an FP32 total in TMEM, over
                // at most kMaxItemChains chains; then (and at the item's end)
                // the total goes to the item's slot instead: stored (FP32
                // slots, items of at most kMaxItemChains chains) or added to
                // the FP64 totals (the first time stored)
                const bool restart = (kk % kMaxItemChains) == 0;
                const bool dump = (kk % kMaxItemChains) == kMaxItemChains - 1 || kk == I.n_chunks - 1;
                if (dump && I.slot_fp64) {
                    const bool first_dump = kk < kMaxItemChains;
                    // 8 columns per round trip; the slot's loads are issued
                    // before the TMEM reads so their latency overlaps them
#pragma unroll 1
                    for (int cc = 0; cc < ncols; cc += 8) {
                        double2 sv[4];
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                            sv[i] = first_dump ? make_double2(0.0, 0.0)
                                               : __ldcg(reinterpret_cast<const double2*>(slot64 + (size_t)(cc + 2 * i) * kM));
                        float dv[8], tv[8];
                        tmem_ld8(acc_col + cc, dv);
                        if (!restart) tmem_ld8(lane_base + kColTotal + cc, tv);
                        tmem_wait_ld();
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const float t0 = restart ? dv[2 * i] : tv[2 * i] + dv[2 * i];
                            const float t1 = restart ? dv[2 * i + 1] : tv[2 * i + 1] + dv[2 * i + 1];
                            __stcg(reinterpret_cast<double2*>(slot64 + (size_t)(cc + 2 * i) * kM),
                                   make_double2(sv[i].x + (double)t0, sv[i].y + (double)t1));
                        }
                    }
                } else {
                    // 32 columns per round trip.  ncols is a multiple of 16, so
                    // the last trip may carry 16 columns past ncols: they stay
                    // inside the accumulator and total regions and are never
                    // stored.
#pragma unroll 1
                    for (int cc = 0; cc < ncols; cc += 32) {
                        float tt[32];
                        if (restart) {
                            tmem_ld32(acc_col + cc, tt);
                            tmem_wait_ld();
                        } else {
                            float dv[32];
                            tmem_ld32(acc_col + cc, dv);
                            tmem_ld32(lane_base + kColTotal + cc, tt);
                            tmem_wait_ld();
#pragma unroll
                            for (int i = 0; i < 32; i += 2) {
                                const float2 t2 =
                                    __fadd2_rn(make_float2(tt[i], tt[i + 1]), make_float2(dv[i], dv[i + 1]));
                                tt[i] = t2.x;
                                tt[i + 1] = t2.y;
                            }
                        }
                        if (!dump) {
                            tmem_st32(lane_base + kColTotal + cc, tt);
                        } else {
                            // ncols is a multiple of 16: whole float4 groups are in or
                            // out; a warp's 32 rows write 512 contiguous bytes per group
#pragma unroll
                            for (int i = 0; i < 32; i += 4)
                                if (cc + i < ncols)
                                    *reinterpret_cast<float4*>(slot32 + (size_t)(cc + i) * kM) =
                                        make_float4(tt[i], tt[i + 1], tt[i + 2], tt[i + 3]);
                        }
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    // kPair: the accumulator release goes straight to CTA 0 (a
                    // forwarding hop would lengthen the MMA's wait); CTA 0's
                    // own warps arrive locally
                    if (rank == 0) mbar_arrive(&acc_empty[b]);
                    else mbar_arrive_leader(&acc_empty[b]);
                }
            }
            C += I.n_chunks;
        }
        tmem_wait_st();  // nothing in flight when TMEM is released (abort path)
    } else if (warp == kLoaderWarp) {
        // ---------------------------------------------------------- loader
        if (lane == 0) {
            int S = 0;
            for (int it = unit; it < a.n_items && !*abort_flag; it += n_units) {
                const TcItem I = tc_item<MODE>(a, it, rank);
                for (int s = 0; s < I.n_stages; ++s, ++S) {
                    const int buf = S % kSlots;
                    // this CTA's producers have read the slot's constants of stage S - kSlots
                    if (S >= kSlots && !mbar_wait(&sfree[buf], ((S / kSlots) - 1) & 1, abort_flag, a.error_flag, a.wait_limit_ns, 32))
                        break;
                    const int block = I.kb / kBlockParticles + s;
                    mbar_arrive_expect_tx(&pdata[buf], kBlockBytes);
                    bulk_copy_g2s(slots + buf * kSlotBytes, I.job->blocks + (size_t)block * kBlockBytes, kBlockBytes,
                                  &pdata[buf]);
                }
            }
        } else if (lane == 1) {
            // the loader's arrival on the barrier the MMA waits on (kPair, CTA 1:
            // the one its forwarder waits on), with the stage's B image where the
            // job has images.  Both wait until the MMA has read the stage
            // buffer's previous contents: the copy may then overwrite them, and
            // the arrival cannot count toward the barrier's previous phase.
            int S = 0;
            for (int it = unit; it < a.n_items && !*abort_flag; it += n_units) {
                const TcItem I = tc_item<MODE>(a, it, rank);
                int s = 0;
                for (; s < I.n_stages; ++s, ++S) {
                    const int bb = S % kBStages;
                    if (!mbar_wait(&b_empty[bb], ((S / kBStages) & 1) ^ 1, abort_flag, a.error_flag, a.wait_limit_ns, 512)) break;
                    uint64_t* fb = rank == 0 ? &full[S % kFull] : &pfull[S % kFull];
                    // test hook (vis_tensor_wait_test_hook): the first stage of
                    // the launch's first unit never completes, so the MMA's
                    // first wait runs out before any MMA is issued
                    if (a.withhold_first_arrival && S == 0 && unit == 0 && rank == 0) continue;
                    if (I.bimg) {
                        const int block = I.kb / kBlockParticles + s;
                        mbar_arrive_expect_tx(fb, (uint32_t)I.img_bytes);
                        bulk_copy_g2s(b_ring + bb * SH::kBStageBytes, I.bimg + (size_t)block * I.img_stride,
                                      (uint32_t)I.img_bytes, fb);
                    } else {
                        mbar_arrive(fb);
                    }
                }
                if (s < I.n_stages) break;
            }
        }
        __syncwarp();
    } else {
        // -------------------------------------------------------- producers
        const int p = tid - 32 * (1 + kFlushWarps);
        const int pp = p & 15;  // particle pair within the stage
        const bool has_a = p < 256;  // A unit: 8-row chunk rc; else B unit: c chunks cb, cb + 8
        const int rc = (p >> 4) & 15;
        const int cb = (p >> 4) & 7;
        int S = 0;
        for (int it = unit; it < a.n_items && !__any_sync(0xffffffffu, *abort_flag != 0); it += n_units) {
            const TcItem I = tc_item<MODE>(a, it, rank);
            const int ky = I.job->ky;
            const bool gauss = I.job->gauss != 0;
            const int rho0 = I.row0 + rc * 8;
            const int a_x = rho0 / ky + I.a_base;
            // the chunk's 8 rows have b = b0, b0 + fold, ..., b0 + 7 fold (the
            // constants' y rotation is the one of fold steps)
            const int b0 = (rho0 % ky) * I.fold + I.b_base;
            const bool a_up = b0 >= 0;
            const int b_s = a_up ? b0 : b0 + 7 * I.fold;
            for (int s = 0; s < I.n_stages; ++s, ++S) {
                const int buf = S % kSlots;
                if (!__all_sync(0xffffffffu, mbar_wait(&pdata[buf], (S / kSlots) & 1, abort_flag, a.error_flag, a.wait_limit_ns, 64)))
                    break;
                uint32_t pqx[2], pqy[2], pqz[2];
                float pamp[2], pgam[2], prho2[2];
                float2 pry[2], prz[2];
                {
                    // the pair's constants: particles 2pp, 2pp+1 of the stage's block
                    const uint8_t* blk = slots + buf * kSlotBytes;
                    const uint2 gq = *reinterpret_cast<const uint2*>(blk + kOffGam + 8 * pp);
                    const uint2 rq = *reinterpret_cast<const uint2*>(blk + kOffRho2 + 8 * pp);
                    pgam[0] = __uint_as_float(gq.x);
                    pgam[1] = __uint_as_float(gq.y);
                    prho2[0] = __uint_as_float(rq.x);
                    prho2[1] = __uint_as_float(rq.y);
                    if (has_a) {
                        const uint2 x = *reinterpret_cast<const uint2*>(blk + kOffQx + 8 * pp);
                        const uint2 y = *reinterpret_cast<const uint2*>(blk + kOffQy + 8 * pp);
                        const uint2 w = *reinterpret_cast<const uint2*>(blk + kOffAmp + 8 * pp);
                        const float4 r = *reinterpret_cast<const float4*>(blk + kOffRy + 16 * pp);
                        pqx[0] = x.x;
                        pqx[1] = x.y;
                        pqy[0] = y.x;
                        pqy[1] = y.y;
                        pamp[0] = __uint_as_float(w.x);
                        pamp[1] = __uint_as_float(w.y);
                        pry[0] = make_float2(r.x, r.y);
                        pry[1] = make_float2(r.z, r.w);
                        pqz[0] = pqz[1] = 0u;
                        prz[0] = prz[1] = make_float2(1.f, 0.f);
                    } else {
                        const uint2 zq = *reinterpret_cast<const uint2*>(blk + kOffQz + 8 * pp);
                        const uint2 yq = *reinterpret_cast<const uint2*>(blk + kOffQy + 8 * pp);
                        const float4 r = *reinterpret_cast<const float4*>(blk + kOffRz + 16 * pp);
                        pqz[0] = zq.x;
                        pqz[1] = zq.y;
                        prz[0] = make_float2(r.x, r.y);
                        prz[1] = make_float2(r.z, r.w);
                        pqy[0] = yq.x;  // row-folded jobs: the phase of a column block's b offset
                        pqy[1] = yq.y;
                        pqx[0] = pqx[1] = 0u;
                        pamp[0] = pamp[1] = 0.f;
                        pry[0] = pry[1] = make_float2(1.f, 0.f);
                    }
                }
                // the slot's constants are in registers: release it to the loader
                __syncwarp();
                if (lane == 0) mbar_arrive(&sfree[buf]);
                // the ring buffer this warp writes: A or B
                const bool waited = has_a ? mbar_wait(&a_empty[S % kAStages], ((S / kAStages) & 1) ^ 1, abort_flag,
                                                      a.error_flag, a.wait_limit_ns, 8)
                                          : mbar_wait(&b_empty[S % kBStages], ((S / kBStages) & 1) ^ 1, abort_flag,
                                                      a.error_flag, a.wait_limit_ns, 8);
                if (!__all_sync(0xffffffffu, waited)) break;
                uint8_t* st = has_a ? a_ring + (S % kAStages) * SH::kAStageBytes
                                    : b_ring + (S % kBStages) * SH::kBStageBytes;
                // the thread's two particles as packed pairs (see split_pair)
                float2 X, Y, RX, RY, Q = make_float2(1.f, 1.f), RHO = make_float2(1.f, 1.f);
                const int col = 8 * pp;  // byte offset of the pair within a 128-byte operand row
                if (has_a) {
                    // ---- A: rows rc*8 .. rc*8+7, particles 2pp, 2pp+1 (amp includes 2^12)
                    float v[2][5];
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        float sn, cs;
                        __sincosf(turns_to_radians((uint32_t)a_x * pqx[e] + (uint32_t)b_s * pqy[e]), &sn, &cs);
                        float g = pamp[e], q = 1.f;
                        if (gauss) {
                            g *= exp2f(pgam[e] * (float)(a_x * a_x + b_s * b_s));
                            q = exp2f(pgam[e] * (float)(2 * (a_up ? b_s : -b_s) + 1));
                        }
                        v[e][0] = g * cs;
                        v[e][1] = -g * sn;
                        v[e][2] = pry[e].x;
                        v[e][3] = a_up ? pry[e].y : -pry[e].y;
                        v[e][4] = q;
                    }
                    X = make_float2(v[0][0], v[1][0]);
                    Y = make_float2(v[0][1], v[1][1]);
                    RX = make_float2(v[0][2], v[1][2]);
                    RY = make_float2(v[0][3], v[1][3]);
                    const float2 NRY = make_float2(-RY.x, -RY.y);
                    uint8_t* base = st + rc * 8 * kRowBytes + (col & 15);
                    const int c16 = col & ~15;
                    if (gauss) {
                        Q = make_float2(v[0][4], v[1][4]);
                        RHO = make_float2(prho2[0], prho2[1]);
                        if (a_up) a_chain<true, true>(base, c16, X, Y, RX, RY, NRY, Q, RHO);
                        else a_chain<true, false>(base, c16, X, Y, RX, RY, NRY, Q, RHO);
                    } else {
                        if (a_up) a_chain<false, true>(base, c16, X, Y, RX, RY, NRY, Q, RHO);
                        else a_chain<false, false>(base, c16, X, Y, RX, RY, NRY, Q, RHO);
                    }
                } else {
                    // ---- B: c chunks cb (and cb + 8, kWide) of this CTA's bnc c values
                    // from bc0 (8 each), scaled by 2^12; rows [0, bnc) hold (Re B, -Im B)
                    // pairs (Re F columns), rows [bnc, 2 bnc) (Im B, Re B) (Im F columns).
                    // Chunks at or beyond bnc are not read by the MMA.
                    uint8_t* bhi = st;
                    RX = make_float2(prz[0].x, prz[1].x);
                    RY = make_float2(prz[0].y, prz[1].y);
                    const float2 NRY = make_float2(-RY.x, -RY.y);
                    if (gauss) RHO = make_float2(prho2[0], prho2[1]);
#pragma unroll 1
                    for (int h = 0; h < SH::kChunksPerThread; ++h) {
                        const int chunk = cb + 8 * h;
                        if (chunk * 8 >= I.bnc || I.bimg) break;  // the loader copies B images
                        b_unit(bhi, I.bnc, chunk, col, I.bc0 + chunk * 8, I.c_base, I.period, I.fold,
                               I.job->coef != nullptr, pqz, pqy, pgam, gauss, RX, RY,
                               NRY, RHO);
                    }
                }
                // each thread makes its stores visible to the tensor core; the
                // warp's lane 0 then arrives for the whole warp
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) {
                    // kPair: CTA 1's warps report to their forwarder (see the MMA role)
                    if (rank == 0) mbar_arrive(&full[S % kFull]);
                    else mbar_arrive(&pfull[S % kFull]);
                }
            }
        }
    }

    // ------------------------------------------------------------- teardown
    // a CTA that gave up a wait may still have bulk copies in flight into its
    // shared memory: give them time to land before anything is released
    if (tid == 0 && *abort_flag) {
        const unsigned long long t0 = global_ns();
        while (global_ns() - t0 < kAbortGraceNs) {
        }
    }
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
        if constexpr (kCtas == 1)
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                         : "memory");
        else
            asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                         : "memory");
    }
    // kPair: neither CTA exits while the other may still signal its barriers
    if constexpr (kCtas == 2) {
        __syncwarp();
        cluster_sync();
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
    int fold;          // the planes' job's row fold (1: none): its y rotation covers fold steps
    int exch;          // the planes' job is axis-exchanged: its blocks carry y and z exchanged
    uint8_t* out;      // ceil(n / 32) blocks
    uint8_t* out_nyq;  // the same with x and z exchanged (the Nyquist-plane job's), or null
};

__global__ void tc_prep_kernel(TcPrepArgs p) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int padded = (p.n + kBlockParticles - 1) / kBlockParticles * kBlockParticles;
    if (j >= padded) return;
    uint8_t* blk = p.out + (size_t)(j / kBlockParticles) * kBlockBytes;
    const int l = j % kBlockParticles;
    uint32_t qx = 0, qy = 0, qz = 0;
    float amp = 0.f, gam = 0.f;
    if (j < p.n) {
        const float4 q = p.particles[j];
        qx = fixed_turns(p.step * (double)q.x);
        qy = fixed_turns(p.step * (double)q.y);
        qz = fixed_turns(p.step * (double)q.z);
        amp = q.w * p.inv_wmax * kOperandScale;
        if (p.gauss) {
            const float h = p.radii[j];
            gam = p.gamma_scale * h * h;
        }
    }
    const uint32_t by = p.exch ? qz : qy, bz = p.exch ? qy : qz;  // the planes job's row and column axes
    reinterpret_cast<uint32_t*>(blk + kOffQx)[l] = qx;
    reinterpret_cast<uint32_t*>(blk + kOffQy)[l] = by;
    reinterpret_cast<uint32_t*>(blk + kOffQz)[l] = bz;
    reinterpret_cast<float*>(blk + kOffAmp)[l] = amp;
    reinterpret_cast<float*>(blk + kOffGam)[l] = gam;
    reinterpret_cast<float*>(blk + kOffRho2)[l] = exp2f(2.f * gam);
    const float2 ry = unit_phase(qy);
    reinterpret_cast<float2*>(blk + kOffRy)[l] = unit_phase((uint32_t)p.fold * by);
    reinterpret_cast<float2*>(blk + kOffRz)[l] = unit_phase(bz);
    if (p.out_nyq) {
        uint8_t* t = p.out_nyq + (size_t)(j / kBlockParticles) * kBlockBytes;
        reinterpret_cast<uint32_t*>(t + kOffQx)[l] = qz;
        reinterpret_cast<uint32_t*>(t + kOffQy)[l] = qy;
        reinterpret_cast<uint32_t*>(t + kOffQz)[l] = qx;
        reinterpret_cast<float*>(t + kOffAmp)[l] = amp;
        reinterpret_cast<float*>(t + kOffGam)[l] = gam;
        reinterpret_cast<float*>(t + kOffRho2)[l] = exp2f(2.f * gam);
        reinterpret_cast<float2*>(t + kOffRy)[l] = ry;
        reinterpret_cast<float2*>(t + kOffRz)[l] = unit_phase(qx);
    }
}

// h-bins of a group whose Phi^ does not separate per axis (SPH, Wendland with
// per-particle radii).  Within bin b (radii in [lo, hi]) Phi^(|k| h) is
// replaced by its Chebyshev interpolant in h on the bin's `order` Chebyshev
// nodes h_p:
//   Phi^(|k| h_j) ~= sum_q c_q(|k|) T_q(t_j),  t_j = (2 h_j - lo - hi) / (hi - lo),
//   c_q(|k|) = (2 / P) sum_p Phi^(|k| h_p) T_q(x_p)  (c_0 halved),
// so the bin's sum is, per q, a separable sum with B-side weights T_q(t_j)
// (one job per bin whose columns are the q blocks), and the reduction
// multiplies block q by c_q(|k|).  The reference's Phi^ switches from a
// quadratic fit to the closed form C at a branch point r0 with a jump in
// slope, which no polynomial in h follows; at frequency k that kink lies in
// the one bin holding r0 / |k|.  For that bin the coefficients are C's, and
// the plain form adds Phi^ - C (zero from r0 on) for the bin's particles at
// that k, over the particles sorted by bin (about 0.5% of the plain form's
// work on the SPH-like set).  The bins and orders are chosen on the host
// (hbin_plan) so the interpolation error stays near 1e-6 of the sum.

struct TcBinnedPrepArgs {
    const float4* particles;
    const float* radii;
    int n;
    double step;
    int nbins;
    const float* edges;    // nbins + 1 classification edges
    const int4* bins;      // (first block, capacity, coef offset, order)
    const float4* spans;   // (lo, hi, 2^12 / W_b, 0): Chebyshev interval and weight scale
    uint8_t* out;          // the group's blocks, bin by bin
    uint8_t* out_nyq;      // the same with x and z exchanged, or null
    const int* first;      // nbins + 1: the bins' first particles in sorted order
    float4* sorted;        // particles sorted by bin (for the branch part)
    float* sorted_radii;
    int* error_flag;
    int fold;              // the bins' planes jobs' row fold (1: none): their y rotation covers fold steps
    const int* order;      // the particles by ascending radius (bins are runs of it)
};

// Sort keys of a binned group: radii (non-negative, so their bits order as
// the values) and the particles' indices.
__global__ void tc_radius_keys_kernel(const float* radii, int n, uint32_t* keys, int* index) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    keys[j] = __float_as_uint(radii[j]);
    index[j] = j;
}

// Writes each particle's constants into its bin's blocks, in ascending radius
// (`order`, from a stable radix sort: the same order on every compute, and
// the branch part can stop at the first radius past r0 / |k|); gam holds t,
// the normalised radius.  The blocks were zeroed first, so padding particles
// have zero amplitude.
__global__ void tc_prep_binned_kernel(TcBinnedPrepArgs p) {
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;  // in the radius order
    if (pos >= p.n) return;
    const int j = p.order[pos];
    const float h = p.radii[j];
    const int b = hbin_of(p.edges, p.nbins, h);
    const int4 bin = p.bins[b];
    const int slot = pos - p.first[b];
    if (slot < 0 || slot >= bin.y) {  // the registered histogram does not hold for these radii
        atomicOr(p.error_flag, 2048);
        return;
    }
    const float4 sp = p.spans[b];
    const float t = sp.y > sp.x ? (2.f * h - sp.x - sp.y) / (sp.y - sp.x) : 0.f;
    const float4 q = p.particles[j];
    p.sorted[p.first[b] + slot] = q;
    p.sorted_radii[p.first[b] + slot] = h;
    const uint32_t qx = fixed_turns(p.step * (double)q.x);
    const uint32_t qy = fixed_turns(p.step * (double)q.y);
    const uint32_t qz = fixed_turns(p.step * (double)q.z);
    const float amp = q.w * sp.z;
    const size_t blk_off = (size_t)(bin.x + slot / kBlockParticles) * kBlockBytes;
    const int l = slot % kBlockParticles;
    const float2 ry = unit_phase(qy);
    const float2 ry_fold = p.fold > 1 ? unit_phase((uint32_t)p.fold * qy) : ry;
    for (int pass = 0; pass < (p.out_nyq ? 2 : 1); ++pass) {
        uint8_t* blk = (pass == 0 ? p.out : p.out_nyq) + blk_off;
        const uint32_t ax = pass == 0 ? qx : qz, az = pass == 0 ? qz : qx;
        reinterpret_cast<uint32_t*>(blk + kOffQx)[l] = ax;
        reinterpret_cast<uint32_t*>(blk + kOffQy)[l] = qy;
        reinterpret_cast<uint32_t*>(blk + kOffQz)[l] = az;
        reinterpret_cast<float*>(blk + kOffAmp)[l] = amp;
        reinterpret_cast<float*>(blk + kOffGam)[l] = t;
        reinterpret_cast<float*>(blk + kOffRho2)[l] = 1.f;
        reinterpret_cast<float2*>(blk + kOffRy)[l] = pass == 0 ? ry_fold : ry;
        reinterpret_cast<float2*>(blk + kOffRz)[l] = unit_phase(az);
    }
}

struct TcCoefArgs {
    int basis;
    double step;
    int nbins;
    int nsq;               // |k|^2 / step^2 = 0 .. nsq - 1
    int total_q;           // the group's Chebyshev blocks over all bins
    const int4* bins;      // (first block, capacity, first Chebyshev block, order)
    const float4* spans;   // (lo, hi, ...)
    const float* edges;    // the bins' classification edges
    float r0;              // the basis's branch point
    float* coef;
};

// Chebyshev coefficients c_q(|k|) of h -> Phi^(|k| h) on each bin, for every
// integer |k|^2 / step^2 of the lattice, in FP64, stored as floats:
// coef[n2 * total_q + q_offset(bin) + q] (one |k|^2's coefficients together,
// as the reduction reads them).  Phi^ is smooth on a bin unless the bin holds
// r0 / |k| (the reference's branch point, where its slope jumps): for that one
// bin the smooth closed form is interpolated instead (phi_smooth_fp64), and
// the plain form adds the rest for the bin's particles at that k
// (kAmpShell, mv_sum.cu).  Both sides find the bin from the same float |k|.
__global__ void tc_coef_kernel(TcCoefArgs c) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)c.nbins * c.nsq) return;
    const int b = (int)(i / c.nsq), n2 = (int)(i % c.nsq);
    const int4 bin = c.bins[b];
    const float4 sp = c.spans[b];
    const int order = bin.w;
    const double k = c.step * sqrt((double)n2);
    const float kf = (float)sqrt(c.step * c.step * (double)n2);
    const bool shell = hbin_of(c.edges, c.nbins, kf > 0.f ? c.r0 / kf : INFINITY) == b;
    const double mid = 0.5 * ((double)sp.x + (double)sp.y), half = 0.5 * ((double)sp.y - (double)sp.x);
    constexpr int kMaxOrder = 16;
    double f[kMaxOrder], x[kMaxOrder];
    for (int p = 0; p < order && p < kMaxOrder; ++p) {
        x[p] = cospi((2.0 * p + 1.0) / (2.0 * order));
        const double r = k * (mid + half * x[p]);
        f[p] = shell ? phi_smooth_fp64(c.basis, r) : phi_fp64(c.basis, r);
    }
    for (int q = 0; q < order && q < kMaxOrder; ++q) {
        double acc = 0.0;
        for (int p = 0; p < order; ++p) acc += f[p] * cospi(q * (2.0 * p + 1.0) / (2.0 * order));
        acc *= 2.0 / order;
        if (q == 0) acc *= 0.5;
        c.coef[(size_t)n2 * c.total_q + bin.z + q] = (float)acc;
    }
}

// B-operand images of one job (layout in TcJob): one CTA per image (n-tile,
// CTA half, 32-particle block); thread (chunk, pair) runs b_unit for 8 c
// values of 2 particles, exactly as a producer warp would into the stage
// buffer.  Each image is written once and copied by the tensor kernel's loader
// for every m-tile of the job.
// All jobs' images in one launch: CTA i makes image i of the concatenation,
// [job with images][n_tile][CTA half][block], the job found by binary search
// over the image offsets (img_first[k]: first image of the k-th such job).
struct TcImageArgs {
    const TcJob* jobs;
    const int* img_jobs;          // the jobs that have images
    const long long* img_first;   // n_img_jobs + 1 offsets
    int n_img_jobs;
};

__global__ void __launch_bounds__(256) tc_bimg_kernel(TcImageArgs g) {
    const long long i = blockIdx.x;
    int lo = 0, hi = g.n_img_jobs;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (g.img_first[mid] <= i) lo = mid;
        else hi = mid;
    }
    const TcJob& J = g.jobs[g.img_jobs[lo]];
    const long long img = i - g.img_first[lo];  // (n_tile * ctas + half) * n_blocks + block
    const int block = (int)(img % J.n_blocks);
    const int nh = (int)(img / J.n_blocks);
    const int half = nh % J.ctas, n_tile = nh / J.ctas;
    const int c0 = n_tile * J.nc_tile;
    const int bnc = min(J.nc_tile, J.lz_tc - c0) / J.ctas;
    const int pp = threadIdx.x & 15, chunk = threadIdx.x >> 4;
    if (chunk * 8 >= bnc) return;
    const unsigned char* blk = J.blocks + (size_t)block * kBlockBytes;
    const uint2 zq = *reinterpret_cast<const uint2*>(blk + kOffQz + 8 * pp);
    const uint2 yq = *reinterpret_cast<const uint2*>(blk + kOffQy + 8 * pp);
    const uint2 gq = *reinterpret_cast<const uint2*>(blk + kOffGam + 8 * pp);
    const uint2 rq = *reinterpret_cast<const uint2*>(blk + kOffRho2 + 8 * pp);
    const float4 r = *reinterpret_cast<const float4*>(blk + kOffRz + 16 * pp);
    const uint32_t pqz[2] = {zq.x, zq.y}, pqy[2] = {yq.x, yq.y};
    const float pgam[2] = {__uint_as_float(gq.x), __uint_as_float(gq.y)};
    const float2 RX = make_float2(r.x, r.z), RY = make_float2(r.y, r.w);
    const float2 NRY = make_float2(-RY.x, -RY.y);
    const bool gauss = J.gauss != 0;
    const float2 RHO = gauss ? make_float2(__uint_as_float(rq.x), __uint_as_float(rq.y)) : make_float2(1.f, 1.f);
    uint8_t* out = const_cast<uint8_t*>(J.bimg) + (size_t)img * J.img_stride;
    b_unit(out, bnc, chunk, 8 * pp, c0 + half * bnc + chunk * 8, J.c_base, J.period, max(1, J.fold), J.coef != nullptr,
           pqz, pqy, pgam, gauss, RX, RY, NRY, RHO);
}

// What the reduction needs of a job, gathered into shared memory once per
// block (the job table's other fields are not read).
struct ReduceJob {
    const void* slots;
    int slot_fp64;
    const int4* colmap;
    const float* coef;  // null unless h-binned
    double scale;       // W x 2^-24
    int slot_stride, n_splits, n_mtiles, n_ntiles;
    int rank_stride;    // floats between the CTAs' parts of a slot: 128 * 2 nc_tile
    int mrows_log2;     // 7 (one CTA) or 8 (CTA pair)
    int period, blocks, coef_stride;
    int fold, ky_full;  // row-folded jobs: the fold and the spectrum's Ky (else 1, 0)
    int exch, rows_a;   // axis-exchanged jobs: 1 and the job rows per a (the planes)
};

__device__ __forceinline__ ReduceJob reduce_job(const TcJob& J) {
    ReduceJob r;
    r.slots = J.slots;
    r.slot_fp64 = J.slot_fp64;
    r.colmap = J.colmap;
    r.coef = J.period > 0 ? J.coef : nullptr;
    r.scale = J.wmax * kInvProductScale;
    r.slot_stride = J.slot_stride;
    r.n_splits = J.n_splits;
    r.n_mtiles = J.n_mtiles;
    r.n_ntiles = J.n_ntiles;
    r.rank_stride = kM * 2 * J.nc_tile;
    r.mrows_log2 = J.ctas == 2 ? 8 : 7;
    r.period = J.period;
    r.blocks = J.period > 0 ? J.lz_tc / J.period / (J.fold > 1 ? J.fold : 1) : 1;
    r.coef_stride = J.coef_stride;
    r.fold = J.fold > 1 ? J.fold : 1;
    r.ky_full = J.exch ? J.lz_tc : J.ky * r.fold;
    r.exch = J.exch;
    r.rows_a = J.ky;
    return r;
}

// Adds one job's contribution at lattice row rho (the spectrum's a_idx Ky +
// b_idx; within the job's rows for unfolded jobs) and the kC consecutive
// frequency columns c0 .. c0 + kC - 1 (c_idx, before the Chebyshev blocks of
// an h-binned job; they share one n-tile and one CTA half, as n-tiles and
// halves hold multiples of 8 columns): the totals of all its particle chunks
// (FP32 or FP64 slots) summed in FP64, each h-binned block weighted by its
// coefficient at |k|^2 = n2[i] step^2, times W 2^-24.  A row-folded job holds
// b_idx = fold bh + bl at job row a_idx (Ky / fold) + bh, in column blocks
// q fold + bl.
constexpr int kReduceC = 4;
__device__ __forceinline__ void reduce_add(const ReduceJob& J, int rho, int c0, const int* n2, int nc, double* sr,
                                           double* si, double sign_im) {
    if (J.exch) {
        // axis-exchanged: plane c0 + i of spectrum row (a_idx, b_idx) is job
        // row a_idx (planes) + c0 + i, job column b_idx; the kC rows share a
        // 128-row CTA half (c0 is a multiple of kC)
        const int a_idx = rho / J.ky_full, b_idx = rho - a_idx * J.ky_full;
        const int4 m = __ldg(J.colmap + b_idx);
        for (int i = 0; i < nc; ++i) {
            const int jr = a_idx * J.rows_a + c0 + i;
            const int m_tile = jr >> J.mrows_log2, within = jr - (m_tile << J.mrows_log2);
            const int rank = within >> 7, rl = within & (kM - 1);
            double tr = 0.0, ti = 0.0;
            for (int ks = 0; ks < J.n_splits; ++ks) {
                const size_t li = ((size_t)ks * J.n_mtiles + m_tile) * J.n_ntiles + m.x;
                const size_t base = li * J.slot_stride + (size_t)rank * J.rank_stride;
                if (J.slot_fp64) {
                    const double* v = static_cast<const double*>(J.slots) + base + rl * 2;
                    tr += __ldg(v + (size_t)(m.y & ~1) * kM + (m.y & 1));
                    ti += __ldg(v + (size_t)(m.z & ~1) * kM + (m.z & 1));
                } else {
                    const float* v = static_cast<const float*>(J.slots) + base + rl * 4;
                    tr += (double)__ldg(v + (size_t)(m.y & ~3) * kM + (m.y & 3));
                    ti += (double)__ldg(v + (size_t)(m.z & ~3) * kM + (m.z & 3));
                }
            }
            sr[i] = fma(J.scale, tr, sr[i]);
            si[i] = fma(J.scale * sign_im, ti, si[i]);
        }
        return;
    }
    int bl = 0;
    if (J.fold > 1) {
        const int a_idx = rho / J.ky_full, b_idx = rho - a_idx * J.ky_full;
        rho = a_idx * (J.ky_full / J.fold) + b_idx / J.fold;
        bl = b_idx % J.fold;
    }
    const int m_tile = rho >> J.mrows_log2, within = rho - (m_tile << J.mrows_log2);
    const int rank = within >> 7, rl = within & (kM - 1);
    // FP32 slot layout [column / 4][128 rows][column % 4]: column n of row rl
    // at (n / 4) * 512 + rl * 4 + n % 4; FP64: [column / 2][128 rows][column %
    // 2], column n at (n / 2) * 256 + rl * 2 + n % 2
    const size_t rbase = (size_t)rank * J.rank_stride;
    const float* row = static_cast<const float*>(J.slots) + rbase + rl * 4;
    const double* row64 = static_cast<const double*>(J.slots) + rbase + rl * 2;
    if (!J.slot_fp64 && nc == kReduceC && J.n_splits == 1) {
        // the common h-bin case (one particle chunk, FP32 slots): two column
        // blocks per round, so each thread has twice the loads in flight
        const size_t lbase = (size_t)m_tile * J.n_ntiles;
        for (int q = 0; q < J.blocks; q += 2) {
            const bool two = q + 1 < J.blocks;
            const int4 m0 = __ldg(J.colmap + (q * J.fold + bl) * J.period + c0);
            const int4 m1 = two ? __ldg(J.colmap + ((q + 1) * J.fold + bl) * J.period + c0) : m0;
            const float* v0 = row + (lbase + m0.x) * J.slot_stride;
            const float* v1 = row + (lbase + m1.x) * J.slot_stride;
            const float4 re0 = __ldg(reinterpret_cast<const float4*>(v0 + (size_t)m0.y * kM));
            const float4 im0 = __ldg(reinterpret_cast<const float4*>(v0 + (size_t)m0.z * kM));
            const float4 re1 = two ? __ldg(reinterpret_cast<const float4*>(v1 + (size_t)m1.y * kM)) : make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 im1 = two ? __ldg(reinterpret_cast<const float4*>(v1 + (size_t)m1.z * kM)) : make_float4(0.f, 0.f, 0.f, 0.f);
            double w0[kReduceC], w1[kReduceC];
#pragma unroll
            for (int i = 0; i < kReduceC; ++i) {
                w0[i] = J.coef ? (double)__ldg(J.coef + (size_t)n2[i] * J.coef_stride + q) * J.scale : J.scale;
                w1[i] = J.coef && two ? (double)__ldg(J.coef + (size_t)n2[i] * J.coef_stride + q + 1) * J.scale
                                      : (two ? J.scale : 0.0);
            }
            const float r0[kReduceC] = {re0.x, re0.y, re0.z, re0.w}, i0[kReduceC] = {im0.x, im0.y, im0.z, im0.w};
            const float r1[kReduceC] = {re1.x, re1.y, re1.z, re1.w}, i1[kReduceC] = {im1.x, im1.y, im1.z, im1.w};
#pragma unroll
            for (int i = 0; i < kReduceC; ++i) {
                sr[i] = fma(w1[i], (double)r1[i], fma(w0[i], (double)r0[i], sr[i]));
                si[i] = fma(w1[i] * sign_im, (double)i1[i], fma(w0[i] * sign_im, (double)i0[i], si[i]));
            }
        }
        return;
    }
    for (int q = 0; q < J.blocks; ++q) {
        // column block q F + bl: Chebyshev block q (h-binned), b offset bl (folded)
        const int4 m = __ldg(J.colmap + (q * J.fold + bl) * J.period + c0);  // the same for a warp's rows
        double tr[kReduceC] = {}, ti[kReduceC] = {};
        for (int ks = 0; ks < J.n_splits; ++ks) {
            const size_t li = ((size_t)ks * J.n_mtiles + m_tile) * J.n_ntiles + m.x;
            if (J.slot_fp64) {
                const double* v = row64 + li * J.slot_stride;
                if (nc == kReduceC) {
                    // two columns per load (m.y, m.z are multiples of 4)
                    const double2 r0 = __ldg(reinterpret_cast<const double2*>(v + (size_t)m.y * kM));
                    const double2 r1 = __ldg(reinterpret_cast<const double2*>(v + (size_t)(m.y + 2) * kM));
                    const double2 i0 = __ldg(reinterpret_cast<const double2*>(v + (size_t)m.z * kM));
                    const double2 i1 = __ldg(reinterpret_cast<const double2*>(v + (size_t)(m.z + 2) * kM));
                    tr[0] += r0.x; tr[1] += r0.y; tr[2] += r1.x; tr[3] += r1.y;
                    ti[0] += i0.x; ti[1] += i0.y; ti[2] += i1.x; ti[3] += i1.y;
                } else {
                    tr[0] += __ldg(v + (size_t)(m.y & ~1) * kM + (m.y & 1));
                    ti[0] += __ldg(v + (size_t)(m.z & ~1) * kM + (m.z & 1));
                }
                continue;
            }
            const float* v = row + li * J.slot_stride;
            if (nc == kReduceC) {
                // four columns in one load (m.y, m.z are multiples of 4); a warp's
                // rows read 512 contiguous bytes
                const float4 re = __ldg(reinterpret_cast<const float4*>(v + (size_t)m.y * kM));
                const float4 im = __ldg(reinterpret_cast<const float4*>(v + (size_t)m.z * kM));
                tr[0] += re.x; tr[1] += re.y; tr[2] += re.z; tr[3] += re.w;
                ti[0] += im.x; ti[1] += im.y; ti[2] += im.z; ti[3] += im.w;
            } else {
                tr[0] += (double)__ldg(v + (size_t)(m.y & ~3) * kM + (m.y & 3));
                ti[0] += (double)__ldg(v + (size_t)(m.z & ~3) * kM + (m.z & 3));
            }
        }
#pragma unroll
        for (int i = 0; i < kReduceC; ++i) {
            if (i < nc) {
                const double w = J.coef ? (double)__ldg(J.coef + (size_t)n2[i] * J.coef_stride + q) * J.scale : J.scale;
                sr[i] = fma(w, tr[i], sr[i]);
                si[i] = fma(w * sign_im, ti[i], si[i]);
            }
        }
    }
}

// The jobs of one output class (same spectrum, same per-frequency factor)
// -> its float2 spectrum, added: planes c in [0, lz_tc) (tc_reduce_planes_kernel),
// or the Nyquist plane c = lz_tc from the transposed jobs (tc_reduce_kernel):
// for a >= 0 the a >= 0 jobs at row b_idx and column a; for a < 0 the
// conjugate of the a < 0 jobs at row Ky - 1 - b_idx (frequency -b) and column
// -a - 1 (frequency -a).  Times the factored Phi^(|k| h) in FP64 and the
// scale.  The kernels gather the class's job descriptors in shared memory
// first.
struct TcReduceArgs {
    const TcJob* jobs;
    const int* list;      // planes: the class's jobs; nyquist: its a >= 0 jobs
    int n_list;
    const int* list_neg;  // nyquist: its a < 0 jobs
    int n_neg;
    int kx, ky, lz_tc, lz_out;
    double step;
    int basis;
    double h;  // radius of the factored Phi^(|k| h); 1 without radii
    bool factored;
    double scale;
    float2* out;
    int warp_rows;  // planes: every warp sums all jobs of its own 32 rows (classes of fewer jobs than warps)
};

// Warps per block of the reduction kernels (each sums every eighth job).
constexpr int kReduceWarps = 8;

// The Nyquist plane of one output class, with the job list split over warps
// as in tc_reduce_planes_kernel: a block takes 32 elements (lanes), warp w
// sums the jobs w, w + 8, ... of the element's sign of a, and the eight
// partial sums are added in warp order (a fixed order).
__global__ void __launch_bounds__(32 * kReduceWarps) tc_reduce_kernel(TcReduceArgs f) {
    extern __shared__ __align__(16) unsigned char s_raw[];  // descriptors, then the partial sums
    ReduceJob* s_jobs = reinterpret_cast<ReduceJob*>(s_raw);
    const int n_all = f.n_list + f.n_neg;
    for (int i = threadIdx.x; i < n_all; i += blockDim.x)
        s_jobs[i] = reduce_job(f.jobs[i < f.n_list ? f.list[i] : f.list_neg[i - f.n_list]]);
    double2* s_part = reinterpret_cast<double2*>(s_raw + (((size_t)n_all * sizeof(ReduceJob) + 15) & ~(size_t)15));
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long rows = (long long)f.kx * f.ky;
    const long long e = (long long)blockIdx.x * 32 + lane;
    const bool active = e < rows;
    const int rho = active ? (int)e : 0;
    const int a_idx = rho / f.ky, b_idx = rho % f.ky;
    const int a = a_idx - f.kx / 2, b = b_idx - f.ky / 2;
    const int c = f.lz_tc;
    int n2[kReduceC];
#pragma unroll
    for (int i = 0; i < kReduceC; ++i) n2[i] = a * a + b * b + (c + i) * (c + i);
    double sr[kReduceC] = {}, si[kReduceC] = {};
    if (active) {
        // for a >= 0 the a >= 0 jobs at row b_idx and column a; for a < 0 the
        // conjugate of the a < 0 jobs at row Ky - 1 - b_idx (frequency -b) and
        // column -a - 1 (frequency -a)
        if (a >= 0) {
            for (int j = warp; j < f.n_list; j += kReduceWarps) reduce_add(s_jobs[j], b_idx, a, n2, 1, sr, si, 1.0);
        } else {
            for (int j = warp; j < f.n_neg; j += kReduceWarps)
                reduce_add(s_jobs[f.n_list + j], f.ky - 1 - b_idx, -a - 1, n2, 1, sr, si, -1.0);
        }
    }
    s_part[warp * 32 + lane] = make_double2(sr[0], si[0]);
    __syncthreads();
    if (warp != 0 || !active) return;
    double tr = 0.0, ti = 0.0;
    for (int w = 0; w < kReduceWarps; ++w) {
        const double2 v = s_part[w * 32 + lane];
        tr += v.x;
        ti += v.y;
    }
    double factor = f.scale;
    if (f.factored) factor *= phi_fp64(f.basis, f.step * sqrt((double)n2[0]) * f.h);
    const size_t idx = (size_t)rho * f.lz_out + c;
    const float2 o = f.out[idx];
    f.out[idx] = make_float2(o.x + (float)(tr * factor), o.y + (float)(ti * factor));
}

// The planes c < lz_tc of one output class.  With the job list split over
// warps (classes of at least 8 jobs): a block takes 32 rows (lanes) x
// kReduceC planes, warp w sums jobs w, w + 8, ..., and the eight partial sums
// are added in warp order (a fixed order: the result does not depend on
// timing), so eight independent load chains per element hide the slots'
// latency.  With fewer jobs (f.warp_rows; one group per class, as in a batch
// of particle sets) a block takes 8 x 32 rows and each warp sums every job of
// its own 32 rows in job order, so no warp idles.
__global__ void __launch_bounds__(32 * kReduceWarps, 2) tc_reduce_planes_kernel(TcReduceArgs f) {
    extern __shared__ __align__(16) unsigned char s_raw[];  // n_list descriptors, then the partial sums
    ReduceJob* s_jobs = reinterpret_cast<ReduceJob*>(s_raw);
    for (int i = threadIdx.x; i < f.n_list; i += blockDim.x) s_jobs[i] = reduce_job(f.jobs[f.list[i]]);
    // [warp][lane][kReduceC], 16-byte aligned after the descriptors
    double2* s_part = reinterpret_cast<double2*>(s_raw + (((size_t)f.n_list * sizeof(ReduceJob) + 15) & ~(size_t)15));
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long rows = (long long)f.kx * f.ky;
    const int block_rows = f.warp_rows ? 32 * kReduceWarps : 32;
    const long long row_blocks = (rows + block_rows - 1) / block_rows;
    const int rho = (int)((blockIdx.x % row_blocks) * block_rows + (f.warp_rows ? warp * 32 : 0) + lane);
    const int c0 = (int)(blockIdx.x / row_blocks) * kReduceC;
    const bool active = rho < rows;
    const int rr = active ? rho : 0;
    const int a = rr / f.ky - f.kx / 2, b = rr % f.ky - f.ky / 2;
    int n2[kReduceC];
#pragma unroll
    for (int i = 0; i < kReduceC; ++i) n2[i] = a * a + b * b + (c0 + i) * (c0 + i);
    double sr[kReduceC] = {}, si[kReduceC] = {};
    // spectrum element (rho, c0 + i) += its FP64 sum, with the factored Phi^
    auto store = [&](int i, double tr, double ti) {
        double factor = f.scale;
        if (f.factored) factor *= phi_fp64(f.basis, f.step * sqrt((double)n2[i]) * f.h);
        const size_t idx = (size_t)rho * f.lz_out + c0 + i;
        const float2 o = f.out[idx];
        f.out[idx] = make_float2(o.x + (float)(tr * factor), o.y + (float)(ti * factor));
    };
    if (f.warp_rows) {  // uniform over the block: no barrier follows
        if (!active) return;
        for (int j = 0; j < f.n_list; ++j) reduce_add(s_jobs[j], rho, c0, n2, kReduceC, sr, si, 1.0);
#pragma unroll
        for (int i = 0; i < kReduceC; ++i) store(i, sr[i], si[i]);
        return;
    }
    if (active)
        for (int j = warp; j < f.n_list; j += kReduceWarps) reduce_add(s_jobs[j], rho, c0, n2, kReduceC, sr, si, 1.0);
#pragma unroll
    for (int i = 0; i < kReduceC; ++i) s_part[(warp * 32 + lane) * kReduceC + i] = make_double2(sr[i], si[i]);
    __syncthreads();
    if (warp != 0 || !active) return;
#pragma unroll
    for (int i = 0; i < kReduceC; ++i) {
        double tr = 0.0, ti = 0.0;
        for (int w = 0; w < kReduceWarps; ++w) {
            const double2 v = s_part[(w * 32 + lane) * kReduceC + i];
            tr += v.x;
            ti += v.y;
        }
        store(i, tr, ti);
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

// kPairDB tiles: MV_TC_DB=0 or a tuned set without kTileDoubleBuffer turns
// them off (those jobs then take kPair).
bool tc_db_enabled() {
    static const bool v = [] {
        const char* e = std::getenv("MV_TC_DB");
        return !(e && e[0] == '0');
    }();
    return v && (active_tune().tc_shapes & kTileDoubleBuffer);
}

// Row folds of pure-phase and h-binned groups: MV_TC_FOLD=0 or a tuned set
// without kTileRowFold turns them off.
bool tc_fold_enabled() {
    static const bool v = [] {
        const char* e = std::getenv("MV_TC_FOLD");
        return !(e && e[0] == '0');
    }();
    return v && (active_tune().tc_shapes & kTileRowFold);
}

// Axis exchange of non-folding groups: MV_TC_EXCHANGE=0 or a tuned set
// without kTileAxisExchange turns it off.
bool tc_exchange_enabled() {
    static const bool v = [] {
        const char* e = std::getenv("MV_TC_EXCHANGE");
        return !(e && e[0] == '0');
    }();
    return v && (active_tune().tc_shapes & kTileAxisExchange);
}

// kPair tiles: MV_TC_PAIRS=0 or a tuned set without kTileCtaPairs turns them
// off (jobs then take kWide tiles).
bool tc_pairs_enabled() {
    static const bool v = [] {
        const char* e = std::getenv("MV_TC_PAIRS");
        return !(e && e[0] == '0');
    }();
    return v && (active_tune().tc_shapes & kTileCtaPairs);
}

// Stages per TMEM accumulation chain before a flush into the FP32 total.
// The single-accumulator tiles (kWide, kPair) stall the MMA for every flush
// and take the tuned value (default 16: 4.1e-6 rel-L2 on C3 against 2.6e-6 at
// 8, for 11% more speed); the double-buffered kNarrow tile hides its flushes
// and keeps chains of at most 8.  MV_TC_FLUSH_STAGES (1..1024) overrides both.
int tc_flush_stages(int mode) {
    static const int env = [] {
        const char* e = std::getenv("MV_TC_FLUSH_STAGES");
        const int x = e ? std::atoi(e) : 0;
        return (x >= 1 && x <= 1024) ? x : 0;
    }();
    if (env) return env;
    return narrow_mode(mode) ? std::min(8, active_tune().tc_flush) : active_tune().tc_flush;
}

// B-operand images are made for jobs whose every image is copied by at
// least this many m-tiles.
constexpr int kImageMinReuse = 4;

long long g_operand_cache_limit = -1;  // bytes; -1: the default policy
// Set by vis_tensor_wait_test_hook; taken by the next tensor launch (one shot).
std::atomic<long long> g_test_wait_limit_ns{0};

}  // namespace

size_t operand_cache_limit() {
    const long long set = __atomic_load_n(&g_operand_cache_limit, __ATOMIC_RELAXED);
    if (set >= 0) return (size_t)set;
    static const long long env = [] {
        // unset or negative: the default below (as vis_set_operand_cache_limit(-1))
        const char* e = std::getenv("MV_TC_OPERAND_CACHE_MB");
        const long long mb = e ? std::atoll(e) : -1LL;
        return mb >= 0 ? std::min(mb, 1LL << 40) << 20 : -1LL;
    }();
    if (env >= 0) return (size_t)env;
    // three eighths of the device's memory (the 51 GB of images of 2^24
    // particles on 384^3 fit a 180 GB device; they are 2.5% faster there than
    // B computed per tile), queried once per device (threads that race here
    // store the same value)
    static size_t total[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    size_t t = __atomic_load_n(&total[dev], __ATOMIC_RELAXED);
    if (!t) {
        size_t free_b = 0;
        if (cudaMemGetInfo(&free_b, &t) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        __atomic_store_n(&total[dev], t, __ATOMIC_RELAXED);
    }
    return t / 8 * 3;
}

extern "C" int vis_tensor_wait_test_hook(long long wait_limit_ns) {
    if (wait_limit_ns < 100000LL || wait_limit_ns > (long long)kWaitLimitNs)
        return set_error(kInvalidValue, "vis_tensor_wait_test_hook: limit outside [1e5, 2e9] ns");
    g_test_wait_limit_ns.store(wait_limit_ns);
    return kOk;
}

extern "C" void vis_set_operand_cache_limit(long long bytes) {
    __atomic_store_n(&g_operand_cache_limit, bytes < 0 ? -1LL : bytes, __ATOMIC_RELAXED);
}

namespace {

// ---------------------------------------------------------------- h-bins
// Chebyshev order of a bin whose radii span dh at the lattice's largest |k|:
// the smallest P with 2 (pi x / 2)^P / P! <= kHBinTau, x = |k|max dh.  That is
// the interpolation error bound for h -> Phi^(|k| h), whose P-th derivative is
// at most (2 pi |k|)^P Phi^(0) (the basis functions have support radius h);
// bins needing more than kHBinMaxOrder nodes are not formed.
constexpr double kHBinTau = 3e-5;
constexpr int kHBinMaxOrder = 12;
// The bins interpolate the closed form C only (the branch's part is summed
// apart, see tc_coef_kernel), which is smooth: CPU models of the scheme
// against the oracle's FP64 Phi^ give 4e-8 rel-L2 on C2's set and up to 7e-7
// on uniform sets with h in [0.01, 0.05].

double hbin_order_limit(int order) {  // largest x that `order` nodes cover
    double f = 1.0;
    for (int i = 2; i <= order; ++i) f *= i;
    return (2.0 / kPi) * std::pow(kHBinTau * f / 2.0, 1.0 / order);
}

int hbin_order(double x) {
    static const std::vector<double> limit = [] {
        std::vector<double> v(kHBinMaxOrder + 1, 0.0);
        for (int p = 1; p <= kHBinMaxOrder; ++p) v[p] = hbin_order_limit(p);
        return v;
    }();
    for (int p = 1; p <= kHBinMaxOrder; ++p)
        if (x <= limit[p]) return p;
    return kHBinMaxOrder + 1;
}

// The largest |k| of a half-spectrum lattice and the largest a^2 + b^2 + c^2.
long long lattice_nsq(const Lattice& L) {
    const long long hx = L.nx / 2, hy = L.ny / 2, hz = L.nz - 1;
    return hx * hx + hy * hy + hz * hz;
}

// Work per particle of a bin of Chebyshev order P whose blocks are `period`
// columns wide, in jobs folded by `fold` rows: the MMAs cost about the same
// per n-tile (at most 128 c values) whatever its width, and a fold puts
// `fold` rows' columns into one job row (1 / fold of the m-tiles); the A and
// B operands' work scales with the columns; in units of one full n-tile.
double hbin_unit_cost(int order, int period, int fold) {
    const double tiles = (double)order * period / Shape<kWide>::kNc;
    return std::ceil(tiles * fold) / fold + tiles;
}

// Row fold of an h-binned group's plane jobs (TcJob::fold): the smallest F of
// {1, 2, 4} whose F planes fill whole n-tiles for every Chebyshev order, if
// Ky / F stays a multiple of 16; else 1.
int hbin_fold(const Lattice& L) {
    const int period = L.nz - 1;
    for (int f : {1, 2, 4})
        if ((f * period) % Shape<kWide>::kNc == 0 && L.ny % (16 * f) == 0) return f > 1 && !tc_fold_enabled() ? 1 : f;
    return 1;
}

// Bins of a group on a lattice: runs of fine bins chosen by dynamic
// programming to minimise, per non-empty bin, count x hbin_unit_cost (the
// tensor work) + order x block_cost (the reduction reads every Chebyshev
// block at every frequency) + job_cost (items, pipeline fills), each bin's
// Chebyshev interval the span of its non-empty fine bins.
HBinPlan hbin_plan_build(const HBinStats& hs, double kmax, int period, int fold, int job_cost, int block_cost) {
    const int F = kHBinFine;
    std::vector<long long> cum(F + 1, 0);
    for (int f = 0; f < F; ++f) cum[f + 1] = cum[f] + hs.count[f];
    std::vector<int> first_ne(F + 1, F), last_ne(F + 1, -1);  // first non-empty >= i, last non-empty < j
    for (int f = F - 1; f >= 0; --f) first_ne[f] = hs.count[f] ? f : first_ne[f + 1];
    for (int f = 0; f < F; ++f) last_ne[f + 1] = hs.count[f] ? f : last_ne[f];
    std::vector<double> best(F + 1, 1e300);
    std::vector<int> arg(F + 1, 0);
    best[0] = 0.0;
    for (int j = 1; j <= F; ++j) {
        for (int i = j - 1; i >= 0; --i) {
            const long long n = cum[j] - cum[i];
            int order = 1;
            if (n > 0) {
                const double lo = hs.edges[first_ne[i]], hi = hs.edges[last_ne[j] + 1];
                order = hbin_order(kmax * (hi - lo));
                if (order > kHBinMaxOrder) break;  // wider runs (smaller i) only need more
            }
            const double c =
                best[i] + (n > 0 ? (double)n * hbin_unit_cost(order, period, fold) + (double)order * block_cost + job_cost : 0.0);
            if (c < best[j]) {
                best[j] = c;
                arg[j] = i;
            }
        }
    }
    HBinPlan plan;
    if (!(best[F] < 1e299)) {  // a single fine bin already needs too many nodes
        plan.feasible = false;
        return plan;
    }
    std::vector<int> cuts;
    for (int j = F; j > 0; j = arg[j]) cuts.push_back(j);
    cuts.push_back(0);
    std::reverse(cuts.begin(), cuts.end());
    long long total = 0, weighted = 0;
    for (size_t k = 0; k + 1 < cuts.size(); ++k) {
        HBin b;
        b.f0 = cuts[k];
        b.f1 = cuts[k + 1];
        b.count = (int)(cum[b.f1] - cum[b.f0]);
        b.wmax = 0.f;
        for (int f = b.f0; f < b.f1; ++f) b.wmax = std::max(b.wmax, hs.wmax[f]);
        if (b.count > 0) {
            b.lo = hs.edges[first_ne[b.f0]];
            b.hi = hs.edges[last_ne[b.f1] + 1];
            b.order = hbin_order(kmax * ((double)b.hi - (double)b.lo));
        } else {
            b.lo = hs.edges[b.f0];
            b.hi = hs.edges[b.f1];
            b.order = 1;
        }
        total += b.count;
        weighted += (long long)b.count * b.order;
        plan.bins.push_back(b);
    }
    plan.cost = total > 0 ? (double)weighted / (double)total : 0.0;
    return plan;
}

// Plans are cached per registration, lattice and job cost.
std::mutex g_hbin_mu;
std::map<std::tuple<unsigned long long, long long, double, long long>, std::shared_ptr<const HBinPlan>> g_hbin_cache;

std::shared_ptr<const HBinPlan> hbin_plan(const SumRequest& r) {
    const long long nsq = lattice_nsq(r.lat);
    const double kmax = r.lat.kx * std::sqrt((double)nsq);
    // MV_HBIN_JOB_COST and MV_HBIN_BLOCK_COST (0 .. 1e6) replace the tuned
    // price of one more bin and of one more Chebyshev block
    auto env = [](const char* name) {
        const char* e = std::getenv(name);
        const long v = e ? std::atol(e) : -1;
        return (v >= 0 && v <= 1000000) ? (int)v : -1;
    };
    static const int env_job = env("MV_HBIN_JOB_COST"), env_block = env("MV_HBIN_BLOCK_COST");
    const int job_cost = env_job >= 0 ? env_job : std::max(0, active_tune().hbin_job_cost);
    const int block_cost = env_block >= 0 ? env_block : std::max(0, active_tune().hbin_block_cost);
    const int period = r.lat.nz - 1;
    const int fold = hbin_fold(r.lat);
    const auto key = std::make_tuple(r.hbins->id, ((nsq * 65536 + period) * 4 + r.basis) * 8 + fold, r.lat.kx,
                                     (long long)job_cost * 2000003LL + block_cost);
    std::lock_guard<std::mutex> lock(g_hbin_mu);
    auto it = g_hbin_cache.find(key);
    if (it != g_hbin_cache.end()) return it->second;
    if (g_hbin_cache.size() >= 256) g_hbin_cache.clear();
    auto plan = std::make_shared<const HBinPlan>(hbin_plan_build(*r.hbins, kmax, period, fold, job_cost, block_cost));
    g_hbin_cache[key] = plan;
    return plan;
}

// A group the tensor form takes through h-bins: SPH or Wendland with varying
// radii and a registered histogram.
bool binned_group(const SumRequest& r) {
    const bool uniform = r.radii && r.radius_min >= 0.f && r.radius_min == r.radius_max;
    return r.radii && !uniform && (r.basis == kSph || r.basis == kWendland) && r.hbins &&
           (int)r.hbins->count.size() == kHBinFine;
}

// The automatic choice takes the h-binned tensor form while its work (terms x
// mean Chebyshev order) stays below what the plain form costs, which does
// about a tenth of the tensor form's terms per second.
constexpr double kHBinAutoMaxCost = 6.0;

}  // namespace

int tensor_sum_available(const SumRequest& r, int form) {
    const Lattice& L = r.lat;
    if (!is_spectrum_lattice(L) || r.wrap != 0) return 0;
    const int lz_tc = L.nz - 1;  // planes [0, Kz/2); the Nyquist plane is planned separately
    if (L.ny % 16 || ((long long)L.nx * L.ny) % kM || lz_tc % 8 || lz_tc < 8) return 0;
    if ((long long)L.nx * L.ny * lz_tc * 2 > (1LL << 31)) return 0;
    if (r.weight_max < 0.f) return 0;  // needs the registered |weight| maximum
    const bool uniform = r.radii && r.radius_min >= 0.f && r.radius_min == r.radius_max;
    const bool separable = !r.radii || uniform || r.basis == kGaussianDecaying;
    if (separable) return 1;
    if (!binned_group(r)) return 0;
    if ((long long)L.nx * L.ny * lz_tc * 2 * kHBinMaxOrder > (1LL << 31)) return 0;
    const std::shared_ptr<const HBinPlan> hp = hbin_plan(r);
    if (!hp->feasible) return 0;
    if (form == VIS_FORM_TENSOR) return 1;
    return hp->cost <= kHBinAutoMaxCost ? 1 : 0;
}

namespace {

// Groups whose slots one reduction sums into one output (an output class):
// same output spectrum and the same per-frequency factor (none for Gaussian
// and h-binned jobs, whose factors are applied per particle or per Chebyshev
// block; Phi^(|k| h) with the same basis and h for factored ones).
struct ClassKey {
    const float2* out;
    int unfactored;
    int basis;
    double h;
    bool operator==(const ClassKey& o) const {
        return out == o.out && unfactored == o.unfactored && (unfactored || (basis == o.basis && h == o.h));
    }
};

}  // namespace

int tensor_plan(const std::vector<SumRequest>& groups, TensorPlan& plan) {
    plan = TensorPlan{};
    std::vector<ClassKey> keys;
    // (tile mode, cost, item): kNarrow items first, then kPair, then kWide;
    // each mode longest first
    struct Item {
        int mode;
        long long cost;
        int2 item;
        int m_tile;  // for the order below
        int split;
        int cost_class = 0, m_block = 0;
    };
    std::vector<Item> items;
    plan.flush_narrow = tc_flush_stages(kNarrow);
    plan.flush = tc_flush_stages(kWide);
    // Tiles and particle splits of a job (rows kx * ky, columns lz_tc), its
    // items appended, B-operand images where the job allows them (image_ok)
    // and they fit the limit; returns the job's index.
    const size_t image_limit = operand_cache_limit();
    // the launch's terms (planes below the Nyquist plane), for the size of
    // its work items
    double launch_terms = 1.0;
    for (const SumRequest& r : groups)
        launch_terms += (double)std::max(0, r.n) * r.lat.nx * r.lat.ny * std::max(1, r.lat.nz - 1);
    auto add_job = [&](TcJob j, int mode, bool image_ok, size_t tp_offset, int cls, int acc_part,
                       size_t coef_offset) {
        // equal n-tiles of at most kNc c values: 192 planes -> 96 + 96 (two
        // N = 192 MMAs) rather than 128 + 64 (an N = 128 one, bound by its
        // shared-memory operand reads); multiples of 16 for kPair
        const int nc_max = narrow_mode(mode) ? Shape<kNarrow>::kNc : Shape<kWide>::kNc;
        const int nc_unit = pair_mode(mode) ? 16 : 8;
        j.n_ntiles = (j.lz_tc + nc_max - 1) / nc_max;
        j.nc_tile = ((j.lz_tc + j.n_ntiles - 1) / j.n_ntiles + nc_unit - 1) / nc_unit * nc_unit;
        j.n_ntiles = (j.lz_tc + j.nc_tile - 1) / j.nc_tile;
        const int ctas = pair_mode(mode) ? 2 : 1;
        // the last m-tile may extend past the rows (Nyquist jobs): the flush
        // skips rows >= kx * ky
        j.n_mtiles = (int)(((long long)j.kx * j.ky + kM * ctas - 1) / (kM * ctas));
        // particle splits: items of at most the launch's terms / (units x
        // tc_waves) (default 4 waves), at least 64 stages each; every split
        // is one more slot to write and reduce
        const long long ftiles = (long long)j.n_mtiles * j.n_ntiles;
        const double item_budget = launch_terms / ((double)(device_sm_count() / ctas) * active_tune().tc_waves);
        long long splits = std::max<long long>(
            1, (long long)std::ceil((double)j.n * kM * ctas * std::min(j.nc_tile, j.lz_tc) / item_budget));
        splits = std::min<long long>(splits, std::max<long long>(1, (j.n + 64 * kKp - 1) / (64 * kKp)));
        // The 128-column tiles keep an item's whole sum in an FP32 total: at
        // most kMaxItemChains chains per item.  The 256-column tiles take items
        // of any length: their items add the FP32 total of every
        // kMaxItemChains chains into FP64 totals in the slot.
        const int flush_stages = narrow_mode(mode) ? plan.flush_narrow : plan.flush;
        const long long max_chunk = (long long)kMaxItemChains * flush_stages * kKp;
        if (narrow_mode(mode)) splits = std::max<long long>(splits, (j.n + max_chunk - 1) / max_chunk);
        const long long chunk = ((j.n + splits - 1) / splits + kKp - 1) / kKp * kKp;
        splits = (j.n + chunk - 1) / chunk;
        j.slot_fp64 = chunk > max_chunk ? 1 : 0;
        // short items of a CTA-pair job: double-buffered accumulators
        if (mode == kPair && (chunk / kKp + flush_stages - 1) / flush_stages <= kDBMaxChains && tc_db_enabled())
            mode = kPairDB;
        j.k_chunk = (int)chunk;
        j.n_splits = (int)splits;
        j.ctas = ctas;
        j.slot_stride = ctas * kM * 2 * j.nc_tile;
        j.n_blocks = (j.n + kBlockParticles - 1) / kBlockParticles;
        j.img_stride = 512 * (j.nc_tile / ctas);
        j.bimg = nullptr;
        size_t img_off = SIZE_MAX;
        const size_t img_total = (size_t)j.n_ntiles * ctas * j.n_blocks * (size_t)j.img_stride;
        if (image_ok && j.n_mtiles >= kImageMinReuse && plan.bimg_bytes + img_total <= image_limit) {
            img_off = plan.bimg_bytes;
            plan.bimg_bytes += img_total;
        }
        const int job_index = (int)plan.jobs.size();
        plan.jobs.push_back(j);
        plan.bimg_offset.push_back(img_off);
        plan.job_tp.push_back(tp_offset);
        plan.job_class.push_back(cls);
        plan.job_acc.push_back(acc_part);
        plan.job_coef.push_back(coef_offset);
        plan.job_slot.push_back(plan.slot_bytes);
        plan.slot_bytes += (size_t)(splits * ftiles) * (size_t)j.slot_stride * (j.slot_fp64 ? 8 : 4);
        // column c of the job -> its n-tile and the slot columns of its Re and
        // Im parts (the accumulator's column order: per CTA half h of the
        // n-tile's c values, Re of its bnc values, then Im)
        plan.job_colmap.push_back(plan.colmaps.size());
        for (int c = 0; c < j.lz_tc; ++c) {
            const int n_tile = c / j.nc_tile, c_in = c - n_tile * j.nc_tile;
            const int bnc = std::min(j.nc_tile, j.lz_tc - n_tile * j.nc_tile) / ctas;
            const int h = c_in / bnc, cc = c_in - h * bnc;
            plan.colmaps.push_back(make_int4(n_tile, h * 2 * bnc + cc, h * 2 * bnc + bnc + cc, 0));
        }
        TensorPlan::Class& cl = plan.classes[cls];
        (acc_part == 0 ? cl.jobs : acc_part == 1 ? cl.nyq_pos : cl.nyq_neg).push_back(job_index);
        const int flush = narrow_mode(mode) ? plan.flush_narrow : plan.flush;
        for (long long ks = 0; ks < splits; ++ks) {
            const long long k0 = ks * chunk, k1 = std::min<long long>(j.n, k0 + chunk);
            const long long stages = (k1 - k0 + kKp - 1) / kKp;
            for (long long t = 0; t < ftiles; ++t)
                items.push_back({mode, stages + (stages + flush - 1) / flush, make_int2(job_index, (int)(ks * ftiles + t)),
                                 (int)(t / j.n_ntiles), (int)ks});
        }
        return job_index;
    };
    // tile mode of a job with `cols` columns over kx * ky rows: kNarrow up to
    // 64 columns; beyond, kPair where every n-tile splits into two halves of
    // 8-c chunks and the rows into 256-row m-tiles, else kWide
    auto mode_of = [](int cols, long long rows) {
        const bool pairs = tc_pairs_enabled() && cols % 16 == 0 && rows % 256 == 0;
        return cols <= Shape<kNarrow>::kNc ? (pairs ? kPairNarrow : kNarrow) : (pairs ? kPair : kWide);
    };
    for (size_t g = 0; g < groups.size(); ++g) {
        const SumRequest& r = groups[g];
        const Lattice& L = r.lat;
        const int kx = L.nx, ky = L.ny, lz_out = L.nz, lz_tc = L.nz - 1;
        const bool uniform = r.radii && r.radius_min >= 0.f && r.radius_min == r.radius_max;
        const bool gauss = r.radii && !uniform && r.basis == kGaussianDecaying;
        const bool binned = !gauss && binned_group(r);
        ClassKey key{r.out, (gauss || binned) ? 1 : 0, r.basis, uniform ? (double)r.radius_max : 1.0};
        int cls = -1;
        for (size_t c = 0; c < keys.size(); ++c)
            if (keys[c] == key) cls = (int)c;
        if (cls < 0) {
            cls = (int)keys.size();
            keys.push_back(key);
            TensorPlan::Class c;
            c.out = r.out;
            c.kx = kx;
            c.ky = ky;
            c.lz_tc = lz_tc;
            c.lz_out = lz_out;
            c.step = L.kx;
            c.basis = r.basis;
            c.h = key.h;
            c.factored = !key.unfactored;
            c.scale = r.scale;
            c.nyquist = false;
            plan.classes.push_back(c);
        }
        plan.group_class.push_back(cls);
        plan.group_binned.push_back(-1);
        plan.nyq_job_of_group.push_back(-1);
        plan.tp_nyq_offset.push_back(0);
        plan.tp_offset.push_back(plan.tp_bytes);
        if (r.n <= 0 || !(r.weight_max > 0.f)) {
            plan.job_of_group.push_back(-1);
            continue;
        }
        const bool nyq_ok = ky % 16 == 0 && kx % 2 == 0 && (kx / 2) % 8 == 0;
        // the class's Nyquist plane comes from transposed jobs
        auto class_nyquist = [&]() { plan.classes[cls].nyquist = true; };
        if (binned) {
            // ------------------------------------------ h-binned group
            const std::shared_ptr<const HBinPlan> hp = hbin_plan(r);
            TensorPlan::Binned bg;
            bg.group = (int)g;
            bg.bins = hp->bins;
            bg.nbins = (int)hp->bins.size();
            for (const HBin& b : bg.bins) bg.edges.push_back(r.hbins->edges[b.f0]);
            bg.edges.push_back(r.hbins->edges[kHBinFine]);
            bg.nsq = (int)(lattice_nsq(L) + 1);
            bg.meta_offset = 0;  // placed by tensor_reserve_upload
            bg.sorted_offset = plan.sorted_bytes;
            {
                // sorted particles, their radii, then the radix sort's keys,
                // indices (in and out) and temporary storage
                size_t temp = 0;
                const int sst = check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, temp, (const uint32_t*)nullptr,
                                                                           (uint32_t*)nullptr, (const int*)nullptr,
                                                                           (int*)nullptr, r.n),
                                           "radius sort size");
                if (sst != kOk) return sst;
                bg.sort_temp_bytes = temp;
                const size_t a4 = ((size_t)r.n * 4 + 255) / 256 * 256;
                plan.sorted_bytes += ((size_t)r.n * sizeof(float4) + 255) / 256 * 256 + 5 * a4 + (temp + 255) / 256 * 256;
            }
            bg.coef_offset = plan.coef_bytes / sizeof(float);
            std::vector<int> first_block(bg.nbins);
            long long blocks = 0;
            bg.total_q = 0;
            for (int b = 0; b < bg.nbins; ++b) {
                first_block[b] = (int)blocks;
                blocks += (bg.bins[b].count + kBlockParticles - 1) / kBlockParticles;
                bg.total_q += bg.bins[b].order;
            }
            bg.coef_count = (size_t)bg.total_q * bg.nsq;  // [n2][bin's blocks]
            plan.coef_bytes += (bg.coef_count * sizeof(float) + 255) / 256 * 256;
            const size_t blocks_bytes = (size_t)blocks * kBlockBytes;
            plan.tp_bytes += blocks_bytes;
            // the Nyquist plane as transposed jobs needs whole 8-c blocks of
            // Kx/2 columns (and 16 for pairs, per job below)
            const bool nyq = nyq_ok;
            if (nyq) {
                plan.tp_nyq_offset.back() = plan.tp_bytes;
                plan.tp_bytes += blocks_bytes;
                class_nyquist();
            }
            size_t coef_at = 0;
            int first_job = -1, first_nyq = -1;
            const int bfold = hbin_fold(L);
            for (int b = 0; b < bg.nbins; ++b) {
                const HBin& bin = bg.bins[b];
                const size_t coef_off = bg.coef_offset + coef_at;  // the bin's first block, within one |k|^2
                coef_at += (size_t)bin.order;
                if (bin.count <= 0 || !(bin.wmax > 0.f)) continue;
                TcJob j{};
                j.kx = kx;
                j.ky = ky / bfold;
                j.lz_tc = bin.order * lz_tc * bfold;  // column blocks q bfold + bl of lz_tc planes
                j.a_base = -kx / 2;
                j.b_base = -ky / 2;
                j.c_base = 0;
                j.n = bin.count;
                j.gauss = 0;
                j.wmax = bin.wmax;
                j.period = lz_tc;
                j.fold = bfold;
                j.coef_stride = bg.total_q;
                const size_t tp = plan.tp_offset.back() + (size_t)first_block[b] * kBlockBytes;
                const int jm = add_job(j, mode_of(j.lz_tc, (long long)kx * j.ky), true, tp, cls, 0, coef_off);
                if (first_job < 0) first_job = jm;
                if (nyq) {
                    TcJob t = j;
                    t.kx = 1;
                    t.ky = ky;
                    t.lz_tc = bin.order * (kx / 2);
                    t.period = kx / 2;
                    t.fold = 0;
                    t.a_base = lz_tc;
                    t.b_base = -ky / 2;
                    t.c_base = 0;
                    const int nmode = mode_of(t.lz_tc, ky);
                    const size_t tpn = plan.tp_nyq_offset.back() + (size_t)first_block[b] * kBlockBytes;
                    const int jn = add_job(t, nmode, false, tpn, cls, 1, coef_off);
                    if (first_nyq < 0) first_nyq = jn;
                    t.a_base = -lz_tc;
                    t.b_base = 1 - ky / 2;
                    t.c_base = 1;
                    add_job(t, nmode, false, tpn, cls, 2, coef_off);
                }
            }
            plan.job_of_group.push_back(first_job);
            plan.nyq_job_of_group.back() = nyq ? first_nyq : -1;
            plan.group_binned.back() = (int)plan.binned.size();
            plan.binned.push_back(std::move(bg));
            continue;
        }
        // ------------------------------------------------ separable group
        const size_t blocks_bytes =
            (size_t)((std::max(0, r.n) + kBlockParticles - 1) / kBlockParticles) * kBlockBytes;
        plan.tp_bytes += blocks_bytes;
        const int mode = mode_of(lz_tc, (long long)kx * ky);
        // Row fold of a group whose terms are pure phases: the F of {1, 2, 4}
        // whose columns F lz_tc fill the MMAs best.  A CTA-pair (or narrow)
        // MMA costs about the same whatever its N up to 256 (128 c values),
        // so the cost per column is n-tiles / columns.
        int fold = 1;
        if (!gauss && tc_fold_enabled()) {
            auto cost = [&](int f) {
                const int cols = f * lz_tc;
                const int nc_max = cols <= Shape<kNarrow>::kNc ? Shape<kNarrow>::kNc : Shape<kWide>::kNc;
                return (double)((cols + nc_max - 1) / nc_max) / cols;
            };
            for (int f : {2, 4})
                if (ky % (16 * f) == 0 && cost(f) < cost(fold) * 0.99) fold = f;
        }
        // Axis exchange of a group that cannot fold (per-particle Gaussian
        // factors): rows (a, c), columns b, where Ky columns fill the MMAs
        // better than the planes (384^3: 3 n-tiles of 128 b values instead of
        // 96 + 96 planes)
        bool exch = false;
        if (fold == 1 && tc_exchange_enabled()) {
            auto cost = [&](int cols) {
                const int nc_max = cols <= Shape<kNarrow>::kNc ? Shape<kNarrow>::kNc : Shape<kWide>::kNc;
                return (double)((cols + nc_max - 1) / nc_max) / cols;
            };
            exch = ky % 16 == 0 && ((long long)kx * lz_tc) % 256 == 0 && cost(ky) < cost(lz_tc) * 0.99;
        }
        TcJob j{};
        j.kx = kx;
        j.ky = exch ? lz_tc : ky / fold;
        j.lz_tc = exch ? ky : fold * lz_tc;
        j.a_base = -kx / 2;
        j.b_base = exch ? 0 : -ky / 2;
        j.c_base = exch ? -ky / 2 : 0;
        j.n = r.n;
        j.gauss = gauss ? 1 : 0;
        j.wmax = r.weight_max;
        j.fold = fold;
        j.period = fold > 1 ? lz_tc : 0;
        j.exch = exch ? 1 : 0;
        plan.job_of_group.push_back(add_job(j, mode_of(j.lz_tc, (long long)kx * j.ky), true, plan.tp_offset.back(),
                                            cls, 0, SIZE_MAX));
        // The Nyquist plane as two transposed jobs (rows b, columns a >= 0 and
        // -a > 0; see TcJob) in the same launch, where the Kx / 2 columns of
        // each split into whole n-tile units (16 c for kPair, else 8);
        // otherwise the plain form sums it.  Their Ky rows (8-row chunks of one
        // sign of b) need not fill the last m-tile.
        if (nyq_ok && (kx / 2) % (pair_mode(mode) ? 16 : 8) == 0) {
            plan.tp_nyq_offset.back() = plan.tp_bytes;
            plan.tp_bytes += blocks_bytes;
            TcJob t = j;
            t.kx = 1;
            t.ky = ky;
            t.lz_tc = kx / 2;
            t.a_base = lz_tc;
            t.b_base = -ky / 2;
            t.c_base = 0;
            t.fold = 0;
            t.period = 0;
            t.exch = 0;
            const size_t tpn = plan.tp_nyq_offset.back();
            plan.nyq_job_of_group.back() = add_job(t, mode, false, tpn, cls, 1, SIZE_MAX);  // one m-tile: no reuse
            t.a_base = -lz_tc;
            t.b_base = 1 - ky / 2;
            t.c_base = 1;
            add_job(t, mode, false, tpn, cls, 2, SIZE_MAX);
            class_nyquist();
        }
    }
    if (items.size() > (size_t)INT32_MAX) return set_error(kInvalidValue, "tensor sum: too many work items");
    // Per tile mode, longest first (round-robin over the persistent CTAs /
    // pairs), in cost classes 5% wide.  Within a class, items run in blocks of
    // as many m-tiles as there are resident units: one wave takes one (job,
    // split) over distinct m-tiles, all of them reading the same B-operand
    // stages (images) at about the same time, and the next waves the other
    // jobs' items of the same m-tiles.
    auto order = [](int m) { return m == kNarrow ? 0 : m == kPairNarrow ? 1 : m == kPair ? 2 : m == kPairDB ? 3 : 4; };
    const int sms = std::max(2, device_sm_count());
    for (Item& it : items) {
        it.cost_class = (int)std::floor(std::log((double)std::max(1LL, it.cost)) / std::log(1.05));
        it.m_block = it.m_tile / (pair_mode(it.mode) ? sms / 2 : sms);
    }
    std::stable_sort(items.begin(), items.end(), [&](const Item& x, const Item& y) {
        if (x.mode != y.mode) return order(x.mode) < order(y.mode);
        if (x.cost_class != y.cost_class) return x.cost_class > y.cost_class;
        if (x.m_block != y.m_block) return x.m_block < y.m_block;
        if (x.item.x != y.item.x) return x.item.x < y.item.x;
        if (x.split != y.split) return x.split < y.split;
        return x.item.y < y.item.y;
    });
    plan.items.reserve(items.size());
    plan.n_narrow = plan.n_pair_narrow = plan.n_pair = plan.n_pair_db = 0;
    for (auto& it : items) {
        plan.items.push_back(it.item);
        plan.n_narrow += it.mode == kNarrow ? 1 : 0;
        plan.n_pair_narrow += it.mode == kPairNarrow ? 1 : 0;
        plan.n_pair += it.mode == kPair ? 1 : 0;
        plan.n_pair_db += it.mode == kPairDB ? 1 : 0;
    }
    const size_t jobs_bytes = ((plan.jobs.size() * sizeof(TcJob) + 255) / 256) * 256;
    plan.meta_bytes = jobs_bytes + ((plan.items.size() * sizeof(int2) + 255) / 256) * 256;
    // the jobs with B-operand images and their first images
    plan.img_jobs.clear();
    plan.img_first.assign(1, 0);
    for (size_t j = 0; j < plan.jobs.size(); ++j) {
        if (plan.bimg_offset[j] == SIZE_MAX) continue;
        const TcJob& J = plan.jobs[j];
        plan.img_jobs.push_back((int)j);
        plan.img_first.push_back(plan.img_first.back() + (long long)J.n_ntiles * J.ctas * J.n_blocks);
    }
    plan.img_jobs_offset = plan.meta_bytes;
    plan.meta_bytes += (plan.img_jobs.size() * sizeof(int) + 255) / 256 * 256;
    plan.img_first_offset = plan.meta_bytes;
    plan.meta_bytes += (plan.img_first.size() * sizeof(long long) + 255) / 256 * 256;
    // the jobs' column maps
    plan.colmap_offset = plan.meta_bytes;
    plan.meta_bytes += (plan.colmaps.size() * sizeof(int4) + 255) / 256 * 256;
    // each class's job lists (planes, Nyquist a >= 0, Nyquist a < 0)
    for (TensorPlan::Class& c : plan.classes) {
        c.list_offset = plan.meta_bytes;
        plan.meta_bytes += ((c.jobs.size() + c.nyq_pos.size() + c.nyq_neg.size()) * sizeof(int) + 255) / 256 * 256;
    }
    // the binned groups' tables: edges, int4 bins, float4 spans, int first
    // particles (16-byte aligned)
    for (TensorPlan::Binned& bg : plan.binned) {
        bg.meta_offset = plan.meta_bytes;
        const size_t edges = ((size_t)(bg.nbins + 1) * sizeof(float) + 15) / 16 * 16;
        plan.meta_bytes += edges + (size_t)bg.nbins * (sizeof(int4) + sizeof(float4)) + (size_t)(bg.nbins + 1) * sizeof(int);
        plan.meta_bytes = (plan.meta_bytes + 255) / 256 * 256;
    }
    return kOk;
}

int tensor_reserve_upload(TensorPlan& plan, TensorWorkspace& ws, cudaStream_t stream) {
    int st = ws.particles.reserve(std::max<size_t>(plan.tp_bytes, 256));
    if (st == kOk) st = ws.meta.reserve(std::max<size_t>(plan.meta_bytes, 256));
    if (st == kOk && plan.bimg_bytes) st = ws.bimg.reserve(plan.bimg_bytes);
    if (st == kOk && plan.coef_bytes) st = ws.coef.reserve(plan.coef_bytes);
    if (st == kOk && plan.sorted_bytes) st = ws.sorted.reserve(plan.sorted_bytes);
    if (st == kOk) st = ws.slots.reserve(std::max<size_t>(plan.slot_bytes, 256));
    if (st != kOk) return st;
    char* tp_base = static_cast<char*>(ws.particles.ptr);
    for (size_t j = 0; j < plan.jobs.size(); ++j) {
        TcJob& job = plan.jobs[j];
        job.bimg = plan.bimg_offset[j] == SIZE_MAX ? nullptr
                                                   : static_cast<const unsigned char*>(ws.bimg.ptr) + plan.bimg_offset[j];
        job.blocks = reinterpret_cast<const unsigned char*>(tp_base + plan.job_tp[j]);
        job.slots = static_cast<char*>(ws.slots.ptr) + plan.job_slot[j];
        job.colmap = reinterpret_cast<const int4*>(static_cast<char*>(ws.meta.ptr) + plan.colmap_offset) +
                     plan.job_colmap[j];
        job.coef = plan.job_coef[j] == SIZE_MAX ? nullptr : static_cast<const float*>(ws.coef.ptr) + plan.job_coef[j];
    }
    std::vector<char> meta(plan.meta_bytes, 0);
    const size_t jobs_bytes = ((plan.jobs.size() * sizeof(TcJob) + 255) / 256) * 256;
    if (!plan.jobs.empty()) std::memcpy(meta.data(), plan.jobs.data(), plan.jobs.size() * sizeof(TcJob));
    if (!plan.items.empty()) std::memcpy(meta.data() + jobs_bytes, plan.items.data(), plan.items.size() * sizeof(int2));
    if (!plan.colmaps.empty())
        std::memcpy(meta.data() + plan.colmap_offset, plan.colmaps.data(), plan.colmaps.size() * sizeof(int4));
    if (!plan.img_jobs.empty()) {
        std::memcpy(meta.data() + plan.img_jobs_offset, plan.img_jobs.data(), plan.img_jobs.size() * sizeof(int));
        std::memcpy(meta.data() + plan.img_first_offset, plan.img_first.data(), plan.img_first.size() * sizeof(long long));
    }
    for (const TensorPlan::Class& c : plan.classes) {
        int* l = reinterpret_cast<int*>(meta.data() + c.list_offset);
        for (int v : c.jobs) *l++ = v;
        for (int v : c.nyq_pos) *l++ = v;
        for (int v : c.nyq_neg) *l++ = v;
    }
    for (const TensorPlan::Binned& bg : plan.binned) {
        float* edges = reinterpret_cast<float*>(meta.data() + bg.meta_offset);
        const size_t edges_bytes = ((size_t)(bg.nbins + 1) * sizeof(float) + 15) / 16 * 16;
        int4* bins = reinterpret_cast<int4*>(meta.data() + bg.meta_offset + edges_bytes);
        float4* spans = reinterpret_cast<float4*>(bins + bg.nbins);
        int* first = reinterpret_cast<int*>(spans + bg.nbins);
        int block = 0, particle = 0;
        int coef_at = 0;
        for (int b = 0; b < bg.nbins; ++b) {
            const HBin& bin = bg.bins[b];
            edges[b] = bg.edges[b];
            bins[b] = make_int4(block, bin.count, coef_at, bin.order);
            spans[b] = make_float4(bin.lo, bin.hi, bin.wmax > 0.f ? kOperandScale / bin.wmax : 0.f, 0.f);
            first[b] = particle;
            block += (bin.count + kBlockParticles - 1) / kBlockParticles;
            particle += bin.count;
            coef_at += bin.order;
        }
        edges[bg.nbins] = bg.edges[bg.nbins];
        first[bg.nbins] = particle;
    }
    plan.d_jobs = static_cast<const void*>(ws.meta.ptr);
    plan.d_items = static_cast<const void*>(static_cast<char*>(ws.meta.ptr) + jobs_bytes);
    if (meta.empty()) return kOk;
    // the same tables as last time (same groups, same buffers): nothing to copy
    if (ws.uploaded_to == ws.meta.ptr && ws.uploaded == meta) return kOk;
    st = check_cuda(cudaMemcpyAsync(ws.meta.ptr, meta.data(), meta.size(), cudaMemcpyHostToDevice, stream),
                    "tensor metadata H2D");
    if (st != kOk) return st;
    // the host vector dies here: make sure the pageable copy has been staged
    st = check_cuda(cudaStreamSynchronize(stream), "tensor metadata H2D");
    if (st != kOk) return st;
    ws.uploaded = std::move(meta);
    ws.uploaded_to = ws.meta.ptr;
    return kOk;
}

int tensor_prepare(const std::vector<SumRequest>& groups, TensorWorkspace& ws, cudaStream_t stream,
                   const TensorPlan** plan) {
    // everything tensor_plan reads, field by field (no padding bytes)
    std::string key;
    auto put = [&key](const void* p, size_t n) { key.append(static_cast<const char*>(p), n); };
    int dev = -1;
    cudaGetDevice(&dev);
    put(&dev, sizeof dev);
    const TuneParams& tp = active_tune();
    const int tune[6] = {tp.plain_waves, tp.tc_waves, tp.tc_flush, tp.hbin_job_cost, tp.hbin_block_cost, tp.tc_shapes};
    put(tune, sizeof tune);
    const size_t limit = operand_cache_limit();
    put(&limit, sizeof limit);
    for (const SumRequest& r : groups) {
        // the histogram by its content id, not its address: a registration of
        // the same data again gives the same plan
        const void* ptrs[5] = {r.particles, r.radii, r.out, r.shell_edges, r.shell_first};
        put(ptrs, sizeof ptrs);
        const unsigned long long hid = r.hbins ? r.hbins->id : 0ull;
        put(&hid, sizeof hid);
        const float f[3] = {r.radius_min, r.radius_max, r.weight_max};
        put(f, sizeof f);
        const long long ll[4] = {r.out_base, r.out_sx, r.out_sy, r.out_sz};
        put(ll, sizeof ll);
        const int in[10] = {r.n, r.basis, r.wrap, r.row, r.accumulate ? 1 : 0, r.kink, r.shell_nbins,
                            r.lat.nx, r.lat.ny, r.lat.nz};
        put(in, sizeof in);
        const int org[3] = {r.lat.x0, r.lat.y0, r.lat.z0};
        put(org, sizeof org);
        const double d[13] = {r.lat.kx, r.lat.ky, r.lat.kz, r.lat.m[0], r.lat.m[1], r.lat.m[2], r.lat.m[3],
                              r.lat.m[4], r.lat.m[5], r.lat.m[6], r.lat.m[7], r.lat.m[8], r.scale};
        put(d, sizeof d);
        put(&r.stream, sizeof r.stream);
        put(&r.error_flag, sizeof r.error_flag);
    }
    if (ws.plan && ws.plan_key == key) {
        *plan = ws.plan.get();
        return kOk;
    }
    ws.plan_key.clear();
    auto fresh = std::make_unique<TensorPlan>();
    int st = tensor_plan(groups, *fresh);
    if (st == kOk) st = tensor_reserve_upload(*fresh, ws, stream);
    if (st != kOk) {
        ws.plan.reset();
        return st;
    }
    ws.plan = std::move(fresh);
    ws.plan_key = std::move(key);
    *plan = ws.plan.get();
    return kOk;
}

namespace {

// One persistent launch of a tile mode: min(items, SMs) CTAs, or for the CTA
// pair modes clusters of 2, as many as can be resident at once.
template <int MODE>
int launch_tile(const TcArgs& a, cudaStream_t stream) {
    using SH = Shape<MODE>;
    int st = check_cuda(
        cudaFuncSetAttribute(tc_sum_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SH::kSmemBytes),
        "cudaFuncSetAttribute");
    if (st != kOk) return st;
    if constexpr (SH::kCtas == 1) {
        const int grid = std::min<int>(a.n_items, device_sm_count());
        tc_sum_kernel<MODE><<<grid, kThreads, SH::kSmemBytes, stream>>>(a);
        return kOk;
    } else {
        cudaLaunchConfig_t lc = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        lc.blockDim = dim3(kThreads);
        lc.dynamicSmemBytes = SH::kSmemBytes;
        lc.stream = stream;
        lc.attrs = attr;
        lc.numAttrs = 1;
        lc.gridDim = dim3(2 * std::max(1, device_sm_count() / 2));
        int clusters = 0;
        st = check_cuda(cudaOccupancyMaxActiveClusters(&clusters, tc_sum_kernel<MODE>, &lc),
                        "cudaOccupancyMaxActiveClusters");
        if (st != kOk) return st;
        if (clusters < 1) return set_error(kCudaError, "tensor sum: no CTA pair fits on this device");
        lc.gridDim = dim3(2 * std::min(a.n_items, clusters));
        return check_cuda(cudaLaunchKernelEx(&lc, tc_sum_kernel<MODE>, a), "tc_sum_kernel (pairs) launch");
    }
}

}  // namespace

namespace {
// Dynamic shared memory of the reduction kernels: the class's job
// descriptors (and the planes kernel's partial sums).
int reduce_smem(void (*kernel)(TcReduceArgs), size_t bytes) {
    if (bytes > 200 * 1024) return set_error(kInvalidValue, "tensor sum: too many jobs in one output class");
    if (bytes <= 48 * 1024) return kOk;
    return check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
                      "cudaFuncSetAttribute(reduction)");
}
}  // namespace

int tensor_enqueue(const std::vector<SumRequest>& groups, const TensorPlan& plan, TensorWorkspace& ws,
                   Workspace& plain_ws, KernelTimer* timer, cudaStream_t stream, int* error_flag) {
    int st = kOk;
    // per-particle constants of every group
    for (size_t g = 0; g < groups.size(); ++g) {
        const int j = plan.job_of_group[g];
        if (j < 0) continue;
        const SumRequest& r = groups[g];
        if (plan.group_binned[g] >= 0) {
            // h-binned: zeroed blocks (padding particles get zero amplitude),
            // the scatter into the bins, and the bins' coefficient tables
            const TensorPlan::Binned& bg = plan.binned[plan.group_binned[g]];
            size_t blocks = 0;
            for (const HBin& b : bg.bins) blocks += (size_t)((b.count + kBlockParticles - 1) / kBlockParticles);
            char* tp = static_cast<char*>(ws.particles.ptr) + plan.tp_offset[g];
            char* tpn = plan.nyq_job_of_group[g] >= 0 ? static_cast<char*>(ws.particles.ptr) + plan.tp_nyq_offset[g]
                                                      : nullptr;
            st = check_cuda(cudaMemsetAsync(tp, 0, blocks * kBlockBytes, stream), "cudaMemsetAsync(binned blocks)");
            if (st == kOk && tpn)
                st = check_cuda(cudaMemsetAsync(tpn, 0, blocks * kBlockBytes, stream), "cudaMemsetAsync(binned blocks)");
            if (st != kOk) return st;
            const char* meta = static_cast<const char*>(ws.meta.ptr) + bg.meta_offset;
            const size_t edges_bytes = ((size_t)(bg.nbins + 1) * sizeof(float) + 15) / 16 * 16;
            TcBinnedPrepArgs bp;
            bp.particles = r.particles;
            bp.radii = r.radii;
            bp.n = r.n;
            bp.step = r.lat.kx;
            bp.nbins = bg.nbins;
            bp.edges = reinterpret_cast<const float*>(meta);
            bp.bins = reinterpret_cast<const int4*>(meta + edges_bytes);
            bp.spans = reinterpret_cast<const float4*>(bp.bins + bg.nbins);
            bp.out = reinterpret_cast<uint8_t*>(tp);
            bp.out_nyq = reinterpret_cast<uint8_t*>(tpn);
            bp.first = reinterpret_cast<const int*>(bp.spans + bg.nbins);
            char* sorted = static_cast<char*>(ws.sorted.ptr) + bg.sorted_offset;
            bp.sorted = reinterpret_cast<float4*>(sorted);
            bp.sorted_radii = reinterpret_cast<float*>(sorted + ((size_t)r.n * sizeof(float4) + 255) / 256 * 256);
            bp.error_flag = error_flag;
            bp.fold = std::max(1, plan.jobs[j].fold);
            {
                // the particles in ascending radius (stable: ties keep their
                // index order), so every bin is a run of it, in the same order
                // on every compute
                const size_t a4 = ((size_t)r.n * 4 + 255) / 256 * 256;
                char* base = sorted + ((size_t)r.n * sizeof(float4) + 255) / 256 * 256 + a4;
                uint32_t* keys_in = reinterpret_cast<uint32_t*>(base);
                uint32_t* keys_out = reinterpret_cast<uint32_t*>(base + a4);
                int* index_in = reinterpret_cast<int*>(base + 2 * a4);
                int* index_out = reinterpret_cast<int*>(base + 3 * a4);
                void* temp = base + 4 * a4;
                size_t temp_bytes = bg.sort_temp_bytes;
                tc_radius_keys_kernel<<<(r.n + 255) / 256, 256, 0, stream>>>(r.radii, r.n, keys_in, index_in);
                count_launch();
                st = check_cuda(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_in, keys_out, index_in, index_out,
                                                                r.n, 0, 32, stream),
                                "radius sort");
                if (st != kOk) return st;
                bp.order = index_out;
            }
            tc_prep_binned_kernel<<<(r.n + 255) / 256, 256, 0, stream>>>(bp);
            count_launch();
            TcCoefArgs ca;
            ca.basis = r.basis;
            ca.step = r.lat.kx;
            ca.nbins = bg.nbins;
            ca.nsq = bg.nsq;
            ca.total_q = bg.total_q;
            ca.bins = bp.bins;
            ca.spans = bp.spans;
            ca.edges = bp.edges;
            ca.r0 = (float)phi_branch_point(r.basis);
            ca.coef = static_cast<float*>(ws.coef.ptr) + bg.coef_offset;
            const long long entries = (long long)bg.nbins * bg.nsq;
            tc_coef_kernel<<<(unsigned)((entries + 127) / 128), 128, 0, stream>>>(ca);
            count_launch();
            continue;
        }
        const Lattice& L = r.lat;
        TcPrepArgs pa;
        pa.particles = r.particles;
        pa.radii = r.radii;
        pa.n = r.n;
        pa.step = L.kx;
        pa.gauss = plan.jobs[j].gauss != 0;
        pa.gamma_scale = pa.gauss ? (float)(-(double)kPiLog2e * L.kx * L.kx) : 0.f;
        pa.inv_wmax = 1.0f / r.weight_max;
        pa.fold = std::max(1, plan.jobs[j].fold);
        pa.exch = plan.jobs[j].exch;
        pa.out = const_cast<unsigned char*>(plan.jobs[j].blocks);
        const int t = plan.nyq_job_of_group[g];
        pa.out_nyq = t < 0 ? nullptr : const_cast<unsigned char*>(plan.jobs[t].blocks);
        tc_prep_kernel<<<(r.n + 255) / 256, 256, 0, stream>>>(pa);
        count_launch();
    }
    st = check_cuda(cudaGetLastError(), "tc_prep_kernel launch");
    if (st != kOk) return st;
    // B-operand images of every job that has them, in one launch (after the
    // constants they are made from)
    if (!plan.img_jobs.empty()) {
        TcImageArgs ia;
        ia.jobs = static_cast<const TcJob*>(plan.d_jobs);
        ia.img_jobs = reinterpret_cast<const int*>(static_cast<const char*>(ws.meta.ptr) + plan.img_jobs_offset);
        ia.img_first = reinterpret_cast<const long long*>(static_cast<const char*>(ws.meta.ptr) + plan.img_first_offset);
        ia.n_img_jobs = (int)plan.img_jobs.size();
        const long long images = plan.img_first.back();
        if (images > 0x7fffffffLL) return set_error(kInvalidValue, "tensor sum: too many B-operand images");
        tc_bimg_kernel<<<(unsigned)images, 256, 0, stream>>>(ia);
        count_launch();
        st = check_cuda(cudaGetLastError(), "tc_bimg_kernel launch");
        if (st != kOk) return st;
    }
    // one persistent launch per tile mode for all groups
    if (!plan.items.empty()) {
        timer_begin(timer, 3, stream);
        const int counts[5] = {plan.n_narrow, plan.n_pair_narrow, plan.n_pair, plan.n_pair_db,
                               (int)plan.items.size() - plan.n_narrow - plan.n_pair_narrow - plan.n_pair -
                                   plan.n_pair_db};
        const int modes[5] = {kNarrow, kPairNarrow, kPair, kPairDB, kWide};
        int first = 0;
        bool hooked = false;
        for (int m = 0; m < 5 && st == kOk; first += counts[m], ++m) {
            TcArgs a;
            a.jobs = static_cast<const TcJob*>(plan.d_jobs);
            a.items = static_cast<const int2*>(plan.d_items) + first;
            a.n_items = counts[m];
            a.flush_stages = narrow_mode(modes[m]) ? plan.flush_narrow : plan.flush;
            a.error_flag = error_flag;
            a.wait_limit_ns = kWaitLimitNs;
            a.withhold_first_arrival = 0;
            if (a.n_items == 0) continue;
            if (!hooked) {
                hooked = true;
                const long long t = g_test_wait_limit_ns.exchange(0);
                if (t > 0) {
                    a.wait_limit_ns = (unsigned long long)t;
                    a.withhold_first_arrival = 1;
                }
            }
            switch (modes[m]) {
            case kNarrow: st = launch_tile<kNarrow>(a, stream); break;
            case kPairNarrow: st = launch_tile<kPairNarrow>(a, stream); break;
            case kPair: st = launch_tile<kPair>(a, stream); break;
            case kPairDB: st = launch_tile<kPairDB>(a, stream); break;
            default: st = launch_tile<kWide>(a, stream); break;
            }
            if (st != kOk) break;
            count_launch();
            st = check_cuda(cudaGetLastError(), "tc_sum_kernel launch");
        }
        timer_end(timer, 3, stream);
        if (st != kOk) return st;
    }
    // the items' tiles -> spectra, summed in FP64 (added to what is there)
    for (const TensorPlan::Class& c : plan.classes) {
        const int* lists = reinterpret_cast<const int*>(static_cast<const char*>(ws.meta.ptr) + c.list_offset);
        TcReduceArgs f;
        f.jobs = static_cast<const TcJob*>(plan.d_jobs);
        f.list = lists;
        f.n_list = (int)c.jobs.size();
        f.list_neg = nullptr;
        f.n_neg = 0;
        f.kx = c.kx;
        f.ky = c.ky;
        f.lz_tc = c.lz_tc;
        f.lz_out = c.lz_out;
        f.step = c.step;
        f.basis = c.basis;
        f.h = c.h;
        f.factored = c.factored;
        f.scale = c.scale;
        f.out = c.out;
        f.warp_rows = f.n_list < kReduceWarps ? 1 : 0;
        if (f.n_list > 0) {
            const int block_rows = f.warp_rows ? 32 * kReduceWarps : 32;
            const long long blocks =
                ((long long)c.kx * c.ky + block_rows - 1) / block_rows * (c.lz_tc / kReduceC);
            const size_t smem = (((size_t)f.n_list * sizeof(ReduceJob) + 15) & ~(size_t)15) +
                                (size_t)kReduceWarps * 32 * kReduceC * sizeof(double2);
            st = reduce_smem(tc_reduce_planes_kernel, smem);
            if (st != kOk) return st;
            tc_reduce_planes_kernel<<<(unsigned)blocks, 32 * kReduceWarps, smem, stream>>>(f);
            count_launch();
        }
        if (c.nyquist) {
            f.list = lists + c.jobs.size();
            f.n_list = (int)c.nyq_pos.size();
            f.list_neg = lists + c.jobs.size() + c.nyq_pos.size();
            f.n_neg = (int)c.nyq_neg.size();
            const long long plane = (long long)c.kx * c.ky;
            const size_t smem = (((size_t)(f.n_list + f.n_neg) * sizeof(ReduceJob) + 15) & ~(size_t)15) +
                                (size_t)32 * kReduceWarps * sizeof(double2);
            st = reduce_smem(tc_reduce_kernel, smem);
            if (st != kOk) return st;
            tc_reduce_kernel<<<(unsigned)((plane + 31) / 32), 32 * kReduceWarps, smem, stream>>>(f);
            count_launch();
        }
    }
    st = check_cuda(cudaGetLastError(), "tc_reduce_kernel launch");
    if (st != kOk) return st;
    // the branch part of h-binned groups with the plain form, over their
    // particles sorted by bin
    for (size_t g = 0; g < groups.size(); ++g) {
        if (plan.group_binned[g] < 0 || plan.job_of_group[g] < 0) continue;
        const TensorPlan::Binned& bg = plan.binned[plan.group_binned[g]];
        const char* meta = static_cast<const char*>(ws.meta.ptr) + bg.meta_offset;
        const size_t edges_bytes = ((size_t)(bg.nbins + 1) * sizeof(float) + 15) / 16 * 16;
        const char* sorted = static_cast<const char*>(ws.sorted.ptr) + bg.sorted_offset;
        SumRequest k = groups[g];
        k.particles = reinterpret_cast<const float4*>(sorted);
        k.radii = reinterpret_cast<const float*>(sorted + ((size_t)k.n * sizeof(float4) + 255) / 256 * 256);
        k.accumulate = true;
        k.kink = 1;
        k.shell_edges = reinterpret_cast<const float*>(meta);
        k.shell_first = reinterpret_cast<const int*>(meta + edges_bytes + (size_t)bg.nbins * (sizeof(int4) + sizeof(float4)));
        k.shell_nbins = bg.nbins;
        // without transposed Nyquist jobs the plain form sums the whole Nyquist
        // plane below (branch included): leave it out here
        if (plan.nyq_job_of_group[g] < 0) k.lat.nz -= 1;
        st = launch_plain_sum(k, plain_ws, timer);
        if (st != kOk) return st;
    }
    // the Nyquist plane l = Kz/2 with the plain form, for groups without a
    // transposed job (groups without particles or weight have neither)
    for (size_t g = 0; g < groups.size(); ++g) {
        if (plan.job_of_group[g] >= 0 && plan.nyq_job_of_group[g] >= 0) continue;
        const SumRequest& r = groups[g];
        SumRequest nyq = r;
        const int lz_tc = r.lat.nz - 1;
        nyq.lat.z0 = lz_tc;
        nyq.lat.nz = 1;
        nyq.out_base = lz_tc;
        nyq.out_sx = (long long)r.lat.ny * r.lat.nz;
        nyq.out_sy = r.lat.nz;
        nyq.out_sz = 1;
        nyq.accumulate = true;
        st = launch_plain_sum(nyq, plain_ws, nullptr);
        if (st != kOk) return st;
    }
    return kOk;
}

}  // namespace mv
