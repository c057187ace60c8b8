// Aliasing cull of the direct slice path: meshless_vis/meshless_vis.cu:39-127
// (cull_fully_aliased_terms), which the reference keeps disabled
// (meshless_vis.cu:336) and whose compaction is broken (the radii copy at
// :110 writes the constraint buffer, and compact() gathers where it should
// scatter).  This restates what it is meant to compute:
//   a particle is kept when the four corners of its footprint square, centre
//   (p.u, p.v) in the image plane and half-side h_j (0 without radii), all lie
//   in the box [0, 1 / (2 step.x)] x [0, 1 / (2 step.y)] (compute_mask and
//   point_in_box, meshless_vis.cu:39-57, :88-89);
// and sums only the kept particles.  Unlike the reference it leaves the
// registered arrays untouched: the kept particles (and radii) are compacted,
// in order, into the config's workspace for this render, so every view culls
// from the full set.
//
// Three launches: per-block kept counts, an exclusive scan of the counts (one
// block), and an order-preserving scatter that ranks kept particles within
// each block by a block-wide prefix sum.  The host then reads the kept count (one
// synchronisation) to size the sum.
#include "mv_internal.h"

namespace mv {
namespace {

constexpr int kCullThreads = 1024;

struct CullArgs {
    const float4* particles;
    const float* radii;
    int n;
    float3 u, v;
    float box_x, box_y;  // the box's upper corner; its lower corner is (0, 0)
    int* block_counts;   // [blocks], then the total
    float4* out_particles;
    float* out_radii;
};

__device__ __forceinline__ bool kept(const CullArgs& a, int j) {
    if (j >= a.n) return false;
    const float4 p = a.particles[j];
    const float r = a.radii ? a.radii[j] : 0.f;
    const float cx = p.x * a.u.x + p.y * a.u.y + p.z * a.u.z;
    const float cy = p.x * a.v.x + p.y * a.v.y + p.z * a.v.z;
    // the four corners (cx +- r, cy +- r) inside [0, box_x] x [0, box_y]
    const float xs[2] = {cx + r, cx - r}, ys[2] = {cy + r, cy - r};
    bool in = true;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int k = 0; k < 2; ++k) in = in && xs[i] >= 0.f && ys[k] >= 0.f && xs[i] <= a.box_x && ys[k] <= a.box_y;
    return in;
}

// Exclusive prefix sum of v over the block (kCullThreads threads: 32 warps);
// *total receives the block's sum.  warp_sums and total are shared memory,
// free again when this returns.
__device__ __forceinline__ int block_exclusive_sum(int v, int* warp_sums, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const int w = warp_sums[lane];
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        warp_sums[lane] = wi - w;
        if (lane == 31) *total = wi;
    }
    __syncthreads();
    const int r = warp_sums[warp] + incl - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kCullThreads) cull_count_kernel(CullArgs a) {
    __shared__ int warp_sums[32];
    __shared__ int total;
    const int j = blockIdx.x * kCullThreads + threadIdx.x;
    block_exclusive_sum(kept(a, j) ? 1 : 0, warp_sums, &total);
    if (threadIdx.x == 0) a.block_counts[blockIdx.x] = total;
}

// Exclusive scan of the block counts in place; the total goes after them.
__global__ void __launch_bounds__(kCullThreads) cull_scan_kernel(int* counts, int blocks) {
    __shared__ int warp_sums[32];
    __shared__ int total;
    int carry = 0;
    for (int base = 0; base < blocks; base += kCullThreads) {
        const int i = base + threadIdx.x;
        const int v = i < blocks ? counts[i] : 0;
        const int excl = block_exclusive_sum(v, warp_sums, &total);
        if (i < blocks) counts[i] = carry + excl;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) counts[blocks] = carry;
}

__global__ void __launch_bounds__(kCullThreads) cull_scatter_kernel(CullArgs a) {
    __shared__ int warp_sums[32];
    __shared__ int total;
    const int j = blockIdx.x * kCullThreads + threadIdx.x;
    const bool keep = kept(a, j);
    const int r = block_exclusive_sum(keep ? 1 : 0, warp_sums, &total);
    if (keep) {
        const int dst = a.block_counts[blockIdx.x] + r;
        a.out_particles[dst] = a.particles[j];
        if (a.radii) a.out_radii[dst] = a.radii[j];
    }
}

}  // namespace

int cull_aliased_terms(const SumRequest& in, float3 u, float3 v, float2 step, Workspace& ws, cudaStream_t stream,
                       SumRequest* out) {
    *out = in;
    if (in.n <= 0) return kOk;
    if (!(step.x > 0.f) || !(step.y > 0.f)) return set_error(kInvalidConfig, "aliasing cull: step_size must be > 0");
    const int blocks = (in.n + kCullThreads - 1) / kCullThreads;
    const size_t counts_bytes = ((size_t)(blocks + 1) * sizeof(int) + 255) / 256 * 256;
    const size_t part_bytes = ((size_t)in.n * sizeof(float4) + 255) / 256 * 256;
    const size_t radii_bytes = in.radii ? ((size_t)in.n * sizeof(float) + 255) / 256 * 256 : 0;
    int st = ws.reserve(counts_bytes + part_bytes + radii_bytes);
    if (st != kOk) return st;
    char* base = static_cast<char*>(ws.ptr);
    CullArgs a;
    a.particles = in.particles;
    a.radii = in.radii;
    a.n = in.n;
    a.u = u;
    a.v = v;
    a.box_x = 0.5f / step.x;
    a.box_y = 0.5f / step.y;
    a.block_counts = reinterpret_cast<int*>(base);
    a.out_particles = reinterpret_cast<float4*>(base + counts_bytes);
    a.out_radii = in.radii ? reinterpret_cast<float*>(base + counts_bytes + part_bytes) : nullptr;
    cull_count_kernel<<<blocks, kCullThreads, 0, stream>>>(a);
    count_launch();
    cull_scan_kernel<<<1, kCullThreads, 0, stream>>>(a.block_counts, blocks);
    count_launch();
    cull_scatter_kernel<<<blocks, kCullThreads, 0, stream>>>(a);
    count_launch();
    st = check_cuda(cudaGetLastError(), "aliasing cull launch");
    if (st != kOk) return st;
    int kept_n = 0;
    st = check_cuda(cudaMemcpyAsync(&kept_n, a.block_counts + blocks, sizeof(int), cudaMemcpyDeviceToHost, stream),
                    "aliasing cull count D2H");
    if (st == kOk) st = check_cuda(cudaStreamSynchronize(stream), "aliasing cull");
    if (st != kOk) return st;
    out->particles = a.out_particles;
    out->radii = a.out_radii;
    out->n = kept_n;
    return kOk;
}

}  // namespace mv
