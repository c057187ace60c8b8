// Internal host-side interfaces between the C API layer (mv_api.cu) and the
// kernel launchers (mv_sum.cu, mv_slice.cu).  Not part of the public ABI.
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace mv {

// Status of an internal call; mirrors enum VisError of meshless_vis_b200.h.
enum Status : int {
    kOk = 0,
    kInvalidValue = 1,
    kInvalidConfig = 2,
    kCudaError = 3,
    kCufftError = 4,
    kOutOfMemory = 5,
    kNotRegistered = 6,
    kUnsupported = 7,
    kNoKernel = 8,
};

// Records an error for vis_get_last_error() on this host thread; returns code.
int set_error(int code, const std::string& message);
// Maps a CUDA error to a Status and records it (kOk if err == cudaSuccess).
int check_cuda(cudaError_t err, const char* what);

// An integer lattice of wavenumbers n = (x, y, z), x in [x0, x0+nx), y in
// [y0, y0+ny), z in [z0, z0+nz).  Sum results are laid out x-major:
// element ((x - x0) * ny + (y - y0)) * nz + (z - z0)  ("lattice order").
struct Lattice {
    int x0, nx;
    int y0, ny;
    int z0, nz;
    // |k| = sqrt((kx x)^2 + (ky y)^2 + (kz z)^2), the argument scale of Phi^.
    double kx, ky, kz;
    // Phase in turns of particle p at n: n . (M p), M row-major 3x3.
    double m[9];
};

// Smoothing-length histogram of a registered group whose transform does not
// separate per axis (SPH, WENDLAND_D3_C2 with per-particle radii): kHBinFine
// log-spaced fine bins between the smallest and the largest radius, with the
// particle count and the largest |weight| of each.  Fine bin of radius h: the
// largest i with edge[i] <= h, clamped to [0, kHBinFine); host and device
// classify by the same float comparisons against the same edges, so counts
// taken at registration hold for the device's scatter at compute time.
constexpr int kHBinFine = 1024;
struct HBinStats {
    float h_min = 0.f, h_max = 0.f;
    std::vector<float> edges;  // kHBinFine + 1
    std::vector<int> count;    // kHBinFine
    std::vector<float> wmax;   // kHBinFine
    unsigned long long id = 0;  // hash of the content (plan cache key); equal data, equal id
};
std::vector<float> hbin_fine_edges(float h_min, float h_max);
int hbin_fine_index(const std::vector<float>& edges, float h);

// One group's Fourier sum over a lattice, written to `out` as
//   out[idx] (=|+=) scale * sum_j w_j Phi^(|k| h_j) exp(-2 pi i n.(M p_j))
// where idx = out_base + (x-x0) out_sx + (y-y0) out_sy + (z-z0) out_sz
// (wrap == 0) or, for the C2R slice layout,
// ((x < 0 ? x + wrap : x) * row + (y - y0)) with nz == 1.
struct SumRequest {
    const float4* particles;  // Constraint AoS
    const float* radii;       // nullptr: Phi^ evaluated at |k|
    float radius_min;         // smallest / largest radius and largest |weight|
    float radius_max;         //   when known (registration), else < 0
    float weight_max;
    const HBinStats* hbins;   // smoothing-length histogram (registration), or null
    int n;
    int basis;
    Lattice lat;
    double scale;
    float2* out;
    long long out_base, out_sx, out_sy, out_sz;
    int wrap;
    int row;
    bool accumulate;
    cudaStream_t stream;
    int* error_flag;  // device word set by kernels that give up a bounded wait
    // The branch part of an h-binned group (SPH / Wendland): kink = 1 sums
    // Phi^ minus its smooth closed form (nonzero below the branch point r0)
    // over particles sorted into shell_nbins h-bins (classification edges
    // shell_edges, first particles shell_first, both device arrays), at each
    // frequency k over the particles of the one bin that holds r0 / |k|.
    int kink;
    const float* shell_edges;
    const int* shell_first;
    int shell_nbins;
};

// Grow-only device scratch owned by one VisConfig.
struct Workspace {
    void* ptr = nullptr;
    size_t bytes = 0;
    int reserve(size_t need);  // Status
    void release();
};

struct KernelTimer;  // per-stage event pairs, see mv_api.cu

// Plain FP32 form.  Uses `ws` for split-K partial sums.
int launch_plain_sum(const SumRequest& req, Workspace& ws, KernelTimer* timer);

// Aliasing cull of the direct path (mv_cull.cu): `out` is `in` restricted to
// the particles whose footprint in the view (u, v) lies in [0, 1/(2 step.x)] x
// [0, 1/(2 step.y)], compacted in order into `ws`; waits for the kept count.
int cull_aliased_terms(const SumRequest& in, float3 u, float3 v, float2 step, Workspace& ws, cudaStream_t stream,
                       SumRequest* out);

// Slice extraction for a batch of views into the C2R layout
// [views][nx][ny/2+1].  views: device array of 8 floats per view
// (u.x, u.y, u.z, v.x, v.y, v.z, step.x, step.y).
struct SliceRequest {
    const float2* spectrum;
    int gx, gy, gz;  // full grid extents Kx, Ky, Kz
    float inv_step;  // 1 / spectral step
    const float* views;
    int number_of_views;
    int cx, cy;
    int nx, ny;
    float2* arranged;
    cudaStream_t stream;
};
int launch_slice_extract(const SliceRequest& req, KernelTimer* timer);

// One view of a batched slice extraction: its spectrum, its image parameters
// and where its C2R-layout slice goes.  Device-resident (96 bytes).
struct SliceView {
    const float2* spectrum;
    float2* arranged;          // float2[nx][ny/2+1]
    long long element_offset;  // prefix sum of nx*(ny/2+1) over the batch's views
    int gx, gy, gz;            // the spectrum's lattice extents
    float inv_step;            // 1 / spectral step
    float u[3], v[3];
    float step[2];
    int cx, cy, nx, ny;
    int pad;
};
// Slices of `number_of_views` views (descriptors in device memory) in one
// launch; total_elements = sum over views of nx*(ny/2+1).
int launch_slice_extract_batch(const SliceView* d_views, int number_of_views, long long total_elements,
                               cudaStream_t stream, KernelTimer* timer);

// Tensor-core form (mv_tc_sum.cu).  A set of groups -- of one or several
// half-spectra -- is summed by one persistent tcgen05 launch:
//   tensor_plan           host only: jobs, work items, output classes;
//   tensor_reserve_upload grows the workspaces and uploads the job and item
//                         tables (not capturable in a CUDA graph);
//   tensor_enqueue        per-particle constants, the persistent launch (each
//                         work item writes its totals into its slot), the FP64
//                         reduction of the slots into the spectra (added), the Nyquist
//                         planes of groups without a Nyquist job and the
//                         branch part of h-binned groups (plain form, added);
//                         stream-ordered and capturable once the workspaces
//                         are large enough.
// The spectra must be zeroed (or hold earlier groups) before tensor_enqueue.
// form: VIS_FORM_TENSOR or VIS_FORM_AUTO (h-binned groups only when cheaper).
int tensor_sum_available(const SumRequest& req, int form);

// One job of the persistent tensor-core kernel: a separable group summed over
// a lattice of rows (a, b) and columns c >= 0 into its work items' slots.  Its
// work items are (split ks, m tile, n tile), local index (ks * n_mtiles +
// m_tile) * n_ntiles + n_tile.  Device-resident.
//
// Frequencies: a = a_idx + a_base, b = b_idx + b_base, c = c_idx + c_base.
// A group's planes c < Kz/2 are one job (a_base = -Kx/2, b_base = -Ky/2,
// c_base = 0).  Its Nyquist plane c = Kz/2 is two transposed jobs over the
// same particles with x and z exchanged, so that their one row index a_idx = 0
// carries the frequency of z and their columns the frequencies of x:
//   a >= 0: a_base = Kz/2, rows b (b_base = -Ky/2), columns 0 .. Kx/2 - 1;
//   a < 0:  F(a, b, Kz/2) = conj F(-a, -b, -Kz/2), so a_base = -Kz/2, rows
//           b' = -b (b_base = 1 - Ky/2), columns -a = 1 .. Kx/2 (c_base = 1).
// Every column frequency is >= 0: the B chains only rise.
//
// B-operand images: where a job's B stages are read by many m-tiles, they are
// computed once (tc_bimg_kernel) into `bimg` in the exact swizzled layout of
// the stage buffer, [n_tile][CTA half][32-particle block][img_stride bytes],
// each image its hi rows then its lo rows (2 x 2 bnc rows of 128 bytes), and
// the loader copies them; otherwise (bimg null) producer warps compute them
// per stage.
struct TcJob {
    const unsigned char* blocks;  // the job's per-particle constants, 32-particle blocks
    // Item results: each work item owns slot [local item * slot_stride ..] of
    // `slots`: per CTA of the item (rank r at r * 128 * 2 nc_tile elements)
    // its 128 rows of every accumulator column n.  A job whose items span at
    // most 64 accumulation chains stores each item's FP32 total once, in
    // quads of columns ([n / 4][row][n % 4] floats); a job with longer items
    // (slot_fp64) adds the item's FP32 total of every 64 chains into FP64
    // totals, in pairs of columns ([n / 2][row][n % 2] doubles).
    // tc_reduce_kernel sums the slots over the items of every job in FP64.
    void* slots;
    int slot_stride;  // elements per item: ctas * 128 * 2 nc_tile
    int slot_fp64;
    int n_splits;     // particle chunks (items per tile)
    int ctas;         // 2 for the CTA-pair tiles
    double wmax;
    int kx, ky, lz_tc;  // row extents (a_idx < kx, b_idx < ky); columns c_idx < lz_tc
    int n_mtiles, n_ntiles;
    int n;        // particles
    int k_chunk;  // particles per item (multiple of 32)
    int gauss;    // per-particle Gaussian factors (GAUSSIAN_DECAYING with radii)
    int nc_tile;  // c values per n-tile (a multiple of 8; the last tile may be narrower)
    int a_base;   // frequency of row index a_idx = 0
    int b_base;   // frequency of row index b_idx = 0 (-Ky/2 or 1 - Ky/2: 8-row chunks never hold both signs)
    int c_base;   // frequency of column c_idx = 0 (>= 0)
    const unsigned char* bimg;  // B-operand images, or null
    int n_blocks;    // 32-particle blocks
    int img_stride;  // bytes per image: 512 x (c values per CTA of a full n-tile)
    // h-binned jobs (period > 0): the job's lz_tc = P x period columns are P
    // blocks of `period` frequency columns, block q weighted on the B side by
    // the Chebyshev polynomial T_q(t_j) of the particle's normalised radius t_j
    // in its bin (kept in the constants' gam field).  The reduction multiplies
    // block q's value at frequency column c by coef[(a^2 + b^2 + c^2) *
    // coef_stride + q], the q-th Chebyshev coefficient of h -> Phi^(|k| h)
    // over the bin (the group's table holds all its bins' q for one |k|^2
    // together).
    const float* coef;
    int period;
    int coef_stride;
    // the slot column of job column c (tc_reduce_kernel): (n-tile, Re column,
    // Im column, 0) per column
    const int4* colmap;
    // Row-folded jobs (fold = F > 1; separable groups without per-particle
    // Gaussian factors, whose terms are pure phases): the spectrum's b axis
    // is split as b = F bh + bl + b_base, job rows (a, bh) (ky = Ky / F of
    // them per a) and job columns bl * period + c_idx (period = the planes).
    // The A operand carries the phase of F bh + b_base, B that of bl and c,
    // so F planes' worth of columns share every A row: more columns per MMA
    // (N = 256 instead of 64 or 128 on small lattices) and less A work per
    // term.  0 or 1: no fold.
    int fold;
    // Axis-exchanged jobs (exch = 1; groups whose amplitudes separate per
    // axis, on lattices with more b values than tensor planes): rows (a,
    // c_idx) with ky = the planes Kz/2 and b_base = 0, columns b_idx with
    // lz_tc = Ky and c_base = -Ky/2 (B chains of negative b fall away from
    // 0); the particle constants carry y and z exchanged.  192 planes with
    // Ky = 384 then run 3 n-tiles of 128 b values (N = 256 MMAs) instead of
    // two of 96 planes.
    int exch;
};

// The h-bins of one binned group on one lattice (tensor_plan): consecutive
// runs of fine bins, each with its Chebyshev order and weight scale.
struct HBin {
    int f0, f1;      // fine bins [f0, f1)
    float lo, hi;    // radius interval (fine edges f0, f1)
    int count;       // particles
    float wmax;      // largest |weight|
    int order;       // Chebyshev nodes P
};
struct HBinPlan {
    std::vector<HBin> bins;
    double cost = 0.0;      // sum over bins of count x order, per particle
    bool feasible = true;   // false: some radii need more Chebyshev nodes than a bin may have
};

struct TensorPlan {
    // A binned group's device tables, uploaded with the job table: bin edges
    // (nbins + 1 floats), then per bin int4 (first block, count, coef offset,
    // order) and float2 (2^12 / W, Chebyshev node scale), then the counters
    // the scatter uses (in the accumulator workspace, zeroed per compute).
    struct Binned {
        int group;
        int nbins;
        size_t meta_offset;     // edges, then int4 bin table, then float2 bin scales
        size_t coef_offset;     // into coef (floats)
        size_t coef_count;
        int nsq;                // |k|^2 / step^2 values: max a^2 + b^2 + c^2 + 1
        int total_q;            // Chebyshev blocks over all bins: the table's stride per |k|^2
        std::vector<HBin> bins;
        std::vector<float> edges;  // nbins + 1: the fine edges where the bins start (classification)
        size_t sorted_offset;      // into TensorWorkspace::sorted: n float4, n radii, then the radius sort's
                                   // keys and indices (in, out) and temporary storage (256-aligned)
        size_t sort_temp_bytes;
    };
    size_t sorted_bytes = 0;
    std::vector<Binned> binned;
    size_t coef_bytes = 0;
    struct Class {
        float2* out;
        int kx, ky, lz_tc, lz_out;
        double step;
        int basis;
        double h;
        bool factored;
        double scale;
        bool nyquist;  // the Nyquist plane is summed by the groups' transposed jobs
        // the class's jobs (indices into jobs): planes, Nyquist a >= 0, Nyquist a < 0
        std::vector<int> jobs, nyq_pos, nyq_neg;
        size_t list_offset = 0;  // those three lists in meta (ints)
    };
    std::vector<TcJob> jobs;
    std::vector<int2> items;  // 128x128-tile items (n_narrow), narrow CTA-pair items (n_pair_narrow),
                              // CTA-pair items (n_pair), then 128x256
    int n_narrow = 0, n_pair_narrow = 0, n_pair = 0, n_pair_db = 0;
    std::vector<Class> classes;
    std::vector<int> group_class, job_of_group;
    std::vector<int> nyq_job_of_group;  // the transposed Nyquist-plane jobs (a >= 0 here, a < 0 next), or -1
    std::vector<int> group_binned;      // index into binned, or -1
    // per job: its particle constants (offset into the particles workspace),
    // accumulator class and part (0 planes, 1 Nyquist a >= 0, 2 Nyquist a < 0),
    // coefficient table (offset in floats into coef, SIZE_MAX for none)
    std::vector<size_t> job_tp, job_coef, job_slot;  // job_slot: byte offset into slots
    std::vector<size_t> job_colmap;                 // the job's column map: index into colmaps
    std::vector<int4> colmaps;                      // all jobs' column maps
    size_t colmap_offset = 0;                       // colmaps in meta
    std::vector<int> img_jobs;                      // the jobs with B-operand images
    std::vector<long long> img_first;               // their first images (and the total last)
    size_t img_jobs_offset = 0, img_first_offset = 0;  // both in meta
    std::vector<int> job_class, job_acc;
    size_t slot_bytes = 0;
    std::vector<size_t> tp_offset, tp_nyq_offset;
    std::vector<size_t> bimg_offset;  // per job: its B-operand images in the workspace, or SIZE_MAX
    size_t bimg_bytes = 0;
    size_t tp_bytes = 0, meta_bytes = 0;
    const void* d_jobs = nullptr;
    const void* d_items = nullptr;
    int flush = 16;        // stages per TMEM accumulation chain of the kWide / kPair tiles, as planned
    int flush_narrow = 8;  // the same for the kNarrow tile
};

struct TensorWorkspace {
    Workspace particles;  // per-particle constants of every group
    Workspace slots;      // work items' totals (FP32 or FP64)
    Workspace meta;       // job and item tables
    Workspace bimg;       // B-operand images
    Workspace coef;       // Chebyshev coefficient tables of h-binned groups
    Workspace sorted;     // h-binned groups' particles and radii sorted by bin
    std::vector<char> uploaded;  // the tables last copied to `meta`
    void* uploaded_to = nullptr;
    // the last plan made here (tensor_prepare), uploaded, and what it was made of
    std::string plan_key;
    std::unique_ptr<TensorPlan> plan;
    void release() {
        uploaded.clear();
        uploaded_to = nullptr;
        plan_key.clear();
        plan.reset();
        particles.release();
        slots.release();
        meta.release();
        bimg.release();
        coef.release();
        sorted.release();
    }
};

int tensor_plan(const std::vector<SumRequest>& groups, TensorPlan& plan);

// Device memory the B-operand images of one plan may take: the limit set with
// vis_set_operand_cache_limit (or MV_TC_OPERAND_CACHE_MB), by default three
// eighths of the current device's memory.
size_t operand_cache_limit();
int tensor_reserve_upload(TensorPlan& plan, TensorWorkspace& ws, cudaStream_t stream);
// tensor_plan + tensor_reserve_upload, skipped when the groups, the launch
// parameters in force and the device are those of the workspace's last plan
// (a compute repeated on the same registered data); *plan points into ws.
int tensor_prepare(const std::vector<SumRequest>& groups, TensorWorkspace& ws, cudaStream_t stream,
                   const TensorPlan** plan);
int tensor_enqueue(const std::vector<SumRequest>& groups, const TensorPlan& plan, TensorWorkspace& ws,
                   Workspace& plain_ws, KernelTimer* timer, cudaStream_t stream, int* error_flag);

// Per-stage timing hooks (no-ops when timer == nullptr or disabled).
void timer_begin(KernelTimer* timer, int stage, cudaStream_t stream);
void timer_end(KernelTimer* timer, int stage, cudaStream_t stream);

int device_sm_count();

// Tile shapes of the tensor form the planner may use; mirrors the VIS_TILE_*
// bits of meshless_vis_b200.h.
enum TileShape : int {
    kTileRowFold = 1,
    kTileAxisExchange = 2,
    kTileDoubleBuffer = 4,
    kTileCtaPairs = 8,
    kTileAll = 15,
};

// Launch parameters chosen per workload shape by the autotuner
// (vis_autotune_spectrum, mv_tune.cu); defaults otherwise.  Only parameters
// that leave results within tolerance are tuned.
struct TuneParams {
    int plain_waves = 6;  // plain form: split-K until the grid holds ~plain_waves blocks per SM
    int tc_waves = 4;     // tensor form: particle splits until the items make ~tc_waves waves
    int tc_flush = 16;    // tensor form, single-accumulator tiles: stages per TMEM chain (8 or 16;
                          // the double-buffered 128x128 tile uses at most 8)
    int hbin_job_cost = 1024;  // h-binned groups: cost of one more bin (a job), in particle x n-tile units
    int hbin_block_cost = 0;  // h-binned groups: cost of one more Chebyshev block (the reduction), same units
    int tc_shapes = kTileAll;  // tensor form: the tile shapes the planner may use (TileShape bits)
};
// The parameters in force on this thread: set by TuneScope around a compute.
const TuneParams& active_tune();
struct TuneScope {
    explicit TuneScope(const TuneParams& p);
    ~TuneScope();
    TuneParams saved;
};
// The table entry for a spectrum shape, or the defaults.
TuneParams tuned_params(int kx, int ky, int kz, long long n_total, int n_groups, int form);

// Statistics of a registered group, recorded by vis_register_meshless_dataset
// and keyed by the group's device particle pointer; all -1 if unknown.
struct GroupStats {
    float radius_min = -1.f, radius_max = -1.f, weight_max = -1.f;
    std::shared_ptr<const HBinStats> hbins;  // SPH / Wendland groups with varying radii
};
GroupStats registered_group_stats(const void* d_constraints);

// Counts a launch of one of this library's kernels (vis_kernel_launch_count).
void count_launch();

}  // namespace mv
