// C API of the drop-in: include/meshless_vis.h (the reference's
// meshless_vis/meshless_vis.cu:129-364 interface) and the additions of
// include/meshless_vis_b200.h.
//
// Host-side design:
//   - VisConfig keeps the reference's public layout; everything new (stream,
//     split-K workspace, batched cuFFT plans, timing events) lives in a side
//     table keyed by the VisConfig pointer.
//   - Every call validates its arguments, never exits, records failures in a
//     thread-local error (vis_get_last_error) and returns early.
//   - All device work of a config is stream-ordered on its stream; only
//     vis_copy_to_host, vis_spectrum_copy_to_host, registration and the
//     host-image variant of vis_spectrum_render_views wait for it.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include <cufft.h>

#include "meshless_vis_b200.h"
#include "mv_internal.h"

namespace mv {

// ------------------------------------------------------------------ errors
namespace {
thread_local int t_last_error = kOk;
thread_local std::string t_last_message;
}  // namespace

int set_error(int code, const std::string& message) {
    t_last_error = code;
    t_last_message = message;
    return code;
}

int check_cuda(cudaError_t err, const char* what) {
    if (err == cudaSuccess) return kOk;
    const int code = (err == cudaErrorMemoryAllocation) ? kOutOfMemory
                     : (err == cudaErrorNoKernelImageForDevice || err == cudaErrorInvalidDeviceFunction) ? kNoKernel
                                                                                                        : kCudaError;
    return set_error(code, std::string(what) + ": " + cudaGetErrorString(err));
}

static int check_cufft(cufftResult r, const char* what) {
    if (r == CUFFT_SUCCESS) return kOk;
    return set_error(r == CUFFT_ALLOC_FAILED ? kOutOfMemory : kCufftError,
                     std::string(what) + ": cuFFT error " + std::to_string((int)r));
}

int device_sm_count() {
    static std::mutex mu;
    static std::map<int, int> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(dev);
    if (it != cache.end()) return it->second;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    cache[dev] = sms;
    return sms;
}

namespace {
std::atomic<unsigned long long> g_launches{0};
std::mutex g_stats_mu;
std::unordered_map<const void*, GroupStats> g_stats;
}  // namespace
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

GroupStats registered_group_stats(const void* d_constraints) {
    if (!d_constraints) return GroupStats{};
    std::lock_guard<std::mutex> lock(g_stats_mu);
    auto it = g_stats.find(d_constraints);
    return it == g_stats.end() ? GroupStats{} : it->second;
}

// kHBinFine + 1 log-spaced edges from h_min to h_max, as floats: the same
// computation every time for the same (h_min, h_max).
std::vector<float> hbin_fine_edges(float h_min, float h_max) {
    std::vector<float> e(kHBinFine + 1);
    const double l0 = std::log((double)h_min), l1 = std::log((double)h_max);
    for (int i = 0; i <= kHBinFine; ++i) e[i] = (float)std::exp(l0 + (l1 - l0) * (double)i / kHBinFine);
    return e;
}

// Largest i with edges[i] <= h, clamped to [0, kHBinFine) (float comparisons
// only: the device scatter classifies the same way against the same floats).
int hbin_fine_index(const std::vector<float>& edges, float h) {
    int lo = 0, hi = kHBinFine;  // edges[lo] <= h < edges[hi] once narrowed
    if (!(h >= edges[1])) return 0;
    if (h >= edges[kHBinFine - 1]) return kHBinFine - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (edges[mid] <= h) lo = mid;
        else hi = mid;
    }
    return lo;
}

namespace {

// Runs fn(part, begin, end) over [0, n) in contiguous ranges, one per host
// thread (up to 16; the calling thread takes part 0), and returns the number
// of parts.  Below 2^16 items, or when no thread can be started, one part
// runs inline.  The registration's statistics are order-independent maxima,
// minima and counts, so the parts' results combine to the serial ones.
template <typename F>
int parallel_parts(long long n, int max_parts, F fn) {
    int parts = 1;
    if (n >= (1LL << 16)) {
        const unsigned hw = std::thread::hardware_concurrency();
        parts = (int)std::min<long long>(std::min<unsigned>(hw ? hw : 1, 16u), n >> 15);
        parts = std::max(1, std::min(parts, max_parts));
    }
    std::vector<std::thread> threads;
    int started = 1;
    auto range = [&](int p) { return std::make_pair(n * p / parts, n * (p + 1) / parts); };
    for (int p = 1; p < parts; ++p) {
        try {
            threads.emplace_back([&fn, p, range] { fn(p, range(p).first, range(p).second); });
            ++started;
        } catch (...) {
            break;
        }
    }
    // parts no thread took run here, after part 0
    fn(0, range(0).first, range(0).second);
    for (int p = started; p < parts; ++p) fn(p, range(p).first, range(p).second);
    for (std::thread& t : threads) t.join();
    return parts;
}

// hbin_fine_index for many radii against the same edges: a guess from the
// logarithm, then float comparisons against the edges up and down to the
// largest i with edges[i] <= h, so the result is the binary search's exactly
// (about 3.5x faster on 262,144 radii: registration cost per frame).
struct FineIndex {
    const float* e;
    double l0, inv;
    explicit FineIndex(const std::vector<float>& edges) : e(edges.data()) {
        l0 = std::log((double)edges[0]);
        inv = kHBinFine / (std::log((double)edges[kHBinFine]) - l0);
    }
    int operator()(float h) const {
        if (!(h >= e[1])) return 0;
        if (h >= e[kHBinFine - 1]) return kHBinFine - 1;
        // e[1] <= h < e[kHBinFine - 1]: the answer is in [1, kHBinFine - 2]
        const double t = (std::log((double)h) - l0) * inv;  // NaN or inf fall to the clamp
        int f = t > 1.0 ? (t < kHBinFine - 2 ? (int)t : kHBinFine - 2) : 1;
        while (e[f + 1] <= h) ++f;
        while (e[f] > h) --f;
        return f;
    }
};

// The smoothing-length histogram of a group whose Phi^ does not separate per
// axis (SPH, WENDLAND_D3_C2) with varying radii; null otherwise.
std::shared_ptr<const HBinStats> hbin_histogram(const Group& grp, const GroupStats& gs) {
    const int b = (int)grp.basis_function_id;
    if (!grp.h_radii || grp.number_of_terms <= 0 || (b != (int)SPH && b != (int)WENDLAND_D3_C2)) return nullptr;
    if (!(gs.radius_min > 0.f) || !(gs.radius_max > gs.radius_min) || !std::isfinite(gs.radius_max)) return nullptr;
    auto hs = std::make_shared<HBinStats>();
    hs->h_min = gs.radius_min;
    hs->h_max = gs.radius_max;
    hs->edges = hbin_fine_edges(gs.radius_min, gs.radius_max);
    hs->count.assign(kHBinFine, 0);
    hs->wmax.assign(kHBinFine, 0.f);
    const FineIndex fine(hs->edges);
    constexpr int kMaxParts = 16;
    std::vector<std::vector<int>> count(kMaxParts);
    std::vector<std::vector<float>> wmax(kMaxParts);
    const int parts = parallel_parts(grp.number_of_terms, kMaxParts, [&](int p, long long b, long long e) {
        count[p].assign(kHBinFine, 0);
        wmax[p].assign(kHBinFine, 0.f);
        for (long long k = b; k < e; ++k) {
            const int f = fine(grp.h_radii[k]);
            count[p][f] += 1;
            wmax[p][f] = std::max(wmax[p][f], std::fabs(grp.h_constraints[k].weight));
        }
    });
    for (int p = 0; p < parts; ++p)
        for (int f = 0; f < kHBinFine; ++f) {
            hs->count[f] += count[p][f];
            hs->wmax[f] = std::max(hs->wmax[f], wmax[p][f]);
        }
    // the id names the content (plans are cached by it): FNV-1a of the range,
    // the counts and the weight maxima, never 0
    uint64_t h = 1469598103934665603ull;
    auto mix = [&h](const void* p, size_t n) {
        const unsigned char* c = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < n; ++i) h = (h ^ c[i]) * 1099511628211ull;
    };
    mix(&hs->h_min, sizeof(float));
    mix(&hs->h_max, sizeof(float));
    mix(hs->count.data(), hs->count.size() * sizeof(int));
    mix(hs->wmax.data(), hs->wmax.size() * sizeof(float));
    hs->id = h ? h : 1;
    return hs;
}
}  // namespace

// ------------------------------------------------------ registration pool
// Registered particle arrays come from a stream-ordered memory pool of the
// library's own, one per device, that keeps freed blocks (release threshold
// unlimited): a register / unregister cycle per frame then reuses device
// memory instead of mapping and unmapping it each time, which made cudaMalloc
// and cudaFree of the same sizes take from under 1 ms to tens of ms.
namespace {
std::mutex g_pool_mu;
std::map<int, cudaMemPool_t> g_pools;

int registration_pool(cudaMemPool_t* pool) {
    int dev = 0;
    int st = check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (st != kOk) return st;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    auto it = g_pools.find(dev);
    if (it != g_pools.end()) {
        *pool = it->second;
        return kOk;
    }
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    st = check_cuda(cudaMemPoolCreate(pool, &props), "cudaMemPoolCreate");
    if (st != kOk) return st;
    uint64_t keep = UINT64_MAX;
    st = check_cuda(cudaMemPoolSetAttribute(*pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
    if (st != kOk) return st;
    g_pools[dev] = *pool;
    return kOk;
}

}  // namespace

// Device blocks of unregistered particle arrays, kept per config for the next
// registration of the same byte size, first in first out: a register /
// unregister cycle per frame of the same datasets in the same order then gets
// back the same device addresses, so a batch of them replays its CUDA graph
// instead of running, capturing and instantiating it again (which the pool's
// own reuse order did not guarantee).  The blocks held plus those registered
// never exceed the most this config had registered at once; the rest go back
// to the pool, and vis_config_destroy returns them all.
struct RegistrationCache {
    std::map<size_t, std::deque<void*>> blocks;
    size_t held = 0, live = 0, peak = 0;

    void* take(size_t bytes) {
        auto it = blocks.find(bytes);
        if (it == blocks.end()) return nullptr;
        void* p = it->second.front();
        it->second.pop_front();
        if (it->second.empty()) blocks.erase(it);
        held -= bytes;
        return p;
    }
    // returns held blocks to the pool, largest first, until held + live <= peak
    void trim(cudaStream_t stream) {
        while (held > 0 && held + live > peak) {
            auto it = std::prev(blocks.end());
            cudaFreeAsync(it->second.front(), stream);
            held -= it->first;
            it->second.pop_front();
            if (it->second.empty()) blocks.erase(it);
        }
    }
    void registered(size_t bytes, cudaStream_t stream) {
        live += bytes;
        peak = std::max(peak, live);
        trim(stream);
    }
    void unregistered(void* p, size_t bytes, cudaStream_t stream) {
        live = live >= bytes ? live - bytes : 0;
        blocks[bytes].push_back(p);
        held += bytes;
        trim(stream);
    }
    void release(cudaStream_t stream) {
        for (auto& kv : blocks)
            for (void* p : kv.second) cudaFreeAsync(p, stream);
        blocks.clear();
        held = live = peak = 0;
    }
};

namespace {
template <typename T>
int registration_alloc(T** p, size_t count, RegistrationCache& cache, cudaStream_t stream) {
    *p = nullptr;
    if (count == 0) return kOk;
    const size_t bytes = sizeof(T) * count;
    if (void* q = cache.take(bytes)) {
        *p = static_cast<T*>(q);
        cache.registered(bytes, stream);
        return kOk;
    }
    cudaMemPool_t pool;
    int st = registration_pool(&pool);
    if (st != kOk) return st;
    cudaError_t e = cudaMallocFromPoolAsync((void**)p, bytes, pool, stream);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return check_cuda(e, "cudaMallocFromPoolAsync");
    }
    cache.registered(bytes, stream);
    return kOk;
}
}  // namespace

// --------------------------------------------------------------- workspace
int Workspace::reserve(size_t need) {
    if (need <= bytes) return kOk;
    if (ptr) {
        // The buffer may still be read by earlier launches on any stream.
        cudaDeviceSynchronize();
        cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    const size_t grow = std::max(need, (size_t)1 << 20);
    cudaError_t e = cudaMalloc(&ptr, grow);
    if (e != cudaSuccess) {
        ptr = nullptr;
        cudaGetLastError();
        return check_cuda(e, "workspace cudaMalloc");
    }
    bytes = grow;
    return kOk;
}

void Workspace::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

// ------------------------------------------------------------------ timing
struct KernelTimer {
    bool enabled = false;
    static constexpr int kStagesTimed = 4;
    cudaEvent_t open[kStagesTimed] = {nullptr, nullptr, nullptr, nullptr};
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> done[kStagesTimed];
    std::vector<cudaEvent_t> pool;

    cudaEvent_t take() {
        cudaEvent_t e = nullptr;
        if (!pool.empty()) {
            e = pool.back();
            pool.pop_back();
        } else if (cudaEventCreate(&e) != cudaSuccess) {
            e = nullptr;
        }
        return e;
    }
    void clear_stage(int s) {
        for (auto& p : done[s]) {
            pool.push_back(p.first);
            pool.push_back(p.second);
        }
        done[s].clear();
    }
    ~KernelTimer() {
        for (int s = 0; s < kStagesTimed; ++s) {
            clear_stage(s);
            if (open[s]) pool.push_back(open[s]);
        }
        for (auto e : pool) cudaEventDestroy(e);
    }
};

void timer_begin(KernelTimer* t, int stage, cudaStream_t stream) {
    if (!t || !t->enabled) return;
    cudaEvent_t e = t->take();
    if (!e) return;
    cudaEventRecord(e, stream);
    if (t->open[stage]) t->pool.push_back(t->open[stage]);
    t->open[stage] = e;
}

void timer_end(KernelTimer* t, int stage, cudaStream_t stream) {
    if (!t || !t->enabled || !t->open[stage]) return;
    cudaEvent_t e = t->take();
    if (!e) return;
    cudaEventRecord(e, stream);
    t->done[stage].emplace_back(t->open[stage], e);
    t->open[stage] = nullptr;
}

// ------------------------------------------------------------- config state
struct ConfigState {
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    Workspace partials;  // split-K partial sums
    Workspace arranged;  // batched C2R inputs of vis_spectrum_render_views
    Workspace images;    // library-owned batched images
    Workspace views;     // per-view parameters
    TensorWorkspace tensor;  // tensor-core form: particle constants, FP64 accumulators, tables
    Workspace post;          // image post-processing (per-image maxima)
    Workspace error_word;  // device int set by kernels that give up a bounded wait
    Workspace cull;        // kept particles of the aliasing cull
    std::map<std::tuple<int, int, int>, cufftHandle> batched_plans;
    KernelTimer timer;
    RegistrationCache registrations;  // blocks of unregistered datasets, for the next registration

    ~ConfigState() {
        if (stream) cudaStreamSynchronize(stream);
        registrations.release(stream);
        if (stream) cudaStreamSynchronize(stream);
        partials.release();
        arranged.release();
        images.release();
        views.release();
        tensor.release();
        post.release();
        error_word.release();
        cull.release();
        for (auto& kv : batched_plans) cufftDestroy(kv.second);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }
};

namespace {
std::mutex g_mu;
std::unordered_map<const VisConfig*, ConfigState*> g_states;

ConfigState* state_of(const VisConfig* cfg) {
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_states.find(cfg);
    return it == g_states.end() ? nullptr : it->second;
}

bool valid_config(const VisConfig* c, std::string* why) {
    // meshless_vis/meshless_vis.cu:191-210
    auto fail = [&](const char* m) {
        if (why) *why = m;
        return false;
    };
    if (c->block_length < 64) return fail("block_length < 64");
    if (c->block_length < 32) return fail("block_length < warp size");
    if (c->block_length > 1024) return fail("block_length > max threads per block");
    if (c->_cutoff_frequency.x < 0 || c->_cutoff_frequency.y < 0) return fail("negative cutoff frequency");
    if ((2LL * c->_cutoff_frequency.x * c->_cutoff_frequency.y) % c->block_length) return fail("2*cx*cy is not a multiple of block_length");
    if (2 * c->_cutoff_frequency.x > c->_number_of_samples.x) return fail("2*cutoff.x > number_of_samples.x");
    if (2 * c->_cutoff_frequency.y > c->_number_of_samples.y) return fail("2*cutoff.y > number_of_samples.y");
    if (c->_number_of_partial_sums < 1) return fail("number_of_partial_sums < 1");
    return true;
}

template <typename T>
int device_alloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) return kOk;
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * count);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return check_cuda(e, "cudaMalloc");
    }
    return kOk;
}

size_t freq_image_count(const VisConfig* c) {
    return 2ULL * std::max(0, c->_cutoff_frequency.x) * std::max(0, c->_cutoff_frequency.y) *
           std::max(1, c->_number_of_partial_sums);
}
size_t arranged_count(const VisConfig* c) {
    return (size_t)std::max(0, c->_number_of_samples.x) * (std::max(0, c->_number_of_samples.y) / 2 + 1);
}
size_t image_count(const VisConfig* c) {
    return (size_t)std::max(0, c->_number_of_samples.x) * std::max(0, c->_number_of_samples.y);
}

int make_plan(VisConfig* c) {
    c->_plan = 0;
    if (c->_number_of_samples.x < 1 || c->_number_of_samples.y < 2) return kOk;
    return check_cufft(cufftPlan2d(&c->_plan, c->_number_of_samples.x, c->_number_of_samples.y, CUFFT_C2R),
                       "cufftPlan2d");
}

}  // namespace

}  // namespace mv

using namespace mv;

// ====================================================================== C ABI
extern "C" {

int vis_get_last_error(void) { return t_last_error; }
const char* vis_get_last_error_message(void) { return t_last_message.c_str(); }
void vis_clear_last_error(void) {
    t_last_error = kOk;
    t_last_message.clear();
}
const char* vis_get_error_string(int code) {
    switch (code) {
    case VIS_SUCCESS: return "success";
    case VIS_ERROR_INVALID_VALUE: return "invalid value";
    case VIS_ERROR_INVALID_CONFIG: return "invalid configuration";
    case VIS_ERROR_CUDA: return "CUDA error";
    case VIS_ERROR_CUFFT: return "cuFFT error";
    case VIS_ERROR_OUT_OF_MEMORY: return "out of device memory";
    case VIS_ERROR_NOT_REGISTERED: return "dataset not registered";
    case VIS_ERROR_UNSUPPORTED: return "unsupported";
    case VIS_ERROR_NO_KERNEL: return "no kernel image for this device";
    default: return "unknown error";
    }
}

// meshless_vis/meshless_vis.cu:129-176 (device-property printout dropped).
VisConfig* vis_config_create(bool automatic_d_image, float2 step_size, int2 cutoff_frequency, float3 u_axis,
                             float3 v_axis, int2 number_of_samples, int block_length, int number_of_partial_sums) {
    if (cutoff_frequency.x < 0 || cutoff_frequency.y < 0 || number_of_samples.x < 1 || number_of_samples.y < 2) {
        set_error(kInvalidValue, "vis_config_create: cutoff must be >= 0 and number_of_samples >= (1, 2)");
        return nullptr;
    }
    VisConfig* c = (VisConfig*)std::calloc(1, sizeof(VisConfig));
    if (!c) {
        set_error(kOutOfMemory, "vis_config_create: host allocation failed");
        return nullptr;
    }
    c->step_size = step_size;
    c->u_axis = u_axis;
    c->v_axis = v_axis;
    c->cull_fully_aliased_terms = false;
    c->_number_of_samples = number_of_samples;
    c->_cutoff_frequency = cutoff_frequency;
    c->block_length = block_length;
    c->_number_of_partial_sums = number_of_partial_sums;
    c->_automatic_d_image = automatic_d_image;
    c->_scale = step_size.x * step_size.y;

    ConfigState* s = new ConfigState();
    int st = check_cuda(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    s->own_stream = st == kOk;
    if (st == kOk) st = s->error_word.reserve(256);
    if (st == kOk) st = check_cuda(cudaMemset(s->error_word.ptr, 0, 256), "cudaMemset");
    if (st == kOk) st = device_alloc(&c->_d_freq_image, freq_image_count(c));
    if (st == kOk) st = device_alloc(&c->_d_freq_image_arranged, arranged_count(c));
    if (st == kOk && automatic_d_image) st = device_alloc(&c->_d_image, image_count(c));
    if (st == kOk) st = make_plan(c);
    if (st != kOk) {
        cudaFree(c->_d_freq_image);
        cudaFree(c->_d_freq_image_arranged);
        if (automatic_d_image) cudaFree(c->_d_image);
        if (c->_plan) cufftDestroy(c->_plan);
        delete s;
        std::free(c);
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    g_states[c] = s;
    return c;
}

// meshless_vis/meshless_vis.cu:178-189 (the CUDA build's defaults).
VisConfig* vis_config_get_default(void) {
    return vis_config_create(true, make_float2(0.1f, 0.1f), make_int2(128, 128), make_float3(1.f, 0.f, 0.f),
                             make_float3(0.f, 1.f, 0.f), make_int2(512, 512), 256, 1);
}

bool vis_config_check(VisConfig* vis_config) {
    if (!vis_config) {
        set_error(kInvalidValue, "vis_config_check: NULL config");
        return false;
    }
    return valid_config(vis_config, nullptr);
}

// The reference overwrites _d_image (meshless_vis/meshless_vis.cu:244-247) and
// would later cudaFree the caller's buffer in vis_config_destroy; here an owned
// image is released first and the caller keeps ownership of theirs.
void vis_config_manual_d_image(VisConfig* vis_config, void* d_image) {
    if (!vis_config) {
        set_error(kInvalidValue, "vis_config_manual_d_image: NULL config");
        return;
    }
    if (vis_config->_automatic_d_image && vis_config->_d_image) {
        ConfigState* s = state_of(vis_config);
        if (s) cudaStreamSynchronize(s->stream);
        cudaFree(vis_config->_d_image);
    }
    vis_config->_automatic_d_image = false;
    vis_config->_d_image = static_cast<float*>(d_image);
}

// meshless_vis/meshless_vis.cu:212-227
void vis_config_change_number_of_samples(VisConfig* c, int2 number_of_samples) {
    if (!c || number_of_samples.x < 1 || number_of_samples.y < 2) {
        set_error(kInvalidValue, "vis_config_change_number_of_samples: bad arguments");
        return;
    }
    ConfigState* s = state_of(c);
    if (s) cudaStreamSynchronize(s->stream);
    c->_number_of_samples = number_of_samples;
    if (c->_automatic_d_image) {
        cudaFree(c->_d_image);
        if (device_alloc(&c->_d_image, image_count(c)) != kOk) return;
    }
    cudaFree(c->_d_freq_image_arranged);
    if (device_alloc(&c->_d_freq_image_arranged, arranged_count(c)) != kOk) return;
    if (c->_plan) cufftDestroy(c->_plan);
    make_plan(c);
}

// meshless_vis/meshless_vis.cu:229-234
void vis_config_change_cutoff_frequency(VisConfig* c, int2 cutoff_frequency) {
    if (!c || cutoff_frequency.x < 0 || cutoff_frequency.y < 0) {
        set_error(kInvalidValue, "vis_config_change_cutoff_frequency: bad arguments");
        return;
    }
    ConfigState* s = state_of(c);
    if (s) cudaStreamSynchronize(s->stream);
    c->_cutoff_frequency = cutoff_frequency;
    cudaFree(c->_d_freq_image);
    device_alloc(&c->_d_freq_image, freq_image_count(c));
}

// meshless_vis/meshless_vis.cu:236-242
void vis_config_change_number_of_partial_sums(VisConfig* c, int number_of_partial_sums) {
    if (!c) {
        set_error(kInvalidValue, "vis_config_change_number_of_partial_sums: NULL config");
        return;
    }
    ConfigState* s = state_of(c);
    if (s) cudaStreamSynchronize(s->stream);
    c->_number_of_partial_sums = number_of_partial_sums;
    cudaFree(c->_d_freq_image);
    device_alloc(&c->_d_freq_image, freq_image_count(c));
}

// meshless_vis/meshless_vis.cu:249-256
void vis_config_destroy(VisConfig* c) {
    if (!c) return;
    ConfigState* s = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        auto it = g_states.find(c);
        if (it != g_states.end()) {
            s = it->second;
            g_states.erase(it);
        }
    }
    delete s;  // waits for the stream
    if (c->_automatic_d_image) cudaFree(c->_d_image);
    cudaFree(c->_d_freq_image_arranged);
    cudaFree(c->_d_freq_image);
    if (c->_plan) cufftDestroy(c->_plan);
    std::free(c);
}

// meshless_vis/meshless_vis.cu:258-262
void vis_config_compute_scale(VisConfig* c) {
    if (!c) {
        set_error(kInvalidValue, "vis_config_compute_scale: NULL config");
        return;
    }
    c->_scale = c->step_size.x * c->step_size.y;
}

int vis_config_set_stream(VisConfig* c, cudaStream_t stream) {
    ConfigState* s = c ? state_of(c) : nullptr;
    if (!s) return set_error(kInvalidValue, "vis_config_set_stream: unknown config");
    cudaStreamSynchronize(s->stream);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    s->own_stream = false;
    s->stream = stream;
    return kOk;
}

cudaStream_t vis_config_get_stream(VisConfig* c) {
    ConfigState* s = c ? state_of(c) : nullptr;
    if (!s) {
        set_error(kInvalidValue, "vis_config_get_stream: unknown config");
        return nullptr;
    }
    return s->stream;
}

// Waits for the config's stream and reports a kernel that gave up one of its
// bounded waits (the word is cleared once reported).
static int sync_and_check(ConfigState* s, const char* what) {
    int rc = check_cuda(cudaStreamSynchronize(s->stream), what);
    if (rc != kOk) return rc;
    int word = 0;
    rc = check_cuda(cudaMemcpy(&word, s->error_word.ptr, sizeof(int), cudaMemcpyDeviceToHost), what);
    if (rc != kOk) return rc;
    if (word != 0) {
        cudaMemset(s->error_word.ptr, 0, sizeof(int));
        return set_error(kCudaError, std::string(what) + ": a tensor-core kernel timed out in a bounded wait (code " +
                                         std::to_string(word) + "); its results are invalid");
    }
    return kOk;
}

int vis_config_synchronize(VisConfig* c) {
    ConfigState* s = c ? state_of(c) : nullptr;
    if (!s) return set_error(kInvalidValue, "vis_config_synchronize: unknown config");
    return sync_and_check(s, "vis_config_synchronize");
}

// meshless_vis/meshless_vis.cu:264-290: device copies padded with zeros to a
// multiple of number_of_partial_sums * block_length (d_number_of_terms).
void vis_register_meshless_dataset(VisConfig* c, MeshlessDataset* ds) {
    ConfigState* s = c ? state_of(c) : nullptr;
    if (!s || !ds || (ds->number_of_groups > 0 && !ds->groups)) {
        set_error(kInvalidValue, "vis_register_meshless_dataset: NULL or unknown argument");
        return;
    }
    const long long multiple = std::max(1LL, (long long)std::max(1, c->_number_of_partial_sums) * std::max(1, c->block_length));
    for (int g = 0; g < ds->number_of_groups; ++g) {
        Group& grp = ds->groups[g];
        grp.d_constraints = nullptr;
        grp.d_radii = nullptr;
        grp.d_number_of_terms = 0;
        if (grp.number_of_terms < 0 || (grp.number_of_terms > 0 && !grp.h_constraints)) {
            set_error(kInvalidValue, "vis_register_meshless_dataset: group without host constraints");
            return;
        }
        const long long padded = (grp.number_of_terms + multiple - 1) / multiple * multiple;
        if (padded > INT32_MAX) {
            set_error(kInvalidValue, "vis_register_meshless_dataset: too many terms");
            return;
        }
        grp.d_number_of_terms = (int)padded;
        if (padded == 0) continue;
        if (registration_alloc(&grp.d_constraints, (size_t)padded, s->registrations, s->stream) != kOk) return;
        cudaMemsetAsync(grp.d_constraints, 0, sizeof(Constraint) * padded, s->stream);
        cudaMemcpyAsync(grp.d_constraints, grp.h_constraints, sizeof(Constraint) * grp.number_of_terms,
                        cudaMemcpyHostToDevice, s->stream);
        GroupStats gs;
        // the largest |weight| and the radius extremes: each part folds from
        // the same start as the serial loop (0, and the first radius), so a
        // NaN is ignored, or kept from the first radius, alike
        {
            constexpr int kMaxParts = 16;
            const bool radii = grp.h_radii && grp.number_of_terms > 0;
            const float r0 = radii ? grp.h_radii[0] : 0.f;
            float wm[kMaxParts], rmin[kMaxParts], rmax[kMaxParts];
            const int parts = parallel_parts(grp.number_of_terms, kMaxParts, [&](int p, long long b, long long e) {
                float w = 0.f, lo = r0, hi = r0;
                for (long long k = b; k < e; ++k) w = std::max(w, std::fabs(grp.h_constraints[k].weight));
                if (radii)
                    for (long long k = b; k < e; ++k) {
                        lo = std::min(lo, grp.h_radii[k]);
                        hi = std::max(hi, grp.h_radii[k]);
                    }
                wm[p] = w;
                rmin[p] = lo;
                rmax[p] = hi;
            });
            gs.weight_max = 0.f;
            for (int p = 0; p < parts; ++p) gs.weight_max = std::max(gs.weight_max, wm[p]);
            if (radii) {
                gs.radius_min = gs.radius_max = r0;
                for (int p = 0; p < parts; ++p) {
                    gs.radius_min = std::min(gs.radius_min, rmin[p]);
                    gs.radius_max = std::max(gs.radius_max, rmax[p]);
                }
                gs.hbins = hbin_histogram(grp, gs);
            }
        }
        {
            std::lock_guard<std::mutex> lock(g_stats_mu);
            g_stats[grp.d_constraints] = gs;
        }
        if (grp.h_radii) {
            if (registration_alloc(&grp.d_radii, (size_t)padded, s->registrations, s->stream) != kOk) return;
            cudaMemsetAsync(grp.d_radii, 0, sizeof(float) * padded, s->stream);
            cudaMemcpyAsync(grp.d_radii, grp.h_radii, sizeof(float) * grp.number_of_terms, cudaMemcpyHostToDevice,
                            s->stream);
        }
    }
    check_cuda(cudaStreamSynchronize(s->stream), "vis_register_meshless_dataset");
}

// meshless_vis/meshless_vis.cu:292-299
void vis_unregister_meshless_dataset(VisConfig* c, MeshlessDataset* ds) {
    ConfigState* s = c ? state_of(c) : nullptr;
    if (!s || !ds) {
        set_error(kInvalidValue, "vis_unregister_meshless_dataset: NULL or unknown argument");
        return;
    }
    // as cudaFree would: no launch on any stream still reads the arrays when
    // their blocks go back to the config's cache (or the pool)
    cudaDeviceSynchronize();
    for (int g = 0; g < ds->number_of_groups; ++g) {
        Group& grp = ds->groups[g];
        const size_t padded = (size_t)std::max(0, grp.d_number_of_terms);
        if (grp.d_constraints) {
            {
                std::lock_guard<std::mutex> lock(g_stats_mu);
                g_stats.erase(grp.d_constraints);
            }
            s->registrations.unregistered(grp.d_constraints, sizeof(Constraint) * padded, s->stream);
        }
        if (grp.d_radii) s->registrations.unregistered(grp.d_radii, sizeof(float) * padded, s->stream);
        grp.d_constraints = nullptr;
        grp.d_radii = nullptr;
    }
}

void vis_opengl_fourier_volume_rendering(MeshlessDataset*, VisConfig*, GLuint) {
    set_error(kUnsupported, "vis_opengl_fourier_volume_rendering: no OpenGL on this build; use vis_config_manual_d_image");
}

// meshless_vis/meshless_vis.cu:334-350: direct slice sum of every group
// (fused with reduce_partial_sums and arrange_samples), then the 2D C2R.
void vis_fourier_volume_rendering(MeshlessDataset* ds, VisConfig* c) {
    ConfigState* s = c ? state_of(c) : nullptr;
    if (!s || !ds || (ds->number_of_groups > 0 && !ds->groups)) {
        set_error(kInvalidValue, "vis_fourier_volume_rendering: NULL or unknown argument");
        return;
    }
    std::string why;
    if (!valid_config(c, &why)) {
        set_error(kInvalidConfig, "vis_fourier_volume_rendering: " + why);
        return;
    }
    if (!c->_d_image || !c->_d_freq_image_arranged) {
        set_error(kInvalidValue, "vis_fourier_volume_rendering: no device image");
        return;
    }
    vis_config_compute_scale(c);
    const int cx = c->_cutoff_frequency.x, cy = c->_cutoff_frequency.y;
    const int nx = c->_number_of_samples.x, ny = c->_number_of_samples.y;
    if (check_cuda(cudaMemsetAsync(c->_d_freq_image_arranged, 0, sizeof(float2) * arranged_count(c), s->stream),
                   "cudaMemsetAsync") != kOk)
        return;
    for (int g = 0; g < ds->number_of_groups; ++g) {
        const Group& grp = ds->groups[g];
        if (grp.number_of_terms > 0 && !grp.d_constraints) {
            set_error(kNotRegistered, "vis_fourier_volume_rendering: group not registered");
            return;
        }
        SumRequest r{};
        r.particles = reinterpret_cast<const float4*>(grp.d_constraints);
        r.radii = grp.d_radii;
        {
            const GroupStats gs = registered_group_stats(grp.d_constraints);
            r.radius_min = gs.radius_min;
            r.radius_max = gs.radius_max;
            r.weight_max = gs.weight_max;
        }
        r.error_flag = static_cast<int*>(s->error_word.ptr);
        r.n = grp.number_of_terms;
        r.basis = (int)grp.basis_function_id;
        // Slice x in (-cx, cx): the reference also evaluates x == cx
        // (fourier_transform.cu:248-249) and then drops it (meshless_vis.cu:323).
        r.lat.x0 = -cx + 1;
        r.lat.nx = cx > 0 ? 2 * cx - 1 : 0;
        r.lat.y0 = 0;
        r.lat.ny = cy;
        r.lat.z0 = 0;
        r.lat.nz = 1;
        r.lat.kx = c->step_size.x;
        r.lat.ky = c->step_size.y;
        r.lat.kz = 0.0;
        const double sx = c->step_size.x, sy = c->step_size.y;
        const double m[9] = {sx * c->u_axis.x, sx * c->u_axis.y, sx * c->u_axis.z,
                             sy * c->v_axis.x, sy * c->v_axis.y, sy * c->v_axis.z, 0.0, 0.0, 0.0};
        std::memcpy(r.lat.m, m, sizeof(m));
        r.scale = (double)c->step_size.x * (double)c->step_size.y;
        r.out = c->_d_freq_image_arranged;
        r.wrap = nx;
        r.row = ny / 2 + 1;
        r.accumulate = g > 0;
        r.stream = s->stream;
        if (c->cull_fully_aliased_terms) {
            // meshless_vis.cu:336 (disabled there): sum only the particles
            // whose footprint lies in the cull box, from a compacted copy
            SumRequest kept;
            if (cull_aliased_terms(r, c->u_axis, c->v_axis, c->step_size, s->cull, s->stream, &kept) != kOk) return;
            r = kept;
        }
        if (launch_plain_sum(r, s->partials, &s->timer) != kOk) return;
    }
    if (check_cufft(cufftSetStream(c->_plan, s->stream), "cufftSetStream") != kOk) return;
    timer_begin(&s->timer, 2, s->stream);
    cufftResult fr = cufftExecC2R(c->_plan, reinterpret_cast<cufftComplex*>(c->_d_freq_image_arranged), c->_d_image);
    timer_end(&s->timer, 2, s->stream);
    check_cufft(fr, "cufftExecC2R");
}

// meshless_vis/meshless_vis.cu:352-355
void vis_copy_to_host(VisConfig* c, float* h_image) {
    ConfigState* s = c ? state_of(c) : nullptr;
    if (!s || !h_image || !c->_d_image) {
        set_error(kInvalidValue, "vis_copy_to_host: NULL or unknown argument");
        return;
    }
    if (check_cuda(cudaMemcpyAsync(h_image, c->_d_image, sizeof(float) * image_count(c), cudaMemcpyDeviceToHost,
                                   s->stream),
                   "vis_copy_to_host") != kOk)
        return;
    check_cuda(cudaStreamSynchronize(s->stream), "vis_copy_to_host");
}

// ------------------------------------------------------------------ timing
unsigned long long vis_kernel_launch_count(void) { return g_launches.load(); }

}  // extern "C"

namespace mv {
// The config's stream and, when bytes > 0, a scratch buffer of the config.
int config_stream_and_scratch(VisConfig* c, cudaStream_t* stream, void** scratch, size_t bytes) {
    ConfigState* s = c ? state_of(c) : nullptr;
    if (!s) return set_error(kInvalidValue, "unknown config");
    *stream = s->stream;
    if (bytes > 0) {
        const int rc = s->post.reserve(bytes);
        if (rc != kOk) return rc;
        *scratch = s->post.ptr;
    }
    return kOk;
}
}  // namespace mv

extern "C" {

int vis_config_enable_kernel_timing(VisConfig* c, int enable) {
    ConfigState* s = c ? state_of(c) : nullptr;
    if (!s) return set_error(kInvalidValue, "vis_config_enable_kernel_timing: unknown config");
    s->timer.enabled = enable != 0;
    return kOk;
}

int vis_config_kernel_timing(VisConfig* c, int stage, float* total_ms, int* launches) {
    ConfigState* s = c ? state_of(c) : nullptr;
    if (!s || stage < 0 || stage >= KernelTimer::kStagesTimed)
        return set_error(kInvalidValue, "vis_config_kernel_timing: bad arguments");
    float total = 0.f;
    int count = 0;
    for (auto& p : s->timer.done[stage]) {
        if (cudaEventSynchronize(p.second) != cudaSuccess) continue;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, p.first, p.second) == cudaSuccess) {
            total += ms;
            ++count;
        }
    }
    s->timer.clear_stage(stage);
    if (total_ms) *total_ms = total;
    if (launches) *launches = count;
    return kOk;
}

}  // extern "C"

// ================================================================ spectrum
struct VisSpectrum {
    int3 grid;
    float step;
    float2* data;
    size_t count;
};

namespace {

// The sum request of one registered group over a half-spectrum lattice
// (accumulating into the spectrum).
SumRequest spectrum_request(const VisSpectrum* sp, const Group& grp, ConfigState* s) {
    SumRequest r{};
    r.particles = reinterpret_cast<const float4*>(grp.d_constraints);
    r.radii = grp.d_radii;
    const GroupStats gs = registered_group_stats(grp.d_constraints);
    r.radius_min = gs.radius_min;
    r.radius_max = gs.radius_max;
    r.weight_max = gs.weight_max;
    r.hbins = gs.hbins.get();  // kept alive by the registration table until unregistered
    r.n = grp.number_of_terms;
    r.basis = (int)grp.basis_function_id;
    r.lat.x0 = -sp->grid.x / 2;
    r.lat.nx = sp->grid.x;
    r.lat.y0 = -sp->grid.y / 2;
    r.lat.ny = sp->grid.y;
    r.lat.z0 = 0;
    r.lat.nz = sp->grid.z / 2 + 1;
    r.lat.kx = r.lat.ky = r.lat.kz = sp->step;
    const double st = sp->step;
    const double m[9] = {st, 0, 0, 0, st, 0, 0, 0, st};
    std::memcpy(r.lat.m, m, sizeof(m));
    r.scale = 1.0;
    r.out = sp->data;
    r.out_base = 0;
    r.out_sx = (long long)sp->grid.y * (sp->grid.z / 2 + 1);
    r.out_sy = sp->grid.z / 2 + 1;
    r.out_sz = 1;
    r.wrap = 0;
    r.row = 0;
    r.accumulate = true;
    r.stream = s->stream;
    r.error_flag = static_cast<int*>(s->error_word.ptr);
    return r;
}

}  // namespace

extern "C" {

VisSpectrum* vis_spectrum_create(int3 grid_size, float step_size) {
    const int3 g = grid_size;
    if (g.x < 2 || g.y < 2 || g.z < 2 || (g.x & 1) || (g.y & 1) || (g.z & 1) || !(step_size > 0.f)) {
        set_error(kInvalidValue, "vis_spectrum_create: grid extents must be even and >= 2, step > 0");
        return nullptr;
    }
    const size_t count = (size_t)g.x * g.y * (g.z / 2 + 1);
    if ((double)g.x * g.y * (g.z / 2 + 1) > (double)INT32_MAX) {
        set_error(kInvalidValue, "vis_spectrum_create: grid too large");
        return nullptr;
    }
    VisSpectrum* sp = new VisSpectrum{g, step_size, nullptr, count};
    if (device_alloc(&sp->data, count) != kOk) {
        delete sp;
        return nullptr;
    }
    return sp;
}

void vis_spectrum_destroy(VisSpectrum* sp) {
    if (!sp) return;
    cudaDeviceSynchronize();
    cudaFree(sp->data);
    delete sp;
}

int3 vis_spectrum_grid_size(VisSpectrum* sp) { return sp ? sp->grid : make_int3(0, 0, 0); }
float2* vis_spectrum_device_data(VisSpectrum* sp) { return sp ? sp->data : nullptr; }

int vis_spectrum_compute(VisSpectrum* sp, VisConfig* c, MeshlessDataset* ds, int form) {
    ConfigState* s = c ? state_of(c) : nullptr;
    if (!sp || !s || !ds || (ds->number_of_groups > 0 && !ds->groups))
        return set_error(kInvalidValue, "vis_spectrum_compute: NULL or unknown argument");
    if (form < VIS_FORM_AUTO || form > VIS_FORM_TENSOR) return set_error(kInvalidValue, "vis_spectrum_compute: bad form");
    // the autotuned launch parameters of this shape, if any (else the defaults)
    long long n_total = 0;
    for (int g = 0; g < ds->number_of_groups; ++g) n_total += std::max(0, ds->groups[g].number_of_terms);
    TuneScope tune(tuned_params(sp->grid.x, sp->grid.y, sp->grid.z, n_total, ds->number_of_groups, form));
    std::vector<SumRequest> tc_groups, plain_groups;
    for (int g = 0; g < ds->number_of_groups; ++g) {
        const Group& grp = ds->groups[g];
        if (grp.number_of_terms > 0 && !grp.d_constraints)
            return set_error(kNotRegistered, "vis_spectrum_compute: group not registered");
        SumRequest r = spectrum_request(sp, grp, s);
        const bool want_tc = form == VIS_FORM_TENSOR || form == VIS_FORM_AUTO;
        if (want_tc && tensor_sum_available(r, form)) tc_groups.push_back(r);
        else plain_groups.push_back(r);
    }
    // every group adds into a zeroed spectrum (the result equals the
    // reference's first-group-assigns, later-groups-accumulate)
    int rc = check_cuda(cudaMemsetAsync(sp->data, 0, sizeof(float2) * sp->count, s->stream), "cudaMemsetAsync");
    if (rc != kOk) return rc;
    if (!tc_groups.empty()) {
        const TensorPlan* plan = nullptr;
        rc = tensor_prepare(tc_groups, s->tensor, s->stream, &plan);
        if (rc == kOk)
            rc = tensor_enqueue(tc_groups, *plan, s->tensor, s->partials, &s->timer, s->stream,
                                static_cast<int*>(s->error_word.ptr));
        if (rc != kOk) return rc;
    }
    for (const SumRequest& r : plain_groups) {
        rc = launch_plain_sum(r, s->partials, &s->timer);
        if (rc != kOk) return rc;
    }
    return kOk;
}

int vis_spectrum_copy_to_host(VisSpectrum* sp, VisConfig* c, float2* h) {
    ConfigState* s = c ? state_of(c) : nullptr;
    if (!sp || !s || !h) return set_error(kInvalidValue, "vis_spectrum_copy_to_host: NULL or unknown argument");
    int rc = check_cuda(cudaMemcpyAsync(h, sp->data, sizeof(float2) * sp->count, cudaMemcpyDeviceToHost, s->stream),
                        "vis_spectrum_copy_to_host");
    if (rc != kOk) return rc;
    return sync_and_check(s, "vis_spectrum_copy_to_host");
}

int vis_spectrum_render_views(VisSpectrum* sp, VisConfig* c, int number_of_views, const float3* u_axes,
                              const float3* v_axes, float* d_images, float* h_images) {
    ConfigState* s = c ? state_of(c) : nullptr;
    if (!sp || !s || number_of_views < 0 || (number_of_views > 0 && (!u_axes || !v_axes)))
        return set_error(kInvalidValue, "vis_spectrum_render_views: NULL or unknown argument");
    if (number_of_views == 0) return kOk;
    const int cx = c->_cutoff_frequency.x, cy = c->_cutoff_frequency.y;
    const int nx = c->_number_of_samples.x, ny = c->_number_of_samples.y;
    if (cx < 0 || cy < 0 || 2 * cx > nx || 2 * cy > ny || nx < 1 || ny < 2)
        return set_error(kInvalidConfig, "vis_spectrum_render_views: cutoff/number_of_samples mismatch");

    std::vector<float> hv((size_t)8 * number_of_views);
    for (int i = 0; i < number_of_views; ++i) {
        float* p = hv.data() + 8 * i;
        p[0] = u_axes[i].x; p[1] = u_axes[i].y; p[2] = u_axes[i].z;
        p[3] = v_axes[i].x; p[4] = v_axes[i].y; p[5] = v_axes[i].z;
        p[6] = c->step_size.x; p[7] = c->step_size.y;
    }
    const size_t per_arr = (size_t)nx * (ny / 2 + 1), per_img = (size_t)nx * ny;
    int rc = s->views.reserve(hv.size() * sizeof(float));
    if (rc == kOk) rc = s->arranged.reserve(per_arr * number_of_views * sizeof(float2));
    if (rc == kOk && !d_images) rc = s->images.reserve(per_img * number_of_views * sizeof(float));
    if (rc != kOk) return rc;
    float* imgs = d_images ? d_images : static_cast<float*>(s->images.ptr);
    rc = check_cuda(cudaMemcpyAsync(s->views.ptr, hv.data(), hv.size() * sizeof(float), cudaMemcpyHostToDevice, s->stream),
                    "view parameters H2D");
    if (rc != kOk) return rc;

    SliceRequest q{};
    q.spectrum = sp->data;
    q.gx = sp->grid.x;
    q.gy = sp->grid.y;
    q.gz = sp->grid.z;
    q.inv_step = 1.0f / sp->step;
    q.views = static_cast<const float*>(s->views.ptr);
    q.number_of_views = number_of_views;
    q.cx = cx;
    q.cy = cy;
    q.nx = nx;
    q.ny = ny;
    q.arranged = static_cast<float2*>(s->arranged.ptr);
    q.stream = s->stream;
    rc = launch_slice_extract(q, &s->timer);
    if (rc != kOk) return rc;

    auto key = std::make_tuple(nx, ny, number_of_views);
    cufftHandle plan;
    auto it = s->batched_plans.find(key);
    if (it == s->batched_plans.end()) {
        if (s->batched_plans.size() >= 4) {
            cudaStreamSynchronize(s->stream);
            for (auto& kv : s->batched_plans) cufftDestroy(kv.second);
            s->batched_plans.clear();
        }
        int n[2] = {nx, ny};
        rc = check_cufft(cufftPlanMany(&plan, 2, n, nullptr, 1, (int)per_arr, nullptr, 1, (int)per_img, CUFFT_C2R,
                                       number_of_views),
                         "cufftPlanMany");
        if (rc != kOk) return rc;
        s->batched_plans[key] = plan;
    } else {
        plan = it->second;
    }
    rc = check_cufft(cufftSetStream(plan, s->stream), "cufftSetStream");
    if (rc != kOk) return rc;
    timer_begin(&s->timer, 2, s->stream);
    cufftResult fr = cufftExecC2R(plan, static_cast<cufftComplex*>(s->arranged.ptr), imgs);
    timer_end(&s->timer, 2, s->stream);
    rc = check_cufft(fr, "cufftExecC2R (batched)");
    if (rc != kOk) return rc;
    if (h_images) {
        rc = check_cuda(cudaMemcpyAsync(h_images, imgs, per_img * number_of_views * sizeof(float),
                                        cudaMemcpyDeviceToHost, s->stream),
                        "images D2H");
        if (rc != kOk) return rc;
        return sync_and_check(s, "vis_spectrum_render_views");
    }
    return kOk;
}

}  // extern "C"

// =================================================================== batch
struct VisBatch {
    VisConfig* cfg = nullptr;
    struct Job {
        MeshlessDataset* ds = nullptr;
        VisSpectrum* sp = nullptr;
        float2 view_step;
        int2 cutoff, samples;
        std::vector<float3> u, v;
        int size_class = -1;
        size_t image_offset = 0;  // floats into the class's image buffer
    };
    struct SizeClass {
        int nx = 0, ny = 0, views = 0;
        cufftHandle plan = 0;
        Workspace arranged, images;
    };
    std::vector<Job> jobs;
    std::vector<SizeClass> classes;
    std::vector<SumRequest> tc_groups, plain_groups;
    TensorPlan plan;
    TensorWorkspace tensor;
    Workspace partials, views_table;
    int n_views = 0;
    long long total_elements = 0;
    std::vector<uint64_t> registered;  // batch_signature of the captured launches
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int mode = -1;  // -1 not built, 0 direct launches, 1 graph

    void drop_build() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        for (SizeClass& c : classes) {
            if (c.plan) cufftDestroy(c.plan);
            c.arranged.release();
            c.images.release();
        }
        classes.clear();
        mode = -1;
    }
};

namespace {

// What a batch's captured launches depend on, per group: the device arrays,
// the term count, and the registration statistics its plan reads (the weight
// and radius extremes and the h-bin histogram).  An execute whose datasets
// match the captured signature replays the graph; a frame registered at the
// same addresses but with other statistics is planned and captured again.
std::vector<uint64_t> batch_signature(const VisBatch* b) {
    std::vector<uint64_t> out;
    auto bits = [](float x) {
        uint32_t u;
        std::memcpy(&u, &x, sizeof u);
        return (uint64_t)u;
    };
    for (const VisBatch::Job& j : b->jobs)
        for (int g = 0; g < j.ds->number_of_groups; ++g) {
            const Group& grp = j.ds->groups[g];
            out.push_back((uint64_t)(uintptr_t)grp.d_constraints);
            out.push_back((uint64_t)(uintptr_t)grp.d_radii);
            out.push_back((uint64_t)(uint32_t)grp.number_of_terms);
            const GroupStats gs = registered_group_stats(grp.d_constraints);
            out.push_back(bits(gs.radius_min) << 32 | bits(gs.radius_max));
            out.push_back(bits(gs.weight_max));
            out.push_back(gs.hbins ? gs.hbins->id : 0);  // the histogram's content hash
        }
    return out;
}

// Everything one execute enqueues; capturable once the workspaces are sized.
int batch_enqueue(VisBatch* b, ConfigState* s) {
    int rc = kOk;
    for (const VisBatch::Job& j : b->jobs) {
        rc = check_cuda(cudaMemsetAsync(j.sp->data, 0, sizeof(float2) * j.sp->count, s->stream), "cudaMemsetAsync");
        if (rc != kOk) return rc;
    }
    int* err = static_cast<int*>(s->error_word.ptr);
    if (!b->tc_groups.empty()) {
        rc = tensor_enqueue(b->tc_groups, b->plan, b->tensor, b->partials, nullptr, s->stream, err);
        if (rc != kOk) return rc;
    }
    for (const SumRequest& r : b->plain_groups) {
        rc = launch_plain_sum(r, b->partials, nullptr);
        if (rc != kOk) return rc;
    }
    rc = launch_slice_extract_batch(static_cast<const SliceView*>(b->views_table.ptr), b->n_views, b->total_elements,
                                    s->stream, nullptr);
    if (rc != kOk) return rc;
    for (VisBatch::SizeClass& c : b->classes) {
        rc = check_cufft(cufftSetStream(c.plan, s->stream), "cufftSetStream");
        if (rc != kOk) return rc;
        rc = check_cufft(cufftExecC2R(c.plan, static_cast<cufftComplex*>(c.arranged.ptr),
                                      static_cast<float*>(c.images.ptr)),
                         "cufftExecC2R (batch)");
        if (rc != kOk) return rc;
    }
    return kOk;
}

int batch_build(VisBatch* b, ConfigState* s, int form) {
    b->drop_build();
    b->tc_groups.clear();
    b->plain_groups.clear();
    for (const VisBatch::Job& j : b->jobs)
        for (int g = 0; g < j.ds->number_of_groups; ++g) {
            const Group& grp = j.ds->groups[g];
            if (grp.number_of_terms > 0 && !grp.d_constraints)
                return set_error(kNotRegistered, "vis_batch_execute: a group of a batch dataset is not registered");
            SumRequest r = spectrum_request(j.sp, grp, s);
            const bool want_tc = form == VIS_FORM_TENSOR || form == VIS_FORM_AUTO;
            if (want_tc && tensor_sum_available(r, form)) b->tc_groups.push_back(r);
            else b->plain_groups.push_back(r);
        }
    int rc = kOk;
    if (!b->tc_groups.empty()) {
        rc = tensor_plan(b->tc_groups, b->plan);
        if (rc == kOk) rc = tensor_reserve_upload(b->plan, b->tensor, s->stream);
        if (rc != kOk) return rc;
    }
    // image size classes, each rendered by one batched C2R
    for (VisBatch::Job& j : b->jobs) {
        int c = -1;
        for (size_t k = 0; k < b->classes.size(); ++k)
            if (b->classes[k].nx == j.samples.x && b->classes[k].ny == j.samples.y) c = (int)k;
        if (c < 0) {
            c = (int)b->classes.size();
            b->classes.emplace_back();
            b->classes.back().nx = j.samples.x;
            b->classes.back().ny = j.samples.y;
        }
        j.size_class = c;
        j.image_offset = (size_t)b->classes[c].views * j.samples.x * j.samples.y;
        b->classes[c].views += (int)j.u.size();
    }
    std::vector<SliceView> views;
    std::vector<int> class_done(b->classes.size(), 0);
    long long elements = 0;
    for (VisBatch::SizeClass& c : b->classes) {
        const size_t per_arr = (size_t)c.nx * (c.ny / 2 + 1), per_img = (size_t)c.nx * c.ny;
        rc = c.arranged.reserve(per_arr * c.views * sizeof(float2));
        if (rc == kOk) rc = c.images.reserve(per_img * c.views * sizeof(float));
        if (rc != kOk) return rc;
        int n[2] = {c.nx, c.ny};
        rc = check_cufft(cufftPlanMany(&c.plan, 2, n, nullptr, 1, (int)per_arr, nullptr, 1, (int)per_img, CUFFT_C2R,
                                       c.views),
                         "cufftPlanMany (batch)");
        if (rc != kOk) return rc;
    }
    for (const VisBatch::Job& j : b->jobs) {
        VisBatch::SizeClass& c = b->classes[j.size_class];
        const size_t per_arr = (size_t)c.nx * (c.ny / 2 + 1);
        for (size_t k = 0; k < j.u.size(); ++k) {
            SliceView v{};
            v.spectrum = j.sp->data;
            v.arranged = static_cast<float2*>(c.arranged.ptr) + per_arr * class_done[j.size_class]++;
            v.element_offset = elements;
            v.gx = j.sp->grid.x;
            v.gy = j.sp->grid.y;
            v.gz = j.sp->grid.z;
            v.inv_step = 1.0f / j.sp->step;
            v.u[0] = j.u[k].x; v.u[1] = j.u[k].y; v.u[2] = j.u[k].z;
            v.v[0] = j.v[k].x; v.v[1] = j.v[k].y; v.v[2] = j.v[k].z;
            v.step[0] = j.view_step.x;
            v.step[1] = j.view_step.y;
            v.cx = j.cutoff.x;
            v.cy = j.cutoff.y;
            v.nx = j.samples.x;
            v.ny = j.samples.y;
            views.push_back(v);
            elements += (long long)per_arr;
        }
    }
    b->n_views = (int)views.size();
    b->total_elements = elements;
    if (!views.empty()) {
        rc = b->views_table.reserve(views.size() * sizeof(SliceView));
        if (rc == kOk)
            rc = check_cuda(cudaMemcpyAsync(b->views_table.ptr, views.data(), views.size() * sizeof(SliceView),
                                            cudaMemcpyHostToDevice, s->stream),
                            "batch view table H2D");
        if (rc == kOk) rc = check_cuda(cudaStreamSynchronize(s->stream), "batch view table H2D");
        if (rc != kOk) return rc;
    }
    // one direct run sizes every workspace (and produces this execute's results)
    rc = batch_enqueue(b, s);
    if (rc != kOk) return rc;
    rc = check_cuda(cudaStreamSynchronize(s->stream), "vis_batch_execute");
    if (rc != kOk) return rc;
    // capture the same sequence
    b->mode = 0;
    if (cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeRelaxed) == cudaSuccess) {
        const int erc = batch_enqueue(b, s);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(s->stream, &g);
        if (erc == kOk && ce == cudaSuccess && g && cudaGraphInstantiate(&b->exec, g, 0) == cudaSuccess) {
            b->graph = g;
            b->mode = 1;
        } else {
            if (g) cudaGraphDestroy(g);
            b->exec = nullptr;
            vis_clear_last_error();
        }
    }
    cudaGetLastError();
    b->registered = batch_signature(b);
    return kOk;
}

}  // namespace

extern "C" {

VisBatch* vis_batch_create(VisConfig* vis_config) {
    if (!vis_config || !state_of(vis_config)) {
        set_error(kInvalidValue, "vis_batch_create: unknown config");
        return nullptr;
    }
    VisBatch* b = new VisBatch();
    b->cfg = vis_config;
    return b;
}

int vis_batch_add(VisBatch* b, MeshlessDataset* ds, int3 grid_size, float spectrum_step, float2 view_step,
                  int2 cutoff, int2 samples, int number_of_views, const float3* u_axes, const float3* v_axes) {
    if (!b || !ds || (ds->number_of_groups > 0 && !ds->groups) || number_of_views < 0 ||
        (number_of_views > 0 && (!u_axes || !v_axes)))
        return -set_error(kInvalidValue, "vis_batch_add: NULL or bad argument");
    if (cutoff.x < 0 || cutoff.y < 0 || samples.x < 1 || samples.y < 2 || 2 * cutoff.x > samples.x ||
        2 * cutoff.y > samples.y)
        return -set_error(kInvalidConfig, "vis_batch_add: cutoff/number_of_samples mismatch");
    VisSpectrum* sp = vis_spectrum_create(grid_size, spectrum_step);
    if (!sp) return -vis_get_last_error();
    VisBatch::Job j;
    j.ds = ds;
    j.sp = sp;
    j.view_step = view_step;
    j.cutoff = cutoff;
    j.samples = samples;
    j.u.assign(u_axes, u_axes + number_of_views);
    j.v.assign(v_axes, v_axes + number_of_views);
    b->jobs.push_back(std::move(j));
    b->drop_build();
    return (int)b->jobs.size() - 1;
}

int vis_batch_execute(VisBatch* b, int form) {
    ConfigState* s = b ? state_of(b->cfg) : nullptr;
    if (!s) return set_error(kInvalidValue, "vis_batch_execute: unknown batch");
    if (form < VIS_FORM_AUTO || form > VIS_FORM_TENSOR) return set_error(kInvalidValue, "vis_batch_execute: bad form");
    if (b->mode < 0 || b->registered != batch_signature(b)) return batch_build(b, s, form);
    if (b->mode == 1) return check_cuda(cudaGraphLaunch(b->exec, s->stream), "cudaGraphLaunch");
    return batch_enqueue(b, s);
}

int vis_batch_uses_graph(VisBatch* b) { return b ? b->mode : -1; }

float* vis_batch_images(VisBatch* b, int job) {
    if (!b || job < 0 || job >= (int)b->jobs.size() || b->jobs[job].size_class < 0 || b->mode < 0) return nullptr;
    const VisBatch::Job& j = b->jobs[job];
    return static_cast<float*>(b->classes[j.size_class].images.ptr) + j.image_offset;
}

float2* vis_batch_spectrum(VisBatch* b, int job) {
    if (!b || job < 0 || job >= (int)b->jobs.size()) return nullptr;
    return b->jobs[job].sp->data;
}

int vis_batch_copy_images_to_host(VisBatch* b, int job, float* h) {
    ConfigState* s = b ? state_of(b->cfg) : nullptr;
    float* d = vis_batch_images(b, job);
    if (!s || !d || !h) return set_error(kInvalidValue, "vis_batch_copy_images_to_host: bad arguments");
    const VisBatch::Job& j = b->jobs[job];
    const size_t bytes = sizeof(float) * j.u.size() * j.samples.x * j.samples.y;
    int rc = check_cuda(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s->stream), "batch images D2H");
    if (rc != kOk) return rc;
    return sync_and_check(s, "vis_batch_copy_images_to_host");
}

void vis_batch_destroy(VisBatch* b) {
    if (!b) return;
    ConfigState* s = state_of(b->cfg);
    if (s) cudaStreamSynchronize(s->stream);
    b->drop_build();
    b->tensor.release();
    b->partials.release();
    b->views_table.release();
    for (VisBatch::Job& j : b->jobs) vis_spectrum_destroy(j.sp);
    delete b;
}

}  // extern "C"
