// Autotuner: picks, per spectrum shape, the launch parameters that the
// kernels otherwise derive from fixed rules (TuneParams in mv_internal.h):
//   plain_waves  split-K of the plain form, in blocks per SM: 2, 4, 6, 8
//   tc_waves     particle splits of the tensor form, in waves: 2, 4, 8
//   tc_flush     tensor-core accumulation chain of the single-accumulator
//                tiles, in stages: 8, 16 (longer chains lose accuracy, so
//                they are not candidates)
//   hbin_job_cost  h-binned groups (SPH / Wendland with per-particle radii):
//                the price of one more h-bin in the bin-count optimisation,
//                256, 1024 (default), 4096: lower gives more, narrower bins
//                with fewer Chebyshev nodes per particle, higher fewer jobs
//                (the accuracy rule on the nodes is the same for all)
//   tc_shapes    tensor form (tensor and auto forms only): the tile shapes
//                the planner may use, VIS_TILE_* bits (all by default); each
//                shape is tried turned off, since the planner's cost rule
//                counts MMAs and not the power cap, L2 reuse or flush stalls
// vis_autotune_spectrum times each candidate on the caller's own data through
// the public compute path (one warm-up and one timed run, CUDA events on the
// config's stream), one parameter at a time starting from the defaults, and
// records the fastest set for the shape: lattice, total particles, number of
// groups and form.  Later vis_spectrum_compute calls of that shape use it.
// The table is process-wide; vis_autotune_clear empties it.
#include <initializer_list>
#include <map>
#include <mutex>
#include <tuple>

#include "meshless_vis_b200.h"
#include "mv_internal.h"

namespace mv {
namespace {

using TuneKey = std::tuple<int, int, int, long long, int, int>;
std::mutex g_tune_mu;
std::map<TuneKey, TuneParams> g_tune_table;
thread_local TuneParams g_active;

long long dataset_terms(const MeshlessDataset* ds, int* groups) {
    long long n = 0;
    *groups = ds->number_of_groups;
    for (int g = 0; g < ds->number_of_groups; ++g) n += std::max(0, ds->groups[g].number_of_terms);
    return n;
}

// Whether some group is SPH or Wendland with registered, varying radii (the
// groups the tensor form takes through h-bins).
bool dataset_has_varying_radii(const MeshlessDataset* ds) {
    for (int g = 0; g < ds->number_of_groups; ++g) {
        const Group& grp = ds->groups[g];
        if (!grp.d_constraints) continue;
        if (registered_group_stats(grp.d_constraints).hbins) return true;
    }
    return false;
}

}  // namespace

const TuneParams& active_tune() { return g_active; }
TuneScope::TuneScope(const TuneParams& p) : saved(g_active) { g_active = p; }
TuneScope::~TuneScope() { g_active = saved; }

TuneParams tuned_params(int kx, int ky, int kz, long long n_total, int n_groups, int form) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_table.find(TuneKey(kx, ky, kz, n_total, n_groups, form));
    return it == g_tune_table.end() ? TuneParams{} : it->second;
}

}  // namespace mv

using namespace mv;

extern "C" {

int vis_autotune_spectrum(VisSpectrum* sp, VisConfig* vis_config, MeshlessDataset* meshless_dataset, int form,
                          float* best_ms) {
    if (!sp || !vis_config || !meshless_dataset)
        return set_error(kInvalidValue, "vis_autotune_spectrum: NULL argument");
    const int3 grid = vis_spectrum_grid_size(sp);
    int rc = kOk;
    cudaStream_t stream = vis_config_get_stream(vis_config);
    int groups = 0;
    const long long n = dataset_terms(meshless_dataset, &groups);
    const TuneKey key(grid.x, grid.y, grid.z, n, groups, form);
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune_table.erase(key);  // time every candidate from the defaults
    }
    cudaEvent_t e0, e1;
    rc = check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
    if (rc != kOk) return rc;
    rc = check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
    if (rc != kOk) {
        cudaEventDestroy(e0);
        return rc;
    }
    // one warm-up and one timed run of a candidate; < 0 on error
    auto time_of = [&](const TuneParams& p) -> float {
        TuneScope scope(p);
        if (vis_spectrum_compute(sp, vis_config, meshless_dataset, form) != kOk) return -1.f;
        cudaEventRecord(e0, stream);
        if (vis_spectrum_compute(sp, vis_config, meshless_dataset, form) != kOk) return -1.f;
        cudaEventRecord(e1, stream);
        if (check_cuda(cudaEventSynchronize(e1), "vis_autotune_spectrum") != kOk) return -1.f;
        float ms = -1.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms;
    };
    TuneParams best;
    float best_t = time_of(best);
    const int plain_c[] = {2, 4, 6, 8}, waves_c[] = {2, 4, 8}, flush_c[] = {16, 8}, hbin_c[] = {256, 1024, 4096};
    const int shape_bits[] = {kTileRowFold, kTileAxisExchange, kTileDoubleBuffer, kTileCtaPairs};
    const bool binned = dataset_has_varying_radii(meshless_dataset);
    for (int field = 0; field < 5 && best_t >= 0.f; ++field) {
        if (field == 3 && !binned) continue;
        if (field == 4 && form == VIS_FORM_PLAIN) continue;
        const int* cand = field == 0 ? plain_c : field == 1 ? waves_c : field == 2 ? flush_c : field == 3 ? hbin_c : shape_bits;
        const int count = field == 0 ? 4 : field == 1 ? 3 : field == 2 ? 2 : field == 3 ? 3 : 4;
        for (int i = 0; i < count && best_t >= 0.f; ++i) {
            TuneParams p = best;
            if (field == 4) {
                // the best set so far with one more shape turned off
                if (!(p.tc_shapes & cand[i])) continue;
                p.tc_shapes &= ~cand[i];
            } else {
                int& v = field == 0 ? p.plain_waves : field == 1 ? p.tc_waves : field == 2 ? p.tc_flush : p.hbin_job_cost;
                if (v == cand[i]) continue;
                v = cand[i];
            }
            const float t = time_of(p);
            if (t < 0.f) best_t = -1.f;
            else if (t < best_t) {
                best_t = t;
                best = p;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best_t < 0.f) return vis_get_last_error() != kOk ? vis_get_last_error() : set_error(kCudaError, "vis_autotune_spectrum");
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune_table[key] = best;
    }
    if (best_ms) *best_ms = best_t;
    return kOk;
}

int vis_autotune_lookup(int3 grid_size, long long number_of_terms, int number_of_groups, int form, int* plain_waves,
                        int* tensor_waves, int* tensor_flush_stages) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_table.find(TuneKey(grid_size.x, grid_size.y, grid_size.z, number_of_terms, number_of_groups, form));
    const TuneParams p = it == g_tune_table.end() ? TuneParams{} : it->second;
    if (plain_waves) *plain_waves = p.plain_waves;
    if (tensor_waves) *tensor_waves = p.tc_waves;
    if (tensor_flush_stages) *tensor_flush_stages = p.tc_flush;
    return it == g_tune_table.end() ? 0 : 1;
}

int vis_autotune_lookup_shapes(int3 grid_size, long long number_of_terms, int number_of_groups, int form,
                               int* tile_shapes, int* hbin_price) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_table.find(TuneKey(grid_size.x, grid_size.y, grid_size.z, number_of_terms, number_of_groups, form));
    const TuneParams p = it == g_tune_table.end() ? TuneParams{} : it->second;
    if (tile_shapes) *tile_shapes = p.tc_shapes;
    if (hbin_price) *hbin_price = p.hbin_job_cost;
    return it == g_tune_table.end() ? 0 : 1;
}

int vis_autotune_store(int3 grid_size, long long number_of_terms, int number_of_groups, int form, int plain_waves,
                       int tensor_waves, int tensor_flush_stages, int tile_shapes, int hbin_price) {
    auto in = [](int v, std::initializer_list<int> set) {
        for (int x : set)
            if (v == x) return true;
        return false;
    };
    if (!in(plain_waves, {2, 4, 6, 8}) || !in(tensor_waves, {2, 4, 8}) || !in(tensor_flush_stages, {8, 16}) ||
        tile_shapes < 0 || tile_shapes > kTileAll || hbin_price < 1 || hbin_price > (1 << 20))
        return set_error(kInvalidValue, "vis_autotune_store: parameter outside its candidate set");
    if (form != VIS_FORM_AUTO && form != VIS_FORM_PLAIN && form != VIS_FORM_TENSOR)
        return set_error(kInvalidValue, "vis_autotune_store: unknown form");
    TuneParams p;
    p.plain_waves = plain_waves;
    p.tc_waves = tensor_waves;
    p.tc_flush = tensor_flush_stages;
    p.tc_shapes = tile_shapes;
    p.hbin_job_cost = hbin_price;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_table[TuneKey(grid_size.x, grid_size.y, grid_size.z, number_of_terms, number_of_groups, form)] = p;
    return kOk;
}

void vis_autotune_clear(void) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_table.clear();
}

}  // extern "C"
