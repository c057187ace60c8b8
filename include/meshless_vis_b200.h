/*
 * meshless_vis_b200.h -- additions of the B200 drop-in that have no
 * counterpart in the reference's C API.  Everything here is extern "C", with
 * plain pointers and sizes.
 *
 *   - error reporting (the reference aborts through cutil macros instead,
 *     meshless_vis/meshless_vis.cu:73-81, :141-146);
 *   - an explicit CUDA stream per VisConfig (the reference uses the default
 *     stream everywhere, meshless_vis/meshless_vis.cu:334-350);
 *   - the 3D Hermitian half-spectrum path: the Fourier sum is evaluated once on
 *     a 3D lattice, and any number of views are then cut from it by
 *     interpolated Fourier slices and rendered by one batched 2D C2R, instead
 *     of redoing the whole sum per view as vis_fourier_volume_rendering does;
 *   - per-stage device timing for benchmarks.
 */
#ifndef MESHLESS_VIS_B200_H
#define MESHLESS_VIS_B200_H

#include "meshless_vis.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- errors */
enum VisError
{
    VIS_SUCCESS = 0,
    VIS_ERROR_INVALID_VALUE = 1, /* bad argument, NULL pointer, size out of range */
    VIS_ERROR_INVALID_CONFIG = 2, /* vis_config_check() would return false */
    VIS_ERROR_CUDA = 3,           /* a CUDA runtime call failed */
    VIS_ERROR_CUFFT = 4,          /* a cuFFT call failed */
    VIS_ERROR_OUT_OF_MEMORY = 5,  /* device allocation failed */
    VIS_ERROR_NOT_REGISTERED = 6, /* dataset not registered with vis_register_meshless_dataset */
    VIS_ERROR_UNSUPPORTED = 7,    /* feature not available (OpenGL interop) */
    VIS_ERROR_NO_KERNEL = 8       /* the library was built without code for this device */
};

/* Code of the last failed call on this host thread (VIS_SUCCESS if none since
 * the last vis_clear_last_error). */
int vis_get_last_error(void);
/* Human-readable detail of the last failure on this host thread. */
const char* vis_get_last_error_message(void);
const char* vis_get_error_string(int code);
void vis_clear_last_error(void);

/* ---------------------------------------------------------------- streams */
/* All work for a VisConfig is issued on its stream (default: a non-blocking
 * stream the library creates).  vis_copy_to_host synchronises it. */
int vis_config_set_stream(VisConfig* vis_config, cudaStream_t stream);
cudaStream_t vis_config_get_stream(VisConfig* vis_config);
int vis_config_synchronize(VisConfig* vis_config);

/* ------------------------------------------------------- 3D half-spectrum */
/* How the Fourier sum is evaluated:
 *   VIS_FORM_PLAIN  -- FP32 SIMT, exact fixed-point phase per term;
 *   VIS_FORM_TENSOR -- per-axis exponential factorisation as complex GEMMs on
 *                      the tensor cores (split FP16 hi+lo, FP32 accumulate);
 *                      needs a separable basis (GAUSSIAN_DECAYING, GAUSSIAN) or
 *                      a group without radii; other groups fall back to PLAIN;
 *   VIS_FORM_AUTO   -- TENSOR where the group allows it, else PLAIN. */
enum VisSumForm
{
    VIS_FORM_AUTO = 0,
    VIS_FORM_PLAIN = 1,
    VIS_FORM_TENSOR = 2
};

typedef struct VisSpectrum VisSpectrum;

/* A device-resident half-spectrum F(k) = sum_j w_j Phi^(|k| h_j)
 * exp(-2 pi i k.x_j) on k = step_size * (i, j, l), i in [-Kx/2, Kx/2),
 * j in [-Ky/2, Ky/2), l in [0, Kz/2]; grid_size = (Kx, Ky, Kz), each even and
 * >= 2.  Storage: float2[Kx][Ky][Kz/2+1], element [i+Kx/2][j+Ky/2][l]. */
VisSpectrum* vis_spectrum_create(int3 grid_size, float step_size);
void vis_spectrum_destroy(VisSpectrum* spectrum);
int3 vis_spectrum_grid_size(VisSpectrum* spectrum);
float2* vis_spectrum_device_data(VisSpectrum* spectrum);

/* Evaluates the spectrum of every group of a registered dataset (the first
 * group overwrites, later groups accumulate), on vis_config's stream. */
int vis_spectrum_compute(VisSpectrum* spectrum, VisConfig* vis_config, MeshlessDataset* meshless_dataset, int form);

/* Copies the whole spectrum to the host (Kx*Ky*(Kz/2+1) float2) and waits. */
int vis_spectrum_copy_to_host(VisSpectrum* spectrum, VisConfig* vis_config, float2* h_spectrum);

/* Renders number_of_views views from the spectrum with vis_config's step_size,
 * cutoff and number of samples: per view, slice sample (x, y) with
 * x in (-cx, cx), y in [0, cy) takes the trilinearly interpolated spectrum at
 * step.x x u + step.y y v (Hermitian fold for k_z < 0, zero outside the
 * lattice), times step.x*step.y, placed in the C2R layout of arrange_samples
 * (meshless_vis/meshless_vis.cu:318-332); then one batched unnormalised 2D C2R.
 * u_axes, v_axes: host arrays of number_of_views float3.
 * d_images: device float[views][Nx][Ny], or NULL to use a library buffer;
 * h_images: if not NULL, the images are also copied there and the call waits. */
int vis_spectrum_render_views(VisSpectrum* spectrum, VisConfig* vis_config, int number_of_views,
                              const float3* u_axes, const float3* v_axes, float* d_images, float* h_images);

/* -------------------------------------------------------------- autotuner */
/* Picks the launch parameters of vis_spectrum_compute for this spectrum's
 * shape (lattice, total particles of the dataset, number of groups, form) by
 * timing candidates on the caller's data: the plain form's split-K (2, 4, 6, 8
 * blocks per SM), the tensor form's particle splits (2, 4, 8 waves), the
 * accumulation chain of its single-accumulator tiles (8 or 16 stages; longer
 * chains lose accuracy; the double-buffered tile keeps at most 8), its tile
 * shapes (each VIS_TILE_* shape turned off in turn, for the tensor and auto
 * forms) and, for datasets with h-binned groups, the price of one more h-bin
 * (256, 1024, 4096: the h-bin count).  Each candidate runs
 * vis_spectrum_compute twice (the spectrum holds the last result); the best
 * set is kept for the process and used by later computes of the same shape.
 * best_ms (may be NULL) receives its time.  No counterpart in the reference,
 * which fixes its launch shape by block_length and number_of_partial_sums
 * (fourier_transform.cu:167-180). */
int vis_autotune_spectrum(VisSpectrum* spectrum, VisConfig* vis_config, MeshlessDataset* meshless_dataset, int form,
                          float* best_ms);
/* The parameters that computes of this shape use; returns 1 if they were
 * tuned, 0 for the defaults (6, 4, 16). */
int vis_autotune_lookup(int3 grid_size, long long number_of_terms, int number_of_groups, int form,
                        int* plain_waves, int* tensor_waves, int* tensor_flush_stages);
/* Tile shapes of the tensor form, as bits: the planner uses a shape where its
 * cost rule finds it cheaper, and only if its bit is set. */
enum {
    VIS_TILE_ROW_FOLD = 1,       /* several b rows of a job as column blocks of one row */
    VIS_TILE_AXIS_EXCHANGE = 2,  /* rows (a, c) and columns b for Gaussian jobs */
    VIS_TILE_DOUBLE_BUFFER = 4,  /* two accumulators per CTA pair for jobs of short items */
    VIS_TILE_CTA_PAIRS = 8,      /* CTA-pair (M = 256) tiles at all */
    VIS_TILE_ALL = 15
};
/* The tile shapes (VIS_TILE_* bits) and the h-bin price that computes of this
 * shape use; returns 1 if they were tuned, 0 for the defaults (VIS_TILE_ALL,
 * 1024).  Either pointer may be NULL. */
int vis_autotune_lookup_shapes(int3 grid_size, long long number_of_terms, int number_of_groups, int form,
                               int* tile_shapes, int* hbin_price);
/* Records a parameter set for a shape, as a tuning run would: for example one
 * read back by the two lookups in an earlier process, or tile shapes a caller
 * wants kept off.  Every value must lie in its candidate set above
 * (tile_shapes 0 .. VIS_TILE_ALL, hbin_price 1 .. 2^20); else
 * VIS_ERROR_INVALID_VALUE and nothing is recorded. */
int vis_autotune_store(int3 grid_size, long long number_of_terms, int number_of_groups, int form, int plain_waves,
                       int tensor_waves, int tensor_flush_stages, int tile_shapes, int hbin_price);
void vis_autotune_clear(void);

/* Device memory the tensor form may use for B-operand images (the c-axis
 * factors of every particle, computed once per compute and copied by each
 * m-tile instead of recomputed).  A job whose images would exceed what is left
 * of the limit computes its B operands per tile instead (same results).
 * bytes < 0 restores the default: MV_TC_OPERAND_CACHE_MB if set, else three
 * eighths of the device's memory; 0 turns the images off.  The images take 16
 * bytes per particle and tensor plane (2 GB for 2^20 particles on 256^3).
 * Process-wide; applies to later computes.  No counterpart in the reference. */
void vis_set_operand_cache_limit(long long bytes);

/* For tests of the tensor form's failure path (no counterpart in the
 * reference).  Every mbarrier wait of the tensor-core kernel is bounded (2 s);
 * a wait that runs out sets a device error word, the kernel's CTAs leave their
 * loops, release their tensor memory and return, and the next synchronising
 * call on the config (vis_config_synchronize, vis_spectrum_copy_to_host, ...)
 * returns VIS_ERROR_CUDA with a message naming the wait.  This hook makes the
 * NEXT tensor-core launch of the process (one shot) bound its waits by
 * wait_limit_ns (1e5 .. 2e9) and withhold one arrival on its first pipeline
 * stage, so that the MMA thread's first wait runs out before any MMA is
 * issued.  Nothing faults; the device stays usable and later computes are
 * unaffected.  That compute's results are invalid.  Returns VIS_SUCCESS or
 * VIS_ERROR_INVALID_VALUE. */
int vis_tensor_wait_test_hook(long long wait_limit_ns);

/* ------------------------------------------------------------------ batch */
/* A batch of jobs, each one registered dataset with its own half-spectrum
 * lattice and its own views and image size (the reference renders one view of
 * one dataset per call).  vis_batch_execute runs the whole batch as one CUDA
 * graph on vis_config's stream: the spectra of every job -- one persistent
 * tensor-core launch for every separable group of every job, the plain form
 * for the rest -- then one slice-extraction launch for every view of every job,
 * then one batched cuFFT C2R per distinct image size.  The first execute (and
 * the first after vis_batch_add, or after a dataset was registered again)
 * plans, reserves memory, runs once and captures the graph; later executes
 * replay it.  Datasets must stay registered while the batch is used. */
typedef struct VisBatch VisBatch;
VisBatch* vis_batch_create(VisConfig* vis_config);
/* Adds a job; returns its index (>= 0) or -VisError.  grid_size and
 * spectrum_step as for vis_spectrum_create; view_step, cutoff_frequency and
 * number_of_samples as in VisConfig; u_axes, v_axes: number_of_views float3
 * each (copied). */
int vis_batch_add(VisBatch* batch, MeshlessDataset* meshless_dataset, int3 grid_size, float spectrum_step,
                  float2 view_step, int2 cutoff_frequency, int2 number_of_samples, int number_of_views,
                  const float3* u_axes, const float3* v_axes);
int vis_batch_execute(VisBatch* batch, int form);
/* 1 if executes replay a captured CUDA graph, 0 if they launch directly (the
 * capture failed), -1 before the first execute. */
int vis_batch_uses_graph(VisBatch* batch);
/* The job's images float[views][Nx][Ny] (device) and half-spectrum (device). */
float* vis_batch_images(VisBatch* batch, int job);
float2* vis_batch_spectrum(VisBatch* batch, int job);
int vis_batch_copy_images_to_host(VisBatch* batch, int job, float* h_images);
void vis_batch_destroy(VisBatch* batch);

/* -------------------------------------------------- image post-processing */
/* Batches of images float[images][Nx][Ny] (device, as rendered) to RGB
 * float[images][Nx][Ny][3] (device), on vis_config's stream. */
/* vis_noninteractive/main.cpp:70-84: grey = max(sample, 0) / (max over the
 * image's raw samples). */
int vis_images_normalize_to_rgb(VisConfig* vis_config, const float* d_images, int number_of_images,
                                int2 number_of_samples, float* d_rgb);
/* vis_wx/local_glsl.h:28-87 (the viewer's display shader): clamp to
 * [intensity_min, intensity_max] -> [0, 1], optional log scale, colour map
 * 1 (fire), 2 (rainbow) or 3 (ice). */
int vis_images_colormap(VisConfig* vis_config, const float* d_images, int number_of_images, int2 number_of_samples,
                        float intensity_min, float intensity_max, int log_scale, int color_map, float* d_rgb);
/* shift_meshless_dataset (include/meshless.h:66) applied to the registered
 * device copy of every group, on vis_config's stream; the host arrays are not
 * changed. */
int vis_shift_registered_dataset(VisConfig* vis_config, MeshlessDataset* meshless_dataset, float x, float y,
                                 float z);
/* Writes one host RGB image (values clamped to [0, 1], 8 bits per channel) as a
 * binary PPM, with the vertical flip the reference's JPEG writer applies
 * (vis_noninteractive/main.cpp:29-35). */
int vis_write_ppm(const char* filename, const float* h_rgb, int2 number_of_samples);

/* ----------------------------------------------------------------- timing */
enum VisTimingStage
{
    VIS_STAGE_SUM = 0,        /* plain-form Fourier-sum kernels (direct slice and 3D spectrum) */
    VIS_STAGE_SLICE = 1,      /* slice extraction into the C2R layout */
    VIS_STAGE_FFT = 2,        /* cuFFT C2R */
    VIS_STAGE_TENSOR_SUM = 3  /* tensor-core Fourier-sum kernels */
};
/* When enabled, CUDA events bracket every launch of each stage on the
 * config's stream.  vis_config_kernel_timing waits for them, returns the summed
 * device time (ms) and launch count of a stage since the last query, and
 * resets that stage. */
int vis_config_enable_kernel_timing(VisConfig* vis_config, int enable);
int vis_config_kernel_timing(VisConfig* vis_config, int stage, float* total_ms, int* launches);

/* Number of this library's own CUDA kernels launched by the process so far
 * (cuFFT's kernels are not counted). */
unsigned long long vis_kernel_launch_count(void);

/* ------------------------------------------------------- no allocation */
/* This entry point has no counterpart in the reference.  It is for callers
 * that cannot allocate device memory: code that must keep a fixed device
 * footprint, renders inside a frame loop where a cudaMalloc (and the
 * device-wide synchronisation that a cudaFree brings) is not acceptable, or
 * lives under another framework's memory pool.
 *
 * It does, for one group, the direct slice sum of vis_fourier_volume_rendering
 * (sample_fourier_transform_over_grid plus arrange_samples): writes (or, with
 * accumulate != 0, adds) step.x*step.y * sum_j w_j Phi^(r h_j)
 * exp(-2 pi i f.x_j) at every slice sample into d_arranged, the C2R layout
 * float2[number_of_samples.x][number_of_samples.y/2 + 1].  Elements that are
 * not slice samples are left untouched: zero the buffer once.  All buffers are
 * the caller's device memory (d_radii may be NULL: Phi^ at r itself).  Work is
 * enqueued on `stream`; the call does not wait.
 *
 * It allocates nothing.  Its scratch (split-K partial sums and the Phi^ table)
 * is a fixed 8 MiB array in the library's device image, which every GPU that
 * loads the library holds until the process exits; slices of more than about
 * 1.04 million samples are rejected with VIS_ERROR_INVALID_VALUE.  The first
 * call on a device looks up the array's device address (cudaGetSymbolAddress)
 * and keeps it for the life of the process, so make that first call before any
 * stream capture; the kept address does not survive a cudaDeviceReset of that
 * device, after which this entry point must not be called.  Groups with SPH or
 * Wendland radii build a 4097-cell Phi^ table per call (64 KiB of shared
 * memory), since no radius maximum is known here.  All calls share the one
 * array: calls whose work overlaps on the GPU (different streams, or different
 * host threads on one device) race and must be serialised by the caller.
 * Returns VIS_SUCCESS or a VisError code. */
int vis_fourier_slice_sum_noalloc(const Constraint* d_constraints, const float* d_radii, int number_of_terms,
                                  BasisFunctionId basis_function_id, float2 step_size, int2 cutoff_frequency,
                                  float3 u_axis, float3 v_axis, int2 number_of_samples, float2* d_arranged,
                                  int accumulate, cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif
