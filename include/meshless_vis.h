/*
 * meshless_vis.h -- Fourier volume rendering API of the B200 libMeshlessVis
 * drop-in.
 *
 * Same names, VisConfig layout (the reference's CUDA-build layout) and
 * signatures as the reference's include/meshless_vis.h, so existing callers
 * (vis_noninteractive/main.cpp, vis_timing_test/main.cpp, vis_wx/main.cpp in
 * the reference) compile and link unchanged.  Differences, all compatible:
 *   - the header does not need <GL/glew.h>: GLuint is declared here;
 *   - vis_config_manual_d_image takes void* (the reference header says float2*,
 *     its implementation float*; both convert);
 *   - errors never exit(): each call records a code readable through
 *     vis_get_last_error() (meshless_vis_b200.h) and returns early.
 * The new 3D-half-spectrum path, batched views and error reporting are
 * declared in meshless_vis_b200.h.
 */
#ifndef MESHLESS_VISh
#define MESHLESS_VISh

#include "meshless.h"
#include <builtin_types.h>
#include <cufft.h>
#include <vector_functions.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned int GLuint;

/* include/meshless_vis.h:39-79 (CUDA build).  Fields prefixed with an
 * underscore are owned by the vis_config_* functions; step_size, u_axis,
 * v_axis and block_length may be written directly between renders, as the
 * reference's viewer does (vis_wx/main.cpp:711, :772, :794). */
typedef struct
{
    float2 step_size;
    int2 _cutoff_frequency;
    float3 u_axis;
    float3 v_axis;

    /* false by default (as the reference).  When true,
     * vis_fourier_volume_rendering sums, per group, only the particles whose
     * footprint square (centre (p.u, p.v), half-side h_j, 0 without radii)
     * lies inside [0, 1/(2 step.x)] x [0, 1/(2 step.y)]: the cull of
     * meshless_vis.cu:39-127, which the reference keeps disabled (:336).  The
     * registered arrays are left untouched; each render culls from the full
     * set and waits once per group for the kept count. */
    bool cull_fully_aliased_terms;

    bool _automatic_d_image;

    cufftHandle _plan;

    int2 _number_of_samples;
    int block_length;
    float _scale;
    float* _d_image;

    float2* _d_freq_image;

    int _number_of_partial_sums;

    float2* _d_freq_image_arranged;
} VisConfig;

/* include/meshless_vis.h:81-94 */
VisConfig* vis_config_create(bool automatic_d_image, float2 step_size, int2 cutoff_frequency, float3 u_axis,
                             float3 v_axis, int2 number_of_samples, int block_length, int number_of_partial_sums);
VisConfig* vis_config_get_default(void);
bool vis_config_check(VisConfig* vis_config);
void vis_config_manual_d_image(VisConfig* vis_config, void* d_image);
void vis_config_change_number_of_samples(VisConfig* vis_config, int2 number_of_samples);
void vis_config_change_cutoff_frequency(VisConfig* vis_config, int2 cutoff_frequency);
void vis_config_change_number_of_partial_sums(VisConfig* vis_config, int number_of_partial_sums);
void vis_config_destroy(VisConfig* vis_config);
void vis_config_compute_scale(VisConfig* vis_config);
void vis_register_meshless_dataset(VisConfig* vis_config, MeshlessDataset* meshless_dataset);
/* Unregistering synchronises the device and keeps the device blocks with the
 * config for its next registration of the same byte size (so that a frame
 * loop gets the same addresses back), up to the most the config had
 * registered at once; vis_config_destroy releases them. */
void vis_unregister_meshless_dataset(VisConfig* vis_config, MeshlessDataset* meshless_dataset);
/* No graphics stack on the target: records VIS_ERROR_UNSUPPORTED and returns
 * without rendering.  Use vis_config_manual_d_image for a caller-owned device
 * image instead of a GL pixel buffer. */
void vis_opengl_fourier_volume_rendering(MeshlessDataset* meshless_dataset, VisConfig* vis_config,
                                         GLuint buffer_object);
void vis_fourier_volume_rendering(MeshlessDataset* meshless_dataset, VisConfig* vis_config);
void vis_copy_to_host(VisConfig* vis_config, float* h_image);

#ifdef __cplusplus
}
#endif

#endif
