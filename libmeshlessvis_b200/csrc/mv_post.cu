// Headless image post-processing after the C2R: the reference's display and
// file-output steps, restated as CUDA kernels over batches of images.
//
//   vis_images_normalize_to_rgb  vis_noninteractive/main.cpp:70-84: per image,
//       m = max over the raw samples (starting from sample 0), negatives
//       clamped to 0, grey RGB = sample / m.
//   vis_images_colormap          vis_wx/local_glsl.h:28-87 (fragment shader of
//       the interactive viewer): a = max(0, (a - min) / (max - min)); with log
//       scale a = (log(alpha a + eps) - log(eps)) / (log(alpha + eps) - log(eps)),
//       eps = 1e-3, alpha = 0.01; then a piecewise-linear colour map with 5
//       knots (maps 1 "fire", 2 "rainbow", 3 "ice"; above the last knot the
//       last colour).
//   vis_shift_registered_dataset shift_meshless_dataset (meshless.cpp:68-84) on
//       the registered device copy, so a frame loop need not re-register.
//   vis_write_ppm                binary PPM (P6) writer on the host, in place of
//       the reference's Magick++ JPEG writer (no image library on the target);
//       rows are written top row first after the same vertical flip the
//       reference applies (main.cpp:31).
// All image batches are float[images][Nx][Ny] with x slow, as vis_copy_to_host
// returns them; RGB outputs are float[images][Nx][Ny][3].
#include <cmath>
#include <cstdio>
#include <vector>

#include "meshless_vis_b200.h"
#include "mv_internal.h"

namespace mv {
namespace {

// Order-preserving map of a float to an unsigned int (for atomicMax).
__device__ __forceinline__ unsigned int ordered(float f) {
    const unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unordered(unsigned int u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

__global__ void image_max_kernel(const float* __restrict__ img, long long per_image, unsigned int* out_max) {
    const int image = blockIdx.y;
    const float* p = img + (size_t)image * per_image;
    float m = p[0];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < per_image;
         i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, p[i]);
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float wm[32];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        float v = threadIdx.x < (blockDim.x >> 5) ? wm[threadIdx.x] : p[0];
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (threadIdx.x == 0) atomicMax(out_max + image, ordered(v));
    }
}

__global__ void init_max_kernel(unsigned int* out_max, int images) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < images) out_max[i] = 0u;  // below every ordered float
}

__global__ void normalize_rgb_kernel(const float* __restrict__ img, long long per_image, int images,
                                     const unsigned int* __restrict__ maxes, float* __restrict__ rgb) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= per_image * images) return;
    const float m = unordered(maxes[q / per_image]);
    float a = img[q];
    if (a < 0.f) a = 0.f;
    const float g = a / m;
    rgb[3 * q] = g;
    rgb[3 * q + 1] = g;
    rgb[3 * q + 2] = g;
}

struct Knots {
    float x[5];
    float c[5][3];
};

__host__ __device__ inline Knots color_knots(int map) {
    if (map == 2) return Knots{{0.f, 0.25f, 0.5f, 0.75f, 1.f},
                               {{0, 0, 1}, {0, 1, 1}, {0, 1, 0}, {1, 1, 0}, {1, 0, 0}}};
    if (map == 3) return Knots{{0.f, 0.475f, 0.694f, 0.745f, 1.f},
                               {{0, 0, 0}, {0.f, 0.004f, 0.686f}, {0.f, 0.42f, 1.f}, {0.f, 0.518f, 1.f}, {1, 1, 1}}};
    return Knots{{0.f, 0.475f, 0.694f, 0.745f, 1.f},
                 {{0, 0, 0}, {0.686f, 0.004f, 0.f}, {1.f, 0.42f, 0.f}, {1.f, 0.518f, 0.f}, {1, 1, 1}}};
}

__global__ void colormap_kernel(const float* __restrict__ img, long long count, float imin, float imax, int log_scale,
                                Knots k, float* __restrict__ rgb) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    float a = fmaxf(0.f, (img[q] - imin) / (imax - imin));
    if (log_scale) {
        const float eps = 1e-3f, alpha = 0.01f;
        a = (-logf(eps) + logf(alpha * a + eps)) / (logf(alpha + eps) - logf(eps));
    }
    float r = k.c[4][0], g = k.c[4][1], b = k.c[4][2];
    for (int i = 1; i < 5; ++i) {
        if (a <= k.x[i]) {
            const float d = k.x[i] - k.x[i - 1];
            const float wi = (a - k.x[i - 1]) / d, wl = (k.x[i] - a) / d;
            r = wi * k.c[i][0] + wl * k.c[i - 1][0];
            g = wi * k.c[i][1] + wl * k.c[i - 1][1];
            b = wi * k.c[i][2] + wl * k.c[i - 1][2];
            break;
        }
    }
    rgb[3 * q] = r;
    rgb[3 * q + 1] = g;
    rgb[3 * q + 2] = b;
}

__global__ void shift_kernel(float4* p, int n, float dx, float dy, float dz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = p[i];
    v.x += dx;
    v.y += dy;
    v.z += dz;
    p[i] = v;
}

}  // namespace

int config_stream_and_scratch(VisConfig* c, cudaStream_t* stream, void** scratch, size_t bytes);  // mv_api.cu

}  // namespace mv

using namespace mv;

extern "C" {

int vis_images_normalize_to_rgb(VisConfig* vis_config, const float* d_images, int number_of_images,
                                int2 number_of_samples, float* d_rgb) {
    const long long per_image = (long long)number_of_samples.x * number_of_samples.y;
    if (!d_images || !d_rgb || number_of_images < 0 || per_image <= 0)
        return set_error(kInvalidValue, "vis_images_normalize_to_rgb: bad arguments");
    if (number_of_images == 0) return kOk;
    cudaStream_t stream;
    void* scratch = nullptr;
    int rc = config_stream_and_scratch(vis_config, &stream, &scratch, sizeof(unsigned int) * number_of_images);
    if (rc != kOk) return rc;
    unsigned int* maxes = static_cast<unsigned int*>(scratch);
    init_max_kernel<<<(number_of_images + 255) / 256, 256, 0, stream>>>(maxes, number_of_images);
    count_launch();
    const int blocks_x = (int)std::min<long long>(64, (per_image + 255) / 256);
    image_max_kernel<<<dim3(blocks_x, number_of_images), 256, 0, stream>>>(d_images, per_image, maxes);
    count_launch();
    const long long count = per_image * number_of_images;
    normalize_rgb_kernel<<<(unsigned)((count + 255) / 256), 256, 0, stream>>>(d_images, per_image, number_of_images,
                                                                              maxes, d_rgb);
    count_launch();
    return check_cuda(cudaGetLastError(), "vis_images_normalize_to_rgb");
}

int vis_images_colormap(VisConfig* vis_config, const float* d_images, int number_of_images, int2 number_of_samples,
                        float intensity_min, float intensity_max, int log_scale, int color_map, float* d_rgb) {
    const long long count = (long long)number_of_samples.x * number_of_samples.y * number_of_images;
    if (!d_images || !d_rgb || number_of_images < 0 || count < 0 || color_map < 1 || color_map > 3 ||
        !(intensity_max != intensity_min))
        return set_error(kInvalidValue, "vis_images_colormap: bad arguments");
    if (count == 0) return kOk;
    cudaStream_t stream;
    int rc = config_stream_and_scratch(vis_config, &stream, nullptr, 0);
    if (rc != kOk) return rc;
    colormap_kernel<<<(unsigned)((count + 255) / 256), 256, 0, stream>>>(d_images, count, intensity_min,
                                                                         intensity_max, log_scale,
                                                                         color_knots(color_map), d_rgb);
    count_launch();
    return check_cuda(cudaGetLastError(), "vis_images_colormap");
}

int vis_shift_registered_dataset(VisConfig* vis_config, MeshlessDataset* meshless_dataset, float x, float y,
                                 float z) {
    if (!meshless_dataset || (meshless_dataset->number_of_groups > 0 && !meshless_dataset->groups))
        return set_error(kInvalidValue, "vis_shift_registered_dataset: NULL dataset");
    cudaStream_t stream;
    int rc = config_stream_and_scratch(vis_config, &stream, nullptr, 0);
    if (rc != kOk) return rc;
    for (int g = 0; g < meshless_dataset->number_of_groups; ++g) {
        const Group& grp = meshless_dataset->groups[g];
        if (grp.number_of_terms <= 0) continue;
        if (!grp.d_constraints)
            return set_error(kNotRegistered, "vis_shift_registered_dataset: group not registered");
        shift_kernel<<<(grp.number_of_terms + 255) / 256, 256, 0, stream>>>(
            reinterpret_cast<float4*>(grp.d_constraints), grp.number_of_terms, x, y, z);
        count_launch();
    }
    return check_cuda(cudaGetLastError(), "vis_shift_registered_dataset");
}

int vis_write_ppm(const char* filename, const float* h_rgb, int2 number_of_samples) {
    const int w = number_of_samples.x, h = number_of_samples.y;
    if (!filename || !h_rgb || w < 1 || h < 1) return set_error(kInvalidValue, "vis_write_ppm: bad arguments");
    FILE* f = std::fopen(filename, "wb");
    if (!f) return set_error(kInvalidValue, std::string("vis_write_ppm: cannot open ") + filename);
    std::fprintf(f, "P6\n%d %d\n255\n", w, h);
    // The reference reads the x-slow image as rows of length Nx (Magick
    // read(width, height, ...)) and flips it vertically before writing.
    std::vector<unsigned char> row((size_t)3 * w);
    for (int r = h - 1; r >= 0; --r) {
        for (int c = 0; c < w; ++c)
            for (int k = 0; k < 3; ++k) {
                float v = h_rgb[3 * ((size_t)r * w + c) + k];
                v = v < 0.f ? 0.f : (v > 1.f ? 1.f : v);
                row[3 * c + k] = (unsigned char)std::lround(v * 255.f);
            }
        if (std::fwrite(row.data(), 1, row.size(), f) != row.size()) {
            std::fclose(f);
            return set_error(kInvalidValue, "vis_write_ppm: write failed");
        }
    }
    std::fclose(f);
    return kOk;
}

}  // extern "C"
