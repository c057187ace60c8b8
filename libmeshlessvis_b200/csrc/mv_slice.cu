// Fourier-slice extraction from the 3D half-spectrum into the 2D C2R layout,
// batched over views.  No reference twin: the reference recomputes the direct
// sum per view (meshless_vis/fourier_transform.cu:67-141); its arrange_samples
// (meshless_vis/meshless_vis.cu:318-332) and the cudaMemset before it (:338)
// are fused here: every element of [view][nx][ny/2+1] is written exactly once.
//
// Element (ix, y) of a view holds slice sample x = ix (ix < cx) or ix - nx
// (ix > nx - cx), y < cy; all other elements (including arrange_samples's
// dropped u-Nyquist x == cx) are zero.  The sample is the trilinear
// interpolation of the spectrum at p = (step.x x u + step.y y v) / step3,
// reflected to conj(F(-p)) when p_z < 0, corners outside the stored lattice
// reading zero, times step.x * step.y.
//
// Bandwidth: per sample 8 corner loads of 8 B (mostly L2 hits for adjacent
// samples) and one 8 B store.
#include "mv_internal.h"

namespace mv {

namespace {

__device__ __forceinline__ float2 corner(const float2* __restrict__ spec, int gx, int gy, int lz, int i, int j, int l) {
    const int ii = i + (gx >> 1), jj = j + (gy >> 1);
    if ((unsigned)ii >= (unsigned)gx || (unsigned)jj >= (unsigned)gy || (unsigned)l >= (unsigned)lz)
        return make_float2(0.f, 0.f);
    return __ldg(spec + ((size_t)ii * gy + jj) * lz + l);
}

__global__ void slice_extract_kernel(SliceRequest r) {
    const int h = r.ny / 2 + 1;
    const long long per_view = (long long)r.nx * h;
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= per_view * r.number_of_views) return;
    const int view = (int)(q / per_view);
    const int e = (int)(q % per_view);
    const int ix = e / h, y = e % h;

    float2 out = make_float2(0.f, 0.f);
    int x = 0;
    bool valid = y < r.cy;
    if (ix < r.cx) x = ix;
    else if (ix > r.nx - r.cx) x = ix - r.nx;
    else valid = false;

    if (valid) {
        const float* v = r.views + 8 * view;
        const float fu = v[6] * (float)x, fv = v[7] * (float)y;
        float p0 = (fu * v[0] + fv * v[3]) * r.inv_step;
        float p1 = (fu * v[1] + fv * v[4]) * r.inv_step;
        float p2 = (fu * v[2] + fv * v[5]) * r.inv_step;
        const bool conj = p2 < 0.f;
        if (conj) {
            p0 = -p0;
            p1 = -p1;
            p2 = -p2;
        }
        const float f0 = floorf(p0), f1 = floorf(p1), f2 = floorf(p2);
        const float t0 = p0 - f0, t1 = p1 - f1, t2 = p2 - f2;
        const int i0 = (int)f0, j0 = (int)f1, l0 = (int)f2;
        const int lz = r.gz / 2 + 1;
        float re = 0.f, im = 0.f;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int di = c & 1, dj = (c >> 1) & 1, dl = (c >> 2) & 1;
            const float w = (di ? t0 : 1.f - t0) * (dj ? t1 : 1.f - t1) * (dl ? t2 : 1.f - t2);
            const float2 s = corner(r.spectrum, r.gx, r.gy, lz, i0 + di, j0 + dj, l0 + dl);
            re = fmaf(w, s.x, re);
            im = fmaf(w, s.y, im);
        }
        const float scale = v[6] * v[7];
        out = make_float2(re * scale, (conj ? -im : im) * scale);
    }
    r.arranged[q] = out;
}

// Batched form: every view has its own spectrum and image size; thread q finds
// its view by binary search over the views' element offsets.
__global__ void slice_extract_batch_kernel(const SliceView* __restrict__ views, int n_views, long long total) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= total) return;
    int lo = 0, hi = n_views - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (views[mid].element_offset <= q) lo = mid;
        else hi = mid - 1;
    }
    const SliceView& V = views[lo];
    const int h = V.ny / 2 + 1;
    const int e = (int)(q - V.element_offset);
    const int ix = e / h, y = e % h;

    float2 out = make_float2(0.f, 0.f);
    int x = 0;
    bool valid = y < V.cy;
    if (ix < V.cx) x = ix;
    else if (ix > V.nx - V.cx) x = ix - V.nx;
    else valid = false;

    if (valid) {
        const float fu = V.step[0] * (float)x, fv = V.step[1] * (float)y;
        float p0 = (fu * V.u[0] + fv * V.v[0]) * V.inv_step;
        float p1 = (fu * V.u[1] + fv * V.v[1]) * V.inv_step;
        float p2 = (fu * V.u[2] + fv * V.v[2]) * V.inv_step;
        const bool conj = p2 < 0.f;
        if (conj) {
            p0 = -p0;
            p1 = -p1;
            p2 = -p2;
        }
        const float f0 = floorf(p0), f1 = floorf(p1), f2 = floorf(p2);
        const float t0 = p0 - f0, t1 = p1 - f1, t2 = p2 - f2;
        const int i0 = (int)f0, j0 = (int)f1, l0 = (int)f2;
        const int lz = V.gz / 2 + 1;
        float re = 0.f, im = 0.f;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int di = c & 1, dj = (c >> 1) & 1, dl = (c >> 2) & 1;
            const float w = (di ? t0 : 1.f - t0) * (dj ? t1 : 1.f - t1) * (dl ? t2 : 1.f - t2);
            const float2 s = corner(V.spectrum, V.gx, V.gy, lz, i0 + di, j0 + dj, l0 + dl);
            re = fmaf(w, s.x, re);
            im = fmaf(w, s.y, im);
        }
        const float scale = V.step[0] * V.step[1];
        out = make_float2(re * scale, (conj ? -im : im) * scale);
    }
    V.arranged[e] = out;
}

}  // namespace

int launch_slice_extract_batch(const SliceView* d_views, int number_of_views, long long total_elements,
                               cudaStream_t stream, KernelTimer* timer) {
    if (number_of_views <= 0 || total_elements <= 0) return kOk;
    timer_begin(timer, 1, stream);
    slice_extract_batch_kernel<<<(unsigned)((total_elements + 255) / 256), 256, 0, stream>>>(d_views, number_of_views,
                                                                                              total_elements);
    count_launch();
    timer_end(timer, 1, stream);
    return check_cuda(cudaGetLastError(), "slice_extract_batch_kernel launch");
}

int launch_slice_extract(const SliceRequest& req, KernelTimer* timer) {
    const long long count = (long long)req.nx * (req.ny / 2 + 1) * req.number_of_views;
    if (count <= 0) return kOk;
    if (count > (1LL << 40)) return set_error(kInvalidValue, "too many slice samples");
    timer_begin(timer, 1, req.stream);
    slice_extract_kernel<<<(unsigned)((count + 255) / 256), 256, 0, req.stream>>>(req);
    count_launch();
    timer_end(timer, 1, req.stream);
    return check_cuda(cudaGetLastError(), "slice_extract_kernel launch");
}

}  // namespace mv
