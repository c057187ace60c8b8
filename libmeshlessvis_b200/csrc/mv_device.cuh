// Device-side building blocks shared by the Fourier-sum kernels:
//   - the reference's basis-function transforms Phi^(r), in FP32 accurate to
//     ~1e-7 of Phi^(0) everywhere (and in FP64 for per-frequency factors);
//   - exact phase reduction with 32-bit fixed-point positions.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "phi_poly.h"
#include "phi_series.h"

namespace mv {

enum Basis : int { kSph = 0, kGaussian = 1, kWendland = 2, kGaussianDecaying = 3, kBasisCount = 4 };

constexpr float kPiF = 3.14159265358979323846f;
constexpr double kPi = 3.14159265358979323846;
// 2*pi / 2^32: converts a signed 32-bit fixed-point turn count to radians.
constexpr float kTwoPiOver2p32 = 1.4629180792671596e-09f;

template <int DEG>
__device__ __forceinline__ float horner(const float* c, float x) {
    float acc = c[DEG];
#pragma unroll
    for (int k = DEG - 1; k >= 0; --k) acc = fmaf(acc, x, c[k]);
    return acc;
}

// SPH transform, meshless_vis/fourier_transform.cu:31-41.  Below 0.06 the
// reference's quadratic; on [0.06, 0.5) a degree-9 polynomial in s^2 of the
// same closed form (the closed form cancels in FP32 there); above, the closed
// form with cos/sin of 2*pi*s from sincospif (exact argument reduction).
__device__ __forceinline__ float phi_sph(float s) {
    if (s < 0.06f) return fmaf(s, fmaf(s, -18.293608272337678f, -0.007968913156311f), kPiF);
    if (s < 0.5f) {
        float x = (s * s - MV_SPH_POLY_T_MID) * MV_SPH_POLY_T_INV_HALF;
        return horner<MV_SPH_POLY_DEG>(MV_SPH_POLY_C, x);
    }
    float sn, cs;
    sincospif(2.0f * s, &sn, &cs);
    float m = kPiF * s;
    float m2 = m * m;
    float m6 = m2 * m2 * m2;
    return (2.3561944901923448f / m6) * (cs - 1.0f) * (cs + m * sn - 1.0f);
}

// Wendland D3 C2 transform, meshless_vis/fourier_transform.cu:48-60.  Below
// 0.24 the reference's quadratic; on [0.24, 1) a degree-9 polynomial in s^2 of
// the closed form; above, the closed form.
__device__ __forceinline__ float phi_wendland(float s) {
    if (s < 0.24f) return fmaf(s, fmaf(s, -0.370530218163545f, -0.002379178586124f), 0.299199300341890f);
    if (s < 1.0f) {
        float x = (s * s - MV_WENDLAND_POLY_T_MID) * MV_WENDLAND_POLY_T_INV_HALF;
        return horner<MV_WENDLAND_POLY_DEG>(MV_WENDLAND_POLY_C, x);
    }
    float sn, cs;
    sincospif(2.0f * s, &sn, &cs);
    float m = kPiF * s;
    float m2 = m * m;
    float m4 = m2 * m2;
    return ((kPiF * 7.5f) / (m4 * m4)) * (4.0f * m2 - 6.0f + (6.0f - m2) * cs + 4.5f * m * sn);
}

// log2(e) * pi: exp(+-pi s^2) = exp2(+-kPiLog2e s^2).
constexpr float kPiLog2e = 4.53236014182719380962f;

template <int BASIS>
__device__ __forceinline__ float phi(float s) {
    if constexpr (BASIS == kSph) return phi_sph(s);
    else if constexpr (BASIS == kGaussian) return exp2f(kPiLog2e * s * s);  // exp(+pi s^2), as the reference
    else if constexpr (BASIS == kWendland) return phi_wendland(s);
    else return exp2f(-kPiLog2e * s * s);
}

// FP64 versions, used once per frequency (for groups without radii, where
// Phi^ factors out of the sum).  Same branch points and constants as above.
__device__ __forceinline__ double phi_fp64(int basis, double r) {
    switch (basis) {
    case kSph:
        if (r >= (double)0.06f) {
            double m = kPi * r, c = cos(2.0 * m), s = sin(2.0 * m);
            return (2.3561944901923448 / (m * m * m * m * m * m)) * (c - 1.0) * (c + m * s - 1.0);
        }
        return kPi + r * (-0.007968913156311 + r * (-18.293608272337678));
    case kGaussian: return exp(kPi * r * r);
    case kWendland:
        if (r >= (double)0.24f) {
            double m = kPi * r, c = cos(2.0 * m), s = sin(2.0 * m);
            double m2 = m * m, m4 = m2 * m2;
            return ((kPi * 7.5) / (m4 * m4)) * (4.0 * m2 - 6.0 + (6.0 - m2) * c + 4.5 * m * s);
        }
        return 0.299199300341890 + r * (-0.002379178586124 + r * (-0.370530218163545));
    default: return exp(-kPi * r * r);
    }
}

// The reference's branch point of SPH (0.06f) and Wendland (0.24f).
__host__ __device__ __forceinline__ double phi_branch_point(int basis) {
    return basis == kSph ? (double)0.06f : (double)0.24f;
}

// SPH and Wendland without the branch: the closed form at every r (smooth),
// from its power series below the branch point (phi_series.h), where the
// closed form cancels, and the closed form above.
__device__ __forceinline__ double phi_smooth_fp64(int basis, double r) {
    if (r >= phi_branch_point(basis)) return phi_fp64(basis, r);
    const double m = kPi * r, m2 = m * m;
    const double* c = basis == kSph ? MV_SPH_SERIES : MV_WENDLAND_SERIES;
    double acc = c[MV_PHI_SERIES_TERMS - 1];
    for (int n = MV_PHI_SERIES_TERMS - 2; n >= 0; --n) acc = fma(acc, m2, c[n]);
    return (basis == kSph ? 2.3561944901923448 : kPi * 7.5) * acc;
}

// What the branch adds: the reference's quadratic fit minus the smooth closed
// form below the branch point, zero above (Phi^ = smooth + kink).
__device__ __forceinline__ double phi_kink_fp64(int basis, double r) {
    if (r >= phi_branch_point(basis)) return 0.0;
    return phi_fp64(basis, r) - phi_smooth_fp64(basis, r);
}

// Bin of radius h among nb bins with edges e[0..nb]: the largest i with
// e[i] <= h, clamped to [0, nb) (the h-binned tensor form's classification;
// the same rule at registration sizes the bins).
__device__ __forceinline__ int hbin_of(const float* e, int nb, float h) {
    if (nb <= 1 || !(h >= e[1])) return 0;
    if (h >= e[nb - 1]) return nb - 1;
    int lo = 0, hi = nb;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (e[mid] <= h) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Fixed-point turn count of q (in turns): round(q * 2^32) mod 2^32.  Exact for
// |q| < 2^31.  Products with integer wavenumbers then wrap mod 2^32, which is
// exactly the phase reduction mod one turn.
__device__ __forceinline__ uint32_t fixed_turns(double q) {
    return (uint32_t)(unsigned long long)__double2ll_rn(q * 4294967296.0);
}

// Radians in [-pi, pi) of a 32-bit fixed-point turn count.
__device__ __forceinline__ float turns_to_radians(uint32_t ph) { return (float)(int32_t)ph * kTwoPiOver2p32; }

}  // namespace mv
