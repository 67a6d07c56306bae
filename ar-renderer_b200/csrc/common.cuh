// Device math shared by every kernel of libprender_gpu: vectors, frames, the PCG32 stream,
// sampled spectra at the 4 hero wavelengths and spectral-table lookups.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/prgpu_api.h"

namespace prb {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kInv2Pi = 0.15915494309189533577f;
constexpr float kInv4Pi = 0.07957747154594766788f;
constexpr float kPiOver2 = 1.57079632679489661923f;
constexpr float kPiOver4 = 0.78539816339744830961f;
constexpr float kOneMinusEps = 0x1.fffffep-1f;
constexpr float kInf = __builtin_huge_valf();

struct V3 {
    float x, y, z;
};
__host__ __device__ __forceinline__ V3 mk(float x, float y, float z) { return {x, y, z}; }
__host__ __device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__host__ __device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__host__ __device__ __forceinline__ float len2(V3 a) { return dot(a, a); }
__device__ __forceinline__ float len(V3 a) { return sqrtf(len2(a)); }
__device__ __forceinline__ V3 normalize(V3 a) { return a * (1.f / len(a)); }
__host__ __device__ __forceinline__ V3 f3(const prgpu::Float3 &f) { return {f.x, f.y, f.z}; }
__device__ __forceinline__ float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ float sqr(float x) { return x * x; }
__device__ __forceinline__ float safe_sqrt(float x) { return sqrtf(fmaxf(0.f, x)); }
__device__ __forceinline__ V3 face_forward(V3 n, V3 v) { return dot(n, v) < 0.f ? -n : n; }
__device__ __forceinline__ float max_abs3(V3 p) { return fmaxf(fabsf(p.x), fmaxf(fabsf(p.y), fabsf(p.z))); }

// Offset scale for spawned rays: 5e-5 * max(1, |p|_inf)  (src/scene/interaction.h:20).
__device__ __forceinline__ float ray_eps(V3 p) { return 5e-5f * fmaxf(1.f, max_abs3(p)); }
// Ray origin pushed off a surface towards w (src/scene/interaction.h:43-50).
__device__ __forceinline__ V3 offset_origin(V3 p, V3 n, V3 w) {
    float e = ray_eps(p);
    return p + (dot(w, n) < 0.f ? -n : n) * e;
}

// Orthonormal frame with z = n (Duff et al. 2017 branchless basis), and the tangent-aligned frame
// used by BSDFs (x from the shading tangent, Gram-Schmidt against z).
struct Frame {
    V3 x, y, z;
    __device__ V3 to_local(V3 v) const { return {dot(v, x), dot(v, y), dot(v, z)}; }
    __device__ V3 from_local(V3 v) const { return x * v.x + y * v.y + z * v.z; }
};
__device__ __forceinline__ Frame frame_from_z(V3 z) {
    float s = copysignf(1.f, z.z);
    float a = -1.f / (s + z.z);
    float b = z.x * z.y * a;
    return {{1.f + s * z.x * z.x * a, s * b, -s * z.x}, {b, s + z.y * z.y * a, -z.y}, z};
}
__device__ __forceinline__ Frame frame_from_xz(V3 xin, V3 z) {
    V3 x = xin - z * dot(xin, z);
    float l2 = len2(x);
    if (l2 < 1e-12f || !isfinite(l2)) return frame_from_z(z);
    x = x * rsqrtf(l2);
    return {x, cross(z, x), z};
}

// ---------------------------------------------------------------------------------------------
// PCG32 (O'Neill) with the MixBits finaliser; per-(pixel, sample) streams seeded as the reference
// GPU module does (src/gpu/prender_gpu.cpp:1507), so sample index drives the stream.

__host__ __device__ __forceinline__ uint64_t mix_bits(uint64_t v) {
    v ^= (v >> 31);
    v *= 0x7fb5d329728ea185ULL;
    v ^= (v >> 27);
    v *= 0x81dadef4bc2dd44dULL;
    v ^= (v >> 33);
    return v;
}

struct Pcg {
    uint64_t state, inc;
    __device__ __forceinline__ uint32_t next() {
        uint64_t old = state;
        state = old * 0x5851f42d4c957f2dULL + inc;
        uint32_t xs = uint32_t(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = uint32_t(old >> 59u);
        return __funnelshift_r(xs, xs, rot);
    }
    __device__ __forceinline__ float uniform() { return fminf(kOneMinusEps, float(next()) * 0x1p-32f); }
    __device__ __forceinline__ void seed(uint64_t seq, uint64_t offset) {
        state = 0;
        inc = (seq << 1u) | 1u;
        next();
        state += offset;
        next();
    }
};

__device__ __forceinline__ Pcg pixel_sample_stream(uint32_t pixel, uint64_t sampleIndex, uint64_t seed) {
    Pcg r;
    r.seed(mix_bits(uint64_t(pixel) * 0x9E3779B97F4A7C15ull ^ seed), mix_bits(sampleIndex + 1));
    return r;
}

// ---------------------------------------------------------------------------------------------
// Sampled spectra at 4 hero wavelengths

struct SS {
    float v[4];
};
__device__ __forceinline__ SS splat(float c) { return {{c, c, c, c}}; }
__device__ __forceinline__ SS operator*(SS a, SS b) {
    return {{a.v[0] * b.v[0], a.v[1] * b.v[1], a.v[2] * b.v[2], a.v[3] * b.v[3]}};
}
__device__ __forceinline__ SS operator*(SS a, float s) { return {{a.v[0] * s, a.v[1] * s, a.v[2] * s, a.v[3] * s}}; }
__device__ __forceinline__ SS operator+(SS a, SS b) {
    return {{a.v[0] + b.v[0], a.v[1] + b.v[1], a.v[2] + b.v[2], a.v[3] + b.v[3]}};
}
__device__ __forceinline__ float max_c(SS a) { return fmaxf(fmaxf(a.v[0], a.v[1]), fmaxf(a.v[2], a.v[3])); }
__device__ __forceinline__ bool nonzero(SS a) { return a.v[0] != 0.f || a.v[1] != 0.f || a.v[2] != 0.f || a.v[3] != 0.f; }
__device__ __forceinline__ float4 to_f4(SS a) { return make_float4(a.v[0], a.v[1], a.v[2], a.v[3]); }
__device__ __forceinline__ SS from_f4(float4 a) { return {{a.x, a.y, a.z, a.w}}; }

// Hero wavelengths and their pdfs. Terminating the secondaries keeps only the hero with its pdf
// divided by 4 (src/core/spectrum.h:111-115).
struct Lambda {
    float l[4], pdf[4];
    __device__ bool terminated() const { return pdf[1] == 0.f && pdf[2] == 0.f && pdf[3] == 0.f; }
    __device__ void terminate_secondary() {
        if (terminated()) return;
        pdf[1] = pdf[2] = pdf[3] = 0.f;
        pdf[0] *= 0.25f;
    }
};

// pbrt-v4 visible-wavelength importance sampling with 4 stratified rotations of one u
// (src/core/spectrum.cpp:11-18, 32-41).
__device__ __forceinline__ Lambda sample_visible(float u) {
    Lambda w;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float up = u + float(i) * 0.25f;
        if (up > 1.f) up -= 1.f;
        float l = 538.f - 138.888889f * atanhf(0.85691062f - 1.82750197f * up);
        l = clampf(l, 360.f, 830.f);
        w.l[i] = l;
        float c = coshf(0.0072f * (l - 538.f));
        w.pdf[i] = 0.0039398042f / (c * c);
    }
    return w;
}

// CIE 1931 matching functions, multi-lobe Gaussian fit of Wyman, Sloan & Shirley (JCGT 2013),
// the same fit the reference uses (src/core/spectrum.cpp:47-57).
__device__ __forceinline__ float g_lobe(float x, float mu, float s1, float s2) {
    float t = (x - mu) / (x < mu ? s1 : s2);
    return __expf(-0.5f * t * t);
}
__device__ __forceinline__ float cie_x(float l) {
    return 1.056f * g_lobe(l, 599.8f, 37.9f, 31.0f) + 0.362f * g_lobe(l, 442.0f, 16.0f, 26.7f) -
           0.065f * g_lobe(l, 501.1f, 20.4f, 26.2f);
}
__device__ __forceinline__ float cie_y(float l) {
    return 0.821f * g_lobe(l, 568.8f, 46.9f, 40.5f) + 0.286f * g_lobe(l, 530.9f, 16.3f, 31.1f);
}
__device__ __forceinline__ float cie_z(float l) {
    return 1.217f * g_lobe(l, 437.0f, 11.8f, 36.0f) + 0.681f * g_lobe(l, 459.0f, 26.0f, 13.8f);
}

// Tabulated spectrum (95 samples at 5 nm from 360 nm), linear interpolation
// (src/gpu/gpu_api.h:19-21; the host tabulates as src/integrators/gpu_path.cpp:148-153 does).
__device__ __forceinline__ float tab(const float *__restrict__ spectra, int id, float lambda) {
    if (id < 0) return 0.f;
    float x = (lambda - prgpu::kSpectrumMin) * (1.f / prgpu::kSpectrumStep);
    x = clampf(x, 0.f, float(prgpu::kSpectrumSamples - 1) - 1e-3f);
    int i = int(x);
    float t = x - float(i);
    const float *v = spectra + size_t(id) * prgpu::kSpectrumSamples;
    return __ldg(v + i) * (1.f - t) + __ldg(v + i + 1) * t;
}
__device__ __forceinline__ SS tab4(const float *__restrict__ spectra, int id, const Lambda &w) {
    return {{tab(spectra, id, w.l[0]), tab(spectra, id, w.l[1]), tab(spectra, id, w.l[2]), tab(spectra, id, w.l[3])}};
}

// sin and cos of a float angle evaluated in double precision and rounded once: the correctly
// rounded float values in all but vanishingly rare cases, as the host C library returns them.
// Used where sampled directions feed sharp lobes (microfacet peaks), so that a one-ulp
// difference in the angle's sine is not amplified.
__device__ __forceinline__ void sincos_rn(float x, float *s, float *c) {
    double sd, cd;
    sincos(double(x), &sd, &cd);
    *s = float(sd);
    *c = float(cd);
}

__device__ __forceinline__ float power_heuristic(float f, float g) {
    float f2 = f * f;
    if (isinf(f2)) return 1.f;
    if (f == 0.f && g == 0.f) return 0.f;
    return f2 / (f2 + g * g);
}

} // namespace prb
