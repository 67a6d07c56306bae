// Improved Perlin noise (K. Perlin, "Improving Noise", SIGGRAPH 2002: his published permutation,
// the quintic fade and the 12-edge gradient hash) and its fractional Brownian motion, as
// pr::PerlinNoise / FBm (src/core/noise.cpp:36-64); the procedural textures and the noise-field
// media both sample it.
#pragma once

#include "common.cuh"

namespace prb {

static __device__ const unsigned char kPerlinPerm[256] = {
    151, 160, 137, 91, 90, 15, 131, 13, 201, 95, 96, 53, 194, 233, 7, 225, 140, 36, 103, 30, 69, 142,
    8, 99, 37, 240, 21, 10, 23, 190, 6, 148, 247, 120, 234, 75, 0, 26, 197, 62, 94, 252, 219, 203, 117, 35,
    11, 32, 57, 177, 33, 88, 237, 149, 56, 87, 174, 20, 125, 136, 171, 168, 68, 175, 74, 165, 71, 134, 139,
    48, 27, 166, 77, 146, 158, 231, 83, 111, 229, 122, 60, 211, 133, 230, 220, 105, 92, 41, 55, 46, 245, 40,
    244, 102, 143, 54, 65, 25, 63, 161, 1, 216, 80, 73, 209, 76, 132, 187, 208, 89, 18, 169, 200, 196, 135,
    130, 116, 188, 159, 86, 164, 100, 109, 198, 173, 186, 3, 64, 52, 217, 226, 250, 124, 123, 5, 202, 38,
    147, 118, 126, 255, 82, 85, 212, 207, 206, 59, 227, 47, 16, 58, 17, 182, 189, 28, 42, 223, 183, 170, 213,
    119, 248, 152, 2, 44, 154, 163, 70, 221, 153, 101, 155, 167, 43, 172, 9, 129, 22, 39, 253, 19, 98, 108,
    110, 79, 113, 224, 232, 178, 185, 112, 104, 218, 246, 97, 228, 251, 34, 242, 193, 238, 210, 144, 12, 191,
    179, 162, 241, 81, 51, 145, 235, 249, 14, 239, 107, 49, 192, 214, 31, 181, 199, 106, 157, 184, 84, 204,
    176, 115, 121, 50, 45, 127, 4, 150, 254, 138, 236, 205, 93, 222, 114, 67, 29, 24, 72, 243, 141, 128, 195,
    78, 66, 215, 61, 156, 180};

__device__ __forceinline__ int perlin_perm(int i) { return kPerlinPerm[i & 255]; }
__device__ __forceinline__ float perlin_fade(float t) { return t * t * t * (t * (t * 6.f - 15.f) + 10.f); }
__device__ __forceinline__ float perlin_grad(int h, float x, float y, float z) {
    h &= 15;
    const float u = h < 8 ? x : y;
    const float v = h < 4 ? y : (h == 12 || h == 14 ? x : z);
    return ((h & 1) ? -u : u) + ((h & 2) ? -v : v);
}
__device__ __forceinline__ float perlin_lerp(float t, float a, float b) { return (1.f - t) * a + t * b; }

static __device__ float perlin_noise(V3 p) {
    const float fx = floorf(p.x), fy = floorf(p.y), fz = floorf(p.z);
    const int X = int(fx) & 255, Y = int(fy) & 255, Z = int(fz) & 255;
    const float x = p.x - fx, y = p.y - fy, z = p.z - fz;
    const float u = perlin_fade(x), v = perlin_fade(y), w = perlin_fade(z);
    const int A = perlin_perm(X) + Y, AA = perlin_perm(A) + Z, AB = perlin_perm(A + 1) + Z;
    const int B = perlin_perm(X + 1) + Y, BA = perlin_perm(B) + Z, BB = perlin_perm(B + 1) + Z;
    const float n0 = perlin_lerp(v, perlin_lerp(u, perlin_grad(perlin_perm(AA), x, y, z),
                                                perlin_grad(perlin_perm(BA), x - 1.f, y, z)),
                                 perlin_lerp(u, perlin_grad(perlin_perm(AB), x, y - 1.f, z),
                                             perlin_grad(perlin_perm(BB), x - 1.f, y - 1.f, z)));
    const float n1 = perlin_lerp(v, perlin_lerp(u, perlin_grad(perlin_perm(AA + 1), x, y, z - 1.f),
                                                perlin_grad(perlin_perm(BA + 1), x - 1.f, y, z - 1.f)),
                                 perlin_lerp(u, perlin_grad(perlin_perm(AB + 1), x, y - 1.f, z - 1.f),
                                             perlin_grad(perlin_perm(BB + 1), x - 1.f, y - 1.f, z - 1.f)));
    return perlin_lerp(w, n0, n1);
}

// Fractional Brownian motion: octaves of noise at doubling frequency and halving amplitude,
// normalised by the amplitude sum; |noise| per octave for turbulence.
static __device__ float fbm_noise(V3 p, int octaves, bool turbulence) {
    float sum = 0.f, amp = 0.5f, freq = 1.f, norm = 0.f;
    const int n = max(1, octaves);
    for (int i = 0; i < n; ++i) {
        const float v = perlin_noise(p * freq);
        sum += amp * (turbulence ? fabsf(v) : v);
        norm += amp;
        amp *= 0.5f;
        freq *= 2.f;
    }
    return sum / norm;
}

} // namespace prb
