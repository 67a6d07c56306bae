// Participating media on the device: homogeneous transmittance and the heterogeneous (voxel grid)
// medium of pr::GridMedium -- trilinear cell-centred density (src/media/medium.cpp:117-128),
// clipping of the segment to the grid bounds in medium space (medium.cpp:182-203), ratio tracking
// with Russian roulette for shadow transmittance (medium.cpp:205-230) and spectral tracking for
// free-flight sampling (medium.cpp:232-285). The reference tracks against the global majorant
// maxDensity * max(sigma_t); these walk a table of per-macro-cell majorants instead (the same
// estimators with a piecewise-constant rate, so the same expectations, with far fewer null
// collisions in sparse media).
#pragma once

#include "noise.cuh"
#include "scene.cuh"

namespace prb {

__device__ __forceinline__ bool is_grid(const DevScene &s, int medium) { return medium >= s.mediumCount; }

__device__ __forceinline__ SS homogeneous_tr(const DevScene &s, int medium, const Lambda &lam, float dist) {
    const prgpu::Medium &md = s.media[medium];
    SS st = (tab4(s.spectra, md.sigmaA, lam) + tab4(s.spectra, md.sigmaS, lam)) * md.scale;
    SS r;
#pragma unroll
    for (int i = 0; i < 4; ++i) r.v[i] = isinf(dist) ? (st.v[i] > 0.f ? 0.f : 1.f) : expf(-st.v[i] * dist);
    return r;
}

__device__ __forceinline__ float grid_at(const DevGrid &g, int x, int y, int z) {
    x = min(max(x, 0), g.nx - 1);
    y = min(max(y, 0), g.ny - 1);
    z = min(max(z, 0), g.nz - 1);
    return __ldg(g.density + (size_t(z) * g.ny + y) * g.nx + x);
}

__device__ __forceinline__ float lerpf(float t, float a, float b) { return (1.f - t) * a + t * b; }

// pr::NoiseField::Density (medium.cpp:168-177) at a medium-space point inside the bounds: the
// remapped fBm, faded towards the bounds' inscribed ellipsoid, thresholded and sharpened.
static __device__ __noinline__ float noise_field_density(const DevGrid &g, V3 p) {
    const V3 q = (p + mk(g.noiseOffset[0], g.noiseOffset[1], g.noiseOffset[2])) * g.noiseFrequency;
    float n = 0.5f + 0.5f * fbm_noise(q, g.noiseOctaves, false) * 1.4f;
    if (g.noiseFalloff) {
        const float ox = (p.x - g.bmin[0]) / (g.bmax[0] - g.bmin[0]) * 2.f - 1.f;
        const float oy = (p.y - g.bmin[1]) / (g.bmax[1] - g.bmin[1]) * 2.f - 1.f;
        const float oz = (p.z - g.bmin[2]) / (g.bmax[2] - g.bmin[2]) * 2.f - 1.f;
        n *= clampf(1.f - (ox * ox + oy * oy + oz * oz), 0.f, 1.f);
    }
    return clampf((n - g.noiseThreshold) * g.noiseSharpness, 0.f, 1.f);
}

// Density of an index-space grid (a densified NanoVDB grid; NanoVDBField::Density,
// nanovdb_field.cpp:27-39): trilinear between voxel centres at integer coordinates, the background
// 0 beyond the array, clamped at 0.
static __device__ __noinline__ float indexed_density(const DevGrid &g, V3 p) {
    const float x = p.x - float(g.org[0]), y = p.y - float(g.org[1]), z = p.z - float(g.org[2]);
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const int x0 = int(fx), y0 = int(fy), z0 = int(fz);
    const float dx = x - fx, dy = y - fy, dz = z - fz;
    auto v = [&](int i, int j, int k) {
        i += x0;
        j += y0;
        k += z0;
        if (i < 0 || j < 0 || k < 0 || i >= g.nx || j >= g.ny || k >= g.nz) return 0.f;
        return __ldg(g.density + (size_t(k) * g.ny + j) * g.nx + i);
    };
    const float c00 = lerpf(dx, v(0, 0, 0), v(1, 0, 0)), c10 = lerpf(dx, v(0, 1, 0), v(1, 1, 0));
    const float c01 = lerpf(dx, v(0, 0, 1), v(1, 0, 1)), c11 = lerpf(dx, v(0, 1, 1), v(1, 1, 1));
    return fmaxf(0.f, lerpf(dz, lerpf(dy, c00, c10), lerpf(dy, c01, c11)));
}

// Density at a medium-space point: 0 outside the bounds, trilinear between cell centres inside
// (or the noise field's, or the index-space grid's).
__device__ __forceinline__ float grid_density(const DevGrid &g, V3 p) {
    if (g.boundless) return noise_field_density(g, p);
    if (!(p.x >= g.bmin[0] && p.x <= g.bmax[0] && p.y >= g.bmin[1] && p.y <= g.bmax[1] && p.z >= g.bmin[2] &&
          p.z <= g.bmax[2]))
        return 0.f;
    if (g.noise) return noise_field_density(g, p);
    if (g.indexed) return indexed_density(g, p);
    float ox = p.x - g.bmin[0], oy = p.y - g.bmin[1], oz = p.z - g.bmin[2];
    if (g.bmax[0] > g.bmin[0]) ox /= g.bmax[0] - g.bmin[0];
    if (g.bmax[1] > g.bmin[1]) oy /= g.bmax[1] - g.bmin[1];
    if (g.bmax[2] > g.bmin[2]) oz /= g.bmax[2] - g.bmin[2];
    float x = ox * g.nx - 0.5f, y = oy * g.ny - 0.5f, z = oz * g.nz - 0.5f;
    int x0 = int(floorf(x)), y0 = int(floorf(y)), z0 = int(floorf(z));
    float dx = x - x0, dy = y - y0, dz = z - z0;
    float c00 = lerpf(dx, grid_at(g, x0, y0, z0), grid_at(g, x0 + 1, y0, z0));
    float c10 = lerpf(dx, grid_at(g, x0, y0 + 1, z0), grid_at(g, x0 + 1, y0 + 1, z0));
    float c01 = lerpf(dx, grid_at(g, x0, y0, z0 + 1), grid_at(g, x0 + 1, y0, z0 + 1));
    float c11 = lerpf(dx, grid_at(g, x0, y0 + 1, z0 + 1), grid_at(g, x0 + 1, y0 + 1, z0 + 1));
    return lerpf(dz, lerpf(dy, c00, c10), lerpf(dy, c01, c11));
}

// Medium-space ray of the world segment [0, tMax) clipped to the bounds; false when it misses.
__device__ __forceinline__ bool grid_clip(const DevGrid &g, V3 o, V3 d, float tMax, V3 *mo, V3 *md, float *t0,
                                          float *t1) {
    const float *m = g.w2m;
    *mo = mk(m[0] * o.x + m[1] * o.y + m[2] * o.z + m[3], m[4] * o.x + m[5] * o.y + m[6] * o.z + m[7],
             m[8] * o.x + m[9] * o.y + m[10] * o.z + m[11]);
    *md = mk(m[0] * d.x + m[1] * d.y + m[2] * d.z, m[4] * d.x + m[5] * d.y + m[6] * d.z,
             m[8] * d.x + m[9] * d.y + m[10] * d.z);
    *t0 = 0.f;
    *t1 = tMax;
    // A field without bounds fills every finite segment (GridMedium::Clip, medium.cpp:182-188).
    if (g.boundless) return isfinite(tMax);
    float oo[3] = {mo->x, mo->y, mo->z}, dd[3] = {md->x, md->y, md->z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float inv = 1.f / dd[a];
        float tn = (g.bmin[a] - oo[a]) * inv, tf = (g.bmax[a] - oo[a]) * inv;
        if (tn > tf) {
            float t = tn;
            tn = tf;
            tf = t;
        }
        if (isnan(tn) || isnan(tf)) {
            if (oo[a] < g.bmin[a] || oo[a] > g.bmax[a]) return false;
            continue;
        }
        *t0 = fmaxf(*t0, tn);
        *t1 = fminf(*t1, tf);
        if (*t0 > *t1) return false;
    }
    return true;
}

__device__ __forceinline__ void grid_sigma(const DevScene &s, const DevGrid &g, const Lambda &lam, SS *sa, SS *ss) {
    *sa = tab4(s.spectra, g.sigmaA, lam) * g.scale;
    *ss = tab4(s.spectra, g.sigmaS, lam) * g.scale;
}

// The free-flight process of a grid medium along its clipped medium-space ray mo + md t,
// t in [t0, t1): a walk over the macro cells the ray crosses (3D DDA) with the piecewise-constant
// rate mu = cell majorant x sMax. Each tentative collision draws a unit-rate exponential optical
// depth and spends it across the cells (mu x length per cell) until it runs out, so a crossing
// costs no random numbers and an empty cell no density lookups. Calls f(t, mu) at each tentative
// collision; f returns false to stop. Bounded: at most 100,000 collisions and mx + my + mz + 3
// cells.
template <class F>
__device__ __forceinline__ void majorant_walk(const DevGrid &g, V3 mo, V3 md, float t0, float t1, float sMax, Pcg &rng,
                                              F &&f) {
    const int M[3] = {g.mx, g.my, g.mz};
    const float o[3] = {mo.x, mo.y, mo.z}, dd[3] = {md.x, md.y, md.z};
    int c[3], step[3];
    float tNext[3], dt[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float ext = g.bmax[a] - g.bmin[a];
        float sc = ext > 0.f ? float(M[a]) / ext : 0.f;
        float u0 = (o[a] + dd[a] * t0 - g.bmin[a]) * sc, du = dd[a] * sc;
        c[a] = min(max(int(floorf(u0)), 0), M[a] - 1);
        if (du > 0.f) {
            tNext[a] = t0 + (float(c[a] + 1) - u0) / du;
            dt[a] = 1.f / du;
            step[a] = 1;
        } else if (du < 0.f) {
            tNext[a] = t0 + (float(c[a]) - u0) / du;
            dt[a] = -1.f / du;
            step[a] = -1;
        } else {
            tNext[a] = INFINITY;
            dt[a] = 0.f;
            step[a] = 0;
        }
    }
    float t = t0;
    float tau = -logf(1.f - rng.uniform());  // optical depth left to the next tentative collision
    int collisions = 0;
    for (int cells = 0; cells < M[0] + M[1] + M[2] + 3; ++cells) {
        int a = tNext[0] < tNext[1] ? (tNext[0] < tNext[2] ? 0 : 2) : (tNext[1] < tNext[2] ? 1 : 2);
        float segEnd = fminf(tNext[a], t1);
        float mu = __ldg(g.majorant + (size_t(c[2]) * M[1] + c[1]) * M[0] + c[0]) * sMax;
        if (mu > 0.f) {
            for (;;) {
                float tc = t + tau / mu;
                if (!(tc < segEnd)) {
                    tau = fmaxf(0.f, tau - mu * fmaxf(0.f, segEnd - t));
                    break;
                }
                t = tc;
                if (!f(t, mu) || ++collisions >= 100000) return;
                tau = -logf(1.f - rng.uniform());
            }
        }
        if (!(tNext[a] < t1)) return;
        t = segEnd;
        c[a] += step[a];
        if (c[a] < 0 || c[a] >= M[a]) return;
        tNext[a] += dt[a];
    }
}

// Ratio-tracking transmittance over [0, dist) along the unit direction d, Russian roulette once
// the largest channel drops below 0.1 (unbiased). rng: a stream for this segment.
static __device__ SS grid_tr(const DevScene &s, const DevGrid &g, const Lambda &lam, V3 o, V3 d, float dist, Pcg &rng) {
    V3 mo, md;
    float t0, t1;
    if (!isfinite(dist) || !grid_clip(g, o, d, dist, &mo, &md, &t0, &t1)) return splat(1.f);
    SS sa, ss;
    grid_sigma(s, g, lam, &sa, &ss);
    SS st = sa + ss;
    float sMax = max_c(st);
    if (!(sMax > 0.f)) return splat(1.f);
    SS T = splat(1.f);
    majorant_walk(g, mo, md, t0, t1, sMax, rng, [&](float t, float mu) {
        float den = grid_density(g, mo + md * t) / mu;
#pragma unroll
        for (int i = 0; i < 4; ++i) T.v[i] *= fmaxf(0.f, 1.f - st.v[i] * den);
        float m = max_c(T);
        if (m <= 0.f) {
            T = splat(0.f);
            return false;
        }
        if (m < 0.1f) {
            if (rng.uniform() < 0.5f) {
                T = splat(0.f);
                return false;
            }
            T = T * 2.f;
        }
        return true;
    });
    return T;
}

// Transmittance of a straight segment of length dist (unit direction d) in medium m.
__device__ __forceinline__ SS medium_transmittance(const DevScene &s, int m, const Lambda &lam, V3 o, V3 d, float dist,
                                                   Pcg &rng) {
    if (!is_grid(s, m)) return homogeneous_tr(s, m, lam, dist);
    return grid_tr(s, s.grids[m - s.mediumCount], lam, o, d, dist, rng);
}

// Spectral tracking (wavelength-neutral event probabilities from the channel averages over the
// live wavelengths, per-wavelength weights sigma_e / (mu P_e)). Returns 1 on a real scattering
// event at *tOut, 2 on absorption, 0 when the segment [0, tMax) is crossed; *weight multiplies
// the throughput in every case.
static __device__ int grid_sample(const DevScene &s, const DevGrid &g, const Lambda &lam, V3 o, V3 d, float tMax, Pcg &rng,
                           float *tOut, SS *weight) {
    *weight = splat(1.f);
    *tOut = tMax;
    V3 mo, md;
    float t0, t1;
    if (!grid_clip(g, o, d, tMax, &mo, &md, &t0, &t1)) return 0;
    SS sa, ss;
    grid_sigma(s, g, lam, &sa, &ss);
    float sMax = max_c(sa + ss);
    if (!(sMax > 0.f)) return 0;
    auto avg = [&](const SS &v) {
        float sum = 0.f;
        int n = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (lam.pdf[i] != 0.f) {
                sum += fabsf(v.v[i]);
                ++n;
            }
        return n ? sum / n : 0.f;
    };
    int event = 0;
    majorant_walk(g, mo, md, t0, t1, sMax, rng, [&](float t, float mu) {
        float den = grid_density(g, mo + md * t);
        SS sA = sa * den, sS = ss * den;
        SS sN = splat(mu) + sA * -1.f + sS * -1.f;
        float pa = avg(sA), ps = avg(sS), pn = avg(sN);
        float norm = pa + ps + pn;
        if (norm <= 0.f) return true;
        float xi = rng.uniform() * norm;
        if (xi < ps) {
            *tOut = t;
            *weight = *weight * sS * (1.f / (mu * ps / norm));
            event = 1;
            return false;
        }
        if (xi < ps + pa) {
            *tOut = t;
            *weight = splat(0.f);
            event = 2;
            return false;
        }
        *weight = *weight * sN * (1.f / (mu * pn / norm));
        return nonzero(*weight);
    });
    if (event == 0) *tOut = tMax;
    return event;
}

// A PCG stream for a shadow segment, from its geometry (ratio tracking needs randomness the path
// state does not carry in the shadow queue).
__device__ __forceinline__ Pcg segment_stream(V3 o, V3 d, uint32_t salt) {
    uint64_t h = mix_bits((uint64_t(__float_as_uint(o.x)) << 32) ^ __float_as_uint(o.y) ^ (uint64_t(salt) << 17));
    h = mix_bits(h ^ (uint64_t(__float_as_uint(o.z)) << 32) ^ __float_as_uint(d.x));
    h = mix_bits(h ^ (uint64_t(__float_as_uint(d.y)) << 32) ^ __float_as_uint(d.z));
    Pcg r;
    r.seed(h, mix_bits(h + 0x9E3779B97F4A7C15ull));
    return r;
}

} // namespace prb
