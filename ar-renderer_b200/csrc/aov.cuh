// Auxiliary (denoiser guide) buffers on the device: pr::RenderAOV (src/integrators/aov.cpp:11-196)
// -- albedo, shading normal, depth or position of the first visible surface, optionally followed
// through perfectly specular chains. One thread per pixel, spp jittered samples, results into an
// RGB float image. Included by render.cu after wavefront.cuh (it uses its traversal and BSDFs).
#pragma once

#include "wavefront.cuh"

namespace prb {

struct AovArgs {
    int type;  // 0 albedo, 1 normal, 2 depth, 3 position (pr::AOVType)
    int spp;
    uint64_t seed;
    int throughSpecular;
    int d65;                  // spectrum index of the D65 illuminant
    float adapt[9], toRGB[9]; // white adaptation, then XYZ -> linear sRGB (row-major)
};

// Nearest non-interface hit along o + t d (NextSurface, aov.cpp:27-35): interfaces only bound
// media, the ray restarts past each. *t is measured from the last restart, as the reference's is.
__device__ __forceinline__ bool next_surface(const DevScene &s, V3 *o, V3 d, Hit *h, bool *overflow) {
    for (int crossings = 0; crossings < 64; ++crossings) {
        TraceRay r = make_trace_ray(*o, d);
        if (!closest4<true>(s, r, kInf, h, overflow)) return false;
        const prgpu::Primitive &pr = s.prims[h->prim];
        if (s.mats[pr.material].type != prgpu::MatInterface) return true;
        Surf sf = shade_point(s, pr, h->t, h->u, h->v, *o, d);
        *o = offset_origin(sf.p, sf.n, d);
    }
    return false;
}

// The end of a guide chain (FollowChain, aov.cpp:44-82): the surface where albedo / normal are
// taken, the chain's throughput, and the medium it entered (-1: none).
struct ChainEnd {
    Surf sf;
    V3 wo;
    int prim;
    int medium;
    SS throughput;
    bool valid;
};

__device__ ChainEnd follow_chain(const DevScene &s, V3 o, V3 d, Hit h, bool throughSpecular, Lambda &lam, Pcg &rng,
                                 bool *overflow) {
    ChainEnd e;
    e.valid = false;
    e.medium = -1;
    e.throughput = splat(1.f);
    for (int bounce = 0;; ++bounce) {
        const prgpu::Primitive &pr = s.prims[h.prim];
        const prgpu::Material &m = s.mats[pr.material];
        Surf sf = shade_point(s, pr, h.t, h.u, h.v, o, d);
        perturb_shading(s, int(&m - s.mats), pr, &sf);
        e.sf = sf;
        e.wo = -d;
        e.prim = h.prim;
        if (!throughSpecular || bounce == 8 || m.type == prgpu::MatBlack || pr.light >= 0) {
            e.valid = true;
            return e;
        }
        Frame fr = frame_from_xz(sf.dpdu, sf.ns);
        V3 wol = fr.to_local(-d);
        BSample bs;
        bool ok;
        float uc = rng.uniform(), u0 = rng.uniform(), u1 = rng.uniform();
        if (full_material(m)) {
            FullBsdf fb;
            make_full(s, m, sf.u, sf.v, lam, &fb);
            textured_full(s, int(&m - s.mats), TexCtx{sf.p, sf.u, sf.v}, lam, &fb);
            if (fb.black || full_non_specular(fb)) {
                e.valid = true;
                return e;
            }
            bool prop;
            ok = wol.z != 0.f && full_sample(fb, wol, uc, u0, u1, &bs, &prop);
        } else {
            Lobe lobe = make_lobe(s, m, sf.u, sf.v, lam);
            textured_lobe(s, int(&m - s.mats), TexCtx{sf.p, sf.u, sf.v}, lam, &lobe);
            if (lobe.flags() == 0u || lobe.non_specular()) {
                e.valid = true;
                return e;
            }
            ok = wol.z != 0.f && lobe_sample(lobe, wol, uc, u0, u1, &bs);
        }
        if (!ok || !(bs.pdf > 0.f)) return e;
        V3 wi = fr.from_local(bs.wi);
        e.throughput = e.throughput * bs.f * (fabsf(dot(wi, sf.ns)) / bs.pdf);
        if (bs.flags & kFlagTransmission) {
            int med = dot(wi, sf.n) > 0.f ? pr.mediumOutside : pr.mediumInside;
            if (med >= 0) {
                int sa, ss;
                float scale;
                if (is_grid(s, med)) {
                    const DevGrid &g = s.grids[med - s.mediumCount];
                    sa = g.sigmaA, ss = g.sigmaS, scale = g.scale;
                } else {
                    sa = s.media[med].sigmaA, ss = s.media[med].sigmaS, scale = s.media[med].scale;
                }
                SS vs = tab4(s.spectra, ss, lam) * scale, va = tab4(s.spectra, sa, lam) * scale;
                if (nonzero(vs)) {
                    e.medium = med;
                    e.valid = true;
                    return e;
                }
                (void)va;
            }
        }
        o = offset_origin(sf.p, sf.n, wi);
        d = wi;
        if (!next_surface(s, &o, d, &h, overflow)) return e;
    }
}

__global__ void __launch_bounds__(128) k_aov(const DevScene *sp, AovArgs a, float *out, int *status) {
    const DevScene &s = *sp;
    const int w = s.cam.width, npix = w * s.cam.height;
    for (int pix = blockIdx.x * blockDim.x + threadIdx.x; pix < npix; pix += gridDim.x * blockDim.x) {
        const int px = pix % w, py = pix / w;
        double sum[3] = {0.0, 0.0, 0.0};
        int hits = 0;
        float minDepth = kInf;
        bool overflow = false;
        for (int smp = 0; smp < a.spp; ++smp) {
            Pcg rng = pixel_sample_stream(uint32_t(pix), uint64_t(smp), a.seed ^ 0xa0f5ull);
            float ux = rng.uniform(), uy = rng.uniform(), l0 = rng.uniform(), l1 = rng.uniform();
            V3 o, d;
            camera_ray(s, float(px) + ux, float(py) + uy, l0, l1, &o, &d);
            Hit h;
            if (!next_surface(s, &o, d, &h, &overflow)) continue;
            ++hits;
            float v[3] = {0.f, 0.f, 0.f};
            if (a.type == 2) {
                minDepth = fminf(minDepth, h.t);
                continue;
            }
            if (a.type == 3) {
                Surf sf = shade_point(s, s.prims[h.prim], h.t, h.u, h.v, o, d);
                v[0] = sf.p.x, v[1] = sf.p.y, v[2] = sf.p.z;
            } else if (a.type == 1) {
                Lambda lam = sample_visible(0.5f);
                ChainEnd e = follow_chain(s, o, d, h, a.throughSpecular != 0, lam, rng, &overflow);
                if (e.valid) {
                    V3 n = e.sf.ns;
                    if (dot(n, e.wo) < 0.f) n = -n;
                    v[0] = n.x, v[1] = n.y, v[2] = n.z;
                }
            } else {
                // Directional albedo: 8 estimates with the BSDF's own sampling, wavelengths
                // resampled each time, as a reflectance under D65 (aov.cpp:108-140).
                float X = 0.f, Y = 0.f, Z = 0.f;
                for (int i = 0; i < 8; ++i) {
                    Lambda lam = sample_visible(rng.uniform());
                    ChainEnd e = follow_chain(s, o, d, h, a.throughSpecular != 0, lam, rng, &overflow);
                    SS alb = splat(0.f);
                    if (e.valid) {
                        const prgpu::Primitive &pr = s.prims[e.prim];
                        const prgpu::Material &m = s.mats[pr.material];
                        if (e.medium >= 0) {
                            int sa, ss;
                            float scale;
                            if (is_grid(s, e.medium)) {
                                const DevGrid &g = s.grids[e.medium - s.mediumCount];
                                sa = g.sigmaA, ss = g.sigmaS, scale = g.scale;
                            } else {
                                sa = s.media[e.medium].sigmaA, ss = s.media[e.medium].sigmaS,
                                scale = s.media[e.medium].scale;
                            }
                            SS vs = tab4(s.spectra, ss, lam) * scale, vt = tab4(s.spectra, sa, lam) * scale + vs;
#pragma unroll
                            for (int k = 0; k < 4; ++k) alb.v[k] = vt.v[k] != 0.f ? vs.v[k] / vt.v[k] : 0.f;
                            alb = e.throughput * alb;
                        } else if (pr.light >= 0) {
                            alb = e.throughput;
                        } else if (m.type != prgpu::MatBlack) {
                            Frame fr = frame_from_xz(e.sf.dpdu, e.sf.ns);
                            V3 wol = fr.to_local(e.wo);
                            float uc = rng.uniform(), u0 = rng.uniform(), u1 = rng.uniform();
                            BSample bs;
                            bool ok;
                            if (full_material(m)) {
                                FullBsdf fb;
                                make_full(s, m, e.sf.u, e.sf.v, lam, &fb);
                                textured_full(s, int(&m - s.mats), TexCtx{e.sf.p, e.sf.u, e.sf.v}, lam, &fb);
                                bool prop;
                                ok = wol.z != 0.f && full_sample(fb, wol, uc, u0, u1, &bs, &prop);
                            } else {
                                Lobe lobe = make_lobe(s, m, e.sf.u, e.sf.v, lam);
                                textured_lobe(s, int(&m - s.mats), TexCtx{e.sf.p, e.sf.u, e.sf.v}, lam, &lobe);
                                ok = wol.z != 0.f && lobe.flags() != 0u && lobe_sample(lobe, wol, uc, u0, u1, &bs);
                            }
                            ok = ok && nonzero(bs.f) && bs.pdf > 0.f && isfinite(bs.pdf) && bs.wi.z != 0.f;
                            if (ok) alb = e.throughput * bs.f * (fabsf(bs.wi.z) / bs.pdf);
                        }
                    }
                    SS lit = alb * tab4(s.spectra, a.d65, lam);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        if (lam.pdf[k] == 0.f) continue;
                        float q = lit.v[k] / lam.pdf[k];
                        X += cie_x(lam.l[k]) * q;
                        Y += cie_y(lam.l[k]) * q;
                        Z += cie_z(lam.l[k]) * q;
                    }
                }
                const float k = s.norm * 0.125f;  // ToXYZ (average over the 4 wavelengths / CIE y integral), / 8
                X *= k, Y *= k, Z *= k;
                const float *A = a.adapt, *M = a.toRGB;
                float ax = A[0] * X + A[1] * Y + A[2] * Z, ay = A[3] * X + A[4] * Y + A[5] * Z,
                      az = A[6] * X + A[7] * Y + A[8] * Z;
                v[0] = M[0] * ax + M[1] * ay + M[2] * az;
                v[1] = M[3] * ax + M[4] * ay + M[5] * az;
                v[2] = M[6] * ax + M[7] * ay + M[8] * az;
                if (a.throughSpecular)
                    for (int c = 0; c < 3; ++c) v[c] = clampf(v[c], 0.f, 1.f);
            }
            for (int c = 0; c < 3; ++c) sum[c] += double(v[c]);
        }
        float r[3];
        if (a.type == 2) {
            float dd = hits > 0 ? minDepth : 1e10f;
            r[0] = r[1] = r[2] = dd;
        } else if (a.type == 1) {
            float l = sqrtf(float(sum[0] * sum[0] + sum[1] * sum[1] + sum[2] * sum[2]));
            for (int c = 0; c < 3; ++c) r[c] = l > 0.f ? float(sum[c]) / l : float(sum[c]);
        } else if (a.type == 3) {
            for (int c = 0; c < 3; ++c) r[c] = hits > 0 ? float(sum[c] / hits) : 0.f;
        } else {
            for (int c = 0; c < 3; ++c) r[c] = float(sum[c] / a.spp);
        }
        out[3 * size_t(pix) + 0] = r[0];
        out[3 * size_t(pix) + 1] = r[1];
        out[3 * size_t(pix) + 2] = r[2];
        if (overflow) atomicOr(status, kStatusStack);
    }
}

} // namespace prb
