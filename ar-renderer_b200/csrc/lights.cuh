// Light-BVH sampling on the device: Conty & Kulla importance of a node's emission bounds at a
// shading point (src/lights/light_bvh.cpp:45-83), stochastic descent picking one light with its
// probability (light_bvh.cpp:179-214), and the exact probability of a given light by the walk
// from its leaf to the root (light_bvh.cpp:216-234) that MIS on emission hits needs.
#pragma once

#include "common.cuh"

namespace prb {

struct LightTree {
    const prgpu::LightBVHNode *nodes;
    int count;
    float prob;          // probability of the BVH branch (1 - probability of infinite lights)
    const int *leafOf;   // light index -> leaf node, -1 when the light is not in the tree
};

// n = 0 for points in media (no cosine factor at the receiver).
__device__ __forceinline__ float lb_importance(const prgpu::LightBVHNode &b, V3 p, V3 n) {
    V3 bmin = f3(b.bmin), bmax = f3(b.bmax);
    V3 pc = (bmin + bmax) * 0.5f;
    float d2 = len2(p - pc);
    d2 = fmaxf(d2, len(bmax - bmin) * 0.5f);
    V3 wi = p - pc;
    float l = len(wi);
    wi = l > 0.f ? wi * (1.f / l) : mk(0.f, 0.f, 1.f);
    float cosW = dot(f3(b.w), wi);
    if (b.twoSided) cosW = fabsf(cosW);
    float sinW = safe_sqrt(1.f - sqr(cosW));
    // Cone subtended by the bounds' bounding sphere.
    float r = len(bmax - pc);
    float cosB = -1.f;
    float dc2 = len2(p - pc);
    if (dc2 >= r * r) cosB = safe_sqrt(1.f - r * r / dc2);
    float sinB = safe_sqrt(1.f - sqr(cosB));
    float sinO = safe_sqrt(1.f - sqr(b.cosThetaO));
    // cos(max(0, a - b)) and sin(max(0, a - b)) from sines and cosines.
    auto cosSub = [](float sA, float cA, float sB, float cB) { return cA > cB ? 1.f : cA * cB + sA * sB; };
    auto sinSub = [](float sA, float cA, float sB, float cB) { return cA > cB ? 0.f : sA * cB - cA * sB; };
    float cosX = cosSub(sinW, cosW, sinO, b.cosThetaO);
    float sinX = sinSub(sinW, cosW, sinO, b.cosThetaO);
    float cosP = cosSub(sinX, cosX, sinB, cosB);
    if (cosP <= b.cosThetaE) return 0.f;
    float imp = b.phi * cosP / d2;
    if (n.x != 0.f || n.y != 0.f || n.z != 0.f) {
        float cosI = fabsf(dot(wi, n));
        float sinI = safe_sqrt(1.f - sqr(cosI));
        imp *= cosSub(sinI, cosI, sinB, cosB);
    }
    return fmaxf(imp, 0.f);
}

// Descent with u already remapped to the BVH branch; returns the light index or -1.
__device__ __forceinline__ int lbvh_sample(const LightTree &t, V3 p, V3 n, float u, float *pmf) {
    int node = 0;
    float prob = t.prob;
    for (int guard = 0; guard < 64; ++guard) {
        const prgpu::LightBVHNode &b = t.nodes[node];
        if (b.light >= 0) {
            if (node > 0 || lb_importance(b, p, n) > 0.f) {
                *pmf = prob;
                return b.light;
            }
            return -1;
        }
        float c0 = lb_importance(t.nodes[node + 1], p, n), c1 = lb_importance(t.nodes[b.child1], p, n);
        if (c0 == 0.f && c1 == 0.f) return -1;
        float p0 = c0 / (c0 + c1);
        if (u < p0) {
            prob *= p0;
            u = fminf(u / p0, kOneMinusEps);
            node = node + 1;
        } else {
            prob *= 1.f - p0;
            u = fminf((u - p0) / (1.f - p0), kOneMinusEps);
            node = b.child1;
        }
    }
    return -1;
}

__device__ __forceinline__ float lbvh_pmf(const LightTree &t, int li, V3 p, V3 n) {
    int leaf = __ldg(t.leafOf + li);
    if (leaf < 0) return 0.f;
    if (leaf == 0) return lb_importance(t.nodes[0], p, n) > 0.f ? t.prob : 0.f;
    float pmf = t.prob;
    int child = leaf;
    for (int guard = 0; guard < 64; ++guard) {
        int parent = t.nodes[child].parent;
        if (parent < 0) break;
        const prgpu::LightBVHNode &b = t.nodes[parent];
        float c0 = lb_importance(t.nodes[parent + 1], p, n), c1 = lb_importance(t.nodes[b.child1], p, n);
        if (c0 == 0.f && c1 == 0.f) return 0.f;
        pmf *= (child == b.child1 ? c1 : c0) / (c0 + c1);
        child = parent;
    }
    return pmf;
}

} // namespace prb
