// Host-side acceleration-structure builders of libprender_host.so (include/prhost_api.h).
//
// prhost_build_bvh: binned surface-area-heuristic BVH. Every split evaluates 32 centroid bins on
// all three axes (the reference bins 16 on the longest axis only, src/geometry/bvh.cpp:56-98),
// with a traversal cost of 1 against one unit per primitive; a node becomes a leaf when no split
// is cheaper and it holds at most maxLeaf primitives. Subtrees of 32K+ primitives near the root
// are built on worker threads into private node arrays and spliced depth-first, so the output is
// the same flattened layout the reference emits (prgpu::BVHNode, gpu_api.h:35-40).
//
// prhost_build_light_bvh: the Conty & Kulla light BVH of pbrt-v4 -- importance bounds (position
// box, emission cone, power) merged with the direction-cone union, split by the surface-area and
// orientation heuristic over 12 buckets per axis -- in the flattened form the reference's
// pr::BVHLightSampler keeps (src/lights/light_bvh.cpp:10-43, 90-177), with parent links for the
// leaf-to-root pmf walk.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <future>
#include <limits>
#include <thread>
#include <vector>

#include "../../include/prhost_api.h"

namespace {

struct Box {
    float lo[3] = {std::numeric_limits<float>::infinity(), std::numeric_limits<float>::infinity(),
                   std::numeric_limits<float>::infinity()};
    float hi[3] = {-std::numeric_limits<float>::infinity(), -std::numeric_limits<float>::infinity(),
                   -std::numeric_limits<float>::infinity()};
    void grow(const Box &b) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], b.lo[a]);
            hi[a] = std::max(hi[a], b.hi[a]);
        }
    }
    void grow(const float *p) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], p[a]);
            hi[a] = std::max(hi[a], p[a]);
        }
    }
    bool empty() const { return lo[0] > hi[0]; }
    float area() const {
        if (empty()) return 0.f;
        float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        return 2.f * (dx * dy + dy * dz + dz * dx);
    }
};

struct Item {
    Box b;
    float c[3];
    int32_t index;
};

struct Builder {
    std::vector<Item> &items;
    int maxLeaf;
    int parallelDepth;
    static constexpr int kBins = 32;
    static constexpr int64_t kParallelMin = 32768;

    int32_t build(int64_t start, int64_t end, std::vector<prgpu::BVHNode> &out, int depth) {
        int32_t nodeIndex = int32_t(out.size());
        out.emplace_back();
        Box bounds, cb;
        for (int64_t i = start; i < end; ++i) {
            bounds.grow(items[size_t(i)].b);
            cb.grow(items[size_t(i)].c);
        }
        prgpu::BVHNode &node0 = out[size_t(nodeIndex)];
        std::memset(&node0, 0, sizeof(node0));
        node0.bmin = {bounds.lo[0], bounds.lo[1], bounds.lo[2]};
        node0.bmax = {bounds.hi[0], bounds.hi[1], bounds.hi[2]};
        const int64_t n = end - start;
        auto leaf = [&]() {
            out[size_t(nodeIndex)].offset = int32_t(start);
            out[size_t(nodeIndex)].nPrims = uint16_t(n);
            return nodeIndex;
        };
        if (n == 1) return leaf();

        // Best binned split over the three axes.
        float bestCost = std::numeric_limits<float>::infinity();
        int bestAxis = -1, bestBin = -1;
        for (int axis = 0; axis < 3; ++axis) {
            float cmin = cb.lo[axis], cmax = cb.hi[axis];
            if (!(cmax > cmin)) continue;
            Box binBox[kBins];
            int64_t binCount[kBins] = {};
            float scale = kBins / (cmax - cmin);
            for (int64_t i = start; i < end; ++i) {
                const Item &it = items[size_t(i)];
                int b = std::min(kBins - 1, int((it.c[axis] - cmin) * scale));
                binCount[b]++;
                binBox[b].grow(it.b);
            }
            float rightArea[kBins];
            int64_t rightCount[kBins];
            Box acc;
            int64_t cnt = 0;
            for (int b = kBins - 1; b > 0; --b) {
                acc.grow(binBox[b]);
                cnt += binCount[b];
                rightArea[b] = acc.area();
                rightCount[b] = cnt;
            }
            Box left;
            int64_t lc = 0;
            for (int b = 0; b < kBins - 1; ++b) {
                left.grow(binBox[b]);
                lc += binCount[b];
                if (lc == 0 || rightCount[b + 1] == 0) continue;
                float cost = float(lc) * left.area() + float(rightCount[b + 1]) * rightArea[b + 1];
                if (cost < bestCost) {
                    bestCost = cost;
                    bestAxis = axis;
                    bestBin = b;
                }
            }
        }
        float rootArea = bounds.area();
        float splitCost = rootArea > 0 ? 1.f + bestCost / rootArea : std::numeric_limits<float>::infinity();
        if (bestAxis < 0) {
            // All centroids coincide: no spatial split exists.
            if (n <= 255) return leaf();
            int64_t mid = (start + end) / 2;
            out[size_t(nodeIndex)].axis = 0;
            children(start, mid, end, out, nodeIndex, depth);
            return nodeIndex;
        }
        if (n <= maxLeaf && float(n) <= splitCost) return leaf();
        float cmin = cb.lo[bestAxis], scale = kBins / (cb.hi[bestAxis] - cmin);
        auto midIt = std::partition(items.begin() + start, items.begin() + end, [&](const Item &it) {
            return std::min(kBins - 1, int((it.c[bestAxis] - cmin) * scale)) <= bestBin;
        });
        int64_t mid = int64_t(midIt - items.begin());
        if (mid == start || mid == end) mid = (start + end) / 2;
        out[size_t(nodeIndex)].axis = uint8_t(bestAxis);
        children(start, mid, end, out, nodeIndex, depth);
        return nodeIndex;
    }

    void children(int64_t start, int64_t mid, int64_t end, std::vector<prgpu::BVHNode> &out, int32_t parent, int depth) {
        if (end - start >= kParallelMin && depth < parallelDepth) {
            std::vector<prgpu::BVHNode> right;
            right.reserve(size_t(2 * (end - mid)));
            auto fut = std::async(std::launch::async, [&] { build(mid, end, right, depth + 1); });
            build(start, mid, out, depth + 1);
            fut.get();
            int32_t base = int32_t(out.size());
            for (prgpu::BVHNode n : right) {
                if (n.nPrims == 0) n.offset += base;
                out.push_back(n);
            }
            out[size_t(parent)].offset = base;
            return;
        }
        build(start, mid, out, depth + 1);
        int32_t second = build(mid, end, out, depth + 1);
        out[size_t(parent)].offset = second;
    }
};

int64_t build_from_items(std::vector<Item> &items, int32_t maxLeaf, int32_t threads, prgpu::BVHNode *nodesOut,
                         int32_t *primOrderOut) {
    if (items.empty()) return 0;
    int hw = int(std::thread::hardware_concurrency());
    int t = threads > 0 ? threads : std::max(1, hw);
    int depth = 0;
    while ((1 << depth) < t && depth < 12) ++depth;
    Builder b{items, std::clamp(int(maxLeaf), 1, 8), depth};
    std::vector<prgpu::BVHNode> nodes;
    nodes.reserve(2 * items.size());
    b.build(0, int64_t(items.size()), nodes, 0);
    std::memcpy(nodesOut, nodes.data(), nodes.size() * sizeof(prgpu::BVHNode));
    for (size_t i = 0; i < items.size(); ++i) primOrderOut[i] = items[i].index;
    return int64_t(nodes.size());
}

// ---------------------------------------------------------------------------------------------
// Light BVH

constexpr float kPi = 3.14159265358979323846f;

struct V {
    float x, y, z;
};
V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V operator*(V a, float s) { return {a.x * s, a.y * s, a.z * s}; }
float dotv(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V crossv(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
float lenv(V a) { return std::sqrt(dotv(a, a)); }
V normv(V a) { return a * (1.f / lenv(a)); }
float safe_acos(float x) { return std::acos(std::clamp(x, -1.f, 1.f)); }
float safe_asin(float x) { return std::asin(std::clamp(x, -1.f, 1.f)); }

struct Cone {
    V w{0, 0, 1};
    float cosTheta = std::numeric_limits<float>::infinity();  // +inf = empty
    bool isEmpty() const { return cosTheta == std::numeric_limits<float>::infinity(); }
};

float angle_between(V a, V b) {
    if (dotv(a, b) < 0) return kPi - 2 * safe_asin(lenv(a + b) / 2);
    return 2 * safe_asin(lenv(b - a) / 2);
}

// Rotation of v by theta about unit axis k (Rodrigues).
V rotate(V v, V k, float theta) {
    float c = std::cos(theta), s = std::sin(theta);
    return v * c + crossv(k, v) * s + k * (dotv(k, v) * (1 - c));
}

Cone cone_union(const Cone &a, const Cone &b) {
    if (a.isEmpty()) return b;
    if (b.isEmpty()) return a;
    float ta = safe_acos(a.cosTheta), tb = safe_acos(b.cosTheta);
    float td = angle_between(a.w, b.w);
    if (std::min(td + tb, kPi) <= ta) return a;
    if (std::min(td + ta, kPi) <= tb) return b;
    float to = (ta + td + tb) / 2;
    if (to >= kPi) return Cone{{0, 0, 1}, -1.f};
    float tr = to - ta;
    V wr = crossv(a.w, b.w);
    if (dotv(wr, wr) == 0) return Cone{{0, 0, 1}, -1.f};
    return Cone{normv(rotate(a.w, normv(wr), tr)), std::cos(to)};
}

struct LB {
    Box b;
    V w{0, 0, 1};
    float phi = 0, cosO = 1, cosE = 0;
    bool twoSided = false;
};

LB lb_union(const LB &a, const LB &b) {
    if (a.phi == 0) return b;
    if (b.phi == 0) return a;
    Cone c = cone_union(Cone{a.w, a.cosO}, Cone{b.w, b.cosO});
    LB r;
    r.b = a.b;
    r.b.grow(b.b);
    r.w = c.w;
    r.phi = a.phi + b.phi;
    r.cosO = c.cosTheta;
    r.cosE = std::min(a.cosE, b.cosE);
    r.twoSided = a.twoSided || b.twoSided;
    return r;
}

float lb_cost(const LB &l, const Box &bounds, int dim) {
    float to = safe_acos(l.cosO), te = safe_acos(l.cosE);
    float tw = std::min(to + te, kPi);
    float so = std::sqrt(std::max(0.f, 1 - l.cosO * l.cosO));
    float mOmega = 2 * kPi * (1 - l.cosO) + kPi / 2 * (2 * tw * so - std::cos(to - 2 * tw) - 2 * to * so + l.cosO);
    float d[3] = {bounds.hi[0] - bounds.lo[0], bounds.hi[1] - bounds.lo[1], bounds.hi[2] - bounds.lo[2]};
    float maxd = std::max(d[0], std::max(d[1], d[2]));
    float kr = d[dim] > 0 ? maxd / d[dim] : 1.f;
    return l.phi * mOmega * kr * l.b.area();
}

struct LightBuilder {
    std::vector<std::pair<int, LB>> items;
    std::vector<prgpu::LightBVHNode> nodes;
    std::vector<LB> lbs;

    int build(int start, int end, int parent) {
        if (end - start == 1) {
            int idx = int(nodes.size());
            prgpu::LightBVHNode n{};
            const LB &l = items[size_t(start)].second;
            fill(n, l);
            n.child1 = -1;
            n.light = items[size_t(start)].first;
            n.parent = parent;
            nodes.push_back(n);
            lbs.push_back(l);
            return idx;
        }
        Box bounds, cb;
        for (int i = start; i < end; ++i) {
            const Box &b = items[size_t(i)].second.b;
            bounds.grow(b);
            float c[3] = {(b.lo[0] + b.hi[0]) * 0.5f, (b.lo[1] + b.hi[1]) * 0.5f, (b.lo[2] + b.hi[2]) * 0.5f};
            cb.grow(c);
        }
        constexpr int kB = 12;
        float minCost = std::numeric_limits<float>::infinity();
        int minBucket = -1, minDim = -1;
        auto bucketOf = [&](const Box &b, int dim) {
            float c = (b.lo[dim] + b.hi[dim]) * 0.5f;
            float off = (c - cb.lo[dim]) / (cb.hi[dim] - cb.lo[dim]);
            return std::clamp(int(kB * off), 0, kB - 1);
        };
        for (int dim = 0; dim < 3; ++dim) {
            if (cb.hi[dim] == cb.lo[dim]) continue;
            LB bucket[kB];
            for (int i = start; i < end; ++i) {
                int b = bucketOf(items[size_t(i)].second.b, dim);
                bucket[b] = lb_union(bucket[b], items[size_t(i)].second);
            }
            for (int i = 0; i < kB - 1; ++i) {
                LB b0, b1;
                for (int j = 0; j <= i; ++j) b0 = lb_union(b0, bucket[j]);
                for (int j = i + 1; j < kB; ++j) b1 = lb_union(b1, bucket[j]);
                float cost = lb_cost(b0, bounds, dim) + lb_cost(b1, bounds, dim);
                if (cost > 0 && cost < minCost) {
                    minCost = cost;
                    minBucket = i;
                    minDim = dim;
                }
            }
        }
        int mid;
        if (minDim == -1) {
            mid = (start + end) / 2;
        } else {
            auto it = std::partition(items.begin() + start, items.begin() + end,
                                     [&](const std::pair<int, LB> &l) { return bucketOf(l.second.b, minDim) <= minBucket; });
            mid = int(it - items.begin());
            if (mid == start || mid == end) mid = (start + end) / 2;
        }
        int idx = int(nodes.size());
        nodes.emplace_back();
        lbs.emplace_back();
        build(start, mid, idx);
        int c1 = build(mid, end, idx);
        LB u = lb_union(lbs[size_t(idx) + 1], lbs[size_t(c1)]);
        lbs[size_t(idx)] = u;
        prgpu::LightBVHNode n{};
        fill(n, u);
        n.child1 = c1;
        n.light = -1;
        n.parent = parent;
        nodes[size_t(idx)] = n;
        return idx;
    }

    static void fill(prgpu::LightBVHNode &n, const LB &l) {
        n.bmin = {l.b.lo[0], l.b.lo[1], l.b.lo[2]};
        n.bmax = {l.b.hi[0], l.b.hi[1], l.b.hi[2]};
        n.w = {l.w.x, l.w.y, l.w.z};
        n.phi = l.phi;
        n.cosThetaO = l.cosO;
        n.cosThetaE = l.cosE;
        n.twoSided = l.twoSided ? 1 : 0;
    }
};

} // namespace

PRHOST_API int64_t prhost_build_bvh(const float *boxMin, const float *boxMax, int64_t primCount, int32_t maxLeaf,
                                    int32_t threads, prgpu::BVHNode *nodesOut, int32_t *primOrderOut) {
    if (primCount < 0 || primCount > (int64_t(1) << 30) || (primCount > 0 && (!boxMin || !boxMax || !nodesOut || !primOrderOut)))
        return -1;
    std::vector<Item> items(static_cast<size_t>(primCount));
    for (int64_t i = 0; i < primCount; ++i) {
        Item &it = items[size_t(i)];
        for (int a = 0; a < 3; ++a) {
            it.b.lo[a] = boxMin[3 * i + a];
            it.b.hi[a] = boxMax[3 * i + a];
            it.c[a] = 0.5f * it.b.lo[a] + 0.5f * it.b.hi[a];
        }
        it.index = int32_t(i);
    }
    return build_from_items(items, maxLeaf, threads, nodesOut, primOrderOut);
}

PRHOST_API int64_t prhost_build_bvh_triangles(const prgpu::Float3 *verts, int64_t primCount, int32_t maxLeaf,
                                              int32_t threads, prgpu::BVHNode *nodesOut, int32_t *primOrderOut) {
    if (primCount < 0 || primCount > (int64_t(1) << 30) || (primCount > 0 && (!verts || !nodesOut || !primOrderOut)))
        return -1;
    std::vector<Item> items(static_cast<size_t>(primCount));
    for (int64_t i = 0; i < primCount; ++i) {
        Item &it = items[size_t(i)];
        for (int k = 0; k < 3; ++k) {
            const prgpu::Float3 &v = verts[3 * i + k];
            float p[3] = {v.x, v.y, v.z};
            it.b.grow(p);
        }
        for (int a = 0; a < 3; ++a) it.c[a] = 0.5f * it.b.lo[a] + 0.5f * it.b.hi[a];
        it.index = int32_t(i);
    }
    return build_from_items(items, maxLeaf, threads, nodesOut, primOrderOut);
}

PRHOST_API int32_t prhost_build_light_bvh(const float *lightBounds13, int32_t lightCount,
                                          prgpu::LightBVHNode *nodesOut) {
    if (lightCount < 0 || (lightCount > 0 && (!lightBounds13 || !nodesOut))) return -1;
    LightBuilder b;
    for (int32_t i = 0; i < lightCount; ++i) {
        const float *x = lightBounds13 + 13 * size_t(i);
        LB l;
        for (int a = 0; a < 3; ++a) {
            l.b.lo[a] = x[a];
            l.b.hi[a] = x[3 + a];
        }
        l.w = {x[6], x[7], x[8]};
        l.phi = x[9];
        l.cosO = x[10];
        l.cosE = x[11];
        l.twoSided = x[12] != 0;
        if (l.phi > 0) b.items.push_back({int(i), l});
    }
    if (b.items.empty()) return 0;
    b.build(0, int(b.items.size()), -1);
    std::memcpy(nodesOut, b.nodes.data(), b.nodes.size() * sizeof(prgpu::LightBVHNode));
    return int32_t(b.nodes.size());
}
