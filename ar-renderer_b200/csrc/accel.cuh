// Conversion of the caller's v4 BVH (prgpu::BVHNode + primOrder, the layout of
// src/gpu/gpu_api.h:35-40 / pr::BVH::Node, src/geometry/bvh.h:31-36) into the traversal layout of
// traverse.cuh, with full validation of the untrusted input so that no malformed tree can make a
// kernel read out of bounds or loop.
#pragma once

#include <limits>

#include <string>
#include <vector>

#include "device.cuh"
#include "traverse.cuh"

namespace prb {

struct RootInfo {
    float box[6];
    int ref;
    int empty;  // 1 = no nodes: every query misses
};

struct HostAccel {
    std::vector<WNode> nodes;
    std::vector<LeafPrim> prims;
    std::vector<QNode> qnodes;  // the same tree collapsed to 4-wide nodes (root = QNode 0 when interior)
    RootInfo root{};
};

// Collapses the binary tree under interior WNode w into 4-wide nodes: a node takes its two
// children and, while it has fewer than four, opens the interior child of largest surface area.
inline int collapse4(const HostAccel &b, int w, std::vector<QNode> *out) {
    struct Kid {
        int ref;
        float lo[3], hi[3];
    };
    auto kidsOf = [&](int wi, Kid *k) {
        const WNode &n = b.nodes[size_t(wi)];
        k[0] = Kid{n.r.x, {n.a.x, n.a.y, n.a.z}, {n.a.w, n.b.x, n.b.y}};
        k[1] = Kid{n.r.y, {n.b.z, n.b.w, n.c.x}, {n.c.y, n.c.z, n.c.w}};
    };
    auto area = [](const Kid &k) {
        float dx = k.hi[0] - k.lo[0], dy = k.hi[1] - k.lo[1], dz = k.hi[2] - k.lo[2];
        return dx * dy + dy * dz + dz * dx;
    };
    Kid kids[4];
    int nk = 2;
    kidsOf(w, kids);
    while (nk < 4) {
        int best = -1;
        float bestA = -1.f;
        for (int i = 0; i < nk; ++i)
            if (kids[i].ref >= 0 && area(kids[i]) > bestA) {
                bestA = area(kids[i]);
                best = i;
            }
        if (best < 0) break;
        Kid two[2];
        kidsOf(kids[best].ref, two);
        kids[best] = two[0];
        kids[nk++] = two[1];
    }
    const int idx = int(out->size());
    out->push_back(QNode{});
    float lo[3][4], hi[3][4];
    int ch[4];
    const float inf = std::numeric_limits<float>::infinity();
    for (int i = 0; i < 4; ++i) {
        for (int a = 0; a < 3; ++a) {
            lo[a][i] = i < nk ? kids[i].lo[a] : inf;
            hi[a][i] = i < nk ? kids[i].hi[a] : -inf;
        }
        ch[i] = 0;
    }
    for (int i = 0; i < nk; ++i) ch[i] = kids[i].ref >= 0 ? collapse4(b, kids[i].ref, out) : kids[i].ref;
    QNode &q = (*out)[size_t(idx)];
    q.lox = make_float4(lo[0][0], lo[0][1], lo[0][2], lo[0][3]);
    q.loy = make_float4(lo[1][0], lo[1][1], lo[1][2], lo[1][3]);
    q.loz = make_float4(lo[2][0], lo[2][1], lo[2][2], lo[2][3]);
    q.hix = make_float4(hi[0][0], hi[0][1], hi[0][2], hi[0][3]);
    q.hiy = make_float4(hi[1][0], hi[1][1], hi[1][2], hi[1][3]);
    q.hiz = make_float4(hi[2][0], hi[2][1], hi[2][2], hi[2][3]);
    q.child = make_int4(ch[0], ch[1], ch[2], ch[3]);
    q.pad = make_int4(0, 0, 0, 0);
    return idx;
}

// Per-primitive geometry accessor for the conversion: fills the leaf record of primitive `prim`.
struct TriangleSoupSource {
    const prgpu::Float3 *verts;  // 3 per primitive
    void operator()(int prim, LeafPrim *out) const {
        const prgpu::Float3 &p0 = verts[3 * size_t(prim)], &p1 = verts[3 * size_t(prim) + 1],
                            &p2 = verts[3 * size_t(prim) + 2];
        // e1 = p1 - p0 and e2 = p2 - p0 are the same float subtractions the reference performs
        // per test (shape.cpp:205), done once here.
        out->v0 = make_float4(p0.x, p0.y, p0.z, __int_as_float_host(prim));
        out->v1 = make_float4(p1.x - p0.x, p1.y - p0.y, p1.z - p0.z, __int_as_float_host(0));
        out->v2 = make_float4(p2.x - p0.x, p2.y - p0.y, p2.z - p0.z, __int_as_float_host(0));
    }
    static float __int_as_float_host(int i) {
        float f;
        std::memcpy(&f, &i, 4);
        return f;
    }
};

struct PrimitiveSource {
    const prgpu::Primitive *prims;
    void operator()(int prim, LeafPrim *out) const {
        const prgpu::Primitive &p = prims[prim];
        if (p.type == prgpu::PrimSphere) {
            out->v0 = make_float4(p.p0.x, p.p0.y, p.p0.z, TriangleSoupSource::__int_as_float_host(prim));
            out->v1 = make_float4(p.r, 0.f, 0.f, TriangleSoupSource::__int_as_float_host(1));
            out->v2 = make_float4(0.f, 0.f, 0.f, TriangleSoupSource::__int_as_float_host(0));
        } else {
            out->v0 = make_float4(p.p0.x, p.p0.y, p.p0.z, TriangleSoupSource::__int_as_float_host(prim));
            out->v1 = make_float4(p.p1.x - p.p0.x, p.p1.y - p.p0.y, p.p1.z - p.p0.z,
                                  TriangleSoupSource::__int_as_float_host(0));
            out->v2 = make_float4(p.p2.x - p.p0.x, p.p2.y - p.p0.y, p.p2.z - p.p0.z,
                                  TriangleSoupSource::__int_as_float_host(0));
        }
    }
};

// Validates the tree and converts it. Returns false with a message for malformed input.
template <typename Source>
bool convert_bvh(const prgpu::BVHNode *nodes, int32_t nodeCount, const int32_t *order, int32_t primCount,
                 const Source &src, HostAccel *out, std::string *err) {
    out->nodes.clear();
    out->prims.clear();
    out->root = RootInfo{};
    if (nodeCount < 0 || primCount < 0) {
        *err = "negative node or primitive count";
        return false;
    }
    if (nodeCount == 0) {
        out->root.empty = 1;
        return true;
    }
    if (!nodes || (primCount > 0 && !order)) {
        *err = "null BVH arrays";
        return false;
    }
    std::vector<int32_t> interiorIndex(size_t(nodeCount), -1);
    int32_t nInterior = 0;
    for (int32_t i = 0; i < nodeCount; ++i) {
        const prgpu::BVHNode &n = nodes[i];
        if (n.nPrims == 0) {
            // Interior: first child i + 1, second child offset; depth-first order means both come
            // after i, which also rules out cycles.
            if (i + 1 >= nodeCount || n.offset <= i || n.offset >= nodeCount || n.axis > 2) {
                *err = "malformed BVH interior node " + std::to_string(i);
                return false;
            }
            interiorIndex[size_t(i)] = nInterior++;
        } else {
            if (n.offset < 0 || int64_t(n.offset) + n.nPrims > primCount) {
                *err = "BVH leaf " + std::to_string(i) + " exceeds the primitive range";
                return false;
            }
        }
    }
    for (int32_t s = 0; s < primCount; ++s)
        if (order[s] < 0 || order[s] >= primCount) {
            *err = "primOrder entry out of range";
            return false;
        }
    // Leaves must cover disjoint slot ranges: each leaf's last slot carries the end mark.
    std::vector<uint8_t> slotOwner(size_t(primCount), 0);
    for (int32_t i = 0; i < nodeCount; ++i) {
        const prgpu::BVHNode &n = nodes[i];
        if (n.nPrims == 0) continue;
        for (int k = 0; k < n.nPrims; ++k) {
            if (slotOwner[size_t(n.offset + k)]) {
                *err = "BVH leaves overlap in primOrder";
                return false;
            }
            slotOwner[size_t(n.offset + k)] = k + 1 == n.nPrims ? 2 : 1;
        }
    }
    auto childRef = [&](int32_t c) {
        const prgpu::BVHNode &n = nodes[c];
        return n.nPrims == 0 ? interiorIndex[size_t(c)] : ~n.offset;
    };
    out->nodes.resize(size_t(nInterior));
    for (int32_t i = 0; i < nodeCount; ++i) {
        const prgpu::BVHNode &n = nodes[i];
        if (n.nPrims != 0) continue;
        const prgpu::BVHNode &a = nodes[i + 1], &b = nodes[n.offset];
        WNode w;
        w.a = make_float4(a.bmin.x, a.bmin.y, a.bmin.z, a.bmax.x);
        w.b = make_float4(a.bmax.y, a.bmax.z, b.bmin.x, b.bmin.y);
        w.c = make_float4(b.bmin.z, b.bmax.x, b.bmax.y, b.bmax.z);
        w.r = make_int4(childRef(i + 1), childRef(n.offset), int(n.axis), 0);
        out->nodes[size_t(interiorIndex[size_t(i)])] = w;
    }
    out->prims.resize(size_t(primCount));
    for (int32_t s = 0; s < primCount; ++s) {
        src(order[s], &out->prims[size_t(s)]);
        int mark = slotOwner[size_t(s)] == 2 ? 1 : 0;
        std::memcpy(&out->prims[size_t(s)].v2.w, &mark, 4);
    }
    const prgpu::BVHNode &r = nodes[0];
    out->root.box[0] = r.bmin.x;
    out->root.box[1] = r.bmin.y;
    out->root.box[2] = r.bmin.z;
    out->root.box[3] = r.bmax.x;
    out->root.box[4] = r.bmax.y;
    out->root.box[5] = r.bmax.z;
    out->root.ref = childRef(0);
    out->root.empty = 0;
    out->qnodes.clear();
    if (out->root.ref >= 0) {
        out->qnodes.reserve(out->nodes.size() / 2 + 1);
        collapse4(*out, out->root.ref, &out->qnodes);
    }
    return true;
}

// Device copy of a converted BVH.
struct DeviceAccel {
    DevBuf nodes, prims, qnodes;
    RootInfo root{};
    int device = -1;
    int64_t bytes = 0;
    void upload(const HostAccel &h, cudaStream_t s) {
        size_t nb = std::max<size_t>(1, h.nodes.size()) * sizeof(WNode);
        size_t pb = std::max<size_t>(1, h.prims.size()) * sizeof(LeafPrim);
        nodes.ensure(nb);
        prims.ensure(pb);
        if (!h.nodes.empty())
            PRB_CUDA(cudaMemcpyAsync(nodes.ptr, h.nodes.data(), h.nodes.size() * sizeof(WNode), cudaMemcpyHostToDevice, s));
        if (!h.prims.empty())
            PRB_CUDA(cudaMemcpyAsync(prims.ptr, h.prims.data(), h.prims.size() * sizeof(LeafPrim), cudaMemcpyHostToDevice, s));
        size_t qb = std::max<size_t>(1, h.qnodes.size()) * sizeof(QNode);
        qnodes.ensure(qb);
        if (!h.qnodes.empty())
            PRB_CUDA(cudaMemcpyAsync(qnodes.ptr, h.qnodes.data(), h.qnodes.size() * sizeof(QNode),
                                     cudaMemcpyHostToDevice, s));
        root = h.root;
        bytes = int64_t(h.qnodes.size() * sizeof(QNode) + h.prims.size() * sizeof(LeafPrim));
    }
    void release() {
        nodes.release();
        prims.release();
        qnodes.release();
    }
};

} // namespace prb
