// BVH traversal for sm_100a: closest-hit and any-hit queries over the caller's binary BVH, with
// results bit-identical to the reference CPU routines pr::BVH::Intersect / IntersectP
// (src/geometry/bvh.cpp:137-232) and pr::Triangle::Intersect (src/geometry/shape.cpp:202-222).
//
// Layout (built on the device from the v4 node array by convert_nodes in accel.cu):
//   WNode, 64 B, one per INTERIOR reference node: both children's boxes plus their references,
//   so one node visit issues four 16-byte loads that bring both child boxes at once. A child
//   reference >= 0 names an interior WNode; < 0 is a leaf whose first leaf slot is ~ref.
//   LeafPrim, 48 B per leaf slot (primOrder order): triangle p0 | e1 = p1 - p0 | e2 = p2 - p0 and
//   the original primitive index; spheres store centre and radius (64-bit test, as the CPU).
//   The last slot of every leaf carries an end mark, so a stack entry is just (ref, entry t).
//
// Parity. The reference pops a node, tests its own box against the CURRENT tMax, and pushes the
// far child before descending into the near one (near = by the sign of the split axis). Here a
// parent tests both child boxes at once, but only the tMax-independent part of the far child's
// test is evaluated early: its entry distance is pushed with it and compared against the tMax
// current at pop time, exactly the reference's final `tMin < tMax` clause. Every arithmetic step
// is an explicitly rounded IEEE operation (__fadd_rn/__fmul_rn/__fdiv_rn, never contracted into
// an FMA), so box decisions, visit order, tMax updates and hits match bit for bit.
#pragma once

#include "common.cuh"

namespace prb {

struct __align__(16) WNode {
    float4 a;  // c0.min.x c0.min.y c0.min.z c0.max.x
    float4 b;  // c0.max.y c0.max.z c1.min.x c1.min.y
    float4 c;  // c1.min.z c1.max.x c1.max.y c1.max.z
    int4 r;    // ref0, ref1, axis, unused
};

struct __align__(16) LeafPrim {
    float4 v0;  // triangle: p0, prim index (int bits); sphere: centre, prim index
    float4 v1;  // triangle: e1, kind 0; sphere: radius, 0, 0, kind 1
    float4 v2;  // triangle: e2, end-of-leaf mark (int bits 1 on a leaf's last slot, else 0)
};

// 4-wide node, collapsed on the host from the binary tree: the four child boxes stored per axis
// (child i in component i of each float4) and the four child references; 128 bytes, one L2 line.
// Unused child slots carry an inverted box (+inf / -inf), which the slab test always rejects.
struct __align__(16) QNode {
    float4 lox, loy, loz, hix, hiy, hiz;
    int4 child;  // >= 0: interior QNode; < 0: leaf whose first slot is ~child
    int4 pad;
};
// The any-hit traversal addresses the plane vectors by byte offset (slab_nf).
static_assert(offsetof(QNode, lox) == 0 && offsetof(QNode, loy) == 16 && offsetof(QNode, loz) == 32 &&
                  offsetof(QNode, hix) == 48 && offsetof(QNode, hiy) == 64 && offsetof(QNode, hiz) == 80 &&
                  sizeof(QNode) == 128,
              "QNode layout");

constexpr int kStackSize = 64;
// 1 + 2 * 1.2e-7f * 3 evaluated in float, the far-distance widening of bvh.cpp:143-151.
constexpr float kWiden = 0x1.00000cp+0f;

struct TraceRay {
    V3 o, d, inv;
    int neg[3];
    bool infInv;  // a direction component is +-0: some slab tests can produce NaN
};

__device__ __forceinline__ TraceRay make_trace_ray(V3 o, V3 d) {
    TraceRay r;
    r.o = o;
    r.d = d;
    r.inv = {__fdiv_rn(1.f, d.x), __fdiv_rn(1.f, d.y), __fdiv_rn(1.f, d.z)};
    r.neg[0] = r.inv.x < 0.f;
    r.neg[1] = r.inv.y < 0.f;
    r.neg[2] = r.inv.z < 0.f;
    r.infInv = isinf(r.inv.x) || isinf(r.inv.y) || isinf(r.inv.z);
    return r;
}

// The tMax-independent part of the reference slab test (bvh.cpp:137-156): returns false when the
// box is rejected for every tMax; otherwise writes the entry distance tMin, and the box is hit
// iff tMin < tMax. Comparison order follows the reference so NaN cases resolve the same way.
__device__ __forceinline__ bool box_entry(const TraceRay &r, float lox, float loy, float loz, float hix, float hiy,
                                          float hiz, float *tEntry) {
    float nx = r.neg[0] ? hix : lox, fx = r.neg[0] ? lox : hix;
    float ny = r.neg[1] ? hiy : loy, fy = r.neg[1] ? loy : hiy;
    float nz = r.neg[2] ? hiz : loz, fz = r.neg[2] ? loz : hiz;
    float tMin = __fmul_rn(__fsub_rn(nx, r.o.x), r.inv.x);
    float tMaxX = __fmul_rn(__fsub_rn(fx, r.o.x), r.inv.x);
    float tyMin = __fmul_rn(__fsub_rn(ny, r.o.y), r.inv.y);
    float tyMax = __fmul_rn(__fsub_rn(fy, r.o.y), r.inv.y);
    tMaxX = __fmul_rn(tMaxX, kWiden);
    tyMax = __fmul_rn(tyMax, kWiden);
    if (tMin > tyMax || tyMin > tMaxX) return false;
    if (tyMin > tMin) tMin = tyMin;
    if (tyMax < tMaxX) tMaxX = tyMax;
    float tzMin = __fmul_rn(__fsub_rn(nz, r.o.z), r.inv.z);
    float tzMax = __fmul_rn(__fsub_rn(fz, r.o.z), r.inv.z);
    tzMax = __fmul_rn(tzMax, kWiden);
    if (tMin > tzMax || tzMin > tMaxX) return false;
    if (tzMin > tMin) tMin = tzMin;
    if (tzMax < tMaxX) tMaxX = tzMax;
    *tEntry = tMin;
    return tMaxX > 0.f;
}

// The same slab test without branches, for rays whose reciprocal direction is finite: the same
// products, and max of the entries / min of the (widened) exits. For such rays every entry is at
// most its own slab's exit unless that exit is negative, so "max entry <= min exit" is the
// reference's pairwise tests and the results (accept, entry distance) are identical; rays with an
// infinite reciprocal use box_entry (its NaN handling differs from fminf / fmaxf).
__device__ __forceinline__ bool box_entry_nb(const TraceRay &r, float lox, float loy, float loz, float hix, float hiy,
                                             float hiz, float *tEntry) {
    float nx = r.neg[0] ? hix : lox, fx = r.neg[0] ? lox : hix;
    float ny = r.neg[1] ? hiy : loy, fy = r.neg[1] ? loy : hiy;
    float nz = r.neg[2] ? hiz : loz, fz = r.neg[2] ? loz : hiz;
    float t0 = fmaxf(fmaxf(__fmul_rn(__fsub_rn(nx, r.o.x), r.inv.x), __fmul_rn(__fsub_rn(ny, r.o.y), r.inv.y)),
                     __fmul_rn(__fsub_rn(nz, r.o.z), r.inv.z));
    float t1 = fminf(fminf(__fmul_rn(__fmul_rn(__fsub_rn(fx, r.o.x), r.inv.x), kWiden),
                           __fmul_rn(__fmul_rn(__fsub_rn(fy, r.o.y), r.inv.y), kWiden)),
                     __fmul_rn(__fmul_rn(__fsub_rn(fz, r.o.z), r.inv.z), kWiden));
    *tEntry = t0;
    return t0 <= t1 && t1 > 0.f;
}

// box_entry_nb with the near and far planes already chosen by the ray's octant (QNode layout:
// lo x, y, z at bytes 0, 16, 32, hi at 48, 64, 80): the same products and comparisons, folded
// with the tMax test; +inf when the box is rejected or entered at or after tMax.
__device__ __forceinline__ float slab_nf(const TraceRay &r, float nx, float fx, float ny, float fy, float nz, float fz,
                                         float tMax) {
    float t0 = fmaxf(fmaxf(__fmul_rn(__fsub_rn(nx, r.o.x), r.inv.x), __fmul_rn(__fsub_rn(ny, r.o.y), r.inv.y)),
                     __fmul_rn(__fsub_rn(nz, r.o.z), r.inv.z));
    float t1 = fminf(fminf(__fmul_rn(__fmul_rn(__fsub_rn(fx, r.o.x), r.inv.x), kWiden),
                           __fmul_rn(__fmul_rn(__fsub_rn(fy, r.o.y), r.inv.y), kWiden)),
                     __fmul_rn(__fmul_rn(__fsub_rn(fz, r.o.z), r.inv.z), kWiden));
    return t0 <= t1 && t1 > 0.f && t0 < tMax ? t0 : __int_as_float(0x7f800000);
}

// Möller-Trumbore in the reference's exact operation order (shape.cpp:202-222).
__device__ __forceinline__ float dot_rn(float ax, float ay, float az, float bx, float by, float bz) {
    return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}
__device__ __forceinline__ bool hit_triangle(const TraceRay &r, float4 v0, float4 v1, float4 v2, float tMax, float *tHit,
                                             float *bu, float *bv) {
    // pvec = d x e2
    float px = __fsub_rn(__fmul_rn(r.d.y, v2.z), __fmul_rn(r.d.z, v2.y));
    float py = __fsub_rn(__fmul_rn(r.d.z, v2.x), __fmul_rn(r.d.x, v2.z));
    float pz = __fsub_rn(__fmul_rn(r.d.x, v2.y), __fmul_rn(r.d.y, v2.x));
    float det = dot_rn(v1.x, v1.y, v1.z, px, py, pz);
    if (det == 0.f || !isfinite(det)) return false;
    float inv = __fdiv_rn(1.f, det);
    float tx = __fsub_rn(r.o.x, v0.x), ty = __fsub_rn(r.o.y, v0.y), tz = __fsub_rn(r.o.z, v0.z);
    float u = __fmul_rn(dot_rn(tx, ty, tz, px, py, pz), inv);
    if (u < 0.f || u > 1.f) return false;
    // qvec = tvec x e1
    float qx = __fsub_rn(__fmul_rn(ty, v1.z), __fmul_rn(tz, v1.y));
    float qy = __fsub_rn(__fmul_rn(tz, v1.x), __fmul_rn(tx, v1.z));
    float qz = __fsub_rn(__fmul_rn(tx, v1.y), __fmul_rn(ty, v1.x));
    float v = __fmul_rn(dot_rn(r.d.x, r.d.y, r.d.z, qx, qy, qz), inv);
    if (v < 0.f || __fadd_rn(u, v) > 1.f) return false;
    float t = __fmul_rn(dot_rn(v2.x, v2.y, v2.z, qx, qy, qz), inv);
    if (t <= 0.f || t >= tMax) return false;
    *tHit = t;
    *bu = u;
    *bv = v;
    return true;
}

// Robust sphere quadratic in double precision, as pr::Sphere::Intersect (shape.cpp:42-61).
__device__ __forceinline__ bool hit_sphere(const TraceRay &r, float4 v0, float4 v1, float tMax, float *tHit) {
    // The origin offset is a float subtraction widened afterwards, as in the reference.
    double ox = __fsub_rn(r.o.x, v0.x), oy = __fsub_rn(r.o.y, v0.y), oz = __fsub_rn(r.o.z, v0.z);
    double dx = r.d.x, dy = r.d.y, dz = r.d.z;
    double rad = v1.x;
    double a = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    double b = __dadd_rn(__dadd_rn(__dmul_rn(ox, dx), __dmul_rn(oy, dy)), __dmul_rn(oz, dz));
    double c = __dsub_rn(__dadd_rn(__dadd_rn(__dmul_rn(ox, ox), __dmul_rn(oy, oy)), __dmul_rn(oz, oz)),
                         __dmul_rn(rad, rad));
    double k = __ddiv_rn(b, a);
    double lx = __dsub_rn(ox, __dmul_rn(k, dx)), ly = __dsub_rn(oy, __dmul_rn(k, dy)),
           lz = __dsub_rn(oz, __dmul_rn(k, dz));
    double disc = __dsub_rn(__dmul_rn(rad, rad),
                            __dadd_rn(__dadd_rn(__dmul_rn(lx, lx), __dmul_rn(ly, ly)), __dmul_rn(lz, lz)));
    if (disc < 0.0) return false;
    double q = __dsub_rn(-b, copysign(__dsqrt_rn(__dmul_rn(a, disc)), b));
    double t0 = __ddiv_rn(c, q), t1 = __ddiv_rn(q, a);
    if (t0 > t1) {
        double s = t0;
        t0 = t1;
        t1 = s;
    }
    double t = t0;
    if (t <= 0.0) t = t1;
    if (t <= 0.0 || t >= double(tMax)) return false;
    *tHit = float(t);
    return true;
}

struct Hit {
    float t, u, v;
    int prim;  // original primitive index, -1 = none
};

// Closest hit (kAny = false) or any hit (kAny = true) with t in (0, tMax). Spheres are tested only
// when kSpheres. rootRef describes the root (interior WNode 0, or a single leaf), rootBox its
// bounds. Sets *overflow (and stops) when the traversal stack would overflow.
template <bool kAny, bool kSpheres>
__device__ __forceinline__ bool traverse(const WNode *__restrict__ nodes, const LeafPrim *__restrict__ prims,
                                         const float *__restrict__ rootBox, int rootRef, const TraceRay &r,
                                         float tMax, Hit *hit, bool *overflow) {
    int stackRef[kStackSize];
    float stackT[kStackSize];
    int sp = 0;
    bool found = false;
    float tEntry;
    if (!box_entry(r, rootBox[0], rootBox[1], rootBox[2], rootBox[3], rootBox[4], rootBox[5], &tEntry) ||
        !(tEntry < tMax))
        return false;
    int ref = rootRef;
    while (true) {
        if (ref >= 0) {
            const WNode *n = nodes + ref;
            float4 a = __ldg(&n->a), b = __ldg(&n->b), c = __ldg(&n->c);
            int4 rr = __ldg(&n->r);
            float t0, t1;
            bool h0 = box_entry(r, a.x, a.y, a.z, a.w, b.x, b.y, &t0);
            bool h1 = box_entry(r, b.z, b.w, c.x, c.y, c.z, c.w, &t1);
            // Near child by the sign of the split axis (bvh.cpp:184-190): the second child first
            // when the ray runs towards -axis.
            bool secondFirst = r.neg[rr.z];
            int nRef = secondFirst ? rr.y : rr.x, fRef = secondFirst ? rr.x : rr.y;
            bool nHit = secondFirst ? h1 : h0, fHit = secondFirst ? h0 : h1;
            float nT = secondFirst ? t1 : t0, fT = secondFirst ? t0 : t1;
            if (fHit) {
                if (sp >= kStackSize) {
                    *overflow = true;
                    return found;
                }
                stackRef[sp] = fRef;
                stackT[sp] = fT;
                ++sp;
            }
            if (nHit && nT < tMax) {
                ref = nRef;
                continue;
            }
        } else {
            const LeafPrim *p = prims + ~ref;
            for (bool last = false; !last; ++p) {
                float4 v0 = __ldg(&p->v0), v1 = __ldg(&p->v1), v2 = __ldg(&p->v2);
                last = __float_as_int(v2.w) != 0;
                float t, u = 0.f, v = 0.f;
                bool h;
                if (kSpheres && __float_as_int(v1.w) == 1)
                    h = hit_sphere(r, v0, v1, tMax, &t);
                else
                    h = hit_triangle(r, v0, v1, v2, tMax, &t, &u, &v);
                if (h) {
                    if (kAny) return true;
                    tMax = t;
                    hit->t = t;
                    hit->u = u;
                    hit->v = v;
                    hit->prim = __float_as_int(v0.w);
                    found = true;
                }
            }
        }
        // Pop: a deferred far child is visited only if its entry is still before tMax.
        bool next = false;
        while (sp > 0) {
            --sp;
            if (stackT[sp] < tMax) {
                ref = stackRef[sp];
                next = true;
                break;
            }
        }
        if (!next) break;
    }
    return found;
}

// The same traversal cut into steps (one interior node or one leaf per call), for persistent
// warps that hand a finished lane a new ray at once instead of waiting for the warp's longest
// ray. Visit order, box and triangle arithmetic are those of traverse(), so results are
// identical. Returns true when the ray's traversal is finished.
struct TravState {
    int ref, sp;
    float tMax;
    bool found;
    bool crossed;  // kSkipTransparent: a transparent primitive was intersected before tMax
    Hit hit;
};

// Bit of a primitive's class byte marking it transparent to shadow rays (a medium interface).
constexpr uint8_t kTransparentBit = 0x80;

template <bool kAny, bool kSpheres>
__device__ __forceinline__ bool traverse_step(const WNode *__restrict__ nodes, const LeafPrim *__restrict__ prims,
                                              const TraceRay &r, TravState &s, int *stackRef, float *stackT,
                                              bool *overflow) {
    if (s.ref >= 0) {
        const WNode *n = nodes + s.ref;
        float4 a = __ldg(&n->a), b = __ldg(&n->b), c = __ldg(&n->c);
        int4 rr = __ldg(&n->r);
        float t0, t1;
        bool h0 = box_entry(r, a.x, a.y, a.z, a.w, b.x, b.y, &t0);
        bool h1 = box_entry(r, b.z, b.w, c.x, c.y, c.z, c.w, &t1);
        bool secondFirst = r.neg[rr.z];
        int nRef = secondFirst ? rr.y : rr.x, fRef = secondFirst ? rr.x : rr.y;
        bool nHit = secondFirst ? h1 : h0, fHit = secondFirst ? h0 : h1;
        float nT = secondFirst ? t1 : t0, fT = secondFirst ? t0 : t1;
        if (fHit) {
            if (s.sp >= kStackSize) {
                *overflow = true;
                return true;
            }
            stackRef[s.sp] = fRef;
            stackT[s.sp] = fT;
            ++s.sp;
        }
        if (nHit && nT < s.tMax) {
            s.ref = nRef;
            return false;
        }
    } else {
        const LeafPrim *p = prims + ~s.ref;
        for (bool last = false; !last; ++p) {
            float4 v0 = __ldg(&p->v0), v1 = __ldg(&p->v1), v2 = __ldg(&p->v2);
            last = __float_as_int(v2.w) != 0;
            float t, u = 0.f, v = 0.f;
            bool h;
            if (kSpheres && __float_as_int(v1.w) == 1)
                h = hit_sphere(r, v0, v1, s.tMax, &t);
            else
                h = hit_triangle(r, v0, v1, v2, s.tMax, &t, &u, &v);
            if (h) {
                s.found = true;
                if (kAny) return true;
                s.tMax = t;
                s.hit.t = t;
                s.hit.u = u;
                s.hit.v = v;
                s.hit.prim = __float_as_int(v0.w);
            }
        }
    }
    while (s.sp > 0) {
        --s.sp;
        if (stackT[s.sp] < s.tMax) {
            s.ref = stackRef[s.sp];
            return false;
        }
    }
    return true;
}

// The step traversal over the 4-wide tree: the children a node's slab tests accept (entry before
// tMax) are visited nearest first, the others pushed with their entry distance, farthest first.
// Box and triangle arithmetic are those of the binary traversal, so a hit's primitive and
// distance are the reference's; only the order among hits at exactly equal distance can differ
// (the binary traversal reproduces the reference's visit order for those).
__device__ __forceinline__ void cswap(float &ta, int &ra, float &tb, int &rb) {
    if (tb < ta) {
        float t = ta;
        ta = tb;
        tb = t;
        int q = ra;
        ra = rb;
        rb = q;
    }
}

// kSkipTransparent: primitives whose class byte (cls) has kTransparentBit do not count as hits;
// intersecting one sets s.crossed.
// The traversal stack as two per-thread arrays (local memory).
struct LocalStack {
    int *ref;
    float *t;
    __device__ __forceinline__ void put(int i, int r, float d) {
        ref[i] = r;
        t[i] = d;
    }
    __device__ __forceinline__ float dist(int i) const { return t[i]; }
    __device__ __forceinline__ int node(int i) const { return ref[i]; }
};

// The bottom kShort entries of a thread's stack in shared memory, the rest in local memory. `sh`
// points at the thread's column of its block's [kShort][kThreads] array, so that the lanes of a
// warp touch consecutive words (no bank conflicts); traversals rarely go deeper than kShort, so
// the local-memory part, which shares the L1 with the node and leaf loads, is rarely touched.
template <int kShort, int kThreads>
struct HybridStack;

// Stack entries per thread in shared memory for the 4-wide traversals: 16 x 8 B x 256 threads =
// 32 KiB per block, 128 KiB per SM at 4 resident blocks (measured on the ray-query benchmark:
// 4 -> 3.27, 8 -> 3.53, 16 -> 3.83, 24 -> 3.79 Grays/s, against 3.36 with the whole stack in local
// memory).
constexpr int kShortStack = 16;

// Persistent traversal kernels refill a warp's idle lanes with new rays once this many lanes are
// idle (or none is busy). The refill (ray load, reciprocal direction, root-box test, the finished
// rays' result stores) run whenever a single lane finished executed with one or two lanes active
// in almost every iteration. Measured on the ray-query benchmark (closest / any hit, Mrays/s):
// 1 lane 3,491 / 4,770, 4 lanes 3,704 / 5,110, 8 lanes 3,829 / 5,319, 16 lanes 3,562 / 4,960.
// Results are unchanged: only the iteration at which a lane starts its next ray moves.
constexpr int kRefillLanes = 8;

template <int kShort, int kThreads>
struct HybridStack {
    int2 *sh;
    int ref[kStackSize - kShort];
    float t[kStackSize - kShort];
    __device__ __forceinline__ void put(int i, int r, float d) {
        if (i < kShort) {
            sh[i * kThreads] = make_int2(r, __float_as_int(d));
        } else {
            ref[i - kShort] = r;
            t[i - kShort] = d;
        }
    }
    __device__ __forceinline__ float dist(int i) const {
        return i < kShort ? __int_as_float(sh[i * kThreads].y) : t[i - kShort];
    }
    __device__ __forceinline__ int node(int i) const { return i < kShort ? sh[i * kThreads].x : ref[i - kShort]; }
};

// kDeferUV (closest hit): a hit records only its leaf slot (s.hit.prim) and distance (s.tMax);
// the caller repeats the winning primitive's test once at the end (finish_hit), which gives the
// same t, u, v bit for bit. Fewer live registers in the loop let the slab planes be selected by
// address as for any hit (ray-query benchmark, closest hit: 3,821 -> 3,926 Mrays/s; either change
// alone was slower: 3,730 and 3,667).
template <bool kAny, bool kSpheres, bool kSkipTransparent = false, bool kDeferUV = false, class Stack>
__device__ __forceinline__ bool traverse4_step_st(const QNode *__restrict__ nodes, const LeafPrim *__restrict__ prims,
                                                  const TraceRay &r, TravState &s, Stack &stack, bool *overflow,
                                                  const uint8_t *__restrict__ cls = nullptr) {
    if (s.ref >= 0) {
        const QNode *n = nodes + s.ref;
        float t0, t1, t2, t3;
        const float inf = __int_as_float(0x7f800000);
        int4 ch;
        if constexpr (kAny || kDeferUV) {
            ch = __ldg(&n->child);
            if (!r.infInv) {
                // The near and far planes chosen by address from the ray's octant (six loads, no
                // per-child selects). Measured on the ray-query benchmark: any hit 5,314 -> 5,689
                // Mrays/s; closest hit only together with kDeferUV (see above); the closest-hit
                // form that keeps t, u, v live loads all six plane vectors below.
                const char *nb = reinterpret_cast<const char *>(n);
                const int ox = r.neg[0] ? 48 : 0, oy = r.neg[1] ? 48 : 0, oz = r.neg[2] ? 48 : 0;
                const float4 nx = __ldg(reinterpret_cast<const float4 *>(nb + ox));
                const float4 fx = __ldg(reinterpret_cast<const float4 *>(nb + 48 - ox));
                const float4 ny = __ldg(reinterpret_cast<const float4 *>(nb + 16 + oy));
                const float4 fy = __ldg(reinterpret_cast<const float4 *>(nb + 64 - oy));
                const float4 nz = __ldg(reinterpret_cast<const float4 *>(nb + 32 + oz));
                const float4 fz = __ldg(reinterpret_cast<const float4 *>(nb + 80 - oz));
                t0 = slab_nf(r, nx.x, fx.x, ny.x, fy.x, nz.x, fz.x, s.tMax);
                t1 = slab_nf(r, nx.y, fx.y, ny.y, fy.y, nz.y, fz.y, s.tMax);
                t2 = slab_nf(r, nx.z, fx.z, ny.z, fy.z, nz.z, fz.z, s.tMax);
                t3 = slab_nf(r, nx.w, fx.w, ny.w, fy.w, nz.w, fz.w, s.tMax);
            } else {
                const float4 lx = __ldg(&n->lox), ly = __ldg(&n->loy), lz = __ldg(&n->loz);
                const float4 hx = __ldg(&n->hix), hy = __ldg(&n->hiy), hz = __ldg(&n->hiz);
                t0 = box_entry(r, lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, &t0) && t0 < s.tMax ? t0 : inf;
                t1 = box_entry(r, lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, &t1) && t1 < s.tMax ? t1 : inf;
                t2 = box_entry(r, lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, &t2) && t2 < s.tMax ? t2 : inf;
                t3 = box_entry(r, lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, &t3) && t3 < s.tMax ? t3 : inf;
            }
        } else {
            const float4 lx = __ldg(&n->lox), ly = __ldg(&n->loy), lz = __ldg(&n->loz);
            const float4 hx = __ldg(&n->hix), hy = __ldg(&n->hiy), hz = __ldg(&n->hiz);
            ch = __ldg(&n->child);
            if (!r.infInv) {
                t0 = box_entry_nb(r, lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, &t0) && t0 < s.tMax ? t0 : inf;
                t1 = box_entry_nb(r, lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, &t1) && t1 < s.tMax ? t1 : inf;
                t2 = box_entry_nb(r, lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, &t2) && t2 < s.tMax ? t2 : inf;
                t3 = box_entry_nb(r, lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, &t3) && t3 < s.tMax ? t3 : inf;
            } else {
                t0 = box_entry(r, lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, &t0) && t0 < s.tMax ? t0 : inf;
                t1 = box_entry(r, lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, &t1) && t1 < s.tMax ? t1 : inf;
                t2 = box_entry(r, lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, &t2) && t2 < s.tMax ? t2 : inf;
                t3 = box_entry(r, lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, &t3) && t3 < s.tMax ? t3 : inf;
            }
        }
        int r0 = ch.x, r1 = ch.y, r2 = ch.z, r3 = ch.w;
        // Sorting network for 4 (5 compare-exchanges); misses sort last at +inf.
        cswap(t0, r0, t1, r1);
        cswap(t2, r2, t3, r3);
        cswap(t0, r0, t2, r2);
        cswap(t1, r1, t3, r3);
        cswap(t1, r1, t2, r2);
        if (t0 < inf) {
            const int extra = (t1 < inf) + (t2 < inf) + (t3 < inf);
            if (s.sp + extra > kStackSize) {
                *overflow = true;
                return true;
            }
            if (t3 < inf) stack.put(s.sp++, r3, t3);
            if (t2 < inf) stack.put(s.sp++, r2, t2);
            if (t1 < inf) stack.put(s.sp++, r1, t1);
            s.ref = r0;
            return false;
        }
    } else {
        const LeafPrim *p = prims + ~s.ref;
        for (bool last = false; !last; ++p) {
            float4 v0 = __ldg(&p->v0), v1 = __ldg(&p->v1), v2 = __ldg(&p->v2);
            last = __float_as_int(v2.w) != 0;
            float t, u = 0.f, v = 0.f;
            bool h;
            if (kSpheres && __float_as_int(v1.w) == 1)
                h = hit_sphere(r, v0, v1, s.tMax, &t);
            else
                h = hit_triangle(r, v0, v1, v2, s.tMax, &t, &u, &v);
            if (h) {
                if (kSkipTransparent && (__ldg(cls + __float_as_int(v0.w)) & kTransparentBit)) {
                    s.crossed = true;
                    continue;
                }
                s.found = true;
                if (kAny) return true;
                s.tMax = t;
                if constexpr (kDeferUV) {
                    s.hit.prim = int(p - prims);
                } else {
                    s.hit.t = t;
                    s.hit.u = u;
                    s.hit.v = v;
                    s.hit.prim = __float_as_int(v0.w);
                }
            }
        }
    }
    while (s.sp > 0) {
        --s.sp;
        if (stack.dist(s.sp) < s.tMax) {
            s.ref = stack.node(s.sp);
            return false;
        }
    }
    return true;
}

// The hit of a kDeferUV traversal: the winning leaf slot's test repeated (no tMax bound), which
// reproduces the distance and barycentrics the traversal computed; prim = the original index.
template <bool kSpheres>
__device__ __forceinline__ Hit finish_hit(const LeafPrim *__restrict__ prims, const TraceRay &r, const TravState &s) {
    Hit h{0.f, 0.f, 0.f, -1};
    if (!s.found) return h;
    const LeafPrim *p = prims + s.hit.prim;
    const float4 v0 = __ldg(&p->v0), v1 = __ldg(&p->v1);
    const float inf = __int_as_float(0x7f800000);
    if (kSpheres && __float_as_int(v1.w) == 1)
        hit_sphere(r, v0, v1, inf, &h.t);
    else
        hit_triangle(r, v0, v1, __ldg(&p->v2), inf, &h.t, &h.u, &h.v);
    h.prim = __float_as_int(v0.w);
    return h;
}

template <bool kAny, bool kSpheres, bool kSkipTransparent = false>
__device__ __forceinline__ bool traverse4_step(const QNode *__restrict__ nodes, const LeafPrim *__restrict__ prims,
                                               const TraceRay &r, TravState &s, int *stackRef, float *stackT,
                                               bool *overflow, const uint8_t *__restrict__ cls = nullptr) {
    LocalStack st{stackRef, stackT};
    return traverse4_step_st<kAny, kSpheres, kSkipTransparent>(nodes, prims, r, s, st, overflow, cls);
}

} // namespace prb
