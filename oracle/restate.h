/* Plain-C restatement of the reference's ray traversal (TEST INFRASTRUCTURE: the oracle).
 * Follows src/geometry/bvh.cpp:137-232 (slab test, stack traversal, child order) and
 * src/geometry/shape.cpp:202-222 (Moller-Trumbore) operation for operation, over the flattened
 * node layout of src/gpu/gpu_api.h:35-40. It also counts visited nodes and tested triangles,
 * the per-ray work figures the roofline accounting uses. Pinned bit-exactly against the
 * reference build in oracle/_ref/libprref.so by tests/test_oracle.py. */
#pragma once
#include <stdint.h>

typedef struct {
    float bmin[3], bmax[3];
    int32_t offset;
    uint16_t nPrims;
    uint8_t axis, pad;
} rs_node;

/* rays: n x 8 floats (o, d, tmax, pad); verts: 9 floats per triangle (original order).
 * Closest hit (anyHit = 0): prim = original index or -1, t, b1 (may be NULL), counters
 * nodesVisited / trisTested per ray (may be NULL). Any hit: prim = 1/0.
 * Returns 0, or 1 if a traversal stack of 64 entries overflowed. */
int rs_trace(const rs_node *nodes, int64_t nodeCount, const int32_t *order, const float *verts, const float *rays,
             int64_t n, int anyHit, int32_t *prim, float *t, int32_t *nodesVisited, int32_t *trisTested);
