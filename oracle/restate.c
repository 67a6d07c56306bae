/* Plain-C restatement of the reference traversal; see restate.h. TEST INFRASTRUCTURE only.
 * Compiled with -ffp-contract=off so that every product is rounded before it is summed, as in the
 * reference's ISO C++ build. */
#include "restate.h"

#include <math.h>
#include <stddef.h>

/* Widening factor of the far slab distances: 1 + 2 * 1.2e-7f * 3 in float (bvh.cpp:143-151). */
static const float kWiden = 1.0f + 2.0f * 1.2e-7f * 3.0f;

/* bvh.cpp:137-156 */
static int box_hit(const rs_node *b, const float o[3], const float inv[3], const int neg[3], float tMax) {
    const float *lo = b->bmin, *hi = b->bmax;
    float tMin = ((neg[0] ? hi : lo)[0] - o[0]) * inv[0];
    float tMaxX = ((neg[0] ? lo : hi)[0] - o[0]) * inv[0];
    float tyMin = ((neg[1] ? hi : lo)[1] - o[1]) * inv[1];
    float tyMax = ((neg[1] ? lo : hi)[1] - o[1]) * inv[1];
    tMaxX *= kWiden;
    tyMax *= kWiden;
    if (tMin > tyMax || tyMin > tMaxX) return 0;
    if (tyMin > tMin) tMin = tyMin;
    if (tyMax < tMaxX) tMaxX = tyMax;
    float tzMin = ((neg[2] ? hi : lo)[2] - o[2]) * inv[2];
    float tzMax = ((neg[2] ? lo : hi)[2] - o[2]) * inv[2];
    tzMax *= kWiden;
    if (tMin > tzMax || tzMin > tMaxX) return 0;
    if (tzMin > tMin) tMin = tzMin;
    if (tzMax < tMaxX) tMaxX = tzMax;
    return (tMin < tMax) && (tMaxX > 0);
}

/* shape.cpp:202-222 */
static int tri_hit(const float *v, const float o[3], const float d[3], float tMax, float *tHit, float *bu) {
    float e1[3] = {v[3] - v[0], v[4] - v[1], v[5] - v[2]};
    float e2[3] = {v[6] - v[0], v[7] - v[1], v[8] - v[2]};
    float p[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]};
    float det = e1[0] * p[0] + e1[1] * p[1] + e1[2] * p[2];
    if (det == 0 || !isfinite(det)) return 0;
    float inv = 1 / det;
    float tv[3] = {o[0] - v[0], o[1] - v[1], o[2] - v[2]};
    float u = (tv[0] * p[0] + tv[1] * p[1] + tv[2] * p[2]) * inv;
    if (u < 0 || u > 1) return 0;
    float q[3] = {tv[1] * e1[2] - tv[2] * e1[1], tv[2] * e1[0] - tv[0] * e1[2], tv[0] * e1[1] - tv[1] * e1[0]};
    float vv = (d[0] * q[0] + d[1] * q[1] + d[2] * q[2]) * inv;
    if (vv < 0 || u + vv > 1) return 0;
    float tt = (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]) * inv;
    if (tt <= 0 || tt >= tMax) return 0;
    *tHit = tt;
    *bu = u;
    return 1;
}

int rs_trace(const rs_node *nodes, int64_t nodeCount, const int32_t *order, const float *verts, const float *rays,
             int64_t n, int anyHit, int32_t *prim, float *t, int32_t *nodesVisited, int32_t *trisTested) {
    int status = 0;
    for (int64_t r = 0; r < n; ++r) {
        const float *ry = rays + 8 * r;
        float o[3] = {ry[0], ry[1], ry[2]}, d[3] = {ry[3], ry[4], ry[5]}, tMax = ry[6];
        float inv[3] = {1 / d[0], 1 / d[1], 1 / d[2]};
        int neg[3] = {inv[0] < 0, inv[1] < 0, inv[2] < 0};
        int stack[64], sp = 0, cur = 0, found = 0, best = -1, visited = 0, tested = 0;
        float bestT = 0;
        if (nodeCount > 0) {
            for (;;) {
                const rs_node *nd = nodes + cur;
                ++visited;
                if (box_hit(nd, o, inv, neg, tMax)) {
                    if (nd->nPrims > 0) {
                        for (int i = 0; i < nd->nPrims; ++i) {
                            int slot = nd->offset + i;
                            float th, bu;
                            ++tested;
                            if (tri_hit(verts + 9 * (size_t)order[slot], o, d, tMax, &th, &bu)) {
                                found = 1;
                                if (anyHit) goto done;
                                tMax = th;
                                bestT = th;
                                best = order[slot];
                            }
                        }
                        if (sp == 0) break;
                        cur = stack[--sp];
                    } else {
                        if (sp >= 64) {
                            status = 1;
                            break;
                        }
                        if (neg[nd->axis]) {
                            stack[sp++] = cur + 1;
                            cur = nd->offset;
                        } else {
                            stack[sp++] = nd->offset;
                            cur = cur + 1;
                        }
                    }
                } else {
                    if (sp == 0) break;
                    cur = stack[--sp];
                }
            }
        }
    done:
        if (anyHit) {
            prim[r] = found;
        } else {
            prim[r] = found ? best : -1;
            if (t) t[r] = found ? bestT : 0;
        }
        if (nodesVisited) nodesVisited[r] = visited;
        if (trisTested) trisTested[r] = tested;
    }
    return status;
}
