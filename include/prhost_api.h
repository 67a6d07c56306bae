// prhost_api.h -- C ABI of libprender_host.so, the C++ host side that prepares scenes for the
// CUDA module: it builds the acceleration structures a SceneDesc carries.
//
// In PRender the host builds its BVH in pr::BVH::Build (src/geometry/bvh.cpp:8-135) and hands the
// flattened nodes to the GPU module (src/integrators/gpu_path.cpp:378-390); its light BVH is
// pr::BVHLightSampler (src/lights/light_bvh.cpp:103-177). These entry points produce the same
// node formats (prgpu::BVHNode, prgpu::LightBVHNode) from plain arrays, so a caller without
// PRender's scene classes can drive libprender_gpu.so.
#pragma once

#include <cstdint>

#include "prgpu_api.h"

#if defined(_WIN32)
#define PRHOST_API extern "C" __declspec(dllexport)
#else
#define PRHOST_API extern "C" __attribute__((visibility("default")))
#endif

// Binned-SAH BVH over primitive bounds (boxMin/boxMax: 3 floats per primitive). Writes at most
// 2 * primCount - 1 nodes in depth-first order (first child follows its parent, offset = second
// child; leaves hold primOrder[offset .. offset + nPrims)) and the leaf-slot permutation.
// maxLeaf bounds primitives per leaf (1..8); threads = 0 uses all hardware threads.
// Returns the node count, or -1 on bad arguments. Replaces pr::BVH::Build (bvh.cpp:8-135).
PRHOST_API int64_t prhost_build_bvh(const float *boxMin, const float *boxMax, int64_t primCount, int32_t maxLeaf,
                                    int32_t threads, prgpu::BVHNode *nodesOut, int32_t *primOrderOut);

// Triangle-soup convenience: bounds from 3 vertices per primitive.
PRHOST_API int64_t prhost_build_bvh_triangles(const prgpu::Float3 *verts, int64_t primCount, int32_t maxLeaf,
                                              int32_t threads, prgpu::BVHNode *nodesOut, int32_t *primOrderOut);

// Light BVH over bounded lights (Conty & Kulla importance, 12-bucket SAOH on 3 axes, as
// src/lights/light_bvh.cpp:90-177). Per light: bounds (6 floats), emission cone axis w (3),
// phi, cosThetaO, cosThetaE, twoSided (as float 0/1): 13 floats. Writes 2 * n - 1 nodes; returns
// the node count or -1.
PRHOST_API int32_t prhost_build_light_bvh(const float *lightBounds13, int32_t lightCount,
                                          prgpu::LightBVHNode *nodesOut);
