// The scene on the device: the caller's SceneDesc (v4 layout, src/gpu/gpu_api.h:120-146) checked,
// converted and kept resident between calls, plus the optional light BVH of the v5 extension.
//
// HBM layout: the traversal arrays of traverse.cuh (64-byte interior nodes, 48-byte leaf
// records in leaf order), the 128-byte Primitive records for shading (read once per hit), and
// the small tables (materials, lights, media, 95-sample spectra, filter CDF, light-BVH nodes).
#pragma once

#include <string>
#include <vector>

#include "accel.cuh"
#include "device.cuh"

namespace prb {

// A heterogeneous medium on the device (GridMediumDesc with its density grid resident in HBM).
constexpr int kMaxWallList = 64;

struct DevGrid {
    float w2m[12];
    float bmin[3], bmax[3];
    int nx, ny, nz;
    float maxDensity;
    float scale, g;
    int sigmaA, sigmaS;
    const float *density;
    // Macro-cell majorants: mx * my * mz cells tiling the bounds, x fastest, each >= the
    // trilinear density anywhere in the cell (a one-voxel margin on every side).
    int mx, my, mz;
    const float *majorant;
    // pr::NoiseField in place of the voxels (noise != 0). boundless: a noise field with empty bounds,
    // which fills every finite segment (medium.cpp:168-177, GridMedium::Clip, medium.cpp:182-188).
    int noise, noiseOctaves, noiseFalloff, boundless;
    float noiseFrequency, noiseThreshold, noiseSharpness;
    float noiseOffset[3];
    // Index-space voxels (indexed != 0): voxel (x, y, z) at integer coordinate org + (x, y, z).
    int indexed;
    int org[3];
};

// Shading classes: the closest-hit kernel files every finished path under one of these, and the
// shading kernel walks the classes in order, so a warp mostly runs one material's code.
enum ShadeClass : int {
    kClassMiss = 0,        // escaped, not in a medium
    kClassDiffuse = 1,
    kClassConductor = 2,
    kClassDielectric = 3,  // smooth, rough or thin
    kClassOther = 4,       // interfaces, black and anything else
    kClassMedium = 5,      // the path is inside a medium (free flight first)
    kClassGuided = 6,      // diffuse, at one of the first diffuse vertices of a path whose render
                           // uses the path guide (its inference runs on this class's queue only)
    kClasses = 7
};

// Image environment on the device: texels (sigmoid-polynomial spectra), and the 2D sampling
// distribution of luminance x sin(theta) as per-row CDFs and a marginal CDF.
struct DevEnvMap {
    int w, h;                  // w = 0: none
    const float4 *texels;      // c0, c1, c2, scale
    const float *func;         // w * h
    const float *rowCdf;       // h x (w + 1)
    const float *rowInt;       // h
    const float *margCdf;      // h + 1
    float margInt;
    int illuminant;
    float scale, pmf;
    float rc, rs;              // cos / sin of the rotation about +y (light to world)
};

struct DevSun {
    V3 x, y, z;                // frame around the sun direction z
    float cosMax;
    int spectrum;              // -1: none
    float scale, pmf;
};

// A spot, distant or goniometric light (prgpu::DeltaLightDesc on the device).
struct DevDelta {
    int type, spectrum;
    float scale, pmf;
    V3 pos, dir;             // dir: spot axis; distant: towards the light
    float cosStart, cosEnd;  // spot falloff
    V3 fx, fy, fz;           // goniometric profile frame
    int nV, nH;
    const float *profile;    // vAngles[nV], hAngles[nH], candela[nH][nV]
};

// An image texture on the device (prgpu::ImageTextureDesc).
struct DevTex {
    int w, h;
    const float *rgb;
    int wrap, flipV;
    float su, sv, ou, ov;
    float scale[3];
};

struct DevScene {
    const WNode *nodes;
    const QNode *qnodes;   // the 4-wide collapse of the same tree
    const LeafPrim *leaves;
    RootInfo root;
    const prgpu::Primitive *prims;
    const uint8_t *primClass;    // shading class of each primitive's material (ShadeClass), | kTransparentBit
                                 // for medium interfaces
    const prgpu::Material *mats;
    const prgpu::Light *lights;
    int lightCount;
    const float *spectra;
    const prgpu::Medium *media;
    int cameraMedium;
    int envSpectrum;
    float envScale;
    float envPmf;         // selection probability of the environment in next-event estimation
    float worldRadius;
    prgpu::Camera cam;
    float norm;           // 1 / (4 * integral of CIE y): XYZ normalisation of one sample
    int hasInterfaces;
    int hasFull;  // some material is coated or has sheen (the kFull shading pass runs)
    // The medium-interface primitives as leaf slots, for the shadow walk's closest-hit queries
    // (brute force over at most kMaxWallList); wallCount < 0: too many, the walk uses the tree.
    const LeafPrim *walls;
    int wallCount;
    const float *sheenTable;  // sheen directional albedo [16 alpha][32 mu], null without sheen
    uint32_t filterType;
    float filterRadius, filterSigma, filterNorm;
    const float *filterCdf;  // kFilterBins + 1
    // Light BVH (lbvhCount > 0 selects importance sampling of the bounded lights).
    const prgpu::LightBVHNode *lbvh;
    int lbvhCount;
    float lbvhProb;          // probability of the BVH branch (1 - probability of the environment)
    const int *lightLeaf;    // light index -> leaf node (-1 when the light is not in the tree)
    // Heterogeneous media: medium index m >= mediumCount names grids[m - mediumCount].
    int mediumCount;
    const DevGrid *grids;
    int gridCount;
    DevEnvMap envMap;
    DevSun sun;
    const DevDelta *deltas;
    int deltaCount;
    // Image textures and procedural texture trees; matTex is null unless a material uses one.
    const DevTex *textures;
    // per material four entries: (reflectance texture, normal map, strength bits, flip green),
    // (bump map, channel, scale bits, reflectance tree), (bump tree, roughness trees u, v, sheen
    // roughness tree) and (coat roughness, thickness, coat albedo, sheen colour trees)
    const int4 *matTex;
    const prgpu::TextureNode *texNodes;
    const float *rgbZ, *rgbCoeffs;
    int texCount;
    // Per-render settings of the batched form (the single-render kernels take them as arguments).
    int maxDepth;            // <= 0: unlimited
    float clampY;            // 0: off
    double *film;            // the render's device FP64 film, 3 doubles per pixel
    int guideMode;           // the render's guide flags (bit 0 sample with the guide, bit 1 train it)
};

struct SceneCache {
    uint64_t key = 0;
    bool valid = false;
    DeviceAccel accel;
    DevBuf prims, primClass, mats, lights, spectra, media, filterCdf, lbvh, lightLeaf, grids, gridData, envTexels,
        envDist, walls, sheen, deltas, deltaProfiles, textures, texData, matTex, texNodes, rgbTable;
    DevScene ds{};
    bool hasSpheres = false;
    int wallCount = 0;
    bool hasSheen = false;
    int64_t deviceBytes = 0;
    void release() {
        accel.release();
        prims.release();
        primClass.release();
        mats.release();
        lights.release();
        spectra.release();
        media.release();
        filterCdf.release();
        lbvh.release();
        lightLeaf.release();
        grids.release();
        gridData.release();
        envTexels.release();
        envDist.release();
        walls.release();
        sheen.release();
        deltas.release();
        deltaProfiles.release();
        textures.release();
        texData.release();
        matTex.release();
        texNodes.release();
        rgbTable.release();
        valid = false;
    }
};

// The sheen directional-albedo table a host passes in SceneDesc::sheenAlbedo, computed on the host.
std::vector<float> sheen_albedo_table();

// Validates sd (and ext) and makes the cache hold it on the device. Throws CudaError on device
// failure; returns false with a message on invalid input.
bool upload_scene(DeviceState &ds, const prgpu::SceneDesc *sd, const prgpu::SceneExt *ext, SceneCache &cache,
                  std::string *err);

} // namespace prb
