// Internal device/host structures of the xtgpu library (sm_100a).
//
// Data layout in HBM (all structure-of-arrays, 16-byte aligned):
//   leaf primitives, in Morton order   3 x float4 (48 B) per primitive
//       triangle: (v0.xyz, id) (v1.xyz, 0) (v2.xyz, 0)
//       sphere:   (c.xyz, id | SPHERE_BIT) (r, 0, 0, 0) (0)
//   FP32 BVH node                      4 x float4 (64 B): both child boxes + refs
//   Q8 BVH node                        2 x uint4 (32 B): origin+exponents, 8-bit
//                                      child bounds rounded outward, refs
//   W8 BVH node (8-wide)               5 x uint4 (80 B): origin+exponents, child
//                                      masks and bases, 48 8-bit child bounds
//   rays                               float4 (org, tmin) + float4 (dir, tmax)
//   hits                               (t, prim, u, v) 16 B
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/xtgpu.h"

namespace xtg {

constexpr uint32_t SPHERE_BIT = 0x80000000u;
constexpr int LEAF_BITS = 3;                  // leaf ref: ~((first << 3) | count)
constexpr int MAX_LEAF = (1 << LEAF_BITS) - 1;
constexpr int32_t EMPTY_REF = ~0;             // leaf of 0 primitives
constexpr int STACK_MAX = 64;

__host__ __device__ inline int32_t leaf_ref(uint32_t first, uint32_t count)
{
    return ~(int32_t)((first << LEAF_BITS) | count);
}
__host__ __device__ inline uint32_t leaf_first(int32_t ref) { return ((uint32_t)~ref) >> LEAF_BITS; }
__host__ __device__ inline uint32_t leaf_count(int32_t ref) { return ((uint32_t)~ref) & MAX_LEAF; }

// A sampler (xtgpu_sampler): kind, texture index, colours a and b.
struct DevSampler {
    int kind, tex;
    float3 a, b;
};

struct DevTexture {
    int32_t width, height, filtering, reserved;
    int64_t offset;
    uint32_t wrap_w, wrap_h;   // 2^64 mod width, 2^64 mod height (bilinear index wrap)
};

// diffuse, specular and emissive are the colours of COLOR samplers; a
// textured material (any other sampler kind) samples s[] at the hit texcoord.
struct DevMaterial {
    int type;
    float3 diffuse, specular, emissive;
    float reflectance, exponent, ior;
    int textured;
    DevSampler s[3];      // diffuse, specular, emissive
};

// Camera basis precomputed on the host in FP64 exactly as
// Perspective::calculate_transform (camera/perspective.cc:26-36).
struct DevCamera {
    int type;             // XTGPU_CAM_*
    double pos[3];
    double rx[3], ry[3], rz[3];
    double dz;            // 1 / tan(fov * RADIAN / 2)
    double rot[3][4];     // ERP, ODS: Matrix4x4f::rotate(orientation) of an identity
    float ipd;            // ODS
    float flength, aperture;   // perspective depth of field (flength > 0)
};
// anti-aliasing levels accepted: grid up to 16 (aa^2 positions per pixel),
// random up to 256 (aa positions)
constexpr int MAX_AA = 16;

// Everything a kernel needs to intersect and shade one scene.
struct DevScene {
    // geometry in the desc order (shading)
    const float4 *tri_v;       // 3 per triangle
    const float4 *tri_n;       // 3 per triangle, or nullptr
    const float4 *spheres;     // (c, r)
    const float4 *planes;      // (n, offset)
    const int32_t *prim_obj;   // object of each primitive id (tris, spheres, planes)
    const int32_t *obj_material;
    const int32_t *prim_mat;   // material of each primitive id (obj_material[prim_obj[i]])
    int32_t has_lobe;          // some material is Phong or BlinnPhong (a specular lobe to sample)
    const DevMaterial *materials;
    const float2 *obj_uvs;     // per object: the surface's (u_scale, v_scale)
    const float2 *tri_uv;      // 3 per triangle, or nullptr (constructor defaults)
    int32_t n_tris, n_spheres, n_planes;
    // BVH
    const float4 *leaf_prims;  // 3 per primitive, Morton order
    const float4 *nodes32;     // 4 per node
    const uint4 *nodes8;       // 2 per node
    int32_t root;              // ref of the root (>= 0 node, < 0 leaf)
    // 8-wide BVH (wide.cu): 5 uint4 per node, its own copy of the primitives
    const uint4 *nodesW;
    const float4 *leafW;
    int32_t rootW;             // 0, or -1 for an empty scene
    int32_t env_type;
    float3 env_a, env_b;
    int32_t env_tex;           // XTGPU_ENV_ERP / XTGPU_ENV_CUBEMAP: its (first) texture
    const DevTexture *textures;
    const float4 *texels;
    DevCamera cam;
};

// Host-side scene object behind the C handle.
struct HostBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

}  // namespace xtg

struct xtgpu_scene {
    xtg::DevScene dev{};
    xtg::HostBuf tri_v, tri_n, spheres, planes, prim_obj, obj_material, prim_mat, materials, obj_uvs, tri_uv;
    xtg::HostBuf textures, texels;
    xtg::HostBuf leaf_prims, nodes32, nodes8, nodesW, leafW;
    xtg::HostBuf morton, order, left, right;   // kept for xtgpu_bvh_export
    int64_t n_prims = 0;
    int32_t depth = 0;
    int32_t leaf_size = 2;
    int32_t layout = 0;
    int32_t builder = 0;
    int32_t last_format = XTGPU_NODES_FP32;
    bool built32 = false, built8 = false, builtW = false;
    int32_t depthW = 0;        // levels of the 8-wide BVH
    int32_t wide_collapse = 1; // how it was collapsed (xtgpu_tuning::wide_collapse)
    float wide_prim_cost = 1.0f;
    int32_t n_wide = 0;        // its nodes
    int device = 0;
    // host copies used by the service and the tests
    int32_t n_objects = 0;
    // tuning picked by xtgpu_autotune for this scene
    xtgpu_tuning tune{};
    bool tuned = false;
};

namespace xtg {

// error plumbing -----------------------------------------------------------
void set_error(const std::string &msg);
xtgpu_status cuda_fail(cudaError_t e, const char *what, const char *file, int line);

#define XTG_CUDA(call)                                                              \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) return xtg::cuda_fail(e_, #call, __FILE__, __LINE__); \
    } while (0)

#define XTG_TRY(call)                          \
    do {                                       \
        xtgpu_status s_ = (call);              \
        if (s_ != XTGPU_OK) return s_;         \
    } while (0)

xtgpu_status dalloc(HostBuf &b, size_t bytes, cudaStream_t s);
void dfree(HostBuf &b);

// BVH build (bvh.cu); the 8-wide collapse of the built binary tree (wide.cu)
// builder: 0 = LBVH (Karras), 1 = PLOC over the same Morton order
xtgpu_status build_bvh(xtgpu_scene *sc, int node_format, int leaf_size, int layout, cudaStream_t s, int builder);
xtgpu_status build_wide(xtgpu_scene *sc, cudaStream_t s);

// node formats
inline bool format_valid(int f) { return f == XTGPU_NODES_FP32 || f == XTGPU_NODES_Q8 || f == XTGPU_NODES_W8; }
inline bool format_built(const xtgpu_scene *sc, int f)
{
    return (f == XTGPU_NODES_FP32 && sc->built32) || (f == XTGPU_NODES_Q8 && sc->built8) ||
           (f == XTGPU_NODES_W8 && sc->builtW);
}
// traversal stack entries (32 or 64) for this scene's tree in format f
int stack_for_scene(const xtgpu_scene *sc, int f, int requested);

// cameras: the device form of a camera, whether a camera description is
// acceptable, and whether a frame size suits a camera and the samples
// (distribution, level, samples per position) are within range
DevCamera make_camera(const xtgpu_camera &c);
bool camera_valid(const xtgpu_camera &c);
bool view_valid(const DevCamera &c, int width, int height, int aa, int dist, int spp);

// the tuning a scene renders with: its own if autotuned, else the process-wide one
const xtgpu_tuning &scene_tuning(const xtgpu_scene *sc);
// xtgpu_render with an explicit launch configuration (the autotuner's probe)
// raygraph: the depth integrator's per-sample records (DevJob::raygraph), or null
xtgpu_status render_impl(xtgpu_scene *sc, const xtgpu_render_params *p, float *rgba, uint64_t *rays,
                         cudaStream_t s, const xtgpu_tuning &T, float *raygraph = nullptr);

}  // namespace xtg
