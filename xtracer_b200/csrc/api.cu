// C ABI entry points (include/xtgpu.h): scene upload, BVH build/export, batched
// closest-hit tracing and single-job frame rendering.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "render.h"

namespace xtg {

static thread_local std::string g_err;

void set_error(const std::string &msg) { g_err = msg; }

xtgpu_status cuda_fail(cudaError_t e, const char *what, const char *file, int line)
{
    char buf[512];
    snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    g_err = buf;
    return e == cudaErrorMemoryAllocation ? XTGPU_ERR_NOMEM : XTGPU_ERR_CUDA;
}

xtgpu_status dalloc(HostBuf &b, size_t bytes, cudaStream_t s)
{
    (void)s;
    dfree(b);
    cudaError_t e = cudaMalloc(&b.p, bytes ? bytes : 16);
    if (e != cudaSuccess) {
        b.p = nullptr;
        return cuda_fail(e, "cudaMalloc", __FILE__, __LINE__);
    }
    b.bytes = bytes;
    return XTGPU_OK;
}

void dfree(HostBuf &b)
{
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
}

// Perspective::calculate_transform (camera/perspective.cc:26-36) in FP64.
struct d3 {
    double x, y, z;
};
static d3 dsub(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static d3 dcross(d3 a, d3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
static d3 dnorm(d3 a)
{
    double l = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
    return l != 0 ? d3{a.x / l, a.y / l, a.z / l} : a;
}

DevCamera make_camera(const xtgpu_camera &c)
{
    DevCamera k;
    d3 pos{c.position[0], c.position[1], c.position[2]};
    d3 tgt{c.target[0], c.target[1], c.target[2]};
    d3 up{c.up[0], c.up[1], c.up[2]};
    d3 rz = dnorm(dsub(tgt, pos));
    d3 rx = dnorm(dcross(up, rz));
    d3 ry = dnorm(dcross(rx, rz));
    k.pos[0] = pos.x; k.pos[1] = pos.y; k.pos[2] = pos.z;
    k.rx[0] = rx.x; k.rx[1] = rx.y; k.rx[2] = rx.z;
    k.ry[0] = ry.x; k.ry[1] = ry.y; k.ry[2] = ry.z;
    k.rz[0] = rz.x; k.rz[1] = rz.y; k.rz[2] = rz.z;
    const double RADIAN = 0.017453292519943;   // lib/nmath/precision.h:111
    k.dz = 1.0 / std::tan(c.fov * RADIAN / 2.0);
    k.type = c.type;
    k.ipd = c.ipd;
    k.flength = c.flength;
    k.aperture = c.aperture;
    // ERP and ODS turn their direction by Matrix4x4f::rotate(orientation)
    // applied to the identity (lib/nmath/matrix.cc:414-427, 485-492):
    // I *= (xrot * yrot * zrot), every product summed left to right.
    const double ex = c.orientation[0], ey = c.orientation[1], ez = c.orientation[2];
    const double xr[3][3] = {{1, 0, 0}, {0, std::cos(ex), -std::sin(ex)}, {0, std::sin(ex), std::cos(ex)}};
    const double yr[3][3] = {{std::cos(ey), 0, std::sin(ey)}, {0, 1, 0}, {-std::sin(ey), 0, std::cos(ey)}};
    const double zr[3][3] = {{std::cos(ez), -std::sin(ez), 0}, {std::sin(ez), std::cos(ez), 0}, {0, 0, 1}};
    double xy[3][3], r3[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) xy[i][j] = xr[i][0] * yr[0][j] + xr[i][1] * yr[1][j] + xr[i][2] * yr[2][j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r3[i][j] = xy[i][0] * zr[0][j] + xy[i][1] * zr[1][j] + xy[i][2] * zr[2][j];
    const double m4[4][4] = {{r3[0][0], r3[0][1], r3[0][2], 0}, {r3[1][0], r3[1][1], r3[1][2], 0},
                             {r3[2][0], r3[2][1], r3[2][2], 0}, {0, 0, 0, 1}};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 4; ++j) {
            const double e0 = i == 0, e1 = i == 1, e2 = i == 2;
            k.rot[i][j] = e0 * m4[0][j] + e1 * m4[1][j] + e2 * m4[2][j] + 0.0 * m4[3][j];
        }
    return k;
}

bool camera_valid(const xtgpu_camera &c)
{
    return c.type >= XTGPU_CAM_PERSPECTIVE && c.type <= XTGPU_CAM_CUBEMAP && std::isfinite(c.ipd) &&
           std::isfinite(c.flength) && std::isfinite(c.aperture) && std::isfinite(c.orientation[0]) &&
           std::isfinite(c.orientation[1]) && std::isfinite(c.orientation[2]);
}

// The frame a camera can render and the grid level: a cubemap is a vertical
// strip of six square faces, so its height must split into them.
bool view_valid(const DevCamera &c, int width, int height, int aa, int dist, int spp)
{
    (void)width;
    if (dist != XTGPU_SAMPLES_GRID && dist != XTGPU_SAMPLES_RANDOM) return false;
    if (aa < 0 || aa > (dist == XTGPU_SAMPLES_RANDOM ? MAX_AA * MAX_AA : MAX_AA)) return false;
    if (spp <= 0 || (int64_t)sample_positions(aa, dist) * spp > INT32_MAX) return false;
    return c.type != XTGPU_CAM_CUBEMAP || (height >= 6 && height % 6 == 0);
}

const xtgpu_tuning &scene_tuning(const xtgpu_scene *sc) { return sc->tuned ? sc->tune : tuning(); }

// One wave runner per process, shared by xtgpu_render calls.
static std::mutex g_runner_mu;
static WaveRunner *g_runner = nullptr;
static int64_t g_runner_cap = 0;

static xtgpu_status get_runner(int64_t cap, cudaStream_t s, WaveRunner **out)
{
    if (!g_runner || g_runner_cap < cap) {
        if (g_runner) {
            // every call ends synchronised (read_ctl), but a failed one may not have
            cudaDeviceSynchronize();
            g_runner->release();
            delete g_runner;
            g_runner = nullptr;
        }
        g_runner = new WaveRunner();
        xtgpu_status st = g_runner->init(cap, 4, 1, s);
        if (st != XTGPU_OK) {
            g_runner->release();
            delete g_runner;
            g_runner = nullptr;
            return st;
        }
        g_runner_cap = cap;
    }
    *out = g_runner;
    return XTGPU_OK;
}

}  // namespace xtg

using namespace xtg;

extern "C" {

const char *xtgpu_last_error(void) { return g_err.c_str(); }

xtgpu_status xtgpu_get_tuning(xtgpu_tuning *t)
{
    if (!t) {
        set_error("xtgpu_get_tuning: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    *t = tuning();
    return XTGPU_OK;
}

xtgpu_status xtgpu_scene_tuning(const xtgpu_scene *sc, xtgpu_tuning *t)
{
    if (!sc || !t) {
        set_error("xtgpu_scene_tuning: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    *t = scene_tuning(sc);
    // the hierarchy the scene was built with, whatever the process-wide values
    if (sc->built32 || sc->built8 || sc->builtW) {
        t->leaf_size = sc->leaf_size;
        t->bvh_builder = sc->builder;
    }
    if (sc->builtW) {
        t->wide_collapse = sc->wide_collapse;
        t->wide_prim_cost = sc->wide_prim_cost;
    }
    return XTGPU_OK;
}

static bool tuning_valid(const xtgpu_tuning *t)
{
    return t && t->extend_variant >= 0 && t->extend_variant <= 2 && t->steps_per_vote >= 1 &&
           t->steps_per_vote <= 64 && t->primary_node_format >= -1 && t->primary_node_format <= XTGPU_NODES_W8 &&
           t->primary_variant >= -1 && t->primary_variant <= 2 && t->extend_block >= 32 && t->extend_block <= 256 &&
           !(t->extend_block & 31) && t->extend_blocks_per_sm >= 1 && t->extend_blocks_per_sm <= 64 && t->tile >= 0 &&
           t->tile <= 256 && t->wave_paths >= 1024 && t->wave_paths <= (1ll << 26) && t->leaf_size >= 1 &&
           t->leaf_size <= MAX_LEAF && t->node_layout >= 0 && t->node_layout <= 1 && t->refill_threshold >= 1 &&
           t->refill_threshold <= 32 &&
           (t->extend_min_blocks == 0 || t->extend_min_blocks == 8 || t->extend_min_blocks == 10) &&
           (t->stack_entries == 0 || t->stack_entries == 32 || t->stack_entries == 64) && t->bvh_builder >= 0 &&
           t->bvh_builder <= 1 && t->wide_collapse >= 0 && t->wide_collapse <= 1 && t->wide_prim_cost >= 0.f &&
           t->wide_prim_cost <= 100.f;
}

xtgpu_status xtgpu_set_tuning(const xtgpu_tuning *t)
{
    if (!tuning_valid(t)) {
        set_error("xtgpu_set_tuning: value out of range");
        return XTGPU_ERR_INVALID;
    }
    tuning() = *t;
    return XTGPU_OK;
}

xtgpu_status xtgpu_scene_set_tuning(xtgpu_scene *sc, const xtgpu_tuning *t)
{
    if (!sc || !tuning_valid(t)) {
        set_error("xtgpu_scene_set_tuning: NULL scene or value out of range");
        return XTGPU_ERR_INVALID;
    }
    if (t->leaf_size != sc->leaf_size || t->bvh_builder != sc->builder ||
        (sc->builtW && (t->wide_collapse != sc->wide_collapse || t->wide_prim_cost != sc->wide_prim_cost))) {
        set_error("xtgpu_scene_set_tuning: leaf_size, bvh_builder or the 8-wide collapse differs from the built BVH "
                  "(rebuild it instead)");
        return XTGPU_ERR_STATE;
    }
    sc->tune = *t;
    sc->tuned = true;
    return XTGPU_OK;
}
const char *xtgpu_version(void) { return "xtgpu 0.1 (sm_100a)"; }

// Materials, samplers, textures and the environment of a description.
static xtgpu_status check_shading(const xtgpu_scene_desc *d, const std::string &who)
{
    if (d->env_type < XTGPU_ENV_NONE || d->env_type > XTGPU_ENV_CUBEMAP) {
        set_error(who + ": bad environment type");
        return XTGPU_ERR_INVALID;
    }
    // textures: every texel of every texture inside texels; samplers name
    // textures that exist (a cubemap six of them)
    if (d->n_textures < 0 || d->n_texels < 0 || (d->n_textures && (!d->textures || !d->texels))) {
        set_error(who + ": inconsistent texture arrays");
        return XTGPU_ERR_INVALID;
    }
    for (int32_t i = 0; i < d->n_textures; ++i) {
        const xtgpu_texture &t = d->textures[i];
        if (t.width <= 0 || t.height <= 0 || t.offset < 0 || (t.filtering != XTGPU_FILTER_NEAREST &&
                                                              t.filtering != XTGPU_FILTER_BILINEAR) ||
            (int64_t)t.width * t.height > d->n_texels - t.offset) {
            set_error(who + ": texture " + std::to_string(i) + " out of bounds or bad filtering");
            return XTGPU_ERR_INVALID;
        }
    }
    auto tex_ok = [&](int kind, int tex) {
        if (kind == XTGPU_SAMPLER_TEXTURE || kind == XTGPU_SAMPLER_ERP) return tex >= 0 && tex < d->n_textures;
        if (kind == XTGPU_SAMPLER_CUBEMAP) return tex >= 0 && (int64_t)tex + 6 <= d->n_textures;
        return kind == XTGPU_SAMPLER_COLOR || kind == XTGPU_SAMPLER_GRADIENT;
    };
    if (d->mat_samplers)
        for (int64_t i = 0; i < 3 * (int64_t)d->n_materials; ++i)
            if (!tex_ok(d->mat_samplers[i].kind, d->mat_samplers[i].texture)) {
                set_error(who + ": material sampler " + std::to_string(i) +
                          ": bad kind or texture index");
                return XTGPU_ERR_INVALID;
            }
    if ((d->env_type == XTGPU_ENV_ERP && !tex_ok(XTGPU_SAMPLER_ERP, d->env_texture)) ||
        (d->env_type == XTGPU_ENV_CUBEMAP && !tex_ok(XTGPU_SAMPLER_CUBEMAP, d->env_texture))) {
        set_error(who + ": environment texture out of range");
        return XTGPU_ERR_INVALID;
    }

    return XTGPU_OK;
}

// Uploads a description's materials (with their samplers), textures, object
// materials, texture-coordinate inputs and environment into new device
// buffers, then swaps them in: the scene's geometry and BVH are untouched.
// material of every primitive id, so that shading reads one table entry per
// hit instead of going through the primitive's object (Scene::get_material,
// scene.cc:55-61, keyed by the hit record's object)
__global__ void k_prim_material(int64_t n, const int32_t *__restrict__ prim_obj,
                                const int32_t *__restrict__ obj_material, int32_t *__restrict__ prim_mat)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        prim_mat[i] = obj_material[prim_obj[i]];
}

static xtgpu_status upload_shading(xtgpu_scene *sc, const xtgpu_scene_desc *d, int64_t nprim, cudaStream_t s)
{
    std::vector<DevMaterial> mats((size_t)std::max(1, d->n_materials));
    for (int32_t i = 0; i < d->n_materials; ++i) {
        const xtgpu_material &m = d->materials[i];
        mats[i].type = m.type;
        mats[i].diffuse = make_float3(m.diffuse[0], m.diffuse[1], m.diffuse[2]);
        mats[i].specular = make_float3(m.specular[0], m.specular[1], m.specular[2]);
        mats[i].emissive = make_float3(m.emissive[0], m.emissive[1], m.emissive[2]);
        mats[i].reflectance = m.reflectance;
        mats[i].exponent = m.exponent;
        mats[i].ior = m.ior;
        mats[i].textured = 0;
        const float3 col[3] = {mats[i].diffuse, mats[i].specular, mats[i].emissive};
        for (int ch = 0; ch < 3; ++ch) {
            DevSampler &k = mats[i].s[ch];
            k = DevSampler{XTGPU_SAMPLER_COLOR, -1, col[ch], make_float3(0.f, 0.f, 0.f)};
            if (!d->mat_samplers) continue;
            const xtgpu_sampler &x = d->mat_samplers[3 * (size_t)i + ch];
            k.kind = x.kind;
            k.tex = x.texture;
            k.a = make_float3(x.a[0], x.a[1], x.a[2]);
            k.b = make_float3(x.b[0], x.b[1], x.b[2]);
            if (x.kind == XTGPU_SAMPLER_COLOR) {
                // the colour replaces the material's (get_sample of the sampler)
                (ch == 0 ? mats[i].diffuse : ch == 1 ? mats[i].specular : mats[i].emissive) = k.a;
            } else {
                mats[i].textured = 1;
            }
        }
    }
    std::vector<DevTexture> texs((size_t)std::max(1, d->n_textures));
    for (int32_t i = 0; i < d->n_textures; ++i)
    {
        const uint64_t W = (uint64_t)d->textures[i].width, Hh = (uint64_t)d->textures[i].height;
        texs[i] = DevTexture{d->textures[i].width, d->textures[i].height, d->textures[i].filtering, 0,
                             d->textures[i].offset, (uint32_t)((UINT64_MAX % W + 1) % W),
                             (uint32_t)((UINT64_MAX % Hh + 1) % Hh)};
    }
    std::vector<int32_t> om((size_t)std::max(1, d->n_objects));
    for (int32_t i = 0; i < d->n_objects; ++i) om[i] = d->obj_material[i];
    // texture-coordinate inputs: the surfaces' u/v scales, the triangles' texcoords
    std::vector<float2> ouv((size_t)std::max(1, d->n_objects), make_float2(0.f, 0.f));
    if (d->obj_uv_scale)
        for (int32_t i = 0; i < d->n_objects; ++i) ouv[i] = make_float2(d->obj_uv_scale[2 * i], d->obj_uv_scale[2 * i + 1]);
    const bool tuv = d->tri_uvs && d->n_tris;
    HostBuf nm, no, nt, nx, nu, nv;
    auto drop = [&](xtgpu_status st) {
        dfree(nm); dfree(no); dfree(nt); dfree(nx); dfree(nu); dfree(nv);
        return st;
    };
    {
        xtgpu_status st;
        if ((st = dalloc(nu, sizeof(float2) * ouv.size(), s)) != XTGPU_OK) return drop(st);
        if (tuv && (st = dalloc(nv, sizeof(float2) * 3 * (size_t)d->n_tris, s)) != XTGPU_OK) return drop(st);
        cudaError_t e = cudaMemcpy(nu.p, ouv.data(), sizeof(float2) * ouv.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && tuv)
            e = cudaMemcpy(nv.p, d->tri_uvs, sizeof(float2) * 3 * (size_t)d->n_tris, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return drop(cuda_fail(e, "cudaMemcpy", __FILE__, __LINE__));
    }
    xtgpu_status st;
    if ((st = dalloc(nm, sizeof(DevMaterial) * mats.size(), s)) != XTGPU_OK) return drop(st);
    if ((st = dalloc(no, sizeof(int32_t) * om.size(), s)) != XTGPU_OK) return drop(st);
    if ((st = dalloc(nt, sizeof(DevTexture) * texs.size(), s)) != XTGPU_OK) return drop(st);
    if ((st = dalloc(nx, sizeof(float4) * (size_t)std::max<int64_t>(1, d->n_texels), s)) != XTGPU_OK) return drop(st);
    cudaError_t e = cudaMemcpy(nm.p, mats.data(), sizeof(DevMaterial) * mats.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(no.p, om.data(), sizeof(int32_t) * om.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(nt.p, texs.data(), sizeof(DevTexture) * texs.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && d->n_texels)
        e = cudaMemcpy(nx.p, d->texels, sizeof(float4) * (size_t)d->n_texels, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return drop(cuda_fail(e, "cudaMemcpy", __FILE__, __LINE__));
    HostBuf npm;
    if ((st = dalloc(npm, sizeof(int32_t) * (size_t)std::max<int64_t>(1, nprim), s)) != XTGPU_OK) return drop(st);
    if (nprim > 0) {
        k_prim_material<<<(int)std::min<int64_t>((nprim + 255) / 256, 4096), 256, 0, s>>>(
            nprim, (const int32_t *)sc->prim_obj.p, (const int32_t *)no.p, (int32_t *)npm.p);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            dfree(npm);
            return drop(cuda_fail(e, "k_prim_material", __FILE__, __LINE__));
        }
    }
    std::swap(sc->materials, nm);
    std::swap(sc->obj_material, no);
    std::swap(sc->prim_mat, npm);
    std::swap(sc->textures, nt);
    std::swap(sc->texels, nx);
    std::swap(sc->obj_uvs, nu);
    std::swap(sc->tri_uv, nv);
    dfree(nm); dfree(no); dfree(npm); dfree(nt); dfree(nx); dfree(nu); dfree(nv);   // the previous buffers
    DevScene &S = sc->dev;
    S.prim_mat = (const int32_t *)sc->prim_mat.p;
    S.has_lobe = 0;
    for (const DevMaterial &m : mats)
        if (m.type == XTGPU_PHONG || m.type == XTGPU_BLINNPHONG) S.has_lobe = 1;
    S.obj_uvs = (const float2 *)sc->obj_uvs.p;
    S.tri_uv = (const float2 *)sc->tri_uv.p;
    S.materials = (const DevMaterial *)sc->materials.p;
    S.obj_material = (const int32_t *)sc->obj_material.p;
    S.textures = (const DevTexture *)sc->textures.p;
    S.texels = (const float4 *)sc->texels.p;
    S.env_type = d->env_type;
    S.env_tex = d->env_texture;
    S.env_a = make_float3(d->env_a[0], d->env_a[1], d->env_a[2]);
    S.env_b = make_float3(d->env_b[0], d->env_b[1], d->env_b[2]);
    return XTGPU_OK;
}

xtgpu_status xtgpu_scene_create(const xtgpu_scene_desc *d, void *stream, xtgpu_scene **out)
{
    if (!d || !out) {
        set_error("xtgpu_scene_create: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    *out = nullptr;
    if (d->n_tris < 0 || d->n_spheres < 0 || d->n_planes < 0 || d->n_objects < 0 || d->n_materials < 0 ||
        (d->n_tris && !d->tris) || (d->n_spheres && !d->spheres) || (d->n_planes && !d->planes) ||
        (d->n_objects && (!d->obj_kind || !d->obj_first || !d->obj_count || !d->obj_material)) ||
        (d->n_materials && !d->materials)) {
        set_error("xtgpu_scene_create: inconsistent sizes or NULL arrays");
        return XTGPU_ERR_INVALID;
    }
    if (!camera_valid(d->camera)) {
        set_error("xtgpu_scene_create: bad camera type or non-finite camera parameters");
        return XTGPU_ERR_INVALID;
    }
    const int64_t nprim = (int64_t)d->n_tris + d->n_spheres + d->n_planes;
    // every primitive must belong to exactly one object with a valid material
    std::vector<int32_t> prim_obj((size_t)std::max<int64_t>(1, nprim), -1);
    for (int32_t o = 0; o < d->n_objects; ++o) {
        int32_t k = d->obj_kind[o], f = d->obj_first[o], c = d->obj_count[o], m = d->obj_material[o];
        if (m < 0 || m >= d->n_materials) {
            set_error("xtgpu_scene_create: object material out of range");
            return XTGPU_ERR_INVALID;
        }
        int64_t base, lim;
        if (k == XTGPU_MESH) { base = 0; lim = d->n_tris; }
        else if (k == XTGPU_SPHERE) { base = d->n_tris; lim = d->n_spheres; c = 1; }
        else if (k == XTGPU_PLANE) { base = (int64_t)d->n_tris + d->n_spheres; lim = d->n_planes; c = 1; }
        else {
            set_error("xtgpu_scene_create: bad object kind");
            return XTGPU_ERR_INVALID;
        }
        if (f < 0 || c < 0 || (int64_t)f + c > lim) {
            set_error("xtgpu_scene_create: object range out of bounds");
            return XTGPU_ERR_INVALID;
        }
        for (int64_t i = 0; i < c; ++i) prim_obj[(size_t)(base + f + i)] = o;
    }
    for (int64_t i = 0; i < nprim; ++i)
        if (prim_obj[(size_t)i] < 0) {
            set_error("xtgpu_scene_create: a primitive belongs to no object");
            return XTGPU_ERR_INVALID;
        }
    XTG_TRY(check_shading(d, "xtgpu_scene_create"));

    cudaStream_t s = (cudaStream_t)stream;
    xtgpu_scene *sc = new xtgpu_scene();
    cudaGetDevice(&sc->device);
    auto fail = [&](xtgpu_status st) {
        xtgpu_scene_destroy(sc);
        return st;
    };
    // triangles as 3 x float4 per triangle
    std::vector<float4> tv((size_t)std::max(1, 3 * d->n_tris));
    for (int32_t i = 0; i < d->n_tris; ++i)
        for (int k = 0; k < 3; ++k)
            tv[3 * i + k] = make_float4(d->tris[9 * (size_t)i + 3 * k], d->tris[9 * (size_t)i + 3 * k + 1],
                                        d->tris[9 * (size_t)i + 3 * k + 2], 0.f);
    xtgpu_status st;
    if ((st = dalloc(sc->tri_v, sizeof(float4) * tv.size(), s)) != XTGPU_OK) return fail(st);
    if (cudaMemcpy(sc->tri_v.p, tv.data(), sizeof(float4) * tv.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(cuda_fail(cudaGetLastError(), "cudaMemcpy", __FILE__, __LINE__));
    if (d->tri_normals && d->n_tris) {
        for (int32_t i = 0; i < d->n_tris; ++i)
            for (int k = 0; k < 3; ++k)
                tv[3 * i + k] = make_float4(d->tri_normals[9 * (size_t)i + 3 * k], d->tri_normals[9 * (size_t)i + 3 * k + 1],
                                            d->tri_normals[9 * (size_t)i + 3 * k + 2], 0.f);
        if ((st = dalloc(sc->tri_n, sizeof(float4) * tv.size(), s)) != XTGPU_OK) return fail(st);
        cudaMemcpy(sc->tri_n.p, tv.data(), sizeof(float4) * tv.size(), cudaMemcpyHostToDevice);
    }
    std::vector<float4> sp((size_t)std::max(1, d->n_spheres)), pl((size_t)std::max(1, d->n_planes));
    for (int32_t i = 0; i < d->n_spheres; ++i)
        sp[i] = make_float4(d->spheres[4 * i], d->spheres[4 * i + 1], d->spheres[4 * i + 2], d->spheres[4 * i + 3]);
    for (int32_t i = 0; i < d->n_planes; ++i)
        pl[i] = make_float4(d->planes[4 * i], d->planes[4 * i + 1], d->planes[4 * i + 2], d->planes[4 * i + 3]);
    if ((st = dalloc(sc->spheres, sizeof(float4) * sp.size(), s)) != XTGPU_OK) return fail(st);
    if ((st = dalloc(sc->planes, sizeof(float4) * pl.size(), s)) != XTGPU_OK) return fail(st);
    if ((st = dalloc(sc->prim_obj, sizeof(int32_t) * prim_obj.size(), s)) != XTGPU_OK) return fail(st);
    cudaMemcpy(sc->spheres.p, sp.data(), sizeof(float4) * sp.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(sc->planes.p, pl.data(), sizeof(float4) * pl.size(), cudaMemcpyHostToDevice);
    if (cudaMemcpy(sc->prim_obj.p, prim_obj.data(), sizeof(int32_t) * prim_obj.size(), cudaMemcpyHostToDevice) !=
        cudaSuccess)
        return fail(cuda_fail(cudaGetLastError(), "cudaMemcpy", __FILE__, __LINE__));
    if ((st = upload_shading(sc, d, nprim, s)) != XTGPU_OK) return fail(st);

    DevScene &S = sc->dev;
    S.tri_v = (const float4 *)sc->tri_v.p;
    S.tri_n = (const float4 *)sc->tri_n.p;
    S.spheres = (const float4 *)sc->spheres.p;
    S.planes = (const float4 *)sc->planes.p;
    S.prim_obj = (const int32_t *)sc->prim_obj.p;
    S.n_tris = d->n_tris;
    S.n_spheres = d->n_spheres;
    S.n_planes = d->n_planes;
    S.root = EMPTY_REF;
    S.cam = make_camera(d->camera);
    sc->n_objects = d->n_objects;
    *out = sc;
    return XTGPU_OK;
}

xtgpu_status xtgpu_scene_update(xtgpu_scene *sc, const xtgpu_scene_desc *d, int32_t what, void *stream)
{
    if (!sc || !d || !what || (what & ~(XTGPU_UPDATE_SHADING | XTGPU_UPDATE_CAMERA))) {
        set_error("xtgpu_scene_update: NULL argument or bad flags");
        return XTGPU_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (what & XTGPU_UPDATE_SHADING) {
        if (d->n_objects != sc->n_objects || d->n_materials < 0 || (d->n_materials && !d->materials) ||
            (d->n_objects && !d->obj_material) || (d->tri_uvs && d->n_tris != sc->dev.n_tris)) {
            set_error("xtgpu_scene_update: the object or triangle count differs from the scene's, or NULL arrays");
            return XTGPU_ERR_INVALID;
        }
        for (int32_t o = 0; o < d->n_objects; ++o)
            if (d->obj_material[o] < 0 || d->obj_material[o] >= d->n_materials) {
                set_error("xtgpu_scene_update: object material out of range");
                return XTGPU_ERR_INVALID;
            }
        XTG_TRY(check_shading(d, "xtgpu_scene_update"));
    }
    if ((what & XTGPU_UPDATE_CAMERA) && !camera_valid(d->camera)) {
        set_error("xtgpu_scene_update: bad camera type or non-finite camera parameters");
        return XTGPU_ERR_INVALID;
    }
    // renders read the buffers being replaced: let those on this stream finish
    XTG_CUDA(cudaStreamSynchronize(s));
    if (what & XTGPU_UPDATE_SHADING)
        XTG_TRY(upload_shading(sc, d, (int64_t)sc->dev.n_tris + sc->dev.n_spheres + sc->dev.n_planes, s));
    if (what & XTGPU_UPDATE_CAMERA) sc->dev.cam = make_camera(d->camera);
    return XTGPU_OK;
}

xtgpu_status xtgpu_bvh_build(xtgpu_scene *sc, const xtgpu_bvh_opts *opts, void *stream)
{
    if (!sc) {
        set_error("xtgpu_bvh_build: NULL scene");
        return XTGPU_ERR_INVALID;
    }
    int fmt = opts ? opts->node_format : XTGPU_NODES_FP32;
    int leaf = opts && opts->leaf_size > 0 ? opts->leaf_size : scene_tuning(sc).leaf_size;
    if (!format_valid(fmt)) {
        set_error("xtgpu_bvh_build: bad node format");
        return XTGPU_ERR_INVALID;
    }
    if (fmt == XTGPU_NODES_W8 && !(opts && opts->leaf_size > 0)) leaf = std::min(leaf, 3);
    if (leaf < 1 || leaf > MAX_LEAF) {
        set_error("xtgpu_bvh_build: leaf_size out of range");
        return XTGPU_ERR_INVALID;
    }
    return build_bvh(sc, fmt, leaf, scene_tuning(sc).node_layout, (cudaStream_t)stream, scene_tuning(sc).bvh_builder);
}

xtgpu_status xtgpu_scene_destroy(xtgpu_scene *sc)
{
    if (!sc) return XTGPU_OK;
    for (HostBuf *b : {&sc->tri_v, &sc->tri_n, &sc->spheres, &sc->planes, &sc->prim_obj, &sc->obj_material,
                       &sc->prim_mat, &sc->obj_uvs, &sc->tri_uv, &sc->materials, &sc->textures, &sc->texels, &sc->leaf_prims, &sc->nodes32, &sc->nodes8, &sc->nodesW, &sc->leafW,
                       &sc->morton, &sc->order, &sc->left, &sc->right})
        dfree(*b);
    delete sc;
    return XTGPU_OK;
}

xtgpu_status xtgpu_scene_device_bytes(const xtgpu_scene *sc, uint64_t *bytes)
{
    if (!sc || !bytes) {
        set_error("xtgpu_scene_device_bytes: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    uint64_t b = 0;
    for (const HostBuf *h : {&sc->tri_v, &sc->tri_n, &sc->spheres, &sc->planes, &sc->prim_obj, &sc->obj_material,
                             &sc->prim_mat, &sc->obj_uvs, &sc->tri_uv, &sc->materials, &sc->textures, &sc->texels, &sc->leaf_prims, &sc->nodes32, &sc->nodes8, &sc->nodesW, &sc->leafW,
                             &sc->morton, &sc->order, &sc->left, &sc->right})
        b += h->bytes;
    *bytes = b;
    return XTGPU_OK;
}

xtgpu_status xtgpu_bvh_export(const xtgpu_scene *sc, xtgpu_bvh_info *info, uint32_t *morton, uint32_t *order,
                              int32_t *left, int32_t *right, void *stream)
{
    if (!sc) {
        set_error("xtgpu_bvh_export: NULL scene");
        return XTGPU_ERR_INVALID;
    }
    if (!sc->built32) {
        set_error("xtgpu_bvh_export: BVH not built");
        return XTGPU_ERR_STATE;
    }
    cudaStream_t s = (cudaStream_t)stream;
    XTG_CUDA(cudaStreamSynchronize(s));
    int64_t n = sc->n_prims;
    if (info) {
        info->n_prims = n;
        info->depth = sc->depth;
        info->leaf_size = sc->leaf_size;
        info->node_bytes_fp32 = sc->nodes32.bytes;
        info->node_bytes_q8 = sc->nodes8.bytes;
        info->node_bytes_w8 = sc->builtW ? (uint64_t)sc->n_wide * 80u : 0u;
        info->depth_w8 = sc->depthW;
    }
    if (n > 0) {
        if (morton) XTG_CUDA(cudaMemcpy(morton, sc->morton.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost));
        if (order) XTG_CUDA(cudaMemcpy(order, sc->order.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost));
        if (n > 1 && left) XTG_CUDA(cudaMemcpy(left, sc->left.p, sizeof(int32_t) * (n - 1), cudaMemcpyDeviceToHost));
        if (n > 1 && right) XTG_CUDA(cudaMemcpy(right, sc->right.p, sizeof(int32_t) * (n - 1), cudaMemcpyDeviceToHost));
    }
    return XTGPU_OK;
}

static xtgpu_status check_format(const xtgpu_scene *sc, int32_t fmt)
{
    if (format_built(sc, fmt)) return XTGPU_OK;
    set_error("node format not built for this scene");
    return XTGPU_ERR_STATE;
}

static xtgpu_status trace_impl(xtgpu_scene *sc, int64_t n, const void *org, const void *dir, xtgpu_hit *hits,
                               int32_t fmt, uint64_t *counts, void *stream);

xtgpu_status xtgpu_trace(xtgpu_scene *sc, int64_t n, const void *org, const void *dir, xtgpu_hit *hits, int32_t fmt,
                         void *stream)
{
    return trace_impl(sc, n, org, dir, hits, fmt, nullptr, stream);
}

xtgpu_status xtgpu_trace_counts(xtgpu_scene *sc, int64_t n, const void *org, const void *dir, xtgpu_hit *hits,
                                int32_t fmt, uint64_t counts[2], void *stream)
{
    if (!counts) {
        set_error("xtgpu_trace_counts: NULL counts");
        return XTGPU_ERR_INVALID;
    }
    return trace_impl(sc, n, org, dir, hits, fmt, counts, stream);
}

static xtgpu_status trace_impl(xtgpu_scene *sc, int64_t n, const void *org, const void *dir, xtgpu_hit *hits,
                               int32_t fmt, uint64_t *counts, void *stream)
{
    if (!sc || n < 0 || (n && (!org || !dir || !hits))) {
        set_error("xtgpu_trace: bad argument");
        return XTGPU_ERR_INVALID;
    }
    XTG_TRY(check_format(sc, fmt));
    if (n == 0) return XTGPU_OK;
    cudaStream_t s = (cudaStream_t)stream;
    int32_t *ctl = nullptr;
    XTG_CUDA(cudaMallocAsync((void **)&ctl, 64 + 16, s));
    unsigned long long *stats = counts ? (unsigned long long *)((char *)ctl + 64) : nullptr;
    if (stats) XTG_CUDA(cudaMemsetAsync(stats, 0, 16, s));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int32_t overflow = 0;
    for (int64_t base = 0; base < n; base += (1ll << 30)) {
        int32_t cnt = (int32_t)std::min<int64_t>(n - base, 1ll << 30);
        WaveQueues q{};
        q.org[0] = (float4 *)((const float4 *)org + base);
        q.dir[0] = (float4 *)((const float4 *)dir + base);
        q.hit = hits + base;
        q.ctl = ctl;
        q.rays = (unsigned long long *)((char *)ctl + 32);
        q.stats = stats;
        int32_t init[4] = {cnt, 0, 0, 0};
        XTG_CUDA(cudaMemcpyAsync(ctl, init, sizeof(init), cudaMemcpyHostToDevice, s));
        const xtgpu_tuning &T = scene_tuning(sc);
        launch_extend(T, fmt, sc->dev, q, 0, sms, stack_for_scene(sc, fmt, T.stack_entries), s);
        XTG_CUDA(cudaGetLastError());
        int32_t back[4];
        XTG_CUDA(cudaMemcpyAsync(back, ctl, sizeof(back), cudaMemcpyDeviceToHost, s));
        XTG_CUDA(cudaStreamSynchronize(s));
        overflow |= back[3];
    }
    if (stats) {
        unsigned long long c[2];
        XTG_CUDA(cudaMemcpy(c, stats, 16, cudaMemcpyDeviceToHost));
        counts[0] = c[0];
        counts[1] = c[1];
    }
    cudaFreeAsync(ctl, s);
    if (overflow) {
        set_error("xtgpu_trace: traversal stack overflow");
        return XTGPU_ERR_LIMIT;
    }
    return XTGPU_OK;
}

xtgpu_status xtgpu_trace_host(xtgpu_scene *sc, int64_t n, const float *org, const float *dir, xtgpu_hit *hits,
                              int32_t fmt, void *stream)
{
    if (!sc || n < 0 || (n && (!org || !dir || !hits))) {
        set_error("xtgpu_trace_host: bad argument");
        return XTGPU_ERR_INVALID;
    }
    if (n == 0) return XTGPU_OK;
    cudaStream_t s = (cudaStream_t)stream;
    float4 *dorg = nullptr, *ddir = nullptr;
    xtgpu_hit *dhit = nullptr;
    XTG_CUDA(cudaMallocAsync((void **)&dorg, sizeof(float4) * n, s));
    XTG_CUDA(cudaMallocAsync((void **)&ddir, sizeof(float4) * n, s));
    XTG_CUDA(cudaMallocAsync((void **)&dhit, sizeof(xtgpu_hit) * n, s));
    XTG_CUDA(cudaMemcpyAsync(dorg, org, sizeof(float4) * n, cudaMemcpyHostToDevice, s));
    XTG_CUDA(cudaMemcpyAsync(ddir, dir, sizeof(float4) * n, cudaMemcpyHostToDevice, s));
    xtgpu_status st = xtgpu_trace(sc, n, dorg, ddir, dhit, fmt, stream);
    if (st == XTGPU_OK) {
        cudaError_t e = cudaMemcpyAsync(hits, dhit, sizeof(xtgpu_hit) * n, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "cudaMemcpyAsync", __FILE__, __LINE__);
    }
    cudaFreeAsync(dorg, s);
    cudaFreeAsync(ddir, s);
    cudaFreeAsync(dhit, s);
    return st;
}

xtgpu_status xtgpu_render(xtgpu_scene *sc, const xtgpu_render_params *p, float *rgba, uint64_t *rays, void *stream)
{
    if (!sc) {
        set_error("xtgpu_render: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    return render_impl(sc, p, rgba, rays, (cudaStream_t)stream, scene_tuning(sc));
}

}  // extern "C"

xtgpu_status xtg::render_impl(xtgpu_scene *sc, const xtgpu_render_params *p, float *rgba, uint64_t *rays,
                              cudaStream_t stream, const xtgpu_tuning &T, float *raygraph)
{
    if (!sc || !p || !rgba) {
        set_error("xtgpu_render: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    if (p->integrator < XTGPU_STENCIL || p->integrator > XTGPU_INTEGRATOR_LAST || p->width <= 0 || p->height <= 0 ||
        p->spp <= 0 || p->rdepth < 0 || (p->integrator == XTGPU_AO && !(p->ao_max_distance > 0.f))) {
        set_error("xtgpu_render: bad parameters");
        return XTGPU_ERR_INVALID;
    }
    if (!view_valid(sc->dev.cam, p->width, p->height, p->aa, p->sample_distribution, p->spp)) {
        set_error("xtgpu_render: sample_distribution not grid or random, aa outside 0..16 (grid) or 0..256 "
                  "(random), samples per pixel above 2^31, or a cubemap height that is not six square faces");
        return XTGPU_ERR_INVALID;
    }
    int x0 = p->x0, y0 = p->y0, x1 = p->x1, y1 = p->y1;
    if (x1 == 0 && y1 == 0) {
        x0 = y0 = 0;
        x1 = p->width;
        y1 = p->height;
    }
    if (x0 < 0 || y0 < 0 || x1 > p->width || y1 > p->height || x0 >= x1 || y0 >= y1) {
        set_error("xtgpu_render: bad rectangle");
        return XTGPU_ERR_INVALID;
    }
    XTG_TRY(check_format(sc, p->node_format));
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t npix = (int64_t)(x1 - x0) * (y1 - y0);
    const int64_t paths = npix * sample_positions(p->aa, p->sample_distribution) * p->spp;
    const int64_t cap = std::min<int64_t>(paths, T.wave_paths);
    std::lock_guard<std::mutex> lock(g_runner_mu);
    WaveRunner *R = nullptr;
    XTG_TRY(get_runner(std::max<int64_t>(cap, 1 << 16), s, &R));
    XTG_TRY(R->set_scenes(&sc->dev, 1, s));
    R->T = T;
    R->stack = stack_for_scene(sc, p->node_format, T.stack_entries);
    R->fmt0 = -1;
    if (T.primary_node_format >= 0 && T.primary_node_format != p->node_format &&
        format_built(sc, T.primary_node_format)) {
        R->fmt0 = T.primary_node_format;
        R->stack0 = stack_for_scene(sc, R->fmt0, T.stack_entries);
    }
    XTG_CUDA(cudaMemsetAsync(R->q.ctl, 0, 64, s));
    XTG_CUDA(cudaMemsetAsync(rgba, 0, sizeof(float4) * npix, s));
    DevJob J{};
    J.integrator = p->integrator;
    J.width = p->width;
    J.height = p->height;
    set_samples(J, p->spp, p->aa, p->sample_distribution);
    J.rdepth = p->rdepth;
    J.ao_maxd = p->ao_max_distance;
    J.seed = p->seed;
    J.x0 = x0;
    J.y0 = y0;
    J.rw = x1 - x0;
    J.rh = y1 - y0;
    J.scene = 0;
    J.bounces = bounces_of(p->integrator, p->rdepth);
    J.tile = T.tile;
    J.frame = (float4 *)rgba;
    J.raygraph = p->integrator == XTGPU_DEPTH ? raygraph : nullptr;
    std::vector<DevJob> jobs(1, J);
    // waves of the tuned size (the shared runner may be larger from an earlier call)
    const int64_t wave = std::max<int64_t>(1, std::min<int64_t>(R->cap, cap));
    for (int64_t first = 0; first < paths; first += wave) {
        jobs[0].first = first;
        jobs[0].count = std::min<int64_t>(wave, paths - first);
        XTG_TRY(R->run_wave(jobs, J.bounces, p->node_format, false, s));
    }
    int32_t overflow = 0;
    unsigned long long nr = 0;
    XTG_TRY(R->read_ctl(&overflow, &nr, s));
    if (rays) *rays = nr;
    if (overflow) {
        set_error("xtgpu_render: traversal stack overflow");
        return XTGPU_ERR_LIMIT;
    }
    return XTGPU_OK;
}

extern "C" {

xtgpu_status xtgpu_render_raygraph(xtgpu_scene *sc, const xtgpu_render_params *p, float *rgba, float *raygraph,
                                   uint64_t *rays, void *stream)
{
    if (!sc || !p || !raygraph) {
        set_error("xtgpu_render_raygraph: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    if (p->integrator != XTGPU_DEPTH) {
        set_error("xtgpu_render_raygraph: the raygraph is recorded by the depth integrator only");
        return XTGPU_ERR_INVALID;
    }
    return render_impl(sc, p, rgba, rays, (cudaStream_t)stream, scene_tuning(sc), raygraph);
}

xtgpu_status xtgpu_render_raygraph_host(xtgpu_scene *sc, const xtgpu_render_params *p, float *rgba_host,
                                        float *raygraph_host, uint64_t *rays, void *stream)
{
    if (!sc || !p || !rgba_host || !raygraph_host) {
        set_error("xtgpu_render_raygraph_host: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    const int64_t w = (p->x1 == 0 && p->y1 == 0) ? p->width : p->x1 - p->x0;
    const int64_t h = (p->x1 == 0 && p->y1 == 0) ? p->height : p->y1 - p->y0;
    if (w <= 0 || h <= 0 || !view_valid(sc->dev.cam, p->width, p->height, p->aa, p->sample_distribution, p->spp)) {
        set_error("xtgpu_render_raygraph_host: bad rectangle or samples");
        return XTGPU_ERR_INVALID;
    }
    const int64_t paths = w * h * sample_positions(p->aa, p->sample_distribution) * p->spp;
    cudaStream_t s = (cudaStream_t)stream;
    float *d = nullptr, *r = nullptr;
    XTG_CUDA(cudaMallocAsync((void **)&d, sizeof(float4) * w * h, s));
    cudaError_t e = cudaMallocAsync((void **)&r, sizeof(float) * 10 * paths, s);
    if (e != cudaSuccess) {
        cudaFreeAsync(d, s);
        return cuda_fail(e, "cudaMallocAsync", __FILE__, __LINE__);
    }
    xtgpu_status st = xtgpu_render_raygraph(sc, p, d, r, rays, stream);
    if (st == XTGPU_OK) {
        e = cudaMemcpyAsync(rgba_host, d, sizeof(float4) * w * h, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(raygraph_host, r, sizeof(float) * 10 * paths, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "cudaMemcpyAsync", __FILE__, __LINE__);
    }
    cudaFreeAsync(d, s);
    cudaFreeAsync(r, s);
    return st;
}

xtgpu_status xtgpu_render_host(xtgpu_scene *sc, const xtgpu_render_params *p, float *rgba_host, uint64_t *rays,
                               void *stream)
{
    if (!sc || !p || !rgba_host) {
        set_error("xtgpu_render_host: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    int64_t w = (p->x1 == 0 && p->y1 == 0) ? p->width : p->x1 - p->x0;
    int64_t h = (p->x1 == 0 && p->y1 == 0) ? p->height : p->y1 - p->y0;
    if (w <= 0 || h <= 0) {
        set_error("xtgpu_render_host: bad rectangle");
        return XTGPU_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    float *d = nullptr;
    XTG_CUDA(cudaMallocAsync((void **)&d, sizeof(float4) * w * h, s));
    xtgpu_status st = xtgpu_render(sc, p, d, rays, stream);
    if (st == XTGPU_OK) {
        cudaError_t e = cudaMemcpyAsync(rgba_host, d, sizeof(float4) * w * h, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "cudaMemcpyAsync", __FILE__, __LINE__);
    }
    cudaFreeAsync(d, s);
    return st;
}

}  // extern "C"
