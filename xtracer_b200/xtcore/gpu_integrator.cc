// GPU integrator for XTracer's xtcore and the Scene flattener behind it.
#include "gpu_integrator.h"

#include <algorithm>
#include <cstdio>
#include <map>

#include <xtcore/log.h>
#include <xtcore/tile.h>
#include <xtcore/util/raygraph.h>
#include <xtcore/mesh.h>
#include <xtcore/octree.h>
#include <xtcore/material.h>
#include <xtcore/sampler_col.h>
#include <xtcore/sampler_gradient.h>
#include <xtcore/sampler_tex.h>
#include <xtcore/sampler_erp.h>
#include <xtcore/sampler_cubemap.h>
#include <xtcore/camera/perspective.h>
#include <xtcore/camera/erp.h>
#include <xtcore/camera/ods.h>
#include <xtcore/camera/cubemap.h>
#include <xtcore/math/sphere.h>
#include <xtcore/math/plane.h>
#include <xtcore/math/triangle.h>
#include <xtcore/matdefs.h>

namespace {

// The triangles of a Mesh live in its private Octree (src/xtcore/mesh.h:38,
// octree.h:61-63), in OBJ face order: m_items is filled by Octree::add in the
// loop of Mesh::build_octree (mesh.cc:70-113).  Inside the XTracer tree a
// maintainer adds a public accessor to Mesh; built against an unmodified tree,
// the members are reached through explicit template instantiation, for which
// C++ does not apply access checks ([temp.explicit]).
typedef xtcore::Octree<xtcore::surface::Triangle> TriOctree;
typedef std::vector<xtcore::OctreeItem<xtcore::surface::Triangle> > TriItems;

template <typename Tag, typename Tag::type Member>
struct Expose {
    friend typename Tag::type member_of(Tag) { return Member; }
};
struct MeshOctreeTag {
    typedef TriOctree xtcore::surface::Mesh::*type;
    friend type member_of(MeshOctreeTag);
};
struct OctreeItemsTag {
    typedef TriItems TriOctree::*type;
    friend type member_of(OctreeItemsTag);
};
template struct Expose<MeshOctreeTag, &xtcore::surface::Mesh::m_octree>;
template struct Expose<OctreeItemsTag, &TriOctree::m_items>;

// The texture samplers keep their images private (sampler_tex.h:34-35,
// sampler_erp.h:20, sampler_cubemap.h:30); reached the same way.
struct TexMapTag {
    typedef nimg::Pixmap xtcore::sampler::Texture2D::*type;
    friend type member_of(TexMapTag);
};
struct TexFilterTag {
    typedef xtcore::sampler::FILTERING xtcore::sampler::Texture2D::*type;
    friend type member_of(TexFilterTag);
};
struct ErpTexTag {
    typedef xtcore::sampler::Texture2D xtcore::sampler::ERP::*type;
    friend type member_of(ErpTexTag);
};
struct CubeTexTag {
    typedef xtcore::sampler::Texture2D (xtcore::sampler::Cubemap::*type)[6];
    friend type member_of(CubeTexTag);
};
template struct Expose<TexMapTag, &xtcore::sampler::Texture2D::m_map>;
template struct Expose<TexFilterTag, &xtcore::sampler::Texture2D::m_filtering>;
template struct Expose<ErpTexTag, &xtcore::sampler::ERP::m_texture>;
template struct Expose<CubeTexTag, &xtcore::sampler::Cubemap::m_textures>;

const TriItems &mesh_triangles(const xtcore::surface::Mesh *m)
{
    const TriOctree &oct = m->*member_of(MeshOctreeTag());
    return oct.*member_of(OctreeItemsTag());
}

// texcoords of a triangle's corners; true if they differ from the Triangle
// constructor's (0,0) (1,0) (0,0) (math/triangle.cc:8-13)
bool put_uvs(std::vector<float> &v, const xtcore::surface::Triangle &t)
{
    static const float dflt[6] = {0.f, 0.f, 1.f, 0.f, 0.f, 0.f};
    bool differs = false;
    for (int k = 0; k < 3; ++k) {
        const float u = (float)t.tc[k].x, w = (float)t.tc[k].y;
        v.push_back(u);
        v.push_back(w);
        differs |= u != dflt[2 * k] || w != dflt[2 * k + 1];
    }
    return differs;
}

void put3(std::vector<float> &v, const nmath::Vector3f &p)
{
    v.push_back((float)p.x);
    v.push_back((float)p.y);
    v.push_back((float)p.z);
}

// Appends the images of n textures (a cubemap's six faces in CUBEMAP_FACE
// order) as consecutive xtgpu_textures; the same sampler object is stored once.
bool add_textures(xtcore::integrator::gpu::FlatScene &F, const void *owner,
                  const xtcore::sampler::Texture2D *const *tex, int n, int32_t &first, std::string &err)
{
    auto it = F.tex_index.find(owner);
    if (it != F.tex_index.end()) {
        first = it->second;
        return true;
    }
    first = (int32_t)F.textures.size();
    for (int k = 0; k < n; ++k) {
        const nimg::Pixmap &pm = tex[k]->*member_of(TexMapTag());
        if (pm.width() == 0 || pm.height() == 0) {
            err = "a texture failed to load (empty image)";
            return false;
        }
        xtgpu_texture t = xtgpu_texture();
        t.width = (int32_t)pm.width();
        t.height = (int32_t)pm.height();
        t.filtering = tex[k]->*member_of(TexFilterTag()) == xtcore::sampler::FILTERING_BILINEAR
                          ? XTGPU_FILTER_BILINEAR : XTGPU_FILTER_NEAREST;
        t.offset = (int64_t)(F.texels.size() / 4);
        for (size_t y = 0; y < pm.height(); ++y)
            for (size_t x = 0; x < pm.width(); ++x) {
                const nimg::ColorRGBAf &c = pm.pixel_ro(x, y);
                F.texels.push_back(c.r());
                F.texels.push_back(c.g());
                F.texels.push_back(c.b());
                F.texels.push_back(c.a());
            }
        F.textures.push_back(t);
    }
    F.tex_index[owner] = first;
    return true;
}

// A sampler (sampler_*.h) as the C ABI's xtgpu_sampler.
bool sampler_of(xtcore::integrator::gpu::FlatScene &F, xtcore::sampler::ISampler *s, xtgpu_sampler &out,
                std::string &err)
{
    using namespace xtcore::sampler;
    out = xtgpu_sampler();
    out.kind = XTGPU_SAMPLER_COLOR;
    out.texture = -1;
    if (!s) {
        // a texture that failed to load leaves a null sampler (parseutil.cc:
        // 492-496), which the CPU integrators would dereference
        err = "a material sampler failed to load";
        return false;
    }
    if (SolidColor *c = dynamic_cast<SolidColor *>(s)) {
        nimg::ColorRGBf v = c->sample(nmath::Vector3f(0, 0, 0));
        out.a[0] = v.r(); out.a[1] = v.g(); out.a[2] = v.b();
    } else if (Gradient *g = dynamic_cast<Gradient *>(s)) {
        out.kind = XTGPU_SAMPLER_GRADIENT;
        out.a[0] = g->a.r(); out.a[1] = g->a.g(); out.a[2] = g->a.b();
        out.b[0] = g->b.r(); out.b[1] = g->b.g(); out.b[2] = g->b.b();
    } else if (Texture2D *t = dynamic_cast<Texture2D *>(s)) {
        out.kind = XTGPU_SAMPLER_TEXTURE;
        const Texture2D *p = t;
        return add_textures(F, s, &p, 1, out.texture, err);
    } else if (ERP *e = dynamic_cast<ERP *>(s)) {
        out.kind = XTGPU_SAMPLER_ERP;
        const Texture2D *p = &(e->*member_of(ErpTexTag()));
        return add_textures(F, s, &p, 1, out.texture, err);
    } else if (Cubemap *cb = dynamic_cast<Cubemap *>(s)) {
        out.kind = XTGPU_SAMPLER_CUBEMAP;
        Texture2D (&faces)[6] = cb->*member_of(CubeTexTag());
        const Texture2D *p[6] = {&faces[0], &faces[1], &faces[2], &faces[3], &faces[4], &faces[5]};
        return add_textures(F, s, p, 6, out.texture, err);
    } else {
        err = "unknown sampler class";
        return false;
    }
    return true;
}

// The material's diffuse, specular and emissive samplers (absent = black, as
// IMaterial::get_sample returns, material.cc:65-70), appended to F.samplers;
// colour samplers also fill the material's colours.
bool samplers_of(xtcore::integrator::gpu::FlatScene &F, const xtcore::asset::IMaterial *m, xtgpu_material &gm,
                 std::string &err)
{
    static const char *names[3] = {MAT_SAMPLER_DIFFUSE, MAT_SAMPLER_SPECULAR, MAT_SAMPLER_EMISSIVE};
    float *colours[3] = {gm.diffuse, gm.specular, gm.emissive};
    for (int ch = 0; ch < 3; ++ch) {
        xtgpu_sampler k = xtgpu_sampler();
        k.texture = -1;
        for (size_t i = 0; m && i < m->get_sampler_count(); ++i) {
            std::string n;
            xtcore::sampler::ISampler *s = const_cast<xtcore::asset::IMaterial *>(m)->get_sampler_by_index(i, &n);
            if (n != names[ch]) continue;
            if (!sampler_of(F, s, k, err)) {
                err = std::string("material sampler '") + names[ch] + "': " + err;
                return false;
            }
            break;
        }
        if (k.kind == XTGPU_SAMPLER_COLOR)
            for (int c = 0; c < 3; ++c) colours[ch][c] = k.a[c];
        else
            F.has_textures = true;
        F.samplers.push_back(k);
    }
    return true;
}

bool material_of(const xtcore::asset::IMaterial *m, xtgpu_material &out, std::string &err)
{
    using namespace xtcore::asset::material;
    out = xtgpu_material();
    if (dynamic_cast<const BlinnPhong *>(m)) out.type = XTGPU_BLINNPHONG;
    else if (dynamic_cast<const Phong *>(m)) out.type = XTGPU_PHONG;
    else if (dynamic_cast<const Lambert *>(m)) out.type = XTGPU_LAMBERT;
    else if (dynamic_cast<const Emissive *>(m)) out.type = XTGPU_EMISSIVE;
    else if (dynamic_cast<const Dielectric *>(m)) out.type = XTGPU_DIELECTRIC;
    else {
        err = "unknown material class";
        return false;
    }
    out.reflectance = m->get_scalar(MAT_SCALART_REFLECTANCE);
    out.exponent = m->get_scalar(MAT_SCALART_EXPONENT);
    out.ior = m->get_scalar(MAT_SCALART_IOR);
    return true;
}

}  // namespace

namespace xtcore {
    namespace integrator {
        namespace gpu {

bool camera_of(xtcore::Scene &scene, HASH_UINT64 camera, xtgpu_camera &out, std::string &err)
{
    out = xtgpu_camera();
    // camera: Perspective (with depth of field when flength > 0,
    // camera/perspective.cc:38-98), ERP (erp.cc:13-31), ODS (ods.cc:17-40) or
    // Cubemap (cubemap.cc:21-69)
    xtcore::asset::ICamera *cam = scene.get_camera(camera);
    if (!cam) {
        err = "no camera";
        return false;
    }
    auto set3 = [](float *o, const nmath::Vector3f &v) {
        o[0] = (float)v.x;
        o[1] = (float)v.y;
        o[2] = (float)v.z;
    };
    set3(out.position, cam->position);
    if (xtcore::camera::Perspective *pc = dynamic_cast<xtcore::camera::Perspective *>(cam)) {
        out.type = XTGPU_CAM_PERSPECTIVE;
        set3(out.target, pc->target);
        set3(out.up, pc->up);
        out.fov = pc->fov;
        out.flength = pc->flength;
        out.aperture = pc->aperture;
    } else if (xtcore::camera::ERP *ec = dynamic_cast<xtcore::camera::ERP *>(cam)) {
        out.type = XTGPU_CAM_ERP;
        set3(out.orientation, ec->orientation);
    } else if (xtcore::camera::ODS *oc = dynamic_cast<xtcore::camera::ODS *>(cam)) {
        out.type = XTGPU_CAM_ODS;
        set3(out.orientation, oc->orientation);
        out.ipd = oc->ipd;
    } else if (dynamic_cast<xtcore::camera::Cubemap *>(cam)) {
        out.type = XTGPU_CAM_CUBEMAP;
    } else {
        err = std::string("unsupported camera type ") + cam->get_type();
        return false;
    }
    return true;
}

xtgpu_status flatten(xtcore::Scene &scene, HASH_UINT64 camera, FlatScene &F, std::string &err)
{
    F = FlatScene();
    auto fail = [&](const std::string &why) {
        err = why;
        return XTGPU_ERR_INVALID;
    };
    // Geometry is grouped by kind in the description (spheres, planes and
    // triangles each in one array) while the objects keep the map order.
    std::map<HASH_UINT64, int32_t> mat_index;
    for (auto it = scene.m_objects.begin(); it != scene.m_objects.end(); ++it) {
        const xtcore::asset::Object *obj = it->second;
        if (!obj) continue;
        auto gs = scene.m_surface.find(obj->surface);
        // Scene::intersection skips objects whose surface is missing
        if (gs == scene.m_surface.end() || !gs->second) continue;
        const xtcore::asset::ISurface *g = gs->second;
        int32_t kind, first, count = 1;
        if (const xtcore::surface::Sphere *s = dynamic_cast<const xtcore::surface::Sphere *>(g)) {
            kind = XTGPU_SPHERE;
            first = (int32_t)(F.spheres.size() / 4);
            put3(F.spheres, s->origin);
            F.spheres.push_back((float)s->radius);
        } else if (const xtcore::surface::Plane *p = dynamic_cast<const xtcore::surface::Plane *>(g)) {
            kind = XTGPU_PLANE;
            first = (int32_t)(F.planes.size() / 4);
            put3(F.planes, p->normal);
            F.planes.push_back((float)p->offset);
        } else if (const xtcore::surface::Triangle *t = dynamic_cast<const xtcore::surface::Triangle *>(g)) {
            kind = XTGPU_MESH;
            first = (int32_t)(F.tris.size() / 9);
            for (int k = 0; k < 3; ++k) put3(F.tris, t->v[k]);
            for (int k = 0; k < 3; ++k) {
                put3(F.tri_normals, t->n[k]);
                F.has_normals |= t->n[k].x != 0 || t->n[k].y != 0 || t->n[k].z != 0;
            }
            F.has_uvs |= put_uvs(F.tri_uvs, *t);
        } else if (const xtcore::surface::Mesh *m = dynamic_cast<const xtcore::surface::Mesh *>(g)) {
            kind = XTGPU_MESH;
            first = (int32_t)(F.tris.size() / 9);
            const TriItems &items = mesh_triangles(m);
            count = (int32_t)items.size();
            for (size_t i = 0; i < items.size(); ++i) {
                const xtcore::surface::Triangle &t = items[i].data;
                for (int k = 0; k < 3; ++k) put3(F.tris, t.v[k]);
                for (int k = 0; k < 3; ++k) {
                    put3(F.tri_normals, t.n[k]);
                    F.has_normals |= t.n[k].x != 0 || t.n[k].y != 0 || t.n[k].z != 0;
                }
                F.has_uvs |= put_uvs(F.tri_uvs, t);
            }
            if (count == 0) continue;   // an empty mesh is never hit
        } else {
            return fail("unsupported surface class");
        }
        // material: shared entries per material id; an object without one
        // gets a black Lambert (the CPU pathtracer dereferences it unchecked)
        int32_t mi;
        auto known = mat_index.find(obj->material);
        if (known != mat_index.end()) {
            mi = known->second;
        } else {
            xtgpu_material gm = xtgpu_material();
            gm.type = XTGPU_LAMBERT;
            auto ms = scene.m_materials.find(obj->material);
            const xtcore::asset::IMaterial *mat = ms != scene.m_materials.end() ? ms->second : 0;
            if (mat && !material_of(mat, gm, err)) return XTGPU_ERR_INVALID;
            if (!samplers_of(F, mat, gm, err)) return XTGPU_ERR_INVALID;
            mi = (int32_t)F.materials.size();
            F.materials.push_back(gm);
            mat_index[obj->material] = mi;
        }
        F.obj_uv_scale.push_back((float)g->uv_scale.x);
        F.obj_uv_scale.push_back((float)g->uv_scale.y);
        F.obj_kind.push_back(kind);
        F.obj_first.push_back(first);
        F.obj_count.push_back(count);
        F.obj_material.push_back(mi);
        F.obj_id.push_back(it->first);
    }
    if (F.tris.size() / 9 > (size_t)INT32_MAX / 4) return fail("too many triangles");

    xtgpu_scene_desc &d = F.desc;
    d = xtgpu_scene_desc();
    d.n_objects = (int32_t)F.obj_kind.size();
    d.obj_kind = F.obj_kind.data();
    d.obj_first = F.obj_first.data();
    d.obj_count = F.obj_count.data();
    d.obj_material = F.obj_material.data();
    d.n_spheres = (int32_t)(F.spheres.size() / 4);
    d.spheres = F.spheres.data();
    d.n_planes = (int32_t)(F.planes.size() / 4);
    d.planes = F.planes.data();
    d.n_tris = (int32_t)(F.tris.size() / 9);
    d.tris = F.tris.data();
    d.tri_normals = F.has_normals ? F.tri_normals.data() : 0;
    d.obj_uv_scale = F.obj_uv_scale.data();
    d.tri_uvs = F.has_uvs ? F.tri_uvs.data() : 0;
    d.n_materials = (int32_t)F.materials.size();
    d.materials = F.materials.data();

    // environment (Scene::sample_environment, scene.cc:142-145)
    d.env_type = XTGPU_ENV_NONE;
    d.env_texture = -1;
    if (scene.m_environment) {
        if (xtcore::sampler::Gradient *gr = dynamic_cast<xtcore::sampler::Gradient *>(scene.m_environment)) {
            d.env_type = XTGPU_ENV_GRADIENT;
            d.env_a[0] = gr->a.r(); d.env_a[1] = gr->a.g(); d.env_a[2] = gr->a.b();
            d.env_b[0] = gr->b.r(); d.env_b[1] = gr->b.g(); d.env_b[2] = gr->b.b();
        } else if (dynamic_cast<xtcore::sampler::SolidColor *>(scene.m_environment)) {
            d.env_type = XTGPU_ENV_COLOR;
            nimg::ColorRGBf c = scene.m_environment->sample(nmath::Vector3f(0, 0, 0));
            d.env_a[0] = c.r(); d.env_a[1] = c.g(); d.env_a[2] = c.b();
        } else if (dynamic_cast<xtcore::sampler::ERP *>(scene.m_environment) ||
                   dynamic_cast<xtcore::sampler::Cubemap *>(scene.m_environment)) {
            xtgpu_sampler k;
            if (!sampler_of(F, scene.m_environment, k, err)) return fail(std::string("environment: ") + err);
            d.env_type = k.kind == XTGPU_SAMPLER_ERP ? XTGPU_ENV_ERP : XTGPU_ENV_CUBEMAP;
            d.env_texture = k.texture;
            F.has_textures = true;
        } else {
            return fail("unsupported environment sampler");
        }
    }
    d.n_textures = (int32_t)F.textures.size();
    d.textures = F.textures.data();
    d.n_texels = (int64_t)(F.texels.size() / 4);
    d.texels = F.texels.data();
    d.mat_samplers = F.has_textures ? F.samplers.data() : 0;

    return camera_of(scene, camera, d.camera, err) ? XTGPU_OK : XTGPU_ERR_INVALID;
}

// ---------------------------------------------------------------------------
Integrator::Integrator(int kind, int node_format)
    : ao_max_distance(100.f), seed(1), record_raygraph(true), m_kind(kind), m_format(node_format), m_scene(0),
      m_uploaded(0), m_camera(0), m_shading_dirty(false), m_x0(0), m_y0(0), m_w(0), m_h(0), m_spx(1), m_served(0),
      m_ready(false), m_empty(false), m_status(XTGPU_OK), m_rays(0)
{}

Integrator::~Integrator()
{
    if (m_scene) xtgpu_scene_destroy(m_scene);
}

void Integrator::invalidate_scene()
{
    std::lock_guard<std::mutex> lock(m_mutex);
    m_uploaded = 0;
}

void Integrator::invalidate_shading()
{
    std::lock_guard<std::mutex> lock(m_mutex);
    m_shading_dirty = true;
}

xtgpu_status Integrator::render_frame()
{
    xtcore::render::params_t &p = ctx->params;
    const bool random = p.sample_distribution == xtcore::antialiasing::SAMPLE_DISTRIBUTION_RANDOM;
    // aa = 0 or samples = 0: antialiasing::produce gives the tiles no samples
    // (aa.cc:9, 67), so the CPU integrators write no pixel
    m_empty = p.aa == 0 || p.samples == 0;
    if (m_empty) return XTGPU_OK;
    if (!m_scene || m_uploaded != &ctx->scene) {
        FlatScene F;
        xtgpu_status st = flatten(ctx->scene, p.camera, F, m_error);
        if (st != XTGPU_OK) return st;
        if (m_scene) xtgpu_scene_destroy(m_scene);
        m_scene = 0;
        if ((st = xtgpu_scene_create(&F.desc, 0, &m_scene)) != XTGPU_OK) {
            m_error = xtgpu_last_error();
            return st;
        }
        xtgpu_bvh_opts o = {m_format, 0};
        if ((st = xtgpu_bvh_build(m_scene, &o, 0)) != XTGPU_OK) {
            m_error = xtgpu_last_error();
            return st;
        }
        m_uploaded = &ctx->scene;
        m_camera = p.camera;
        m_shading_dirty = false;
    } else if (m_shading_dirty) {
        // materials, samplers, textures, environment and camera again, the
        // geometry and BVH kept
        FlatScene F;
        xtgpu_status st = flatten(ctx->scene, p.camera, F, m_error);
        if (st != XTGPU_OK) return st;
        if ((st = xtgpu_scene_update(m_scene, &F.desc, XTGPU_UPDATE_SHADING | XTGPU_UPDATE_CAMERA, 0)) !=
            XTGPU_OK) {
            m_error = xtgpu_last_error();
            return st;
        }
        m_camera = p.camera;
        m_shading_dirty = false;
    } else if (p.camera != m_camera) {
        // the context renders through another camera of the scene
        xtgpu_scene_desc d = xtgpu_scene_desc();
        if (!camera_of(ctx->scene, p.camera, d.camera, m_error)) return XTGPU_ERR_INVALID;
        xtgpu_status st = xtgpu_scene_update(m_scene, &d, XTGPU_UPDATE_CAMERA, 0);
        if (st != XTGPU_OK) {
            m_error = xtgpu_last_error();
            return st;
        }
        m_camera = p.camera;
    }
    // bounding rectangle of the context's tiles
    size_t x0 = (size_t)-1, y0 = (size_t)-1, x1 = 0, y1 = 0;
    for (size_t i = 0; i < ctx->tiles.size(); ++i) {
        const xtcore::render::tile_t &t = ctx->tiles[i];
        x0 = std::min(x0, t.x0());
        y0 = std::min(y0, t.y0());
        x1 = std::max(x1, t.x1());
        y1 = std::max(y1, t.y1());
    }
    if (x1 <= x0 || y1 <= y0) {
        m_error = "no tiles";
        return XTGPU_ERR_INVALID;
    }
    xtgpu_render_params rp = xtgpu_render_params();
    rp.integrator = m_kind;
    rp.width = (int32_t)p.width;
    rp.height = (int32_t)p.height;
    rp.spp = (int32_t)p.samples;
    rp.rdepth = (int32_t)p.rdepth;
    rp.ao_max_distance = ao_max_distance;
    rp.seed = seed;
    rp.node_format = m_format;
    rp.x0 = (int32_t)x0;
    rp.y0 = (int32_t)y0;
    rp.x1 = (int32_t)x1;
    rp.y1 = (int32_t)y1;
    rp.aa = (int32_t)p.aa;
    rp.sample_distribution = random ? XTGPU_SAMPLES_RANDOM : XTGPU_SAMPLES_GRID;
    m_x0 = x0;
    m_y0 = y0;
    m_w = x1 - x0;
    m_h = y1 - y0;
    m_frame.assign(4 * m_w * m_h, 0.f);
    xtgpu_status st;
    m_spx = (size_t)(random ? p.aa : p.aa * p.aa) * p.samples;
    if (m_kind == XTGPU_DEPTH && record_raygraph) {
        // the depth integrator's raygraph (depth/integrator.cc:43-51)
        m_raygraph.assign(10 * m_w * m_h * m_spx, 0.f);
        st = xtgpu_render_raygraph_host(m_scene, &rp, m_frame.data(), m_raygraph.data(), &m_rays, 0);
    } else {
        m_raygraph.clear();
        st = xtgpu_render_host(m_scene, &rp, m_frame.data(), &m_rays, 0);
    }
    if (st != XTGPU_OK) m_error = xtgpu_last_error();
    return st;
}

void Integrator::render_tile(xtcore::render::tile_t *tile)
{
    {
        std::lock_guard<std::mutex> lock(m_mutex);
        if (!m_ready) {
            m_error.clear();
            m_rays = 0;
            m_status = render_frame();
            if (m_status != XTGPU_OK)
                xtcore::Log::handle().post_warning("gpu integrator: %s", m_error.c_str());
            m_served = 0;
            m_ready = true;
        }
    }
    // the produce/pop contract: every sample the tile was given is consumed
    while (tile->samples.count() > 0) {
        xtcore::antialiasing::sample_rgba_t s;
        tile->samples.pop(s);
    }
    if (m_status == XTGPU_OK && !m_empty) {
        for (size_t y = tile->y0(); y < tile->y1(); ++y)
            for (size_t x = tile->x0(); x < tile->x1(); ++x) {
                const float *c = &m_frame[4 * ((y - m_y0) * m_w + (x - m_x0))];
                tile->write(x, y, nimg::ColorRGBAf(c[0], c[1], c[2], c[3]));
            }
        if (!m_raygraph.empty()) {
            // one two-sample path per sample, in the order the tile's queue
            // held them (antialiasing::produce, aa.cc:55-75: column by column,
            // each pixel's grid positions and repeats in order), appended as
            // the CPU depth integrator appends them
            for (size_t x = tile->x0(); x < tile->x1(); ++x)
                for (size_t y = tile->y0(); y < tile->y1(); ++y)
                    for (size_t k = 0; k < m_spx; ++k) {
                        const float *r = &m_raygraph[10 * (((y - m_y0) * m_w + (x - m_x0)) * m_spx + k)];
                        xtcore::raygraph::path_t path;
                        xtcore::raygraph::sample_t s0, s1;
                        s0.position = nmath::Vector3f(r[0], r[1], r[2]);
                        s1.position = nmath::Vector3f(r[3], r[4], r[5]);
                        s1.color = nimg::ColorRGBAf(r[6], r[7], r[8], r[9]);
                        path.samples.push_back(s0);
                        path.samples.push_back(s1);
                        tile->raygraph_bundle.paths.push_back(path);
                    }
        }
    }
    std::lock_guard<std::mutex> lock(m_mutex);
    if (++m_served >= ctx->tiles.size()) m_ready = false;
}

        } /* namespace gpu */
    } /* namespace integrator */
} /* namespace xtcore */
