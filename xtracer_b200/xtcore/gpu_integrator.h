// GPU integrator for XTracer's xtcore: stencil, depth, AO and pathtracer
// rendered by libxtgpu.so on a B200, behind the reference's own interface
// xtcore::render::IIntegrator (src/xtcore/integrator.h:10-24).
//
// IIntegrator::render() (src/xtcore/integrator.cc:29-53) is not virtual: it
// runs the OpenMP tile loop (tile->init, antialiasing::produce, render_tile,
// tile->submit).  The first render_tile of a frame renders the bounding
// rectangle of the context's tiles on the GPU in one call; every render_tile
// then drains its tile's sample queue, as the CPU integrators do, and writes
// its pixels from that frame.  When the last tile has been served the frame is
// dropped, so the next render() renders again.
//
// The loaded Scene is flattened (objects in Scene::m_objects order, the order
// Scene::intersection visits them, scene.cc:191-216) and uploaded once; call
// invalidate_scene() after changing its geometry, invalidate_shading() after
// changing only materials, samplers, the environment or cameras.  A context
// that switches to another camera of the scene is followed on its own.
//
// Supported: perspective (with depth of field), ERP, ODS and cubemap cameras
// (a cubemap's height a multiple of 6), spheres (and points, which the loader
// makes spheres of radius 0), planes, triangles, meshes, colour, gradient,
// texture, ERP and cubemap material samplers, no / colour / gradient / ERP /
// cubemap environment, any aa with the grid
// sample distribution (aa <= 1 with the random one).  Anything else makes the
// frame fail: status() and error() say why, the tiles stay as tile->init()
// left them, and a warning goes to xtcore's log.  The depth-of-field lens
// draws come from the GPU's sample streams, not from the C library's rand().
#ifndef XTGPU_XTCORE_GPU_INTEGRATOR_H
#define XTGPU_XTCORE_GPU_INTEGRATOR_H

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <xtgpu.h>
#include <xtcore/integrator.h>
#include <xtcore/scene.h>

namespace xtcore {
    namespace integrator {
        namespace gpu {

// A loaded Scene as the C ABI's scene description; desc points into the
// vectors, so it lives as long as the FlatScene.
struct FlatScene {
    std::vector<int32_t> obj_kind, obj_first, obj_count, obj_material;
    std::vector<HASH_UINT64> obj_id;          // Scene::m_objects key of each object
    std::vector<float> spheres, planes, tris, tri_normals;
    std::vector<float> obj_uv_scale, tri_uvs;   // 2 per object, 6 per triangle
    std::vector<xtgpu_material> materials;
    std::vector<xtgpu_texture> textures;
    std::vector<float> texels;                 // 4 per texel
    std::vector<xtgpu_sampler> samplers;       // 3 per material
    std::map<const void *, int32_t> tex_index; // sampler object -> its first texture
    bool has_textures = false;                 // a non-colour sampler is used
    bool has_normals = false;
    bool has_uvs = false;     // a triangle's texcoords differ from the constructor's
    xtgpu_scene_desc desc;
};

// The scene camera `camera` as the C ABI's camera; false (reason in err) for a
// missing or unsupported camera.
bool camera_of(xtcore::Scene &scene, HASH_UINT64 camera, xtgpu_camera &out, std::string &err);

// Flattens ctx.scene with the given camera.  Returns XTGPU_OK, or
// XTGPU_ERR_INVALID with the reason in err for what the GPU path cannot render.
xtgpu_status flatten(xtcore::Scene &scene, HASH_UINT64 camera, FlatScene &out, std::string &err);

class Integrator : public xtcore::render::IIntegrator
{
    public:
    // kind: XTGPU_STENCIL .. XTGPU_WIREFRAME (stencil, depth, ao, pathtracer,
    // normal, uv, emission, wireframe);
    // node_format: XTGPU_NODES_FP32, XTGPU_NODES_Q8 or XTGPU_NODES_W8
    explicit Integrator(int kind, int node_format = XTGPU_NODES_FP32);
    ~Integrator();

    void render_tile(xtcore::render::tile_t *tile);

    float ao_max_distance;   // AO occlusion distance; the CPU integrator's is 100
    uint64_t seed;           // sample streams are keyed by (seed, pixel, sample)
    // depth: append each sample's raygraph path to its tile's bundle, as the
    // CPU depth integrator does (depth/integrator.cc:43-51); on by default
    bool record_raygraph;

    // after the scene's geometry changed: flatten, upload and rebuild the BVH
    void invalidate_scene();
    // after materials, samplers, the environment or cameras changed (an edit
    // or a -mod of those): re-upload them, keep the geometry and BVH
    void invalidate_shading();
    xtgpu_status status() const { return m_status; }   // of the last frame
    const std::string &error() const { return m_error; }
    uint64_t rays() const { return m_rays; }           // rays traced by the last frame

    private:
    xtgpu_status render_frame();

    int m_kind, m_format;
    std::mutex m_mutex;
    xtgpu_scene *m_scene;
    const xtcore::Scene *m_uploaded;
    HASH_UINT64 m_camera;              // the camera uploaded
    bool m_shading_dirty;
    std::vector<float> m_frame;        // RGBA of the rectangle, row-major
    std::vector<float> m_raygraph;     // depth: 10 floats per sample, pixels row-major
    size_t m_x0, m_y0, m_w, m_h;
    size_t m_spx;                      // samples per pixel (aa^2 x samples)
    size_t m_served;                   // tiles served from the current frame
    bool m_ready;
    bool m_empty;                      // the context gives the tiles no samples
    xtgpu_status m_status;
    std::string m_error;
    uint64_t m_rays;
};

        } /* namespace gpu */
    } /* namespace integrator */
} /* namespace xtcore */

#endif
