// xtgpu-xtcore: a minimal XTracer front end that renders a .scn through the
// reference host (io::scn::load, params, tiles, IIntegrator::render, assemble)
// with the GPU integrator, or with one of the reference's CPU integrators for
// comparison, as the GUI does it (src/frontend/gui/workspace.cc:55-81).
//
//   xtgpu-xtcore render <scn> <integrator> W H spp rdepth <out.bin> [options]
//       integrator: stencil | depth | ao | pathtracer | normal | uv | emission | wireframe
//       --cpu          the reference's CPU integrator instead of the GPU one
//       --q8           binary BVH with 8-bit quantised nodes (GPU)
//       --w8           8-wide BVH with 8-bit quantised nodes (GPU)
//       --seed N       sample stream key (GPU), default 1
//       --ao-distance D  AO occlusion distance (GPU), default 100
//       --threads N    OpenMP threads of the tile loop, default all
//       --tile N       tile size, default 32 (context.cc:5)
//       --aa N         anti-aliasing level, default 1
//       --random       the random sample distribution (aa jittered positions
//                      per pixel) instead of the grid
//       --raygraph P   the depth integrator's raygraph as PLY, exported the
//                      GUI's way (render::assemble + raygraph::write)
//       --then-camera N  render once more through the scene's camera N (the
//                      output is that second frame)
//       --png P        the assembled frame as PNG through the GPU quantiser
//       --exr P        the assembled frame as OpenEXR (this library's writer)
//       --ref-png P, --ref-exr P   the same frame through XTracer's own writers
//                      (nimg::io::save::png / exr), for comparison
//   xtgpu-xtcore flatten <scn> <out.bin>
//       writes the flattened scene description (see write_flat)
//
// render writes int32 width, height, then width*height RGBA float32 pixels,
// row-major (the assembled Pixmap), and prints one JSON line.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <omp.h>

#include <xtcore/xtcore.h>
#include <xtcore/log.h>
#include <xtcore/context.h>
#include <xtcore/integrator.h>
#include <xtcore/integrator/wireframe/integrator.h>
#include <xtcore/parseutil.h>
#include <xtcore/strpool.h>
#include <xtcore/util/raygraph.h>
#include <nimg/img.h>

#include "gpu_integrator.h"

namespace {

int load(xtcore::render::context_t &ctx, const char *scn)
{
    xtcore::Log::handle().echo(false);
    if (xtcore::io::scn::load(&ctx.scene, scn, 0)) {
        fprintf(stderr, "xtgpu-xtcore: failed to load %s\n", scn);
        return 1;
    }
    if (ctx.scene.m_cameras.empty()) {
        fprintf(stderr, "xtgpu-xtcore: no camera in %s\n", scn);
        return 1;
    }
    // the GUI's fallback (gui/workspace.cc:33-39): the first camera
    ctx.params.camera = ctx.scene.m_cameras.begin()->first;
    return 0;
}

template <typename T>
void put(FILE *f, const T *p, size_t n)
{
    if (n) fwrite(p, sizeof(T), n, f);
}

// int32 n_objects, n_spheres, n_planes, n_tris, n_materials, has_normals,
// env_type, has_uvs; int32 obj_kind/first/count/material [n_objects each];
// float32 spheres [4n], planes [4n], tris [9n], tri_normals [9n] when
// has_normals, obj_uv_scale [2 n_objects], tri_uvs [6n] when has_uvs;
// per material int32 type + float32 diffuse[3] specular[3] emissive[3]
// reflectance exponent ior; float32 env_a[3] env_b[3]; float32 camera
// position[3] target[3] up[3] fov; int32 camera type; float32 orientation[3]
// ipd flength aperture; int32 n_textures, has_samplers, env_texture; per
// texture int32 width height filtering, int64 offset; int64 n_texels; float32
// texels [4n]; when has_samplers, per material 3 x (int32 kind texture,
// float32 a[3] b[3]).
int write_flat(const xtcore::integrator::gpu::FlatScene &F, const char *out)
{
    const xtgpu_scene_desc &d = F.desc;
    FILE *f = fopen(out, "wb");
    if (!f) return 1;
    int32_t head[8] = {d.n_objects, d.n_spheres, d.n_planes, d.n_tris, d.n_materials, d.tri_normals ? 1 : 0,
                       d.env_type, d.tri_uvs ? 1 : 0};
    put(f, head, 8);
    put(f, d.obj_kind, (size_t)d.n_objects);
    put(f, d.obj_first, (size_t)d.n_objects);
    put(f, d.obj_count, (size_t)d.n_objects);
    put(f, d.obj_material, (size_t)d.n_objects);
    put(f, d.spheres, 4 * (size_t)d.n_spheres);
    put(f, d.planes, 4 * (size_t)d.n_planes);
    put(f, d.tris, 9 * (size_t)d.n_tris);
    if (d.tri_normals) put(f, d.tri_normals, 9 * (size_t)d.n_tris);
    put(f, d.obj_uv_scale, 2 * (size_t)d.n_objects);
    if (d.tri_uvs) put(f, d.tri_uvs, 6 * (size_t)d.n_tris);
    for (int32_t i = 0; i < d.n_materials; ++i) {
        const xtgpu_material &m = d.materials[i];
        put(f, &m.type, 1);
        put(f, m.diffuse, 3);
        put(f, m.specular, 3);
        put(f, m.emissive, 3);
        float sc[3] = {m.reflectance, m.exponent, m.ior};
        put(f, sc, 3);
    }
    put(f, d.env_a, 3);
    put(f, d.env_b, 3);
    put(f, d.camera.position, 3);
    put(f, d.camera.target, 3);
    put(f, d.camera.up, 3);
    put(f, &d.camera.fov, 1);
    put(f, &d.camera.type, 1);
    put(f, d.camera.orientation, 3);
    float lens[3] = {d.camera.ipd, d.camera.flength, d.camera.aperture};
    put(f, lens, 3);
    int32_t th[3] = {d.n_textures, d.mat_samplers ? 1 : 0, d.env_texture};
    put(f, th, 3);
    for (int32_t i = 0; i < d.n_textures; ++i) {
        int32_t t3[3] = {d.textures[i].width, d.textures[i].height, d.textures[i].filtering};
        put(f, t3, 3);
        put(f, &d.textures[i].offset, 1);
    }
    put(f, &d.n_texels, 1);
    put(f, d.texels, 4 * (size_t)d.n_texels);
    if (d.mat_samplers)
        for (int32_t i = 0; i < 3 * d.n_materials; ++i) {
            const xtgpu_sampler &k = d.mat_samplers[i];
            int32_t kt[2] = {k.kind, k.texture};
            put(f, kt, 2);
            put(f, k.a, 3);
            put(f, k.b, 3);
        }
    fclose(f);
    return 0;
}

int mode_flatten(int argc, char **argv)
{
    if (argc < 4) return 2;
    xtcore::init();
    xtcore::render::context_t ctx;
    if (load(ctx, argv[2])) return 1;
    xtcore::integrator::gpu::FlatScene F;
    std::string err;
    if (xtcore::integrator::gpu::flatten(ctx.scene, ctx.params.camera, F, err) != XTGPU_OK) {
        fprintf(stderr, "xtgpu-xtcore: %s\n", err.c_str());
        return 1;
    }
    return write_flat(F, argv[3]);
}

int mode_render(int argc, char **argv)
{
    if (argc < 9) return 2;
    const char *scn = argv[2];
    std::string integ = argv[3];
    size_t w = strtoul(argv[4], 0, 10), h = strtoul(argv[5], 0, 10);
    size_t spp = strtoul(argv[6], 0, 10), rdepth = strtoul(argv[7], 0, 10);
    const char *out = argv[8];
    bool cpu = false, q8 = false, w8 = false, random = false;
    unsigned long long seed = 1;
    float aod = 100.f;
    size_t threads = 0, tile = 32, aa = 1;
    std::string png, exr, ref_png, ref_exr, raygraph, then_camera;
    for (int i = 9; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "--cpu") cpu = true;
        else if (a == "--q8") q8 = true;
        else if (a == "--w8") w8 = true;
        else if (a == "--seed" && i + 1 < argc) seed = strtoull(argv[++i], 0, 10);
        else if (a == "--ao-distance" && i + 1 < argc) aod = (float)atof(argv[++i]);
        else if (a == "--threads" && i + 1 < argc) threads = strtoul(argv[++i], 0, 10);
        else if (a == "--tile" && i + 1 < argc) tile = strtoul(argv[++i], 0, 10);
        else if (a == "--aa" && i + 1 < argc) aa = strtoul(argv[++i], 0, 10);
        else if (a == "--random") random = true;
        else if (a == "--raygraph" && i + 1 < argc) raygraph = argv[++i];
        else if (a == "--then-camera" && i + 1 < argc) then_camera = argv[++i];
        else if (a == "--png" && i + 1 < argc) png = argv[++i];
        else if (a == "--exr" && i + 1 < argc) exr = argv[++i];
        else if (a == "--ref-png" && i + 1 < argc) ref_png = argv[++i];
        else if (a == "--ref-exr" && i + 1 < argc) ref_exr = argv[++i];
        else {
            fprintf(stderr, "xtgpu-xtcore: unknown option %s\n", a.c_str());
            return 2;
        }
    }
    if (!w || !h || !spp || !tile) return 2;

    xtcore::init();
    xtcore::render::context_t ctx;
    if (load(ctx, scn)) return 1;
    ctx.params.width = w;
    ctx.params.height = h;
    ctx.params.samples = spp;
    ctx.params.rdepth = rdepth;
    ctx.params.threads = threads;
    ctx.params.tile_size = tile;
    ctx.params.aa = aa;
    ctx.params.sample_distribution = random ? xtcore::antialiasing::SAMPLE_DISTRIBUTION_RANDOM
                                            : xtcore::antialiasing::SAMPLE_DISTRIBUTION_GRID;
    ctx.init();   // segments the frame into tiles (context.cc)

    xtcore::render::IIntegrator *ig = 0;
    xtcore::integrator::gpu::Integrator *gi = 0;
    int kind = integ == "stencil" ? XTGPU_STENCIL : integ == "depth" ? XTGPU_DEPTH : integ == "ao" ? XTGPU_AO
             : integ == "pathtracer" ? XTGPU_PATHTRACER : integ == "normal" ? XTGPU_NORMAL : integ == "uv" ? XTGPU_UV
             : integ == "emission" ? XTGPU_EMISSION : integ == "wireframe" ? XTGPU_WIREFRAME : -1;
    if (kind < 0) {
        fprintf(stderr, "xtgpu-xtcore: unknown integrator %s\n", integ.c_str());
        return 2;
    }
    if (cpu) {
        if (kind == XTGPU_STENCIL) ig = new xtcore::integrator::stencil::Integrator();
        else if (kind == XTGPU_DEPTH) ig = new xtcore::integrator::depth::Integrator();
        else if (kind == XTGPU_AO) ig = new xtcore::integrator::ao::Integrator();
        else if (kind == XTGPU_NORMAL) ig = new xtcore::integrator::normal::Integrator();
        else if (kind == XTGPU_UV) ig = new xtcore::integrator::uv::Integrator();
        else if (kind == XTGPU_EMISSION) ig = new xtcore::integrator::emission::Integrator();
        else if (kind == XTGPU_WIREFRAME) ig = new xtcore::integrator::wireframe::Integrator();
        else ig = new xtcore::integrator::pathtracer::Integrator();
    } else {
        gi = new xtcore::integrator::gpu::Integrator(kind, w8 ? XTGPU_NODES_W8 : q8 ? XTGPU_NODES_Q8 : XTGPU_NODES_FP32);
        gi->seed = seed;
        gi->ao_max_distance = aod;
        ig = gi;
    }
    ig->setup(ctx);
    auto t0 = std::chrono::steady_clock::now();
    ig->render();
    auto t1 = std::chrono::steady_clock::now();
    if (!then_camera.empty()) {
        // the GUI's camera selection (workspace.cc): another camera of the
        // loaded scene, the same integrator
        ctx.params.camera = xtcore::pool::str::add(then_camera.c_str());
        if (ctx.scene.m_cameras.find(ctx.params.camera) == ctx.scene.m_cameras.end()) {
            fprintf(stderr, "xtgpu-xtcore: no camera %s\n", then_camera.c_str());
            return 1;
        }
        t0 = std::chrono::steady_clock::now();
        ig->render();
        t1 = std::chrono::steady_clock::now();
    }
    double secs = std::chrono::duration<double>(t1 - t0).count();

    nimg::Pixmap pm;
    xtcore::render::assemble(pm, ctx);
    FILE *f = fopen(out, "wb");
    if (!f) return 1;
    int32_t wh[2] = {(int32_t)w, (int32_t)h};
    put(f, wh, 2);
    std::vector<float> row(4 * w);
    for (size_t y = 0; y < h; ++y) {
        for (size_t x = 0; x < w; ++x) {
            const nimg::ColorRGBAf &c = pm.pixel_ro(x, y);
            row[4 * x] = c.r();
            row[4 * x + 1] = c.g();
            row[4 * x + 2] = c.b();
            row[4 * x + 3] = c.a();
        }
        put(f, row.data(), row.size());
    }
    fclose(f);
    int rc = 0;
    if (!png.empty() || !exr.empty()) {
        std::vector<float> frame(4 * w * h);
        for (size_t y = 0; y < h; ++y)
            for (size_t x = 0; x < w; ++x) {
                const nimg::ColorRGBAf &c = pm.pixel_ro(x, y);
                float *o = &frame[4 * (y * w + x)];
                o[0] = c.r();
                o[1] = c.g();
                o[2] = c.b();
                o[3] = c.a();
            }
        if (!png.empty() && xtgpu_save_png_host(png.c_str(), (int32_t)w, (int32_t)h, frame.data(), 0) != XTGPU_OK) {
            fprintf(stderr, "xtgpu-xtcore: %s\n", xtgpu_last_error());
            rc = 1;
        }
        if (!exr.empty() && xtgpu_write_exr(exr.c_str(), (int32_t)w, (int32_t)h, frame.data()) != XTGPU_OK) {
            fprintf(stderr, "xtgpu-xtcore: %s\n", xtgpu_last_error());
            rc = 1;
        }
    }
    if (!raygraph.empty()) {
        xtcore::raygraph::raygraph_t rg;
        xtcore::render::assemble(rg, ctx);
        if (xtcore::raygraph::write(raygraph.c_str(), rg)) rc = 1;
    }
    if (!ref_png.empty() && nimg::io::save::png(ref_png.c_str(), pm)) rc = 1;
    if (!ref_exr.empty() && nimg::io::save::exr(ref_exr.c_str(), pm)) rc = 1;
    if (gi) {
        printf("{\"integrator\": \"gpu:%s\", \"render_s\": %.9f, \"rays\": %llu, \"status\": %d, \"error\": \"%s\"}\n",
               integ.c_str(), secs, (unsigned long long)gi->rays(), (int)gi->status(), gi->error().c_str());
        if (gi->status() != XTGPU_OK) rc = 1;
    } else {
        printf("{\"integrator\": \"cpu:%s\", \"render_s\": %.9f, \"threads\": %d}\n", integ.c_str(), secs,
               threads ? (int)threads : omp_get_max_threads());
    }
    delete ig;
    return rc;
}

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 2) {
        fprintf(stderr, "usage: xtgpu-xtcore render|flatten ...\n");
        return 2;
    }
    std::string m = argv[1];
    int rc = 2;
    if (m == "render") rc = mode_render(argc, argv);
    else if (m == "flatten") rc = mode_flatten(argc, argv);
    if (rc == 2) fprintf(stderr, "xtgpu-xtcore: bad arguments\n");
    return rc;
}
