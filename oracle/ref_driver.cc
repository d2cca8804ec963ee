// Harness driver for the reference renderer (XTracer's xtcore, compiled from its
// own sources by oracle/ref.mk).  TEST INFRASTRUCTURE: it produces the golden
// fixtures that pin the oracle restatement and it is the timed CPU baseline.
//
// The reference CLI cannot render (its integrator pointer is left NULL,
// src/frontend/cli/xtracer.cc:91-117), so this driver does what the GUI does
// (src/frontend/gui/workspace.cc:55-81): io::scn::load -> params -> tiles ->
// IIntegrator::setup/render, then reads the tile pixels back.
//
// Modes
//   xtref render <scn> <integrator> W H spp aa rdepth threads seed <tiles.txt|-> <out.bin> [ao_maxdist]
//                [raygraph.ply|-] [distribution: 0 grid, 1 random]
//   xtref hits   <scn> W H <tiles.txt|-> <out.bin> [mesh.obj]
//   xtref kat    <in.txt> <out.txt>
//   xtref bench  <scn> <integrator> W H spp rdepth threads seed <tiles.txt|-> repeats
//                (the CPU baseline: the scene is loaded once, its load and
//                octree build timed on their own, then IIntegrator::render runs
//                `repeats` times over the same tiles, each timed)
//
// Two link-time hooks (-Wl,--wrap, no reference source is modified):
//   * Scene::intersection is counted, so the ray count of a render is exact;
//   * time() returns the seed, so the reference's srand(time(NULL)) on the first
//     prng_c call of each translation unit (lib/nmath/prng.inl:75-79) becomes
//     reproducible for single-threaded runs.
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>
#include <omp.h>

#include <xtcore/xtcore.h>
#include <xtcore/log.h>
#include <xtcore/strpool.h>
#include <xtcore/context.h>
#include <xtcore/integrator.h>
#include <xtcore/integrator/wireframe/integrator.h>
#include <xtcore/parseutil.h>
#include <xtcore/mesh.h>
#include <xtcore/octree.h>
#include <xtcore/math/sphere.h>
#include <xtcore/math/plane.h>
#include <xtcore/math/triangle.h>
#include <xtcore/math/aabb.h>
#include <xtcore/camera/perspective.h>
#include <xtcore/camera/erp.h>
#include <xtcore/camera/ods.h>
#include <xtcore/camera/cubemap.h>
#include <xtcore/sampler_col.h>
#include <xtcore/sampler_gradient.h>
#include <xtcore/sampler_tex.h>
#include <xtcore/sampler_erp.h>
#include <xtcore/sampler_cubemap.h>
#include <xtcore/util/raygraph.h>
#include <xtcore/material/lambert.h>
#include <xtcore/material/phong.h>
#include <xtcore/material/blinnphong.h>
#include <xtcore/material/emissive.h>
#include <nmesh/obj.h>
#include <nmath/sample.h>

#define SCENE_INTERSECTION _ZN6xtcore5Scene12intersectionERKNS_3RayERNS_12hit_record_tE
#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)

static std::atomic<unsigned long long> g_rays(0);
static time_t g_fixed_time = 1;

extern "C" bool CAT(__real_, SCENE_INTERSECTION)(xtcore::Scene *, const xtcore::Ray &, xtcore::hit_record_t &);
extern "C" bool CAT(__wrap_, SCENE_INTERSECTION)(xtcore::Scene *s, const xtcore::Ray &r, xtcore::hit_record_t &h)
{
    g_rays.fetch_add(1, std::memory_order_relaxed);
    return CAT(__real_, SCENE_INTERSECTION)(s, r, h);
}

extern "C" time_t __wrap_time(time_t *t)
{
    if (t) *t = g_fixed_time;
    return g_fixed_time;
}

using xtcore::Ray;
using xtcore::hit_record_t;
using nmath::Vector3f;

// ---------------------------------------------------------------------------
// AO with the maximum distance as a parameter.  The shipped integrator has it as
// a #define of 100 (src/xtcore/integrator/ao/integrator.cc:10); this restates that
// render_tile (ao/integrator.cc:12-53) with the distance passed in, calling the
// reference's Scene::intersection and nmath::sample::hemisphere unchanged.
class AoWithDistance : public xtcore::render::IIntegrator
{
public:
    explicit AoWithDistance(float d) : maxd(d) {}
    float maxd;
    void render_tile(xtcore::render::tile_t *tile)
    {
        xtcore::asset::ICamera *cam = ctx->scene.get_camera(ctx->params.camera);
        while (tile->samples.count() > 0) {
            xtcore::antialiasing::sample_rgba_t sample;
            tile->samples.pop(sample);
            hit_record_t hr;
            nimg::ColorRGBAf px;
            tile->read(sample.pixel.x, sample.pixel.y, px);
            Vector3f acc(px.r(), px.g(), px.b());
            Ray ray = cam->get_primary_ray(sample.coords.x, sample.coords.y,
                                           (float)ctx->params.width, (float)ctx->params.height);
            float w = 1.0f;
            if (ctx->scene.intersection(ray, hr)) {
                Ray ao;
                ao.direction = nmath::sample::hemisphere(hr.normal, hr.normal);
                ao.origin = hr.point + hr.normal * EPSILON;
                hit_record_t ahr;
                if (ctx->scene.intersection(ao, ahr)) {
                    float dist = (ahr.point - ao.origin).length();
                    w = nmath::min(dist, maxd) / maxd;
                }
            }
            acc += w * sample.weight;
            px = nimg::ColorRGBAf(acc.x, acc.y, acc.z, 1.f);
            tile->write(floor(sample.pixel.x), floor(sample.pixel.y), px);
        }
    }
};

// ---------------------------------------------------------------------------
static bool read_tiles(const char *path, size_t w, size_t h, xtcore::render::Tileset &tiles)
{
    tiles.clear();
    if (!strcmp(path, "-")) {
        xtcore::render::segment_framebuffer(tiles, w, h, 32);
        return true;
    }
    FILE *f = fopen(path, "r");
    if (!f) return false;
    unsigned long x0, y0, x1, y1;
    while (fscanf(f, "%lu %lu %lu %lu", &x0, &y0, &x1, &y1) == 4) {
        if (x1 > w || y1 > h || x0 >= x1 || y0 >= y1) { fclose(f); return false; }
        tiles.push_back(xtcore::render::tile_t(x0, y0, x1, y1));
    }
    fclose(f);
    return true;
}

static int load_scene(xtcore::render::context_t &ctx, const char *scn)
{
    xtcore::Log::handle().echo(false);
    if (xtcore::io::scn::load(&ctx.scene, scn, 0)) {
        fprintf(stderr, "xtref: failed to load %s\n", scn);
        return 1;
    }
    if (ctx.scene.m_cameras.empty()) {
        fprintf(stderr, "xtref: no camera in %s\n", scn);
        return 1;
    }
    // Same fallback as the GUI (gui/workspace.cc:33-39): the first camera.
    ctx.params.camera = ctx.scene.m_cameras.begin()->first;
    return 0;
}

static xtcore::render::IIntegrator *make_integrator(const std::string &integ, float ao_maxd)
{
    if (integ == "stencil") return new xtcore::integrator::stencil::Integrator();
    if (integ == "depth") return new xtcore::integrator::depth::Integrator();
    if (integ == "pathtracer") return new xtcore::integrator::pathtracer::Integrator();
    if (integ == "normal") return new xtcore::integrator::normal::Integrator();
    if (integ == "uv") return new xtcore::integrator::uv::Integrator();
    if (integ == "emission") return new xtcore::integrator::emission::Integrator();
    if (integ == "wireframe") return new xtcore::integrator::wireframe::Integrator();
    if (integ == "ao") {
        if (ao_maxd == 100.0f) return new xtcore::integrator::ao::Integrator();
        return new AoWithDistance(ao_maxd);
    }
    return 0;
}

static int mode_render(int argc, char **argv)
{
    if (argc < 13) return 2;
    const char *scn = argv[2];
    std::string integ = argv[3];
    size_t w = atol(argv[4]), h = atol(argv[5]), spp = atol(argv[6]), aa = atol(argv[7]);
    size_t rdepth = atol(argv[8]), threads = atol(argv[9]);
    g_fixed_time = (time_t)atoll(argv[10]);
    const char *tiles_path = argv[11], *out = argv[12];
    float ao_maxd = argc > 13 ? (float)atof(argv[13]) : 100.0f;
    const char *raygraph_out = argc > 14 ? argv[14] : 0;
    const int random = argc > 15 && atoi(argv[15]) == 1;

    xtcore::init();
    xtcore::render::context_t ctx;
    if (load_scene(ctx, scn)) return 1;
    HASH_UINT64 cam = ctx.params.camera;
    ctx.params.width = w;
    ctx.params.height = h;
    ctx.params.samples = spp;
    ctx.params.aa = aa;
    ctx.params.sample_distribution = random ? xtcore::antialiasing::SAMPLE_DISTRIBUTION_RANDOM
                                            : xtcore::antialiasing::SAMPLE_DISTRIBUTION_GRID;
    ctx.params.rdepth = rdepth;
    ctx.params.threads = threads;
    ctx.params.camera = cam;
    if (!read_tiles(tiles_path, w, h, ctx.tiles)) {
        fprintf(stderr, "xtref: bad tiles %s\n", tiles_path);
        return 1;
    }

    xtcore::render::IIntegrator *ig = make_integrator(integ, ao_maxd);
    if (!ig) { fprintf(stderr, "xtref: unknown integrator %s\n", integ.c_str()); return 1; }

    ig->setup(ctx);
    g_rays = 0;
    auto t0 = std::chrono::steady_clock::now();
    ig->render();
    auto t1 = std::chrono::steady_clock::now();
    double secs = std::chrono::duration<double>(t1 - t0).count();

    FILE *f = fopen(out, "wb");
    if (!f) return 1;
    long long npx = 0;
    for (size_t i = 0; i < ctx.tiles.size(); ++i) npx += (long long)(ctx.tiles[i].width() * ctx.tiles[i].height());
    fwrite(&npx, 8, 1, f);
    for (size_t i = 0; i < ctx.tiles.size(); ++i) {
        const xtcore::render::tile_t &t = ctx.tiles[i];
        for (size_t y = t.y0(); y < t.y1(); ++y)
            for (size_t x = t.x0(); x < t.x1(); ++x) {
                nimg::ColorRGBAf c;
                t.read(x, y, c);
                int xy[2] = {(int)x, (int)y};
                float rgba[4] = {c.r(), c.g(), c.b(), c.a()};
                fwrite(xy, 4, 2, f);
                fwrite(rgba, 4, 4, f);
            }
    }
    fclose(f);
    if (raygraph_out && strcmp(raygraph_out, "-")) {
        // the GUI's raygraph export (gui/action.cc:65-85): the tiles' bundles
        // in tile order, written by raygraph::write (util/raygraph.cc:8-75)
        xtcore::raygraph::raygraph_t rg;
        xtcore::render::assemble(rg, ctx);
        if (xtcore::raygraph::write(raygraph_out, rg)) return 1;
    }
    int nthr = threads ? (int)threads : omp_get_max_threads();
    printf("{\"render_s\": %.9f, \"rays\": %llu, \"pixels\": %lld, \"threads\": %d}\n",
           secs, (unsigned long long)g_rays.load(), npx, nthr);
    delete ig;
    return 0;
}

// Mesh replica: the triangle loop of Mesh::build_octree (src/xtcore/mesh.cc:70-113)
// with the same insertion order and limits, so the returned OctreeItem* gives the
// primitive index the reference's Scene::intersection does not expose.
struct MeshReplica {
    xtcore::Octree<xtcore::surface::Triangle> oct;
};

static int build_replica(const char *objpath, MeshReplica &rep)
{
    nmesh::object_t obj;
    if (nmesh::io::import::obj(objpath, obj)) return 1;
    size_t tris_added = 0;
    for (auto it = obj.shapes.begin(); it != obj.shapes.end(); ++it) {
        for (size_t i = 0; i < it->mesh.indices.size() / 3; ++i) {
            nmesh::attrib_t *d = &obj.attributes;
            xtcore::surface::Triangle p;
            for (int k = 0; k < 3; ++k) {
                int vi = it->mesh.indices[3 * i + k].v;
                int ni = it->mesh.indices[3 * i + k].n;
                if (vi != -1) p.v[k] = Vector3f(d->v[3 * vi], d->v[3 * vi + 1], d->v[3 * vi + 2]);
                if (ni != -1) p.n[k] = Vector3f(d->n[3 * ni], d->n[3 * ni + 1], d->n[3 * ni + 2]);
            }
            // tc[0] is only read to interpolate the hit record's texcoord
            // (triangle.cc:108-110); it carries the insertion index here.
            p.tc[0] = nmath::Vector2f((double)tris_added++, 0.0);
            p.calc_aabb();
            rep.oct.add(p.aabb, p);
        }
    }
    rep.oct.max_items_per_node(LIMITS_MAX_ITEMS_PER_NODE);
    rep.oct.max_depth(LIMITS_MAX_DEPTH);
    rep.oct.build();
    return 0;
}

static int mode_hits(int argc, char **argv)
{
    if (argc < 7) return 2;
    const char *scn = argv[2];
    size_t w = atol(argv[3]), h = atol(argv[4]);
    const char *tiles_path = argv[5], *out = argv[6];
    const char *objpath = argc > 7 ? argv[7] : 0;

    xtcore::init();
    xtcore::render::context_t ctx;
    if (load_scene(ctx, scn)) return 1;
    xtcore::asset::ICamera *cam = ctx.scene.get_camera(ctx.params.camera);
    if (!read_tiles(tiles_path, w, h, ctx.tiles)) return 1;

    // Object ids in the order Scene::intersection visits them (std::map order).
    std::vector<HASH_UINT64> order;
    for (auto it = ctx.scene.m_objects.begin(); it != ctx.scene.m_objects.end(); ++it) order.push_back(it->first);

    MeshReplica rep;
    bool have_rep = false;
    if (objpath) {
        if (build_replica(objpath, rep)) { fprintf(stderr, "xtref: bad obj %s\n", objpath); return 1; }
        have_rep = true;
    }

    FILE *f = fopen(out, "wb");
    if (!f) return 1;
    long long n = 0;
    for (size_t i = 0; i < ctx.tiles.size(); ++i) n += (long long)(ctx.tiles[i].width() * ctx.tiles[i].height());
    int nobj = (int)order.size();
    fwrite(&n, 8, 1, f);
    fwrite(&nobj, 4, 1, f);
    for (int i = 0; i < nobj; ++i) {
        const char *name = xtcore::pool::str::get(order[i]);
        char buf[64] = {0};
        strncpy(buf, name ? name : "", 63);
        fwrite(buf, 1, 64, f);
    }
    auto t0 = std::chrono::steady_clock::now();
    for (size_t ti = 0; ti < ctx.tiles.size(); ++ti) {
        const xtcore::render::tile_t &t = ctx.tiles[ti];
        for (size_t y = t.y0(); y < t.y1(); ++y)
            for (size_t x = t.x0(); x < t.x1(); ++x) {
                Ray ray = cam->get_primary_ray(x + 0.5f, y + 0.5f, (float)w, (float)h);
                hit_record_t hr;
                bool hit = ctx.scene.intersection(ray, hr);
                int obj = -1, prim = -1;
                double trep = -1.0;
                if (hit) {
                    for (int k = 0; k < nobj; ++k) if (order[k] == hr.id_object) obj = k;
                    if (have_rep) {
                        hit_record_t rr;
                        const xtcore::OctreeItem<xtcore::surface::Triangle> *it = rep.oct.intersection(ray, &rr);
                        if (it) {
                            prim = (int)it->data.tc[0].x;
                            trep = rr.t;
                        }
                    }
                }
                int xy[2] = {(int)x, (int)y};
                fwrite(xy, 4, 2, f);
                double rec[14] = {ray.origin.x, ray.origin.y, ray.origin.z,
                                  ray.direction.x, ray.direction.y, ray.direction.z,
                                  hit ? hr.t : -1.0, hr.point.x, hr.point.y, hr.point.z,
                                  hr.normal.x, hr.normal.y, hr.normal.z, trep};
                int hi[3] = {hit ? 1 : 0, obj, prim};
                fwrite(hi, 4, 3, f);
                fwrite(rec, 8, 14, f);
            }
    }
    auto t1 = std::chrono::steady_clock::now();
    fclose(f);
    printf("{\"trace_s\": %.9f, \"rays\": %lld}\n", std::chrono::duration<double>(t1 - t0).count(), n);
    return 0;
}

// ---------------------------------------------------------------------------
// Known-answer mode.  Each input line names a reference function and its
// arguments as C99 hex floats; the output line holds the results as hex floats.
static std::vector<double> parse_nums(char *s)
{
    std::vector<double> v;
    char *tok = strtok(s, " \t\n");
    while (tok) { v.push_back(strtod(tok, 0)); tok = strtok(0, " \t\n"); }
    return v;
}

static void put(FILE *f, double x) { fprintf(f, " %a", x); }
static void put3(FILE *f, const Vector3f &v) { put(f, v.x); put(f, v.y); put(f, v.z); }

// samplers loaded by the tex_load / erp_load / cube_load lines
static xtcore::sampler::Texture2D g_tex[16];
static xtcore::sampler::ERP g_erp[4];
static xtcore::sampler::Cubemap g_cube[4];

static int mode_kat(int argc, char **argv)
{
    if (argc < 4) return 2;
    FILE *in = fopen(argv[2], "r"), *out = fopen(argv[3], "w");
    if (!in || !out) return 1;
    xtcore::init();
    xtcore::Log::handle().echo(false);

    // Touch every sampling path once so each translation unit's prng_c has done
    // its one-time srand(time(NULL)) before any srand(seed) below.
    {
        Vector3f n(0, 1, 0);
        xtcore::camera::Perspective lens;   // the thin-lens ray draws in perspective.cc's unit
        lens.position = Vector3f(0, 0, -5);
        lens.target = Vector3f(0, 0, 0);
        lens.up = Vector3f(0, 1, 0);
        lens.fov = 45.f;
        lens.flength = 5.f;
        lens.aperture = 0.5f;
        lens.get_primary_ray(1.f, 1.f, 4.f, 4.f);
        for (int i = 0; i < 4; ++i) {
            nmath::sample::hemisphere(n, n);
            nmath::sample::diffuse(n);
            nmath::sample::lobe(n, Vector3f(0, 1, 1).normalized(), 10.0);
        }
        xtcore::asset::material::Lambert l;
        xtcore::asset::material::Phong p;
        xtcore::asset::material::BlinnPhong b;
        xtcore::hit_result_t r;
        hit_record_t hr;
        hr.normal = n;
        hr.incident_direction = Vector3f(0, -1, 1).normalized();
        for (int i = 0; i < 8; ++i) {
            l.sample_path(r, hr);
            p.sample_path(r, hr);
            b.sample_path(r, hr);
        }
    }

    char line[8192];
    while (fgets(line, sizeof(line), in)) {
        char kind[64];
        if (sscanf(line, "%63s", kind) != 1) continue;
        char raw[8192];
        memcpy(raw, line, sizeof(raw));
        std::vector<double> a = parse_nums(line + strlen(kind));
        fprintf(out, "%s", kind);
        if (!strcmp(kind, "rand")) {
            srand((unsigned)a[0]);
            int n = (int)a[1];
            for (int i = 0; i < n; ++i) fprintf(out, " %d", rand());
            fprintf(out, " %d", RAND_MAX);
        } else if (!strcmp(kind, "camera")) {
            xtcore::camera::Perspective c;
            c.position = Vector3f(a[0], a[1], a[2]);
            c.target = Vector3f(a[3], a[4], a[5]);
            c.up = Vector3f(a[6], a[7], a[8]);
            c.fov = (float)a[9];
            Ray r = c.get_primary_ray((float)a[12], (float)a[13], (float)a[10], (float)a[11]);
            put3(out, r.origin);
            put3(out, r.direction);
        } else if (!strcmp(kind, "camera_dof")) {
            // seed, position, target, up, fov, flength, aperture, w, h, x, y:
            // the thin-lens ray draws two prng_c values (perspective.cc:73-82)
            srand((unsigned)a[0]);
            xtcore::camera::Perspective c;
            c.position = Vector3f(a[1], a[2], a[3]);
            c.target = Vector3f(a[4], a[5], a[6]);
            c.up = Vector3f(a[7], a[8], a[9]);
            c.fov = (float)a[10];
            c.flength = (float)a[11];
            c.aperture = (float)a[12];
            Ray r = c.get_primary_ray((float)a[15], (float)a[16], (float)a[13], (float)a[14]);
            put3(out, r.origin);
            put3(out, r.direction);
        } else if (!strcmp(kind, "camera_erp") || !strcmp(kind, "camera_ods")) {
            // position, orientation, ipd, w, h, x, y
            xtcore::asset::ICamera *c;
            xtcore::camera::ERP erp;
            xtcore::camera::ODS ods;
            if (!strcmp(kind, "camera_erp")) {
                erp.position = Vector3f(a[0], a[1], a[2]);
                erp.orientation = Vector3f(a[3], a[4], a[5]);
                c = &erp;
            } else {
                ods.position = Vector3f(a[0], a[1], a[2]);
                ods.orientation = Vector3f(a[3], a[4], a[5]);
                ods.ipd = (float)a[6];
                c = &ods;
            }
            Ray r = c->get_primary_ray((float)a[9], (float)a[10], (float)a[7], (float)a[8]);
            put3(out, r.origin);
            put3(out, r.direction);
        } else if (!strcmp(kind, "camera_cubemap")) {
            // position, w, h, x, y
            xtcore::camera::Cubemap c;
            c.position = Vector3f(a[0], a[1], a[2]);
            Ray r = c.get_primary_ray((float)a[5], (float)a[6], (float)a[3], (float)a[4]);
            put3(out, r.origin);
            put3(out, r.direction);
        } else if (!strcmp(kind, "sphere")) {
            // Members set directly, as the .scn loader does (parseutil.cc:371-383),
            // so a radius of 0 (a "point" light) is kept.
            xtcore::surface::Sphere s;
            s.origin = Vector3f(a[0], a[1], a[2]);
            s.radius = a[3];
            Ray r;
            r.origin = Vector3f(a[4], a[5], a[6]);
            r.direction = Vector3f(a[7], a[8], a[9]);
            hit_record_t hr;
            bool hit = s.intersection(r, &hr);
            fprintf(out, " %d", hit ? 1 : 0);
            put(out, hr.t); put3(out, hr.point); put3(out, hr.normal);
        } else if (!strcmp(kind, "plane")) {
            xtcore::surface::Plane p;
            p.normal = Vector3f(a[0], a[1], a[2]);
            p.offset = a[3];
            Ray r;
            r.origin = Vector3f(a[4], a[5], a[6]);
            r.direction = Vector3f(a[7], a[8], a[9]);
            hit_record_t hr;
            bool hit = p.intersection(r, &hr);
            fprintf(out, " %d", hit ? 1 : 0);
            put(out, hr.t); put3(out, hr.point); put3(out, hr.normal);
        } else if (!strcmp(kind, "triangle")) {
            xtcore::surface::Triangle t;
            for (int k = 0; k < 3; ++k) t.v[k] = Vector3f(a[3 * k], a[3 * k + 1], a[3 * k + 2]);
            for (int k = 0; k < 3; ++k) t.n[k] = Vector3f(a[9 + 3 * k], a[10 + 3 * k], a[11 + 3 * k]);
            Ray r;
            r.origin = Vector3f(a[18], a[19], a[20]);
            r.direction = Vector3f(a[21], a[22], a[23]);
            hit_record_t hr;
            bool hit = t.intersection(r, &hr);
            fprintf(out, " %d", hit ? 1 : 0);
            put(out, hr.t); put3(out, hr.point); put3(out, hr.normal);
        } else if (!strcmp(kind, "aabb")) {
            xtcore::AABB3 b(Vector3f(a[0], a[1], a[2]), Vector3f(a[3], a[4], a[5]));
            Ray r;
            r.origin = Vector3f(a[6], a[7], a[8]);
            r.direction = Vector3f(a[9], a[10], a[11]);
            fprintf(out, " %d", b.intersection(r) ? 1 : 0);
        } else if (!strcmp(kind, "hemisphere")) {
            srand((unsigned)a[0]);
            Vector3f n(a[1], a[2], a[3]);
            put3(out, nmath::sample::hemisphere(n, n));
        } else if (!strcmp(kind, "diffuse")) {
            srand((unsigned)a[0]);
            put3(out, nmath::sample::diffuse(Vector3f(a[1], a[2], a[3])));
        } else if (!strcmp(kind, "lobe")) {
            srand((unsigned)a[0]);
            put3(out, nmath::sample::lobe(Vector3f(a[1], a[2], a[3]), Vector3f(a[4], a[5], a[6]), a[7]));
        } else if (!strcmp(kind, "material")) {
            // material <type 0 lambert,1 phong,2 blinn,3 emissive> seed diffuse3 specular3 emissive3
            //          reflectance exponent  point3 normal3 incident3
            int type = (int)a[0];
            xtcore::asset::IMaterial *m = 0;
            if (type == 0) m = new xtcore::asset::material::Lambert();
            if (type == 1) m = new xtcore::asset::material::Phong();
            if (type == 2) m = new xtcore::asset::material::BlinnPhong();
            if (type == 3) m = new xtcore::asset::material::Emissive();
            nimg::ColorRGBf cd((float)a[2], (float)a[3], (float)a[4]);
            nimg::ColorRGBf cs((float)a[5], (float)a[6], (float)a[7]);
            nimg::ColorRGBf ce((float)a[8], (float)a[9], (float)a[10]);
            xtcore::sampler::SolidColor *sd = new xtcore::sampler::SolidColor(); sd->set(cd);
            xtcore::sampler::SolidColor *ss = new xtcore::sampler::SolidColor(); ss->set(cs);
            xtcore::sampler::SolidColor *se = new xtcore::sampler::SolidColor(); se->set(ce);
            m->add_sampler("diffuse", sd);
            m->add_sampler("specular", ss);
            m->add_sampler("emissive", se);
            m->add_scalar("reflectance", (float)a[11]);
            m->add_scalar("exponent", (float)a[12]);
            hit_record_t hr;
            hr.point = Vector3f(a[13], a[14], a[15]);
            hr.normal = Vector3f(a[16], a[17], a[18]);
            hr.incident_direction = Vector3f(a[19], a[20], a[21]);
            xtcore::hit_result_t res;
            srand((unsigned)a[1]);
            bool cont = m->sample_path(res, hr);
            fprintf(out, " %d", cont ? 1 : 0);
            put3(out, res.ray.origin);
            put3(out, res.ray.direction);
            put(out, res.intensity.r()); put(out, res.intensity.g()); put(out, res.intensity.b());
            delete m;
        } else if (!strcmp(kind, "tex_load")) {
            // tex_load slot filtering flip_x flip_y path: Texture2D as
            // deserialize_texture sets it up (parseutil.cc:478-508)
            int slot, filt, fx, fy;
            char path[4096];
            if (sscanf(raw + strlen(kind), "%d %d %d %d %4095s", &slot, &filt, &fx, &fy, path) != 5 || slot < 0 ||
                slot >= 16) {
                fprintf(out, " bad");
            } else {
                g_tex[slot] = xtcore::sampler::Texture2D();
                int r = g_tex[slot].load(path);
                g_tex[slot].set_filtering(filt ? xtcore::sampler::FILTERING_BILINEAR
                                               : xtcore::sampler::FILTERING_NEAREST);
                if (fx) g_tex[slot].flip_horizontal();
                if (fy) g_tex[slot].flip_vertical();
                fprintf(out, " %d", r);
            }
        } else if (!strcmp(kind, "tex_sample")) {
            nimg::ColorRGBf c = g_tex[(int)a[0] & 15].sample(Vector3f(a[1], a[2], 0));
            put(out, c.r()); put(out, c.g()); put(out, c.b());
        } else if (!strcmp(kind, "erp_load")) {
            int slot;
            char path[4096];
            if (sscanf(raw + strlen(kind), "%d %4095s", &slot, path) != 2 || slot < 0 || slot >= 4) {
                fprintf(out, " bad");
            } else {
                fprintf(out, " %d", g_erp[slot].load(path));
            }
        } else if (!strcmp(kind, "erp_sample")) {
            nimg::ColorRGBf c = g_erp[(int)a[0] & 3].sample(Vector3f(a[1], a[2], a[3]));
            put(out, c.r()); put(out, c.g()); put(out, c.b());
        } else if (!strcmp(kind, "cube_load")) {
            // cube_load slot left right top bottom front back
            int slot;
            char p[6][1024];
            if (sscanf(raw + strlen(kind), "%d %1023s %1023s %1023s %1023s %1023s %1023s", &slot, p[0], p[1], p[2],
                       p[3], p[4], p[5]) != 7 || slot < 0 || slot >= 4) {
                fprintf(out, " bad");
            } else {
                for (int f = 0; f < 6; ++f)
                    fprintf(out, " %d", g_cube[slot].load(p[f], (xtcore::sampler::CUBEMAP_FACE)f));
            }
        } else if (!strcmp(kind, "cube_sample")) {
            nimg::ColorRGBf c = g_cube[(int)a[0] & 3].sample(Vector3f(a[1], a[2], a[3]));
            put(out, c.r()); put(out, c.g()); put(out, c.b());
        } else if (!strcmp(kind, "gradient")) {
            xtcore::sampler::Gradient g;
            g.a = nimg::ColorRGBf((float)a[0], (float)a[1], (float)a[2]);
            g.b = nimg::ColorRGBf((float)a[3], (float)a[4], (float)a[5]);
            nimg::ColorRGBf c = g.sample(Vector3f(a[6], a[7], a[8]));
            put(out, c.r()); put(out, c.g()); put(out, c.b());
        } else {
            fprintf(out, " unknown");
        }
        fprintf(out, "\n");
    }
    fclose(in);
    fclose(out);
    return 0;
}

static int mode_bench(int argc, char **argv)
{
    if (argc < 12) return 2;
    const char *scn = argv[2];
    std::string integ = argv[3];
    size_t w = atol(argv[4]), h = atol(argv[5]), spp = atol(argv[6]);
    size_t rdepth = atol(argv[7]), threads = atol(argv[8]);
    g_fixed_time = (time_t)atoll(argv[9]);
    const char *tiles_path = argv[10];
    int repeats = atoi(argv[11]);
    if (repeats < 1) return 2;

    xtcore::init();
    xtcore::render::context_t ctx;
    auto l0 = std::chrono::steady_clock::now();
    if (load_scene(ctx, scn)) return 1;
    double load_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - l0).count();
    HASH_UINT64 cam = ctx.params.camera;
    ctx.params.width = w;
    ctx.params.height = h;
    ctx.params.samples = spp;
    ctx.params.aa = 1;
    ctx.params.rdepth = rdepth;
    ctx.params.threads = threads;
    ctx.params.camera = cam;
    if (!read_tiles(tiles_path, w, h, ctx.tiles)) {
        fprintf(stderr, "xtref: bad tiles %s\n", tiles_path);
        return 1;
    }
    xtcore::render::IIntegrator *ig = make_integrator(integ, 100.0f);
    if (!ig) { fprintf(stderr, "xtref: unknown integrator %s\n", integ.c_str()); return 1; }
    ig->setup(ctx);
    printf("{\"load_s\": %.9f, \"threads\": %d, \"renders\": [", load_s,
           threads ? (int)threads : omp_get_max_threads());
    for (int r = 0; r < repeats; ++r) {
        g_rays = 0;
        auto t0 = std::chrono::steady_clock::now();
        ig->render();
        double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        printf("%s{\"render_s\": %.9f, \"rays\": %llu}", r ? ", " : "", secs, (unsigned long long)g_rays.load());
    }
    printf("]}\n");
    delete ig;
    return 0;
}

int main(int argc, char **argv)
{
    if (argc < 2) {
        fprintf(stderr, "usage: xtref render|hits|kat|bench ...\n");
        return 2;
    }
    std::string m = argv[1];
    int rc = 2;
    if (m == "render") rc = mode_render(argc, argv);
    else if (m == "hits") rc = mode_hits(argc, argv);
    else if (m == "kat") rc = mode_kat(argc, argv);
    else if (m == "bench") rc = mode_bench(argc, argv);
    if (rc == 2) fprintf(stderr, "xtref: bad arguments\n");
    return rc;
}
