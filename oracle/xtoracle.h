/*
 * xtoracle — CPU restatement of XTracer's ray-scene intersection and integrator
 * hot path, in FP64 like the reference (lib/nmath/precision.h:45-80).
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that the GPU path is compared
 * against; it is never called by the product library.  It is pinned against the
 * reference itself: tests/golden/ holds known-answer vectors and renders made by
 * the reference's own code (oracle/ref_driver.cc, built by oracle/ref.mk), and
 * tests/test_oracle_golden.py checks this file against them.
 *
 * Every function cites the reference file:line it restates.  File paths are
 * relative to the XTracer source tree.
 */
#ifndef XTORACLE_H
#define XTORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { XO_SPHERE = 0, XO_PLANE = 1, XO_MESH = 2 };
enum { XO_LAMBERT = 0, XO_PHONG = 1, XO_BLINNPHONG = 2, XO_EMISSIVE = 3, XO_DIELECTRIC = 4 };
enum { XO_ENV_NONE = 0, XO_ENV_COLOR = 1, XO_ENV_GRADIENT = 2, XO_ENV_ERP = 3, XO_ENV_CUBEMAP = 4 };
/* material samplers (sampler_col.cc, sampler_gradient.cc, sampler_tex.cc,
 * sampler_erp.cc, sampler_cubemap.cc); texture filtering (sampler.h:11-15) */
enum { XO_SAMPLER_COLOR = 0, XO_SAMPLER_GRADIENT = 1, XO_SAMPLER_TEXTURE = 2, XO_SAMPLER_ERP = 3,
       XO_SAMPLER_CUBEMAP = 4 };
enum { XO_FILTER_NEAREST = 0, XO_FILTER_BILINEAR = 1 };
enum { XO_STENCIL = 0, XO_DEPTH = 1, XO_AO = 2, XO_PATHTRACER = 3,
       XO_NORMAL = 4, XO_UV = 5, XO_EMISSION = 6, XO_WIREFRAME = 7 };
/* mesh intersector: 0 = octree restatement (exact reference order), 1 = FP64 BVH
 * with the reference's triangle test (same closest hit except exact t ties). */
enum { XO_ACCEL_OCTREE = 0, XO_ACCEL_BVH = 1 };
/* random source: 0 = table of libc rand() values (known-answer tests),
 * 1 = the counter stream shared with the GPU path (SplitMix64 of key+counter). */
enum { XO_RNG_TABLE = 0, XO_RNG_STREAM = 1 };
/* cameras (src/xtcore/camera/): thin-lens perspective, equirectangular,
 * omni-directional stereo, cubemap vertical strip */
enum { XO_CAM_PERSPECTIVE = 0, XO_CAM_ERP = 1, XO_CAM_ODS = 2, XO_CAM_CUBEMAP = 3 };

typedef struct {
    int32_t type;
    float diffuse[3], specular[3], emissive[3];
    float reflectance, exponent, ior;
} xo_material;

/* A loaded Texture2D: its Pixmap (RGBA float per texel, rows top first, as
 * nimg::io::load::image fills it after the flips) and its filtering. */
typedef struct {
    int32_t width, height, filtering, pad;
    int64_t offset;              /* first texel in xo_scene_desc::texels */
} xo_texture;

/* A material sampler: COLOR a; GRADIENT a, b; TEXTURE and ERP one texture;
 * CUBEMAP six consecutive textures in CUBEMAP_FACE order (left, right, top,
 * bottom, front, back; sampler_cubemap.h:11-19). */
typedef struct {
    int32_t kind, texture;
    float a[3], b[3];
} xo_sampler;

typedef struct {
    int32_t n_objects;
    const int32_t *obj_kind;     /* XO_SPHERE / XO_PLANE / XO_MESH */
    const int32_t *obj_first;    /* sphere index, plane index or first triangle */
    const int32_t *obj_count;    /* triangles of a mesh (1 for sphere/plane) */
    const int32_t *obj_material;
    int32_t n_spheres;
    const float *spheres;        /* cx cy cz r */
    int32_t n_planes;
    const float *planes;         /* nx ny nz offset */
    int32_t n_tris;
    const float *tris;           /* 9 floats per triangle */
    const float *tri_normals;    /* 9 floats per triangle, or NULL */
    int32_t n_materials;
    const xo_material *materials;
    int32_t env_type;
    float env_a[3], env_b[3];
    float cam_pos[3], cam_target[3], cam_up[3];
    float cam_fov;
    const float *obj_uv_scale;   /* 2 floats per object (ISurface::uv_scale), or NULL = (0, 0),
                                    what the loader sets without uscale/vscale */
    const float *tri_uvs;        /* 6 floats per triangle (Triangle::tc[0..2].xy), or NULL = the
                                    Triangle constructor's (0,0) (1,0) (0,0), triangle.cc:8-13 */
    int32_t cam_type;            /* XO_CAM_* */
    float cam_orientation[3];    /* ERP, ODS: euler angles (Matrix4x4f::rotate) */
    float cam_ipd;               /* ODS */
    float cam_flength, cam_aperture;   /* perspective: depth of field when flength > 0 */
    int32_t n_textures;
    const xo_texture *textures;
    const float *texels;         /* 4 floats (r g b a) per texel */
    const xo_sampler *mat_samplers;    /* 3 per material (diffuse, specular, emissive), or
                                          NULL = the materials' colours */
    int32_t env_texture;         /* XO_ENV_ERP: its texture; XO_ENV_CUBEMAP: the first of six */
} xo_scene_desc;

typedef struct xo_scene xo_scene;

int  xo_scene_create(const xo_scene_desc *desc, int accel, xo_scene **out);
void xo_scene_destroy(xo_scene *s);

/* Closest hit of n rays (Scene::intersection, scene.cc:191-216).  Per ray:
 * hit (0/1), t, object index, primitive index (triangle index for meshes, sphere
 * or plane index otherwise), point and normal. */
void xo_trace(const xo_scene *s, int64_t n, const double *org, const double *dir,
              int32_t *hit, double *t, int32_t *obj, int32_t *prim, double *point, double *normal);

/* Primary ray of the pinhole camera (Perspective::get_primary_ray,
 * camera/perspective.cc:38-98, flength = 0). */
void xo_camera_ray(const float pos[3], const float target[3], const float up[3], float fov,
                   float x, float y, float w, float h, double org[3], double dir[3]);

typedef struct {
    int32_t integrator;    /* XO_STENCIL .. XO_WIREFRAME */
    int32_t width, height, spp, rdepth;
    int32_t aa;            /* anti-aliasing level; grid (aa.cc:7-32): 0 or 1 = pixel centre */
    float ao_max_distance; /* 100 in the shipped AO integrator */
    uint64_t seed;         /* XO_RNG_STREAM key */
    int32_t distribution;  /* XO_SAMPLES_GRID or XO_SAMPLES_RANDOM (aa.h SAMPLE_DISTRIBUTION) */
} xo_render_params;

/* Sample distributions (aa.cc:7-48).  RANDOM takes aa positions per pixel at
 * offsets drawn from a stream keyed by (seed ^ XO_JITTER_SALT, position,
 * pixel) where the reference draws libc rand(). */
enum { XO_SAMPLES_GRID = 0, XO_SAMPLES_RANDOM = 1 };
#define XO_JITTER_SALT 0xA0761D6478BD642FULL

/* Renders the listed pixels (x,y pairs): aa^2 grid positions per pixel, each
 * taken `spp` times with weight 1/(aa^2 spp) (aa.cc:7-32, 51-77).  Output RGBA
 * per listed pixel; *rays = number of Scene::intersection calls. */
int xo_render(const xo_scene *s, const xo_render_params *p, int64_t npix, const int32_t *px,
              float *rgba, uint64_t *rays);
/* The depth integrator (whatever p->integrator says) recording its raygraph:
 * 10 doubles per sample (origin, hit point, colour after the sample), pixels
 * in px order, each pixel's samples in order. */
int xo_render_raygraph(const xo_scene *s, const xo_render_params *p, int64_t npix, const int32_t *px,
                       float *rgba, double *raygraph, uint64_t *rays);

/* Known-answer hooks for single reference functions.  `table` holds libc rand()
 * values (consumed in order) and rand_max their RAND_MAX. */
int  xo_kat_sphere(const double sph[4], const double o[3], const double d[3], double out[7]);
int  xo_kat_plane(const double pl[4], const double o[3], const double d[3], double out[7]);
int  xo_kat_triangle(const double v[9], const double n[9], const double o[3], const double d[3], double out[7]);
int  xo_kat_aabb(const double mn[3], const double mx[3], const double o[3], const double d[3]);
void xo_kat_hemisphere(const int32_t *table, int32_t rand_max, const double n[3], double out[3]);
void xo_kat_diffuse(const int32_t *table, int32_t rand_max, const double n[3], double out[3]);
void xo_kat_lobe(const int32_t *table, int32_t rand_max, const double n[3], const double d[3], double e, double out[3]);
int  xo_kat_material(const xo_material *m, const int32_t *table, int32_t rand_max, const double p[3],
                     const double n[3], const double inc[3], double out[9]);
void xo_kat_gradient(const float a[3], const float b[3], const double d[3], float out[3]);
/* Texture2D::sample (sampler_tex.cc:37-45: nimg::sample::nearest / bilinear),
 * ERP::sample (sampler_erp.cc:13-26) and Cubemap::sample (sampler_cubemap.cc:
 * 13-36) on textures of the given layout; faces: six textures. */
void xo_kat_texture(const xo_texture *t, const float *texels, double u, double v, float out[3]);
void xo_kat_erp(const xo_texture *t, const float *texels, const double d[3], float out[3]);
void xo_kat_cubemap(const xo_texture *faces, const float *texels, const double d[3], float out[3]);

/* Camera rays of every camera type, known-answer hooks: perspective with depth
 * of field (the two prng_c draws from `table`), equirectangular, ODS, cubemap. */
void xo_kat_camera_dof(const int32_t *table, int32_t rand_max, const float pos[3], const float target[3],
                       const float up[3], float fov, float flength, float aperture, float x, float y, float w,
                       float h, double org[3], double dir[3]);
void xo_kat_camera_erp(const float pos[3], const float orient[3], float x, float y, float w, float h,
                       double org[3], double dir[3]);
void xo_kat_camera_ods(const float pos[3], const float orient[3], float ipd, float x, float y, float w, float h,
                       double org[3], double dir[3]);
void xo_kat_camera_cubemap(const float pos[3], float x, float y, float w, float h, double org[3], double dir[3]);

/* The counter stream shared with the GPU path, exposed for tests. */
double xo_stream_uniform(uint64_t key, uint32_t counter);
uint64_t xo_path_key(uint64_t seed, uint64_t path);
/* Key of the random distribution's offsets of one position of one pixel. */
uint64_t xo_jitter_key(uint64_t seed, int32_t position, int32_t width, int32_t height, int32_t x, int32_t y);

#ifdef __cplusplus
}
#endif
#endif
