/*
 * xtgpu.h — C ABI of the B200 ray-scene intersection and integrator backend for
 * XTracer (4rknova/xtracer).
 *
 * XTracer's C++ host (the .scn loader, Scene, IIntegrator, tiles, image output)
 * stays as it is.  A GPU integrator (an IIntegrator subclass built into
 * XTracer's tree) flattens the loaded Scene into an xtgpu_scene_desc and calls
 * the entry points below.  Plain
 * pointers and sizes only; every call returns an xtgpu_status and never throws;
 * xtgpu_last_error() gives the text of the last failure on the calling thread.
 *
 * Reference interfaces replaced (paths relative to the XTracer source tree):
 *   xtgpu_scene_create     the Scene built by io::scn::load
 *                          (src/xtcore/parseutil.cc:697-822, scene.h:35-86):
 *                          objects, surfaces, materials, environment, camera
 *   xtgpu_bvh_build        Mesh::build_octree / Octree<Triangle>::build
 *                          (src/xtcore/mesh.cc:70-113, octree.tml:118-198)
 *   xtgpu_trace            Scene::intersection (src/xtcore/scene.cc:191-216)
 *                          over a batch of rays, including the per-mesh
 *                          Octree::r_intersection (octree.tml:206-249)
 *   xtgpu_render           IIntegrator::render + render_tile of the stencil,
 *                          depth, ao and pathtracer integrators
 *                          (src/xtcore/integrator.cc:29-53,
 *                          integrator/{stencil,depth,ao,pathtracer}/integrator.cc)
 *   xtgpu_service_*        no reference counterpart: a persistent render
 *                          service (resident scenes, memory-budget admission,
 *                          merged wavefront launches in CUDA graphs)
 *
 * Device pointers are CUDA global-memory pointers on the current device;
 * `stream` is a cudaStream_t (NULL = legacy default stream).
 */
#ifndef XTGPU_H
#define XTGPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define XTGPU_API __attribute__((visibility("default")))
#else
#define XTGPU_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    XTGPU_OK = 0,
    XTGPU_ERR_INVALID = 1,   /* bad argument: NULL handle, size out of range, bad enum */
    XTGPU_ERR_CUDA = 2,      /* a CUDA runtime call failed */
    XTGPU_ERR_NOMEM = 3,     /* device allocation failed or a memory budget is exceeded */
    XTGPU_ERR_LIMIT = 4,     /* a fixed capacity was exceeded (traversal stack, queue) */
    XTGPU_ERR_TIMEOUT = 5,   /* a bounded wait expired */
    XTGPU_ERR_NOT_FOUND = 6, /* unknown job or scene id */
    XTGPU_ERR_STATE = 7      /* call not valid in the object's current state */
} xtgpu_status;

/* Surface kinds (src/xtcore/math/{sphere,plane}.cc, mesh.cc). */
enum { XTGPU_SPHERE = 0, XTGPU_PLANE = 1, XTGPU_MESH = 2 };
/* Materials (src/xtcore/material/, names in matdefs.h:4-12). */
enum { XTGPU_LAMBERT = 0, XTGPU_PHONG = 1, XTGPU_BLINNPHONG = 2, XTGPU_EMISSIVE = 3, XTGPU_DIELECTRIC = 4 };
/* Environment samplers (sampler_col.cc, sampler_gradient.cc, sampler_erp.cc,
 * sampler_cubemap.cc); none = black (scene.cc:142-145). */
enum { XTGPU_ENV_NONE = 0, XTGPU_ENV_COLOR = 1, XTGPU_ENV_GRADIENT = 2, XTGPU_ENV_ERP = 3, XTGPU_ENV_CUBEMAP = 4 };
/* Material samplers (IMaterial::get_sample, material.cc:65-70, at the hit's
 * texcoord) and texture filtering (sampler.h:11-15). */
enum { XTGPU_SAMPLER_COLOR = 0, XTGPU_SAMPLER_GRADIENT = 1, XTGPU_SAMPLER_TEXTURE = 2, XTGPU_SAMPLER_ERP = 3,
       XTGPU_SAMPLER_CUBEMAP = 4 };
enum { XTGPU_FILTER_NEAREST = 0, XTGPU_FILTER_BILINEAR = 1 };
/* Cameras (src/xtcore/camera/): thin-lens perspective, equirectangular,
 * omni-directional stereo (upper half one eye, lower the other), cubemap
 * vertical strip (faces +x -x +y -y +z -z, height a multiple of 6). */
enum { XTGPU_CAM_PERSPECTIVE = 0, XTGPU_CAM_ERP = 1, XTGPU_CAM_ODS = 2, XTGPU_CAM_CUBEMAP = 3 };
/* Sample distributions (aa.h:14-18, aa.cc:7-48): GRID takes aa^2 positions per
 * pixel on a regular grid of weight 1/aa^2; RANDOM takes aa positions of weight
 * 1/aa, each at offsets in [0,1)^2 from the pixel corner drawn from a random
 * stream keyed by (seed, position, pixel) where the reference draws libc
 * rand().  Either way each position is taken spp times at 1/spp. */
enum { XTGPU_SAMPLES_GRID = 0, XTGPU_SAMPLES_RANDOM = 1 };
/* Integrators. */
enum { XTGPU_STENCIL = 0, XTGPU_DEPTH = 1, XTGPU_AO = 2, XTGPU_PATHTRACER = 3,
       /* primary-ray integrators (integrator/{normal,uv,emission,wireframe}) */
       XTGPU_NORMAL = 4, XTGPU_UV = 5, XTGPU_EMISSION = 6, XTGPU_WIREFRAME = 7 };
#define XTGPU_INTEGRATOR_LAST XTGPU_WIREFRAME
/* BVH node formats: binary nodes with 64-byte FP32 child boxes or 32-byte
 * boxes quantised to 8 bits per bound with outward rounding; or 8-wide nodes
 * (80 bytes) with 8-bit quantised child boxes, collapsed from the binary tree
 * (leaves of at most 3 primitives). */
enum { XTGPU_NODES_FP32 = 0, XTGPU_NODES_Q8 = 1, XTGPU_NODES_W8 = 2 };

typedef struct {
    int32_t type;                  /* XTGPU_LAMBERT ... */
    float diffuse[3], specular[3], emissive[3];
    float reflectance, exponent, ior;
} xtgpu_material;

typedef struct {
    float position[3], target[3], up[3];
    float fov;                     /* degrees, horizontal (perspective.cc:48-50) */
    int32_t type;                  /* XTGPU_CAM_PERSPECTIVE (default) .. XTGPU_CAM_CUBEMAP */
    float orientation[3];          /* ERP, ODS: euler angles in radians (Matrix4x4f::rotate) */
    float ipd;                     /* ODS: inter-pupillary distance (ods.cc:20-23) */
    float flength, aperture;       /* perspective: depth of field when flength > 0
                                      (perspective.cc:73-95); lens draws come first on
                                      each sample's random stream */
} xtgpu_camera;

/* A loaded Texture2D (sampler_tex.h:14-37): its Pixmap as RGBA floats, rows
 * top first, after the loader's flips, and its filtering. */
typedef struct {
    int32_t width, height;
    int32_t filtering;             /* XTGPU_FILTER_NEAREST / XTGPU_FILTER_BILINEAR */
    int32_t reserved;
    int64_t offset;                /* first texel in xtgpu_scene_desc::texels */
} xtgpu_texture;

/* A sampler: COLOR a; GRADIENT a, b (over the normalised texcoord); TEXTURE
 * and ERP one texture; CUBEMAP six consecutive textures in CUBEMAP_FACE order
 * (left, right, top, bottom, front, back; sampler_cubemap.h:11-19). */
typedef struct {
    int32_t kind;                  /* XTGPU_SAMPLER_* */
    int32_t texture;
    float a[3], b[3];
} xtgpu_sampler;

/* A flattened Scene.  Objects are listed in the order Scene::intersection
 * visits them (the std::map order of their ids).  Host pointers; copied. */
typedef struct {
    int32_t n_objects;
    const int32_t *obj_kind;       /* XTGPU_SPHERE / XTGPU_PLANE / XTGPU_MESH */
    const int32_t *obj_first;      /* sphere index, plane index, or first triangle */
    const int32_t *obj_count;      /* triangle count of a mesh, 1 otherwise */
    const int32_t *obj_material;   /* index into materials */
    int32_t n_spheres;
    const float *spheres;          /* 4 floats each: centre xyz, radius */
    int32_t n_planes;
    const float *planes;           /* 4 floats each: normal xyz, offset */
    int32_t n_tris;
    const float *tris;             /* 9 floats each: v0 v1 v2 */
    const float *tri_normals;      /* 9 floats each, or NULL (face normals) */
    int32_t n_materials;
    const xtgpu_material *materials;
    int32_t env_type;
    float env_a[3], env_b[3];
    xtgpu_camera camera;
    const float *obj_uv_scale;     /* 2 floats per object: the surface's uv_scale (u_scale,
                                      v_scale), or NULL = (0, 0), the loader's default */
    const float *tri_uvs;          /* 6 floats per triangle: texcoords of its corners (OBJ vt),
                                      or NULL = the Triangle constructor's (0,0) (1,0) (0,0) */
    int32_t n_textures;
    const xtgpu_texture *textures;
    int64_t n_texels;
    const float *texels;           /* 4 floats (r g b a) per texel */
    const xtgpu_sampler *mat_samplers;  /* 3 per material (diffuse, specular, emissive), or
                                           NULL = the materials' colours */
    int32_t env_texture;           /* XTGPU_ENV_ERP: its texture; XTGPU_ENV_CUBEMAP: the first
                                      of its six faces */
} xtgpu_scene_desc;

typedef struct xtgpu_scene xtgpu_scene;

typedef struct {
    int32_t node_format;           /* XTGPU_NODES_FP32 or XTGPU_NODES_Q8 */
    int32_t leaf_size;             /* primitives per leaf, 1..4 (0 = default 2) */
} xtgpu_bvh_opts;

/* Uploads the scene (geometry, materials, camera) to the current device. */
XTGPU_API xtgpu_status xtgpu_scene_create(const xtgpu_scene_desc *desc, void *stream, xtgpu_scene **out);
/* Re-uploads the parts of a scene that need no BVH rebuild, from a
 * description of the same geometry (an edited Scene, or one loaded with other
 * -mod values): XTGPU_UPDATE_SHADING replaces the materials, their samplers,
 * the textures, the objects' materials, the u/v scales and triangle texcoords
 * (texturing only) and the environment; XTGPU_UPDATE_CAMERA
 * the camera.  Geometry fields are ignored.  Work on `stream` is waited for;
 * renders of the scene on other streams must have finished.  A service that
 * holds the scene sees the change after xtgpu_service_update_scene. */
enum { XTGPU_UPDATE_SHADING = 1, XTGPU_UPDATE_CAMERA = 2 };
XTGPU_API xtgpu_status xtgpu_scene_update(xtgpu_scene *scene, const xtgpu_scene_desc *desc, int32_t what,
                                          void *stream);
/* Builds the scene's LBVH on the device: 30-bit Morton codes, in-house radix
 * sort, Karras hierarchy, bottom-up refit, optional 8-bit quantisation.  Both
 * node formats can be built and kept; the last one built is used by default. */
XTGPU_API xtgpu_status xtgpu_bvh_build(xtgpu_scene *scene, const xtgpu_bvh_opts *opts, void *stream);
/* Frees every device buffer of the scene. */
XTGPU_API xtgpu_status xtgpu_scene_destroy(xtgpu_scene *scene);
/* Bytes of device memory the scene holds (geometry + built BVHs). */
XTGPU_API xtgpu_status xtgpu_scene_device_bytes(const xtgpu_scene *scene, uint64_t *bytes);

/* BVH statistics and intermediate build arrays, copied to host memory (any
 * pointer may be NULL).  morton/order: n_prims each (sorted codes, sorted
 * primitive ids); left/right: n_prims-1 each, Karras child references
 * (>= 0 internal node, < 0 leaf ~index); depth: maximum root-to-leaf depth. */
typedef struct {
    int64_t n_prims;               /* triangles + spheres (planes are tested apart) */
    int32_t depth;
    int32_t leaf_size;
    uint64_t node_bytes_fp32, node_bytes_q8;
    uint64_t node_bytes_w8;        /* 8-wide nodes (0 if not built) */
    int32_t depth_w8;              /* levels of the 8-wide tree */
} xtgpu_bvh_info;
XTGPU_API xtgpu_status xtgpu_bvh_export(const xtgpu_scene *scene, xtgpu_bvh_info *info, uint32_t *morton,
                              uint32_t *order, int32_t *left, int32_t *right, void *stream);

/* Ray batch in device memory, structure of arrays of float4:
 *   org_tmin[i] = (origin.xyz, tmin), dir_tmax[i] = (direction.xyz, tmax)
 * Hit output per ray: t (inf on a miss), primitive id (triangles 0..T-1, then
 * spheres T..T+S-1, then planes), barycentric u, v of the hit triangle.
 * Primitive ids follow the desc arrays, so the object of a hit is found from
 * obj_first/obj_count. */
typedef struct {
    float t;
    uint32_t prim;
    float u, v;
} xtgpu_hit;

/* Closest hit of n rays: Scene::intersection semantics (nearest hit over every
 * object; spheres hit only from outside, planes from both sides).  node_format
 * picks the BVH to traverse (it must have been built). */
XTGPU_API xtgpu_status xtgpu_trace(xtgpu_scene *scene, int64_t n, const void *org_tmin_dev, const void *dir_tmax_dev,
                         xtgpu_hit *hits_dev, int32_t node_format, void *stream);
/* xtgpu_trace with a counting traversal: also returns the BVH nodes visited
 * (counts[0]) and primitives tested (counts[1]) summed over the batch, the
 * per-ray figures behind the extend kernel's algorithmic bytes. */
XTGPU_API xtgpu_status xtgpu_trace_counts(xtgpu_scene *scene, int64_t n, const void *org_tmin_dev,
                                          const void *dir_tmax_dev, xtgpu_hit *hits_dev, int32_t node_format,
                                          uint64_t counts[2], void *stream);
/* The same with host buffers (pinned or pageable), copies included. */
XTGPU_API xtgpu_status xtgpu_trace_host(xtgpu_scene *scene, int64_t n, const float *org_tmin, const float *dir_tmax,
                              xtgpu_hit *hits, int32_t node_format, void *stream);

typedef struct {
    int32_t integrator;            /* XTGPU_STENCIL .. XTGPU_WIREFRAME */
    int32_t width, height;         /* frame size (params_t, context.h:18-34) */
    int32_t spp;                   /* samples per pixel, weight 1/spp each (aa.cc:66-74) */
    int32_t rdepth;                /* pathtracer recursion depth */
    float ao_max_distance;         /* AO: 100 in the shipped integrator (ao/integrator.cc:10) */
    uint64_t seed;                 /* random stream key: results depend only on (seed, pixel, sample) */
    int32_t node_format;           /* BVH to traverse */
    int32_t x0, y0, x1, y1;        /* pixel rectangle to render; x1 = y1 = 0 means the whole frame */
    int32_t aa;                    /* anti-aliasing level (params_t::aa): grid, 0..16, 0 or 1 =
                                      the pixel centre (aa.cc:7-32); random, 0..256 */
    int32_t sample_distribution;   /* XTGPU_SAMPLES_GRID (0) or XTGPU_SAMPLES_RANDOM
                                      (params_t::sample_distribution, aa.h:14-18) */
} xtgpu_render_params;

/* Renders the rectangle and writes RGBA float per pixel of the rectangle
 * (row-major) into rgba_dev (device memory).  Each pixel takes P positions
 * of the sample distribution (aa^2 on the grid, aa random), each spp times,
 * of weight 1/(P spp) (aa.cc:51-77).
 * rays_traced (optional, host) receives the number of rays traced. */
XTGPU_API xtgpu_status xtgpu_render(xtgpu_scene *scene, const xtgpu_render_params *params, float *rgba_dev,
                          uint64_t *rays_traced, void *stream);
/* The same into host memory (copy included). */
XTGPU_API xtgpu_status xtgpu_render_host(xtgpu_scene *scene, const xtgpu_render_params *params, float *rgba_host,
                               uint64_t *rays_traced, void *stream);
/* The depth integrator recording its raygraph (depth/integrator.cc:43-51),
 * which the GUI exports as PLY: params->integrator must be XTGPU_DEPTH.
 * raygraph_dev receives 10 floats per sample: the ray origin, the hit point
 * ((0,0,0) on a miss) and the pixel's RGBA after the sample; rectangle pixels
 * row-major, each pixel's positions x spp samples in order. */
XTGPU_API xtgpu_status xtgpu_render_raygraph(xtgpu_scene *scene, const xtgpu_render_params *params, float *rgba_dev,
                                             float *raygraph_dev, uint64_t *rays_traced, void *stream);
XTGPU_API xtgpu_status xtgpu_render_raygraph_host(xtgpu_scene *scene, const xtgpu_render_params *params,
                                                  float *rgba_host, float *raygraph_host, uint64_t *rays_traced,
                                                  void *stream);
/* raygraph::write (util/raygraph.cc:8-75): n_paths two-vertex paths as ASCII
 * PLY, records (10 floats each, as above) in the order they are listed. */
XTGPU_API xtgpu_status xtgpu_write_raygraph_ply(const char *path, int64_t n_paths, const float *records);

/* xtgpu_render for one rectangle without allocating any memory.  No
 * counterpart in the reference.  For callers that cannot allocate device
 * memory at render time: a render_tile on XTracer's OpenMP tile threads, where
 * a cudaMalloc would synchronise the device and stall every other tile; a
 * process that reserved its device memory at start-up under a fixed budget (or
 * leaves it to another allocator); a render loop that must not meet an
 * allocation failure mid-frame.  Scratch is one static device array of about
 * 11.5 MB held by every GPU that loads the library; a call renders at most
 * XTGPU_NOALLOC_MAX_PATHS paths (rectangle pixels x positions x spp) and larger requests
 * return XTGPU_ERR_LIMIT.  Calls that overlap on the GPU race on the shared
 * array.  The first call on a device looks up the array's address; make it
 * before any stream capture.  Every call copies its job from host memory and
 * waits for `stream` before it returns; a stream that is capturing is refused
 * (XTGPU_ERR_STATE).  Output: rgba_dev as in xtgpu_render. */
#define XTGPU_NOALLOC_MAX_PATHS 65536
XTGPU_API xtgpu_status xtgpu_render_tile_noalloc(xtgpu_scene *scene, const xtgpu_render_params *params,
                                                 float *rgba_dev, uint64_t *rays_traced, void *stream);

/* ---------------------------------------------------------------------- */
/* Output side (lib/nimg/img.cc:72-179, the save::png and save::exr writers
 * fed by context.cc:38-52 assemble).  The frame is width*height RGBA floats,
 * row-major, as xtgpu_render writes it. */
/* 8-bit RGBA of a device frame, on the device: channel * 255, clamped at 255,
 * truncated (the PNG writer's arithmetic; NaN gives 0). */
XTGPU_API xtgpu_status xtgpu_frame_rgba8(const float *rgba_dev, int64_t n_pixels, uint8_t *rgba8_dev, void *stream);
/* PNG file (8-bit RGBA) from host 8-bit pixels. */
XTGPU_API xtgpu_status xtgpu_write_png(const char *path, int32_t width, int32_t height, const uint8_t *rgba8_host);
/* OpenEXR file (uncompressed scanlines, float B, G, R) from a host frame. */
XTGPU_API xtgpu_status xtgpu_write_exr(const char *path, int32_t width, int32_t height, const float *rgba_host);
/* PNG of a host frame: uploaded, quantised by xtgpu_frame_rgba8, written. */
XTGPU_API xtgpu_status xtgpu_save_png_host(const char *path, int32_t width, int32_t height, const float *rgba_host,
                                           void *stream);

/* ---------------------------------------------------------------------- */
/* Render service.  Scenes stay resident; jobs are admitted while their
 * accumulation buffers fit the memory budget and a job slot is free; the rays of
 * all admitted jobs are merged into shared wavefront launches (camera, extend,
 * shade, accumulate) replayed as CUDA graphs.  Results depend only on the job
 * (seed, pixel, sample), never on what else is in flight.  No counterpart in
 * the reference, whose IIntegrator::render (integrator.cc:29-53) renders one
 * frame per blocking call.
 *
 * Threads: one thread at a time runs xtgpu_service_run.  While it runs, any
 * other thread may call xtgpu_service_submit, _poll, _result, _result_host,
 * _release, _open and _get_stats; a job submitted then is admitted as slots
 * and memory free up and joins the next wave launched.  One job's result and
 * release come from one thread.  xtgpu_service_add_scene, _update_scene,
 * _reset_stats and _destroy must not overlap a run.                         */
typedef struct xtgpu_service xtgpu_service;

typedef struct {
    uint64_t memory_budget_bytes;  /* for job accumulation buffers and queues */
    int32_t max_jobs;              /* concurrent job slots (<= 1024) */
    int64_t wave_paths;            /* paths per merged wavefront (0 = autotuned) */
    int32_t node_format;           /* BVH format used by the service */
    int32_t use_graphs;            /* 1 = replay each wave as a CUDA graph */
    int32_t merge_jobs;            /* 0 = one job per launch (the plain path) */
    int32_t host_results;          /* 1 = copy each finished frame to pinned host memory
                                      (asynchronously, reused between jobs) and free its
                                      device buffer at once (frees budget early) */
    int32_t time_kernels;          /* 1 = time every extend launch with CUDA events */
    int32_t count_visits;          /* 1 = count BVH nodes visited / primitives tested */
    int32_t policy;                /* wave planning: 0 = fewest remaining paths first,
                                      1 = equal share per running job */
    int32_t waves_in_flight;       /* 1 = one wave at a time; 2 (or 0) up to
                                      XTGPU_MAX_WAVES_IN_FLIGHT = the next waves are launched
                                      on streams of their own while the earlier ones drain,
                                      so their kernels fill the earlier waves' tails */
} xtgpu_service_opts;
#define XTGPU_MAX_WAVES_IN_FLIGHT 4

typedef struct {
    int32_t scene;                 /* id from xtgpu_service_add_scene */
    int32_t integrator;
    int32_t width, height, spp, rdepth;
    float ao_max_distance;
    uint64_t seed;
    int32_t aa;                    /* anti-aliasing level, as xtgpu_render_params::aa */
    int32_t sample_distribution;   /* XTGPU_SAMPLES_GRID or XTGPU_SAMPLES_RANDOM */
} xtgpu_job_desc;

typedef struct {
    int32_t state;                 /* 0 queued, 1 running, 2 done, 3 failed */
    uint64_t rays;                 /* rays traced for the job */
    double submit_s, start_s, finish_s;   /* service clock (seconds): arrival, admission,
                                             result available (on the host with host_results) */
    double render_done_s;          /* the job's last wave retired (device work done) */
} xtgpu_job_status;

XTGPU_API xtgpu_status xtgpu_service_create(const xtgpu_service_opts *opts, void *stream, xtgpu_service **out);
XTGPU_API xtgpu_status xtgpu_service_add_scene(xtgpu_service *svc, xtgpu_scene *scene, int32_t *scene_id);
/* Refreshes the service's copy of a resident scene's tables after
 * xtgpu_scene_update, and after a BVH rebuild of the scene (xtgpu_bvh_build,
 * xtgpu_autotune or a tuning change that rebuilds): the service's waves read
 * node and leaf buffers through that copy, and its captured graphs that hold
 * the old buffers are dropped.  Waits for the waves in flight. */
XTGPU_API xtgpu_status xtgpu_service_update_scene(xtgpu_service *service, int32_t scene);
/* Queues a job; submit_s is the arrival time on the service clock (seconds
 * since xtgpu_service_create), or a negative value for "now". */
XTGPU_API xtgpu_status xtgpu_service_submit(xtgpu_service *svc, const xtgpu_job_desc *job, double submit_s, int64_t *job_id);
/* Runs admission + waves until every queued job whose arrival time has passed
 * is done, or max_seconds of service clock elapsed (0 = no limit).  While the
 * service is open (xtgpu_service_open), running out of work does not end the
 * run: it waits for submissions until the service is closed. */
XTGPU_API xtgpu_status xtgpu_service_run(xtgpu_service *svc, double max_seconds);
/* Opens (1) or closes (0) the service to live submissions: while open, a
 * running xtgpu_service_run waits for new jobs when it has none; once closed
 * it returns after the jobs already submitted are done.  Callable from any
 * thread. */
XTGPU_API xtgpu_status xtgpu_service_open(xtgpu_service *svc, int32_t open);
XTGPU_API xtgpu_status xtgpu_service_poll(xtgpu_service *svc, int64_t job_id, xtgpu_job_status *status);
/* Copies a finished job's RGBA frame (width*height*4 floats) to host memory. */
XTGPU_API xtgpu_status xtgpu_service_result(xtgpu_service *svc, int64_t job_id, float *rgba_host);
/* With host_results: the finished job's frame in the service's pinned host
 * memory, without a copy; valid until xtgpu_service_release. */
XTGPU_API xtgpu_status xtgpu_service_result_host(xtgpu_service *svc, int64_t job_id, const float **rgba_host);
/* Releases a finished job's frame buffer. */
XTGPU_API xtgpu_status xtgpu_service_release(xtgpu_service *svc, int64_t job_id);
XTGPU_API xtgpu_status xtgpu_service_destroy(xtgpu_service *svc);

typedef struct {
    uint64_t rays;                 /* rays traced since the last reset */
    uint64_t waves;                /* merged wavefront launches */
    uint64_t kernel_launches;      /* camera + extend + shade + accumulate kernels */
    double extend_ms;              /* device time of the extend launches (time_kernels) */
    uint64_t extend_launches;
    uint64_t node_visits, prim_tests;   /* count_visits */
} xtgpu_service_stats;
/* Counters of the service since creation or the last reset. */
XTGPU_API xtgpu_status xtgpu_service_get_stats(xtgpu_service *svc, xtgpu_service_stats *stats);
XTGPU_API xtgpu_status xtgpu_service_reset_stats(xtgpu_service *svc);

/* ---------------------------------------------------------------------- */
/* Launch configuration of the wavefront kernels (process-wide).            */
typedef struct {
    int32_t extend_variant;        /* 0 = warp-batched ray fetch, 1 = lanes refilled when
                                      refill_threshold of them are idle (binary nodes),
                                      2 = the same, voting every steps_per_vote steps */
    int32_t extend_block;          /* threads per block of the extend kernel (32..256) */
    int32_t extend_blocks_per_sm;  /* resident extend blocks per SM, in 128-thread units */
    int32_t tile;                  /* camera ray order: square pixel tiles of this edge (0 = rows) */
    int64_t wave_paths;            /* paths per wave of xtgpu_render */
    int32_t leaf_size;             /* default primitives per BVH leaf */
    int32_t node_layout;           /* BVH node order: 0 = Karras index, 1 = depth-first */
    int32_t refill_threshold;      /* variants 1, 2: idle lanes (1..32) that trigger a refill */
    int32_t extend_min_blocks;     /* variant 0: 0, 8 or 10 resident 128-thread blocks per SM
                                      requested from the compiler (caps registers) */
    int32_t stack_entries;         /* traversal stack: 32 or 64 entries (0 = smallest that
                                      holds the scene's BVH depth) */
    int32_t steps_per_vote;        /* variant 2: traversal steps between refill votes (1..64) */
    int32_t primary_node_format;   /* node format of the first extend pass of a wave (the
                                      coherent camera rays) when every scene of the wave
                                      has it built; -1 = the wave's format */
    int32_t primary_variant;       /* extend kernel of that pass; -1 = extend_variant */
    int32_t bvh_builder;           /* hierarchy over the Morton order: 0 = LBVH (Karras radix
                                      splits), 1 = PLOC agglomerative clustering (Meister and
                                      Bittner 2018; a lower-cost tree, same closest hits) */
    int32_t wide_collapse;         /* 8-wide nodes from the binary tree: 1 = cost-optimal
                                      (surface-area costs by dynamic programming, subtrees of
                                      up to 3 primitives as leaves; Ylitie, Karras and Laine
                                      2017), 0 = greedy largest-area opening */
    float wide_prim_cost;          /* that cost of a primitive test, in node visits (0 = 1; 1 measured
                                      best of 0.3, 0.6, 1 and 1.5 over the served scenes) */
} xtgpu_tuning;
XTGPU_API xtgpu_status xtgpu_get_tuning(xtgpu_tuning *t);
XTGPU_API xtgpu_status xtgpu_set_tuning(const xtgpu_tuning *t);
/* Autotuner.  Picks for one scene the primitives per BVH leaf, the traversal
 * stack size, the camera tile, the extend kernel's register cap and the wave
 * size, by timing a probe pathtracer job (512x512, 4 spp, depth 4) for every
 * candidate of one knob at a time (coordinate descent from the process-wide
 * tuning, within budget_ms of wall time).  The result stays with the scene: the
 * BVH is rebuilt with the chosen leaf size, xtgpu_render uses it, and the service
 * uses its tile for the scene's jobs.  *best receives it. */
XTGPU_API xtgpu_status xtgpu_autotune(xtgpu_scene *scene, int32_t node_format, double budget_ms, xtgpu_tuning *best,
                                      void *stream);
/* Tuning stored with a scene (the process-wide one if it was never tuned),
 * with the leaf size and builder of the BVH the scene was built with. */
XTGPU_API xtgpu_status xtgpu_scene_tuning(const xtgpu_scene *scene, xtgpu_tuning *t);
/* Sets the tuning the scene renders with (as xtgpu_autotune does); its
 * leaf_size and bvh_builder must be those the scene's BVH was built with. */
XTGPU_API xtgpu_status xtgpu_scene_set_tuning(xtgpu_scene *scene, const xtgpu_tuning *tuning);

/* Text of the last error on this thread ("" if none). */
XTGPU_API const char *xtgpu_last_error(void);
/* Library version string. */
XTGPU_API const char *xtgpu_version(void);

#ifdef __cplusplus
}
#endif
#endif /* XTGPU_H */
