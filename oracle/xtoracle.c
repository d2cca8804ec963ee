/*
 * xtoracle.c — CPU restatement (FP64) of XTracer's intersection and integrator
 * hot path.  TEST INFRASTRUCTURE ONLY: the checker for the GPU path, never called
 * by the product library.  Pinned against the reference's own code through the
 * fixtures in tests/golden/ (made by oracle/ref_driver.cc from the reference
 * sources).  Build: oracle/build_oracle.sh (plain gcc -O2, no -march, so that,
 * like the reference built the same way, no FMA contraction happens).
 *
 * Arithmetic follows the reference operation by operation (same association,
 * same float/double conversions) so that results are bit-identical to it.
 * File:line citations are relative to the XTracer source tree.
 */
#include "xtoracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define XO_EPS 1e-8                    /* EPSILON, lib/nmath/precision.h:87-89 */
#define XO_PI 3.14159265358979323846   /* nmath::PI, lib/nmath/precision.h:101 */
#define XO_PI_DOUBLE 6.283185307179586232   /* nmath::PI_DOUBLE, lib/nmath/precision.h:100 */
#define XO_RADIAN 0.017453292519943    /* RADIAN, lib/nmath/precision.h:111 */
#define XO_OCT_MAX_ITEMS 10            /* LIMITS_MAX_ITEMS_PER_NODE, mesh.h:11 */
#define XO_OCT_MAX_DEPTH 10            /* LIMITS_MAX_DEPTH, mesh.h:12 */

/* ------------------------------------------------------------------------ */
/* Vector3f in double (lib/nmath/vector.h:86-150, vector.inl)                 */
typedef struct { double x, y, z; } v3;

static v3 V(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 mul(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static v3 muls(v3 a, double s) { return V(a.x * s, a.y * s, a.z * s); }   /* vector.inl:323-331 */
static v3 divs(v3 a, double s) { return V(a.x / s, a.y / s, a.z / s); }   /* vector.inl:333-336 */
static v3 neg(v3 a) { return V(-a.x, -a.y, -a.z); }
static double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }   /* vector.inl:489-492 */
static v3 cross(v3 a, v3 b)                                                     /* vector.inl:494-497 */
{
    return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static double length(v3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); } /* vector.inl:422-425 */
static v3 normalized(v3 a)                                                      /* vector.inl:444-448 */
{
    double l = length(a);
    return (l != 0) ? V(a.x / l, a.y / l, a.z / l) : a;
}
static v3 normalize(v3 a)                                                       /* vector.inl:432-442 */
{
    double l = length(a);
    if (!l) return a;
    a.x /= l; a.y /= l; a.z /= l;
    return a;
}
static v3 reflected(v3 d, v3 n)                                                 /* vector.inl:455-460 */
{
    v3 i = normalized(d), nn = normalized(n);
    return sub(muls(nn, 2 * dot(i, nn)), i);
}
static v3 vf(const float *f) { return V(f[0], f[1], f[2]); }

/* Colour channels are floats clamped at 0 (lib/nimg/color.cc:6-10, color.inl:48-61). */
typedef struct { float r, g, b; } c3;
static float clamp0(float v) { return v < 0.f ? 0.f : v; }
static c3 C(float r, float g, float b) { c3 c = {clamp0(r), clamp0(g), clamp0(b)}; return c; }
static c3 cmul(c3 a, c3 b) { return C(a.r * b.r, a.g * b.g, a.b * b.b); }   /* color.inl:29-36 */
static c3 cmuls(c3 a, float s) { return C(a.r * s, a.g * s, a.b * s); }     /* color.inl:39-46 */
static c3 cadd(c3 a, c3 b) { return C(a.r + b.r, a.g + b.g, a.b + b.b); }   /* color.inl:11-18 */
static float clamp01(float a) { return a < 0.f ? 0.f : (a > 1.f ? 1.f : a); } /* color.inl:160-163 */

/* ------------------------------------------------------------------------ */
/* Random sources.                                                            */
typedef struct {
    int kind;
    const int32_t *table;   /* XO_RNG_TABLE */
    int32_t rand_max;
    int pos;
    uint64_t key;           /* XO_RNG_STREAM */
    uint32_t counter;
} rng_t;

/* SplitMix64 finaliser (Steele, Lea, Flood, "Fast splittable pseudorandom number
 * generators", OOPSLA 2014).  The GPU path uses the identical function. */
static uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

uint64_t xo_path_key(uint64_t seed, uint64_t path)
{
    return mix64(seed ^ mix64(path + 0x9E3779B97F4A7C15ULL));
}

double xo_stream_uniform(uint64_t key, uint32_t counter)
{
    uint64_t x = mix64(key + (uint64_t)(counter + 1u) * 0x9E3779B97F4A7C15ULL);
    return (double)(uint32_t)(x >> 40) * (1.0 / 16777216.0);
}

uint64_t xo_jitter_key(uint64_t seed, int32_t position, int32_t width, int32_t height, int32_t x, int32_t y)
{
    return xo_path_key(seed ^ XO_JITTER_SALT, (uint64_t)position * (uint64_t)width * (uint64_t)height +
                                                 (uint64_t)y * (uint64_t)width + (uint64_t)x);
}

/* prng_c(a, b) (lib/nmath/prng.inl:54-83): rand() * ((b - a) / RAND_MAX) + a. */
static double prng(rng_t *r, double a, double b)
{
    if (r->kind == XO_RNG_TABLE) {
        double v = (double)r->table[r->pos++];
        return v * ((b - a) / (double)r->rand_max) + a;
    }
    double u = xo_stream_uniform(r->key, r->counter++);
    return u * (b - a) + a;
}

/* ------------------------------------------------------------------------ */
/* Sampling (lib/nmath/sample.inl)                                            */

/* sample::hemisphere, sample.inl:28-59 */
static v3 s_hemisphere(rng_t *r, v3 normal, v3 direction)
{
    double u = prng(r, 0.0f, 1.0f);
    double v = prng(r, 0.0f, 1.0f);
    float phi = (float)acos(sqrt(u));
    float theta = (float)(2.0 * M_PI * v);
    v3 d = V(cos(theta) * sin(phi), cos(phi), sin(theta) * sin(phi));
    v3 norm = normalized(normal);
    v3 xvec = normalized(cross(add(norm, V(XO_EPS, XO_EPS, XO_EPS)), norm));
    v3 yvec = norm;
    v3 zvec = normalized(cross(xvec, yvec));
    /* Matrix3x3f with columns x,y,z; Vector3f::transformed (vector.inl:504-510) */
    v3 t = V(xvec.x * d.x + yvec.x * d.y + zvec.x * d.z,
             xvec.y * d.x + yvec.y * d.y + zvec.y * d.z,
             xvec.z * d.x + yvec.z * d.y + zvec.z * d.z);
    v3 dirc = normalized(direction);
    float ndotl = (float)dot(norm, dirc);
    return normalized(muls(t, (double)(ndotl > 0 ? ndotl : 0)));
}

/* sample::lobe, sample.inl:61-90 */
static v3 s_lobe(rng_t *r, v3 normal, v3 direction, double exponent)
{
    double m[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    v3 refl = reflected(direction, normal);
    if (1.0f - dot(direction, normal) > XO_EPS) {
        v3 ivec = normalized(cross(direction, refl));
        v3 kvec = cross(refl, ivec);
        m[0][0] = ivec.x; m[1][0] = ivec.y; m[2][0] = ivec.z;
        m[0][1] = refl.x; m[1][1] = refl.y; m[2][1] = refl.z;
        m[0][2] = kvec.x; m[1][2] = kvec.y; m[2][2] = kvec.z;
    }
    double u = prng(r, 0.0f, 1.0f);
    double v = prng(r, 0.0f, 1.0f);
    double theta = 2.0 * M_PI * u;
    double phi = acos(pow(v, 1.0 / (exponent + 1)));
    v3 vc = V(cos(theta) * sin(phi), cos(phi), sin(theta) * sin(phi));
    vc = V(m[0][0] * vc.x + m[0][1] * vc.y + m[0][2] * vc.z,
           m[1][0] * vc.x + m[1][1] * vc.y + m[1][2] * vc.z,
           m[2][0] * vc.x + m[2][1] * vc.y + m[2][2] * vc.z);
    double vdotr = dot(refl, vc);
    if (vdotr < 0.0) vdotr = 0.0;
    return normalized(muls(vc, pow(vdotr, exponent)));
}

/* sample::diffuse, sample.inl:92-107.  The three prng_c calls are arguments of
 * one Vector3f constructor; g++ on x86-64 evaluates them last-to-first, so the
 * first value drawn lands in z (checked by the known-answer tests). */
static v3 s_diffuse(rng_t *r, v3 normal)
{
    v3 p;
    float l = 1.0;
    do {
        double c = prng(r, 0, 1);
        double b = prng(r, 0, 1);
        double a = prng(r, 0, 1);
        p = sub(muls(V(a, b, c), 2.0), V(1, 1, 1));
        l = (float)length(mul(p, p));
        l *= l;
    } while (l >= 1.0);
    p = add(p, normal);
    return normalize(p);
}

/* ------------------------------------------------------------------------ */
/* Primitives                                                                 */
typedef struct {
    int hit;
    double t;
    v3 point, normal;
    double tu, tv;   /* hit_record_t::texcoord */
} hrec;

/* Sphere::intersection, math/sphere.cc:25-62 (the active #if 1 branch); usc is
 * the surface's uv_scale (math/surface.h:26). */
static int hit_sphere(v3 c, double radius, const double usc[2], v3 o, v3 d, hrec *h)
{
    double b = 2 * dot(sub(o, c), d);
    double cc = dot(c, c) + dot(o, o) + 2 * dot(neg(c), o) - radius * radius;
    double discr = (b * b - 4 * cc);
    if (discr > 0.0) {
        double sq = sqrt(discr);
        double t1 = (-b + sq) / 2.0;
        double t2 = (-b - sq) / 2.0;
        double t = t1 < t2 ? t1 : t2;
        if (t > XO_EPS) {
            h->t = t;
            h->point = add(o, muls(d, t));
            h->normal = muls(divs(sub(h->point, c), radius), (t1 * t2 > 0. ? 1. : -1));
            h->tu = asin(h->normal.x / (usc[0] != 0.0f ? usc[0] : 1.0f)) / XO_PI + 0.5;
            h->tv = asin(h->normal.y / (usc[1] != 0.0f ? usc[1] : 1.0f)) / XO_PI + 0.5;
            return 1;
        }
    }
    return 0;
}

/* Plane::intersection, math/plane.cc:19-61 */
static int hit_plane(v3 n, double offset, const double usc[2], v3 o, v3 d, hrec *h)
{
    double n_dot_dir = dot(n, d);
    if (fabs(n_dot_dir) < XO_EPS) return 0;
    v3 v = muls(V(fabs(n.x), fabs(n.y), fabs(n.z)), offset);
    v3 vorigin = sub(v, o);
    double n_dot_vo = dot(vorigin, n);
    double t = n_dot_vo / n_dot_dir;
    if (t < XO_EPS) return 0;
    h->t = t;
    h->point = add(o, muls(d, t));
    h->normal = n;
    /* texture coordinates, plane.cc:47-58 */
    v3 nn = normalized(n);
    v3 uvec = V(nn.y, nn.z, -nn.x);
    v3 vvec = cross(uvec, nn);
    double tu = dot(uvec, add(v, h->point)) * usc[0];
    double tv = dot(vvec, add(v, h->point)) * usc[1];
    if (tu > 1.f) tu -= (float)(int)tu;
    if (tv > 1.f) tv -= (float)(int)tv;
    if (tu < -1.f) tu -= (float)(int)tu;
    if (tv < -1.f) tv -= (float)(int)tv;
    if (tu < 0.f) tu = 1.f + tu;
    if (tv < 0.f) tv = 1.f + tv;
    h->tu = tu;
    h->tv = tv;
    return 1;
}

/* Triangle::calc_barycentric, math/triangle.cc:149-184 */
static v3 tri_bary(const v3 *v, v3 p)
{
    v3 v1 = sub(v[1], v[0]), v2 = sub(v[2], v[0]);
    v3 x = cross(v1, v2);
    v3 norm = normalized(x);
    double area = fabs(dot(x, norm)) * 0.5;
    if (area < XO_EPS) return V(0, 0, 0);
    v3 pv0 = sub(v[0], p), pv1 = sub(v[1], p), pv2 = sub(v[2], p);
    v3 x12 = cross(pv1, pv2), x20 = cross(pv2, pv0), x01 = cross(pv0, pv1);
    double a0 = fabs(dot(x12, norm)) * 0.5;
    double a1 = fabs(dot(x20, norm)) * 0.5;
    double a2 = fabs(dot(x01, norm)) * 0.5;
    return V(a0 / area, a1 / area, a2 / area);
}

/* Triangle::intersection, math/triangle.cc:82-123 (normal: calc_normal :142-147);
 * vt: the three texcoords (tc), z = 0 */
static int hit_triangle(const v3 *v, const v3 *vn, const v3 *vt, v3 o, v3 d, hrec *h)
{
    v3 normal = normalized(cross(sub(v[1], v[0]), sub(v[2], v[0])));
    double n_dot_dir = dot(normal, d);
    if (fabs(n_dot_dir) < XO_EPS) return 0;
    v3 vo = sub(o, v[0]);
    double t = -dot(normal, vo) / n_dot_dir;
    if (t < XO_EPS) return 0;
    v3 pos = add(o, muls(d, t));
    v3 bc = tri_bary(v, pos);
    double s = bc.x + bc.y + bc.z;
    if (s < 1.0 - XO_EPS || s > 1.0 + XO_EPS) return 0;
    h->t = t;
    h->point = pos;
    v3 tc = add(add(muls(vt[0], bc.x), muls(vt[1], bc.y)), muls(vt[2], bc.z));
    h->tu = tc.x;
    h->tv = tc.y;
    v3 pn = add(add(muls(vn[0], bc.x), muls(vn[1], bc.y)), muls(vn[2], bc.z));
    h->normal = length(pn) ? pn : normal;
    return 1;
}

/* AABB3::intersection, math/aabb.cc:32-71 (float inverse directions). */
static int hit_aabb(v3 mn, v3 mx, v3 o, v3 d)
{
    if (o.x > mn.x && o.y > mn.y && o.z > mn.z && o.x < mx.x && o.y < mx.y && o.z < mx.z) return 1;
    v3 bb[2] = {mn, mx};
    const float t0 = 0.0;
    int xs = (int)(d.x < 0.0), ys = (int)(d.y < 0.0);
    float ix = (float)(1.0 / d.x), iy = (float)(1.0 / d.y);
    float tmin = (float)((bb[xs].x - o.x) * ix);
    float tmax = (float)((bb[1 - xs].x - o.x) * ix);
    float tymin = (float)((bb[ys].y - o.y) * iy);
    float tymax = (float)((bb[1 - ys].y - o.y) * iy);
    if ((tmin > tymax) || (tymin > tmax)) return 0;
    if (tymin > tmin) tmin = tymin;
    if (tymax < tmax) tmax = tymax;
    int zs = (int)(d.z < 0.0);
    float iz = (float)(1.0 / d.z);
    float tzmin = (float)((bb[zs].z - o.z) * iz);
    float tzmax = (float)((bb[1 - zs].z - o.z) * iz);
    if ((tmin > tzmax) || (tzmin > tmax)) return 0;
    if (tzmin > tmin) tmin = tzmin;
    if (tzmax < tmax) tmax = tzmax;
    return (tmax > t0);
}

/* ------------------------------------------------------------------------ */
/* Octree<Triangle> (octree.h:12-62, octree.tml:118-249) for one mesh.        */
typedef struct onode {
    v3 mn, mx;
    int32_t *items;   /* triangle indices (into the mesh), list order */
    int32_t nitems;
    int32_t child[8]; /* -1 = none */
} onode;

typedef struct {
    onode *nodes;
    int32_t nnodes, cap;
    v3 *tv;           /* 3 vertices per triangle (double) */
    v3 *tn;           /* 3 normals per triangle */
    v3 *tt;           /* 3 texcoords per triangle (z = 0) */
    v3 *amin, *amax;  /* item AABBs (Triangle::calc_aabb, triangle.cc:125-140) */
    int32_t ntris;
    /* FP64 BVH (XO_ACCEL_BVH) */
    struct bnode { v3 mn, mx; int32_t left, right, first, count; } *bvh;
    int32_t *bidx;
    int32_t nbvh;
} mesh_t;

static int contains(v3 mn, v3 mx, v3 p)   /* AABB3::contains, aabb.inl:38-41 */
{
    return (p.x >= mn.x) && (p.y >= mn.y) && (p.z >= mn.z) && (p.x <= mx.x) && (p.y <= mx.y) && (p.z <= mx.z);
}

static v3 vmin(v3 a, v3 b) { return V(a.x <= b.x ? a.x : b.x, a.y <= b.y ? a.y : b.y, a.z <= b.z ? a.z : b.z); }
static v3 vmax(v3 a, v3 b) { return V(a.x >= b.x ? a.x : b.x, a.y >= b.y ? a.y : b.y, a.z >= b.z ? a.z : b.z); }

static int32_t onew(mesh_t *m)
{
    if (m->nnodes == m->cap) {
        m->cap = m->cap ? m->cap * 2 : 1024;
        m->nodes = (onode *)realloc(m->nodes, sizeof(onode) * (size_t)m->cap);
    }
    onode *n = &m->nodes[m->nnodes];
    memset(n, 0, sizeof(*n));
    for (int i = 0; i < 8; ++i) n->child[i] = -1;
    return m->nnodes++;
}

/* Octree::subdivide, octree.tml:138-198.  Child box 7 takes the ROOT's max.z
 * (octree.tml:166), as in the reference. */
static void osubdivide(mesh_t *m, int32_t ni, size_t level, v3 root_max)
{
    if (m->nodes[ni].nitems <= XO_OCT_MAX_ITEMS || level >= XO_OCT_MAX_DEPTH) return;
    v3 mn = m->nodes[ni].mn, mx = m->nodes[ni].mx;
    v3 c = divs(add(mn, mx), 2.f);
    v3 cmn[8], cmx[8];
#define BOX(i, a, b) do { cmn[i] = vmin(a, b); cmx[i] = vmax(a, b); } while (0)
    BOX(0, mn, c);
    BOX(1, V(c.x, mn.y, mn.z), V(mx.x, c.y, c.z));
    BOX(2, V(c.x, c.y, mn.z), V(mx.x, mx.y, c.z));
    BOX(3, V(mn.x, c.y, mn.z), V(c.x, mx.y, c.z));
    BOX(4, V(mn.x, mn.y, c.z), V(c.x, c.y, mx.z));
    BOX(5, V(c.x, mn.y, c.z), V(mx.x, c.y, mx.z));
    BOX(6, c, mx);
    BOX(7, V(mn.x, c.y, c.z), V(c.x, mx.y, root_max.z));
#undef BOX
    for (int i = 0; i < 8; ++i) {
        int32_t ci = onew(m);
        onode *cn = &m->nodes[ci];
        onode *pn = &m->nodes[ni];
        pn->child[i] = ci;
        cn->mn = cmn[i];
        cn->mx = cmx[i];
        int32_t keep = 0;
        cn->items = (int32_t *)malloc(sizeof(int32_t) * (size_t)(pn->nitems ? pn->nitems : 1));
        for (int32_t k = 0; k < pn->nitems; ++k) {
            int32_t it = pn->items[k];
            const v3 *tv = &m->tv[3 * it];
            if (contains(cmn[i], cmx[i], tv[0]) && contains(cmn[i], cmx[i], tv[1]) && contains(cmn[i], cmx[i], tv[2]))
                cn->items[cn->nitems++] = it;
            else
                pn->items[keep++] = it;
        }
        pn->nitems = keep;
    }
    for (int i = 0; i < 8; ++i) osubdivide(m, m->nodes[ni].child[i], level + 1, root_max);
}

/* Octree::add + build, octree.tml:103-136; the root box starts at the origin
 * because clear() zeroes m_aabb (octree.tml:94-96) before add() augments it. */
static void obuild(mesh_t *m)
{
    v3 mn = V(0, 0, 0), mx = V(0, 0, 0);
    for (int32_t i = 0; i < m->ntris; ++i) {
        v3 a = m->amin[i], b = m->amax[i];
        if (b.x > mx.x) mx.x = b.x;
        if (a.x < mn.x) mn.x = a.x;
        if (b.y > mx.y) mx.y = b.y;
        if (a.y < mn.y) mn.y = a.y;
        if (b.z > mx.z) mx.z = b.z;
        if (a.z < mn.z) mn.z = a.z;
    }
    int32_t r = onew(m);
    m->nodes[r].mn = mn;
    m->nodes[r].mx = mx;
    m->nodes[r].items = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m->ntris ? m->ntris : 1));
    for (int32_t i = 0; i < m->ntris; ++i) m->nodes[r].items[i] = i;
    m->nodes[r].nitems = m->ntris;
    if (m->nodes[r].nitems > XO_OCT_MAX_ITEMS) osubdivide(m, r, 0, mx);
}

/* Octree::r_intersection, octree.tml:206-249 */
static int32_t otrace(const mesh_t *m, int32_t ni, v3 o, v3 d, hrec *out)
{
    if (ni < 0) return -1;
    const onode *n = &m->nodes[ni];
    if (!hit_aabb(n->mn, n->mx, o, d)) return -1;
    hrec best;
    best.t = FLT_MAX;
    int32_t closest = -1;
    for (int32_t k = 0; k < n->nitems; ++k) {
        hrec h;
        int32_t it = n->items[k];
        if (hit_triangle(&m->tv[3 * it], &m->tn[3 * it], &m->tt[3 * it], o, d, &h) && h.t < best.t) {
            best = h;
            closest = it;
        }
    }
    for (int i = 0; i < 8; ++i) {
        hrec h;
        int32_t it = otrace(m, n->child[i], o, d, &h);
        if (it >= 0 && h.t < best.t) {
            best = h;
            closest = it;
        }
    }
    if (closest >= 0) *out = best;
    return closest;
}

/* ------------------------------------------------------------------------ */
/* FP64 BVH over a mesh, used only to make the oracle fast on large meshes.   */
/* Same triangle test; boxes padded so no hit can be culled by rounding.      */
static int32_t bbuild(mesh_t *m, int32_t first, int32_t count)
{
    int32_t ni = m->nbvh++;
    v3 mn = V(INFINITY, INFINITY, INFINITY), mx = V(-INFINITY, -INFINITY, -INFINITY);
    v3 cmn = mn, cmx = mx;
    for (int32_t k = first; k < first + count; ++k) {
        int32_t i = m->bidx[k];
        mn = vmin(mn, m->amin[i]);
        mx = vmax(mx, m->amax[i]);
        v3 c = muls(add(m->amin[i], m->amax[i]), 0.5);
        cmn = vmin(cmn, c);
        cmx = vmax(cmx, c);
    }
    double pad = 1e-9 * (1.0 + fmax(fmax(fabs(mn.x), fabs(mx.x)), fmax(fmax(fabs(mn.y), fabs(mx.y)), fmax(fabs(mn.z), fabs(mx.z)))));
    m->bvh[ni].mn = sub(mn, V(pad, pad, pad));
    m->bvh[ni].mx = add(mx, V(pad, pad, pad));
    m->bvh[ni].first = first;
    m->bvh[ni].count = count;
    m->bvh[ni].left = m->bvh[ni].right = -1;
    if (count <= 4) return ni;
    v3 ext = sub(cmx, cmn);
    int axis = (ext.x >= ext.y && ext.x >= ext.z) ? 0 : (ext.y >= ext.z ? 1 : 2);
    double mid = axis == 0 ? (cmn.x + cmx.x) * 0.5 : axis == 1 ? (cmn.y + cmx.y) * 0.5 : (cmn.z + cmx.z) * 0.5;
    int32_t lo = first, hi = first + count - 1;
    while (lo <= hi) {
        int32_t i = m->bidx[lo];
        v3 c = muls(add(m->amin[i], m->amax[i]), 0.5);
        double cv = axis == 0 ? c.x : axis == 1 ? c.y : c.z;
        if (cv < mid) ++lo;
        else { int32_t t = m->bidx[hi]; m->bidx[hi] = m->bidx[lo]; m->bidx[lo] = t; --hi; }
    }
    int32_t nl = lo - first;
    if (nl == 0 || nl == count) nl = count / 2;
    int32_t l = bbuild(m, first, nl);
    int32_t r = bbuild(m, first + nl, count - nl);
    m->bvh[ni].left = l;
    m->bvh[ni].right = r;
    return ni;
}

static int box_t(v3 mn, v3 mx, v3 o, v3 d, double tmax)
{
    double t0 = 0.0, t1 = tmax;
    double oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z}, lo[3] = {mn.x, mn.y, mn.z}, hi[3] = {mx.x, mx.y, mx.z};
    for (int a = 0; a < 3; ++a) {
        if (dd[a] == 0.0) {
            if (oo[a] < lo[a] || oo[a] > hi[a]) return 0;
            continue;
        }
        double inv = 1.0 / dd[a];
        double ta = (lo[a] - oo[a]) * inv, tb = (hi[a] - oo[a]) * inv;
        if (ta > tb) { double t = ta; ta = tb; tb = t; }
        ta -= 1e-12 * fabs(ta);
        tb += 1e-12 * fabs(tb);
        if (ta > t0) t0 = ta;
        if (tb < t1) t1 = tb;
        if (t0 > t1) return 0;
    }
    return 1;
}

/* Closest hit in the mesh with the reference triangle test.  Among equal t the
 * lowest triangle index wins (the octree would pick by node order instead;
 * exact-t ties are the only place the two can differ). */
static int32_t btrace(const mesh_t *m, v3 o, v3 d, hrec *out)
{
    int32_t stack[128];
    int sp = 0;
    stack[sp++] = 0;
    hrec best;
    best.t = INFINITY;
    int32_t closest = -1;
    while (sp) {
        const struct bnode *n = &m->bvh[stack[--sp]];
        if (!box_t(n->mn, n->mx, o, d, best.t)) continue;
        if (n->left < 0) {
            for (int32_t k = n->first; k < n->first + n->count; ++k) {
                int32_t it = m->bidx[k];
                hrec h;
                if (hit_triangle(&m->tv[3 * it], &m->tn[3 * it], &m->tt[3 * it], o, d, &h) &&
                    (h.t < best.t || (h.t == best.t && it < closest))) {
                    best = h;
                    closest = it;
                }
            }
        } else {
            stack[sp++] = n->right;
            stack[sp++] = n->left;
        }
    }
    if (closest >= 0) *out = best;
    return closest;
}

/* ------------------------------------------------------------------------ */
struct xo_scene {
    xo_scene_desc d;
    int accel;
    mesh_t *meshes;   /* one per object (only XO_MESH objects filled) */
};

int xo_scene_create(const xo_scene_desc *desc, int accel, xo_scene **out)
{
    xo_scene *s = (xo_scene *)calloc(1, sizeof(xo_scene));
    if (!s) return 1;
    s->d = *desc;
    s->accel = accel;
    s->meshes = (mesh_t *)calloc((size_t)(desc->n_objects ? desc->n_objects : 1), sizeof(mesh_t));
    for (int32_t oi = 0; oi < desc->n_objects; ++oi) {
        if (desc->obj_kind[oi] != XO_MESH) continue;
        mesh_t *m = &s->meshes[oi];
        int32_t first = desc->obj_first[oi], count = desc->obj_count[oi];
        m->ntris = count;
        m->tv = (v3 *)malloc(sizeof(v3) * 3 * (size_t)(count ? count : 1));
        m->tn = (v3 *)calloc(3 * (size_t)(count ? count : 1), sizeof(v3));
        m->tt = (v3 *)calloc(3 * (size_t)(count ? count : 1), sizeof(v3));
        m->amin = (v3 *)malloc(sizeof(v3) * (size_t)(count ? count : 1));
        m->amax = (v3 *)malloc(sizeof(v3) * (size_t)(count ? count : 1));
        for (int32_t i = 0; i < count; ++i) {
            const float *t = desc->tris + 9 * (size_t)(first + i);
            for (int k = 0; k < 3; ++k) {
                m->tv[3 * i + k] = vf(t + 3 * k);
                if (desc->tri_normals) m->tn[3 * i + k] = vf(desc->tri_normals + 9 * (size_t)(first + i) + 3 * k);
                if (desc->tri_uvs) {
                    const float *uv = desc->tri_uvs + 6 * (size_t)(first + i) + 2 * k;
                    m->tt[3 * i + k] = V(uv[0], uv[1], 0.0);
                } else {
                    /* the Triangle constructor's texcoords (math/triangle.cc:8-13):
                     * tc[1] is set twice, tc[2] stays zero */
                    m->tt[3 * i + k] = k == 1 ? V(1.0, 0.0, 0.0) : V(0.0, 0.0, 0.0);
                }
            }
            /* Triangle::calc_aabb, triangle.cc:125-140 */
            v3 mn = V(INFINITY, INFINITY, INFINITY), mx = V(-INFINITY, -INFINITY, -INFINITY);
            for (int k = 0; k < 3; ++k) {
                v3 p = m->tv[3 * i + k];
                if (p.x < mn.x) mn.x = p.x;
                if (p.y < mn.y) mn.y = p.y;
                if (p.z < mn.z) mn.z = p.z;
                if (p.x > mx.x) mx.x = p.x;
                if (p.y > mx.y) mx.y = p.y;
                if (p.z > mx.z) mx.z = p.z;
            }
            m->amin[i] = mn;
            m->amax[i] = mx;
        }
        if (accel == XO_ACCEL_OCTREE) {
            obuild(m);
        } else {
            m->bidx = (int32_t *)malloc(sizeof(int32_t) * (size_t)(count ? count : 1));
            for (int32_t i = 0; i < count; ++i) m->bidx[i] = i;
            m->bvh = malloc(sizeof(*m->bvh) * (size_t)(2 * (count ? count : 1)));
            if (count) bbuild(m, 0, count);
        }
    }
    *out = s;
    return 0;
}

void xo_scene_destroy(xo_scene *s)
{
    if (!s) return;
    for (int32_t oi = 0; oi < s->d.n_objects; ++oi) {
        mesh_t *m = &s->meshes[oi];
        for (int32_t i = 0; i < m->nnodes; ++i) free(m->nodes[i].items);
        free(m->nodes); free(m->tv); free(m->tn); free(m->tt); free(m->amin); free(m->amax); free(m->bvh); free(m->bidx);
    }
    free(s->meshes);
    free(s);
}

/* Scene::intersection, scene.cc:191-216: linear loop over objects in map order,
 * `res.t > test.t` keeps the first of equal hits. */
static int scene_hit(const xo_scene *s, v3 o, v3 d, hrec *res, int32_t *obj, int32_t *prim)
{
    const xo_scene_desc *D = &s->d;
    int hit = 0;
    res->t = INFINITY;
    *obj = -1;
    *prim = -1;
    for (int32_t oi = 0; oi < D->n_objects; ++oi) {
        hrec h;
        int ok = 0;
        int32_t p = D->obj_first[oi];
        const double usc[2] = {D->obj_uv_scale ? (double)D->obj_uv_scale[2 * oi] : 0.0,
                               D->obj_uv_scale ? (double)D->obj_uv_scale[2 * oi + 1] : 0.0};
        if (D->obj_kind[oi] == XO_SPHERE) {
            const float *sp = D->spheres + 4 * (size_t)p;
            ok = hit_sphere(V(sp[0], sp[1], sp[2]), (double)sp[3], usc, o, d, &h);
        } else if (D->obj_kind[oi] == XO_PLANE) {
            const float *pl = D->planes + 4 * (size_t)p;
            ok = hit_plane(V(pl[0], pl[1], pl[2]), (double)pl[3], usc, o, d, &h);
        } else {
            const mesh_t *m = &s->meshes[oi];
            int32_t it = (s->accel == XO_ACCEL_OCTREE) ? otrace(m, m->nnodes ? 0 : -1, o, d, &h)
                                                       : (m->nbvh ? btrace(m, o, d, &h) : -1);
            ok = it >= 0;
            p = D->obj_first[oi] + it;
        }
        if (ok) {
            hit = 1;
            if (res->t > h.t) {
                *res = h;
                *obj = oi;
                *prim = p;
            }
        }
    }
    return hit;
}

void xo_trace(const xo_scene *s, int64_t n, const double *org, const double *dir,
              int32_t *hit, double *t, int32_t *obj, int32_t *prim, double *point, double *normal)
{
    for (int64_t i = 0; i < n; ++i) {
        hrec h;
        int32_t oi, pi;
        int ok = scene_hit(s, V(org[3 * i], org[3 * i + 1], org[3 * i + 2]),
                           V(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]), &h, &oi, &pi);
        hit[i] = ok;
        t[i] = ok ? h.t : -1.0;
        obj[i] = oi;
        prim[i] = pi;
        if (point) { point[3 * i] = ok ? h.point.x : 0; point[3 * i + 1] = ok ? h.point.y : 0; point[3 * i + 2] = ok ? h.point.z : 0; }
        if (normal) { normal[3 * i] = ok ? h.normal.x : 0; normal[3 * i + 1] = ok ? h.normal.y : 0; normal[3 * i + 2] = ok ? h.normal.z : 0; }
    }
}

/* ------------------------------------------------------------------------ */
/* Perspective::get_primary_ray, camera/perspective.cc:26-98 (flength = 0). */
void xo_camera_ray(const float pos[3], const float target[3], const float up[3], float fov,
                   float x, float y, float w, float h, double org[3], double dir[3])
{
    double aspect = (double)w / (double)h;
    v3 d = V((2.0 * (double)x / (double)w) - 1.0,
             ((2.0 * (double)y / (double)h) - 1.0) / aspect,
             1.0 / tan(fov * XO_RADIAN / 2.0));
    v3 p = vf(pos);
    v3 rz = normalized(sub(vf(target), p));
    v3 rx = normalized(cross(vf(up), rz));
    v3 ry = normalized(cross(rx, rz));
    /* Vector3f::transformed(Matrix4x4f) adds the zero translation column
     * (vector.inl:517-523). */
    v3 t = V(rx.x * d.x + ry.x * d.y + rz.x * d.z + 0.0,
             rx.y * d.x + ry.y * d.y + rz.y * d.z + 0.0,
             rx.z * d.x + ry.z * d.y + rz.z * d.z + 0.0);
    t = normalize(t);
    org[0] = p.x; org[1] = p.y; org[2] = p.z;
    dir[0] = t.x; dir[1] = t.y; dir[2] = t.z;
}

/* Perspective with depth of field (camera/perspective.cc:38-98, flength > 0):
 * the direction in camera space is the lens point (two prng_c draws, x then y,
 * within half the aperture) to the focal-plane point; the origin is the lens
 * point transformed and moved to the position. */
static void camera_dof(rng_t *r, const float pos[3], const float target[3], const float up[3], float fov,
                       float flength, float aperture, float x, float y, float w, float h, double org[3],
                       double dir[3])
{
    double aspect = (double)w / (double)h;
    v3 d = V((2.0 * (double)x / (double)w) - 1.0,
             ((2.0 * (double)y / (double)h) - 1.0) / aspect,
             1.0 / tan(fov * XO_RADIAN / 2.0));
    v3 p = vf(pos);
    v3 rz = normalized(sub(vf(target), p));
    v3 rx = normalized(cross(vf(up), rz));
    v3 ry = normalized(cross(rx, rz));
    v3 lo = d;
    double half = aperture / 2.f;
    lo.x += prng(r, -half, half);
    lo.y += prng(r, -half, half);
    v3 fpip = add(d, muls(normalized(d), (double)flength));
    v3 fd = sub(fpip, lo);
    v3 t = V(rx.x * fd.x + ry.x * fd.y + rz.x * fd.z + 0.0,
             rx.y * fd.x + ry.y * fd.y + rz.y * fd.z + 0.0,
             rx.z * fd.x + ry.z * fd.y + rz.z * fd.z + 0.0);
    t = normalize(t);
    v3 o = V(rx.x * lo.x + ry.x * lo.y + rz.x * lo.z + 0.0,
             rx.y * lo.x + ry.y * lo.y + rz.y * lo.z + 0.0,
             rx.z * lo.x + ry.z * lo.y + rz.z * lo.z + 0.0);
    o = add(o, p);
    org[0] = o.x; org[1] = o.y; org[2] = o.z;
    dir[0] = t.x; dir[1] = t.y; dir[2] = t.z;
}

/* Matrix4x4f::rotate(euler) applied to an identity matrix (lib/nmath/matrix.cc:
 * 485-492, 414-427): I *= (xrot * yrot * zrot), products summed left to right. */
static void euler_rotation(const float e3[3], double m[3][4])
{
    double ex = e3[0], ey = e3[1], ez = e3[2];
    double xr[3][3] = {{1, 0, 0}, {0, cos(ex), -sin(ex)}, {0, sin(ex), cos(ex)}};
    double yr[3][3] = {{cos(ey), 0, sin(ey)}, {0, 1, 0}, {-sin(ey), 0, cos(ey)}};
    double zr[3][3] = {{cos(ez), -sin(ez), 0}, {sin(ez), cos(ez), 0}, {0, 0, 1}};
    double t[3][3], r3[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t[i][j] = xr[i][0] * yr[0][j] + xr[i][1] * yr[1][j] + xr[i][2] * yr[2][j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r3[i][j] = t[i][0] * zr[0][j] + t[i][1] * zr[1][j] + t[i][2] * zr[2][j];
    double m4[4][4] = {{r3[0][0], r3[0][1], r3[0][2], 0}, {r3[1][0], r3[1][1], r3[1][2], 0},
                       {r3[2][0], r3[2][1], r3[2][2], 0}, {0, 0, 0, 1}};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 4; ++j) {
            double id0 = i == 0, id1 = i == 1, id2 = i == 2;
            m[i][j] = id0 * m4[0][j] + id1 * m4[1][j] + id2 * m4[2][j] + 0.0 * m4[3][j];
        }
}

static v3 transform4(const double m[3][4], v3 v)   /* Vector3f::transformed(Matrix4x4f), vector.inl:517-523 */
{
    return V(m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z + m[0][3],
             m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z + m[1][3],
             m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z + m[2][3]);
}

/* ERP::get_primary_ray, camera/erp.cc:13-31 (angles in float, trig in double) */
static void camera_erp(const float pos[3], const float orient[3], float x, float y, float w, float h,
                       double org[3], double dir[3])
{
    float phi = (float)((x / w) * XO_PI * 2.f);
    float theta = (float)((y / h) * XO_PI);
    v3 d = V(sin(theta) * cos(phi), cos(theta), sin(theta) * sin(phi));
    double m[3][4];
    euler_rotation(orient, m);
    d = transform4(m, d);
    org[0] = pos[0]; org[1] = pos[1]; org[2] = pos[2];
    dir[0] = d.x; dir[1] = d.y; dir[2] = d.z;
}

/* ODS::get_primary_ray, camera/ods.cc:17-40: the upper half of the frame is
 * one eye, the lower the other, each origin on a circle of radius ipd/2 */
static void camera_ods(const float pos[3], const float orient[3], float ipd, float x, float y, float w, float h,
                       double org[3], double dir[3])
{
    float hh = h * .5f;
    float scale = ipd * .5f * ((y < hh) ? -1 : 1);
    if (y > hh) y = y - hh;
    float theta = (float)((x / w) * 2.f * XO_PI);
    float phi = (float)(XO_PI * .5f - (y / hh) * XO_PI);
    v3 o = add(muls(V(cos(theta), 0, sin(theta)), (double)scale), vf(pos));
    v3 d = V(sin(theta) * cos(phi), sin(phi), -cos(theta) * cos(phi));
    double m[3][4];
    euler_rotation(orient, m);
    d = transform4(m, d);
    org[0] = o.x; org[1] = o.y; org[2] = o.z;
    dir[0] = d.x; dir[1] = d.y; dir[2] = d.z;
}

/* Cubemap::get_primary_ray, camera/cubemap.cc:21-69 (vertical strip of six
 * square faces +x -x +y -y +z -z) */
static void camera_cubemap(const float pos[3], float x, float y, float w, float h, double org[3], double dir[3])
{
    size_t face_size = (size_t)(h) / 6;
    size_t face = (size_t)(y) / face_size;
    v3 camdir = V(0, 0, 0), up = V(0, 0, 0);
    switch (face) {
    case 0: camdir = V(1, 0, 0); up = V(0, 1, 0); break;
    case 1: camdir = V(-1, 0, 0); up = V(0, 1, 0); break;
    case 2: camdir = V(0, 1, 0); up = V(0, 0, -1); break;
    case 3: camdir = V(0, -1, 0); up = V(0, 0, 1); break;
    case 4: camdir = V(0, 0, 1); up = V(0, 1, 0); break;
    case 5: camdir = V(0, 0, -1); up = V(0, 1, 0); break;
    }
    y -= (float)(face * face_size);
    v3 d = V((2.f * (double)x / (double)w) - 1.f, (2.f * (double)y / (double)face_size) - 1.f, 1.f);
    d = normalize(d);
    v3 rz = camdir;
    v3 rx = normalize(cross(up, rz));
    v3 ry = normalize(cross(rx, rz));
    d = V(rx.x * d.x + ry.x * d.y + rz.x * d.z + 0.0, rx.y * d.x + ry.y * d.y + rz.y * d.z + 0.0,
          rx.z * d.x + ry.z * d.y + rz.z * d.z + 0.0);
    d = normalize(d);
    org[0] = pos[0]; org[1] = pos[1]; org[2] = pos[2];
    dir[0] = d.x; dir[1] = d.y; dir[2] = d.z;
}

/* The scene's camera at (x, y); r supplies the depth-of-field draws. */
static void camera_any(const xo_scene_desc *D, rng_t *r, float x, float y, float w, float h, double o[3],
                       double d[3])
{
    switch (D->cam_type) {
    case XO_CAM_ERP: camera_erp(D->cam_pos, D->cam_orientation, x, y, w, h, o, d); return;
    case XO_CAM_ODS: camera_ods(D->cam_pos, D->cam_orientation, D->cam_ipd, x, y, w, h, o, d); return;
    case XO_CAM_CUBEMAP: camera_cubemap(D->cam_pos, x, y, w, h, o, d); return;
    default:
        if (D->cam_flength > 0)
            camera_dof(r, D->cam_pos, D->cam_target, D->cam_up, D->cam_fov, D->cam_flength, D->cam_aperture, x, y,
                       w, h, o, d);
        else
            xo_camera_ray(D->cam_pos, D->cam_target, D->cam_up, D->cam_fov, x, y, w, h, o, d);
    }
}

void xo_kat_camera_dof(const int32_t *table, int32_t rand_max, const float pos[3], const float target[3],
                       const float up[3], float fov, float flength, float aperture, float x, float y, float w,
                       float h, double org[3], double dir[3])
{
    rng_t r;
    memset(&r, 0, sizeof(r));
    r.kind = XO_RNG_TABLE;
    r.table = table;
    r.rand_max = rand_max;
    camera_dof(&r, pos, target, up, fov, flength, aperture, x, y, w, h, org, dir);
}

void xo_kat_camera_erp(const float pos[3], const float orient[3], float x, float y, float w, float h,
                       double org[3], double dir[3])
{
    camera_erp(pos, orient, x, y, w, h, org, dir);
}

void xo_kat_camera_ods(const float pos[3], const float orient[3], float ipd, float x, float y, float w, float h,
                       double org[3], double dir[3])
{
    camera_ods(pos, orient, ipd, x, y, w, h, org, dir);
}

void xo_kat_camera_cubemap(const float pos[3], float x, float y, float w, float h, double org[3], double dir[3])
{
    camera_cubemap(pos, x, y, w, h, org, dir);
}

/* ------------------------------------------------------------------------ */
/* Materials: IMaterial::sample_path (src/xtcore/material/).                  */
typedef struct {
    v3 org, dir;
    c3 intensity;
} hres;

/* ------------------------------------------------------------------------ */
/* Samplers                                                                   */

/* The x86-64 conversion the reference's (int) cast of a float compiles to
 * (cvttss2si): a value outside int's range, NaN included, gives INT_MIN. */
static int32_t f2i_x86(float f)
{
    return (f != f || f >= 2147483648.f || f < -2147483648.f) ? INT32_MIN : (int32_t)f;
}

/* Pixmap::pixel_ro clamps both coordinates to the last column / row
 * (lib/nimg/pixmap.cc:44-50). */
static const float *texel(const xo_texture *t, const float *tx, uint64_t x, uint64_t y)
{
    uint64_t nx = x >= (uint64_t)t->width ? (uint64_t)t->width - 1 : x;
    uint64_t ny = y >= (uint64_t)t->height ? (uint64_t)t->height - 1 : y;
    return tx + 4 * (t->offset + (int64_t)(ny * (uint64_t)t->width + nx));
}

/* nimg::sample::nearest, lib/nimg/sample.cc:8-17: wrap into [0, 1], then
 * (size_t)(u * (float)width); a NaN coordinate converts to 2^63 on x86-64
 * and is clamped to the last texel. */
static c3 tex_nearest(const xo_texture *t, const float *tx, double u, double v)
{
    u = u < 0 ? 0 : (u > 1 ? u - floor(u) : u);
    v = v < 0 ? 0 : (v > 1 ? v - floor(v) : v);
    double fx = u * (float)t->width, fy = v * (float)t->height;
    uint64_t x = fx == fx ? (uint64_t)fx : (1ull << 63);
    uint64_t y = fy == fy ? (uint64_t)fy : (1ull << 63);
    const float *c = texel(t, tx, x, y);
    return C(c[0], c[1], c[2]);
}

/* nimg::sample::bilinear, lib/nimg/sample.cc:19-52: the int texel index is
 * taken modulo the size_t width (so a negative index wraps through 2^64), the
 * four colours scaled and summed as ColorRGBAf, each step clamped at 0. */
static c3 tex_bilinear(const xo_texture *t, const float *tx, double u, double v)
{
    const uint64_t w = (uint64_t)t->width, h = (uint64_t)t->height;
    float fu = (float)(u * (double)w);
    float fv = (float)(v * (double)h);
    int32_t u1 = (int32_t)((uint64_t)(int64_t)f2i_x86(fu) % w);
    int32_t v1 = (int32_t)((uint64_t)(int64_t)f2i_x86(fv) % h);
    int32_t u2 = (int32_t)((uint64_t)(int64_t)(u1 + 1) % w);
    int32_t v2 = (int32_t)((uint64_t)(int64_t)(v1 + 1) % h);
    float fracu = fu - floorf(fu);
    float fracv = fv - floorf(fv);
    float w1 = (1 - fracu) * (1 - fracv);
    float w2 = fracu * (1 - fracv);
    float w3 = (1 - fracu) * fracv;
    float w4 = fracu * fracv;
    const float *a = texel(t, tx, (uint64_t)u1, (uint64_t)v1), *b = texel(t, tx, (uint64_t)u2, (uint64_t)v1);
    const float *c = texel(t, tx, (uint64_t)u1, (uint64_t)v2), *d = texel(t, tx, (uint64_t)u2, (uint64_t)v2);
    c3 s = cadd(cadd(cadd(cmuls(C(a[0], a[1], a[2]), w1), cmuls(C(b[0], b[1], b[2]), w2)),
                     cmuls(C(c[0], c[1], c[2]), w3)), cmuls(C(d[0], d[1], d[2]), w4));
    return s;
}

/* Texture2D::sample, sampler_tex.cc:37-45 */
static c3 tex_sample(const xo_texture *t, const float *tx, double u, double v)
{
    return t->filtering == XO_FILTER_BILINEAR ? tex_bilinear(t, tx, u, v) : tex_nearest(t, tx, u, v);
}

/* ERP::sample, sampler_erp.cc:13-26 (angles rounded to float) */
static c3 erp_sample(const xo_texture *t, const float *tx, v3 tc)
{
    v3 dir = normalized(tc);
    float theta = (float)acos(dir.y);
    float phi = (float)atan2(dir.x, -dir.z);
    float u = (float)(0.5f + phi / XO_PI_DOUBLE);
    float v = (float)(theta / XO_PI);
    return tex_sample(t, tx, u, v);
}

/* Cubemap::sample, sampler_cubemap.cc:13-36: the face of the largest
 * component, u and v from the other two (faces in CUBEMAP_FACE order:
 * 0 left, 1 right, 2 top, 3 bottom, 4 front, 5 back). */
static c3 cube_sample(const xo_texture *faces, const float *tx, v3 tc)
{
    v3 dir = normalized(tc);
    int face = 2;
    float u = 0.f, v = 0.f;
    double ax = fabs(dir.x), ay = fabs(dir.y), az = fabs(dir.z);
    if ((ax >= ay) && (ax >= az)) {
        if (dir.x > 0.0f) { face = 1; u = (float)((dir.z / dir.x + 1.0f) * 0.5f); v = (float)(1.f - (dir.y / dir.x + 1.0f) * 0.5f); }
        else if (dir.x < 0.0f) { face = 0; u = (float)((dir.z / dir.x + 1.0f) * 0.5f); v = (float)((dir.y / dir.x + 1.0f) * 0.5f); }
    } else if ((ay >= ax) && (ay >= az)) {
        if (dir.y > 0.0f) { face = 2; u = (float)((dir.x / dir.y + 1.0f) * 0.5f); v = (float)(1.f - (dir.z / dir.y + 1.0f) * 0.5f); }
        else if (dir.y < 0.0f) { face = 3; u = (float)(1. - (dir.x / dir.y + 1.0f) * 0.5f); v = (float)(1.f - (dir.z / dir.y + 1.0f) * 0.5f); }
    } else if ((az >= ax) && (az >= ay)) {
        if (dir.z > 0.0f) { face = 5; u = (float)(1. - (dir.x / dir.z + 1.0f) * 0.5f); v = (float)(1.f - (dir.y / dir.z + 1.0f) * 0.5f); }
        else if (dir.z < 0.0f) { face = 4; u = (float)(1. - (dir.x / dir.z + 1.0f) * 0.5f); v = (float)((dir.y / dir.z + 1.0f) * 0.5f); }
    }
    return tex_sample(&faces[face], tx, u, v);
}

/* Gradient::sample, sampler_gradient.cc:11-17, on a direction or texcoord */
static c3 gradient_sample(const float a3[3], const float b3[3], v3 tc)
{
    v3 d = normalized(tc);
    float t = (float)(0.5f * d.y + 1.0);
    c3 a = C(a3[0], a3[1], a3[2]), b = C(b3[0], b3[1], b3[2]);
    return cadd(cmuls(a, (float)(1.0 - t)), cmuls(b, t));
}

static c3 sampler_eval(const xo_scene_desc *D, const xo_sampler *sm, v3 tc)
{
    switch (sm->kind) {
    case XO_SAMPLER_GRADIENT: return gradient_sample(sm->a, sm->b, tc);
    case XO_SAMPLER_TEXTURE: return tex_sample(&D->textures[sm->texture], D->texels, tc.x, tc.y);
    case XO_SAMPLER_ERP: return erp_sample(&D->textures[sm->texture], D->texels, tc);
    case XO_SAMPLER_CUBEMAP: return cube_sample(&D->textures[sm->texture], D->texels, tc);
    default: return C(sm->a[0], sm->a[1], sm->a[2]);
    }
}

/* IMaterial::get_sample, material.cc:65-70, at hit_record_t::texcoord (tu, tv,
 * 0); ch 0 diffuse, 1 specular, 2 emissive.  An absent sampler is black. */
static c3 mat_sample(const xo_scene_desc *D, int32_t mi, int ch, double tu, double tv)
{
    if (!D->mat_samplers) {
        const xo_material *m = &D->materials[mi];
        const float *c = ch == 0 ? m->diffuse : (ch == 1 ? m->specular : m->emissive);
        return C(c[0], c[1], c[2]);
    }
    return sampler_eval(D, &D->mat_samplers[3 * mi + ch], V(tu, tv, 0.0));
}

void xo_kat_texture(const xo_texture *t, const float *texels, double u, double v, float out[3])
{
    c3 c = tex_sample(t, texels, u, v);
    out[0] = c.r; out[1] = c.g; out[2] = c.b;
}

void xo_kat_erp(const xo_texture *t, const float *texels, const double d[3], float out[3])
{
    c3 c = erp_sample(t, texels, V(d[0], d[1], d[2]));
    out[0] = c.r; out[1] = c.g; out[2] = c.b;
}

void xo_kat_cubemap(const xo_texture *faces, const float *texels, const double d[3], float out[3])
{
    c3 c = cube_sample(faces, texels, V(d[0], d[1], d[2]));
    out[0] = c.r; out[1] = c.g; out[2] = c.b;
}

/* The material's three samples are resolved by the caller (samplers draw no
 * random numbers, so resolving all three changes nothing). */
static int sample_path_c(const xo_material *m, c3 dif, c3 spe, c3 emi, rng_t *r, v3 point, v3 normal,
                         v3 incident, hres *out)
{
    switch (m->type) {
    case XO_LAMBERT:   /* lambert.cc:30-40 */
        out->org = add(point, muls(normal, XO_EPS));
        out->dir = normalized(s_diffuse(r, normal));
        out->intensity = cmuls(dif, (float)dot(normal, out->dir));
        return 1;
    case XO_PHONG:     /* phong.cc:35-55 */
    case XO_BLINNPHONG: { /* blinnphong.cc:34-61 */
        out->org = add(point, muls(normal, XO_EPS));
        double s = m->reflectance;
        double k = prng(r, 0.0f, 1.0f);
        if (k > s) {
            out->intensity = dif;
            out->dir = s_diffuse(r, normal);
        } else {
            out->intensity = spe;
            double e = m->exponent;
            out->dir = s_lobe(r, normal, neg(incident), e);
            if (m->type == XO_BLINNPHONG) out->dir = normalized(out->dir);
        }
        return 1;
    }
    case XO_EMISSIVE:  /* emissive.cc:20-27 */
        out->intensity = emi;
        return 0;
    default:
        /* dielectric.cc:22-31 leaves the intensity at its default 0, so the path's
         * value is 0 whatever follows; the path is ended here instead of tracing
         * the refracted continuation (its rays are not counted). */
        out->intensity = C(0, 0, 0);
        return 0;
    }
}

static int sample_path(const xo_material *m, rng_t *r, v3 point, v3 normal, v3 incident, hres *out)
{
    return sample_path_c(m, C(m->diffuse[0], m->diffuse[1], m->diffuse[2]),
                         C(m->specular[0], m->specular[1], m->specular[2]),
                         C(m->emissive[0], m->emissive[1], m->emissive[2]), r, point, normal, incident, out);
}

static c3 environment(const xo_scene_desc *D, v3 dir)
{
    if (D->env_type == XO_ENV_COLOR) return C(D->env_a[0], D->env_a[1], D->env_a[2]);
    if (D->env_type == XO_ENV_GRADIENT) return gradient_sample(D->env_a, D->env_b, dir);
    if (D->env_type == XO_ENV_ERP) return erp_sample(&D->textures[D->env_texture], D->texels, dir);
    if (D->env_type == XO_ENV_CUBEMAP) return cube_sample(&D->textures[D->env_texture], D->texels, dir);
    return C(0, 0, 0);   /* scene.cc:142-145 */
}

/* pathtracer::Integrator::eval, integrator/pathtracer/integrator.cc:21-47 */
static c3 pt_eval(const xo_scene *s, size_t depth, c3 in_int, v3 o, v3 d, rng_t *r, uint64_t *rays)
{
    if (depth == 0) return C(0, 0, 0);
    hrec h;
    int32_t oi, pi;
    ++*rays;
    int hit = scene_hit(s, o, d, &h, &oi, &pi);
    if (hit) {
        const int32_t mi = s->d.obj_material[oi];
        const xo_material *m = &s->d.materials[mi];
        hres res;
        res.org = V(0, 0, 0);
        res.dir = V(0, 0, 1);
        res.intensity = C(0, 0, 0);
        int cont = sample_path_c(m, mat_sample(&s->d, mi, 0, h.tu, h.tv), mat_sample(&s->d, mi, 1, h.tu, h.tv),
                                 mat_sample(&s->d, mi, 2, h.tu, h.tv), r, h.point, h.normal, d, &res);
        c3 value = cmul(in_int, res.intensity);
        if (cont) value = cmul(value, pt_eval(s, depth - 1, res.intensity, res.org, res.dir, r, rays));
        return value;
    }
    return environment(&s->d, d);
}

static int render_impl(const xo_scene *s, const xo_render_params *p, int64_t npix, const int32_t *px,
                       float *rgba, uint64_t *rays, double *raygraph);

int xo_render(const xo_scene *s, const xo_render_params *p, int64_t npix, const int32_t *px,
              float *rgba, uint64_t *rays)
{
    return render_impl(s, p, npix, px, rgba, rays, NULL);
}

/* The depth integrator with the raygraph it records (depth/integrator.cc:
 * 43-51): per sample, in pixel then sample order, the ray origin, the hit
 * point ((0,0,0) on a miss: Scene::intersection copies a default record,
 * scene.cc:212) and the pixel's colour after the sample: 10 doubles. */
int xo_render_raygraph(const xo_scene *s, const xo_render_params *p, int64_t npix, const int32_t *px,
                       float *rgba, double *raygraph, uint64_t *rays)
{
    xo_render_params q = *p;
    q.integrator = XO_DEPTH;
    return render_impl(s, &q, npix, px, rgba, rays, raygraph);
}

static int render_impl(const xo_scene *s, const xo_render_params *p, int64_t npix, const int32_t *px,
                       float *rgba, uint64_t *rays, double *raygraph)
{
    const xo_scene_desc *D = &s->d;
    uint64_t nr = 0;
    /* aa.cc:7-48, 51-77: per pixel P positions, each taken spp times: the
     * grid's aa^2 (rows of the grid in order) or the random distribution's aa
     * jittered ones; weight 1/P as a float, times 1/spp */
    const int random = p->distribution == XO_SAMPLES_RANDOM;
    const int32_t L = p->aa > 1 ? p->aa : 1;
    const int32_t P = random ? L : L * L;
    double weight = P == 1 ? 1.f : (double)(1.f / (float)P);
    weight *= 1. / (double)p->spp;
    const float sub_pixel = 1.f / (float)L, offset = sub_pixel * 0.5f;
    for (int64_t i = 0; i < npix; ++i) {
        int32_t x = px[2 * i], y = px[2 * i + 1];
        float col[4] = {0, 0, 0, 0};
        for (int32_t si = 0; si < P * p->spp; ++si) {
            rng_t r;
            memset(&r, 0, sizeof(r));
            r.kind = XO_RNG_STREAM;
            r.key = xo_path_key(p->seed, (uint64_t)si * (uint64_t)p->width * (uint64_t)p->height +
                                             (uint64_t)y * (uint64_t)p->width + (uint64_t)x);
            const int32_t gi = si / p->spp;   /* position of the sample */
            double cx = (double)x + 0.5f, cy = (double)y + 0.5f;
            if (random) {
                /* gen_samples_random (aa.cc:34-48): pixel + (float)prng_c(0, 1) per axis */
                const uint64_t jk = xo_jitter_key(p->seed, gi, p->width, p->height, x, y);
                cx = (double)x + (double)(float)xo_stream_uniform(jk, 0);
                cy = (double)y + (double)(float)xo_stream_uniform(jk, 1);
            } else if (L > 1) {
                cx = ((double)x + (double)(gi % L) * (double)sub_pixel) + (double)offset;
                cy = ((double)y + (double)(gi / L) * (double)sub_pixel) + (double)offset;
            }
            double o[3], d[3];
            camera_any(D, &r, (float)cx, (float)cy, (float)p->width, (float)p->height, o, d);
            v3 O = V(o[0], o[1], o[2]), Dd = V(d[0], d[1], d[2]);
            hrec h;
            int32_t oi, pi;
            if (p->integrator == XO_STENCIL) {          /* stencil/integrator.cc:13-33 */
                ++nr;
                if (scene_hit(s, O, Dd, &h, &oi, &pi)) {
                    col[0] = col[1] = col[2] = 1.f;
                    col[3] = clamp01((float)(col[3] + weight));
                }
            } else if (p->integrator == XO_DEPTH) {     /* depth/integrator.cc:15-54 */
                ++nr;
                float depth = 0.f;
                const int dhit = scene_hit(s, O, Dd, &h, &oi, &pi);
                if (dhit) {
                    depth = (float)(1. / log(length(sub(O, h.point))));
                    depth = (float)(col[0] + depth * weight);
                    col[0] = col[1] = col[2] = clamp0(depth);
                    col[3] = 1;
                }
                col[3] = 1;
                if (raygraph) {
                    double *rg = raygraph + 10 * (i * (int64_t)P * p->spp + si);
                    rg[0] = O.x; rg[1] = O.y; rg[2] = O.z;
                    rg[3] = dhit ? h.point.x : 0.0; rg[4] = dhit ? h.point.y : 0.0; rg[5] = dhit ? h.point.z : 0.0;
                    for (int k = 0; k < 4; ++k) rg[6 + k] = col[k];
                }
            } else if (p->integrator == XO_AO) {        /* ao/integrator.cc:14-52 */
                v3 acc = V(col[0], col[1], col[2]);
                float w = 1.0f;
                ++nr;
                if (scene_hit(s, O, Dd, &h, &oi, &pi)) {
                    v3 ad = s_hemisphere(&r, h.normal, h.normal);
                    v3 ao = add(h.point, muls(h.normal, XO_EPS));
                    hrec h2;
                    ++nr;
                    if (scene_hit(s, ao, ad, &h2, &oi, &pi)) {
                        float dist = (float)length(sub(h2.point, ao));
                        /* nmath::min works in scalar_t (lib/nmath/mutil.inl:44) */
                        double md = (double)p->ao_max_distance;
                        double mn = (md > (double)dist ? (double)dist : md);
                        w = (float)(mn / md);
                    }
                }
                acc = V(acc.x + w * weight, acc.y + w * weight, acc.z + w * weight);
                col[0] = clamp0((float)acc.x);
                col[1] = clamp0((float)acc.y);
                col[2] = clamp0((float)acc.z);
                col[3] = 1.f;
            } else if (p->integrator == XO_NORMAL) {    /* normal/integrator.cc:10-39 */
                v3 acc = V(col[0], col[1], col[2]);
                acc = V(acc.x * 2.0f - 1.0f, acc.y * 2.0f - 1.0f, acc.z * 2.0f - 1.0f);
                ++nr;
                if (scene_hit(s, O, Dd, &h, &oi, &pi)) {
                    v3 nw = muls(add(h.normal, acc), 0.5f);
                    v3 u = normalized(nw);
                    acc = V((u.x + 1.0f) * 0.5f, (u.y + 1.0f) * 0.5f, (u.z + 1.0f) * 0.5f);
                }
                col[0] = clamp0((float)acc.x);
                col[1] = clamp0((float)acc.y);
                col[2] = clamp0((float)acc.z);
                col[3] = 1.f;
            } else if (p->integrator == XO_UV) {        /* uv/integrator.cc:10-42 */
                v3 acc = V(col[0], col[1], col[2]);
                double alpha = col[3], alpha_sample = 0.f;
                ++nr;
                if (scene_hit(s, O, Dd, &h, &oi, &pi)) {
                    /* hit_record_t::texcoord is a Vector3f with z = 0 (hitrecord.h:33),
                     * so the blue channel gains (0 * 0.5 + 0.5) * weight */
                    acc = V(acc.x + (h.tu * 0.5f + 0.5f) * weight, acc.y + (h.tv * 0.5f + 0.5f) * weight,
                            acc.z + (0.0 * 0.5f + 0.5f) * weight);
                    alpha_sample += weight;
                }
                col[0] = clamp0((float)acc.x);
                col[1] = clamp0((float)acc.y);
                col[2] = clamp0((float)acc.z);
                col[3] = clamp01((float)(alpha + weight * alpha_sample));
            } else if (p->integrator == XO_EMISSION) {  /* emission/integrator.cc:10-38 */
                ++nr;
                if (scene_hit(s, O, Dd, &h, &oi, &pi)) {
                    c3 e = cmuls(mat_sample(D, D->obj_material[oi], 2, h.tu, h.tv), (float)weight);
                    col[0] = clamp0(col[0] + e.r);
                    col[1] = clamp0(col[1] + e.g);
                    col[2] = clamp0(col[2] + e.b);
                }
                col[3] = 1.f;
            } else if (p->integrator == XO_WIREFRAME) { /* wireframe/integrator.cc:10-35 */
                ++nr;
                if (scene_hit(s, O, Dd, &h, &oi, &pi)) {
                    col[0] = col[1] = col[2] = 1.f;
                    col[3] = clamp01((float)(col[3] + weight));
                }
            } else {                                    /* pathtracer/integrator.cc:49-74 */
                c3 v = pt_eval(s, (size_t)p->rdepth, C(1, 1, 1), O, Dd, &r, &nr);
                c3 add_ = cmuls(v, (float)weight);
                col[0] = clamp0(col[0] + add_.r);
                col[1] = clamp0(col[1] + add_.g);
                col[2] = clamp0(col[2] + add_.b);
                col[3] = 1;
            }
        }
        memcpy(rgba + 4 * i, col, sizeof(col));
    }
    if (rays) *rays = nr;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Known-answer hooks                                                         */
static void put_hit(int ok, const hrec *h, double out[7])
{
    out[0] = ok ? h->t : 0;
    out[1] = ok ? h->point.x : 0; out[2] = ok ? h->point.y : 0; out[3] = ok ? h->point.z : 0;
    out[4] = ok ? h->normal.x : 0; out[5] = ok ? h->normal.y : 0; out[6] = ok ? h->normal.z : 0;
}

int xo_kat_sphere(const double sph[4], const double o[3], const double d[3], double out[7])
{
    hrec h;
    const double usc[2] = {0.0, 0.0};
    int ok = hit_sphere(V(sph[0], sph[1], sph[2]), sph[3], usc, V(o[0], o[1], o[2]), V(d[0], d[1], d[2]), &h);
    put_hit(ok, &h, out);
    return ok;
}

int xo_kat_plane(const double pl[4], const double o[3], const double d[3], double out[7])
{
    hrec h;
    const double usc[2] = {0.0, 0.0};
    int ok = hit_plane(V(pl[0], pl[1], pl[2]), pl[3], usc, V(o[0], o[1], o[2]), V(d[0], d[1], d[2]), &h);
    put_hit(ok, &h, out);
    return ok;
}

int xo_kat_triangle(const double v[9], const double n[9], const double o[3], const double d[3], double out[7])
{
    v3 tv[3] = {V(v[0], v[1], v[2]), V(v[3], v[4], v[5]), V(v[6], v[7], v[8])};
    v3 tn[3] = {V(n[0], n[1], n[2]), V(n[3], n[4], n[5]), V(n[6], n[7], n[8])};
    hrec h;
    const v3 tt[3] = {V(0, 0, 0), V(0, 0, 0), V(0, 0, 0)};
    int ok = hit_triangle(tv, tn, tt, V(o[0], o[1], o[2]), V(d[0], d[1], d[2]), &h);
    put_hit(ok, &h, out);
    return ok;
}

int xo_kat_aabb(const double mn[3], const double mx[3], const double o[3], const double d[3])
{
    /* AABB3(a, b) orders the corners (aabb.cc:21-25) */
    v3 a = V(mn[0], mn[1], mn[2]), b = V(mx[0], mx[1], mx[2]);
    return hit_aabb(vmin(a, b), vmax(a, b), V(o[0], o[1], o[2]), V(d[0], d[1], d[2]));
}

static rng_t table_rng(const int32_t *table, int32_t rand_max)
{
    rng_t r;
    memset(&r, 0, sizeof(r));
    r.kind = XO_RNG_TABLE;
    r.table = table;
    r.rand_max = rand_max;
    return r;
}

void xo_kat_hemisphere(const int32_t *table, int32_t rand_max, const double n[3], double out[3])
{
    rng_t r = table_rng(table, rand_max);
    v3 v = s_hemisphere(&r, V(n[0], n[1], n[2]), V(n[0], n[1], n[2]));
    out[0] = v.x; out[1] = v.y; out[2] = v.z;
}

void xo_kat_diffuse(const int32_t *table, int32_t rand_max, const double n[3], double out[3])
{
    rng_t r = table_rng(table, rand_max);
    v3 v = s_diffuse(&r, V(n[0], n[1], n[2]));
    out[0] = v.x; out[1] = v.y; out[2] = v.z;
}

void xo_kat_lobe(const int32_t *table, int32_t rand_max, const double n[3], const double d[3], double e, double out[3])
{
    rng_t r = table_rng(table, rand_max);
    v3 v = s_lobe(&r, V(n[0], n[1], n[2]), V(d[0], d[1], d[2]), e);
    out[0] = v.x; out[1] = v.y; out[2] = v.z;
}

int xo_kat_material(const xo_material *m, const int32_t *table, int32_t rand_max, const double p[3],
                    const double n[3], const double inc[3], double out[9])
{
    rng_t r = table_rng(table, rand_max);
    hres res;
    res.org = V(0, 0, 0);
    res.dir = V(0, 0, 1);
    res.intensity = C(0, 0, 0);
    int cont = sample_path(m, &r, V(p[0], p[1], p[2]), V(n[0], n[1], n[2]), V(inc[0], inc[1], inc[2]), &res);
    out[0] = res.org.x; out[1] = res.org.y; out[2] = res.org.z;
    out[3] = res.dir.x; out[4] = res.dir.y; out[5] = res.dir.z;
    out[6] = res.intensity.r; out[7] = res.intensity.g; out[8] = res.intensity.b;
    return cont;
}

void xo_kat_gradient(const float a[3], const float b[3], const double d[3], float out[3])
{
    xo_scene_desc D;
    memset(&D, 0, sizeof(D));
    D.env_type = XO_ENV_GRADIENT;
    memcpy(D.env_a, a, sizeof(D.env_a));
    memcpy(D.env_b, b, sizeof(D.env_b));
    c3 c = environment(&D, V(d[0], d[1], d[2]));
    out[0] = c.r; out[1] = c.g; out[2] = c.b;
}
