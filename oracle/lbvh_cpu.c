/*
 * lbvh_cpu.c — CPU re-implementation of the GPU BVH build's deterministic steps
 * (xtracer_b200/csrc/bvh.cu): primitive boxes, 30-bit Morton codes, stable sort,
 * Karras hierarchy, and the PLOC hierarchy with its depth-first leaf order.
 * TEST INFRASTRUCTURE: the GPU build must reproduce these arrays bit for bit.  The reference renderer has no BVH (its BVH file,
 * src/xtcore/bvh.cc, is commented out); this checks the new builder only.
 *
 * Float steps use the same operations as the device code, in round-to-nearest
 * (gcc -O2 without -march: SSE, no contraction); sphere boxes are rounded
 * outward like __fsub_rd/__fadd_ru.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

static float round_down(double d) { float f = (float)d; if ((double)f > d) f = nextafterf(f, -INFINITY); return f; }
static float round_up(double d)   { float f = (float)d; if ((double)f < d) f = nextafterf(f, INFINITY); return f; }

static void prim_box(int i, int n_tris, const float *tris, const float *sph, float lo[3], float hi[3])
{
    if (i < n_tris) {
        const float *t = tris + 9 * (size_t)i;
        for (int a = 0; a < 3; ++a) {
            float x = t[a], y = t[3 + a], z = t[6 + a];
            lo[a] = fminf(fminf(x, y), z);
            hi[a] = fmaxf(fmaxf(x, y), z);
        }
    } else {
        const float *s = sph + 4 * (size_t)(i - n_tris);
        for (int a = 0; a < 3; ++a) {
            lo[a] = round_down((double)s[a] - (double)s[3]);
            hi[a] = round_up((double)s[a] + (double)s[3]);
        }
    }
}

static uint32_t expand10(uint32_t v)
{
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

static uint32_t quant10(float c, float lo, float scale)
{
    float q = (c - lo) * scale;
    uint32_t u = (uint32_t)q;
    return u > 1023u ? 1023u : u;
}

typedef struct { uint32_t key, idx; } kv;
static int cmp_kv(const void *a, const void *b)
{
    const kv *x = (const kv *)a, *y = (const kv *)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

static int delta(const uint32_t *k, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    uint32_t a = k[i], b = k[j];
    return a != b ? __builtin_clz(a ^ b) : 32 + __builtin_clz((uint32_t)(i ^ j));
}

/* Outputs (caller-allocated): keys[n] sorted Morton codes, order[n] sorted
 * primitive ids, left/right[n-1] child refs (>= 0 internal, < 0 leaf ~index). */
int xo_lbvh_build(int n_tris, const float *tris, int n_sph, const float *sph,
                  uint32_t *keys, uint32_t *order, int32_t *left, int32_t *right)
{
    int n = n_tris + n_sph;
    if (n <= 0) return 0;
    float (*lo)[3] = malloc(sizeof(float[3]) * (size_t)n), (*hi)[3] = malloc(sizeof(float[3]) * (size_t)n);
    float cmn[3] = {INFINITY, INFINITY, INFINITY}, cmx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < n; ++i) {
        prim_box(i, n_tris, tris, sph, lo[i], hi[i]);
        for (int a = 0; a < 3; ++a) {
            float c = (lo[i][a] + hi[i][a]) * 0.5f;
            cmn[a] = fminf(cmn[a], c);
            cmx[a] = fmaxf(cmx[a], c);
        }
    }
    float sc[3];
    for (int a = 0; a < 3; ++a) {
        float e = cmx[a] - cmn[a];
        sc[a] = e > 0.f ? 1024.0f / e : 0.f;
    }
    kv *v = malloc(sizeof(kv) * (size_t)n);
    for (int i = 0; i < n; ++i) {
        float c[3];
        for (int a = 0; a < 3; ++a) c[a] = (lo[i][a] + hi[i][a]) * 0.5f;
        v[i].key = (expand10(quant10(c[0], cmn[0], sc[0])) << 2) | (expand10(quant10(c[1], cmn[1], sc[1])) << 1) |
                   expand10(quant10(c[2], cmn[2], sc[2]));
        v[i].idx = (uint32_t)i;
    }
    qsort(v, (size_t)n, sizeof(kv), cmp_kv);
    for (int i = 0; i < n; ++i) { keys[i] = v[i].key; order[i] = v[i].idx; }
    free(v); free(lo); free(hi);
    /* Karras 2012 */
    for (int i = 0; i < n - 1; ++i) {
        int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
        int dmin = delta(keys, n, i, i - d);
        int lmax = 2;
        while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
        int j = i + l * d;
        int dnode = delta(keys, n, i, j);
        int s = 0, t = l;
        do {
            t = (t + 1) >> 1;
            if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
        } while (t > 1);
        int g = i + s * d + (d < 0 ? d : 0);
        int mn = i < j ? i : j, mx = i < j ? j : i;
        left[i] = (mn == g) ? ~g : g;
        right[i] = (mx == g + 1) ? ~(g + 1) : g + 1;
    }
    return 0;
}

/* PLOC (Meister and Bittner, TVCG 2018) as the GPU runs it (bvh.cu k_ploc_*):
 * clusters in Morton order; per iteration each cluster's nearest neighbour
 * within PLOC_R positions by the half surface area of the merged box (operation
 * by operation in float; ties to nearer positions, then pairs starting at an
 * even position, then the lower position); mutual pairs merge at
 * the lower position into inner node base-1-rank (rank = position order of the
 * merges of the iteration); survivors compacted in order.  Then the leaves are
 * renumbered in depth-first order (left before right) and keys, order and the
 * leaf references follow. */
#define PLOC_R 16
static float half_area(const float alo[3], const float ahi[3], const float blo[3], const float bhi[3])
{
    float dx = fmaxf(ahi[0], bhi[0]) - fminf(alo[0], blo[0]);
    float dy = fmaxf(ahi[1], bhi[1]) - fminf(alo[1], blo[1]);
    float dz = fmaxf(ahi[2], bhi[2]) - fminf(alo[2], blo[2]);
    float a = dx * dy;
    float b = dy * dz;
    float c = dz * dx;
    return (a + b) + c;
}

int xo_ploc_build(int n_tris, const float *tris, int n_sph, const float *sph,
                  uint32_t *keys, uint32_t *order, int32_t *left, int32_t *right)
{
    int n = n_tris + n_sph;
    if (n <= 0) return 0;
    int32_t *tl = malloc(sizeof(int32_t) * (size_t)(n > 1 ? n - 1 : 1));
    int32_t *tr = malloc(sizeof(int32_t) * (size_t)(n > 1 ? n - 1 : 1));
    /* the Morton order of the LBVH build */
    xo_lbvh_build(n_tris, tris, n_sph, sph, keys, order, tl, tr);
    if (n == 1) { free(tl); free(tr); return 0; }
    float (*clo)[3] = malloc(sizeof(float[3]) * (size_t)n), (*chi)[3] = malloc(sizeof(float[3]) * (size_t)n);
    float (*olo)[3] = malloc(sizeof(float[3]) * (size_t)n), (*ohi)[3] = malloc(sizeof(float[3]) * (size_t)n);
    int32_t *cid = malloc(sizeof(int32_t) * (size_t)n), *oid = malloc(sizeof(int32_t) * (size_t)n);
    int32_t *nn = malloc(sizeof(int32_t) * (size_t)n), *cnt = malloc(sizeof(int32_t) * (size_t)n);
    int32_t *pint = malloc(sizeof(int32_t) * (size_t)n), *pleaf = malloc(sizeof(int32_t) * (size_t)n);
    for (int i = 0; i < n; ++i) {
        prim_box((int)order[i], n_tris, tris, sph, clo[i], chi[i]);
        cid[i] = ~i;
    }
    for (int i = 0; i < n - 1; ++i) pint[i] = -1;
    int m = n, base = n - 1, rc = 0;
    while (m > 1) {
        for (int i = 0; i < m; ++i) {
            float best = INFINITY;
            uint64_t bkey = ~0ull;
            int bj = -1;
            for (int o = -PLOC_R; o <= PLOC_R; ++o) {
                int j = i + o;
                if (o == 0 || j < 0 || j >= m) continue;
                float a = half_area(clo[i], chi[i], clo[j], chi[j]);
                /* ties: nearer positions, then pairs at an even position, then lower */
                uint32_t lo = (uint32_t)(i < j ? i : j), d = (uint32_t)(o < 0 ? -o : o);
                uint64_t key = ((uint64_t)d << 33) | ((uint64_t)(lo & 1u) << 32) | lo;
                if (a < best || (a == best && key < bkey)) { best = a; bkey = key; bj = j; }
            }
            nn[i] = bj;
        }
        int merges = 0, pos = 0;
        for (int i = 0; i < m; ++i) {
            int j = nn[i];
            int mutual = j >= 0 && nn[j] == i;
            if (mutual && i > j) continue;
            if (!mutual) {
                for (int a = 0; a < 3; ++a) { olo[pos][a] = clo[i][a]; ohi[pos][a] = chi[i][a]; }
                oid[pos++] = cid[i];
                continue;
            }
            int k = base - 1 - merges++;
            int32_t a_ = cid[i], b_ = cid[j];
            tl[k] = a_;
            tr[k] = b_;
            cnt[k] = (a_ < 0 ? 1 : cnt[a_]) + (b_ < 0 ? 1 : cnt[b_]);
            if (a_ < 0) pleaf[~a_] = k; else pint[a_] = k;
            if (b_ < 0) pleaf[~b_] = k; else pint[b_] = k;
            for (int a = 0; a < 3; ++a) {
                olo[pos][a] = fminf(clo[i][a], clo[j][a]);
                ohi[pos][a] = fmaxf(chi[i][a], chi[j][a]);
            }
            oid[pos++] = k;
        }
        if (merges == 0) { rc = 1; break; }
        base -= merges;
        m = pos;
        float (*t3)[3] = clo; clo = olo; olo = t3;
        t3 = chi; chi = ohi; ohi = t3;
        int32_t *ti = cid; cid = oid; oid = ti;
    }
    if (!rc) {
        /* leaf offsets in depth-first order */
        int32_t *newpos = malloc(sizeof(int32_t) * (size_t)n);
        for (int i = 0; i < n; ++i) {
            int32_t child = ~i, node = pleaf[i];
            int off = 0;
            for (;;) {
                if (tr[node] == child) off += tl[node] < 0 ? 1 : cnt[tl[node]];
                if (node == 0) break;
                child = node;
                node = pint[node];
            }
            newpos[i] = off;
        }
        uint32_t *k2 = malloc(sizeof(uint32_t) * (size_t)n), *o2 = malloc(sizeof(uint32_t) * (size_t)n);
        for (int i = 0; i < n; ++i) { k2[newpos[i]] = keys[i]; o2[newpos[i]] = order[i]; }
        for (int i = 0; i < n; ++i) { keys[i] = k2[i]; order[i] = o2[i]; }
        for (int i = 0; i < n - 1; ++i) {
            left[i] = tl[i] < 0 ? ~newpos[~tl[i]] : tl[i];
            right[i] = tr[i] < 0 ? ~newpos[~tr[i]] : tr[i];
        }
        free(k2); free(o2); free(newpos);
    }
    free(clo); free(chi); free(olo); free(ohi); free(cid); free(oid); free(nn); free(cnt); free(pint);
    free(pleaf); free(tl); free(tr);
    return rc;
}
