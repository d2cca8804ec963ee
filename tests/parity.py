"""Helpers shared by the parity tests: primitive bookkeeping and the FP64
classification of GPU/reference disagreements (tie, grazing, or GPU error)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from oracle import pyoracle as po
from xtracer_b200 import scenes


def P(a):
    return np.ascontiguousarray(a, np.float64).ctypes.data_as(C.c_void_p)


def global_prim(spec, obj, prim_in_obj_or_global, is_mesh_local=True):
    """Global primitive id (triangles, then spheres, then planes) of an object hit."""
    kind = spec.obj_kind[obj]
    first = spec.obj_first[obj]
    if kind == scenes.MESH:
        return int(first + prim_in_obj_or_global) if is_mesh_local else int(prim_in_obj_or_global)
    if kind == scenes.SPHERE:
        return spec.n_tris + int(first)
    return spec.n_tris + spec.spheres.shape[0] + int(first)


def oracle_global_prim(spec, obj, prim):
    """xo_trace returns prim = triangle index (global) for meshes, sphere/plane
    index otherwise; convert to the GPU's global id."""
    out = np.full(obj.shape, -1, np.int64)
    for i in range(obj.size):
        o = obj[i]
        if o < 0:
            continue
        k = spec.obj_kind[o]
        if k == scenes.MESH:
            out[i] = prim[i]
        elif k == scenes.SPHERE:
            out[i] = spec.n_tris + prim[i]
        else:
            out[i] = spec.n_tris + spec.spheres.shape[0] + prim[i]
    return out


def ref_t_of(spec, gid, o, d):
    """(hit, t, margin) of the reference's FP64 test of primitive gid; margin is
    the smallest barycentric (triangles) or relative discriminant (spheres)."""
    L = po.lib()
    out = np.zeros(7)
    nt, ns = spec.n_tris, spec.spheres.shape[0]
    if gid < nt:
        v = spec.tris[gid].astype(np.float64).ravel()
        n = np.zeros(9) if spec.tri_normals is None else spec.tri_normals[gid].astype(np.float64).ravel()
        h = L.xo_kat_triangle(P(v), P(n), P(o), P(d), P(out))
        # watertight FP64 barycentric margin at the ray's crossing of the plane
        V = v.reshape(3, 3)
        e1, e2 = V[1] - V[0], V[2] - V[0]
        pv = np.cross(d, e2)
        det = e1 @ pv
        if abs(det) < 1e-300:
            return h, out[0], 0.0
        tv = o - V[0]
        u = (tv @ pv) / det
        qv = np.cross(tv, e1)
        w = (d @ qv) / det
        margin = min(u, w, 1 - u - w)
        return h, out[0], margin
    if gid < nt + ns:
        s = spec.spheres[gid - nt].astype(np.float64)
        h = L.xo_kat_sphere(P(s), P(o), P(d), P(out))
        f = o - s[:3]
        b = f @ d
        disc = b * b - (f @ f - s[3] ** 2)
        return h, out[0], disc / max(s[3] ** 2, 1e-300)
    pl = spec.planes[gid - nt - ns].astype(np.float64)
    h = L.xo_kat_plane(P(pl), P(o), P(d), P(out))
    return h, out[0], abs(pl[:3] @ d)


def classify(spec, org, dirs, g_hit, g_gid, g_t, r_hit, r_gid, r_t, tie_rel=1e-5, graze=1e-5):
    """Returns (n_agree, n_tie, n_graze, unexplained_indices) over all rays."""
    agree = (g_hit == r_hit) & ((g_hit == 0) | (g_gid == r_gid))
    tie = graze_n = 0
    bad = []
    for i in np.nonzero(~agree)[0]:
        o, d = org[i], dirs[i]
        if g_hit[i] and r_hit[i]:
            h, t_alt, m = ref_t_of(spec, int(g_gid[i]), o, d)
            if h and abs(t_alt - r_t[i]) <= tie_rel * r_t[i]:
                tie += 1
                continue
            _, _, mg = ref_t_of(spec, int(g_gid[i]), o, d)
            _, _, mr = ref_t_of(spec, int(r_gid[i]), o, d)
            if abs(mg) < graze or abs(mr) < graze:
                graze_n += 1
                continue
            bad.append(i)
        else:
            gid = int(g_gid[i]) if g_hit[i] else int(r_gid[i])
            _, _, m = ref_t_of(spec, gid, o, d)
            if abs(m) < graze:
                graze_n += 1
            else:
                bad.append(i)
    return int(agree.sum()), tie, graze_n, bad


def random_distribution_agreement(R, O, channel, aa=None):
    """Checks frames of the random sample distribution (aa.cc:34-48) from two
    sources of jitter offsets against each other: R, the reference's frames at
    several seeds (libc rand()), and O, frames from this library's stream at as
    many seeds, both (seeds, pixels, 4) in the same pixel order.

    * the frame mean of `channel` agrees within 4.5 standard errors (the
      per-pixel variance across seeds of both sides);
    * the per-pixel mean over seeds differs between the sources by at most 1.5
      times what it differs between two halves of the seeds of one source;
    * for stencil (channel 3, given aa): every coverage value is a multiple of
      1/aa (each position's spp samples see the same ray), the sources use the
      same values, and the fraction of partly covered pixels agrees within
      4.5 binomial standard errors."""
    r = np.asarray(R, np.float64)[..., channel]
    o = np.asarray(O, np.float64)[..., channel]
    n, npix = r.shape
    assert o.shape == r.shape
    se = np.sqrt((r.var(0, ddof=1).sum() + o.var(0, ddof=1).sum()) / n) / npix
    assert abs(r.mean() - o.mean()) <= 4.5 * se + 1e-6, (r.mean(), o.mean(), se)
    h = n // 2
    split = 0.5 * (np.abs(r[:h].mean(0) - r[h:].mean(0)).mean() + np.abs(o[:h].mean(0) - o[h:].mean(0)).mean())
    cross = np.abs(r.mean(0) - o.mean(0)).mean()
    assert cross <= 1.5 * split + 1e-6, (cross, split)
    if aa is not None:
        for x in (r, o):
            k = x * aa
            assert np.allclose(k, np.round(k), atol=1e-5), np.unique(x)
        assert set(np.round(r * aa).astype(int).ravel()) == set(np.round(o * aa).astype(int).ravel())
        pr, po_ = ((r > 0) & (r < 1)).mean(), ((o > 0) & (o < 1)).mean()
        p = 0.5 * (pr + po_)
        assert abs(pr - po_) <= 4.5 * np.sqrt(p * (1 - p) * 2.0 / r.size) + 1e-9, (pr, po_)


def rmse(a, b):
    """Per-pixel RMSE over the colour channels of two (npix, 4) frames."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a[:, :3] - b[:, :3]) ** 2)))


def converged_rmse_bar(frames, truth, ref_rmse, label="", tol=1.05):
    """The stochastic bar as the hot-path contract words it: per-pixel RMSE
    against a 4096-spp render must sit within the sampling noise of the
    reference CPU renderer at equal spp.

    frames: (k >= 2, npix, 4) frames under test at that spp (different seeds);
    truth: (npix, 4) the converged render; ref_rmse: the reference's own RMSE
    against the same truth, one per reference seed.  Asserts
    * the mean RMSE of the frames <= (tol + 3 cv) x the largest reference
      RMSE, where cv is the relative spread of the reference's RMSEs between
      its seeds (at least 1 %): the noise estimate is itself a sample, whose
      spread runs from 1-3 % on busy frames to 25 % where few pixels vary;
    * per channel, the frames' mean minus the truth's mean within 4.5 standard
      errors (from the per-pixel variance between the frames).
    Prints and returns (mean RMSE, reference RMSEs)."""
    F = np.asarray(frames, np.float64)
    T = np.asarray(truth, np.float64)
    k, npix = F.shape[0], F.shape[1]
    assert k >= 2
    got = [rmse(F[i], T) for i in range(k)]
    ref = [float(x) for x in np.asarray(ref_rmse).ravel()]
    cv = max(0.01, float(np.std(ref, ddof=1) / np.mean(ref))) if len(ref) > 1 else 0.01
    bar = tol + 3.0 * cv
    print("[%s] RMSE vs 4096-spp: frames %s, reference %s, ratio %.3f (bar %.3f x max)" %
          (label, np.round(got, 5), np.round(ref, 5), np.mean(got) / max(ref), bar))
    assert np.mean(got) <= bar * max(ref), (got, ref, bar)
    for ch in range(3):
        se = np.sqrt(F[:, :, ch].var(0, ddof=1).mean() / npix / k)
        bias = F[:, :, ch].mean() - T[:, ch].mean()
        assert abs(bias) <= 4.5 * se + 1e-6, (label, ch, bias, se)
    return float(np.mean(got)), ref


def same_stream_bar(gpu, oracle, oracle_other, label="", frac=0.25):
    """GPU (FP32) and oracle (FP64) frames drawn from the same random stream
    differ only where rounding sends a path another way: an edge or grazing
    hit, a tie between primitives, a secondary ray's origin offset.  Bar: the
    RMSE between them is at most `frac` of one frame's sampling noise at that
    spp, measured as the RMSE between the oracle's frames at two seeds over
    sqrt(2); the divergence then adds at most frac^2 to the frame's variance.
    Prints the ratio and the share of pixels equal within 1e-3."""
    g = np.asarray(gpu, np.float64).reshape(-1, 4)
    o = np.asarray(oracle, np.float64).reshape(-1, 4)
    o2 = np.asarray(oracle_other, np.float64).reshape(-1, 4)
    noise = rmse(o, o2) / np.sqrt(2.0)
    div = rmse(g, o)
    same = float(np.mean(np.abs(g[:, :3] - o[:, :3]).max(axis=1) < 1e-3))
    print("[%s] same stream: RMSE(gpu, oracle) %.3g = %.3f of the noise %.3g (bar %.2f); %.4f of pixels within 1e-3"
          % (label, div, div / max(noise, 1e-30), noise, frac, same))
    assert div <= frac * noise, (label, div, noise)
    return div / max(noise, 1e-30), same
