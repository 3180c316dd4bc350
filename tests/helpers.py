"""Comparison helpers shared by the parity tests.

The gates restate the reference's own: block sets exact
(cpp/tests/test_cuda_analytic.cu:244-245), vertex counts within 1 % (:247-249),
symmetric surface distance with stride-8 queries, mean < voxel/100 and
Hausdorff < voxel/10 (:251-283), analytic sphere error mean < voxel/4 and
max < voxel (cpp/tests/test_analytic.cpp:86-104).
"""
from __future__ import annotations

import numpy as np

TSDF_TOL = 1e-5  # mean TSDF (tsdf_sum / weight), FP32; the bar for float parity


def sorted_voxels(vol):
    """(coords, tsdf, weight, r, g, b) with blocks sorted by coordinate."""
    coords, *arrs = vol.voxels()
    order = np.lexsort(coords.T[::-1]) if coords.shape[0] else np.zeros(0, dtype=np.int64)
    return (coords[order], *(a[order] for a in arrs))


def assert_same_blocks(gpu, ref):
    g = gpu.coords()
    r = ref.coords()
    assert g.shape == r.shape, f"block counts differ: gpu {g.shape[0]} oracle {r.shape[0]}"
    gs = g[np.lexsort(g.T[::-1])]
    rs = r[np.lexsort(r.T[::-1])]
    assert np.array_equal(gs, rs), "block coordinate sets differ"


def assert_same_voxels(gpu, ref, tol=TSDF_TOL, exact_tsdf=False):
    """Weights and colour sums exact; mean TSDF within tol (or bit-exact)."""
    gc, gt, gw, gr, gg, gb = sorted_voxels(gpu)
    rc, rt, rw, rr, rg, rb = sorted_voxels(ref)
    assert np.array_equal(gc, rc), "block coordinate sets differ"
    bad = np.argwhere(gw != rw)
    assert bad.shape[0] == 0, (
        f"{bad.shape[0]} weights differ, first at block {gc[bad[0][0]]} voxel {bad[0][1]}: "
        f"gpu {gw[tuple(bad[0])]} oracle {rw[tuple(bad[0])]}")
    for name, a, b in (("r", gr, rr), ("g", gg, rg), ("b", gb, rb)):
        assert np.array_equal(a, b), f"colour sum {name} differs"
    seen = rw > 0
    if exact_tsdf:
        assert np.array_equal(gt.view(np.uint32), rt.view(np.uint32)), "tsdf sums differ"
    mg = gt[seen] / gw[seen]
    mr = rt[seen] / rw[seen]
    err = float(np.max(np.abs(mg - mr))) if mg.size else 0.0
    assert err <= tol, f"mean TSDF differs by {err:.3e} > {tol:.1e}"
    # Unobserved voxels must stay exactly zero.
    assert not np.any(gt[~seen]), "tsdf written where weight is zero"
    return err


# Mean normalised TSDF of FP16 storage against the oracle: four half ulps of
# [-1, 1] (FP16 rounding of the running mean) plus the FP32 parity bar.
FP16_ORACLE_TOL = 4 * 2.0 ** -11 + TSDF_TOL


def assert_matches_oracle(vol, ref, tol=TSDF_TOL):
    """Any storage mode against the CPU oracle: block set and weights exact,
    mean normalised TSDF within tol. Returns the largest mean difference."""
    from what_irregularity_costs_b200 import precision
    gc, gm, gw = precision._aligned(vol)
    rc, rt, rw, *_ = sorted_voxels(ref)
    assert gc.shape == rc.shape and np.array_equal(gc, rc), "block sets differ from the oracle"
    bad = int(np.sum(gw != rw))
    assert bad == 0, f"{bad} weights differ from the oracle"
    seen = rw > 0
    err = float(np.max(np.abs(gm[seen] - rt[seen] / rw[seen]))) if seen.any() else 0.0
    assert err <= tol, f"mean TSDF differs from the oracle by {err:.3e} > {tol:.1e}"
    return err


def sphere_errors(mesh, center, radius):
    p = mesh[:, :3].astype(np.float64) - np.asarray(center, dtype=np.float64)
    e = np.abs(np.linalg.norm(p, axis=1) - radius)
    return float(e.mean()), float(e.max())


def surface_distance(a, b, stride=8):
    """Symmetric nearest-neighbour distance between two vertex sets (metres)."""
    from scipy.spatial import cKDTree
    pa = a[:, :3].astype(np.float64)
    pb = b[:, :3].astype(np.float64)
    ta, tb = cKDTree(pa), cKDTree(pb)
    dab, _ = tb.query(pa[::stride])
    dba, _ = ta.query(pb[::stride])
    return 0.5 * (dab.mean() + dba.mean()), max(dab.max(), dba.max())


def canonical_triangles(mesh):
    """Triangles as a sorted array of their 9 position floats (order-free compare)."""
    tri = mesh[:, :3].reshape(-1, 9)
    order = np.lexsort(tri.T[::-1])
    return tri[order]
