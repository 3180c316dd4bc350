"""Precision of a volume against the FP64 on-device oracle.

The oracle is a volume created with ``STORAGE_FP64`` and fed the same
batches: same samples, blocks and accepted contributions, signed distances
evaluated in double, sums in double. ``tsdf_errors`` compares the mean
normalised TSDF of two volumes voxel by voxel (matched by block
coordinate) and reports the error in metres (normalised error x truncation
distance); ``mesh_errors`` gives the symmetric surface distance between
their extracted meshes.
"""
from __future__ import annotations

import numpy as np


def _aligned(vol):
    coords, mean, w = vol.means()
    order = np.lexsort(coords.T[::-1]) if coords.shape[0] else np.zeros(0, dtype=np.int64)
    return coords[order], mean[order], w[order]


def tsdf_errors(vol, oracle64, trunc_m: float) -> dict:
    """Max and RMS mean-TSDF error (metres) of `vol` against `oracle64` over
    the voxels both observe; raises if the block sets or weights differ."""
    ca, ma, wa = _aligned(vol)
    cb, mb, wb = _aligned(oracle64)
    if ca.shape != cb.shape or not np.array_equal(ca, cb):
        raise AssertionError("block sets differ from the FP64 oracle")
    if not np.array_equal(wa, wb):
        raise AssertionError("weights differ from the FP64 oracle")
    seen = wb > 0
    err = np.abs(ma[seen] - mb[seen]) * float(trunc_m)
    if err.size == 0:
        return {"max_m": 0.0, "rms_m": 0.0, "voxels": 0}
    return {"max_m": float(err.max()), "rms_m": float(np.sqrt(np.mean(err * err))),
            "voxels": int(err.size)}


def mesh_errors(mesh_a, mesh_b, stride: int = 1) -> dict:
    """Symmetric nearest-vertex distance (metres) between two triangle soups
    (posnor arrays): mean (Chamfer) and maximum (Hausdorff)."""
    from scipy.spatial import cKDTree
    if mesh_a is None or mesh_b is None or not len(mesh_a) or not len(mesh_b):
        return {"chamfer_m": None, "hausdorff_m": None}
    pa = np.asarray(mesh_a[:, :3], dtype=np.float64)
    pb = np.asarray(mesh_b[:, :3], dtype=np.float64)
    dab, _ = cKDTree(pb).query(pa[::stride])
    dba, _ = cKDTree(pa).query(pb[::stride])
    return {"chamfer_m": float(0.5 * (dab.mean() + dba.mean())),
            "hausdorff_m": float(max(dab.max(), dba.max())),
            "vertices": [int(len(pa)), int(len(pb))]}
