"""The raw "OSN1" mesh file: the reference harness's geometry dump
(cpp/bench/bench_arms.cu:506-523), read and written on the host.

Layout, little-endian: uint32 magic 0x314e534f (the bytes b"OSN1"), uint32
vertex count n, then n * 6 float32 -- each vertex's position and face normal
interleaved, exactly as extraction produced them (a triangle soup: vertices
3k, 3k+1, 3k+2 form triangle k). CudaVolume.write_mesh_osn1 writes the file
straight from the library (osn_tsdf_cuda_write_mesh_osn1).
"""
from __future__ import annotations

import numpy as np

MAGIC = 0x314E534F


def write_osn1(path: str, posnor: np.ndarray) -> int:
    """Write an (n, 6) float32 position/normal array; returns n."""
    a = np.ascontiguousarray(np.asarray(posnor, dtype="<f4"))
    if a.ndim != 2 or a.shape[1] != 6:
        raise ValueError("posnor must have shape (n, 6)")
    with open(path, "wb") as f:
        f.write(np.array([MAGIC, a.shape[0]], dtype="<u4").tobytes())
        f.write(a.tobytes())
    return int(a.shape[0])


def read_osn1(path: str) -> np.ndarray:
    """The (n, 6) float32 position/normal array of an OSN1 file."""
    with open(path, "rb") as f:
        head = np.frombuffer(f.read(8), dtype="<u4")
        if head.size != 2 or int(head[0]) != MAGIC:
            raise ValueError(f"{path}: not an OSN1 mesh file")
        n = int(head[1])
        body = np.frombuffer(f.read(), dtype="<f4")
    if body.size != 6 * n:
        raise ValueError(f"{path}: {body.size} floats for {n} vertices")
    return body.reshape(n, 6).copy()
