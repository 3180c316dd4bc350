"""The OSN1 mesh file (the reference harness's raw geometry dump,
cpp/bench/bench_arms.cu:506-523): header bytes, round trip, malformed files,
and the library's own writer (osn_tsdf_cuda_write_mesh_osn1) against the mesh
that extraction returns.
"""
import numpy as np
import pytest

from helpers import canonical_triangles
from what_irregularity_costs_b200 import CudaVolume, meshio, scenes


def test_osn1_header_and_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    posnor = rng.standard_normal((12, 6)).astype(np.float32)
    path = str(tmp_path / "mesh.raw")
    assert meshio.write_osn1(path, posnor) == 12
    raw = open(path, "rb").read()
    assert raw[:4] == b"OSN1"
    assert int.from_bytes(raw[4:8], "little") == 12
    assert len(raw) == 8 + 12 * 6 * 4
    back = meshio.read_osn1(path)
    assert back.dtype == np.float32 and np.array_equal(back, posnor)


def test_osn1_empty_and_malformed(tmp_path):
    empty = str(tmp_path / "empty.raw")
    meshio.write_osn1(empty, np.zeros((0, 6), dtype=np.float32))
    assert meshio.read_osn1(empty).shape == (0, 6)
    bad = tmp_path / "bad.raw"
    bad.write_bytes(b"OSN2" + (1).to_bytes(4, "little") + bytes(24))
    with pytest.raises(ValueError):
        meshio.read_osn1(str(bad))
    short = tmp_path / "short.raw"
    short.write_bytes(b"OSN1" + (2).to_bytes(4, "little") + bytes(24))
    with pytest.raises(ValueError):
        meshio.read_osn1(str(short))
    with pytest.raises(ValueError):
        meshio.write_osn1(str(tmp_path / "x.raw"), np.zeros((3, 5), dtype=np.float32))


@pytest.mark.gpu
def test_library_writes_the_extracted_mesh(cuda, tmp_path):
    frame = scenes.sphere_frame()
    vol = CudaVolume(0.01, 1 << 15, 0.04, 64.0)
    vol.integrate(cuda.from_numpy(scenes.frame_points(frame)).cuda(), frame.cam)
    mesh = vol.extract_mesh(1 << 20, 0.5, 0.0)
    path = str(tmp_path / "sphere.raw")
    n = vol.write_mesh_osn1(path, 1 << 20, 0.5, 0.0)
    dumped = meshio.read_osn1(path)
    assert n == mesh.shape[0] == dumped.shape[0] > 0
    # Triangle order follows the extraction's block compaction; the set is fixed.
    assert np.array_equal(canonical_triangles(dumped), canonical_triangles(mesh[:, :6]))
    with pytest.raises(ValueError):
        vol.write_mesh_osn1(str(tmp_path / "small.raw"), 16)  # vert_cap too small
    assert vol.status() == 0
