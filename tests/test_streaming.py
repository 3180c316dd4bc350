"""Streaming by chunk id: evict the blocks of chunks left behind to host
memory, keep integrating with the freed pool, stream them back in.

The scene is a row of six spheres 3 m apart (the reference's analytic sphere,
cpp/tests/analytic_scenes.hpp:19-33, each seen from its centre), one chunk
per sphere, so no chunk re-observes another's blocks. A pool that holds
about two and a half spheres integrates all six by evicting, after each
call, the chunk before it; the resident blocks plus the evicted packs must then
be exactly the oracle's volume of all six spheres (block set, weights; mean
TSDF within 1e-5), and streaming every pack back into a large volume must
give a volume bit-identical to integrating all six without eviction, even
with resident chunks integrated again in between.
"""
import numpy as np
import pytest

import oracle
from helpers import TSDF_TOL, sorted_voxels
from what_irregularity_costs_b200 import CudaVolume

pytestmark = pytest.mark.gpu

N_CHUNKS = 6
VOXEL, CAP = 0.01, 32.0


def _chunks():
    pts = oracle.sphere_points(0.5, 100, 200)
    out = []
    for k in range(N_CHUNKS):
        off = np.float32([3.0 * k, 0.0, 0.0])
        out.append((np.ascontiguousarray(pts + off), tuple(float(x) for x in off)))
    return out


def _blocks(coords, *arrays):
    """{coordinate: (array rows...)} for comparisons independent of pool order."""
    return {tuple(c): tuple(a[i] for a in arrays) for i, c in enumerate(coords.tolist())}


def test_evict_keeps_a_small_pool_integrating(cuda):
    chunks = _chunks()
    ref = oracle.OracleVolume(VOXEL, 1 << 14, -1.0, CAP)
    for p, cam in chunks:
        ref.integrate(p, cam)
    assert ref.drop_count() == 0

    vol = CudaVolume(VOXEL, 2800, -1.0, CAP)  # about 2.5 spheres' blocks
    packs = []
    for k, (p, cam) in enumerate(chunks):
        vol.set_chunk(k)
        vol.integrate(cuda.from_numpy(p).cuda(), cam)
        if k >= 1:
            packs.append(vol.evict_chunks(k - 1, k - 1))  # the chunk behind
    vol.synchronize()
    assert vol.status() == 0 and vol.drop_count() == 0
    assert len(packs) == N_CHUNKS - 1

    # Resident blocks are the last chunk's; the packs hold the others.
    rc, rt, rw, *_ = sorted_voxels(ref)
    want = _blocks(rc, rt, rw)
    got = _blocks(*vol.voxels()[:3])
    for pk in packs:
        coords, chunk_ids, arrays = vol.unpack_chunks(pk)
        assert len(set(chunk_ids.tolist())) == 1
        for c, row in _blocks(coords, arrays[0], arrays[1]).items():
            assert c not in got, "a block is both resident and evicted"
            got[c] = row
    assert set(got) == set(want), "resident + evicted blocks differ from the oracle's block set"
    for c, (t, w) in want.items():
        gt, gw = got[c]
        assert np.array_equal(gw, w), f"weights of block {c} differ"
        seen = w > 0
        assert np.max(np.abs(gt[seen] / gw[seen] - t[seen] / w[seen]), initial=0.0) <= TSDF_TOL


def test_stream_in_restores_bit_identically(cuda):
    chunks = _chunks()
    whole = CudaVolume(VOXEL, 1 << 14, -1.0, CAP)
    vol = CudaVolume(VOXEL, 1 << 14, -1.0, CAP)
    for k, (p, cam) in enumerate(chunks):
        d = cuda.from_numpy(p).cuda()
        whole.integrate(d, cam)
        vol.set_chunk(k)
        vol.integrate(d, cam)
    n_all = vol.block_count()
    pack = vol.evict_chunks(1, 3)
    left = vol.block_count()
    assert 0 < left < n_all
    # The resident chunks keep integrating after the compaction.
    p, cam = chunks[5]
    extra = cuda.from_numpy(p).cuda()
    vol.integrate(extra, cam)
    whole.integrate(extra, cam)
    assert vol.stream_in(pack) == 0
    assert vol.block_count() == n_all == whole.block_count()
    for x, y in zip(sorted_voxels(vol), sorted_voxels(whole)):
        assert x.shape == y.shape and np.array_equal(x.view(np.uint8), y.view(np.uint8))
    # Streaming the same pack again: every block is present, all skipped.
    assert vol.stream_in(pack) == len(vol.unpack_chunks(pack)[0])
    assert vol.block_count() == n_all
    assert vol.status() == 0


def test_pack_of_another_volume_is_refused(cuda):
    a = CudaVolume(VOXEL, 1 << 12, -1.0, CAP)
    b = CudaVolume(0.02, 1 << 12, -1.0, CAP)
    p, cam = _chunks()[0]
    a.integrate(cuda.from_numpy(p).cuda(), cam)
    pack = a.evict_chunks(0, 0)
    assert a.block_count() == 0 and len(a.unpack_chunks(pack)[0]) > 1000
    with pytest.raises(ValueError):  # another voxel size: a bad pack (code 1)
        b.stream_in(pack)
    empty = a.evict_chunks(7, 9)  # nothing in range: a header-only pack
    assert len(a.unpack_chunks(empty)[0]) == 0 and a.stream_in(empty) == 0
