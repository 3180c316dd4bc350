"""Host logic of bench.py's headline arm: frames grouped for
osn_tsdf_cuda_integrate_frames (no GPU needed)."""
import numpy as np
import pytest

import bench


@pytest.mark.parametrize("fpc", [1, 2, 3, 7, 100, 150])
def test_frame_groups_cover_every_frame_once(fpc):
    rng = np.random.default_rng(fpc)
    sizes = rng.integers(0, 500, size=100)
    offsets = np.concatenate([[0], np.cumsum(sizes)])
    cams = rng.standard_normal((100, 3))
    groups = bench.frame_groups(offsets, [tuple(c) for c in cams], fpc)
    assert [g[0] for g in groups] == list(range(0, 100, fpc))
    assert groups[-1][1] == 100
    for lo, hi, a, b, begin, gcams in groups:
        assert 0 < hi - lo <= fpc
        assert (a, b) == (offsets[lo], offsets[hi])
        assert begin.dtype == np.int32 and begin.shape == (hi - lo + 1,)
        assert begin[0] == 0 and begin[-1] == b - a and np.all(np.diff(begin) >= 0)
        assert np.array_equal(begin, offsets[lo:hi + 1] - offsets[lo])
        assert gcams.dtype == np.float32 and gcams.shape == (hi - lo, 3)
        assert np.array_equal(gcams, cams[lo:hi].astype(np.float32))
    # Consecutive groups tile the trajectory's points.
    assert all(groups[k][3] == groups[k + 1][2] for k in range(len(groups) - 1))
