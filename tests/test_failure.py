"""Failure detection without a GPU fault: a device-side wait that runs out.

The reference spins without a bound while another thread publishes a block
it inserted (cpp/src/volume_cuda.cu:71-72). Here every such wait is bounded
(osn_tsdf_cuda_set_spin_limit, default 2^20 iterations of ~100 ns); a wait
that runs out drops its samples and sets bit 0 of the status word, and the
call returns normally. The test plants a slot that is claimed but never
published -- the block's key with block_idx -1, written from the host into
the table through the device view while the volume is idle -- so the insert
of that block waits on a flag nothing will set, with a 64-iteration bound.
"""
import numpy as np
import pytest

import oracle
from what_irregularity_costs_b200 import CudaVolume

pytestmark = pytest.mark.gpu

BIAS = 1 << 20


def _key(bx, by, bz):
    return ((bx + BIAS) << 42) | ((by + BIAS) << 21) | (bz + BIAS)


def _home_slot(bx, by, bz, mask):
    """types.hpp:150-155 in uint32 arithmetic."""
    h = ((bx * 73856093) & 0xFFFFFFFF) ^ ((by * 19349663) & 0xFFFFFFFF) ^ ((bz * 83492791) & 0xFFFFFFFF)
    return h & mask


def _write_slot(view, slot, key, block_idx):
    from cuda.bindings import runtime as rt
    entry = np.zeros(2, dtype=np.int64)
    entry[0] = key
    entry.view(np.int32)[2] = block_idx
    (err,) = rt.cudaMemcpy(view.table + slot * 16, entry.ctypes.data, 16,
                           rt.cudaMemcpyKind.cudaMemcpyHostToDevice)
    assert err == rt.cudaError_t.cudaSuccess


def test_unpublished_slot_wait_runs_out(cuda):
    # One point whose five band samples (1 cm voxels, trunc 2 cm) all fall in
    # block (0, 0, 5), as the oracle confirms.
    pts = np.float32([[0.04, 0.04, 0.44]])
    ref = oracle.OracleVolume(0.01, 1 << 10, 0.02, 64.0)
    ref.integrate(pts, (0.0, 0.0, 0.0))
    assert ref.coords().tolist() == [[0, 0, 5]] and ref.voxels()[2].sum() == 5.0

    vol = CudaVolume(0.01, 1 << 10, 0.02, 64.0)
    vol.set_spin_limit(64)
    view = vol.device_view()
    vol.synchronize()
    _write_slot(view, _home_slot(0, 0, 5, view.hash_mask), _key(0, 0, 5), -1)

    d = cuda.from_numpy(pts).cuda()
    vol.integrate(d, (0.0, 0.0, 0.0))
    vol.synchronize()  # returns: the wait was bounded
    assert vol.status() & 1, "the bounded wait must report that it ran out"
    assert vol.block_count() == 0
    assert vol.drop_count() == 5  # every sample of the unpublished block dropped
    assert float(vol.voxels()[2].sum()) == 0.0

    # The volume stays usable: a point in another block integrates as usual,
    # and lookups of the unpublished block (update without allocation) do not
    # wait at all.
    other = np.float32([[0.04, 0.04, 0.84]])
    vol.integrate(cuda.from_numpy(other).cuda(), (0.0, 0.0, 0.0))
    vol.update_voxels(d, (0.0, 0.0, 0.0))
    vol.synchronize()
    ref2 = oracle.OracleVolume(0.01, 1 << 10, 0.02, 64.0)
    ref2.integrate(other, (0.0, 0.0, 0.0))
    assert vol.coords().tolist() == ref2.coords().tolist()
    assert float(vol.voxels()[2].sum()) == float(ref2.voxels()[2].sum())


def test_spin_limit_bounds(cuda):
    vol = CudaVolume(0.01, 1 << 10, 0.02, 64.0)
    for bad in (0, -1, (1 << 20) + 1):
        with pytest.raises(ValueError):
            vol.set_spin_limit(bad)
    vol.set_spin_limit(1 << 20)
    vol.set_spin_limit(1)
