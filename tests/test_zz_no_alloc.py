"""sfd_forward_noalloc, the single-shot forward that allocates no device memory (for callers
that cannot allocate when they model a shot: a framework that has reserved the device memory
for its own allocator, a process at its device-memory quota, a real-time loop that forbids
allocation after start-up).  Its output must equal the context-based sfd_forward with
SFD_EXACT (the same reference-order kernel) bit for bit, on two different calls in a row --
the second call must not see the first call's leftovers in the shared device array.

This file is collected last (test_zz_*): if it fails, a run that stops at the first failure
has already run every other test."""
import ctypes

import numpy as np
import pytest

from conftest import bits_equal
from seismic_code_github_b200 import seisfd as S
from seismic_code_github_b200 import workloads as W

pytestmark = pytest.mark.gpu


def reference_records(case, sx, sz, rx, rz, w, den=True):
    with S.Engine(S.ACOUSTIC_2D, case.Nx, case.Nz, case.dx, case.dz, case.dt, case.PML, order=16,
                  flags=S.EXACT) as e:
        e.set_model(case.vp, case.den if den else None)
        e.set_shots([S.ShotSpec(sx, sz, rx, rz, w)])
        return e.forward().reshape(len(rx), len(w))


def noalloc_call(case, sx, sz, rx, rz, w, den=True, check_free=False):
    """One call through the C ABI with torch-owned device buffers; returns (rc, records).
    check_free: also assert that the call left the device's free memory unchanged."""
    import torch
    dev = torch.device("cuda:0")
    vp = torch.from_numpy(np.ascontiguousarray(case.vp)).to(dev)
    dn = torch.from_numpy(np.ascontiguousarray(case.den)).to(dev) if den else None
    wd = torch.from_numpy(np.ascontiguousarray(w)).to(dev)
    out = torch.full((len(rx) * len(w),), float("nan"), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    g = S.Grid(S.ACOUSTIC_2D, case.Nx, 1, case.Nz, case.PML, case.dx, 0.0, case.dz, case.dt, 16, S.EXACT, 0.0)
    rxa = np.ascontiguousarray(rx, np.int32)
    rza = np.ascontiguousarray(rz, np.int32)
    free0 = torch.cuda.mem_get_info(0)[0]
    rc = S.load().sfd_forward_noalloc(ctypes.byref(g), vp.data_ptr(), dn.data_ptr() if den else None, wd.data_ptr(),
                                      len(w), sx, sz, len(rxa), S._ip(rxa), S._ip(rza), out.data_ptr(), None)
    if check_free:
        assert torch.cuda.mem_get_info(0)[0] == free0, "the call changed the device's free memory"
    return rc, out.cpu().numpy().reshape(len(rx), len(w))


def noalloc_records(case, sx, sz, rx, rz, w, den=True, check_free=False):
    rc, rec = noalloc_call(case, sx, sz, rx, rz, w, den, check_free)
    assert rc == S.OK, rc
    return rec


def test_noalloc_equals_forward_on_two_calls():
    case = W.small_varden()
    rx, rz = case.receivers()
    calls = [
        (case.src_x[0], case.src_z[0], rx, rz, S.wavelet(S.WAVELET_RIC, 220, case.dt, 20.0, 40)),
        (case.PML + 55, case.PML + 30, rx[::3].copy(), (rz[::3] + 5).copy(),
         S.wavelet(S.WAVELET_RIC, 140, case.dt, 27.0, 30)),
    ]
    for sx, sz, rxs, rzs, w in calls:
        got = noalloc_records(case, sx, sz, rxs, rzs, w)
        ref = reference_records(case, sx, sz, rxs, rzs, w)
        assert np.isfinite(got).all() and np.abs(got).max() > 0
        assert bits_equal(got, ref)


def test_noalloc_constant_density_allocates_nothing():
    """den_dev = NULL (constant density 2400, the reference's DEN, AFD:140-142) against
    sfd_forward on a model given without density, on two calls in a row.  The calls after the
    first allocate nothing: the device's free memory is the same before and after each."""
    case = W.small_varden()
    rx, rz = case.receivers()
    w = S.wavelet(S.WAVELET_RIC, 180, case.dt, 22.0, 40)
    noalloc_records(case, case.src_x[0], case.src_z[0], rx, rz, w, den=False)  # first call: address set-up
    for sz in (case.src_z[0], case.src_z[0] + 7):
        got = noalloc_records(case, case.src_x[0], sz, rx, rz, w, den=False, check_free=True)
        ref = reference_records(case, case.src_x[0], sz, rx, rz, w, den=False)
        assert np.isfinite(got).all() and np.abs(got).max() > 0
        assert bits_equal(got, ref)


def test_noalloc_rejects_sizes_beyond_its_array():
    """A grid and record larger than the 32 MiB array are refused with SFD_ERR_NOMEM before any
    device work: the output buffer keeps its contents."""
    case = W.small_varden()
    rx, rz = case.receivers()
    w = np.zeros(120000, np.float32)  # the nrec x nt records alone (38 MB) exceed 32 MiB
    rc, out = noalloc_call(case, case.src_x[0], case.src_z[0], rx, rz, w)
    assert rc == S.ERR_NOMEM
    assert np.isnan(out).all()
