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


def reference_records(case, sx, sz, rx, rz, w):
    with S.Engine(S.ACOUSTIC_2D, case.Nx, case.Nz, case.dx, case.dz, case.dt, case.PML, order=16,
                  flags=S.EXACT) as e:
        e.set_model(case.vp, case.den)
        e.set_shots([S.ShotSpec(sx, sz, rx, rz, w)])
        return e.forward().reshape(len(rx), len(w))


def noalloc_records(case, sx, sz, rx, rz, w):
    import torch
    dev = torch.device("cuda:0")
    vp = torch.from_numpy(np.ascontiguousarray(case.vp)).to(dev)
    den = torch.from_numpy(np.ascontiguousarray(case.den)).to(dev)
    wd = torch.from_numpy(np.ascontiguousarray(w)).to(dev)
    out = torch.full((len(rx) * len(w),), float("nan"), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    g = S.Grid(S.ACOUSTIC_2D, case.Nx, 1, case.Nz, case.PML, case.dx, 0.0, case.dz, case.dt, 16, S.EXACT, 0.0)
    rxa = np.ascontiguousarray(rx, np.int32)
    rza = np.ascontiguousarray(rz, np.int32)
    rc = S.load().sfd_forward_noalloc(ctypes.byref(g), vp.data_ptr(), den.data_ptr(), wd.data_ptr(), len(w),
                                      sx, sz, len(rxa), S._ip(rxa), S._ip(rza), out.data_ptr(), None)
    assert rc == S.OK, rc
    return out.cpu().numpy().reshape(len(rx), len(w))


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
