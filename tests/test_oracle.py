"""Pins the CPU oracle (oracle/afd_oracle.cpp) against the reference's own outputs.

  - forward/Acoustic_FD_by_ss/file/{record,Snap}.dat (shipped with the reference, copied to
    tests/golden/afd_default/): bit-exact;
  - the patched reference build (oracle/ref_build.py) on config 1 and on a non-square,
    variable-density case (tests/golden/*_record.f32): bit-exact;
  - tools/ricker.cpp output (tests/golden/ric_trace255.f32): bit-exact.
"""
import json
import os

import numpy as np
import pytest

import oracle_lib as ol
from conftest import bits_equal, rel_l2
from seismic_code_github_b200 import workloads as W


def afd_default_setup():
    NX = NZ = 100
    PML = 20
    Nx = Nz = NX + 2 * PML
    vp = np.full((Nx, Nz), 2000, np.float32)
    den = np.full((Nx, Nz), 2400, np.float32)
    w = ol.wavelet_afd(2000, 0.0005, 28.0)
    rx = np.full(NX, Nx // 2)
    rz = np.arange(PML, Nx - PML)
    return NX, NZ, PML, Nx, Nz, vp, den, w, rx, rz


def test_manifest(golden):
    import hashlib
    with open(os.path.join(golden, "manifest.json")) as f:
        man = json.load(f)
    for name, meta in man.items():
        with open(os.path.join(golden, name), "rb") as f:
            data = f.read()
        assert len(data) == meta["bytes"]
        assert hashlib.sha256(data).hexdigest() == meta["sha256"], name


def test_afd_default_record_and_snapshot_bitexact(golden):
    NX, NZ, PML, Nx, Nz, vp, den, w, rx, rz = afd_default_setup()
    rec, snap, _ = ol.afd_forward(Nx, Nz, PML, 2000, 10.0, 10.0, 0.0005, vp, den, w, Nx // 2, Nz // 2, rx, rz,
                                  radius=8, snap_step=500)
    ref = np.fromfile(os.path.join(golden, "afd_default", "record.dat"), np.float32).reshape(NX, 2000)
    assert bits_equal(rec, ref)
    sref = np.fromfile(os.path.join(golden, "afd_default", "Snap.dat"), np.float32).reshape(NX, NZ)
    assert bits_equal(snap[PML:-PML, PML:-PML], sref)
    model = np.fromfile(os.path.join(golden, "afd_default", "Model.dat"), np.float32).reshape(NX, NZ)
    assert bits_equal(vp[PML:-PML, PML:-PML], model)


def test_fp64_oracle_close_to_reference(golden):
    """The FP64 oracle of the same scheme differs from the FP32 reference only by rounding
    (about 1e-6 relative L2 on the shipped record)."""
    NX, NZ, PML, Nx, Nz, vp, den, w, rx, rz = afd_default_setup()
    rec, _, _ = ol.afd_forward(Nx, Nz, PML, 2000, 10.0, 10.0, 0.0005, vp, den, w, Nx // 2, Nz // 2, rx, rz,
                               fp64=True)
    ref = np.fromfile(os.path.join(golden, "afd_default", "record.dat"), np.float32).reshape(NX, 2000)
    assert rel_l2(ref, rec) < 5e-6


def test_ricker_tool_bitexact(golden):
    ref = np.fromfile(os.path.join(golden, "ric_trace255.f32"), np.float32)
    assert bits_equal(ol.wavelet_ric(1024, 0.002, 35, 150), ref)


@pytest.mark.parametrize("case_fn,fname", [(W.small_varden, "small_varden_record.f32"),
                                           (W.config1, "config1_record.f32")])
def test_patched_reference_cases_bitexact(golden, case_fn, fname):
    case = case_fn()
    w = ol.wavelet_ric(case.nt, case.dt, int(case.f0), 150)
    rx, rz = case.receivers()
    rec, _, _ = ol.afd_forward(case.Nx, case.Nz, case.PML, case.nt, case.dx, case.dz, case.dt, case.vp, case.den,
                               w, case.src_x[0], case.src_z[0], rx, rz)
    ref = np.fromfile(os.path.join(golden, fname), np.float32).reshape(rec.shape)
    assert bits_equal(rec, ref)


def test_oracle_rejects_bad_config():
    vp = np.full((20, 20), 2000, np.float32)
    with pytest.raises(ValueError):
        ol.afd_forward(20, 20, 2, 5, 10, 10, 1e-3, vp, vp, np.zeros(5, np.float32), 25, 5, [5], [5])


def test_planted_error_is_detected(golden):
    """A mistake planted in the oracle's inputs (one model cell changed) must break the
    bit-exact comparison -- the pin is sensitive."""
    case = W.small_varden()
    w = ol.wavelet_ric(case.nt, case.dt, int(case.f0), 150)
    rx, rz = case.receivers()
    vp = case.vp.copy()
    vp[case.src_x[0] + 3, case.src_z[0] + 2] *= 1.001
    rec, _, _ = ol.afd_forward(case.Nx, case.Nz, case.PML, case.nt, case.dx, case.dz, case.dt, vp, case.den,
                               w, case.src_x[0], case.src_z[0], rx, rz)
    ref = np.fromfile(os.path.join(golden, "small_varden_record.f32"), np.float32).reshape(rec.shape)
    assert not bits_equal(rec, ref)
