"""GPU parity of the VTI pseudo-acoustic modeller (sfd_vti_forward, csrc/vti2d.cu) with the FP32
restatement (oracle/vti_oracle.cpp): with SFD_EXACT the records must be equal bit for bit, in
the default mode (FMA contraction, approximate divisions) within relative L2 1e-5 of the FP32
and the FP64 restatement.  The cases cover
the reference's own layout (no top PML, receivers on row 6 because nrz0 + nz_bound_u < 6,
VM:446-453), a top PML with the receivers below it, apertures clamped at both model edges
(VS:298-300), and a batch of shots against the per-shot restatement."""
import numpy as np
import pytest

import oracle_lib as ol
from conftest import rel_l2
from seismic_code_github_b200 import seisfd as S

pytestmark = pytest.mark.gpu


def model(nxv=140, nzv=90, seed=11):
    rng = np.random.default_rng(seed)
    z = np.arange(nzv)
    vz = np.tile(np.where(z < 30, 1800.0, np.where(z < 60, 2400.0, 3000.0)), (nxv, 1)).astype(np.float32)
    vz += (40.0 * rng.standard_normal(vz.shape)).astype(np.float32)
    eps = np.tile(np.where(z < 45, 0.12, 0.22), (nxv, 1)).astype(np.float32)
    de = np.tile(np.where(z < 45, 0.04, 0.09), (nxv, 1)).astype(np.float32)
    eps += (0.01 * rng.random(eps.shape)).astype(np.float32)
    return vz, eps, de


CASES = {
    # bounds (l, r, u, d), shot (nsx, nsz0, nrz0, xmin, xmax)
    "reference_layout": ((25, 25, 0, 25), (70, 1, 1, 10, 129)),
    "top_pml": ((20, 22, 12, 20), (60, 4, 3, 0, 139)),
    "clamped_aperture": ((20, 20, 8, 20), (30, 2, 2, -15, 104)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_single_shot_bitexact(name):
    bounds, shot = CASES[name]
    vz, eps, de = model()
    nt = 600
    rec, t = S.vti_forward(vz, eps, de, 5.0, 5.0, 5e-4, 30.0, nt, bounds, [shot], exact=True)
    ref = ol.vti_forward(vz, eps, de, 5.0, 5.0, 5e-4, 30.0, nt, bounds, *shot)
    diff = np.abs(rec[0] - ref).max()
    print(f"{name}: max |GPU - restatement| {diff:.3e}, peak {np.abs(ref).max():.3e}, {t['launches']} launches, "
          f"{t['loop_ms']:.2f} ms")
    assert np.abs(ref).max() > 0
    assert np.array_equal(rec[0].view(np.uint32), ref.view(np.uint32))
    assert t["kernel_variant"] == 71


def test_batched_shots_equal_per_shot_restatement():
    vz, eps, de = model(180, 80, seed=5)
    bounds = (20, 20, 0, 20)
    nt = 500
    shots = [(nsx, 1, 1, nsx - 60, nsx + 59) for nsx in (40, 90, 150)]
    rec, t = S.vti_forward(vz, eps, de, 5.0, 5.0, 5e-4, 30.0, nt, bounds, shots, exact=True)
    for k, sh in enumerate(shots):
        ref = ol.vti_forward(vz, eps, de, 5.0, 5.0, 5e-4, 30.0, nt, bounds, *sh)
        assert np.array_equal(rec[k].view(np.uint32), ref.view(np.uint32)), k
    # one launch per step for all shots, plus the source injections
    nwt = int(round(2 * 0.07 / 5e-4)) + 1
    assert t["launches"] == nt + (nwt - 1) // 2 + nwt


@pytest.mark.parametrize("name", list(CASES))
def test_fast_mode_within_tolerance(name):
    bounds, shot = CASES[name]
    vz, eps, de = model()
    nt = 600
    rec, t = S.vti_forward(vz, eps, de, 5.0, 5.0, 5e-4, 30.0, nt, bounds, [shot])
    ref = ol.vti_forward(vz, eps, de, 5.0, 5.0, 5e-4, 30.0, nt, bounds, *shot)
    r64 = ol.vti_forward(vz, eps, de, 5.0, 5.0, 5e-4, 30.0, nt, bounds, *shot, fp64=True)
    e32, e64 = rel_l2(rec[0], ref), rel_l2(rec[0], r64)
    print(f"{name}: fast mode relL2 vs FP32 restatement {e32:.2e}, vs FP64 {e64:.2e}")
    assert t["kernel_variant"] == 70
    assert e32 <= 1e-5 and e64 <= 1e-5


def test_fast_mode_long_record():
    """The default mode over 3000 samples (the error of approximate divisions and FMA contraction
    accumulates with the record length): still within relative L2 1e-5 of the FP64 restatement."""
    bounds, shot = CASES["reference_layout"]
    vz, eps, de = model()
    nt = 3000
    rec, _ = S.vti_forward(vz, eps, de, 5.0, 5.0, 5e-4, 30.0, nt, bounds, [shot])
    r64 = ol.vti_forward(vz, eps, de, 5.0, 5.0, 5e-4, 30.0, nt, bounds, *shot, fp64=True)
    r32 = ol.vti_forward(vz, eps, de, 5.0, 5.0, 5e-4, 30.0, nt, bounds, *shot)
    e64, e32 = rel_l2(rec[0], r64), rel_l2(r32, r64)
    print(f"nt {nt}: fast mode relL2 vs FP64 {e64:.2e} (FP32 restatement vs FP64 {e32:.2e})")
    assert e64 <= 1e-5


def test_invalid_arguments():
    vz, eps, de = model(60, 40)
    with pytest.raises(S.SfdError) as e:  # shots of one call share the grid
        S.vti_forward(vz, eps, de, 5.0, 5.0, 5e-4, 30.0, 10, (10, 10, 0, 10), [(20, 1, 1, 0, 39), (30, 1, 1, 0, 29)])
    assert e.value.status == 1
    with pytest.raises(S.SfdError) as e:
        S.vti_forward(vz, eps, de, 5.0, 5.0, 5e-4, 30.0, 10, (10, 10, 0, 10), [(20, 1, 1, 0, 39)], orders=(8, 9, 10))
    assert e.value.status == 7
    bad = vz.copy()
    bad[3, 3] = 0.0
    with pytest.raises(S.SfdError) as e:
        S.vti_forward(bad, eps, de, 5.0, 5.0, 5e-4, 30.0, 10, (10, 10, 0, 10), [(20, 1, 1, 0, 39)])
    assert e.value.status == 1
