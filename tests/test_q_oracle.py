"""CPU checks of the viscoacoustic restatement (oracle/q_oracle.cpp).  The Fortran reference
cannot be compiled here, so these are physics and consistency pins (parity unpinned):
vs = 0 makes strxx and strzz identical (the acoustic reduction the GPU path implements), FP32
agrees with FP64, lower Q attenuates, and the elastic case (vs > 0) stays finite."""
import numpy as np
import pytest

import oracle_lib as ol


def model(nx=60, nz=50, q=50.0, vs_frac=0.0, seed=0):
    rng = np.random.default_rng(seed)
    z = np.arange(nz)
    vp = np.tile(np.where(z < nz // 2, 2000.0, 2600.0), (nx, 1)).astype(np.float32)
    vp += (40.0 * rng.standard_normal((nx, nz))).astype(np.float32)
    vs = (vs_frac * vp).astype(np.float32)
    rho = np.full((nx, nz), 2000.0, np.float32)
    qp = np.full((nx, nz), q, np.float32)
    return vp, vs, rho, qp, qp.copy()


def run(q=50.0, vs_frac=0.0, fp64=False, override=False, nt=200):
    vp, vs, rho, qp, qs = model(q=q, vs_frac=vs_frac)
    npx = npz = 11
    return ol.q_forward(vp, vs, rho, qp, qs, 10.0, 10.0, 1e-3, 20.0, nt, npx, npz, isxe=npx + 30, isze=npz + 3,
                        fp64=fp64, q_override=override)


def test_decay_rule():
    assert ol.q_decay(10.0, 1e-3) == 120
    assert ol.q_decay(20.0, 5e-4) == 120


def test_viscoacoustic_reduction_strxx_equals_strzz():
    r1, r2, _ = run(q=30.0, vs_frac=0.0)
    assert np.abs(r1).max() > 0
    assert np.array_equal(r1.view(np.uint32), r2.view(np.uint32))


def test_fp32_against_fp64():
    r32, _, _ = run(q=40.0)
    r64, _, _ = run(q=40.0, fp64=True)
    err = np.linalg.norm(r32 - r64) / np.linalg.norm(r64)
    assert err < 1e-5, err


def test_attenuation_increases_as_q_drops():
    e = [float(np.sum(run(q=q, nt=300)[0].astype(np.float64) ** 2)) for q in (1e5, 100.0, 20.0)]
    assert e[0] > e[1] > e[2]


def test_q_override_matches_large_q():
    r_big, _, _ = run(q=100000.0)
    r_ovr, _, _ = run(q=15.0, override=True)
    assert np.array_equal(r_big.view(np.uint32), r_ovr.view(np.uint32))


def test_elastic_case_is_finite_and_differs():
    r_el, r_el2, _ = run(q=50.0, vs_frac=0.5)
    r_ac, _, _ = run(q=50.0, vs_frac=0.0)
    assert np.isfinite(r_el).all() and np.isfinite(r_el2).all()
    assert not np.allclose(r_el, r_ac)
