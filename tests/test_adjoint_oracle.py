"""CPU checks of the FP64 adjoint oracle (oracle/adj_oracle.cpp) before it is used to check
the GPU gradient: its forward equals the FP64 forward restatement, the adjoint passes the
dot-product test, and the gradient matches central finite differences of the misfit."""
import numpy as np
import pytest

import oracle_lib as ol
from seismic_code_github_b200 import workloads as W


def small_case(seed=0, nt=160):
    NX, NZ, PML = 40, 30, 10
    rng = np.random.default_rng(seed)
    v = W.layered_model(NX, NZ, 3, 1800.0, 2600.0, seed=seed, anomalies=1, radius=5.0, amp=150.0)
    vp = W.pad_edges(v, PML, PML)
    den = W.pad_edges((2000.0 + 300.0 * rng.random((NX, NZ))).astype(np.float32), PML, PML)
    Nx, Nz = vp.shape
    w = ol.wavelet_ric(nt, 1e-3, 25, 40)
    rx = np.arange(PML, Nx - PML, 3, dtype=np.int32)
    rz = np.full_like(rx, PML + 2)
    return dict(nx=Nx, nz=Nz, pml=PML, nt=nt, dx=10.0, dz=10.0, dt=1e-3, vp=vp, den=den, wavelet=w,
                sx=PML + 12, sz=PML + 4, rec_x=rx, rec_z=rz)


@pytest.mark.parametrize("radius", [8, 4])
def test_oracle_adjoint_forward_matches_fp64_forward(radius):
    c = small_case()
    obs = np.zeros((len(c["rec_x"]), c["nt"]), np.float32)
    _, _, _, rec = ol.afd_gradient_f64(**c, obs=obs, radius=radius)
    ref, _, _ = ol.afd_forward(c["nx"], c["nz"], c["pml"], c["nt"], c["dx"], c["dz"], c["dt"], c["vp"], c["den"],
                               c["wavelet"], c["sx"], c["sz"], c["rec_x"], c["rec_z"], radius=radius, fp64=True)
    np.testing.assert_allclose(rec, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("radius", [8, 5])
def test_oracle_dot_product(radius):
    """<F w2, r> = <w2, F^T r>: F maps the wavelet to the records (linear for a fixed model);
    F^T r is the wavelet gradient of 0.5|F w1 - obs|^2 with obs = F w1 - r."""
    c = small_case(seed=1)
    rng = np.random.default_rng(42)
    nrec, nt = len(c["rec_x"]), c["nt"]
    r = rng.standard_normal((nrec, nt)).astype(np.float32)
    w1 = c["wavelet"]
    _, _, _, rec1 = ol.afd_gradient_f64(**c, obs=np.zeros((nrec, nt), np.float32), radius=radius)
    obs = (rec1 - r.astype(np.float64)).astype(np.float32)
    res = rec1 - obs  # the residual the adjoint actually sees (r up to float rounding of obs)
    _, _, dw, _ = ol.afd_gradient_f64(**c, obs=obs, radius=radius)
    w2 = rng.standard_normal(nt).astype(np.float32)
    c2 = dict(c, wavelet=w2)
    _, _, _, rec2 = ol.afd_gradient_f64(**c2, obs=np.zeros((nrec, nt), np.float32), radius=radius)
    lhs = float(np.sum(rec2 * res))
    rhs = float(np.sum(w2.astype(np.float64) * dw))
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), abs(rhs)), (lhs, rhs)


def test_oracle_gradient_finite_differences():
    c = small_case(seed=2, nt=140)
    nrec, nt = len(c["rec_x"]), c["nt"]
    true = dict(c, vp=(c["vp"] * 1.03).astype(np.float32))
    _, _, _, obs = ol.afd_gradient_f64(**true, obs=np.zeros((nrec, nt), np.float32))
    obs = obs.astype(np.float32)
    J0, g, _, _ = ol.afd_gradient_f64(**c, obs=obs)
    rng = np.random.default_rng(7)
    for trial in range(3):
        d = rng.standard_normal(c["vp"].shape)
        d[np.abs(d) < 0] = 0
        dvp = (d * 2.0).astype(np.float64)  # m/s
        eps = 1.0
        Jp, _, _, _ = ol.afd_gradient_f64(**dict(c, vp=(c["vp"] + eps * dvp).astype(np.float32)), obs=obs)
        Jm, _, _, _ = ol.afd_gradient_f64(**dict(c, vp=(c["vp"] - eps * dvp).astype(np.float32)), obs=obs)
        fd = (Jp - Jm) / (2 * eps)
        an = float(np.sum(g * dvp))
        assert abs(fd - an) <= 2e-3 * abs(an), (trial, fd, an)


def test_oracle_source_in_frozen_rim():
    """Source inside the never-updated rim: the transpose reaches the rim cells; the wavelet
    gradient must still pass the dot-product test."""
    c = small_case(seed=3, nt=80)
    c["sx"], c["sz"] = 3, 5
    rng = np.random.default_rng(5)
    nrec, nt = len(c["rec_x"]), c["nt"]
    _, _, _, rec1 = ol.afd_gradient_f64(**c, obs=np.zeros((nrec, nt), np.float32))
    r = rng.standard_normal((nrec, nt))
    obs = (rec1 - r).astype(np.float32)
    res = rec1 - obs
    _, _, dw, _ = ol.afd_gradient_f64(**c, obs=obs)
    w2 = rng.standard_normal(nt).astype(np.float32)
    _, _, _, rec2 = ol.afd_gradient_f64(**dict(c, wavelet=w2), obs=np.zeros((nrec, nt), np.float32))
    lhs, rhs = float(np.sum(rec2 * res)), float(np.sum(w2 * dw))
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), abs(rhs), 1e-300)
