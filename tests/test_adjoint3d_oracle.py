"""CPU checks of the FP64 3-D adjoint oracle (oracle/adj3d_oracle.cpp) before it checks the GPU
3-D gradient: its forward equals the FP64 forward restatement (oracle/afd3d_oracle.cpp), its
wavelet gradient passes the dot-product test, and its model gradient matches central finite
differences of its own misfit along a seeded smooth perturbation."""
import numpy as np
from scipy.ndimage import gaussian_filter

import oracle_lib as ol
from seismic_code_github_b200 import seisfd as S

PML, D, DT = 6, 10.0, 1e-3


def case(seed=0, n=(26, 24, 28), nt=90, radius=4):
    rng = np.random.default_rng(seed)
    vp = (2000.0 + 500.0 * gaussian_filter(rng.random(n), 2)).astype(np.float32)
    den = (1900.0 + 300.0 * rng.random(n)).astype(np.float32)
    rx = np.arange(PML, n[0] - PML, 2, dtype=np.int32)
    ry = rng.integers(PML, n[1] - PML, len(rx)).astype(np.int32)
    rz = np.full_like(rx, PML + 1)
    w = S.wavelet(S.WAVELET_RIC, nt, DT, 30.0, 25)
    src = (n[0] // 2, n[1] // 2 - 1, PML + 3)
    return dict(vp=vp, den=den, wavelet=w, src=src, rec_x=rx, rec_y=ry, rec_z=rz, pml=PML, dx=D, dy=D, dz=D, dt=DT,
                radius=radius)


def test_forward_matches_fp64_restatement():
    c = case()
    out = ol.afd3d_gradient_f64(**c)
    ref, _ = ol.afd3d_forward(c["vp"], c["den"], c["wavelet"], c["src"], c["rec_x"], c["rec_y"], c["rec_z"],
                              PML, D, D, D, DT, radius=c["radius"], fp64=True)
    assert np.abs(ref).max() > 0
    np.testing.assert_allclose(out["records"], ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_dot_product():
    c = case(seed=1)
    rng = np.random.default_rng(3)
    rec1 = ol.afd3d_gradient_f64(**c)["records"]
    r = rng.standard_normal(rec1.shape)
    obs = (rec1 - r).astype(np.float32)
    res = rec1 - obs
    dw = ol.afd3d_gradient_f64(**c, obs=obs)["dw"]
    w2 = rng.standard_normal(len(c["wavelet"])).astype(np.float32)
    rec2 = ol.afd3d_gradient_f64(**dict(c, wavelet=w2))["records"]
    lhs, rhs = float(np.sum(rec2 * res)), float(np.dot(w2.astype(np.float64), dw))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs), (lhs, rhs)


def test_model_gradient_finite_differences():
    c = case(seed=2, nt=100)
    obs = (ol.afd3d_gradient_f64(**dict(c, vp=(c["vp"] * 1.03).astype(np.float32)))["records"]).astype(np.float32)
    out = ol.afd3d_gradient_f64(**c, obs=obs)
    rng = np.random.default_rng(9)
    d = gaussian_filter(rng.standard_normal(c["vp"].shape), 3)
    d /= np.abs(d).max()
    # the injection scale (dt den) vp is rounded to float (AFD:250), so the misfit is a staircase
    # in vp at the source cell; the perturbation leaves that cell out
    d[c["src"]] = 0.0
    eps = 1.0
    vpp, vpm = (c["vp"] + eps * d).astype(np.float32), (c["vp"] - eps * d).astype(np.float32)
    J = lambda m: ol.afd3d_gradient_f64(**dict(c, vp=m), obs=obs)["misfit"]
    fd = (J(vpp) - J(vpm)) / (2 * eps)
    pred = float(np.sum(out["grad_vp"] * (vpp.astype(np.float64) - vpm) / (2 * eps)))
    assert abs(pred) > 0
    assert abs(fd - pred) <= 1e-6 * abs(pred), (fd, pred)
