"""CPU checks of the FP64 viscoacoustic gradient oracle (oracle/q_adj_oracle.cpp), the checker of
the GPU d misfit / d vp and d misfit / d (1/Q):
  * its forward equals the FP32 restatement of Q_forward (oracle/q_oracle.cpp) to FP32 round-off;
  * its wavelet gradient is the transpose of the wavelet-to-records map (dot-product test);
  * its model gradients match central finite differences of its own misfit along seeded smooth
    perturbations of vp and of 1/Q.
"""
import numpy as np
import pytest
from scipy.ndimage import gaussian_filter

import oracle_lib as ol
from conftest import rel_l2
from seismic_code_github_b200 import seisfd as S

NPX, F0, DT, DX = 8, 20.0, 5e-4, 10.0


def model(seed=0, nx=36, nz=32):
    rng = np.random.default_rng(seed)
    vp_i = (2000 + 400 * gaussian_filter(rng.random((nx, nz)), 3)).astype(np.float32)
    rho_i = (1900 + 400 * rng.random((nx, nz))).astype(np.float32)
    q_i = (30 + 120 * gaussian_filter(rng.random((nx, nz)), 2)).astype(np.float32)
    pad = lambda a: S.pad_model(a, NPX, NPX, NPX, NPX)
    return vp_i, rho_i, q_i, pad(vp_i), pad(rho_i), pad(q_i)


def test_forward_equals_fp32_restatement():
    vp_i, rho_i, q_i, vp, rho, q = model()
    dec = ol.q_decay(F0, DT)
    nt = 140
    isxe, isze, nrz0 = NPX + 15, NPX + 5, 2
    r1, _, _ = ol.q_forward(vp_i, vp_i * 0, rho_i, q_i, q_i, DX, DX, DT, F0, nt, NPX, NPX, isxe, isze, nrz0=nrz0)
    w = S.wavelet(S.WAVELET_Q, nt + dec, DT, F0)
    rx = np.arange(NPX, NPX + vp_i.shape[0], dtype=np.int32)
    out = ol.q_gradient_f64(vp, rho, q, w, (isxe - 1, isze - 1), rx, np.full_like(rx, NPX + nrz0), NPX, DX, DX, DT, F0)
    got = out["records"][:, dec:]
    assert np.abs(got).max() > 0
    assert rel_l2(r1, got) < 1e-5


def setup_case(seed=1, nt=160):
    _, _, _, vp, rho, q = model(seed)
    w = S.wavelet(S.WAVELET_Q, nt, DT, F0)
    rx = np.arange(NPX, vp.shape[0] - NPX, 3, dtype=np.int32)
    rz = np.full_like(rx, NPX + 2)
    return vp, rho, q, w, (22, 14), rx, rz


def test_wavelet_gradient_dot_product():
    vp, rho, q, w, src, rx, rz = setup_case()
    rng = np.random.default_rng(5)
    r = rng.standard_normal((len(rx), len(w))).astype(np.float32)
    fw = ol.q_gradient_f64(vp, rho, q, w, src, rx, rz, NPX, DX, DX, DT, F0)["records"]
    obs = (fw - r).astype(np.float32)  # residual = F w - obs = r (up to the float32 rounding of obs)
    res = fw - obs.astype(np.float64)
    dw = ol.q_gradient_f64(vp, rho, q, w, src, rx, rz, NPX, DX, DX, DT, F0, obs=obs)["dw"]
    dwv = rng.standard_normal(len(w)).astype(np.float32)
    fdw = ol.q_gradient_f64(vp, rho, q, dwv, src, rx, rz, NPX, DX, DX, DT, F0)["records"]
    lhs, rhs = float(np.sum(res * fdw)), float(np.dot(dwv.astype(np.float64), dw))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


@pytest.mark.parametrize("which", ["vp", "invq"])
def test_model_gradient_finite_differences(which):
    vp, rho, q, w, src, rx, rz = setup_case(seed=2)
    obs = (0.8 * ol.q_gradient_f64(vp, rho, q, w, src, rx, rz, NPX, DX, DX, DT, F0)["records"]).astype(np.float32)
    out = ol.q_gradient_f64(vp, rho, q, w, src, rx, rz, NPX, DX, DX, DT, F0, obs=obs)
    rng = np.random.default_rng(9)
    d = gaussian_filter(rng.standard_normal(vp.shape), 4)
    d /= np.abs(d).max()
    if which == "vp":
        eps = 1.0  # m/s; the step actually taken is the float32-rounded one
        vpp, vpm = (vp + eps * d).astype(np.float32), (vp - eps * d).astype(np.float32)
        J = lambda m: ol.q_gradient_f64(m, rho, q, w, src, rx, rz, NPX, DX, DX, DT, F0, obs=obs)["misfit"]
        fd = (J(vpp) - J(vpm)) / (2 * eps)
        pred = float(np.sum(out["grad_vp"] * (vpp.astype(np.float64) - vpm) / (2 * eps)))
    else:
        invq = 1.0 / q.astype(np.float64)
        eps = 1e-4
        J = lambda e: ol.q_gradient_f64(vp, rho, (1.0 / (invq + e * d)).astype(np.float32), w, src, rx, rz, NPX,
                                        DX, DX, DT, F0, obs=obs)["misfit"]
        pred = float(np.sum(out["grad_invq"] * d))
        fd = (J(eps) - J(-eps)) / (2 * eps)
    assert abs(pred) > 0
    assert abs(fd - pred) <= 1e-4 * abs(pred), (fd, pred)
