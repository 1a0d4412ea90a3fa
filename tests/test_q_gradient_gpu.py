"""GPU gradient of the viscoacoustic scheme (SFD_VISCOAC_2D, the vs = 0 reduction of
forward/Q_forward) through the C ABI (sfd_gradient with grad_invq): d misfit / d vp and
d misfit / d (1/Q) against the FP64 adjoint oracle (oracle/q_adj_oracle.cpp, relative L2 <= 1e-4),
the dot-product test of the wavelet gradient, central finite differences of the GPU misfit along
seeded smooth perturbations, and invariance to the checkpoint interval and to batching."""
import numpy as np
import pytest
from scipy.ndimage import gaussian_filter

import oracle_lib as ol
from conftest import rel_l2
from seismic_code_github_b200 import seisfd as S

pytestmark = pytest.mark.gpu

TOL_GRAD = 1e-4
NPX, F0, DT, DX = 8, 20.0, 5e-4, 10.0


def model(seed=0, nx=44, nz=36):
    rng = np.random.default_rng(seed)
    vp_i = (2000 + 400 * gaussian_filter(rng.random((nx, nz)), 3)).astype(np.float32)
    rho_i = (1900 + 400 * rng.random((nx, nz))).astype(np.float32)
    q_i = (30 + 120 * gaussian_filter(rng.random((nx, nz)), 2)).astype(np.float32)
    pad = lambda a: S.pad_model(a, NPX, NPX, NPX, NPX)
    return pad(vp_i), pad(rho_i), pad(q_i)


def shots_for(vp, nts, seed=1):
    rng = np.random.default_rng(seed)
    nx, nz = vp.shape
    out = []
    for i, nt in enumerate(nts):
        sx = int(rng.integers(NPX + 3, nx - NPX - 3))
        sz = int(rng.integers(NPX + 2, NPX + 8))
        rx = np.arange(NPX, nx - NPX, 2, dtype=np.int32)
        rz = np.full_like(rx, NPX + 2 + (i % 2))
        out.append(S.ShotSpec(sx, sz, rx, rz, S.wavelet(S.WAVELET_Q, nt, DT, F0)))
    return out


def engine(vp, rho, q):
    # the gradient is the adjoint of the reference-order scheme (its forward passes run those kernels
    # in either mode), so the forwards these tests compare with it run in SFD_EXACT mode too
    e = S.Engine(S.VISCOAC_2D, vp.shape[0], vp.shape[1], DX, DX, DT, NPX, order=10, f0=F0, flags=S.EXACT)
    e.set_model(vp, rho, q)
    return e


def observed(vp, rho, q, shots):
    with engine(vp, rho, q) as e:
        e.set_shots(shots)
        return e.forward()


def oracle(vp, rho, q, shots, obs_list):
    J, gv, gq = 0.0, np.zeros(vp.shape), np.zeros(vp.shape)
    for s, o in zip(shots, obs_list):
        out = ol.q_gradient_f64(vp, rho, q, s.wavelet, (s.sx, s.sz), s.rec_x, s.rec_z, NPX, DX, DX, DT, F0,
                                obs=o.reshape(len(s.rec_x), s.nt))
        J += out["misfit"]
        gv += out["grad_vp"]
        gq += out["grad_invq"]
    return J, gv, gq


@pytest.mark.parametrize("nts,interval", [([170], 0), ([180, 130, 150], 17)])
def test_gradient_matches_fp64_oracle(nts, interval):
    vp, rho, q = model(0)
    shots = shots_for(vp, nts)
    vp_true = (vp * 1.02).astype(np.float32)
    q_true = (q * 0.8).astype(np.float32)
    obs = observed(vp_true, rho, q_true, shots)
    with engine(vp, rho, q) as e:
        e.set_shots(shots)
        e.set_checkpoint_interval(interval)
        J, gv, gq = e.gradient(obs, want_invq=True)
        obs_list = e.split_records(obs)
        t = e.timing()
    Jo, gvo, gqo = oracle(vp, rho, q, shots, obs_list)
    ev, eq = rel_l2(gv, gvo), rel_l2(gq, gqo)
    print(f"shots {nts}: misfit {J:.6e} vs {Jo:.6e}; relL2 d/dvp {ev:.2e}, d/d(1/Q) {eq:.2e}; "
          f"{t['launches']} launches, {t['loop_ms']:.2f} ms")
    assert np.abs(gqo).max() > 0
    assert abs(J - Jo) <= 1e-4 * Jo
    assert ev <= TOL_GRAD
    assert eq <= TOL_GRAD


def test_dot_product_adjoint():
    """<F w2, r> = <w2, F^T r> for F: wavelet -> records at a fixed model; F^T r is the wavelet
    gradient of 0.5 |F w1 - obs|^2 with obs = F w1 - r."""
    vp, rho, q = model(3)
    rng = np.random.default_rng(11)
    shots = shots_for(vp, [160], seed=4)
    with engine(vp, rho, q) as e:
        e.set_shots(shots)
        d1 = e.forward()
        r = rng.standard_normal(d1.size).astype(np.float32)
        obs = (d1 - r).astype(np.float32)
        e.gradient(obs)
        ftr = e.wavelet_gradient(0).astype(np.float64)
        res = d1.astype(np.float64) - obs
        w2 = rng.standard_normal(160).astype(np.float32)
        s0 = shots[0]
        e.set_shots([S.ShotSpec(s0.sx, s0.sz, s0.rec_x, s0.rec_z, w2)])
        d2 = e.forward().astype(np.float64)
    lhs, rhs = float(np.dot(d2, res)), float(np.dot(w2.astype(np.float64), ftr))
    print(f"dot test: {lhs:.9e} vs {rhs:.9e} (rel {abs(lhs - rhs) / abs(lhs):.2e})")
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


@pytest.mark.parametrize("which", ["vp", "invq"])
def test_finite_differences_along_random_smooth_perturbations(which):
    vp, rho, q = model(5)
    shots = shots_for(vp, [200, 200], seed=3)
    obs = observed((vp * 1.03).astype(np.float32), rho, (q * 0.7).astype(np.float32), shots)
    rng = np.random.default_rng(8)
    with engine(vp, rho, q) as e:
        e.set_shots(shots)
        _, gv, gq = e.gradient(obs, want_invq=True)
        for trial in range(3):
            d = gaussian_filter(rng.standard_normal(vp.shape), 4)
            d /= np.abs(d).max()
            Js = []
            if which == "vp":
                dm = 1e-3 * vp * d
                for sgn in (1, -1):
                    e.set_model((vp + sgn * dm).astype(np.float32), rho, q)
                    Js.append(e.gradient(obs)[0])
                an = float(np.sum(gv.astype(np.float64) * dm))
            else:
                invq = 1.0 / q.astype(np.float64)
                dm = 3e-2 * invq * d
                for sgn in (1, -1):
                    e.set_model(vp, rho, (1.0 / (invq + sgn * dm)).astype(np.float32))
                    Js.append(e.gradient(obs)[0])
                an = float(np.sum(gq.astype(np.float64) * dm))
            e.set_model(vp, rho, q)
            fd = (Js[0] - Js[1]) / 2.0
            print(f"{which} trial {trial}: FD {fd:.6e} adjoint {an:.6e} rel {abs(fd - an) / abs(an):.2e}")
            assert abs(fd - an) <= 2e-2 * abs(an)


def test_checkpoint_interval_and_batched_vs_per_shot():
    vp, rho, q = model(7)
    shots = shots_for(vp, [150, 120, 150, 90], seed=6)
    obs = observed((vp * 0.98).astype(np.float32), rho, q, shots)
    out = {}
    with engine(vp, rho, q) as e:
        e.set_shots(shots)
        for key, interval, per_shot in [("a", 0, False), ("b", 7, False), ("c", 150, False), ("d", 11, True)]:
            e.set_checkpoint_interval(interval)
            out[key] = e.gradient(obs, want_invq=True, per_shot=per_shot)
    for key in "bcd":
        assert abs(out[key][0] - out["a"][0]) <= 1e-5 * out["a"][0]
        assert rel_l2(out[key][1], out["a"][1]) <= 1e-5
        assert rel_l2(out[key][2], out["a"][2]) <= 1e-5
