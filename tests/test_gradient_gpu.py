"""GPU gradient of the 2-D acoustic scheme through the C ABI (sfd_gradient): against the FP64
CPU adjoint oracle (relative L2 <= 1e-4, the gradient bar), the dot-product adjoint test,
central finite differences along seeded random smooth perturbations, invariance to the
checkpoint interval, and batched = per-shot."""
import numpy as np
import pytest

import oracle_lib as ol
from conftest import bits_equal, rel_l2
from seismic_code_github_b200 import seisfd as S
from seismic_code_github_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL_GRAD = 1e-4


def small_model(seed=0, NX=40, NZ=30, PML=10):
    rng = np.random.default_rng(seed)
    v = W.layered_model(NX, NZ, 3, 1800.0, 2600.0, seed=seed, anomalies=1, radius=5.0, amp=150.0)
    vp = W.pad_edges(v, PML, PML)
    den = W.pad_edges((2000.0 + 300.0 * rng.random((NX, NZ))).astype(np.float32), PML, PML)
    return vp, den, PML


def engine(vp, den, pml, dt=1e-3, dx=10.0, order=16):
    e = S.Engine(S.ACOUSTIC_2D, vp.shape[0], vp.shape[1], dx, dx, dt, pml, order=order)
    e.set_model(vp, den)
    return e


def shots_for(vp, pml, nts, seed=1, f0=25.0):
    rng = np.random.default_rng(seed)
    Nx, Nz = vp.shape
    out = []
    for i, nt in enumerate(nts):
        sx = int(rng.integers(pml + 2, Nx - pml - 2))
        sz = int(rng.integers(pml + 1, pml + 6))
        rx = np.arange(pml, Nx - pml, 2, dtype=np.int32)
        rz = np.full_like(rx, pml + 2 + (i % 2))
        w = S.wavelet(S.WAVELET_RIC, nt, 1e-3, f0, 40)
        out.append(S.ShotSpec(sx, sz, rx, rz, w))
    return out


def oracle_grad(vp, den, pml, shots, obs_list, dt=1e-3, dx=10.0, radius=8):
    J, g = 0.0, np.zeros(vp.shape)
    for s, obs in zip(shots, obs_list):
        j, gs, _, _ = ol.afd_gradient_f64(vp.shape[0], vp.shape[1], pml, s.nt, dx, dx, dt, vp, den, s.wavelet,
                                          s.sx, s.sz, s.rec_x, s.rec_z, obs, radius=radius)
        J += j
        g += gs
    return J, g


def observed(vp_true, den, pml, shots):
    with engine(vp_true, den, pml) as e:
        e.set_shots(shots)
        return e.forward()


@pytest.mark.parametrize("order", [16, 8])
def test_gradient_matches_fp64_oracle(order):
    vp, den, pml = small_model(0)
    shots = shots_for(vp, pml, [180, 140, 200])
    obs = observed((vp * 1.02).astype(np.float32), den, pml, shots)
    with engine(vp, den, pml, order=order) as e:
        e.set_shots(shots)
        e.set_checkpoint_interval(13)
        J, g, _ = e.gradient(obs)
        obs_list = e.split_records(obs)
        t = e.timing()
    Jo, go = oracle_grad(vp, den, pml, shots, obs_list, radius=order // 2)
    err = rel_l2(g, go)
    print(f"order {order}: misfit {J:.6e} vs {Jo:.6e}; gradient relL2 vs FP64 oracle {err:.3e}; "
          f"{t['launches']} launches, {t['loop_ms']:.2f} ms")
    assert abs(J - Jo) <= 1e-4 * Jo
    assert err <= TOL_GRAD


def test_dot_product_adjoint():
    """<F w2, r> = <w2, F^T r> with F: wavelet -> records at a fixed model; F^T r is the
    wavelet gradient of 0.5|F w1 - obs|^2 with obs = F w1 - r."""
    vp, den, pml = small_model(3)
    rng = np.random.default_rng(11)
    nt = 160
    shots = shots_for(vp, pml, [nt])
    with engine(vp, den, pml) as e:
        e.set_shots(shots)
        d1 = e.forward()
        r = rng.standard_normal(d1.size).astype(np.float32)
        obs = (d1 - r).astype(np.float32)
        e.gradient(obs)
        ftr = e.wavelet_gradient(0).astype(np.float64)
        res = (d1.astype(np.float64) - obs)  # what the adjoint saw
        w2 = rng.standard_normal(nt).astype(np.float32)
        s2 = S.ShotSpec(shots[0].sx, shots[0].sz, shots[0].rec_x, shots[0].rec_z, w2)
        e.set_shots([s2])
        d2 = e.forward().astype(np.float64)
    lhs = float(np.dot(d2, res))
    rhs = float(np.dot(w2.astype(np.float64), ftr))
    print(f"dot test: {lhs:.9e} vs {rhs:.9e} (rel {abs(lhs - rhs) / abs(lhs):.2e})")
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


def test_finite_differences_along_random_smooth_perturbations():
    vp, den, pml = small_model(5, NX=60, NZ=40)
    shots = shots_for(vp, pml, [220, 220], seed=3)
    obs = observed(W.pad_edges(W.layered_model(60, 40, 3, 1850.0, 2700.0, seed=9, anomalies=2, radius=6.0,
                                               amp=200.0), pml, pml), den, pml, shots)
    rng = np.random.default_rng(8)
    with engine(vp, den, pml) as e:
        e.set_shots(shots)
        J0, g, _ = e.gradient(obs)
        for trial in range(4):
            # smooth perturbation: a few random Gaussians, 1e-3 relative
            x = np.arange(vp.shape[0])[:, None]
            z = np.arange(vp.shape[1])[None, :]
            d = np.zeros(vp.shape)
            for _ in range(3):
                cx, cz = rng.uniform(pml, vp.shape[0] - pml), rng.uniform(pml, vp.shape[1] - pml)
                d += rng.standard_normal() * np.exp(-((x - cx) ** 2 + (z - cz) ** 2) / (2 * 6.0 ** 2))
            dvp = 1e-3 * vp * d / np.abs(d).max()
            Js = []
            for sgn in (1, -1):
                e.set_model((vp + sgn * dvp).astype(np.float32), den)
                Js.append(e.gradient(obs)[0])
            e.set_model(vp, den)
            fd = (Js[0] - Js[1]) / 2.0
            an = float(np.sum(g.astype(np.float64) * dvp))
            print(f"trial {trial}: FD {fd:.6e} adjoint {an:.6e} rel {abs(fd - an) / abs(an):.2e}")
            assert abs(fd - an) <= 2e-2 * abs(an)


def test_checkpoint_interval_and_batched_vs_per_shot():
    vp, den, pml = small_model(7)
    shots = shots_for(vp, pml, [150, 97, 150, 61], seed=5)
    obs = observed((vp * 0.99).astype(np.float32), den, pml, shots)
    with engine(vp, den, pml) as e:
        e.set_shots(shots)
        grads = {}
        for C in (1, 7, 0, 150):
            e.set_checkpoint_interval(C)
            grads[C] = e.gradient(obs)[1]
        e.set_checkpoint_interval(0)
        Jb, gb, _ = e.gradient(obs)
        Jp, gp, _ = e.gradient(obs, per_shot=True)
    for C, g in grads.items():
        assert rel_l2(g, grads[0]) < 1e-6, C
    assert bits_equal(gb, gp)
    assert Jb == Jp


def test_config4_geometry_short_record_properties():
    """Config-4 geometry (384 x 1536 interior, 50-cell sponge, dx 10 m, dt 1 ms), 8 shots and
    120 steps: the batched gradient equals the per-shot gradient and agrees with central
    finite differences along a smooth perturbation."""
    NX, NZ, PML = 1536, 384, 50
    v = W.layered_model(NX, NZ, 8, 1500.0, 3500.0, seed=44, anomalies=3, radius=30.0, amp=300.0, dx=10.0)
    vp = W.pad_edges(v, PML, PML)
    den = np.full_like(vp, 2200.0)
    rng = np.random.default_rng(4)
    shots = []
    for i in range(8):
        sx = PML + int((i + 0.5) * NX / 8)
        rx = np.arange(PML, PML + NX, 4, dtype=np.int32)
        rz = np.full_like(rx, PML + 2)
        shots.append(S.ShotSpec(sx, PML + 2, rx, rz, S.wavelet(S.WAVELET_RIC, 120, 1e-3, 25.0, 40)))
    true = (vp * (1.0 + 0.02 * rng.standard_normal() )).astype(np.float32)
    obs = observed(true, den, PML, shots)
    with engine(vp, den, PML) as e:
        e.set_shots(shots)
        Jb, gb, _ = e.gradient(obs)
        Jp, gp, _ = e.gradient(obs, per_shot=True)
        assert bits_equal(gb, gp) and Jb == Jp
        x = np.arange(vp.shape[0])[:, None]
        z = np.arange(vp.shape[1])[None, :]
        d = np.exp(-((x - 600) ** 2 + (z - 120) ** 2) / (2 * 40.0 ** 2))
        dvp = 1e-3 * vp * d
        Js = []
        for sgn in (1, -1):
            e.set_model((vp + sgn * dvp).astype(np.float32), den)
            Js.append(e.gradient(obs)[0])
    fd = (Js[0] - Js[1]) / 2.0
    an = float(np.sum(gb.astype(np.float64) * dvp))
    print(f"config-4 geometry: FD {fd:.6e} adjoint {an:.6e}")
    assert abs(fd - an) <= 2e-2 * abs(an)
