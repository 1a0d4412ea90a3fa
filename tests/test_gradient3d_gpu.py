"""GPU gradient of the 3-D acoustic scheme (SFD_ACOUSTIC_3D) through the C ABI: d misfit / d vp
against the FP64 3-D adjoint oracle (oracle/adj3d_oracle.cpp, relative L2 <= 1e-4), the
dot-product test of the wavelet gradient, central finite differences of the GPU misfit, and the
memory-planned schedules (shot groups, one or two checkpoint levels) against each other."""
import numpy as np
import pytest
from scipy.ndimage import gaussian_filter

import oracle_lib as ol
from conftest import rel_l2
from seismic_code_github_b200 import seisfd as S

pytestmark = pytest.mark.gpu

TOL_GRAD = 1e-4
D, DT, PML = 10.0, 1e-3, 7


def model(seed=0, n=(36, 32, 40), varden=True):
    rng = np.random.default_rng(seed)
    vp = (2000.0 + 600.0 * gaussian_filter(rng.random(n), 2)).astype(np.float32)
    den = (1900.0 + 300.0 * rng.random(n)).astype(np.float32) if varden else None
    return vp, den


def shots_for(vp, nts, seed=1):
    rng = np.random.default_rng(seed)
    nx, ny, nz = vp.shape
    out = []
    for i, nt in enumerate(nts):
        src = (int(rng.integers(PML + 2, nx - PML - 2)), int(rng.integers(PML + 2, ny - PML - 2)),
               int(rng.integers(PML + 1, PML + 5)))
        rx = np.repeat(np.arange(PML, nx - PML, 3, dtype=np.int32), 3)
        ry = np.tile(np.array([PML + 2, ny // 2, ny - PML - 3], np.int32), len(rx) // 3)
        rz = np.full_like(rx, PML + 1 + (i % 2))
        w = S.wavelet(S.WAVELET_RIC, nt, DT, 28.0, 25)
        out.append(S.ShotSpec(src[0], src[2], rx, rz, w, sy=src[1], rec_y=ry))
    return out


def engine(vp, den, order=8):
    nx, ny, nz = vp.shape
    e = S.Engine(S.ACOUSTIC_3D, nx, nz, D, D, DT, PML, order=order, ny=ny, dy=D)
    e.set_model(vp, den)
    return e


def observed(vp, den, shots, order=8):
    with engine(vp, den, order) as e:
        e.set_shots(shots)
        return e.forward()


def oracle(vp, den, shots, obs_list, order=8):
    J, g = 0.0, np.zeros(vp.shape)
    for s, o in zip(shots, obs_list):
        out = ol.afd3d_gradient_f64(vp, den, s.wavelet, (s.sx, s.sy, s.sz), s.rec_x, s.rec_y, s.rec_z, PML, D, D, D,
                                    DT, obs=o.reshape(len(s.rec_x), s.nt), radius=order // 2)
        J += out["misfit"]
        g += out["grad_vp"]
    return J, g


@pytest.mark.parametrize("order,nts,varden", [(8, [110], True), (4, [120, 90, 105], False)])
def test_gradient_matches_fp64_oracle(order, nts, varden):
    vp, den = model(0, varden=varden)
    shots = shots_for(vp, nts)
    obs = observed((vp * 1.02).astype(np.float32), den, shots, order)
    with engine(vp, den, order) as e:
        e.set_shots(shots)
        J, g, _ = e.gradient(obs)
        obs_list = e.split_records(obs)
        t = e.timing()
    Jo, go = oracle(vp, den, shots, obs_list, order)
    err = rel_l2(g, go)
    print(f"order {order} shots {nts}: misfit {J:.6e} vs {Jo:.6e}; relL2 {err:.2e}; variant {t['kernel_variant']}, "
          f"{t['launches']} launches, {t['loop_ms']:.2f} ms")
    assert abs(J - Jo) <= 1e-4 * Jo
    assert err <= TOL_GRAD


def test_dot_product_adjoint():
    vp, den = model(3)
    shots = shots_for(vp, [100], seed=4)
    rng = np.random.default_rng(11)
    with engine(vp, den) as e:
        e.set_shots(shots)
        d1 = e.forward()
        r = rng.standard_normal(d1.size).astype(np.float32)
        obs = (d1 - r).astype(np.float32)
        e.gradient(obs)
        ftr = e.wavelet_gradient(0).astype(np.float64)
        res = d1.astype(np.float64) - obs
        w2 = rng.standard_normal(100).astype(np.float32)
        s0 = shots[0]
        e.set_shots([S.ShotSpec(s0.sx, s0.sz, s0.rec_x, s0.rec_z, w2, sy=s0.sy, rec_y=s0.rec_y)])
        d2 = e.forward().astype(np.float64)
    lhs, rhs = float(np.dot(d2, res)), float(np.dot(w2.astype(np.float64), ftr))
    print(f"dot test: {lhs:.9e} vs {rhs:.9e} (rel {abs(lhs - rhs) / abs(lhs):.2e})")
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


def test_finite_differences():
    vp, den = model(5)
    shots = shots_for(vp, [120], seed=3)
    obs = observed((vp * 1.03).astype(np.float32), den, shots)
    rng = np.random.default_rng(8)
    with engine(vp, den) as e:
        e.set_shots(shots)
        _, g, _ = e.gradient(obs)
        for trial in range(2):
            d = gaussian_filter(rng.standard_normal(vp.shape), 3)
            d /= np.abs(d).max()
            s0 = shots[0]
            d[s0.sx, s0.sy, s0.sz] = 0.0  # the float-rounded injection scale is a staircase in vp there
            dm = 1e-3 * vp * d
            Js = []
            for sgn in (1, -1):
                e.set_model((vp + sgn * dm).astype(np.float32), den)
                Js.append(e.gradient(obs)[0])
            e.set_model(vp, den)
            fd = (Js[0] - Js[1]) / 2.0
            an = float(np.sum(g.astype(np.float64) * dm))
            print(f"trial {trial}: FD {fd:.6e} adjoint {an:.6e} rel {abs(fd - an) / abs(an):.2e}")
            assert abs(fd - an) <= 2e-2 * abs(an)


def test_memory_planned_schedules_agree():
    """The largest-group one-level schedule, one shot per group with two checkpoint levels (forced
    by a memory budget) and the per-shot schedule give the same gradient."""
    vp, den = model(7, varden=False)
    shots = shots_for(vp, [120, 100, 120], seed=6)
    obs = observed((vp * 0.98).astype(np.float32), den, shots)
    nx, ny, nz = vp.shape
    F = 4 * nx * ny * ((nz + 3) // 4 * 4)
    nrec = sum(s.nrec * s.nt for s in shots)
    fixed = 8 * nx * ny * nz + 16 * nrec + 4 * len(shots) * 120
    out = {}
    with engine(vp, den) as e:
        e.set_shots(shots)
        out["batched"] = e.gradient(obs) + (e.timing()["kernel_variant"],)
        e.set_checkpoint_interval(6)
        e.set_memory_limit(fixed + 80 * F)  # one slot: one level needs 105 F, two levels 61 F
        out["two_level"] = e.gradient(obs) + (e.timing()["kernel_variant"],)
        e.set_memory_limit(0)
        e.set_checkpoint_interval(0)
        out["per_shot"] = e.gradient(obs, per_shot=True) + (e.timing()["kernel_variant"],)
        fwd = e.forward()  # the forward grows the wavefields back after the gradient shrank them
    assert out["batched"][3] == 61 and out["two_level"][3] == 62
    assert np.array_equal(fwd, observed(vp, den, shots)) and np.abs(fwd).max() > 0
    for k in ("two_level", "per_shot"):
        assert abs(out[k][0] - out["batched"][0]) <= 1e-5 * out["batched"][0]
        assert rel_l2(out[k][1], out["batched"][1]) <= 1e-5, k
