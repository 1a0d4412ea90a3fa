"""GPU parity of every schedule of the FMA step kernel (SFD_ACOUSTIC_2D without SFD_EXACT).  The
tuner picks the faster schedule at run time; SFD_FMA_STAGES forces one, so each is checked here:
1 = one tile per CTA with two CTAs per SM, 2 = persistent CTAs with double-buffered TMA.  Each
must stay within the forward tolerance of the oracle restatement (relative L2 <= 1e-5), at every
order, with variable density, on sponge-free interior tiles and for uneven shots, and carry the
adjoint gradient to within 1e-4 of the FP64 adjoint oracle (the gradient's forward and its
recomputation run under the forced schedule).  Forward steps number their CTAs tile-major by
default (SFD_TILE_MAJOR=0 selects shot-major); every case runs under both numberings, and the
two must give the same bits."""
import numpy as np
import pytest

import oracle_lib as ol
from conftest import bits_equal, rel_l2
from seismic_code_github_b200 import seisfd as S
from seismic_code_github_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL_FWD = 1e-5
SCHEDULES = [1, 2]


@pytest.fixture(params=[(s, m) for s in SCHEDULES for m in (1, 0)], ids=lambda p: f"s{p[0]}-tm{p[1]}")
def schedule(request, monkeypatch):
    s, m = request.param
    monkeypatch.setenv("SFD_FMA_STAGES", str(s))
    monkeypatch.setenv("SFD_TILE_MAJOR", str(m))
    return s


@pytest.mark.parametrize("order", [16, 10, 8, 4, 2])
def test_all_orders_variable_density(schedule, order):
    case = W.small_varden()
    w = S.wavelet(S.WAVELET_RIC, 200, case.dt, case.f0, 60)
    rx, rz = case.receivers()
    with S.Engine(S.ACOUSTIC_2D, case.Nx, case.Nz, case.dx, case.dz, case.dt, case.PML, order=order) as e:
        e.set_model(case.vp, case.den)
        e.set_shots([S.ShotSpec(case.src_x[0], case.src_z[0], rx, rz, w)])
        rec = e.forward().reshape(len(rx), 200)
        t = e.timing()
    ref, _, _ = ol.afd_forward(case.Nx, case.Nz, case.PML, 200, case.dx, case.dz, case.dt, case.vp, case.den, w,
                               case.src_x[0], case.src_z[0], rx, rz, radius=order // 2)
    err = rel_l2(rec, ref)
    print(f"schedule {schedule} order {order}: relL2 vs oracle {err:.3e}")
    assert t["kernel_variant"] == 10 + schedule
    assert err <= TOL_FWD


def uneven_shots_case():
    NX, NZ, PML = 300, 200, 20
    v = W.layered_model(NX, NZ, 5, 1800.0, 3500.0, seed=5, anomalies=2, radius=12.0, amp=250.0, dx=10.0)
    vp = W.pad_edges(v, PML, PML)
    den = np.full_like(vp, 2200.0)
    rx = np.arange(PML, vp.shape[0] - PML, dtype=np.int32)
    rz = np.full_like(rx, PML + 2)
    shots = []
    for i, (sx, sz, nt) in enumerate(((PML + 40, PML + 3, 260), (PML + 150, PML + 100, 200), (PML + 290, PML + 5, 130))):
        w = S.wavelet(S.WAVELET_RIC, nt, 1e-3, 20.0 + i, 50)
        shots.append(S.ShotSpec(sx, sz, rx, rz, w))
    return vp, den, PML, shots


def test_interior_tiles_uneven_shots(schedule):
    vp, den, PML, shots = uneven_shots_case()
    refs = [ol.afd_forward(vp.shape[0], vp.shape[1], PML, s.nt, 10.0, 10.0, 1e-3, vp, den, s.wavelet, s.sx, s.sz,
                           s.rec_x, s.rec_z)[0] for s in shots]
    with S.Engine(S.ACOUSTIC_2D, vp.shape[0], vp.shape[1], 10.0, 10.0, 1e-3, PML, order=16) as e:
        e.set_model(vp, den)
        e.set_shots(shots)
        got = e.split_records(e.forward())
    for g, r in zip(got, refs):
        assert rel_l2(g, r) <= TOL_FWD


def test_gradient_against_fp64_adjoint(schedule):
    NX, NZ, PML = 60, 48, 12
    vt = W.pad_edges(W.layered_model(NX, NZ, 3, 1900.0, 2700.0, seed=8, anomalies=1, radius=5.0, amp=200.0), PML, PML)
    vp = (vt * 0.97).astype(np.float32)
    den = (2000.0 + 200.0 * np.random.default_rng(2).random(vp.shape)).astype(np.float32)
    rx = np.arange(PML, vp.shape[0] - PML, 2, dtype=np.int32)
    rz = np.full_like(rx, PML + 2)
    shots = [S.ShotSpec(PML + 10 + 15 * i, PML + 3, rx, rz, S.wavelet(S.WAVELET_RIC, nt, 1e-3, 25.0, 40))
             for i, nt in enumerate((220, 170))]
    obs = [ol.afd_forward(vp.shape[0], vp.shape[1], PML, s.nt, 10.0, 10.0, 1e-3, vt, den, s.wavelet, s.sx, s.sz, rx,
                          rz)[0].astype(np.float32) for s in shots]
    with S.Engine(S.ACOUSTIC_2D, vp.shape[0], vp.shape[1], 10.0, 10.0, 1e-3, PML, order=16) as e:
        e.set_model(vp, den)
        e.set_shots(shots)
        e.set_checkpoint_interval(20)
        misfit, g, _ = e.gradient(np.concatenate([o.ravel() for o in obs]))
    J, g64 = 0.0, np.zeros(vp.shape)
    for s, o in zip(shots, obs):
        j, gs, _, _ = ol.afd_gradient_f64(vp.shape[0], vp.shape[1], PML, s.nt, 10.0, 10.0, 1e-3, vp, den, s.wavelet,
                                          s.sx, s.sz, rx, rz, o)
        J += j
        g64 += gs
    err = rel_l2(g, g64)
    print(f"schedule {schedule}: gradient relL2 vs FP64 adjoint {err:.2e}")
    assert err <= 1e-4 and abs(misfit - J) <= 1e-3 * J


def test_tile_numbering_gives_identical_bits(monkeypatch):
    """Tile-major and shot-major CTA numbering visit the same tiles with the same arithmetic: the
    records of a multi-shot forward and the batched gradient agree bit for bit."""
    vp, den, PML, shots = uneven_shots_case()
    out = {}
    for m in (1, 0):
        monkeypatch.setenv("SFD_TILE_MAJOR", str(m))
        with S.Engine(S.ACOUSTIC_2D, vp.shape[0], vp.shape[1], 10.0, 10.0, 1e-3, PML, order=16) as e:
            e.set_model(vp, den)
            e.set_shots(shots)
            rec = e.forward().copy()
            e.set_model((vp * 1.01).astype(np.float32), den)
            J, g, _ = e.gradient(rec)
        out[m] = (rec, J, g)
    assert bits_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1] and bits_equal(out[0][2], out[1][2])


def test_second_device_in_the_same_process():
    """The step kernels' shared-memory size attribute is set per device: a forward on device 0 and
    then on device 1 of the same process both run (needs two visible GPUs)."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("one GPU visible")
    case = W.small_varden()
    w = S.wavelet(S.WAVELET_RIC, 80, case.dt, case.f0, 40)
    rx, rz = case.receivers()
    recs = []
    for dev in (0, 1):
        with S.Engine(S.ACOUSTIC_2D, case.Nx, case.Nz, case.dx, case.dz, case.dt, case.PML, order=16,
                      device=dev) as e:
            e.set_model(case.vp, case.den)
            e.set_shots([S.ShotSpec(case.src_x[0], case.src_z[0], rx, rz, w)])
            recs.append(e.forward().copy())
    assert bits_equal(recs[0], recs[1])
