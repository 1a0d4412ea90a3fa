"""GPU parity of the x-marching forward kernel of the default (FMA) scheme.

The x-marching kernel (a CTA walks down x over one 64-wide z strip of one shot, 16 columns per
chunk, double-buffered TMA) stages the fields differently from the tile kernel but performs the
same operations on the same values, so its records, snapshots and gradients must equal the tile
kernel's bit for bit -- at every order, with constant and variable density, for uneven shots with
apertures, and for segment lengths down to a single chunk (16 columns, where every segment starts
with its warm-up chunk).  It must also stay within the forward tolerance (relative L2 <= 1e-5) of
the oracle restatement of forward/Acoustic_FD_by_ss/src/Acoustic_1order_FD.cpp:237-380."""
import numpy as np
import pytest

import oracle_lib as ol
from conftest import bits_equal, rel_l2
from seismic_code_github_b200 import seisfd as S
from seismic_code_github_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL_FWD = 1e-5
SEGS = [16, 48, 128, 512]


def run_forward(monkeypatch, kind, vp, den, pml, shots, order=16, dx=10.0, dt=1e-3, snap=None):
    """kind: ("tile",) or ("march", seg).  Returns (records, kernel_variant, snapshots or None)."""
    if kind[0] == "tile":
        monkeypatch.delenv("SFD_MARCH_SEG", raising=False)
        monkeypatch.setenv("SFD_FMA_STAGES", "1")
    else:
        monkeypatch.delenv("SFD_FMA_STAGES", raising=False)
        monkeypatch.setenv("SFD_MARCH_SEG", str(kind[1]))
    with S.Engine(S.ACOUSTIC_2D, vp.shape[0], vp.shape[1], dx, dx, dt, pml, order=order) as e:
        e.set_model(vp, den)
        e.set_shots(shots)
        if snap:
            e.set_snapshots(0, S.FIELD_P, *snap)
        rec = e.forward().copy()
        v = e.timing()["kernel_variant"]
        sn = e.snapshots(0, 0).copy() if snap else None
    return rec, v, sn


def uneven_case():
    NX, NZ, PML = 300, 200, 20
    v = W.layered_model(NX, NZ, 5, 1800.0, 3500.0, seed=5, anomalies=2, radius=12.0, amp=250.0, dx=10.0)
    vp = W.pad_edges(v, PML, PML)
    den = (2100.0 + 300.0 * np.random.default_rng(4).random(vp.shape)).astype(np.float32)
    rx = np.arange(PML, vp.shape[0] - PML, dtype=np.int32)
    rz = np.full_like(rx, PML + 2)
    shots = []
    for i, (sx, sz, nt) in enumerate(((PML + 40, PML + 3, 260), (PML + 150, PML + 100, 200), (PML + 290, PML + 5, 130))):
        w = S.wavelet(S.WAVELET_RIC, nt, 1e-3, 20.0 + i, 50)
        shots.append(S.ShotSpec(sx, sz, rx, rz, w))
    return vp, den, PML, shots


@pytest.mark.parametrize("order", [16, 10, 8, 4, 2])
@pytest.mark.parametrize("varden", [True, False])
def test_march_equals_tile_all_orders(monkeypatch, order, varden):
    case = W.small_varden()
    w = S.wavelet(S.WAVELET_RIC, 180, case.dt, case.f0, 60)
    rx, rz = case.receivers()
    den = case.den if varden else None
    shots = [S.ShotSpec(case.src_x[0], case.src_z[0], rx, rz, w)]
    tile, vt, _ = run_forward(monkeypatch, ("tile",), case.vp, den, case.PML, shots, order, case.dx, case.dt)
    assert vt == 11
    ref, _, _ = ol.afd_forward(case.Nx, case.Nz, case.PML, 180, case.dx, case.dz, case.dt, case.vp,
                               case.den if varden else np.full_like(case.vp, 2400.0), w, case.src_x[0],
                               case.src_z[0], rx, rz, radius=order // 2)
    for seg in (16, 48):
        got, v, _ = run_forward(monkeypatch, ("march", seg), case.vp, den, case.PML, shots, order, case.dx, case.dt)
        assert v == 13
        assert bits_equal(got, tile), f"order {order} seg {seg}: max diff {np.abs(got - tile).max()}"
        assert rel_l2(got.reshape(ref.shape), ref) <= TOL_FWD


@pytest.mark.parametrize("seg", SEGS)
def test_march_uneven_shots_apertures(monkeypatch, seg):
    """Three shots with different record lengths and apertures, a P snapshot stream of the first
    shot, and a source near the grid edge: records and snapshots equal the tile kernel's."""
    vp, den, PML, shots = uneven_case()
    nx = vp.shape[0]
    ap = [(0, nx), (60, 200), (150, nx - 150)]
    sh = []
    for s, (x0, w) in zip(shots, ap):
        rx = np.arange(PML, w - PML, dtype=np.int32)
        sh.append(S.ShotSpec(min(s.sx, w - PML - 3), s.sz, rx, np.full_like(rx, PML + 2 + (x0 % 7)), s.wavelet,
                             ap_x0=x0, ap_nx=w))
    snap = (10, 40, 4)
    tile, _, tsn = run_forward(monkeypatch, ("tile",), vp, den, PML, sh, snap=snap)
    got, v, gsn = run_forward(monkeypatch, ("march", seg), vp, den, PML, sh, snap=snap)
    assert v == 13
    assert bits_equal(got, tile)
    assert bits_equal(gsn, tsn)
    # and the oracle for the full-width shot
    r0 = ol.afd_forward(nx, vp.shape[1], PML, sh[0].nt, 10.0, 10.0, 1e-3, vp, den, sh[0].wavelet, sh[0].sx, sh[0].sz,
                        sh[0].rec_x, sh[0].rec_z)[0]
    n0 = sh[0].nrec * sh[0].nt
    assert rel_l2(got[:n0].reshape(r0.shape), r0) <= TOL_FWD


def test_march_config2_geometry(monkeypatch):
    """The benchmark geometry (512 x 2048 interior, 612 x 2148 padded, 16th order) with 3 shots and
    60 steps: the last z strip is partly outside the grid, segments of 256 columns."""
    case = W.config2(nshot=3, nt=60)
    w = S.wavelet(S.WAVELET_RIC, case.nt, case.dt, case.f0, 20)
    rx, rz = case.receivers()
    shots = [S.ShotSpec(sx, sz, rx, rz, w) for sx, sz in zip(case.src_x, case.src_z)]
    tile, _, _ = run_forward(monkeypatch, ("tile",), case.vp, case.den, case.PML, shots, 16, case.dx, case.dt)
    got, v, _ = run_forward(monkeypatch, ("march", 256), case.vp, case.den, case.PML, shots, 16, case.dx, case.dt)
    assert v == 13 and np.abs(tile).max() > 0
    assert bits_equal(got, tile)


def test_march_gradient_bits(monkeypatch):
    """The gradient's forward and recomputation run on the x-marching kernel (with the D_k output):
    misfit and gradient equal the tile kernel's bit for bit."""
    vp, den, PML, shots = uneven_case()
    out = {}
    for kind in (("tile",), ("march", 48)):
        if kind[0] == "tile":
            monkeypatch.delenv("SFD_MARCH_SEG", raising=False)
            monkeypatch.setenv("SFD_FMA_STAGES", "1")
        else:
            monkeypatch.delenv("SFD_FMA_STAGES", raising=False)
            monkeypatch.setenv("SFD_MARCH_SEG", str(kind[1]))
        with S.Engine(S.ACOUSTIC_2D, vp.shape[0], vp.shape[1], 10.0, 10.0, 1e-3, PML, order=16) as e:
            e.set_model(vp, den)
            e.set_shots(shots)
            rec = e.forward().copy()
            e.set_model((vp * 1.01).astype(np.float32), den)
            e.set_checkpoint_interval(30)
            J, g, _ = e.gradient(rec)
        out[kind[0]] = (rec, J, g.copy())
    assert bits_equal(out["tile"][0], out["march"][0])
    assert out["tile"][1] == out["march"][1] and bits_equal(out["tile"][2], out["march"][2])


def test_tuner_candidates_agree():
    """Whatever the tuner picks for this shot set, the records equal the tile kernel's; the pick is
    reported as kernel_variant 11, 12 (tile schedules) or 13 (x-marching)."""
    vp, den, PML, shots = uneven_case()
    with S.Engine(S.ACOUSTIC_2D, vp.shape[0], vp.shape[1], 10.0, 10.0, 1e-3, PML, order=16) as e:
        e.set_model(vp, den)
        e.set_shots(shots)
        rec = e.forward().copy()
        v = e.timing()["kernel_variant"]
    with S.Engine(S.ACOUSTIC_2D, vp.shape[0], vp.shape[1], 10.0, 10.0, 1e-3, PML, order=16) as e:
        e.set_model(vp, den)
        e.set_shots(shots)
        ref = e.forward_per_shot().copy()
    assert v in (11, 12, 13)
    assert bits_equal(rec, ref)
