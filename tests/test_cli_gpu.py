"""GPU checks of the file-contract programs and of the in-loop snapshots.

  * afd_fd with no options writes the reference's own record.dat / Snap.dat / Model.dat
    (forward/Acoustic_FD_by_ss/file/) bit for bit; on a reduced grid with Pall.dat switched on
    it matches the patched reference build (fixture tests/golden/afd_small) file for file.
  * q_forward on a parameter card of three aperture shots writes merged SU files whose traces
    equal the FP32 restatement of Q_forward per shot (bit for bit) and whose headers follow
    QS:1502-1533; the per-shot parts are deleted as in QS:1582.
  * sfd_set_snapshots: each recorded interior equals the wavefield of a run stopped after that
    step (both schemes, batched and per-shot paths).
"""
import os
import subprocess

import numpy as np
import pytest

import oracle_lib as ol
from conftest import GOLDEN, ROOT, bits_equal, rel_l2
from seismic_code_github_b200 import seisfd as S
from seismic_code_github_b200 import workloads as W
from test_fileio import CARD, expected_header

pytestmark = pytest.mark.gpu
BIN = os.path.join(ROOT, "seismic_code_github_b200", "bin")


def run(cmd, cwd):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return r


def read(path, shape=None):
    a = np.fromfile(path, np.float32)
    return a if shape is None else a.reshape(shape)


def test_afd_fd_default_reproduces_the_shipped_outputs(tmp_path):
    (tmp_path / "file").mkdir()
    (tmp_path / "bin").mkdir()
    run([os.path.join(BIN, "afd_fd")], cwd=tmp_path / "bin")  # writes ../file like the reference
    for f in ("record.dat", "Snap.dat", "Model.dat"):
        got, ref = read(tmp_path / "file" / f), read(os.path.join(GOLDEN, "afd_default", f))
        assert bits_equal(got, ref), f
    assert read(tmp_path / "file" / "Pall.dat").size == 200 * 100 * 100


def test_afd_fd_small_case_with_pall_matches_the_reference_build(tmp_path):
    run([os.path.join(BIN, "afd_fd"), "--nx", "40", "--nz", "40", "--pml", "10", "--nt", "150", "--dt", "0.001",
         "--snap", "100", "--out", str(tmp_path)], cwd=tmp_path)
    for f in ("record.dat", "Snap.dat", "Model.dat", "Pall.dat"):
        got, ref = read(tmp_path / f), read(os.path.join(GOLDEN, "afd_small", f))
        assert got.shape == ref.shape and bits_equal(got, ref), f


def test_afd_fd_fast_path_within_tolerance(tmp_path):
    run([os.path.join(BIN, "afd_fd"), "--fast", "--out", str(tmp_path), "--pall-every", "0"], cwd=tmp_path)
    got, ref = read(tmp_path / "record.dat"), read(os.path.join(GOLDEN, "afd_default", "record.dat"))
    assert rel_l2(got, ref) <= 1e-5
    assert not (tmp_path / "Pall.dat").exists()


def qcard_case(tmp_path, elastic=False):
    nx, nz = 120, 80
    rng = np.random.default_rng(11)
    z = np.arange(nz)
    vp = np.tile(np.where(z < 40, 2000.0, 2600.0), (nx, 1)).astype(np.float32)
    vp += rng.uniform(-50, 50, vp.shape).astype(np.float32)
    rho = (2000.0 + 300.0 * rng.random((nx, nz))).astype(np.float32)
    qp = (30.0 + 150.0 * rng.random((nx, nz))).astype(np.float32)
    vs = (vp / 1.8).astype(np.float32) if elastic else vp * 0
    qs = (0.7 * qp).astype(np.float32) if elastic else qp
    for name, a in (("vp", vp), ("vs", vs), ("rho", rho), ("qp", qp), ("qs", qs)):
        a.tofile(tmp_path / f"{name}.bin")
    card = CARD.format(d=str(tmp_path)).replace("0.001\n", "0.0005\n").replace("500\n!*dt", "400\n!*dt")
    (tmp_path / "card.par").write_text(card)
    return S.read_qpar(str(tmp_path / "card.par")), vp, vs, rho, qp, qs


@pytest.mark.parametrize("use_q,elastic", [(False, False), (True, False), (True, True)])
def test_q_forward_program_against_restatement(tmp_path, use_q, elastic):
    p, vp, vs, rho, qp, qs = qcard_case(tmp_path, elastic)
    assert p.nt == 400 and np.float32(p.dt) == np.float32(0.0005)
    cmd = [os.path.join(BIN, "q_forward"), str(tmp_path / "card.par")] + (["--use-q"] if use_q else [])
    run(cmd, cwd=tmp_path)
    nint = lambda v: int(np.floor(abs(v) + 0.5)) * (1 if v >= 0 else -1)
    np_ = nint(p.pml_xn / p.dx) + 1
    isx0, nsz0, nrz0 = nint(p.sx0 / p.dx) + 1, nint(p.sz0 / p.dz) + 1, nint(p.rz0 / p.dz) + 1
    for stem in ("pz", "px"):
        assert not (tmp_path / f"{stem}_tmp1.su").exists()
        raw = open(tmp_path / f"shot_{stem}.su", "rb").read()
        off = 0
        for i in range(1, p.nshot + 1):
            isx = isx0 + nint((i - 1) * p.dsx / p.dx)
            ixmine, ixmaxe = isx + nint(p.offset_min / p.dx), isx + nint(p.offset_max / p.dx)
            nxe = ixmaxe - ixmine + 1
            r1, r2, _ = ol.q_forward(vp, vs, rho, qp, qs, p.dx, p.dz, p.dt, p.f0, p.nt, np_, np_,
                                     isx - ixmine + np_ + 1, nsz0 + np_ + 1, nrz0=nrz0, ixmine=ixmine,
                                     ixmaxe=ixmaxe, q_override=not use_q)
            ref = r1 if stem == "pz" else r2
            for t in range(nxe):
                rec = raw[off:off + 240 + 4 * p.nt]
                off += 240 + 4 * p.nt
                assert rec[:240] == expected_header(i, isx, ixmine, p.dx, p.dt, p.nt, t + 1)
                assert bits_equal(np.frombuffer(rec[240:], np.float32), ref[t]), (stem, i, t)
        assert off == len(raw)


def test_snapshots_equal_truncated_runs_acoustic():
    case = W.small_varden()
    rx, rz = case.receivers()
    w = S.wavelet(S.WAVELET_RIC, 60, case.dt, 20.0, 20)
    shots = [S.ShotSpec(case.src_x[0], case.src_z[0], rx, rz, w),
             S.ShotSpec(case.src_x[0] + 9, case.src_z[0] - 5, rx, rz, w[:45])]
    pml = case.PML
    with S.Engine(S.ACOUSTIC_2D, case.Nx, case.Nz, case.dx, case.dz, case.dt, pml, flags=S.EXACT) as e:
        e.set_model(case.vp, case.den)
        e.set_shots(shots)
        e.set_snapshots(0, S.FIELD_P, 3, 7, 6)
        e.set_snapshots(1, S.FIELD_VX, 10, 20, 3)
        e.forward()
        got = [[e.snapshots(sid, s) for s in range(2)] for sid in range(2)]
        e.forward_per_shot()
        per = [[e.snapshots(sid, s) for s in range(2)] for sid in range(2)]
    assert [g.shape[0] for g in got[0]] == [6, 6] and [g.shape[0] for g in got[1]] == [3, 2]
    for a, b in zip(sum(got, []), sum(per, [])):
        assert bits_equal(a, b)
    for sid, field, first, every in ((0, S.FIELD_P, 3, 7), (1, S.FIELD_VX, 10, 20)):
        for s in range(2):
            for j, snap in enumerate(got[sid][s]):
                k = first + j * every
                with S.Engine(S.ACOUSTIC_2D, case.Nx, case.Nz, case.dx, case.dz, case.dt, pml, flags=S.EXACT) as e:
                    e.set_model(case.vp, case.den)
                    sh = shots[s]
                    e.set_shots([S.ShotSpec(sh.sx, sh.sz, rx, rz, sh.wavelet[:k + 1])])
                    e.forward()
                    full = e.wavefield(0, field)
                assert bits_equal(snap, full[pml:-pml, pml:-pml]), (sid, s, k)


@pytest.mark.parametrize("flags", [0, S.EXACT], ids=["fused", "exact"])
def test_snapshots_equal_truncated_runs_viscoacoustic(flags):
    rng = np.random.default_rng(3)
    npx, f0, dt, dx = 8, 20.0, 5e-4, 10.0
    vp = S.pad_model((2000 + 300 * rng.random((40, 36))).astype(np.float32), npx, npx, npx, npx)
    rho = np.full_like(vp, 2100.0)
    q = S.pad_model((40 + 100 * rng.random((40, 36))).astype(np.float32), npx, npx, npx, npx)
    r = np.arange(npx, vp.shape[0] - npx, dtype=np.int32)
    w = S.wavelet(S.WAVELET_Q, 90, dt, f0)
    with S.Engine(S.VISCOAC_2D, vp.shape[0], vp.shape[1], dx, dx, dt, npx, order=10, f0=f0, flags=flags) as e:
        e.set_model(vp, rho, q)
        e.set_shots([S.ShotSpec(20, 12, r, np.full_like(r, 10), w)])
        e.set_snapshots(2, S.FIELD_P, 9, 40, 3)
        e.set_snapshots(3, S.FIELD_R, 49, 50, 1)
        e.forward()
        snaps = e.snapshots(2, 0), e.snapshots(3, 0)
    for (sid, field, first, every), got in zip(((2, S.FIELD_P, 9, 40), (3, S.FIELD_R, 49, 50)), snaps):
        for j, snap in enumerate(got):
            k = first + j * every
            with S.Engine(S.VISCOAC_2D, vp.shape[0], vp.shape[1], dx, dx, dt, npx, order=10, f0=f0, flags=flags) as e:
                e.set_model(vp, rho, q)
                e.set_shots([S.ShotSpec(20, 12, r, np.full_like(r, 10), w[:k + 1])])
                e.forward()
                full = e.wavefield(0, field)
            assert bits_equal(snap, full[npx:-npx, npx:-npx]), (field, k)


@pytest.mark.parametrize("mode,hilly", [("abc", False), ("fsbc", False), ("abc", True), ("fsbc", True)])
def test_iso_forward_program_against_restatement(tmp_path, mode, hilly):
    """iso_forward on a yang_version card of three aperture shots, flat or with topography: the
    merged SU files hold the FP32 restatement's vx / vz traces bit for bit, with YPUB:1555-1596's
    headers (no cdp); the last snapshot of the last shot equals the restatement's wavefield after
    that step."""
    from test_fileio import ISOCARD
    nx, nz = 120, 80
    rng = np.random.default_rng(12)
    z = np.arange(nz)
    vp = np.tile(np.where(z < 40, 2000.0, 2700.0), (nx, 1)).astype(np.float32)
    vp += rng.uniform(-50, 50, vp.shape).astype(np.float32)
    vs = (vp / 1.8).astype(np.float32)
    rho = (2000.0 + 300.0 * rng.random((nx, nz))).astype(np.float32)
    for name, a in (("vp", vp), ("vs", vs), ("rho", rho)):
        a.tofile(tmp_path / f"{name}.bin")
    x = np.arange(nx)
    topo = (10.0 * np.round(2 + 1.5 * np.cos(x / 10.0))).astype(np.float32) if hilly else np.zeros(nx, np.float32)
    topo.tofile(tmp_path / "topo.bin")
    (tmp_path / "snap").mkdir()
    card = ISOCARD.format(d=str(tmp_path), mode=mode, ztop="90.0" if mode == "abc" else "0000.0", rgau=12)
    (tmp_path / "iso.par").write_text(card)
    p = S.read_isopar(str(tmp_path / "iso.par"))
    run([os.path.join(BIN, "iso_forward"), str(tmp_path / "iso.par"), "--snapshots", str(tmp_path / "snap")],
        cwd=tmp_path)
    nint = lambda v: int(np.floor(abs(v) + 0.5)) * (1 if v >= 0 else -1)
    np_ = nint(p.pml_xn / p.dx) + 1
    top = nint(p.pml_zn / p.dz) + 1
    isx0, isz0, irz0 = nint(p.sx0 / p.dx) + 1, nint(p.sz0 / p.dz) + 1, nint(p.rz0 / p.dz) + 1
    idecay, idtsnap = nint(p.decay / p.dt), nint(p.dtsnap / p.dt)
    fs = mode == "fsbc"
    kw = dict(nrz0=irz0, idecay=idecay, rgau=p.rgau, fsbc=fs, npz_top=top, topo=topo)
    itopo_at = lambda col: nint(float(np.float32(topo[min(max(col, 1), nx) - 1]) / np.float32(p.dz))) + top
    refs = []
    for i in range(1, p.nshot + 1):
        isx = isx0 + nint((i - 1) * p.dsx / p.dx)
        ixmine, ixmaxe = isx + nint(p.offset_min / p.dx), isx + nint(p.offset_max / p.dx)
        args = (vp, vs, rho, p.dx, p.dz, p.dt, p.f0)
        isze = isz0 + itopo_at(isx + 1)  # isz + itopoe(isxe): window column isxe reads model column isx + 1
        r1, r2, _ = ol.iso_forward(*args, p.nt, np_, np_, isx - ixmine + np_ + 1, isze, ixmine=ixmine,
                                   ixmaxe=ixmaxe, **kw)
        refs.append((isx, ixmine, ixmaxe - ixmine + 1, r1, r2, isze))
    for stem, which in (("vx", 3), ("vz", 4)):
        assert not (tmp_path / f"{stem}_tmp1.su").exists()
        raw = open(tmp_path / f"shot_{stem}.su", "rb").read()
        off = 0
        for i, ref in enumerate(refs, start=1):
            isx, ixmine, nxe = ref[:3]
            for t in range(nxe):
                rec = raw[off:off + 240 + 4 * p.nt]
                off += 240 + 4 * p.nt
                want = bytearray(expected_header(i, isx, ixmine, p.dx, p.dt, p.nt, t + 1))
                want[20:24] = b"\0\0\0\0"
                assert rec[:240] == bytes(want)
                assert bits_equal(np.frombuffer(rec[240:], np.float32), ref[which][t]), (stem, i, t)
        assert off == len(raw)
    # snapshots of the last shot: vx after step it = k * idtsnap (YPRI:212-224)
    isx, ixmine, nxe = refs[-1][:3]
    last = idtsnap * ((p.nt + idecay) // idtsnap)
    snap = read(tmp_path / "snap" / f"vx_{last}", (nxe, nz))
    _, _, fin = ol.iso_forward(vp, vs, rho, p.dx, p.dz, p.dt, p.f0, last - idecay, np_, np_, isx - ixmine + np_ + 1,
                               refs[-1][5], ixmine=ixmine, ixmaxe=ixmine + nxe - 1, want_final=True, **kw)
    assert bits_equal(snap, fin[np_:np_ + nxe, top:top + nz])


def test_vti_forward_program_against_restatement(tmp_path):
    """vti_forward on a card of three shots whose apertures reach past the model's left edge: the
    merged SU file holds the FP32 restatement's records bit for bit, computed with epsilon and
    delta zero as read_data leaves them (VS:147-148), with VS:184-214's headers (fldr, trid, sx,
    gx, ns, dt; no offset, no cdp)."""
    from test_fileio import VTICARD, expected_header
    nx, nz, nt = 200, 80, 300
    rng = np.random.default_rng(21)
    z = np.arange(nz)
    vz = np.tile(np.where(z < 40, 1900.0, 2600.0), (nx, 1)).astype(np.float32)
    vz += rng.uniform(-40, 40, vz.shape).astype(np.float32)
    vz.tofile(tmp_path / "vz.bin")
    (0.2 * rng.random((nx, nz))).astype(np.float32).tofile(tmp_path / "eps.bin")
    (0.1 * rng.random((nx, nz))).astype(np.float32).tofile(tmp_path / "delta.bin")
    (tmp_path / "vti.par").write_text(VTICARD.format(d=str(tmp_path), nx=nx, nz=nz, nt=nt))
    run([os.path.join(BIN, "vti_forward"), str(tmp_path / "vti.par")], cwd=tmp_path)
    assert not (tmp_path / "vti_tmp1.su").exists()
    raw = open(tmp_path / "vti_all.su", "rb").read()
    zero = np.zeros_like(vz)
    rec_bytes = 240 + 4 * nt
    off = 0
    for i in range(1, 4):
        nsx = 21 + (i - 1) * 10  # nint(100/5) + 1 + nint((i-1) 50/5)
        xmin, xmax = nsx - 60, nsx + 59
        ref = ol.vti_forward(vz, zero, zero, 5.0, 5.0, 0.0005, 30.0, nt, (20, 20, 0, 20), nsx, 1, 1, xmin, xmax)
        for tr in range(1, xmax - xmin + 2):
            rec = raw[off:off + rec_bytes]
            off += rec_bytes
            want = bytearray(expected_header(i, nsx, xmin, 5.0, 0.0005, nt, tr))
            want[20:24] = b"\0\0\0\0"
            want[36:40] = b"\0\0\0\0"
            assert rec[:240] == bytes(want), (i, tr)
            assert np.array_equal(np.frombuffer(rec[240:], np.uint32), ref[tr - 1].view(np.uint32)), (i, tr)
    assert off == len(raw)
