"""GPU viscoacoustic path (SFD_VISCOAC_2D, the vs = 0 reduction of forward/Q_forward) through
the C ABI, against the restatement of the Fortran code (oracle/q_oracle.cpp).  With SFD_EXACT the
two kernels per step keep the reference's operation order, so records must be bit-identical to
the FP32 restatement.  The default mode (x-marching step kernel and sponge-band kernel, merged stress and memory
variable away from the sponge bands, FMA contraction) must stay within relative L2 <= 1e-5 of
the FP64 restatement."""
import numpy as np
import pytest

import oracle_lib as ol
from conftest import bits_equal, rel_l2
from seismic_code_github_b200 import seisfd as S

pytestmark = pytest.mark.gpu


def qmodel(nx=70, nz=56, seed=0, qlo=20.0, qhi=200.0, lens=True):
    rng = np.random.default_rng(seed)
    z = np.arange(nz)
    x = np.arange(nx)
    vp = np.tile(np.where(z < nz // 2, 2000.0, 3000.0), (nx, 1)).astype(np.float32)
    vp += (30.0 * rng.standard_normal((nx, nz))).astype(np.float32)
    rho = (2000.0 + 200.0 * rng.random((nx, nz))).astype(np.float32)
    q = qlo + (qhi - qlo) * rng.random((nx, nz))
    if lens:
        q = np.where((x[:, None] - nx / 2) ** 2 + (z[None, :] - nz / 2) ** 2 < (nz / 5) ** 2, qlo, q)
    return vp, rho, q.astype(np.float32)


TOL_FAST = 1e-5


def run_gpu(vp, rho, q, npx, f0, dt, dx, shots_spec, flags=S.EXACT):
    """shots_spec: list of (isxe, isze, nt_total, nrz0); interior model arrays (nx, nz)."""
    vpp, rhop, qp = (S.pad_model(a, npx, npx, npx, npx) for a in (vp, rho, q))
    nx, nz = vpp.shape
    e = S.Engine(S.VISCOAC_2D, nx, nz, dx, dx, dt, npx, order=10, f0=f0, flags=flags)
    e.set_model(vpp, rhop, qp)
    shots = []
    for isxe, isze, ntot, nrz0 in shots_spec:
        rx = np.arange(npx, nx - npx, dtype=np.int32)
        rz = np.full_like(rx, npx + nrz0)
        w = S.wavelet(S.WAVELET_Q, ntot, dt, f0)
        shots.append(S.ShotSpec(isxe - 1, isze - 1, rx, rz, w))
    e.set_shots(shots)
    recs = e.split_records(e.forward())
    t = e.timing()
    e.close()
    return recs, t


@pytest.mark.parametrize("seed", [0, 1])
def test_single_shot_bitexact_against_restatement(seed):
    vp, rho, q = qmodel(seed=seed)
    npx, f0, dt, dx, nt = 11, 20.0, 5e-4, 10.0, 160
    decay = ol.q_decay(f0, dt)
    isxe, isze, nrz0 = npx + 25, npx + 4, 1
    recs, t = run_gpu(vp, rho, q, npx, f0, dt, dx, [(isxe, isze, nt + decay, nrz0)])
    r1, r2, _ = ol.q_forward(vp, vp * 0, rho, q, q, dx, dx, dt, f0, nt, npx, npx, isxe, isze, nrz0=nrz0)
    r64, _, _ = ol.q_forward(vp, vp * 0, rho, q, q, dx, dx, dt, f0, nt, npx, npx, isxe, isze, nrz0=nrz0, fp64=True)
    got = recs[0][:, decay:]
    print(f"seed {seed}: GPU vs FP32 restatement relL2 {rel_l2(got, r1):.2e}; vs FP64 {rel_l2(got, r64):.2e}; "
          f"{t['launches']} launches {t['loop_ms']:.2f} ms")
    assert np.abs(got).max() > 0
    assert bits_equal(got, r1)
    assert bits_equal(r1, r2)  # strzz == strxx in the acoustic reduction


def test_batched_uneven_shots_and_q_override():
    vp, rho, q = qmodel(seed=3, nx=80, nz=50)
    npx, f0, dt, dx = 10, 25.0, 5e-4, 10.0
    decay = ol.q_decay(f0, dt)
    spec = [(npx + 12, npx + 3, 150, 1), (npx + 60, npx + 8, 90, 2), (npx + 40, npx + 20, 120, 1)]
    recs, _ = run_gpu(vp, rho, q, npx, f0, dt, dx, [(a, b, n + decay, c) for a, b, n, c in spec])
    for (isxe, isze, nt, nrz0), got in zip(spec, recs):
        ref, _, _ = ol.q_forward(vp, vp * 0, rho, q, q, dx, dx, dt, f0, nt, npx, npx, isxe, isze, nrz0=nrz0)
        assert bits_equal(got[:, decay:], ref), (isxe, isze, nt)


def test_attenuation_on_gpu():
    vp, rho, _ = qmodel(seed=4, lens=False)
    npx, f0, dt, dx, nt = 11, 20.0, 5e-4, 10.0, 300
    decay = ol.q_decay(f0, dt)
    energies = []
    for qv in (1e5, 60.0, 15.0):
        q = np.full_like(vp, qv)
        recs, _ = run_gpu(vp, rho, q, npx, f0, dt, dx, [(npx + 30, npx + 4, nt + decay, 1)])
        energies.append(float(np.sum(recs[0][:, decay:].astype(np.float64) ** 2)))
    assert energies[0] > energies[1] > energies[2]


def test_wavefield_readback():
    vp, rho, q = qmodel(seed=5, nx=40, nz=40)
    npx, f0, dt, dx = 8, 20.0, 5e-4, 10.0
    vpp, rhop, qp = (S.pad_model(a, npx, npx, npx, npx) for a in (vp, rho, q))
    with S.Engine(S.VISCOAC_2D, vpp.shape[0], vpp.shape[1], dx, dx, dt, npx, order=10, f0=f0) as e:
        e.set_model(vpp, rhop, qp)
        rx = np.array([20], np.int32)
        e.set_shots([S.ShotSpec(25, 12, rx, rx, S.wavelet(S.WAVELET_Q, 150, dt, f0))])
        rec = e.forward()
        p = e.wavefield(0, S.FIELD_P)
        r = e.wavefield(0, S.FIELD_R)
        vx = e.wavefield(0, S.FIELD_VX)
    assert np.isfinite(p).all() and np.abs(p).max() > 0 and np.abs(r).max() > 0 and np.abs(vx).max() > 0
    assert p[20, 20] == rec[-1]


@pytest.mark.parametrize("seed", [0, 1])
def test_fused_single_shot_against_fp64(seed):
    vp, rho, q = qmodel(seed=seed)
    npx, f0, dt, dx, nt = 11, 20.0, 5e-4, 10.0, 160
    decay = ol.q_decay(f0, dt)
    isxe, isze, nrz0 = npx + 25, npx + 4, 1
    recs, t = run_gpu(vp, rho, q, npx, f0, dt, dx, [(isxe, isze, nt + decay, nrz0)], flags=0)
    r64, _, _ = ol.q_forward(vp, vp * 0, rho, q, q, dx, dx, dt, f0, nt, npx, npx, isxe, isze, nrz0=nrz0, fp64=True)
    got = recs[0][:, decay:]
    err = rel_l2(got, r64)
    print(f"seed {seed}: fused vs FP64 restatement relL2 {err:.2e}, kernel {t['kernel_variant']}, "
          f"{t['launches']} launches")
    assert t["kernel_variant"] == 41 and np.abs(got).max() > 0
    assert err <= TOL_FAST


def test_fused_batched_uneven_shots_apertures_against_fp64():
    """Shots of different record lengths and sources near the sponge bands and a grid corner, on
    a grid whose width is not a multiple of the strip or segment sizes."""
    vp, rho, q = qmodel(seed=3, nx=300, nz=150)
    npx, f0, dt, dx = 20, 25.0, 5e-4, 10.0
    decay = ol.q_decay(f0, dt)
    # (isxe, isze, nt, nrz0): each shot's receiver row lies a few cells above its source, so that the
    # records hold the wave itself within the record length
    spec = [(npx + 12, npx + 3, 150, 1), (npx + 160, npx + 60, 90, 55), (npx + 290, npx + 140, 120, 134),
            (3, 4, 100, 1)]
    recs, _ = run_gpu(vp, rho, q, npx, f0, dt, dx, [(a, b, n + decay, c) for a, b, n, c in spec], flags=0)
    for (isxe, isze, nt, nrz0), got in zip(spec, recs):
        r64, _, _ = ol.q_forward(vp, vp * 0, rho, q, q, dx, dx, dt, f0, nt, npx, npx, isxe, isze, nrz0=nrz0,
                                 fp64=True)
        err = rel_l2(got[:, decay:], r64)
        print(f"shot at ({isxe}, {isze}): relL2 {err:.2e}")
        assert err <= TOL_FAST, (isxe, isze, err)


@pytest.mark.parametrize("seg", ["16", "64", "512"])
def test_fused_segment_length_keeps_bits(monkeypatch, seg):
    """The step kernel's segment length (the engine halves it for steps with few active shots; a
    first chunk per segment recomputes the velocities it needs) does not change any bit of the
    records of the uneven batch above."""
    vp, rho, q = qmodel(seed=3, nx=300, nz=150)
    npx, f0, dt, dx = 20, 25.0, 5e-4, 10.0
    spec = [(npx + 12, npx + 3, 150, 1), (npx + 160, npx + 60, 90, 55), (npx + 290, npx + 140, 120, 134),
            (3, 4, 100, 1)]
    monkeypatch.delenv("SFD_QFAST_SEG", raising=False)
    ref, _ = run_gpu(vp, rho, q, npx, f0, dt, dx, spec, flags=0)
    monkeypatch.setenv("SFD_QFAST_SEG", seg)
    got, _ = run_gpu(vp, rho, q, npx, f0, dt, dx, spec, flags=0)
    for a, b in zip(ref, got):
        assert np.abs(a).max() > 0 and bits_equal(a, b)


def test_fused_final_wavefields_against_fp64():
    """The final stress field (sigma = strxx) after the loop, everywhere on the padded grid
    (sponge bands, corners and interior), against the FP64 restatement."""
    vp, rho, q = qmodel(seed=6, nx=90, nz=76)
    npx, f0, dt, dx, nt = 12, 20.0, 5e-4, 10.0, 200
    decay = ol.q_decay(f0, dt)
    isxe, isze = npx + 30, npx + 20
    vpp, rhop, qp = (S.pad_model(a, npx, npx, npx, npx) for a in (vp, rho, q))
    with S.Engine(S.VISCOAC_2D, vpp.shape[0], vpp.shape[1], dx, dx, dt, npx, order=10, f0=f0) as e:
        e.set_model(vpp, rhop, qp)
        rx = np.arange(npx, vpp.shape[0] - npx, dtype=np.int32)
        e.set_shots([S.ShotSpec(isxe - 1, isze - 1, rx, np.full_like(rx, npx + 1),
                                S.wavelet(S.WAVELET_Q, nt + decay, dt, f0))])
        e.forward()
        p = e.wavefield(0, S.FIELD_P)
    _, _, fin = ol.q_forward(vp, vp * 0, rho, q, q, dx, dx, dt, f0, nt, npx, npx, isxe, isze, fp64=True,
                             want_final=True)
    assert np.abs(p).max() > 0
    assert rel_l2(p, fin) <= TOL_FAST
