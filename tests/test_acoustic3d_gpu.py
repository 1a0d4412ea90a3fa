"""GPU parity of the 3-D acoustic path (SFD_ACOUSTIC_3D) through the C ABI.

The reference has no 3-D modeller, so the bar is the FP64 restatement of the same scheme
(oracle/afd3d_oracle.cpp): relative L2 <= 1e-5 on the receiver traces and on the final
pressure (max-abs printed).  The cases cover partial tiles (grid sizes that are not multiples
of the 32 x 32 column), columns wholly inside the sponge-free interior, variable density, both
built orders, sources near the rim, several shots of different lengths in one batch (equal bit
for bit to the per-shot path) and the wavefield read-back.
"""
import numpy as np
import pytest

import oracle_lib as ol
from conftest import bits_equal, rel_l2
from seismic_code_github_b200 import seisfd as S

pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative L2, FP32 CUDA vs FP64 restatement


def model3d(nx, ny, nz, seed, varden=False):
    rng = np.random.default_rng(seed)
    z = np.arange(nz)
    vp = np.empty((nx, ny, nz), np.float32)
    vp[:] = (1800.0 + 1200.0 * z / nz)[None, None, :]
    vp += (150.0 * rng.standard_normal((nx, ny, nz))).astype(np.float32) * 0.3
    den = (1900.0 + 500.0 * rng.random((nx, ny, nz))).astype(np.float32) if varden else None
    return vp.astype(np.float32), den


def receivers(nx, ny, nz, seed, n=60):
    rng = np.random.default_rng(seed + 100)
    rx = rng.integers(0, nx, n).astype(np.int32)
    ry = rng.integers(0, ny, n).astype(np.int32)
    rz = rng.integers(0, nz, n).astype(np.int32)
    return rx, ry, rz


def run_gpu(vp, den, shots, pml, d, dt, order=8, per_shot=False):
    nx, ny, nz = vp.shape
    with S.Engine(S.ACOUSTIC_3D, nx, nz, d, d, dt, pml, order=order, ny=ny, dy=d) as e:
        e.set_model(vp, den)
        e.set_shots(shots)
        rec = e.forward_per_shot() if per_shot else e.forward()
        fin = [e.wavefield(i, S.FIELD_P) for i in range(len(shots))]
        t = e.timing()
    return rec, fin, t


def check_case(nx, ny, nz, pml, nt, src, seed, order=8, varden=False, d=10.0, dt=1e-3):
    vp, den = model3d(nx, ny, nz, seed, varden)
    rx, ry, rz = receivers(nx, ny, nz, seed)
    w = S.wavelet(S.WAVELET_RIC, nt, dt, 25.0, 30)
    shot = S.ShotSpec(src[0], src[2], rx, rz, w, sy=src[1], rec_y=ry)
    rec, fin, _ = run_gpu(vp, den, [shot], pml, d, dt, order)
    ref, pref = ol.afd3d_forward(vp, den, w, src, rx, ry, rz, pml, d, d, d, dt, radius=order // 2, want_final=True)
    rec = rec.reshape(len(rx), nt)
    e_rec, e_fin = rel_l2(rec, ref), rel_l2(fin[0], pref)
    print(f"3-D {nx}x{ny}x{nz} pml={pml} order={order} varden={varden}: rec relL2={e_rec:.2e} "
          f"maxabs={np.abs(rec - ref).max():.2e} (max {np.abs(ref).max():.2e}); final P relL2={e_fin:.2e}")
    assert np.abs(ref).max() > 0
    assert e_rec <= TOL and e_fin <= TOL


def test_small_partial_tiles():
    check_case(44, 40, 52, 8, 120, (20, 18, 12), seed=0)


def test_interior_columns_and_sponge():
    # y and z of 100 / 110 give 4 x 4 columns of 32 with interior ones (no sponge, no rim)
    check_case(72, 100, 110, 10, 90, (36, 50, 40), seed=1)


def test_variable_density():
    check_case(40, 45, 38, 6, 100, (19, 22, 17), seed=2, varden=True)


def test_order4():
    check_case(38, 36, 41, 6, 110, (15, 20, 18), seed=3, order=4)


def test_source_next_to_rim():
    check_case(30, 34, 36, 5, 80, (4, 4, 4), seed=4)


def test_batched_equals_per_shot_and_each_matches_oracle():
    nx, ny, nz, pml, d, dt = 40, 44, 48, 8, 10.0, 1e-3
    vp, den = model3d(nx, ny, nz, 5)
    rx, ry, rz = receivers(nx, ny, nz, 5, n=40)
    spec = [((12, 20, 14), 70), ((25, 10, 30), 110), ((30, 33, 8), 50)]
    shots = [S.ShotSpec(s[0], s[2], rx, rz, S.wavelet(S.WAVELET_RIC, nt, dt, 20.0, 25), sy=s[1], rec_y=ry)
             for s, nt in spec]
    rec_b, fin_b, tb = run_gpu(vp, den, shots, pml, d, dt)
    rec_p, fin_p, tp = run_gpu(vp, den, shots, pml, d, dt, per_shot=True)
    assert tb["graph"] == 1 and tp["graph"] == 0
    assert bits_equal(rec_b, rec_p)
    for a, b in zip(fin_b, fin_p):
        assert bits_equal(a, b)
    off = 0
    for (src, nt), sh in zip(spec, shots):
        n = len(rx) * nt
        got = rec_b[off:off + n].reshape(len(rx), nt)
        off += n
        ref, _ = ol.afd3d_forward(vp, None, sh.wavelet, src, rx, ry, rz, pml, d, d, d, dt)
        assert rel_l2(got, ref) <= TOL


def test_velocity_readback_is_damped_field():
    nx, ny, nz, pml, d, dt, nt = 36, 38, 40, 7, 10.0, 1e-3, 60
    vp, _ = model3d(nx, ny, nz, 6)
    w = S.wavelet(S.WAVELET_RIC, nt, dt, 25.0, 20)
    r = np.array([18], np.int32)
    with S.Engine(S.ACOUSTIC_3D, nx, nz, d, d, dt, pml, order=8, ny=ny, dy=d) as e:
        e.set_model(vp)
        e.set_shots([S.ShotSpec(18, 20, r, r, w, sy=19, rec_y=r)])
        rec = e.forward()
        p = e.wavefield(0, S.FIELD_P)
        vx = e.wavefield(0, S.FIELD_VX)
        vy = e.wavefield(0, S.FIELD_VY)
        vz = e.wavefield(0, S.FIELD_VZ)
    assert p[18, 18, 18] == rec[-1]
    a = ol.afd3d_sponge(nx, ny, nz, pml)
    # velocities come back damped: zero on the frozen rim, finite and non-zero inside
    for v in (vx, vy, vz):
        assert np.isfinite(v).all() and np.abs(v).max() > 0
        assert np.all(v[:4] == 0) and np.all(v[:, :, -4:] == 0)
    assert a.min() > 0
