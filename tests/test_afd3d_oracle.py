"""CPU checks of the 3-D restatement (oracle/afd3d_oracle.cpp), the checker of the 3-D CUDA path.

No 3-D reference exists, so the restatement is tied to the reference through the parts it
shares with the 2-D scheme and checked for the symmetries the discrete scheme has:
  * its sponge equals the reference's 2-D sponge (AFD:164-194) on every x-z plane outside the y
    pads (the x factor wins over the z factor, as in AFD's corners);
  * FP32 and FP64 instances agree to FP32 round-off;
  * with no sponge, dy = dz and a model symmetric under swapping y and z, the wavefield of a
    source on the diagonal is symmetric (the scheme treats the two axes identically);
  * the records are linear in the wavelet.
"""
import numpy as np

import oracle_lib as ol
from conftest import rel_l2
from seismic_code_github_b200 import seisfd as S


def test_sponge_reduces_to_the_2d_reference_rule():
    nx, ny, nz, pml = 40, 30, 36, 8
    a3 = ol.afd3d_sponge(nx, ny, nz, pml)
    a2 = ol.afd_sponge(nx, nz, pml)
    for y in range(pml, ny - pml):
        assert np.array_equal(a3[:, y, :], a2)
    # inside the y pads the y taper applies except where the x pad wins
    y = 2
    q = pml - y - 1
    ty = np.float32(-0.38 * q * q / (1.0 * pml * pml) + 1)
    assert np.all(a3[pml:nx - pml, y, :] == ty)
    assert np.array_equal(a3[:pml, y, :], a2[:pml, :])


def case(seed=0, n=(30, 28, 32)):
    rng = np.random.default_rng(seed)
    vp = (2200.0 + 400.0 * rng.random(n)).astype(np.float32)
    rx = rng.integers(0, n[0], 20).astype(np.int32)
    ry = rng.integers(0, n[1], 20).astype(np.int32)
    rz = rng.integers(0, n[2], 20).astype(np.int32)
    return vp, rx, ry, rz


def test_fp32_matches_fp64():
    vp, rx, ry, rz = case()
    w = S.wavelet(S.WAVELET_RIC, 80, 1e-3, 25.0, 20)
    r64, f64 = ol.afd3d_forward(vp, None, w, (15, 14, 16), rx, ry, rz, 6, 10.0, 10.0, 10.0, 1e-3, want_final=True)
    r32, f32 = ol.afd3d_forward(vp, None, w, (15, 14, 16), rx, ry, rz, 6, 10.0, 10.0, 10.0, 1e-3, fp64=False,
                                want_final=True)
    assert np.abs(r64).max() > 0
    assert rel_l2(r32, r64) < 1e-5 and rel_l2(f32, f64) < 1e-5


def test_y_z_swap_symmetry_without_sponge():
    n = 30
    rng = np.random.default_rng(3)
    v = (2000.0 + 500.0 * rng.random((n, n, n))).astype(np.float32)
    v = 0.5 * (v + v.transpose(0, 2, 1))  # symmetric in (y, z)
    w = S.wavelet(S.WAVELET_RIC, 60, 1e-3, 30.0, 15)
    r = np.array([3], np.int32)
    _, fin = ol.afd3d_forward(v, None, w, (15, 12, 12), r, r, r, 0, 10.0, 10.0, 10.0, 1e-3, want_final=True)
    assert np.abs(fin).max() > 0
    assert rel_l2(fin.transpose(0, 2, 1), fin) < 1e-12


def test_records_are_linear_in_the_wavelet():
    vp, rx, ry, rz = case(seed=1)
    w1 = S.wavelet(S.WAVELET_RIC, 60, 1e-3, 25.0, 20)
    w2 = S.wavelet(S.WAVELET_RIC, 60, 1e-3, 15.0, 30)
    f = lambda w: ol.afd3d_forward(vp, None, w, (14, 13, 15), rx, ry, rz, 5, 10.0, 10.0, 10.0, 1e-3)[0]
    assert rel_l2(f(w1) + 2.0 * f(w2), f((w1 + 2.0 * w2).astype(np.float32))) < 1e-6
