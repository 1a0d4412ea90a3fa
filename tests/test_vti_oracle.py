"""CPU checks of the restated VTI pseudo-acoustic modeller (oracle/vti_oracle.cpp, after
de-multiple/convolution_srm/vti_qa_2d_c3_demo1).  Its main program does not compile and the folder
ships no output, so the restatement is pinned by mathematics and physics instead: the
Sherman-Morrison coefficients against the exact central-difference weights, FP32 against FP64,
mirror symmetry about the source, and absorption by the PML.  The library's host-side coefficient
routine (sfd_vti_coefficients, no GPU needed) must equal the restatement's bit for bit."""
from fractions import Fraction

import numpy as np
import pytest

import oracle_lib as ol
from conftest import rel_l2


def exact_weights(k, first):
    """Central-difference weights c_m, m = 1..k, solving sum_m c_m 2 m^p / p! = delta(p, p0)
    for p = 2j (second derivative) or 2j-1 (first derivative), in exact rationals."""
    from math import factorial
    A = [[Fraction(2 * m ** (2 * j - 1 if first else 2 * j), factorial(2 * j - 1 if first else 2 * j))
          for m in range(1, k + 1)] for j in range(1, k + 1)]
    b = [Fraction(1 if j == 0 else 0) for j in range(k)]
    n = k
    M = [row[:] + [b[r]] for r, row in enumerate(A)]
    for c in range(n):
        p = next(r for r in range(c, n) if M[r][c] != 0)
        M[c], M[p] = M[p], M[c]
        for r in range(n):
            if r != c and M[r][c] != 0:
                f = M[r][c] / M[c][c]
                M[r] = [x - f * y for x, y in zip(M[r], M[c])]
    return [float(M[r][n] / M[r][r]) for r in range(n)]


@pytest.mark.parametrize("order,first", [(10, 0), (9, 1), (10, 1), (8, 0), (6, 0)])
def test_coefficients_against_exact_weights(order, first):
    k = (order + 1) // 2 if first else order // 2
    ex = np.array(exact_weights(k, bool(first)))
    c64 = ol.vti_coefficients(order, first, fp64=True)
    c32 = ol.vti_coefficients(order, first)
    assert np.allclose(c64, ex, rtol=1e-9, atol=0)
    assert np.allclose(c32, ex, rtol=3e-6, atol=0)


def test_library_coefficients_equal_restatement():
    from seismic_code_github_b200 import seisfd as S
    for order, first in ((10, 0), (9, 1), (10, 1)):
        a = S.vti_coefficients(order, bool(first))
        b = ol.vti_coefficients(order, first)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (order, first)


def layered(nxv=120, nzv=80, seed=3):
    rng = np.random.default_rng(seed)
    z = np.arange(nzv)
    vz = np.tile(np.where(z < nzv // 2, 2000.0, 2600.0), (nxv, 1)).astype(np.float32)
    eps = np.tile(np.where(z < nzv // 2, 0.15, 0.25), (nxv, 1)).astype(np.float32)
    de = np.tile(np.where(z < nzv // 2, 0.05, 0.10), (nxv, 1)).astype(np.float32)
    vz += (30.0 * rng.standard_normal(vz.shape)).astype(np.float32)
    return vz, eps, de


def test_fp32_restatement_within_1e5_of_fp64():
    vz, eps, de = layered()
    kw = dict(dx=5.0, dz=5.0, dt=5e-4, f0=30.0, nt=700, bounds=(20, 20, 0, 20), nsx=60, nsz0=1, nrz0=1, xmin=0,
              xmax=119)
    r = ol.vti_forward(vz, eps, de, **kw)
    r64 = ol.vti_forward(vz, eps, de, fp64=True, **kw)
    err = rel_l2(r, r64)
    print(f"VTI FP32 vs FP64 relL2 {err:.2e}")
    assert np.abs(r64).max() > 0 and err <= 1e-5


def test_mirror_symmetry_about_the_source():
    """A laterally homogeneous model and the source on the grid's centre column: the traces k
    columns either side agree bit for bit.  The grid is nx = range + nxl + nxr - 2 wide (VM:248)
    with the model in columns nxl+1 .. nxl+range, so the right PML covers the last two model
    columns and the centre (nx + 1) / 2 is grid column nxl + 60 for range 121: source nsx = 60
    (xmin 0), record trace 60 (index 59).  Epsilon and delta exist only inside the window
    (VS:297-302; the pads keep zero), which is not symmetric about that centre, so the anisotropic
    case is only near-symmetric and the exact check runs with epsilon = delta = 0."""
    nxv, nzv = 121, 70
    z = np.arange(nzv)
    vz = np.tile(np.where(z < 35, 2000.0, 2500.0), (nxv, 1)).astype(np.float32)
    z0 = np.zeros_like(vz)
    r = ol.vti_forward(vz, z0, z0, 5.0, 5.0, 5e-4, 30.0, 500, (20, 20, 10, 20), 60, 5, 3, 0, 120)
    mid = 59
    for k in (5, 20, 45):
        assert np.array_equal(r[mid - k], r[mid + k]), k
    eps = np.tile(np.where(z < 35, 0.1, 0.2), (nxv, 1)).astype(np.float32)
    de = np.tile(np.where(z < 35, 0.05, 0.08), (nxv, 1)).astype(np.float32)
    ra = ol.vti_forward(vz, eps, de, 5.0, 5.0, 5e-4, 30.0, 500, (20, 20, 10, 20), 60, 5, 3, 0, 120)
    assert rel_l2(ra[mid - 5], ra[mid + 5]) < 0.05
    assert rel_l2(ra[mid], r[mid]) > 1e-3  # the anisotropy changes the record


def test_pml_absorbs():
    """Homogeneous isotropic model: after the direct wave has left the grid the record energy is a
    small fraction of its peak (the PML of VS:565-663 absorbs on the left, right and bottom)."""
    nxv, nzv = 100, 60
    vz = np.full((nxv, nzv), 2500.0, np.float32)
    z0 = np.zeros_like(vz)
    r = ol.vti_forward(vz, z0, z0, 5.0, 5.0, 5e-4, 30.0, 2400, (25, 25, 0, 25), 50, 1, 1, 0, 99)
    e = (r.astype(np.float64) ** 2).sum(axis=0)
    peak = e.max()
    assert e[-300:].max() < 1e-3 * peak


def test_invalid_configurations_rejected():
    vz, eps, de = layered(40, 30)
    with pytest.raises(ValueError):  # nx_bound_r < 2 leaves no room for the right pad (VM:248)
        ol.vti_forward(vz, eps, de, 5.0, 5.0, 5e-4, 30.0, 10, (10, 1, 0, 10), 20, 1, 1, 0, 39)
    with pytest.raises(ValueError):  # the stencils are written for order 10 only
        ol.vti_forward(vz, eps, de, 5.0, 5.0, 5e-4, 30.0, 10, (10, 10, 0, 10), 20, 1, 1, 0, 39, orders=(8, 9, 10))
