"""CPU checks of the restated isotropic elastic standard-staggered-grid modeller
(oracle/iso_oracle.cpp: forward/yang_version_2016_2_2, abc mode, flat surface).  The Fortran
cannot be built here, so the restatement is checked by (1) an independent float32 Python
restatement of its model preparation -- substagger (YPUB:323-547) and the in-place Gaussian
smoothing of the top sponge rows in the one-thread order (YPUB:549-634) -- bit for bit, and
(2) physics: FP32 against FP64, P arrival time, mirror symmetry about the source."""
import ctypes
import ctypes.util

import numpy as np
import pytest

import oracle_lib as ol
from conftest import rel_l2

F = np.float32
_libm = ctypes.CDLL(ctypes.util.find_library("m"))
_libm.expf.argtypes = [ctypes.c_float]
_libm.expf.restype = ctypes.c_float


def expf(x):
    """The C library's single-precision exp (the one the restatement calls)."""
    return F(_libm.expf(float(x)))


def py_prepare(vp, vs, rho, npx, npz, rgau):
    """Float32 Python restatement of YPUB:188-634 for a whole-model window (tiny sizes only)."""
    pad = lambda a: np.pad(a, ((npx, npx), (npz, npz)), mode="edge")
    vpe, vse, rhoe = pad(vp).T.copy(), pad(vs).T.copy(), pad(rho).T.copy()  # (NZ, NX), Fortran (k, i)
    NZ, NX = vpe.shape
    mu = np.zeros_like(vpe); lamb = np.zeros_like(vpe)
    for i in range(NX):
        for k in range(NZ):
            mu[k, i] = rhoe[k, i] * vse[k, i] * vse[k, i]
            lamb[k, i] = rhoe[k, i] * vpe[k, i] * vpe[k, i] - F(2.0) * mu[k, i]
    b1 = np.zeros_like(vpe)
    for i in range(NX - 1):
        for k in range(NZ - 1):
            b1[k, i] = F(0.25) * (rhoe[k, i] + rhoe[k + 1, i] + rhoe[k + 1, i + 1] + rhoe[k, i + 1])
    b1[NZ - 1, :] = b1[NZ - 2, :]
    b1[:, NX - 1] = b1[:, NX - 2]
    b1 = (F(1.0) / b1).astype(F)
    b1e = np.zeros_like(vpe)
    for k in range(1, NZ):
        b1e[k] = F(0.5) * (b1[k] + b1[k - 1])
    b1e[0] = b1[0]
    b2 = (F(1.0) / rhoe).astype(F)
    b2e = np.zeros_like(vpe)
    for i in range(NX - 1):
        b2e[:, i] = F(0.5) * (b2[:, i] + b2[:, i + 1])
    b2e[:, NX - 1] = b2[:, NX - 1]
    musg = np.zeros_like(vpe)
    for k in range(NZ - 1):
        musg[k] = F(0.5) * (mu[k + 1] + mu[k])
    musg[NZ - 1] = mu[NZ - 1]
    musge = np.zeros_like(vpe)
    for i in range(NX - 1):
        for k in range(1, NZ):
            q = (musg[k, i], musg[k, i + 1], musg[k - 1, i + 1], musg[k - 1, i])
            musge[k, i] = F(4.0) / (F(1.0) / q[0] + F(1.0) / q[1] + F(1.0) / q[2] + F(1.0) / q[3]) if all(q) else F(0)
    musge[0] = musg[0]
    musge[:, NX - 1] = musg[:, NX - 1]
    lambsg = np.zeros_like(vpe)
    for i in range(NX - 1):
        lambsg[:, i] = F(0.5) * (lamb[:, i + 1] + lamb[:, i])
    lambsg[:, NX - 1] = lamb[:, NX - 1]
    lambmusg = np.zeros_like(vpe)
    for i in range(NX - 1):
        for k in range(NZ):
            lambmusg[k, i] = F(0.5) * (lamb[k, i] + F(2) * mu[k, i] + lamb[k, i + 1] + F(2) * mu[k, i + 1])
    lambmusg[:, NX - 1] = lamb[:, NX - 1] + F(2) * mu[:, NX - 1]
    out = [b2e, b1e, lambmusg, lambsg, musge]
    itopo = npz  # 1-based row itopo = npzn
    for a in out:  # rows above itopo refilled (YPUB:484-501)
        for k in range(itopo - 1, 0, -1):
            a[k - 1] = a[k]
    # Gaussian coefficients (YPUB:1470-1501), sigma = 2
    w = 2 * rgau - 1
    cen = (w + 1) // 2
    pi = F(3.1415926)
    s2 = F(2.0) * F(2.0)
    g = np.zeros((w, w), F)
    for j in range(1, w + 1):
        for i in range(1, w + 1):
            dis = F((j - cen) ** 2 + (i - cen) ** 2)
            g[i - 1, j - 1] = F(1) / (F(2) * pi * s2) * expf(-(dis / (F(2) * s2)))
    tot = F(0)
    for j in range(w):
        for i in range(w):
            tot = tot + g[i, j]
    g = (g / tot).astype(F)
    for a in (out[3], out[4], out[2], out[1], out[0]):  # modipapml order; arrays are independent
        for i in range(NX):
            for k in range(itopo):
                s = F(0)
                for n in range(i - (rgau - 1), i + rgau):
                    for m in range(k - (rgau - 1), k + rgau):
                        if 0 <= n < NX and 0 <= m < NZ:
                            s = s + a[m, n] * g[m - k + rgau - 1, n - i + rgau - 1]
                a[k, i] = s
    return [x.T for x in out]  # back to (NX, NZ)


def tiny_model(nx=14, nz=12, seed=0):
    rng = np.random.default_rng(seed)
    vp = (2000 + 800 * rng.random((nx, nz))).astype(F)
    vs = (vp / (1.6 + 0.3 * rng.random((nx, nz)))).astype(F)
    rho = (1800 + 500 * rng.random((nx, nz))).astype(F)
    return vp, vs, rho


@pytest.mark.parametrize("seed,rgau", [(0, 3), (1, 4)])
def test_prepare_bitexact_against_python_restatement(seed, rgau):
    vp, vs, rho = tiny_model(seed=seed)
    npx = npz = 4
    nx, nz = vp.shape
    NX, NZ = nx + 2 * npx, nz + 2 * npz
    L = ol.lib()
    L.oracle_iso_prepare_f32.argtypes = [ctypes.POINTER(ol.OracleIsoCfg)] + [ol._F32P] * 4
    cfg = ol.OracleIsoCfg(nx, nz, 10.0, 10.0, 1e-3, 20.0, 10, npx, npx, npz, npz, 0, nx - 1, npx + 3, npz + 2, 1, 0,
                          rgau)
    out = np.zeros((5, NX, NZ), F)
    assert L.oracle_iso_prepare_f32(ctypes.byref(cfg), ol._p(vp), ol._p(vs), ol._p(rho), ol._p(out)) == 0
    ref = py_prepare(vp, vs, rho, npx, npz, rgau)
    for a in range(5):
        assert np.array_equal(out[a].view(np.uint32), ref[a].view(np.uint32)), a
    # the smoothing changed the top rows and left the rest alone
    unsm = py_prepare(vp, vs, rho, npx, npz, 1)
    assert not np.array_equal(out[3][:, :npz], unsm[3][:, :npz])
    assert np.array_equal(out[3][:, npz:], unsm[3][:, npz:])


def layered(nx=90, nz=70, seed=2):
    rng = np.random.default_rng(seed)
    z = np.arange(nz)
    vp = np.tile(np.where(z < nz // 3, 1800.0, np.where(z < 2 * nz // 3, 2600.0, 3300.0)), (nx, 1)).astype(F)
    vp += (40.0 * rng.standard_normal((nx, nz))).astype(F)
    vs = (vp / 1.8).astype(F)
    rho = (1900.0 + 300.0 * rng.random((nx, nz))).astype(F)
    return vp, vs, rho


def test_fp32_restatement_within_1e5_of_fp64():
    vp, vs, rho = layered()
    kw = dict(dx=10.0, dz=10.0, dt=1e-3, f0=20.0, nt=260, npx=12, npz=12, isxe=12 + 45, isze=12 + 3, nrz0=2,
              idecay=60, rgau=12)
    r1, r2, _ = ol.iso_forward(vp, vs, rho, **kw)
    d1, d2, _ = ol.iso_forward(vp, vs, rho, fp64=True, **kw)
    e1, e2 = rel_l2(r1, d1), rel_l2(r2, d2)
    print(f"FP32 vs FP64: vx {e1:.2e}, vz {e2:.2e}")
    assert np.abs(d1).max() > 0 and e1 <= 1e-5 and e2 <= 1e-5


def test_homogeneous_arrival_and_mirror_symmetry():
    nx, nz = 120, 80
    vp = np.full((nx, nz), 3000.0, F)
    vs = (vp / 1.732).astype(F)
    rho = np.full((nx, nz), 2000.0, F)
    npx, dt, idecay = 15, 1e-3, 60
    r1, r2, _ = ol.iso_forward(vp, vs, rho, 10.0, 10.0, dt, 20.0, 300, npx, npx, isxe=npx + 60, isze=npx + 10, nrz0=11,
                               idecay=idecay, rgau=20)
    # the source sits on trace 59: vz (on the source's x nodes) is symmetric, vx (half a cell to the
    # left, YPUB:1115 u(i) - u(i-1)) antisymmetric about it
    assert rel_l2(r2[59 - 30], r2[59 + 30]) < 1e-3
    assert rel_l2(r1[59 - 30], -r1[60 + 30]) < 1e-4
    # the Ricker peak (it = idecay) reaches the trace 40 cells away 400 m / 3000 m/s later
    tr = r2[59 + 40]
    peak = int(np.argmax(np.abs(tr)))
    assert abs(peak - 400.0 / 3000.0 / dt) <= 8


def test_zero_density_rejected():
    vp, vs, rho = tiny_model()
    rho[3, 3] = 0.0
    with pytest.raises(ValueError):
        ol.iso_forward(vp, vs, rho, 10.0, 10.0, 1e-3, 20.0, 10, 4, 4, isxe=8, isze=6, rgau=3)


def test_free_surface_stable_and_close_to_fp64():
    """fsbc mode (YPRI:57-230): the restated free surface stays stable over a long record and
    agrees with its FP64 restatement; before the direct wave reaches the surface the records
    match the abc mode's to FP32 round-off."""
    nx, nz = 100, 90
    vp = np.full((nx, nz), 3000.0, F)
    vs = (vp / 1.732).astype(F)
    rho = np.full((nx, nz), 2000.0, F)
    kw = dict(dx=10.0, dz=10.0, dt=1e-3, f0=20.0, npx=15, npz=15, isxe=15 + 50, nrz0=2, idecay=60, rgau=20)
    for top in (1, 4):
        f1, f2, _ = ol.iso_forward(vp, vs, rho, nt=2000, isze=top + 40, npz_top=top, fsbc=True, **kw)
        peaks = [np.abs(f2[:, i:i + 250]).max() for i in range(0, 2000, 250)]
        assert peaks[-1] < 1e-4 * peaks[0], peaks
        d1, d2, _ = ol.iso_forward(vp, vs, rho, nt=300, isze=top + 40, npz_top=top, fsbc=True, fp64=True, **kw)
        assert rel_l2(f1[:, :300], d1) <= 1e-5 and rel_l2(f2[:, :300], d2) <= 1e-5
        a1, a2, _ = ol.iso_forward(vp, vs, rho, nt=300, isze=top + 40, npz_top=top, **kw)
        early = 40  # 40 samples after the Ricker peak: the wave is still 25 cells below the surface
        assert np.abs(f2[:, :early] - a2[:, :early]).max() <= 1e-5 * np.abs(f2).max()
