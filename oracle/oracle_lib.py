"""ctypes bindings of the CPU restatements (oracle/_build/liboracle.so).

ORACLE -- test infrastructure only: imported by tests/, by __graft_entry__.smoke() as the
checker and by bench.py's cpu_baseline leg. The product never imports this module.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_F32P = ctypes.POINTER(ctypes.c_float)
_F64P = ctypes.POINTER(ctypes.c_double)
_I32P = ctypes.POINTER(ctypes.c_int)


class OracleAfdCfg(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("nz", ctypes.c_int), ("pml", ctypes.c_int), ("nt", ctypes.c_int),
        ("dx", ctypes.c_float), ("dz", ctypes.c_float), ("dt", ctypes.c_float),
        ("radius", ctypes.c_int), ("sx", ctypes.c_int), ("sz", ctypes.c_int),
        ("nrec", ctypes.c_int), ("rec_x", _I32P), ("rec_z", _I32P), ("snap_step", ctypes.c_int),
    ]


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.oracle_afd_f32.argtypes = [ctypes.POINTER(OracleAfdCfg), _F32P, _F32P, _F32P, _F32P, _F32P, _F32P]
        _lib.oracle_afd_f64.argtypes = [ctypes.POINTER(OracleAfdCfg), _F32P, _F32P, _F32P, _F64P, _F64P, _F64P]
        _lib.oracle_afd_sponge.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _F32P]
        _lib.oracle_afd_coeffs.argtypes = [ctypes.c_int, _F32P]
        _lib.oracle_wavelet_afd.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_float, _F32P]
        _lib.oracle_wavelet_ric.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_int, _F32P]
        _lib.oracle_wavelet_afd.restype = None
        _lib.oracle_wavelet_ric.restype = None
    return _lib


def _p(a, t=_F32P):
    return a.ctypes.data_as(t) if a is not None else None


def afd_sponge(nx: int, nz: int, pml: int) -> np.ndarray:
    out = np.empty((nx, nz), np.float32)
    assert lib().oracle_afd_sponge(nx, nz, pml, _p(out)) == 0
    return out


def afd_coeffs(radius: int) -> np.ndarray:
    out = np.zeros(8, np.float32)
    assert lib().oracle_afd_coeffs(radius, _p(out)) == 0
    return out[:radius]


def wavelet_afd(nt: int, dt: float, freq: float) -> np.ndarray:
    out = np.empty(nt, np.float32)
    lib().oracle_wavelet_afd(nt, dt, freq, _p(out))
    return out


def wavelet_ric(nt: int, dt: float, f0: int, delay: int = 150) -> np.ndarray:
    out = np.empty(nt, np.float32)
    lib().oracle_wavelet_ric(nt, dt, int(f0), int(delay), _p(out))
    return out


def afd_forward(nx, nz, pml, nt, dx, dz, dt, vp, den, wavelet, sx, sz, rec_x, rec_z,
                radius=8, snap_step=-1, fp64=False, want_state=False):
    """Run the restated AFD time loop. Returns (record[nrec, nt], snap_vx[nx, nz] or None,
    final_state[3, nx, nz] (P, Vx, Vz after the sponge) or None)."""
    rec_x = np.ascontiguousarray(rec_x, np.int32)
    rec_z = np.ascontiguousarray(rec_z, np.int32)
    vp = np.ascontiguousarray(vp, np.float32)
    den = np.ascontiguousarray(den, np.float32)
    wavelet = np.ascontiguousarray(wavelet, np.float32)
    assert vp.shape == (nx, nz) and den.shape == (nx, nz) and wavelet.shape[0] >= nt
    cfg = OracleAfdCfg(nx, nz, pml, nt, dx, dz, dt, radius, sx, sz, len(rec_x),
                       _p(rec_x, _I32P), _p(rec_z, _I32P), snap_step)
    dt_ = np.float64 if fp64 else np.float32
    tp = _F64P if fp64 else _F32P
    rec = np.zeros((len(rec_x), nt), dt_)
    snap = np.zeros((nx, nz), dt_) if snap_step >= 0 else None
    state = np.zeros((3, nx, nz), dt_) if want_state else None
    fn = lib().oracle_afd_f64 if fp64 else lib().oracle_afd_f32
    rc = fn(ctypes.byref(cfg), _p(vp), _p(den), _p(wavelet), _p(rec, tp), _p(snap, tp), _p(state, tp))
    if rc != 0:
        raise ValueError(f"oracle_afd rejected the configuration (rc={rc})")
    return rec, snap, state


def afd_gradient_f64(nx, nz, pml, nt, dx, dz, dt, vp, den, wavelet, sx, sz, rec_x, rec_z, obs, radius=8):
    """FP64 misfit, d misfit/d vp (padded grid), d misfit/d wavelet and FP64 records
    (oracle/adj_oracle.cpp)."""
    L = lib()
    if not hasattr(L, "_grad_sig"):
        L.oracle_afd_gradient_f64.argtypes = [ctypes.POINTER(OracleAfdCfg), _F32P, _F32P, _F32P, _F32P, _F64P,
                                              _F64P, _F64P, _F64P]
        L._grad_sig = True
    rec_x = np.ascontiguousarray(rec_x, np.int32)
    rec_z = np.ascontiguousarray(rec_z, np.int32)
    vp = np.ascontiguousarray(vp, np.float32)
    den = np.ascontiguousarray(den, np.float32)
    wavelet = np.ascontiguousarray(wavelet, np.float32)
    obs = np.ascontiguousarray(obs, np.float32)
    assert obs.shape == (len(rec_x), nt)
    cfg = OracleAfdCfg(nx, nz, pml, nt, dx, dz, dt, radius, sx, sz, len(rec_x), _p(rec_x, _I32P),
                       _p(rec_z, _I32P), -1)
    mis = np.zeros(1, np.float64)
    g = np.zeros((nx, nz), np.float64)
    dw = np.zeros(nt, np.float64)
    rec = np.zeros((len(rec_x), nt), np.float64)
    rc = L.oracle_afd_gradient_f64(ctypes.byref(cfg), _p(vp), _p(den), _p(wavelet), _p(obs), _p(mis, _F64P),
                                   _p(g, _F64P), _p(dw, _F64P), _p(rec, _F64P))
    if rc != 0:
        raise ValueError(f"oracle_afd_gradient_f64 rejected the configuration (rc={rc})")
    return float(mis[0]), g, dw, rec


class OracleQCfg(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("nz", ctypes.c_int), ("dx", ctypes.c_float), ("dz", ctypes.c_float),
                ("dt", ctypes.c_float), ("f0", ctypes.c_float), ("nt", ctypes.c_int), ("npxn", ctypes.c_int),
                ("npxp", ctypes.c_int), ("npzn", ctypes.c_int), ("npzp", ctypes.c_int), ("ixmine", ctypes.c_int),
                ("ixmaxe", ctypes.c_int), ("isxe", ctypes.c_int), ("isze", ctypes.c_int), ("nrz0", ctypes.c_int),
                ("q_override", ctypes.c_int)]


def q_decay(f0: float, dt: float) -> int:
    """QM:279-280: nwt = 2*nint(1.2/(f0*dt)) in single precision, decay = nint(nwt/2)."""
    x = float(np.float32(1.2) / (np.float32(f0) * np.float32(dt)))
    nwt = 2 * int(np.floor(x + 0.5))
    return int(np.floor(nwt / 2.0 + 0.5))


def q_forward(vp, vs, rho, qp, qs, dx, dz, dt, f0, nt, npx, npz, isxe, isze, nrz0=1, ixmine=None, ixmaxe=None,
              q_override=False, fp64=False, want_final=False):
    """Restated Q_forward single-shot modelling (oracle/q_oracle.cpp). Model arrays are the
    interior (nx, nz) float32 x-major arrays; returns (record1 = strzz, record2 = strxx, final
    strxx or None), records [nxe][nt]."""
    L = lib()
    if not hasattr(L, "_q_sig"):
        tp = ctypes.POINTER(OracleQCfg)
        L.oracle_q_f32.argtypes = [tp, _F32P, _F32P, _F32P, _F32P, _F32P, _F32P, _F32P, _F32P]
        L.oracle_q_f64.argtypes = [tp, _F32P, _F32P, _F32P, _F32P, _F32P, _F64P, _F64P, _F64P]
        L._q_sig = True
    arrs = [np.ascontiguousarray(a, np.float32) for a in (vp, vs, rho, qp, qs)]
    nx, nz = arrs[0].shape
    ixmine = 0 if ixmine is None else ixmine
    ixmaxe = nx - 1 if ixmaxe is None else ixmaxe
    nxe = ixmaxe - ixmine + 1
    cfg = OracleQCfg(nx, nz, dx, dz, dt, f0, nt, npx, npx, npz, npz, ixmine, ixmaxe, isxe, isze, nrz0,
                     1 if q_override else 0)
    dt_ = np.float64 if fp64 else np.float32
    tp = _F64P if fp64 else _F32P
    r1 = np.zeros((nxe, nt), dt_)
    r2 = np.zeros((nxe, nt), dt_)
    fin = np.zeros((nx + 2 * npx if ixmine == 0 and ixmaxe == nx - 1 else nxe + 2 * npx, nz + 2 * npz), dt_) \
        if want_final else None
    fn = L.oracle_q_f64 if fp64 else L.oracle_q_f32
    rc = fn(ctypes.byref(cfg), *[_p(a) for a in arrs], _p(r1, tp), _p(r2, tp), _p(fin, tp))
    if rc != 0:
        raise ValueError(f"oracle_q rejected the configuration (rc={rc})")
    return r1, r2, fin


class OracleIsoCfg(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("nz", ctypes.c_int), ("dx", ctypes.c_float), ("dz", ctypes.c_float),
                ("dt", ctypes.c_float), ("f0", ctypes.c_float), ("nt", ctypes.c_int), ("npxn", ctypes.c_int),
                ("npxp", ctypes.c_int), ("npzn", ctypes.c_int), ("npzp", ctypes.c_int), ("ixmine", ctypes.c_int),
                ("ixmaxe", ctypes.c_int), ("isxe", ctypes.c_int), ("isze", ctypes.c_int), ("nrz0", ctypes.c_int),
                ("idecay", ctypes.c_int), ("rgau", ctypes.c_int), ("fsbc", ctypes.c_int), ("topo", _F32P)]


def iso_forward(vp, vs, rho, dx, dz, dt, f0, nt, npx, npz, isxe, isze, nrz0=1, idecay=0, rgau=50, ixmine=None,
                ixmaxe=None, fp64=False, want_final=False, fsbc=False, npz_top=None, topo=None):
    """Restated yang_version isotropic elastic modelling, abc mode, flat surface
    (oracle/iso_oracle.cpp).  Model arrays are the interior (nx, nz) float32 x-major arrays; npx /
    npz are the sponge cells on both sides (npxn = npxp, npzn = npzp; npz_top overrides npzn, the
    1-based surface row itopo of the fsbc mode); topo: surface depth (m) per model column (None:
    flat); source row 1-based as in the Fortran (isz + itopoe(isxe)), receivers at
    itopo(i) + nrz0.  Returns (record1 = vx, record2 = vz, final vx or None), records [nxe][nt]."""
    L = lib()
    if not hasattr(L, "_iso_sig"):
        tp = ctypes.POINTER(OracleIsoCfg)
        L.oracle_iso_f32.argtypes = [tp, _F32P, _F32P, _F32P, _F32P, _F32P, _F32P]
        L.oracle_iso_f64.argtypes = [tp, _F32P, _F32P, _F32P, _F64P, _F64P, _F64P]
        L._iso_sig = True
    arrs = [np.ascontiguousarray(a, np.float32) for a in (vp, vs, rho)]
    nx, nz = arrs[0].shape
    ixmine = 0 if ixmine is None else ixmine
    ixmaxe = nx - 1 if ixmaxe is None else ixmaxe
    nxe = ixmaxe - ixmine + 1
    top = npz if npz_top is None else npz_top
    topo_a = None if topo is None else np.ascontiguousarray(topo, np.float32)
    cfg = OracleIsoCfg(nx, nz, dx, dz, dt, f0, nt, npx, npx, top, npz, ixmine, ixmaxe, isxe, isze, nrz0, idecay, rgau,
                       1 if fsbc else 0, _p(topo_a))
    dt_ = np.float64 if fp64 else np.float32
    tp = _F64P if fp64 else _F32P
    r1 = np.zeros((nxe, nt), dt_)
    r2 = np.zeros((nxe, nt), dt_)
    fin = np.zeros((nxe + 2 * npx, nz + top + npz), dt_) if want_final else None
    fn = L.oracle_iso_f64 if fp64 else L.oracle_iso_f32
    rc = fn(ctypes.byref(cfg), *[_p(a) for a in arrs], _p(r1, tp), _p(r2, tp), _p(fin, tp))
    if rc != 0:
        raise ValueError(f"oracle_iso rejected the configuration (rc={rc})")
    return r1, r2, fin


class OracleVtiCfg(ctypes.Structure):
    _fields_ = [("nx_v", ctypes.c_int), ("nz_v", ctypes.c_int), ("nt", ctypes.c_int), ("dx", ctypes.c_float),
                ("dz", ctypes.c_float), ("dt", ctypes.c_float), ("f0", ctypes.c_float), ("nx_bound_l", ctypes.c_int),
                ("nx_bound_r", ctypes.c_int), ("nz_bound_u", ctypes.c_int), ("nz_bound_d", ctypes.c_int),
                ("order_explicit", ctypes.c_int), ("order_pml_1st", ctypes.c_int), ("order_pml_2nd", ctypes.c_int),
                ("nsx", ctypes.c_int), ("nsz0", ctypes.c_int), ("nrz0", ctypes.c_int), ("xmin", ctypes.c_int),
                ("xmax", ctypes.c_int)]


def vti_coefficients(order, first, fp64=False):
    """The FD coefficients of coefficient_2nd (first = 0) / coefficient_1st (first = 1)
    (oracle/vti_oracle.cpp, VS:1264-1472)."""
    L = lib()
    k = (order + 1) // 2 if first else order // 2
    out = np.zeros(k, np.float64 if fp64 else np.float32)
    fn = L.oracle_vti_coef_f64 if fp64 else L.oracle_vti_coef_f32
    fn.argtypes = [ctypes.c_int, ctypes.c_int, _F64P if fp64 else _F32P]
    if fn(order, 1 if first else 0, _p(out, _F64P if fp64 else _F32P)) != 0:
        raise ValueError("unsupported order")
    return out


def vti_forward(vz, eps, delta, dx, dz, dt, f0, nt, bounds, nsx, nsz0, nrz0, xmin, xmax, orders=(10, 9, 10),
                fp64=False):
    """Restated VTI pseudo-acoustic modelling of one shot (oracle/vti_oracle.cpp).  Model arrays
    (nx_v, nz_v) float32 x-major; bounds = (nx_bound_l, nx_bound_r, nz_bound_u, nz_bound_d) in
    cells; nsx, nsz0, nrz0, xmin, xmax the reference's 1-based grid numbers.  Returns the record
    [xmax - xmin + 1][nt] (u on the receiver row)."""
    L = lib()
    if not hasattr(L, "_vti_sig"):
        tp = ctypes.POINTER(OracleVtiCfg)
        L.oracle_vti_f32.argtypes = [tp, _F32P, _F32P, _F32P, _F32P]
        L.oracle_vti_f64.argtypes = [tp, _F32P, _F32P, _F32P, _F64P]
        L._vti_sig = True
    arrs = [np.ascontiguousarray(a, np.float32) for a in (vz, eps, delta)]
    nx_v, nz_v = arrs[0].shape
    cfg = OracleVtiCfg(nx_v, nz_v, nt, dx, dz, dt, f0, *bounds, *orders, nsx, nsz0, nrz0, xmin, xmax)
    rec = np.zeros((xmax - xmin + 1, nt), np.float64 if fp64 else np.float32)
    fn = L.oracle_vti_f64 if fp64 else L.oracle_vti_f32
    if fn(ctypes.byref(cfg), *[_p(a) for a in arrs], _p(rec, _F64P if fp64 else _F32P)) != 0:
        raise ValueError("oracle_vti rejected the configuration")
    return rec


class OracleAfd3Cfg(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("pml", ctypes.c_int),
                ("nt", ctypes.c_int), ("radius", ctypes.c_int), ("dx", ctypes.c_float), ("dy", ctypes.c_float),
                ("dz", ctypes.c_float), ("dt", ctypes.c_float), ("sx", ctypes.c_int), ("sy", ctypes.c_int),
                ("sz", ctypes.c_int), ("nrec", ctypes.c_int), ("rec_x", _I32P), ("rec_y", _I32P),
                ("rec_z", _I32P), ("den_c", ctypes.c_float)]


def afd3d_sponge(nx: int, ny: int, nz: int, pml: int) -> np.ndarray:
    a = np.empty((nx, ny, nz), np.float32)
    if lib().oracle_afd3d_sponge(nx, ny, nz, pml, _p(a)) != 0:
        raise ValueError("bad sponge size")
    return a


def afd3d_gradient_f64(vp, den, wavelet, src, rec_x, rec_y, rec_z, pml, dx, dy, dz, dt, obs=None, radius=4,
                       den_c=2400.0):
    """FP64 3-D records, misfit, d misfit/d vp and d misfit/d wavelet (oracle/adj3d_oracle.cpp).
    Returns dict(records, misfit, grad_vp, dw); the gradients are None without obs."""
    L = lib()
    if not hasattr(L, "_a3g_sig"):
        L.oracle_afd3d_gradient_f64.argtypes = [ctypes.POINTER(OracleAfd3Cfg), _F32P, _F32P, _F32P, _F32P, _F64P,
                                                _F64P, _F64P, _F64P]
        L._a3g_sig = True
    vp = np.ascontiguousarray(vp, np.float32)
    nx, ny, nz = vp.shape
    den = None if den is None else np.ascontiguousarray(den, np.float32)
    w = np.ascontiguousarray(wavelet, np.float32)
    rx, ry, rz = (np.ascontiguousarray(a, np.int32) for a in (rec_x, rec_y, rec_z))
    cfg = OracleAfd3Cfg(nx, ny, nz, pml, len(w), radius, dx, dy, dz, dt, src[0], src[1], src[2], len(rx),
                        rx.ctypes.data_as(_I32P), ry.ctypes.data_as(_I32P), rz.ctypes.data_as(_I32P), den_c)
    rec = np.zeros((len(rx), len(w)), np.float64)
    mis = np.zeros(1, np.float64)
    g = np.zeros((nx, ny, nz), np.float64) if obs is not None else None
    dw = np.zeros(len(w), np.float64) if obs is not None else None
    o = None if obs is None else np.ascontiguousarray(obs, np.float32)
    rc = L.oracle_afd3d_gradient_f64(ctypes.byref(cfg), _p(vp), None if den is None else _p(den), _p(w),
                                     None if o is None else _p(o), _p(mis, _F64P), None if g is None else _p(g, _F64P),
                                     None if dw is None else _p(dw, _F64P), _p(rec, _F64P))
    if rc != 0:
        raise ValueError("oracle_afd3d_gradient_f64 rejected the configuration")
    return {"records": rec, "misfit": float(mis[0]), "grad_vp": g, "dw": dw}


def afd3d_forward(vp, den, wavelet, src, rec_x, rec_y, rec_z, pml, dx, dy, dz, dt, radius=4, fp64=True,
                  den_c=2400.0, want_final=False):
    """Restated 3-D scheme (oracle/afd3d_oracle.cpp) for one shot on the padded (nx, ny, nz) grid.
    Returns records [nrec][nt] (float64 or float32) and the final P (or None)."""
    L = lib()
    if not hasattr(L, "_a3_sig"):
        tp = ctypes.POINTER(OracleAfd3Cfg)
        L.oracle_afd3d_f32.argtypes = [tp, _F32P, _F32P, _F32P, _F32P, _F32P]
        L.oracle_afd3d_f64.argtypes = [tp, _F32P, _F32P, _F32P, _F64P, _F64P]
        L._a3_sig = True
    vp = np.ascontiguousarray(vp, np.float32)
    nx, ny, nz = vp.shape
    den = None if den is None else np.ascontiguousarray(den, np.float32)
    w = np.ascontiguousarray(wavelet, np.float32)
    rx, ry, rz = (np.ascontiguousarray(a, np.int32) for a in (rec_x, rec_y, rec_z))
    cfg = OracleAfd3Cfg(nx, ny, nz, pml, len(w), radius, dx, dy, dz, dt, src[0], src[1], src[2], len(rx),
                        rx.ctypes.data_as(_I32P), ry.ctypes.data_as(_I32P), rz.ctypes.data_as(_I32P), den_c)
    dt_ = np.float64 if fp64 else np.float32
    tp = _F64P if fp64 else _F32P
    rec = np.zeros((len(rx), len(w)), dt_)
    fin = np.zeros((nx, ny, nz), dt_) if want_final else None
    fn = L.oracle_afd3d_f64 if fp64 else L.oracle_afd3d_f32
    rc = fn(ctypes.byref(cfg), _p(vp), None if den is None else _p(den), _p(w), _p(rec, tp),
            None if fin is None else _p(fin, tp))
    if rc != 0:
        raise ValueError("oracle_afd3d rejected the configuration")
    return rec, fin


class OracleQGradCfg(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("nz", ctypes.c_int), ("np", ctypes.c_int), ("dx", ctypes.c_float),
                ("dz", ctypes.c_float), ("dt", ctypes.c_float), ("f0", ctypes.c_float), ("nt", ctypes.c_int),
                ("sx", ctypes.c_int), ("sz", ctypes.c_int), ("nrec", ctypes.c_int), ("rec_x", _I32P),
                ("rec_z", _I32P)]


def q_gradient_f64(vp, rho, q, wavelet, src, rec_x, rec_z, np_, dx, dz, dt, f0, obs=None):
    """FP64 viscoacoustic forward (+ gradient when obs is given) on the padded grid
    (oracle/q_adj_oracle.cpp).  Returns dict(records, misfit, grad_vp, grad_invq, dw)."""
    L = lib()
    if not hasattr(L, "_qg_sig"):
        L.oracle_q_gradient_f64.argtypes = [ctypes.POINTER(OracleQGradCfg), _F32P, _F32P, _F32P, _F32P, _F32P,
                                            _F64P, _F64P, _F64P, _F64P, _F64P]
        L._qg_sig = True
    vp = np.ascontiguousarray(vp, np.float32)
    nx, nz = vp.shape
    rho = np.ascontiguousarray(rho, np.float32)
    q = None if q is None else np.ascontiguousarray(q, np.float32)
    w = np.ascontiguousarray(wavelet, np.float32)
    rx, rz = np.ascontiguousarray(rec_x, np.int32), np.ascontiguousarray(rec_z, np.int32)
    cfg = OracleQGradCfg(nx, nz, np_, dx, dz, dt, f0, len(w), src[0], src[1], len(rx), rx.ctypes.data_as(_I32P),
                         rz.ctypes.data_as(_I32P))
    rec = np.zeros((len(rx), len(w)), np.float64)
    mis = np.zeros(1, np.float64)
    g1 = np.zeros((nx, nz), np.float64) if obs is not None else None
    g2 = np.zeros((nx, nz), np.float64) if obs is not None else None
    dw = np.zeros(len(w), np.float64) if obs is not None else None
    o = None if obs is None else np.ascontiguousarray(obs, np.float32)
    rc = L.oracle_q_gradient_f64(ctypes.byref(cfg), _p(vp), _p(rho), None if q is None else _p(q), _p(w),
                                 None if o is None else _p(o), _p(mis, _F64P), None if g1 is None else _p(g1, _F64P),
                                 None if g2 is None else _p(g2, _F64P), None if dw is None else _p(dw, _F64P),
                                 _p(rec, _F64P))
    if rc:
        raise ValueError(f"oracle_q_gradient_f64 rejected the configuration (rc={rc})")
    return {"records": rec, "misfit": float(mis[0]), "grad_vp": g1, "grad_invq": g2, "dw": dw}
