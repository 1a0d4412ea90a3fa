"""ctypes binding of the C ABI in include/seisfd.h (libseisfd.so, built by build.py).

There is no CPU fallback: if the native library is missing, importing this module raises.
"""
import ctypes
import os
from typing import List, Optional, Sequence

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libseisfd.so")

OK, ERR_ARG, ERR_IO, ERR_CUDA, ERR_TIMEOUT, ERR_NAN, ERR_NOMEM, ERR_UNSUPPORTED, ERR_STATE = range(9)
ACOUSTIC_2D, VISCOAC_2D, ACOUSTIC_3D, VISCOEL_2D, ELASTIC_2D = 0, 1, 2, 3, 4
EXACT, NAN_CHECK = 0x1, 0x2
WAVELET_AFD, WAVELET_RIC, WAVELET_Q, WAVELET_ISO = 0, 1, 2, 3
FIELD_P, FIELD_VX, FIELD_VZ, FIELD_VY, FIELD_R, FIELD_SZZ, FIELD_SXZ = 0, 1, 2, 3, 4, 5, 6

_F32P = ctypes.POINTER(ctypes.c_float)
_I32P = ctypes.POINTER(ctypes.c_int)


class Grid(ctypes.Structure):
    _fields_ = [("scheme", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("pml", ctypes.c_int), ("dx", ctypes.c_float), ("dy", ctypes.c_float), ("dz", ctypes.c_float),
                ("dt", ctypes.c_float), ("order", ctypes.c_int), ("flags", ctypes.c_int), ("f0", ctypes.c_float)]


class Shot(ctypes.Structure):
    _fields_ = [("sx", ctypes.c_int), ("sy", ctypes.c_int), ("sz", ctypes.c_int), ("nt", ctypes.c_int),
                ("nrec", ctypes.c_int), ("rec_x", _I32P), ("rec_y", _I32P), ("rec_z", _I32P),
                ("wavelet", _F32P), ("ap_x0", ctypes.c_int), ("ap_nx", ctypes.c_int)]


class QPar(ctypes.Structure):
    """sfd_qpar: the Q_forward parameter card."""
    _fields_ = [(n, ctypes.c_char * 256) for n in ("vp", "vs", "rho", "qp", "qs", "shot1", "shot2", "shot3", "shot4")] + \
               [("nshot", ctypes.c_int), ("offset_min", ctypes.c_float), ("offset_max", ctypes.c_float),
                ("sx0", ctypes.c_float), ("sz0", ctypes.c_float), ("rz0", ctypes.c_float), ("dsx", ctypes.c_float),
                ("nx", ctypes.c_int), ("nz", ctypes.c_int), ("dx", ctypes.c_float), ("dz", ctypes.c_float),
                ("nt", ctypes.c_int), ("dt", ctypes.c_float), ("f0", ctypes.c_float),
                ("pml_xn", ctypes.c_float), ("pml_xp", ctypes.c_float), ("pml_zn", ctypes.c_float),
                ("pml_zp", ctypes.c_float), ("fdo2", ctypes.c_int), ("fdo1", ctypes.c_int)]


def read_qpar(path: str) -> QPar:
    p = QPar()
    rc = load().sfd_qpar_read(path.encode(), ctypes.byref(p))
    if rc:
        raise SfdError(rc, f"sfd_qpar_read({path})")
    return p


class IsoPar(ctypes.Structure):
    """sfd_isopar: the yang_version parameter card."""
    _fields_ = [("molmod", ctypes.c_char * 16)] + \
               [(n, ctypes.c_char * 256) for n in ("vp", "vs", "rho", "topo", "snapx", "snapz", "shot1", "shot2",
                                                   "shot3", "shot4")] + \
               [("nshot", ctypes.c_int), ("offset_min", ctypes.c_float), ("offset_max", ctypes.c_float),
                ("sx0", ctypes.c_float), ("sz0", ctypes.c_float), ("rz0", ctypes.c_float), ("dsx", ctypes.c_float),
                ("nx", ctypes.c_int), ("nz", ctypes.c_int), ("dx", ctypes.c_float), ("dz", ctypes.c_float),
                ("nt", ctypes.c_int), ("dt", ctypes.c_float), ("dtsnap", ctypes.c_float), ("f0", ctypes.c_float),
                ("decay", ctypes.c_float), ("pml_xn", ctypes.c_float), ("pml_xp", ctypes.c_float),
                ("pml_zn", ctypes.c_float), ("pml_zp", ctypes.c_float), ("rgau", ctypes.c_int)]


def read_isopar(path: str) -> IsoPar:
    p = IsoPar()
    rc = load().sfd_isopar_read(path.encode(), ctypes.byref(p))
    if rc:
        raise SfdError(rc, f"sfd_isopar_read({path})")
    return p


SU_CDP = 0x1
SU_NO_OFFSET = 0x2  # leave offset 0, as the VTI modeller's writer does (VS:163-217)


def su_write(path: str, traces: np.ndarray, shot_no: int, isx: int, ixmin: int, dx: float, dt: float,
             flags: int = SU_CDP):
    """One shot's SU file; flags = SU_CDP sets the cdp header word as QS does, 0 leaves it 0 as
    the yang_version writer does."""
    tr = np.ascontiguousarray(traces, np.float32)
    rc = load().sfd_su_write_ex(path.encode(), _fp(tr), tr.shape[0], tr.shape[1], shot_no, isx, ixmin, dx, dt, flags)
    if rc:
        raise SfdError(rc, f"sfd_su_write({path})")


def su_merge(out_path: str, parts: Sequence[str], delete_inputs: bool = True):
    arr = (ctypes.c_char_p * len(parts))(*[p.encode() for p in parts])
    rc = load().sfd_su_merge(out_path.encode(), arr, len(parts), 1 if delete_inputs else 0)
    if rc:
        raise SfdError(rc, f"sfd_su_merge({out_path})")


class Timing(ctypes.Structure):
    _fields_ = [("loop_ms", ctypes.c_double), ("device_ms", ctypes.c_double), ("total_ms", ctypes.c_double), ("point_updates", ctypes.c_double),
                ("launches", ctypes.c_longlong), ("h2d_bytes", ctypes.c_longlong), ("d2h_bytes", ctypes.c_longlong),
                ("graph", ctypes.c_int), ("kernel_variant", ctypes.c_int)]


class VtiPar(ctypes.Structure):
    """sfd_vti_par: the VTI modeller's .par fields (VS:342-425) in cells and seconds."""
    _fields_ = [("nx_v", ctypes.c_int), ("nz_v", ctypes.c_int), ("dx", ctypes.c_float), ("dz", ctypes.c_float),
                ("dt", ctypes.c_float), ("f0", ctypes.c_float), ("nt", ctypes.c_int), ("nx_bound_l", ctypes.c_int),
                ("nx_bound_r", ctypes.c_int), ("nz_bound_u", ctypes.c_int), ("nz_bound_d", ctypes.c_int),
                ("order_explicit", ctypes.c_int), ("order_pml_1st", ctypes.c_int), ("order_pml_2nd", ctypes.c_int),
                ("flags", ctypes.c_int)]


class VtiCardFields(ctypes.Structure):
    """sfd_vtipar: the VTI modeller's parameter card (VS:342-425) as sfd_vtipar_read fills it."""
    _fields_ = [("vz", ctypes.c_char * 256), ("epsilon", ctypes.c_char * 256), ("delta", ctypes.c_char * 256),
                ("shot1", ctypes.c_char * 256), ("shot2", ctypes.c_char * 256), ("nshot", ctypes.c_int),
                ("offset_min", ctypes.c_float), ("offset_max", ctypes.c_float), ("sx0", ctypes.c_float),
                ("sz0", ctypes.c_float), ("rz0", ctypes.c_float), ("dsx", ctypes.c_float), ("nx_v", ctypes.c_int),
                ("nz_v", ctypes.c_int), ("dx_v", ctypes.c_float), ("dz_v", ctypes.c_float), ("nt", ctypes.c_int),
                ("dt", ctypes.c_float), ("f0", ctypes.c_float), ("bound_x_l", ctypes.c_float),
                ("bound_x_r", ctypes.c_float), ("bound_z_u", ctypes.c_float), ("bound_z_d", ctypes.c_float),
                ("order_explicit", ctypes.c_int), ("order_pml_1st", ctypes.c_int), ("order_pml_2nd", ctypes.c_int)]


class VtiShot(ctypes.Structure):
    """sfd_vti_shot: the reference's 1-based source column / row, receiver row and aperture."""
    _fields_ = [("nsx", ctypes.c_int), ("nsz0", ctypes.c_int), ("nrz0", ctypes.c_int), ("xmin", ctypes.c_int),
                ("xmax", ctypes.c_int)]


# Every symbol include/seisfd.h declares, with (restype, argtypes).
SIGNATURES = {
    "sfd_abi_version": (ctypes.c_int, []),
    "sfd_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "sfd_create": (ctypes.c_int, [ctypes.POINTER(Grid), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "sfd_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "sfd_last_error": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "sfd_set_model": (ctypes.c_int, [ctypes.c_void_p, _F32P, _F32P, _F32P]),
    "sfd_set_model_elastic": (ctypes.c_int, [ctypes.c_void_p, _F32P, _F32P, _F32P, _F32P, _F32P]),
    "sfd_get_records": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _F32P]),
    "sfd_set_shots": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(Shot)]),
    "sfd_forward": (ctypes.c_int, [ctypes.c_void_p, _F32P]),
    "sfd_forward_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "sfd_forward_per_shot": (ctypes.c_int, [ctypes.c_void_p, _F32P]),
    "sfd_get_wavefield": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _F32P]),
    "sfd_gradient": (ctypes.c_int, [ctypes.c_void_p, _F32P, _F32P, _F32P, _F32P]),
    "sfd_gradient_per_shot": (ctypes.c_int, [ctypes.c_void_p, _F32P, _F32P, _F32P, _F32P]),
    "sfd_gradient_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p]),
    "sfd_get_wavelet_gradient": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _F32P]),
    "sfd_set_checkpoint_interval": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "sfd_test_wait_timeout": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double]),
    "sfd_set_memory_limit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong]),
    "sfd_set_gauss_radius": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "sfd_set_free_surface": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "sfd_set_topography": (ctypes.c_int, [ctypes.c_void_p, _I32P]),
    "sfd_get_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Timing)]),
    "sfd_set_snapshots": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int]),
    "sfd_get_snapshots": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _F32P,
                                         ctypes.POINTER(ctypes.c_int)]),
    "sfd_forward_noalloc": (ctypes.c_int, [ctypes.POINTER(Grid), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _I32P, _I32P,
                                           ctypes.c_void_p, ctypes.c_void_p]),
    "sfd_qpar_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p]),
    "sfd_isopar_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p]),
    "sfd_read_floats": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_longlong, _F32P]),
    "sfd_write_floats": (ctypes.c_int, [ctypes.c_char_p, _F32P, ctypes.c_longlong, ctypes.c_int]),
    "sfd_su_write": (ctypes.c_int, [ctypes.c_char_p, _F32P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_float, ctypes.c_float]),
    "sfd_su_write_ex": (ctypes.c_int, [ctypes.c_char_p, _F32P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int]),
    "sfd_su_merge": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int, ctypes.c_int]),
    "sfd_wavelet": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int, _F32P]),
    "sfd_afd_sponge": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _F32P]),
    "sfd_fd_coeffs": (ctypes.c_int, [ctypes.c_int, _F32P]),
    "sfd_pad_model": (ctypes.c_int, [_F32P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, _F32P]),
    "sfd_vtipar_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p]),
    "sfd_vti_coefficients": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _F32P]),
    "sfd_vti_forward": (ctypes.c_int, [ctypes.POINTER(VtiPar), _F32P, _F32P, _F32P, ctypes.c_int,
                                       ctypes.POINTER(VtiShot), ctypes.c_int, _F32P, ctypes.POINTER(Timing)]),
}

_lib = None


def load():
    """Load libseisfd.so; raises if it has not been built (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m seismic_code_github_b200.build`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class SfdError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{load().sfd_status_string(status).decode()} ({status}): {msg}")
        self.status = status


def _fp(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_F32P)


def _ip(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_I32P)


def wavelet(convention: int, nt: int, dt: float, f0: float, delay: int = 150) -> np.ndarray:
    out = np.empty(nt, np.float32)
    rc = load().sfd_wavelet(convention, nt, dt, f0, delay, _fp(out))
    if rc:
        raise SfdError(rc, "sfd_wavelet")
    return out


def vti_coefficients(order: int, first: bool) -> np.ndarray:
    """coefficient_2nd (first False) / coefficient_1st (first True) of the VTI modeller, as it
    computes them in single precision (VS:1264-1472)."""
    out = np.zeros((order + 1) // 2 if first else order // 2, np.float32)
    rc = load().sfd_vti_coefficients(order, 1 if first else 0, _fp(out))
    if rc:
        raise SfdError(rc, "sfd_vti_coefficients")
    return out


def vti_forward(vz: np.ndarray, epsilon: np.ndarray, delta: np.ndarray, dx: float, dz: float, dt: float, f0: float,
                nt: int, bounds, shots, orders=(10, 9, 10), device: int = 0, exact: bool = False):
    """VTI pseudo-acoustic modelling of a survey (sfd_vti_forward): model arrays (nx_v, nz_v)
    x-major; bounds = (nx_bound_l, nx_bound_r, nz_bound_u, nz_bound_d) PML cells; shots a list of
    (nsx, nsz0, nrz0, xmin, xmax) in the reference's 1-based grid numbers, all with the same
    xmax - xmin.  exact: the reference's operation order, bit-exact with the restatement
    (SFD_EXACT); otherwise FMA contraction and approximate divisions (relative L2 <= 1e-5).
    Returns (records [nshot][xmax - xmin + 1][nt], timing dict)."""
    arrs = [np.ascontiguousarray(a, np.float32) for a in (vz, epsilon, delta)]
    nx_v, nz_v = arrs[0].shape
    for a in arrs[1:]:
        if a.shape != (nx_v, nz_v):
            raise ValueError("vz, epsilon and delta must have the same shape")
    par = VtiPar(nx_v, nz_v, dx, dz, dt, f0, nt, *bounds, *orders, EXACT if exact else 0)
    sh = (VtiShot * len(shots))(*[VtiShot(*s) for s in shots])
    rng = shots[0][4] - shots[0][3] + 1
    out = np.zeros((len(shots), rng, nt), np.float32)
    t = Timing()
    rc = load().sfd_vti_forward(ctypes.byref(par), *[_fp(a) for a in arrs], len(shots), sh, device, _fp(out),
                                ctypes.byref(t))
    if rc:
        raise SfdError(rc, "sfd_vti_forward")
    return out, {k: getattr(t, k) for k, _ in Timing._fields_}


def afd_sponge(nx: int, nz: int, pml: int) -> np.ndarray:
    out = np.empty((nx, nz), np.float32)
    rc = load().sfd_afd_sponge(nx, nz, pml, _fp(out))
    if rc:
        raise SfdError(rc, "sfd_afd_sponge")
    return out


def fd_coeffs(order: int) -> np.ndarray:
    out = np.zeros(8, np.float32)
    rc = load().sfd_fd_coeffs(order, _fp(out))
    if rc:
        raise SfdError(rc, "sfd_fd_coeffs")
    return out[: order // 2]


def pad_model(a: np.ndarray, pxn: int, pxp: int, pzn: int, pzp: int) -> np.ndarray:
    a = np.ascontiguousarray(a, np.float32)
    out = np.empty((a.shape[0] + pxn + pxp, a.shape[1] + pzn + pzp), np.float32)
    rc = load().sfd_pad_model(_fp(a), a.shape[0], a.shape[1], pxn, pxp, pzn, pzp, _fp(out))
    if rc:
        raise SfdError(rc, "sfd_pad_model")
    return out


class ShotSpec:
    """One shot: source cell, receiver cells, wavelet (nt samples), optional aperture."""

    def __init__(self, sx: int, sz: int, rec_x: Sequence[int], rec_z: Sequence[int], wavelet: np.ndarray,
                 sy: int = 0, rec_y: Optional[Sequence[int]] = None, ap_x0: int = 0, ap_nx: int = 0):
        self.sx, self.sy, self.sz = int(sx), int(sy), int(sz)
        self.rec_x = np.ascontiguousarray(rec_x, np.int32)
        self.rec_z = np.ascontiguousarray(rec_z, np.int32)
        self.rec_y = None if rec_y is None else np.ascontiguousarray(rec_y, np.int32)
        self.wavelet = np.ascontiguousarray(wavelet, np.float32)
        self.ap_x0, self.ap_nx = int(ap_x0), int(ap_nx)

    @property
    def nt(self) -> int:
        return int(self.wavelet.shape[0])

    @property
    def nrec(self) -> int:
        return int(self.rec_x.shape[0])


class Engine:
    """Owns one sfd_ctx (one device, one stream)."""

    def __init__(self, scheme: int, nx: int, nz: int, dx: float, dz: float, dt: float, pml: int, order: int = 16,
                 ny: int = 1, dy: float = 0.0, flags: int = 0, f0: float = 0.0, device: int = 0):
        self._lib = load()
        self.grid = Grid(scheme, nx, ny, nz, pml, dx, dy, dz, dt, order, flags, f0)
        h = ctypes.c_void_p()
        rc = self._lib.sfd_create(ctypes.byref(self.grid), device, ctypes.byref(h))
        if rc:
            raise SfdError(rc, "sfd_create")
        self._h = h
        self._shots: List[ShotSpec] = []

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sfd_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def last_error(self) -> str:
        buf = ctypes.create_string_buffer(1024)
        self._lib.sfd_last_error(self._h, buf, 1024)
        return buf.value.decode(errors="replace")

    def _check(self, rc: int, what: str):
        if rc:
            raise SfdError(rc, f"{what}: {self.last_error()}")

    def set_model(self, vp: np.ndarray, den: Optional[np.ndarray] = None, q: Optional[np.ndarray] = None):
        vp = np.ascontiguousarray(vp, np.float32)
        den = None if den is None else np.ascontiguousarray(den, np.float32)
        q = None if q is None else np.ascontiguousarray(q, np.float32)
        self._keep_model = (vp, den, q)
        self._check(self._lib.sfd_set_model(self._h, _fp(vp), _fp(den), _fp(q)), "sfd_set_model")

    def set_model_elastic(self, vp: np.ndarray, vs: np.ndarray, den: Optional[np.ndarray] = None,
                          qp: Optional[np.ndarray] = None, qs: Optional[np.ndarray] = None):
        """P and S velocities, density and quality factors of the visco-elastic scheme (the
        isotropic elastic scheme takes no quality factors)."""
        arrs = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (vp, vs, den, qp, qs)]
        self._keep_model = tuple(arrs)
        self._check(self._lib.sfd_set_model_elastic(self._h, *[_fp(a) for a in arrs]), "sfd_set_model_elastic")

    def records(self, field: int) -> np.ndarray:
        """Records of one component from the last forward, in the layout of forward(): FIELD_SZZ
        (record1, strzz) or FIELD_P (record2, strxx) for the Q_forward schemes, FIELD_VX (record1)
        or FIELD_VZ (record2) for the isotropic elastic scheme."""
        out = np.empty(self.record_size(), np.float32)
        self._check(self._lib.sfd_get_records(self._h, field, _fp(out)), "sfd_get_records")
        return out

    def set_shots(self, shots: Sequence[ShotSpec]):
        arr = (Shot * len(shots))()
        for i, s in enumerate(shots):
            arr[i] = Shot(s.sx, s.sy, s.sz, s.nt, s.nrec, _ip(s.rec_x), _ip(s.rec_y), _ip(s.rec_z),
                          _fp(s.wavelet), s.ap_x0, s.ap_nx)
        self._shots = list(shots)
        self._check(self._lib.sfd_set_shots(self._h, len(shots), arr), "sfd_set_shots")

    def record_size(self) -> int:
        return sum(s.nrec * s.nt for s in self._shots)

    def split_records(self, flat: np.ndarray) -> List[np.ndarray]:
        out, off = [], 0
        for s in self._shots:
            n = s.nrec * s.nt
            out.append(flat[off:off + n].reshape(s.nrec, s.nt))
            off += n
        return out

    def forward(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        rec = out if out is not None else np.empty(self.record_size(), np.float32)
        self._check(self._lib.sfd_forward(self._h, _fp(rec)), "sfd_forward")
        return rec

    def forward_per_shot(self) -> np.ndarray:
        rec = np.empty(self.record_size(), np.float32)
        self._check(self._lib.sfd_forward_per_shot(self._h, _fp(rec)), "sfd_forward_per_shot")
        return rec

    def forward_device(self, dev_ptr: int):
        self._check(self._lib.sfd_forward_device(self._h, ctypes.c_void_p(dev_ptr)), "sfd_forward_device")

    def wavefield(self, shot: int, field: int) -> np.ndarray:
        s = self._shots[shot]
        nx = s.ap_nx if s.ap_nx > 0 else self.grid.nx
        out = np.empty((nx, self.grid.ny, self.grid.nz) if self.grid.ny > 1 else (nx, self.grid.nz), np.float32)
        self._check(self._lib.sfd_get_wavefield(self._h, shot, field, _fp(out)), "sfd_get_wavefield")
        return out

    def gradient(self, obs: np.ndarray, want_invq: bool = False, per_shot: bool = False):
        """misfit 0.5*sum (pred - obs)^2 and its gradient w.r.t. vp (and 1/Q for the
        viscoacoustic scheme); obs in the record layout of forward()."""
        obs = np.ascontiguousarray(obs, np.float32).reshape(-1)
        assert obs.size == self.record_size()
        mis = np.zeros(1, np.float32)
        n = self.grid.nx * self.grid.ny * self.grid.nz
        g = np.empty(n, np.float32)
        gq = np.empty(n, np.float32) if want_invq else None
        fn = self._lib.sfd_gradient_per_shot if per_shot else self._lib.sfd_gradient
        self._check(fn(self._h, _fp(obs), _fp(mis), _fp(g), _fp(gq)), "sfd_gradient")
        shape = (self.grid.nx, self.grid.nz) if self.grid.ny == 1 else (self.grid.nx, self.grid.ny, self.grid.nz)
        return float(mis[0]), g.reshape(shape), (None if gq is None else gq.reshape(shape))

    def gradient_device(self, obs_dev: int, misfit_dev: int, grad_vp_dev: int, grad_invq_dev: Optional[int] = None):
        """sfd_gradient_device: every argument is a device address on this engine's device (for
        torch tensors, tensor.data_ptr()): obs in the record layout of forward(), misfit one
        float32, grad_vp / grad_invq the model grid in float32."""
        self._check(self._lib.sfd_gradient_device(self._h, obs_dev, misfit_dev, grad_vp_dev, grad_invq_dev),
                    "sfd_gradient_device")

    def wavelet_gradient(self, shot: int) -> np.ndarray:
        out = np.empty(self._shots[shot].nt, np.float32)
        self._check(self._lib.sfd_get_wavelet_gradient(self._h, shot, _fp(out)), "sfd_get_wavelet_gradient")
        return out

    def test_wait_timeout(self, cta: int, step: int, limit_s: float = 1e-4):
        """Test hook (sfd_test_wait_timeout): CTA `cta` of step `step` issues no tile loads and
        gives up its bounded wait after limit_s seconds; cta < 0 removes the hook."""
        self._check(self._lib.sfd_test_wait_timeout(self._h, cta, step, limit_s), "sfd_test_wait_timeout")

    def set_checkpoint_interval(self, steps: int):
        self._check(self._lib.sfd_set_checkpoint_interval(self._h, steps), "sfd_set_checkpoint_interval")

    def set_gauss_radius(self, rgau: int):
        """Half-width of the source / top-sponge Gaussian of the isotropic elastic scheme
        (YPUB:1470-1501; default 50)."""
        self._check(self._lib.sfd_set_gauss_radius(self._h, int(rgau)), "sfd_set_gauss_radius")

    def set_free_surface(self, top: int):
        """Boundary mode of the isotropic elastic scheme: 0 = absorbing on all sides ('abc'),
        top >= 1 = free surface at padded row top - 1 ('fsbc', the reference's itopo = top)."""
        self._check(self._lib.sfd_set_free_surface(self._h, int(top)), "sfd_set_free_surface")

    def set_topography(self, itopo):
        """Surface row per padded model column for the isotropic elastic scheme (the reference's
        1-based itopoe = nint(topo/dz) + npzn); None restores the flat surface."""
        if itopo is None:
            self._check(self._lib.sfd_set_topography(self._h, None), "sfd_set_topography")
            return
        a = np.ascontiguousarray(itopo, np.int32)
        self._check(self._lib.sfd_set_topography(self._h, a.ctypes.data_as(_I32P)), "sfd_set_topography")

    def set_memory_limit(self, nbytes: int):
        """Device-memory budget of gradient() (0: the free device memory)."""
        self._check(self._lib.sfd_set_memory_limit(self._h, int(nbytes)), "sfd_set_memory_limit")

    def set_snapshots(self, stream: int, field: int, first: int, every: int, count: int):
        self._check(self._lib.sfd_set_snapshots(self._h, stream, field, first, every, count), "sfd_set_snapshots")

    def snapshots(self, stream: int, shot: int) -> np.ndarray:
        """(n, nx_shot - 2 pml, nz - 2 pml) interior snapshots of one shot from the last forward."""
        n = ctypes.c_int()
        self._check(self._lib.sfd_get_snapshots(self._h, stream, shot, None, ctypes.byref(n)), "sfd_get_snapshots")
        s = self._shots[shot]
        nx = (s.ap_nx if s.ap_nx > 0 else self.grid.nx) - 2 * self.grid.pml
        out = np.empty((n.value, nx, self.grid.nz - 2 * self.grid.pml), np.float32)
        self._check(self._lib.sfd_get_snapshots(self._h, stream, shot, _fp(out), ctypes.byref(n)), "sfd_get_snapshots")
        return out

    def timing(self) -> dict:
        t = Timing()
        self._check(self._lib.sfd_get_timing(self._h, ctypes.byref(t)), "sfd_get_timing")
        return {k: getattr(t, k) for k, _ in Timing._fields_}
