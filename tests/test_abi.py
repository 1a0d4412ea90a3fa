"""CPU checks of the C ABI: the library loads, exports every symbol include/seisfd.h declares,
the host helpers agree bit-for-bit with the oracle and the reference tools, and invalid
arguments are rejected with status codes before any device work."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle_lib as ol
from conftest import ROOT, bits_equal
from seismic_code_github_b200 import seisfd as S


def declared_symbols():
    syms = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            with open(os.path.join(ROOT, "include", fn)) as f:
                txt = f.read()
            syms |= set(re.findall(r"^\s*(?:int|const char\*|void)\s+(sfd_\w+)\s*\(", txt, re.M))
    return syms


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(S.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 18
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # and the Python binding covers all of them
    assert syms <= set(S.SIGNATURES), syms - set(S.SIGNATURES)


def test_abi_version_and_status_strings():
    lib = S.load()
    assert lib.sfd_abi_version() == 1
    assert lib.sfd_status_string(S.ERR_TIMEOUT) == b"device wait timed out"
    assert lib.sfd_status_string(99) == b"unknown status"


def test_wavelets_match_reference_formulas(golden):
    ric = np.fromfile(os.path.join(golden, "ric_trace255.f32"), np.float32)
    assert bits_equal(S.wavelet(S.WAVELET_RIC, 1024, 0.002, 35, 150), ric)
    assert bits_equal(S.wavelet(S.WAVELET_AFD, 2000, 0.0005, 28.0), ol.wavelet_afd(2000, 0.0005, 28.0))
    q = S.wavelet(S.WAVELET_Q, 500, 0.001, 10.0)
    b = np.float32(3.1415926) * np.float32(10.0) * (np.arange(1, 501, dtype=np.float32) * np.float32(0.001)
                                                    - np.float32(1.2) / np.float32(10.0))
    np.testing.assert_allclose(q, np.exp(-(b * b)) * (1 - 2 * (b * b)), rtol=0, atol=2e-7)


@pytest.mark.parametrize("nx,nz,pml", [(140, 140, 20), (120, 90, 15), (351, 351, 50), (60, 200, 10)])
def test_sponge_matches_oracle(nx, nz, pml):
    assert bits_equal(S.afd_sponge(nx, nz, pml), ol.afd_sponge(nx, nz, pml))


@pytest.mark.parametrize("order", [16, 10, 8, 4, 2])
def test_coefficients_match_oracle(order):
    assert bits_equal(S.fd_coeffs(order), ol.afd_coeffs(order // 2))


def test_pad_model_edge_replication():
    a = np.arange(12, dtype=np.float32).reshape(3, 4)
    p = S.pad_model(a, 2, 1, 1, 3)
    np.testing.assert_array_equal(p, np.pad(a, ((2, 1), (1, 3)), mode="edge"))


def test_helpers_reject_bad_arguments():
    lib = S.load()
    out = np.zeros(10, np.float32)
    assert lib.sfd_wavelet(9, 10, 0.001, 10.0, 0, S._fp(out)) == S.ERR_ARG
    assert lib.sfd_wavelet(S.WAVELET_RIC, 10, 0.001, -1.0, 0, S._fp(out)) == S.ERR_ARG
    assert lib.sfd_fd_coeffs(7, S._fp(out)) == S.ERR_ARG
    assert lib.sfd_afd_sponge(10, 10, 6, S._fp(out)) == S.ERR_ARG


@pytest.mark.parametrize("kw", [dict(nx=0), dict(order=7), dict(dt=0.0), dict(pml=-1), dict(pml=200),
                                dict(scheme=9), dict(nx=10, order=16)])
def test_create_rejects_bad_grid(kw):
    args = dict(scheme=S.ACOUSTIC_2D, nx=100, nz=100, pml=20, dx=10.0, dz=10.0, dt=1e-3, order=16)
    args.update(kw)
    g = S.Grid(args["scheme"], args["nx"], 1, args["nz"], args["pml"], args["dx"], 0.0, args["dz"], args["dt"],
               args["order"], 0, 0.0)
    h = ctypes.c_void_p()
    assert S.load().sfd_create(ctypes.byref(g), 0, ctypes.byref(h)) == S.ERR_ARG
    assert not h.value


def test_null_context_is_rejected():
    lib = S.load()
    assert lib.sfd_forward(None, None) == S.ERR_ARG
    assert lib.sfd_set_model(None, None, None, None) == S.ERR_ARG
    assert lib.sfd_destroy(None) == S.OK


def test_noalloc_rejects_sizes_beyond_its_array_before_any_device_work():
    """sfd_forward_noalloc checks the grid against its fixed 32 MiB array before touching the
    device (the pointers below are never dereferenced)."""
    g = S.Grid(S.ACOUSTIC_2D, 3000, 1, 3000, 20, 10.0, 0.0, 10.0, 1e-3, 16, S.EXACT, 0.0)
    rx = np.zeros(1, np.int32)
    fake = ctypes.c_void_p(256)
    lib = S.load()
    assert lib.sfd_forward_noalloc(ctypes.byref(g), fake, None, fake, 10, 5, 5, 1, S._ip(rx), S._ip(rx), fake,
                                   None) == S.ERR_NOMEM
    assert lib.sfd_forward_noalloc(ctypes.byref(g), None, None, fake, 10, 5, 5, 1, S._ip(rx), S._ip(rx), fake,
                                   None) == S.ERR_ARG
