"""CPU checks of the file contract helpers (seismic_code_github_b200/csrc/fileio.cpp): the
Q_forward parameter card reader (QS:121-234), the yang_version card reader (YPUB:48-145), the VTI
modeller's card reader (VS:342-425), the SU shot writer (QS:1476-1546, YPUB:1533-1604 without the
cdp word, VS:163-217 without cdp and offset), the merge (QS:1550-1624) and the raw float32 files.  The expected SU headers are built here from the
Fortran statements of QS:1502-1533 with numpy float32 arithmetic."""
import ctypes
import os
import struct

import numpy as np
import pytest

from conftest import REFERENCE, ROOT
from seismic_code_github_b200 import seisfd as S

CARD = """!*P-wave velocity filename*!
{d}/vp.bin
!*S-wave velocity filename*!
{d}/vs.bin
!*Density velocity filename*!
{d}/rho.bin
!*P-wave quality factor filename*!
{d}/qp.bin
!*S-wave quality factor filename*!
{d}/qs.bin
!*NO.1 shot record filename(tmp)*!
{d}/pz_tmp
!*NO.2 shot record filename(all)*!
{d}/shot_pz
!*NO.3 shot record filename(tmp)*!
{d}/px_tmp
!*NO.4 shot record filename(all)*!
{d}/shot_px
!*nshot(samples)*!
3
!*offset_min,offset_max*!
-150.0  250.0
!*sx0,sz0,rz0(m)*!
200.0 10.0 20.0
!*dsx(m)*!
50.0
!*nx_v,nz_v(samples)*!
120 80
!*dx_v,dz_v(m)*!
10.0 10.0
!*nt(samples)*!
500
!*dt(s)*!
0.001
!*f0(Hz)*!
15
!*pml_thick x left and right direction(m)*!
100.0 100.0
!*pml_thick z up and down direction(m)*!
100.0 100.0
!*order_2nd*!
10
!*order_1st*!
9
"""


@pytest.mark.parametrize("eol", ["\n", "\r\n"])
def test_parameter_card(tmp_path, eol):
    p = tmp_path / "card.par"
    p.write_bytes(CARD.format(d=str(tmp_path)).replace("\n", eol).encode())
    q = S.read_qpar(str(p))
    assert q.vp.decode() == f"{tmp_path}/vp.bin" and q.shot4.decode() == f"{tmp_path}/shot_px"
    assert (q.nshot, q.nx, q.nz, q.nt, q.fdo2, q.fdo1) == (3, 120, 80, 500, 10, 9)
    assert (q.offset_min, q.offset_max, q.sx0, q.sz0, q.rz0, q.dsx) == (-150.0, 250.0, 200.0, 10.0, 20.0, 50.0)
    assert (q.dx, q.dz, q.f0) == (10.0, 10.0, 15.0) and np.float32(q.dt) == np.float32(0.001)
    assert (q.pml_xn, q.pml_xp, q.pml_zn, q.pml_zp) == (100.0, 100.0, 100.0, 100.0)


def test_reference_parameter_card():
    """The card shipped with the reference (forward/Q_forward/isoq_2d_modelling_simple.par)."""
    path = os.path.join(REFERENCE, "forward/Q_forward/isoq_2d_modelling_simple.par")
    if not os.path.exists(path):
        pytest.skip("reference tree not present")
    q = S.read_qpar(path)
    assert q.vp.decode() == "./model/vp2d_2l.dat" and q.shot2.decode() == "./shot_vz"
    assert (q.nshot, q.nx, q.nz, q.nt, q.f0, q.dsx) == (1, 401, 401, 2000, 10.0, 10.0)
    assert (q.offset_min, q.offset_max, q.pml_xn, q.pml_zp) == (0.0, 50.0, 200.0, 200.0)


def test_card_errors(tmp_path):
    assert S.load().sfd_qpar_read(str(tmp_path / "missing.par").encode(), None) == S.ERR_ARG
    p = tmp_path / "short.par"
    p.write_text("\n".join(CARD.format(d="x").splitlines()[:25]))
    with pytest.raises(S.SfdError):
        S.read_qpar(str(p))


def expected_header(shot_no, isx, ixmin, dx, dt, nt, i):
    f32 = np.float32
    sx = int(f32(isx - 1) * f32(dx))  # real(4) product, truncated on assignment
    gx = int(f32(ixmin - 1 + i - 1) * f32(dx))
    q = f32(gx + sx) / f32(dx)
    cdp = int(np.floor(abs(q) + 0.5)) * (1 if q >= 0 else -1) + 1  # nint: halves away from zero
    h = bytearray(240)
    struct.pack_into("<i", h, 8, shot_no)
    struct.pack_into("<i", h, 20, cdp)
    struct.pack_into("<h", h, 28, 1)
    struct.pack_into("<i", h, 36, gx - sx)
    struct.pack_into("<i", h, 72, sx)
    struct.pack_into("<i", h, 80, gx)
    struct.pack_into("<h", h, 114, nt)
    struct.pack_into("<h", h, 116, int(f32(dt) * f32(1.0e6)))
    return bytes(h)


@pytest.mark.parametrize("isx,ixmin,dx", [(21, 6, 10.0), (1, -4, 12.5), (300, 301, 3.3)])
def test_su_shot_file(tmp_path, isx, ixmin, dx):
    nt, ntr = 37, 9
    tr = np.random.default_rng(0).standard_normal((ntr, nt)).astype(np.float32)
    path = str(tmp_path / "shot7.su")
    S.su_write(path, tr, 7, isx, ixmin, dx, 0.0005)
    raw = open(path, "rb").read()
    assert len(raw) == ntr * (240 + 4 * nt)  # records of nt + 60 four-byte words
    for i in range(1, ntr + 1):
        rec = raw[(i - 1) * (240 + 4 * nt):i * (240 + 4 * nt)]
        assert rec[:240] == expected_header(7, isx, ixmin, dx, 0.0005, nt, i), i
        assert np.array_equal(np.frombuffer(rec[240:], np.float32), tr[i - 1])


def test_su_merge_and_delete(tmp_path):
    parts = []
    for s in range(3):
        p = str(tmp_path / f"pz_tmp{s + 1}.su")
        S.su_write(p, np.full((4, 10), s, np.float32), s + 1, 10 + s, 5, 10.0, 0.001)
        parts.append(p)
    blobs = [open(p, "rb").read() for p in parts]
    S.su_merge(str(tmp_path / "keep.su"), parts, delete_inputs=False)
    assert open(tmp_path / "keep.su", "rb").read() == b"".join(blobs)
    assert all(os.path.exists(p) for p in parts)
    S.su_merge(str(tmp_path / "all.su"), parts)
    assert open(tmp_path / "all.su", "rb").read() == b"".join(blobs)
    assert not any(os.path.exists(p) for p in parts)


def test_raw_float_files(tmp_path):
    lib = S.load()
    a = np.arange(12, dtype=np.float32)
    p = str(tmp_path / "a.dat").encode()
    assert lib.sfd_write_floats(p, S._fp(a), 12, 0) == S.OK
    assert lib.sfd_write_floats(p, S._fp(a), 5, 1) == S.OK
    b = np.empty(17, np.float32)
    assert lib.sfd_read_floats(p, 17, S._fp(b)) == S.OK
    assert np.array_equal(b, np.concatenate([a, a[:5]]))
    assert lib.sfd_read_floats(p, 18, S._fp(np.empty(18, np.float32))) == S.ERR_IO


ISOCARD = """!*Modeling mode:fsbc(free surface bc).or.abc(absorbing bc)*!
{mode}
!*P-wave velocity filename*!
{d}/vp.bin
!*S-wave velocity filename*!
{d}/vs.bin
!*Density velocity filename*!
{d}/rho.bin
!*Topography velocity filename*!
{d}/topo.bin
!*Vx snapshot  filename*!
{d}/snap/vx_
!*Vz snapshot filename*!
{d}/snap/vz_
!*NO.1 shot record filename(tmp)*!
{d}/vx_tmp
!*NO.2 shot record filename(all)*!
{d}/shot_vx
!*NO.3 shot record filename(tmp)*!
{d}/vz_tmp
!*NO.4 shot record filename(all)*!
{d}/shot_vz
!*nshot(samples)*!
3
!*offset_min,offset_max*!
-150.0  250.0
!*sx0,sz0,rz0(m)*!
200.0 30.0 10.0
!*dsx(m)*!
50.0
!*nx_v,nz_v(samples)*!
120 80
!*dx_v,dz_v(m)*!
10.0 10.0
!*nt(samples)*!
300
!*dt(s),desnap(s)*!
0.0005 0.025
!*f0(Hz)*!
20.0
!*decay(s) recommending decay=(1.2/f0)s*!
0.02
!*pml_thick x left and right direction(m)*!
90.0 90.0
!*pml_thick z up and down direction(m)*!
{ztop} 90.0
!*rad of gauss smooth*!
{rgau}
"""


def test_yang_parameter_card(tmp_path):
    p = tmp_path / "iso.par"
    p.write_text(ISOCARD.format(d=str(tmp_path), mode="fsbc", ztop="0000.0", rgau=12))
    q = S.read_isopar(str(p))
    assert q.molmod.decode() == "fsbc" and q.topo.decode() == f"{tmp_path}/topo.bin"
    assert q.snapz.decode() == f"{tmp_path}/snap/vz_" and q.shot4.decode() == f"{tmp_path}/shot_vz"
    assert (q.nshot, q.nx, q.nz, q.nt, q.rgau) == (3, 120, 80, 300, 12)
    assert (q.offset_min, q.offset_max, q.sx0, q.sz0, q.rz0, q.dsx) == (-150.0, 250.0, 200.0, 30.0, 10.0, 50.0)
    assert np.float32(q.dt) == np.float32(0.0005) and np.float32(q.dtsnap) == np.float32(0.025)
    assert (q.f0, np.float32(q.decay)) == (20.0, np.float32(0.02))
    assert (q.pml_xn, q.pml_xp, q.pml_zn, q.pml_zp) == (90.0, 90.0, 0.0, 90.0)


def test_reference_yang_parameter_card():
    """The card shipped with the reference (forward/yang_version_2016_2_2/iso_2d_modelling_sin_test.par)."""
    path = os.path.join(REFERENCE, "forward/yang_version_2016_2_2/iso_2d_modelling_sin_test.par")
    if not os.path.exists(path):
        pytest.skip("reference tree not present")
    q = S.read_isopar(path)
    assert q.molmod.decode() == "fsbc" and q.shot1.decode().endswith("/vx_tmp")
    assert (q.nshot, q.nx, q.nz, q.nt, q.rgau) == (1, 501, 401, 3001, 50)
    assert (q.offset_min, q.offset_max, q.sx0, q.dsx, q.dx, q.f0) == (-1250.0, 1250.0, 1250.0, 100.0, 5.0, 25.0)
    assert np.float32(q.decay) == np.float32(0.048) and np.float32(q.dtsnap) == np.float32(0.01)
    assert (q.pml_xn, q.pml_xp, q.pml_zn, q.pml_zp) == (1000.0, 1000.0, 0.0, 1000.0)


def test_su_without_cdp(tmp_path):
    nt, ntr = 21, 5
    tr = np.random.default_rng(1).standard_normal((ntr, nt)).astype(np.float32)
    path = str(tmp_path / "shot3.su")
    S.su_write(path, tr, 3, 40, 12, 5.0, 0.001, flags=0)
    raw = open(path, "rb").read()
    for i in range(1, ntr + 1):
        rec = raw[(i - 1) * (240 + 4 * nt):i * (240 + 4 * nt)]
        want = bytearray(expected_header(3, 40, 12, 5.0, 0.001, nt, i))
        want[20:24] = b"\0\0\0\0"  # YPUB:1555-1572 never sets cdp
        assert rec[:240] == bytes(want), i


# A VTI modeller card in the layout of VS:383-421 (label line, value line), values of this test.
VTICARD = """!*velocity filename*!
{d}/vz.bin
!*epsilon filename*!
{d}/eps.bin
!*delta filename*!
{d}/delta.bin
!*NO.1 shot record filename(tmp)*!
{d}/vti_tmp
!*NO.2 shot record filename(all)*!
{d}/vti_all
!*nshot(samples)*!
3
!*offset_min,offset_max*!
-300  295.0
!*sx0,sz0,rz0(m)*!
100.0 0.0 0.0
!*dsx(m)*!
50.0
!*nx_v,nz_v(samples)*!
{nx} {nz}
!*dx_v,dz_v(m)*!
5.0 5.0
!*nt(samples)*!
{nt}
!*dt(s)*!
0.0005
!*f0(Hz)*!
30.0
!*pml_thick x left and right direction(m)*!
100.0 100.0
!*pml_thick z up and down direction(m)*
0.0 100.0
!*fd_order_explicit*!
10
!*order_pml_1st*!
9
!*order_pml_2nd*!
10
"""


def test_vti_card_reader(tmp_path):
    (tmp_path / "vti.par").write_text(VTICARD.format(d="/data", nx=300, nz=200, nt=10000))
    p = S.VtiCardFields()
    assert S.load().sfd_vtipar_read(str(tmp_path / "vti.par").encode(), ctypes.byref(p)) == 0
    assert p.vz.decode() == "/data/vz.bin" and p.delta.decode() == "/data/delta.bin"
    assert p.shot1.decode() == "/data/vti_tmp" and p.shot2.decode() == "/data/vti_all"
    assert (p.nshot, p.nx_v, p.nz_v, p.nt) == (3, 300, 200, 10000)
    assert (p.offset_min, p.offset_max, p.sx0, p.dsx) == (-300.0, 295.0, 100.0, 50.0)
    assert np.float32(p.dt) == np.float32(0.0005) and p.f0 == 30.0
    assert (p.bound_x_l, p.bound_x_r, p.bound_z_u, p.bound_z_d) == (100.0, 100.0, 0.0, 100.0)
    assert (p.order_explicit, p.order_pml_1st, p.order_pml_2nd) == (10, 9, 10)
    (tmp_path / "short.par").write_text("\n".join(VTICARD.splitlines()[:20]))
    assert S.load().sfd_vtipar_read(str(tmp_path / "short.par").encode(), ctypes.byref(p)) != 0


def test_su_without_offset(tmp_path):
    """The VTI modeller's writer (VS:184-214) sets fldr, trid, sx, gx, ns and dt only."""
    nt, ntr = 17, 4
    tr = np.random.default_rng(2).standard_normal((ntr, nt)).astype(np.float32)
    path = str(tmp_path / "shot2.su")
    S.su_write(path, tr, 2, 61, -239, 5.0, 0.0005, flags=S.SU_NO_OFFSET)
    raw = open(path, "rb").read()
    for i in range(1, ntr + 1):
        rec = raw[(i - 1) * (240 + 4 * nt):i * (240 + 4 * nt)]
        want = bytearray(expected_header(2, 61, -239, 5.0, 0.0005, nt, i))
        want[20:24] = b"\0\0\0\0"
        want[36:40] = b"\0\0\0\0"
        assert rec[:240] == bytes(want), i


def test_programs_are_built():
    for name in ("afd_fd", "q_forward", "iso_forward", "vti_forward"):
        assert os.access(os.path.join(ROOT, "seismic_code_github_b200", "bin", name), os.X_OK)
