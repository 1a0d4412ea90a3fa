"""sfd_gradient_device: the gradient with every buffer in the caller's device memory (torch
tensors here), against sfd_gradient with host buffers -- bit for bit, for the 2-D acoustic scheme
(several shots with apertures, variable density), the viscoacoustic scheme (d/dvp and d/d(1/Q))
and the 3-D scheme; and the sharded form (sharding.sharded_gradient_device) through a one-rank
NCCL group, whose in-place all-reduce leaves the values unchanged."""
import datetime
import os
import socket

import numpy as np
import pytest

from conftest import bits_equal
from seismic_code_github_b200 import seisfd as S
from seismic_code_github_b200 import sharding as SH
from seismic_code_github_b200 import workloads as W

pytestmark = pytest.mark.gpu


def device_gradient(e, obs, shape, want_invq=False):
    import torch
    dev = torch.device("cuda:0")
    o = torch.from_numpy(np.ascontiguousarray(obs, np.float32).reshape(-1)).to(dev)
    mis = torch.full((1,), float("nan"), dtype=torch.float32, device=dev)
    g = torch.full(shape, float("nan"), dtype=torch.float32, device=dev)
    gq = torch.full(shape, float("nan"), dtype=torch.float32, device=dev) if want_invq else None
    torch.cuda.synchronize()
    e.gradient_device(o.data_ptr(), mis.data_ptr(), g.data_ptr(), gq.data_ptr() if want_invq else None)
    return float(mis.item()), g.cpu().numpy(), (gq.cpu().numpy() if want_invq else None)


def test_acoustic_2d_device_equals_host():
    case = W.small_varden()
    rx, rz = case.receivers()
    w = S.wavelet(S.WAVELET_RIC, 150, case.dt, case.f0, 40)
    shots = [S.ShotSpec(case.src_x[0], case.src_z[0], rx, rz, w),
             S.ShotSpec(case.src_x[0] - 10, case.src_z[0] + 6, rx, rz, w),
             S.ShotSpec(20, 14, rx[:40] - 10, rz[:40], w[:110], ap_x0=10, ap_nx=80)]
    with S.Engine(S.ACOUSTIC_2D, case.Nx, case.Nz, case.dx, case.dz, case.dt, case.PML, order=16) as e:
        e.set_model((case.vp * 1.02).astype(np.float32), case.den)
        e.set_shots(shots)
        obs = e.forward().copy()
        e.set_model(case.vp, case.den)
        e.set_checkpoint_interval(17)
        mh, gh, _ = e.gradient(obs)
        md, gd, _ = device_gradient(e, obs, gh.shape)
        md2, gd2, _ = device_gradient(e, obs, gh.shape)  # a second call on the same context
    assert np.abs(gh).max() > 0
    assert mh == md == md2
    assert bits_equal(gd, gh) and bits_equal(gd2, gh)


def test_viscoacoustic_device_equals_host():
    rng = np.random.default_rng(3)
    nx, nz, npx, dt, f0 = 60, 48, 10, 5e-4, 20.0
    vp = S.pad_model((2000.0 + 40.0 * rng.standard_normal((nx, nz))).astype(np.float32), npx, npx, npx, npx)
    rho = S.pad_model(np.full((nx, nz), 2100.0, np.float32), npx, npx, npx, npx)
    q = S.pad_model((30.0 + 50.0 * rng.random((nx, nz))).astype(np.float32), npx, npx, npx, npx)
    rx = np.arange(npx, vp.shape[0] - npx, dtype=np.int32)
    rz = np.full_like(rx, npx + 2)
    shots = [S.ShotSpec(npx + 15 + 12 * i, npx + 3, rx, rz, S.wavelet(S.WAVELET_Q, 220 - 40 * i, dt, f0))
             for i in range(2)]
    with S.Engine(S.VISCOAC_2D, vp.shape[0], vp.shape[1], 10.0, 10.0, dt, npx, order=10, f0=f0) as e:
        e.set_model((vp * 1.02).astype(np.float32), rho, q)
        e.set_shots(shots)
        obs = e.forward().copy()
        e.set_model(vp, rho, q)
        mh, gh, gqh = e.gradient(obs, want_invq=True)
        md, gd, gqd = device_gradient(e, obs, gh.shape, want_invq=True)
    assert np.abs(gh).max() > 0 and np.abs(gqh).max() > 0
    assert mh == md and bits_equal(gd, gh) and bits_equal(gqd, gqh)


def test_acoustic_3d_device_equals_host():
    n, pml, dt = 48, 8, 1e-3
    z = np.arange(n)
    vp = np.empty((n, n, n), np.float32)
    vp[:] = (1800.0 + 900.0 * z / n)[None, None, :]
    w = S.wavelet(S.WAVELET_RIC, 70, dt, 20.0, 30)
    r = np.arange(pml, n - pml, 3, dtype=np.int32)
    shots = [S.ShotSpec(n // 2, pml + 3, r, np.full_like(r, pml + 2), w, sy=n // 2 - 4 + 8 * i, rec_y=r)
             for i in range(2)]
    with S.Engine(S.ACOUSTIC_3D, n, n, 10.0, 10.0, dt, pml, order=8, ny=n, dy=10.0) as e:
        e.set_model((vp * 1.03).astype(np.float32))
        e.set_shots(shots)
        obs = e.forward().copy()
        e.set_model(vp)
        mh, gh, _ = e.gradient(obs)
        md, gd, _ = device_gradient(e, obs, gh.shape)
    assert np.abs(gh).max() > 0
    assert mh == md and bits_equal(gd, gh)


def test_sharded_device_gradient_one_rank_nccl():
    import torch
    import torch.distributed as dist
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        case = W.small_varden()
        rx, rz = case.receivers()
        w = S.wavelet(S.WAVELET_RIC, 120, case.dt, case.f0, 40)
        with S.Engine(S.ACOUSTIC_2D, case.Nx, case.Nz, case.dx, case.dz, case.dt, case.PML, order=16) as e:
            e.set_model((case.vp * 1.02).astype(np.float32), case.den)
            e.set_shots([S.ShotSpec(case.src_x[0], case.src_z[0], rx, rz, w)])
            obs = e.forward().copy()
            e.set_model(case.vp, case.den)
            mh, gh, _ = e.gradient(obs)
            mt, gt, _ = SH.sharded_gradient_device(e, torch.from_numpy(obs).cuda(), gh.shape)
            torch.cuda.synchronize()
        assert gt.is_cuda and float(mt.item()) == mh
        assert bits_equal(gt.cpu().numpy(), gh)
    finally:
        dist.destroy_process_group()
