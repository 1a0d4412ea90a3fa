"""Multi-GPU plumbing on the host: round-robin shot sharding (forward/Q_forward/
Q_multishot_fd_main_fsbc_zy_rotated.f90:124-141) and the gradient all-reduce, run as two gloo ranks
on CPU.  Each rank sums the FP64 oracle gradients of its own shots; after the all-reduce every rank
holds the gradient of the whole shot set, equal to the serial sum to float32 round-off."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle_lib as ol
from conftest import rel_l2
from seismic_code_github_b200 import sharding as SH
from seismic_code_github_b200 import workloads as W


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_round_robin_shards_cover_every_shot_once(world):
    for nshot in range(0, 21):
        seen = []
        for r in range(world):
            mine = SH.shard_shots(nshot, r, world)
            assert all(i % world == r for i in mine)
            seen += mine
        assert sorted(seen) == list(range(nshot))
    with pytest.raises(ValueError):
        SH.shard_shots(4, 2, 2)


def test_local_record_gather():
    sizes = [3, 5, 2, 4]
    rec = np.arange(sum(sizes), dtype=np.float32)
    parts = SH.split_records(rec, sizes)
    assert [p.size for p in parts] == sizes
    loc = SH.gather_local_records(rec, sizes, [1, 3])
    assert np.array_equal(loc, np.concatenate([parts[1], parts[3]]))


def small_problem(nshot=5):
    NX, NZ, PML, nt = 36, 28, 8, 90
    vp = W.pad_edges(W.layered_model(NX, NZ, 3, 1800.0, 2600.0, seed=3, anomalies=1, radius=5.0, amp=150.0), PML,
                     PML)
    den = np.full(vp.shape, 2100.0, np.float32)
    Nx, Nz = vp.shape
    rx = np.arange(PML, Nx - PML, 2, dtype=np.int32)
    rz = np.full_like(rx, PML + 2)
    w = ol.wavelet_ric(nt, 1e-3, 25, 30)
    srcs = [(PML + 4 + 5 * i, PML + 3) for i in range(nshot)]
    obs = []
    for sx, sz in srcs:
        rec, _, _ = ol.afd_forward(Nx, Nz, PML, nt, 10.0, 10.0, 1e-3, (vp * 1.03).astype(np.float32), den, w, sx, sz,
                                   rx, rz, radius=4, fp64=True)
        obs.append(rec.astype(np.float32))
    return dict(Nx=Nx, Nz=Nz, PML=PML, nt=nt, vp=vp, den=den, w=w, srcs=srcs, rx=rx, rz=rz, obs=obs)


def shot_gradients(p, shots):
    J, g = 0.0, np.zeros(p["vp"].shape)
    for i in shots:
        sx, sz = p["srcs"][i]
        j, gs, _, _ = ol.afd_gradient_f64(p["Nx"], p["Nz"], p["PML"], p["nt"], 10.0, 10.0, 1e-3, p["vp"], p["den"],
                                          p["w"], sx, sz, p["rx"], p["rz"], p["obs"][i], radius=4)
        J += j
        g += gs
    return J, g


def _rank(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        p = small_problem()
        mine = SH.shard_shots(len(p["srcs"]), rank, world)
        J, g = shot_gradients(p, mine)
        Jt, gt, _ = SH.allreduce_gradient(J, g.astype(np.float32), device="cpu")
        np.save(os.path.join(out_dir, f"g{rank}.npy"), gt)
        np.save(os.path.join(out_dir, f"J{rank}.npy"), np.array([Jt]))
    finally:
        dist.destroy_process_group()


def rank_payload(rank):
    """A rank's partial misfit and gradient for the tensor all-reduce test (seeded per rank)."""
    rng = np.random.default_rng(100 + rank)
    return float(rng.random()), rng.standard_normal((44, 36)).astype(np.float32)


def _rank_tensors(rank, world, port, out_dir):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        J, g = rank_payload(rank)
        mis = torch.tensor([J], dtype=torch.float32)
        gv = torch.from_numpy(g.copy())
        gq = torch.from_numpy(2.0 * g)
        out = SH.allreduce_gradient_tensors(mis, gv, gq)
        assert out[1] is gv  # reduced in place
        np.save(os.path.join(out_dir, f"t{rank}.npy"), np.stack([gv.numpy(), gq.numpy()]))
        np.save(os.path.join(out_dir, f"m{rank}.npy"), mis.numpy())
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_gradient_allreduce_two_gloo_ranks(tmp_path):
    world = 2
    mp.spawn(_rank, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True)
    p = small_problem()
    J, g = shot_gradients(p, range(len(p["srcs"])))
    for r in range(world):
        gr = np.load(tmp_path / f"g{r}.npy")
        Jr = float(np.load(tmp_path / f"J{r}.npy")[0])
        assert abs(Jr - J) <= 1e-12 * J
        assert rel_l2(gr, g) <= 1e-6


def test_tensor_allreduce_two_gloo_ranks(tmp_path):
    """The in-place tensor form used on GPUs (sharding.allreduce_gradient_tensors, which NCCL runs
    on device tensors) with CPU tensors over gloo: every rank ends with the sums."""
    world = 2
    mp.spawn(_rank_tensors, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True)
    parts = [rank_payload(r) for r in range(world)]
    J = sum(p[0] for p in parts)
    g = sum(p[1].astype(np.float64) for p in parts)
    for r in range(world):
        t = np.load(tmp_path / f"t{r}.npy")
        assert rel_l2(t[0], g) <= 1e-6 and rel_l2(t[1], 2.0 * g) <= 1e-6
        assert abs(float(np.load(tmp_path / f"m{r}.npy")[0]) - J) <= 1e-6 * J
