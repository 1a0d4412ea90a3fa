"""Shot sharding over GPUs and the gradient all-reduce.

The reference distributes shots round-robin over MPI ranks, one process per rank
(forward/Q_forward/Q_multishot_fd_main_fsbc_zy_rotated.f90:124-141: rank r models shots
r, r + size, r + 2 size, ...).  Here one process drives one GPU: each rank models its own
shots in one batched launch (no data-path collective for the forward), and for the gradient each
rank's partial sum over its shots is added across ranks by one all-reduce (sum) of the
d misfit / d vp field, the d misfit / d (1/Q) field when present and the misfit, issued in one
coalesced group over torch.distributed (NCCL over NVLink between GPUs, gloo on the host).  On
GPUs the gradient stays in device memory: sfd_gradient_device writes it into torch tensors and
NCCL reduces them in place (sharded_gradient_device); allreduce_gradient is the host-array form.
"""
from typing import List, Optional, Sequence, Tuple

import numpy as np


def shard_shots(nshot: int, rank: int, world: int) -> List[int]:
    """Indices of the shots rank `rank` of `world` models, round-robin as QM:124-141."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return list(range(rank, nshot, world))


def split_records(records: np.ndarray, sizes: Sequence[int]) -> List[np.ndarray]:
    """Cut a flat record buffer (shots concatenated in order) into per-shot pieces."""
    offs = np.concatenate([[0], np.cumsum(sizes)])
    if offs[-1] != records.size:
        raise ValueError(f"records hold {records.size} values, the shots {offs[-1]}")
    return [records[offs[i]:offs[i + 1]] for i in range(len(sizes))]


def gather_local_records(records: np.ndarray, sizes: Sequence[int], local: Sequence[int]) -> np.ndarray:
    """The records of the shots in `local`, concatenated in that order (the layout of an engine
    whose shot list is `local`)."""
    parts = split_records(records, sizes)
    return np.concatenate([parts[i] for i in local]) if local else np.zeros(0, records.dtype)


def allreduce_gradient_tensors(misfit, grad_vp, grad_invq=None, group=None):
    """Sum the per-rank misfit and gradient tensors over the process group in place, where they
    live: CUDA tensors written by Engine.gradient_device are reduced by NCCL on the device (no
    host copy of the gradient); CPU tensors by gloo.  One coalesced group of all-reduces."""
    import torch.distributed as dist
    tensors = [t for t in (misfit, grad_vp, grad_invq) if t is not None]
    works = [dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group, async_op=True) for t in tensors]
    for w in works:
        w.wait()
    return misfit, grad_vp, grad_invq


def sharded_gradient_device(engine, obs_dev, grad_shape, want_invq=False, group=None):
    """One rank's part of a sharded gradient, kept on its GPU: the engine (holding this rank's
    shots) writes the misfit and gradient of its shots into device tensors (sfd_gradient_device),
    which are then summed over the ranks by NCCL in place.  obs_dev: this rank's observed records
    as a CUDA float32 tensor.  Returns (misfit, grad_vp, grad_invq) as device tensors."""
    import torch
    dev = obs_dev.device
    misfit = torch.zeros(1, dtype=torch.float32, device=dev)
    gvp = torch.empty(grad_shape, dtype=torch.float32, device=dev)
    gq = torch.empty(grad_shape, dtype=torch.float32, device=dev) if want_invq else None
    torch.cuda.synchronize(dev)  # obs_dev is complete before the library's stream reads it
    engine.gradient_device(obs_dev.data_ptr(), misfit.data_ptr(), gvp.data_ptr(), gq.data_ptr() if gq is not None else None)
    return allreduce_gradient_tensors(misfit, gvp, gq, group=group)


def allreduce_gradient(misfit: float, grad_vp: np.ndarray, grad_invq: Optional[np.ndarray] = None,
                       device: Optional[str] = None, group=None) -> Tuple[float, np.ndarray, Optional[np.ndarray]]:
    """Sum the per-rank misfit and gradients over the process group.  The fields travel as one
    float32 buffer per tensor (misfit in float64) in one coalesced all-reduce; `device` is the
    torch device of the collective ("cuda:k" for NCCL, "cpu" for gloo)."""
    import torch
    import torch.distributed as dist
    dev = torch.device(device or ("cuda" if torch.cuda.is_available() else "cpu"))
    tensors = [torch.tensor([misfit], dtype=torch.float64, device=dev),
               torch.from_numpy(np.ascontiguousarray(grad_vp, np.float32)).to(dev)]
    if grad_invq is not None:
        tensors.append(torch.from_numpy(np.ascontiguousarray(grad_invq, np.float32)).to(dev))
    works = [dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group, async_op=True) for t in tensors]
    for w in works:
        w.wait()
    out_q = tensors[2].cpu().numpy().reshape(grad_invq.shape) if grad_invq is not None else None
    return float(tensors[0].item()), tensors[1].cpu().numpy().reshape(grad_vp.shape), out_q
