"""Runs the reference's own AFD executable (built by oracle/ref_build.py) on a configuration.

Test infrastructure and CPU-baseline timing only: nothing in the product imports this.

The executable writes to ../file/{record,Snap,Model,Pall}.dat relative to its working
directory (forward/Acoustic_FD_by_ss/src/Acoustic_1order_FD.cpp:146,347,361,386), so each run
gets a private <tmp>/bin + <tmp>/file pair.
"""
import os
import resource
import shutil
import subprocess
import tempfile
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def ric_wavelet(nt: int, dt: float, f0: float, delay: int = 150) -> np.ndarray:
    """The Ricker trace of tools/ricker.cpp:44 (pi = 3.1415926, integer frequency, double
    arithmetic, delay in samples), rounded to float32: the wavelet fed to the reference build."""
    pi = 3.1415926
    j = np.arange(nt, dtype=np.float64)
    a = pi * float(int(f0)) * (j - delay) * np.float64(np.float32(dt))
    return ((1 - 2 * a * a) * np.exp(-a * a)).astype(np.float32)


def ref_binary(name: str = "afd_ref") -> str:
    return os.path.join(REF_DIR, name)


def available(name: str = "afd_ref") -> bool:
    return os.access(ref_binary(name), os.X_OK)


@dataclass
class AfdRefConfig:
    """Parameters of the patched reference (oracle/ref_build.py). Grid sizes are AFD's
    NX/NZ (interior) and PML; the padded grid is (NX+2*PML) x (NZ+2*PML)."""
    NX: int = 100
    NZ: int = 100
    PML: int = 20
    Nt: int = 2000
    dx: float = 10.0
    dz: float = 10.0
    dt: float = 0.0005
    vp: Optional[np.ndarray] = None       # padded (Nx, Nz) f32, x-major
    den: Optional[np.ndarray] = None      # padded (Nx, Nz) f32
    wavelet: Optional[np.ndarray] = None  # (Nt,) f32
    sx: Optional[int] = None              # padded source cell
    sz: Optional[int] = None
    rec_z: int = -1                       # >=0: horizontal receiver line at this padded z
    snap: int = 500
    pall: bool = False
    extra_env: dict = field(default_factory=dict)


def _raise_stack():
    # AFD keeps absorb[Nx][Nz] and signal[Nt] on the stack (AFD:47,199)
    try:
        resource.setrlimit(resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
    except (ValueError, OSError):
        pass


def launch(cfg: AfdRefConfig, workdir: str, binary: str = "afd_ref") -> subprocess.Popen:
    """Start one run in `workdir` (created) and return the process."""
    bindir = os.path.join(workdir, "bin")
    os.makedirs(bindir, exist_ok=True)
    os.makedirs(os.path.join(workdir, "file"), exist_ok=True)
    env = dict(os.environ)
    env.update({
        "AFD_NX": str(cfg.NX), "AFD_NZ": str(cfg.NZ), "AFD_PML": str(cfg.PML),
        "AFD_NT": str(cfg.Nt), "AFD_DX": repr(float(cfg.dx)), "AFD_DZ": repr(float(cfg.dz)),
        "AFD_DT": repr(float(cfg.dt)), "AFD_SNAP": str(cfg.snap),
        "AFD_PALL": "1" if cfg.pall else "0", "AFD_REC_Z": str(cfg.rec_z),
    })
    if cfg.sx is not None:
        env["AFD_SX"] = str(cfg.sx)
    if cfg.sz is not None:
        env["AFD_SZ"] = str(cfg.sz)
    for key, arr, name in (("AFD_VP_FILE", cfg.vp, "vp.bin"), ("AFD_DEN_FILE", cfg.den, "den.bin"),
                           ("AFD_WAVELET_FILE", cfg.wavelet, "wavelet.bin")):
        if arr is not None:
            fn = os.path.join(workdir, name)
            np.ascontiguousarray(arr, dtype=np.float32).tofile(fn)
            env[key] = fn
    env.update(cfg.extra_env)
    return subprocess.Popen([ref_binary(binary)], cwd=bindir, env=env, stdout=subprocess.DEVNULL,
                            stderr=subprocess.PIPE, preexec_fn=_raise_stack)


def collect(cfg: AfdRefConfig, workdir: str) -> dict:
    fdir = os.path.join(workdir, "file")
    out = {"record": np.fromfile(os.path.join(fdir, "record.dat"), np.float32).reshape(cfg.NX, cfg.Nt)}
    snap = os.path.join(fdir, "Snap.dat")
    if os.path.exists(snap):
        out["snap"] = np.fromfile(snap, np.float32).reshape(cfg.NX, cfg.NZ)
    out["model"] = np.fromfile(os.path.join(fdir, "Model.dat"), np.float32).reshape(cfg.NX, cfg.NZ)
    pall = os.path.join(fdir, "Pall.dat")
    if os.path.exists(pall):
        out["pall"] = np.fromfile(pall, np.float32).reshape(-1, cfg.NX, cfg.NZ)
    return out


def run(cfg: AfdRefConfig, binary: str = "afd_ref", keep: Optional[str] = None) -> dict:
    """Run one configuration to completion; returns record/snap/model arrays and wall time."""
    work = keep or tempfile.mkdtemp(prefix="afdref_")
    try:
        t0 = time.perf_counter()
        p = launch(cfg, work, binary)
        _, err = p.communicate()
        wall = time.perf_counter() - t0
        if p.returncode != 0:
            raise RuntimeError(f"{binary} exited {p.returncode}: {err.decode(errors='replace')}")
        out = collect(cfg, work)
        out["wall_s"] = wall
        return out
    finally:
        if keep is None:
            shutil.rmtree(work, ignore_errors=True)


def run_many(cfgs, binary: str = "afd_ref", procs: Optional[int] = None) -> dict:
    """Run independent configurations (shots) as concurrent processes, one per host core,
    round-robin like forward/Q_forward/Q_multishot_fd_main_fsbc_zy_rotated.f90:124.
    Returns the wall time and the per-run records."""
    procs = procs or os.cpu_count() or 1
    work = tempfile.mkdtemp(prefix="afdref_many_")
    try:
        pending = list(enumerate(cfgs))
        running = []
        records = [None] * len(cfgs)
        t0 = time.perf_counter()
        while pending or running:
            while pending and len(running) < procs:
                i, c = pending.pop(0)
                d = os.path.join(work, f"s{i}")
                running.append((i, c, d, launch(c, d, binary)))
            i, c, d, p = running.pop(0)
            _, err = p.communicate()
            if p.returncode != 0:
                raise RuntimeError(f"{binary} exited {p.returncode}: {err.decode(errors='replace')}")
            records[i] = collect(c, d)["record"]
        wall = time.perf_counter() - t0
        return {"wall_s": wall, "records": records, "procs": procs}
    finally:
        shutil.rmtree(work, ignore_errors=True)
