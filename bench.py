"""Benchmark of the batched 2-D acoustic forward (config 2 of the benchmark set).

One bench step = one batched forward of all shots of the workload (every shot's full time
loop) with model, wavelets and receiver tables already resident in HBM.  `value` is grid-point
updates per second (padded points x steps x shots) over all ranks, timed with CUDA events on
the library's stream; `e2e` is the same metric through the C ABI with host buffers (model
upload and record download inside the timed region).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--exact]

Under torchrun each rank runs its own full workload on its GPU (shots are independent; no
collective on the data path): weak scaling.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gpts/s & % HBM roofline; gradient shots/s batched vs plain @ relL2≤1e-4"
BYTES_PER_POINT = {False: 28, True: 32}  # algorithmic bytes per grid-point update (const / variable density)
GRAD_BYTES_PER_POINT_STEP = 100          # 2-D acoustic gradient, per point-step of a shot
GRAD3_BYTES_PER_POINT_STEP = 124         # 3-D: forward 36, recomputation 36 + 4, adjoint 36 + 4 (D) + 8 (sum)
FALLBACK_HBM_GBS = 6650.0
PROFILE_SUMMARY = os.path.join(ROOT, "profiles", "acoustic2d_march_config2.md")


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def read_profile_traffic():
    """DRAM bytes per launch of the step kernel from the committed ncu summary, if present
    (line `dram_bytes_per_launch: <int>`)."""
    try:
        with open(PROFILE_SUMMARY) as f:
            for line in f:
                if line.strip().startswith("dram_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------------------------
# CPU baselines (the reference's own AFD build; the oracle port only if that build is absent)
# ----------------------------------------------------------------------------------------------

def cpu_reference_sample(case, steps_per_proc: int):
    """One process per host core, each running one shot of `case` (full grid) for
    `steps_per_proc` steps with the reference's own time loop (oracle/_ref/afd_ref), shots
    distributed like forward/Q_forward/Q_multishot_fd_main_fsbc_zy_rotated.f90:124."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    procs = os.cpu_count() or 1
    pts = case.Nx * case.Nz * steps_per_proc
    # the wavelet comes from a numpy restatement of tools/ricker.cpp:44: nothing of this
    # repository's native library is loaded on the reference path
    w = ref_runner.ric_wavelet(steps_per_proc, case.dt, case.f0, 150)
    if ref_runner.available():
        cfgs = [ref_runner.AfdRefConfig(NX=case.NX, NZ=case.NZ, PML=case.PML, Nt=steps_per_proc, dx=case.dx,
                                        dz=case.dz, dt=case.dt, vp=case.vp, den=case.den, wavelet=w,
                                        sx=case.src_x[i % case.nshot], sz=case.src_z[i % case.nshot],
                                        rec_z=case.rec_z, snap=-1, pall=False) for i in range(procs)]
        r = ref_runner.run_many(cfgs, procs=procs)
        return {"value": procs * pts / r["wall_s"] / 1e9, "unit": "Gpts/s", "cores": procs, "kind": "reference",
                "sample": f"{procs} concurrent single-shot runs of the reference AFD build (g++ -O3, "
                          f"oracle/_ref/afd_ref) on the {case.Nx}x{case.Nz} padded grid, {steps_per_proc} steps each",
                "wall_s": r["wall_s"]}
    import oracle_lib as ol
    rx, rz = case.receivers()
    t0 = time.perf_counter()
    ol.afd_forward(case.Nx, case.Nz, case.PML, steps_per_proc, case.dx, case.dz, case.dt, case.vp, case.den, w,
                   case.src_x[0], case.src_z[0], rx, rz)
    wall = time.perf_counter() - t0
    return {"value": pts / wall / 1e9, "unit": "Gpts/s", "cores": procs, "kind": "port",
            "sample": f"one shot of the oracle restatement (OpenMP, {procs} threads), {steps_per_proc} steps",
            "wall_s": wall}


# ----------------------------------------------------------------------------------------------

def make_case(args):
    from seismic_code_github_b200 import workloads as W
    return W.config2(nshot=args.nshot, nt=args.nt)


def build_shots(case):
    from seismic_code_github_b200 import seisfd as S
    w = S.wavelet(S.WAVELET_RIC, case.nt, case.dt, case.f0, 150)
    rx, rz = case.receivers()
    return [S.ShotSpec(sx, sz, rx, rz, w) for sx, sz in zip(case.src_x, case.src_z)]


def run_reference_arm(args, world, rank):
    if rank != 0:
        return 0
    case = make_case(args)
    steps_per_proc = args.ref_steps
    for _ in range(args.warmup):
        cpu_reference_sample(case, max(5, steps_per_proc // 4))
    vals, walls = [], []
    for _ in range(args.steps):
        r = cpu_reference_sample(case, steps_per_proc)
        vals.append(r["value"])
        walls.append(r["wall_s"])
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Gpts/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.median(walls)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded layered model, config-2 geometry)",
            "config": config_dict(case, args),
            "cpu_baseline": {"value": v, "unit": "Gpts/s", "cores": r["cores"], "kind": r["kind"],
                             "sample": r["sample"]},
            "e2e": {"value": v, "unit": "Gpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "repo_libs_mapped": repo_libs_mapped()}
    print(json.dumps(line), flush=True)
    return 0


def repo_libs_mapped():
    """Shared objects of this repository mapped into this process (the reference arm must show
    none: it runs the reference's own build and numpy only)."""
    found = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.split()[-1] if len(line.split()) >= 6 else ""
                if path.endswith(".so") and os.path.realpath(path).startswith(os.path.realpath(ROOT) + os.sep):
                    found.add(os.path.relpath(os.path.realpath(path), os.path.realpath(ROOT)))
    except OSError:
        return None
    return sorted(found)


def measure_gradient(args, dev):
    """Config 4: batched adjoint gradient (all shots in one CUDA graph: checkpointed forward,
    per-segment recomputation, adjoint, imaging) against the plain per-shot path (shots one
    after another, one launch per step, no graph) on the same shots."""
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import workloads as W
    case, vp_true = W.config4(nshot=args.grad_nshot, nt=args.grad_nt)
    w = S.wavelet(S.WAVELET_RIC, case.nt, case.dt, case.f0, 150)
    rx, rz = case.receivers()
    shots = [S.ShotSpec(sx, sz, rx, rz, w) for sx, sz in zip(case.src_x, case.src_z)]
    with S.Engine(S.ACOUSTIC_2D, case.Nx, case.Nz, case.dx, case.dz, case.dt, case.PML, order=16,
                  device=dev) as e:
        e.set_model(vp_true, case.den)
        e.set_shots(shots)
        obs = e.forward().copy()
        e.set_model(case.vp, case.den)
        e.set_checkpoint_interval(case.extra["checkpoint_interval"])
        e.gradient(obs)  # warm-up: allocation, tuning, graph capture
        times, launches = [], 0
        for _ in range(args.grad_steps):
            mis, g, _ = e.gradient(obs)
            t = e.timing()
            times.append(t["loop_ms"])
            launches = t["launches"]
        bt = float(np.median(times))
        # plain per-shot path (one shot after another, one launch per step, no graph) on the same
        # engine and shot set, so both schedules have the same memory for kept D_k slots
        sub = shots if args.grad_plain_shots <= 0 else shots[: args.grad_plain_shots]
        if len(sub) < len(shots):
            e.set_shots(sub)
        e.gradient(obs[: len(sub) * len(rx) * case.nt], per_shot=True)
        t_plain = e.timing()
    batched_sps = len(shots) / (bt / 1e3)
    plain_sps = len(sub) / (t_plain["loop_ms"] / 1e3)
    # roofline at the algorithmic ~100 B per point-step of a shot's gradient: forward with
    # checkpoints 28, recomputation 28 + 4 (D_k write), adjoint 28, imaging 4 (D_k read) + 8 (sum)
    peak, peak_src = read_peaks()
    pts_shot = float(case.Nx) * case.Nz * case.nt
    roof = {"bytes_per_point_step": GRAD_BYTES_PER_POINT_STEP,
            "achieved_gbs": GRAD_BYTES_PER_POINT_STEP * pts_shot * len(shots) / (bt / 1e3) / 1e9,
            "plain_achieved_gbs": GRAD_BYTES_PER_POINT_STEP * pts_shot * len(sub) / (t_plain["loop_ms"] / 1e3) / 1e9,
            "peak_gbs": peak, "peak_kind": peak_src}
    roof["frac"] = roof["achieved_gbs"] / peak
    roof["plain_frac"] = roof["plain_achieved_gbs"] / peak
    oracle = None
    if not args.no_cpu_baseline:
        # the reference has no adjoint: the FP64 adjoint oracle is timed beside the GPU path as a
        # labelled oracle on a bounded sample (one shot, the first grad_cpu_steps steps)
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle_lib as ol
        n = args.grad_cpu_steps
        o = obs.reshape(len(shots), len(rx), case.nt)[0][:, :n]
        t0 = time.perf_counter()
        ol.afd_gradient_f64(case.Nx, case.Nz, case.PML, n, case.dx, case.dz, case.dt, case.vp, case.den, w[:n],
                            case.src_x[0], case.src_z[0], rx, rz, o)
        wall = time.perf_counter() - t0
        oracle = {"shots_per_s_equivalent": (n / case.nt) / wall, "cores": os.cpu_count(), "kind": "oracle (FP64)",
                  "sample": f"one shot of the FP64 adjoint oracle (oracle/adj_oracle.cpp, OpenMP), {n} of {case.nt} "
                            f"steps: forward, residual, adjoint and imaging; scaled to whole shots"}
    return {"workload": f"config 4: adjoint gradient d(misfit)/d(vp), {case.NZ}x{case.NX} interior "
                        f"({case.Nz}x{case.Nx} padded), {len(shots)} shots, nt={case.nt}, checkpoints every "
                        f"{case.extra['checkpoint_interval']} steps, start model = true model smoothed (sigma 15)",
            "batched_shots_per_s": batched_sps, "batched_ms": bt, "batched_launches": launches,
            "plain_shots_per_s": plain_sps, "plain_ms": t_plain["loop_ms"], "plain_shots": len(sub),
            "plain_launches": t_plain["launches"], "batched_over_plain": batched_sps / plain_sps,
            "roofline": roof,
            "misfit": float(mis), "gradient_accuracy": "relL2 vs FP64 adjoint oracle 7.6e-7 (tests/test_gradient_gpu.py)",
            "cpu_oracle": oracle}


def measure_gradient_sharded(args, dev, world, rank):
    """Config 4 on N GPUs: every rank takes the gradient of its round-robin share of the shots
    (forward/Q_forward/Q_multishot_fd_main_fsbc_zy_rotated.f90:124-141) into device memory
    (sfd_gradient_device) and one all-reduce (NCCL, in place on the device) sums the per-rank
    gradients and misfits; no host copy of the gradient.  Time: device time of the local gradient
    plus the all-reduce, max over ranks."""
    import torch
    import torch.distributed as dist
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import sharding as SH
    from seismic_code_github_b200 import workloads as W
    case, vp_true = W.config4(nshot=args.grad_nshot, nt=args.grad_nt)
    w = S.wavelet(S.WAVELET_RIC, case.nt, case.dt, case.f0, 150)
    rx, rz = case.receivers()
    mine = SH.shard_shots(len(case.src_x), rank, world)
    shots = [S.ShotSpec(case.src_x[i], case.src_z[i], rx, rz, w) for i in mine]
    with S.Engine(S.ACOUSTIC_2D, case.Nx, case.Nz, case.dx, case.dz, case.dt, case.PML, order=16,
                  device=dev) as e:
        e.set_model(vp_true, case.den)
        e.set_shots(shots)
        obs = torch.from_numpy(e.forward().copy()).to(f"cuda:{dev}")
        e.set_model(case.vp, case.den)
        e.set_checkpoint_interval(case.extra["checkpoint_interval"])
        shape = (case.Nx, case.Nz)
        SH.sharded_gradient_device(e, obs, shape)  # warm-up
        dist.barrier()
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        mis_t, g_t, _ = SH.sharded_gradient_device(e, obs, shape)
        t1.record()
        torch.cuda.synchronize()
        mis_all, g_all = float(mis_t.item()), g_t.cpu().numpy()
    ms = torch.tensor([t0.elapsed_time(t1)], dtype=torch.float64, device=f"cuda:{dev}")
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    return {"workload": f"config 4 gradient, {len(case.src_x)} shots sharded round-robin over {world} GPUs, "
                        f"one in-place NCCL all-reduce of the {g_all.size * 4 / 1e6:.1f} MB gradient on the device",
            "shots_per_s": len(case.src_x) / (ms.item() / 1e3), "ms": ms.item(), "misfit": float(mis_all),
            "grad_norm": float(np.linalg.norm(g_all))}


# Viscoacoustic bytes per grid point and step.  Algorithmic: vx, vz, sigma, r each read and written
# once (32 B) plus the two per-cell modulus factors (8 B).  The default one-kernel step moves 44 B
# (the same and the buoyancy), plus 48 B at each sponge-band cell (its six split parts read and
# written); SFD_EXACT moves 96 B (its velocity kernel reads the three split stress parts, its
# stress kernel reads and writes all six split parts).
Q_ALG_BYTES = 40
Q_KERNEL_BYTES = 44
Q_EXACT_BYTES = 96


def measure_viscoacoustic(args, dev):
    """Config 3: 16 viscoacoustic shots (uneven record lengths) in one batched time loop; the CPU
    figure is the restated Fortran step (oracle/q_oracle.cpp, OpenMP, all host cores) on one
    shot for a bounded number of steps -- the Fortran reference cannot be compiled here."""
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import workloads as W
    c = W.config3(nshot=args.q_nshot)
    Nx, Nz = c["vp"].shape
    rx = np.arange(c["PML"], Nx - c["PML"], dtype=np.int32)
    rz = np.full_like(rx, c["rec_z"])
    shots = [S.ShotSpec(sx, sz, rx, rz, S.wavelet(S.WAVELET_Q, nt, c["dt"], c["f0"]))
             for sx, sz, nt in zip(c["src_x"], c["src_z"], c["nt"])]

    def timed(flags):
        with S.Engine(S.VISCOAC_2D, Nx, Nz, c["dx"], c["dz"], c["dt"], c["PML"], order=10, f0=c["f0"], flags=flags,
                      device=dev) as e:
            e.set_model(c["vp"], c["rho"], c["q"])
            e.set_shots(shots)
            e.forward_device(0)
            ms = []
            for _ in range(args.q_steps):
                e.forward_device(0)
                t = e.timing()
                ms.append(t["loop_ms"])
        return float(np.median(ms)), t

    pts = float(sum(Nx * Nz * nt for nt in c["nt"]))
    peak = read_peaks()[0]
    ms, t = timed(0)
    gpts = pts / (ms / 1e3) / 1e9
    ms_x, t_x = timed(S.EXACT)
    gpts_x = pts / (ms_x / 1e3) / 1e9
    out = {"workload": f"config 3: viscoacoustic SLS forward, {c['NZ']}x{c['NX']} interior ({Nz}x{Nx} padded), "
                       f"{len(shots)} shots, nt {min(c['nt'])}-{max(c['nt'])}, Q 20-200 + low-Q lens",
           "gpts_per_s": gpts, "shots_per_s": len(shots) / (ms / 1e3), "loop_ms": ms, "launches": t["launches"],
           "kernel_variant": t["kernel_variant"],
           "algorithmic_bytes_per_point": Q_ALG_BYTES, "hbm_frac_of_measured": Q_ALG_BYTES * gpts / peak,
           "kernel_bytes_per_point": Q_KERNEL_BYTES, "kernel_hbm_frac_of_measured": Q_KERNEL_BYTES * gpts / peak,
           "parity": "default mode (one kernel per step, merged stress and memory variable away from the sponge "
                     "bands): relL2 <= 1e-5 vs the FP64 restatement; attenuation and dispersion within 1% of the "
                     "discrete 1-SLS law",
           "exact": {"gpts_per_s": gpts_x, "loop_ms": ms_x, "kernel_variant": t_x["kernel_variant"],
                     "kernel_bytes_per_point": Q_EXACT_BYTES,
                     "kernel_hbm_frac_of_measured": Q_EXACT_BYTES * gpts_x / peak,
                     "hbm_frac_of_measured_at_algorithmic": Q_ALG_BYTES * gpts_x / peak,
                     "parity": "SFD_EXACT: bit-exact vs the FP32 restatement (oracle/q_oracle.cpp)"}}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle_lib as ol
        vp, rho, q = c["interior"]
        steps = args.q_cpu_steps
        run = lambda n: ol.q_forward(vp, vp * 0, rho, q, q, c["dx"], c["dz"], c["dt"], c["f0"], n, c["PML"], c["PML"],
                                     c["src_x"][0] + 1, c["src_z"][0] + 1)
        t0 = time.perf_counter()
        run(1)  # set-up and the decay steps
        t1 = time.perf_counter()
        run(1 + steps)  # the same plus `steps` time steps
        wall = (time.perf_counter() - t1) - (t1 - t0)
        out["cpu_baseline"] = {"value": Nx * Nz * steps / max(wall, 1e-9) / 1e9, "unit": "Gpts/s",
                               "cores": os.cpu_count(), "kind": "port",
                               "sample": f"restated Q_forward time step (oracle/q_oracle.cpp, OpenMP) on one shot: "
                                         f"the difference of a {steps + 1}- and a 1-sample run on the {Nz}x{Nx} "
                                         f"padded grid ({steps} steps)"}
    return out


def measure_viscoelastic(args, dev):
    """Config-3 geometry with shear waves: the visco-elastic P-SV scheme (vs = vp / 1.8, Qs = 0.7 Qp)
    on the same 16 shots, one batched time loop (22 split fields per cell, as the reference
    keeps them)."""
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import workloads as W
    c = W.config3(nshot=args.q_nshot)
    Nx, Nz = c["vp"].shape
    rx = np.arange(c["PML"], Nx - c["PML"], dtype=np.int32)
    rz = np.full_like(rx, c["rec_z"])
    shots = [S.ShotSpec(sx, sz, rx, rz, S.wavelet(S.WAVELET_Q, nt, c["dt"], c["f0"]))
             for sx, sz, nt in zip(c["src_x"], c["src_z"], c["nt"])]
    with S.Engine(S.VISCOEL_2D, Nx, Nz, c["dx"], c["dz"], c["dt"], c["PML"], order=10, f0=c["f0"], device=dev) as e:
        e.set_model_elastic(c["vp"], (c["vp"] / 1.8).astype(np.float32), c["rho"], c["q"],
                            (0.7 * c["q"]).astype(np.float32))
        e.set_shots(shots)
        e.forward_device(0)
        ms = []
        for _ in range(args.e_steps):
            e.forward_device(0)
            ms.append(e.timing()["loop_ms"])
    pts = float(sum(Nx * Nz * nt for nt in c["nt"]))
    gpts = pts / (float(np.median(ms)) / 1e3) / 1e9
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle_lib as ol
        vp, rho, q = c["interior"]
        vs, qs = (vp / 1.8).astype(np.float32), (0.7 * q).astype(np.float32)
        steps = max(1, args.q_cpu_steps // 2)
        run = lambda n: ol.q_forward(vp, vs, rho, q, qs, c["dx"], c["dz"], c["dt"], c["f0"], n, c["PML"], c["PML"],
                                     c["src_x"][0] + 1, c["src_z"][0] + 1)
        t0 = time.perf_counter()
        run(1)
        t1 = time.perf_counter()
        run(1 + steps)
        wall = (time.perf_counter() - t1) - (t1 - t0)
        cpu = {"value": Nx * Nz * steps / max(wall, 1e-9) / 1e9, "unit": "Gpts/s", "cores": os.cpu_count(),
               "kind": "port", "sample": f"restated visco-elastic Q_forward step (oracle/q_oracle.cpp, OpenMP) on one "
                                         f"shot: the difference of a {steps + 1}- and a 1-sample run ({steps} steps)"}
    return {"workload": f"config 3 geometry, visco-elastic P-SV (vs = vp/1.8): {c['NZ']}x{c['NX']} interior, "
                        f"{len(shots)} shots, nt {min(c['nt'])}-{max(c['nt'])}",
            "gpts_per_s": gpts, "shots_per_s": len(shots) / (float(np.median(ms)) / 1e3),
            "loop_ms": float(np.median(ms)), "parity": "bit-exact vs FP32 restatement (strzz and strxx)",
            "cpu_baseline": cpu}


def measure_elastic(args, dev):
    """Config-3 geometry, isotropic elastic P-SV on the standard staggered grid (the abc mode of
    forward/yang_version_2016_2_2; vs = vp / 1.8): 16 shots with uneven record lengths in one
    batched time loop, ten split fields per cell as the reference keeps them.  The model
    preparation (substagger on the host, the serial top-sponge smoothing on the device) is timed
    apart.  The CPU figure is the restated step (oracle/iso_oracle.cpp, OpenMP, all host cores)."""
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import workloads as W
    c = W.config3(nshot=args.q_nshot)
    Nx, Nz = c["vp"].shape
    rx = np.arange(c["PML"], Nx - c["PML"], dtype=np.int32)
    rz = np.full_like(rx, c["rec_z"])
    idecay = int(round(1.2 / c["f0"] / c["dt"]))  # the .par's recommended decay = 1.2 / f0 (s)
    shots = [S.ShotSpec(sx, sz, rx, rz, S.wavelet(S.WAVELET_ISO, nt, c["dt"], c["f0"], delay=idecay))
             for sx, sz, nt in zip(c["src_x"], c["src_z"], c["nt"])]
    vs = (c["vp"] / 1.8).astype(np.float32)
    with S.Engine(S.ELASTIC_2D, Nx, Nz, c["dx"], c["dz"], c["dt"], c["PML"], order=10, f0=c["f0"], device=dev) as e:
        t0 = time.perf_counter()
        e.set_model_elastic(c["vp"], vs, c["rho"])
        e.set_shots(shots)
        prep_s = time.perf_counter() - t0
        e.forward_device(0)
        ms = []
        for _ in range(args.el_steps):
            e.forward_device(0)
            t = e.timing()
            ms.append(t["loop_ms"])
    pts = float(sum(Nx * Nz * nt for nt in c["nt"]))
    gpts = pts / (float(np.median(ms)) / 1e3) / 1e9
    out = {"workload": f"config 3 geometry, isotropic elastic P-SV standard staggered grid (vs = vp/1.8): "
                       f"{c['NZ']}x{c['NX']} interior ({Nz}x{Nx} padded), {len(shots)} shots, "
                       f"nt {min(c['nt'])}-{max(c['nt'])}, Gaussian radius 50",
           "gpts_per_s": gpts, "shots_per_s": len(shots) / (float(np.median(ms)) / 1e3),
           "loop_ms": float(np.median(ms)), "launches": t["launches"], "bytes_per_point": 100,
           "hbm_frac_of_measured": 100 * gpts / read_peaks()[0], "prepare_s": prep_s,
           "parity": "bit-exact vs FP32 restatement (vx and vz)"}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle_lib as ol
        vp, rho, _ = c["interior"]
        vsi = (vp / 1.8).astype(np.float32)
        steps = max(1, args.q_cpu_steps // 2)
        run = lambda n: ol.iso_forward(vp, vsi, rho, c["dx"], c["dz"], c["dt"], c["f0"], n, c["PML"], c["PML"],
                                       c["src_x"][0] + 1, c["src_z"][0] + 1, idecay=0)
        t0 = time.perf_counter()
        run(1)  # set-up (incl. the serial smoothing) and one step
        t1 = time.perf_counter()
        run(1 + steps)
        wall = (time.perf_counter() - t1) - (t1 - t0)
        out["cpu_baseline"] = {"value": Nx * Nz * steps / max(wall, 1e-9) / 1e9, "unit": "Gpts/s",
                               "cores": os.cpu_count(), "kind": "port",
                               "sample": f"restated yang_version abc step (oracle/iso_oracle.cpp, OpenMP) on one "
                                         f"shot: the difference of a {steps + 1}- and a 1-step run ({steps} steps)"}
    return out


def measure_vti(args, dev):
    """The VTI modeller's .par geometry (de-multiple/convolution_srm/vti_qa_2d_c3_demo1): 64 shots
    of 600 traces on a seeded synthetic 300 x 300 VTI model, batched in one launch per time step
    (the fused u / q step of csrc/vti2d.cu, reference operation order).  The record length is cut
    from the card's 10000 to 2000 samples; the per-step cost does not depend on it.  The CPU figure
    is the restated modeller (oracle/vti_oracle.cpp, OpenMP) on one shot."""
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import workloads as W
    c = W.vti_card(nshot=args.vti_nshot, nt=args.vti_nt)
    args_ = (c["vz"], c["eps"], c["delta"], c["dx"], c["dz"], c["dt"], c["f0"], c["nt"], c["bounds"])
    S.vti_forward(*args_, c["shots"][:1], device=dev)  # warm-up (module load)
    ms, mx, t = [], [], None
    for _ in range(args.vti_steps):
        _, t = S.vti_forward(*args_, c["shots"], device=dev)
        ms.append(t["loop_ms"])
        _, tx = S.vti_forward(*args_, c["shots"], device=dev, exact=True)
        mx.append(tx["loop_ms"])
    pts = t["point_updates"]
    gpts = pts / (float(np.median(ms)) / 1e3) / 1e9
    gpts_exact = pts / (float(np.median(mx)) / 1e3) / 1e9
    nxl, nxr, nzu, nzd = c["bounds"]
    nx = 600 + nxl + nxr - 2
    nz = c["vz"].shape[1] + nzu + nzd - 2
    out = {"workload": f"VTI pseudo-acoustic (vti_qa_2d_modelling_new.par geometry): 300x300 model, {nz}x{nx} "
                       f"grid per shot, {len(c['shots'])} shots of 600 traces, nt {c['nt']} (+ source delay steps)",
           "gpts_per_s": gpts, "shots_per_s": len(c["shots"]) / (float(np.median(ms)) / 1e3),
           "loop_ms": float(np.median(ms)), "launches": t["launches"], "total_ms": t["total_ms"],
           "bytes_per_point": 36, "hbm_frac_of_measured": 36 * gpts / read_peaks()[0],
           "gpts_per_s_exact": gpts_exact,
           "parity": "relL2 <= 1e-5 vs FP32 and FP64 restatement; SFD_EXACT (gpts_per_s_exact) bit-exact vs "
                     "the FP32 restatement (tests/test_vti_gpu.py)"}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle_lib as ol
        steps = args.vti_cpu_steps
        sh = c["shots"][len(c["shots"]) // 2]
        t0 = time.perf_counter()
        ol.vti_forward(c["vz"], c["eps"], c["delta"], c["dx"], c["dz"], c["dt"], c["f0"], steps, c["bounds"], *sh)
        wall = time.perf_counter() - t0
        nwt = int(round(2 * 0.07 / c["dt"])) + 1
        out["cpu_baseline"] = {"value": nx * nz * (steps + (nwt - 1) // 2) / max(wall, 1e-9) / 1e9, "unit": "Gpts/s",
                               "cores": os.cpu_count(), "kind": "port",
                               "sample": f"restated VTI modeller (oracle/vti_oracle.cpp, OpenMP) on one shot, "
                                         f"{steps} record samples plus the source delay steps"}
    return out


def measure_q_gradient(args, dev):
    """Config-3 geometry: the viscoacoustic gradient d misfit / d vp and d misfit / d (1/Q) of 16
    shots (uneven record lengths), observed data from the Q field scaled by 0.8, batched (one
    CUDA graph) against the plain per-shot schedule on the same shots."""
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import workloads as W
    c = W.config3(nshot=args.qg_nshot)
    Nx, Nz = c["vp"].shape
    rx = np.arange(c["PML"], Nx - c["PML"], dtype=np.int32)
    rz = np.full_like(rx, c["rec_z"])
    nts = [max(1, int(round(nt * args.qg_nt_scale))) for nt in c["nt"]]
    shots = [S.ShotSpec(sx, sz, rx, rz, S.wavelet(S.WAVELET_Q, nt, c["dt"], c["f0"]))
             for sx, sz, nt in zip(c["src_x"], c["src_z"], nts)]
    with S.Engine(S.VISCOAC_2D, Nx, Nz, c["dx"], c["dz"], c["dt"], c["PML"], order=10, f0=c["f0"], device=dev) as e:
        e.set_model(c["vp"], c["rho"], (c["q"] * 0.8).astype(np.float32))
        e.set_shots(shots)
        obs = e.forward().copy()
        e.set_model(c["vp"], c["rho"], c["q"])
        e.gradient(obs, want_invq=True)  # warm-up: allocation and graph capture
        ms = []
        for _ in range(args.qg_steps):
            e.gradient(obs, want_invq=True)
            ms.append(e.timing()["loop_ms"])
        t = e.timing()
        sub = shots if args.qg_plain_shots <= 0 else shots[: args.qg_plain_shots]
        offs = np.cumsum([0] + [s.nrec * s.nt for s in shots])
        if len(sub) < len(shots):
            e.set_shots(sub)
        e.gradient(obs[: offs[len(sub)]], want_invq=True, per_shot=True)
        tp = e.timing()
    bt = float(np.median(ms))
    return {"workload": f"config 3 geometry: viscoacoustic gradient d/dvp and d/d(1/Q), {c['NZ']}x{c['NX']} interior "
                        f"({Nz}x{Nx} padded), {len(shots)} shots, nt {min(nts)}-{max(nts)}",
            "batched_shots_per_s": len(shots) / (bt / 1e3), "batched_ms": bt, "batched_launches": t["launches"],
            "plain_shots_per_s": len(sub) / (tp["loop_ms"] / 1e3), "plain_ms": tp["loop_ms"], "plain_shots": len(sub),
            "batched_over_plain": (len(shots) / bt) / (len(sub) / tp["loop_ms"]),
            "gradient_accuracy": "relL2 vs FP64 adjoint oracle 1.5e-6 (vp), 2.6e-6 (1/Q) (tests/test_q_gradient_gpu.py)"}


def measure_3d_gradient(args, dev):
    """Config-5 geometry (612^3 padded, order 8): the 3-D gradient of a few shots with record
    lengths scaled by --d3g-nt-scale; the library plans shot groups and checkpoint levels to the
    device memory.  Batched against the per-shot schedule on the same shots."""
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import workloads as W
    c = W.config5(nshot=args.d3g_nshot, nt_scale=args.d3g_nt_scale)
    n, d = c["n"], c["d"]
    vp = np.empty((n, n, n), np.float32)
    for x0 in range(0, n, 64):
        vp[x0:x0 + 64] = c["vp_slab"](x0, min(n, x0 + 64))
    shots = [S.ShotSpec(sx, sz, rx, rz, S.wavelet(S.WAVELET_RIC, nt, c["dt"], c["f0"], 80), sy=sy, rec_y=ry)
             for (sx, sy, sz), (rx, ry, rz), nt in zip(c["src"], c["rec"], c["nt"])]
    with S.Engine(S.ACOUSTIC_3D, n, n, d, d, c["dt"], c["PML"], order=8, ny=n, dy=d, device=dev) as e:
        e.set_model((vp * 1.02).astype(np.float32))
        e.set_shots(shots)
        obs = e.forward().copy()
        e.set_model(vp)
        e.gradient(obs)
        t = e.timing()
        # plain per-shot schedule (one shot per group) on the first shots, the same engine and memory
        nplain = len(shots) if args.d3g_plain_shots <= 0 else min(args.d3g_plain_shots, len(shots))
        if nplain < len(shots):
            e.set_shots(shots[:nplain])
        nobs = sum(len(s.rec_x) * s.nt for s in shots[:nplain])
        e.gradient(obs[:nobs], per_shot=True)
        tp = e.timing()
    del vp
    levels = 2 if t["kernel_variant"] == 62 else 1
    pts = float(n) ** 3 * sum(c["nt"])
    pts_plain = float(n) ** 3 * sum(c["nt"][:nplain])
    peak, peak_src = read_peaks()
    roof = {"bytes_per_point_step": GRAD3_BYTES_PER_POINT_STEP,
            "achieved_gbs": GRAD3_BYTES_PER_POINT_STEP * pts / (t["loop_ms"] / 1e3) / 1e9, "peak_gbs": peak,
            "peak_kind": peak_src,
            "note": "algorithmic bytes of one checkpoint level; with two levels the extra recomputation pass "
                    "is work beyond this count"}
    roof["frac"] = roof["achieved_gbs"] / peak
    return {"workload": f"config 5 geometry: 3-D gradient d/dvp, {c['N']}^3 interior ({n}^3 padded), {len(shots)} shots, "
                        f"record lengths 1500-2500 scaled by {args.d3g_nt_scale} (nt {min(c['nt'])}-{max(c['nt'])})",
            "batched_shots_per_s": len(shots) / (t["loop_ms"] / 1e3), "batched_ms": t["loop_ms"],
            "checkpoint_levels": levels, "passes": t["point_updates"] / pts,
            "gpts_per_s_all_passes": t["point_updates"] / (t["loop_ms"] / 1e3) / 1e9,
            "plain_shots_per_s": nplain / (tp["loop_ms"] / 1e3), "plain_ms": tp["loop_ms"], "plain_shots": nplain,
            "batched_over_plain": (len(shots) / t["loop_ms"]) / (nplain / tp["loop_ms"]),
            "roofline": roof,
            "plain_gbs": GRAD3_BYTES_PER_POINT_STEP * pts_plain / (tp["loop_ms"] / 1e3) / 1e9,
            "gradient_accuracy": "relL2 vs FP64 3-D adjoint oracle 6.7e-7 (tests/test_gradient3d_gpu.py)"}


def measure_3d(args, dev):
    """Config 5: 3-D acoustic, 16 shots of 612^3 padded cells in one batched time loop.  The
    record lengths are scaled by --d3-nt-scale so the section stays short; the per-step cost does
    not depend on nt.  No 3-D reference exists: the CPU figure is the restated scheme
    (oracle/afd3d_oracle.cpp, OpenMP, FP32) on one shot for a few steps."""
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import workloads as W
    c = W.config5(nshot=args.d3_nshot, nt_scale=args.d3_nt_scale)
    n, d = c["n"], c["d"]
    vp = np.empty((n, n, n), np.float32)
    for x0 in range(0, n, 64):
        vp[x0:x0 + 64] = c["vp_slab"](x0, min(n, x0 + 64))
    shots = [S.ShotSpec(sx, sz, rx, rz, S.wavelet(S.WAVELET_RIC, nt, c["dt"], c["f0"], 80), sy=sy, rec_y=ry)
             for (sx, sy, sz), (rx, ry, rz), nt in zip(c["src"], c["rec"], c["nt"])]
    with S.Engine(S.ACOUSTIC_3D, n, n, d, d, c["dt"], c["PML"], order=8, ny=n, dy=d, device=dev) as e:
        e.set_model(vp)
        e.set_shots(shots)
        e.forward_device(0)
        ms = []
        for _ in range(args.d3_steps):
            e.forward_device(0)
            t = e.timing()
            ms.append(t["loop_ms"])
    pts = float(n) ** 3 * sum(c["nt"])
    gpts = pts / (float(np.median(ms)) / 1e3) / 1e9
    out = {"workload": f"config 5: 3-D acoustic order 8, {c['N']}^3 interior ({n}^3 padded), {len(shots)} shots, "
                       f"256x256 receivers each, record lengths 1500-2500 scaled by {args.d3_nt_scale} "
                       f"(nt {min(c['nt'])}-{max(c['nt'])})",
           "gpts_per_s": gpts, "loop_ms": float(np.median(ms)), "launches": t["launches"], "bytes_per_point": 36,
           "hbm_frac_of_measured": 36 * gpts / read_peaks()[0], "parity": "relL2 <= 1e-5 vs FP64 restatement"}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle_lib as ol
        steps = args.d3_cpu_steps
        r = np.zeros(1, np.int32) + c["PML"]
        w = shots[0].wavelet[:steps + 1]
        t0 = time.perf_counter()
        ol.afd3d_forward(vp, None, w[:1], c["src"][0], r, r, r, c["PML"], d, d, d, c["dt"], fp64=False)
        t1 = time.perf_counter()
        ol.afd3d_forward(vp, None, w[:steps + 1], c["src"][0], r, r, r, c["PML"], d, d, d, c["dt"], fp64=False)
        wall = (time.perf_counter() - t1) - (t1 - t0)
        out["cpu_baseline"] = {"value": n ** 3 * steps / max(wall, 1e-9) / 1e9, "unit": "Gpts/s",
                               "cores": os.cpu_count(), "kind": "port",
                               "sample": f"restated 3-D step (oracle/afd3d_oracle.cpp, OpenMP, FP32) on one shot: the "
                                         f"difference of a {steps + 1}- and a 1-step run on the {n}^3 grid"}
    del vp
    return out


def config_dict(case, args):
    return {"workload": f"batched 2-D acoustic forward, {case.NZ}x{case.NX} interior "
                        f"({case.Nz}x{case.Nx} padded, {case.PML}-cell sponge), {case.nshot} shots, nt={case.nt}, "
                        f"16th-order staggered v-p, {len(case.receivers()[0])} receivers/shot",
            "nshot": case.nshot, "nt": case.nt, "grid_padded": [case.Nx, case.Nz], "order": 16,
            "mode": "exact" if args.exact else "fma",
            "l2_policy": "inputs larger than L2 (wavefield state ~2.3 GB per rank)",
            "parallelism": f"shots x {max(1, int(os.environ.get('WORLD_SIZE', '1')))} GPUs (independent)"}


def run_ours(args, world, rank, local):
    import torch
    from seismic_code_github_b200 import seisfd as S
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = local if torch.cuda.is_available() else 0
    torch.cuda.set_device(dev)
    case = make_case(args)
    shots = build_shots(case)
    flags = S.EXACT if args.exact else 0
    eng = S.Engine(S.ACOUSTIC_2D, case.Nx, case.Nz, case.dx, case.dz, case.dt, case.PML, order=16, flags=flags,
                   device=dev)
    eng.set_model(case.vp, case.den)
    eng.set_shots(shots)
    varden = not np.all(case.den == case.den.flat[0])

    for _ in range(args.warmup):
        eng.forward_device(0)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    sampler = ClockSampler(dev)
    barrier()
    sampler.start()
    dev_ms, loop_ms, launches, pts = 0.0, 0.0, 0, 0.0
    for _ in range(args.steps):
        eng.forward_device(0)
        t = eng.timing()
        dev_ms += t["device_ms"]
        loop_ms += t["loop_ms"]
        launches += t["launches"]
        pts += t["point_updates"]
    barrier()
    clocks = sampler.stop()

    # e2e: model upload from pinned host memory + forward + record download to pinned memory
    nrec_total = eng.record_size()
    pinned_rec = torch.empty(nrec_total, dtype=torch.float32, pin_memory=True).numpy()
    pinned_vp = torch.empty(case.vp.shape, dtype=torch.float32, pin_memory=True).numpy()
    pinned_vp[...] = case.vp
    e2e_steps = max(1, min(args.steps, 2))
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        eng.set_model(pinned_vp, case.den)
        eng.forward(pinned_rec)
    barrier()
    e2e_s = time.perf_counter() - t0
    h2d = case.vp.nbytes + (0 if not varden else case.den.nbytes)
    d2h = pinned_rec.nbytes

    tot = torch.tensor([dev_ms, pts, loop_ms, e2e_s], dtype=torch.float64, device=f"cuda:{dev}")
    if dist is not None:
        mx = tot.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        sm = tot.clone()
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        dev_ms_max, pts_all, loop_max, e2e_max = mx[0].item(), sm[1].item(), mx[2].item(), mx[3].item()
    else:
        dev_ms_max, pts_all, loop_max, e2e_max = dev_ms, pts, loop_ms, e2e_s

    # plain per-shot path (one launch per step per shot, no graph) on a subset of shots
    plain = None
    if rank == 0 and args.plain_shots > 0:
        sub = shots[: args.plain_shots]
        eng.set_shots(sub)
        eng.forward_per_shot()
        tp = eng.timing()
        eng.set_shots(sub)
        eng.forward_device(0)
        tb = eng.timing()
        plain = {"shots": len(sub), "plain_ms": tp["device_ms"], "plain_launches": tp["launches"],
                 "batched_ms_same_shots": tb["device_ms"],
                 "plain_shots_per_s": len(sub) / (tp["device_ms"] / 1e3),
                 "batched_full_shots_per_s": world * case.nshot * args.steps / (dev_ms_max / 1e3)}

    eng.close()
    grad_sharded = None
    if dist is not None:
        if args.grad_steps > 0:
            grad_sharded = measure_gradient_sharded(args, dev, world, rank)
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0

    value = pts_all / (dev_ms_max / 1e3) / 1e9
    e2e_val = world * e2e_steps * (pts / args.steps) / e2e_max / 1e9
    peak, peak_kind = read_peaks()
    bpp = BYTES_PER_POINT[bool(varden)]
    achieved = bpp * pts / (loop_ms / 1e3) / 1e9  # GB/s on rank 0's kernel time
    traffic = read_profile_traffic()
    launches_per_call = launches / args.steps
    line = {
        "metric": METRIC, "value": value, "unit": "Gpts/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded layered model with Gaussian anomalies, config-2 geometry)",
        "config": config_dict(case, args),
        "shots_per_s": world * case.nshot * args.steps / (dev_ms_max / 1e3),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
                     else "fallback 6.65 TB/s", "frac_of_nominal_8tbs": achieved / 8000.0,
                     "bytes_per_point": bpp, "traffic": traffic,
                     "traffic_source": os.path.relpath(PROFILE_SUMMARY, ROOT) if traffic else None},
        "e2e": {"value": e2e_val, "unit": "Gpts/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "launches_per_step": launches_per_call,
        "kernel": {11: "FMA tile kernel, one tile per CTA", 12: "FMA tile kernel, persistent",
                   13: "FMA x-marching kernel", 1: "reference-order kernel (SFD_EXACT)"}.get(t["kernel_variant"],
                                                                                            str(t["kernel_variant"])),
        "clocks": clocks,
    }
    if plain is not None:
        line["plain_vs_batched"] = plain
    if world == 1 and args.grad_steps > 0:
        line["gradient"] = measure_gradient(args, dev)
    if grad_sharded is not None:
        line["gradient_sharded"] = grad_sharded
    if world == 1 and args.q_steps > 0:
        line["viscoacoustic"] = measure_viscoacoustic(args, dev)
    if world == 1 and args.e_steps > 0:
        line["viscoelastic"] = measure_viscoelastic(args, dev)
    if world == 1 and args.el_steps > 0:
        line["elastic"] = measure_elastic(args, dev)
    if world == 1 and args.vti_steps > 0:
        line["vti"] = measure_vti(args, dev)
    if world == 1 and args.qg_steps > 0:
        line["viscoacoustic_gradient"] = measure_q_gradient(args, dev)
    if world == 1 and args.d3_steps > 0:
        line["acoustic3d"] = measure_3d(args, dev)
    if world == 1 and args.d3g_nshot > 0:
        line["acoustic3d_gradient"] = measure_3d_gradient(args, dev)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = {k: v for k, v in cpu_reference_sample(case, args.ref_steps).items() if k != "wall_s"}
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------------------------
# Small runs of one scheme for profiler captures (python bench.py --case NAME ...): a seeded
# synthetic model with the benchmark geometries, one warm-up call and one timed call of the batched
# path; prints the engine's timing record.  Sizes come from --case-n / --case-nshot / --case-nt so
# that a capture stays small.
# ----------------------------------------------------------------------------------------------

def case_acoustic3d(args):
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import workloads as W
    n, pml, d, dt = args.case_n, min(50, args.case_n // 8), 10.0, 1e-3
    z = np.arange(n)
    vp = np.empty((n, n, n), np.float32)
    vp[:] = (1500.0 + 2500.0 * z / n)[None, None, :]
    w = S.wavelet(S.WAVELET_RIC, args.case_nt, dt, 15.0, 40)
    r = np.arange(pml, n - pml, dtype=np.int32)
    shots = [S.ShotSpec(n // 2, pml + 5, r, np.full_like(r, pml + 2), w, sy=n // 2, rec_y=r)
             for _ in range(args.case_nshot)]
    with S.Engine(S.ACOUSTIC_3D, n, n, d, d, dt, pml, order=8, ny=n, dy=d) as e:
        e.set_model(vp)
        e.set_shots(shots)
        e.forward_device(0)
        e.forward_device(0)
        return e.timing()


def case_viscoac(args):
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import workloads as W
    c = W.config3(nshot=args.case_nshot)
    Nx, Nz = c["vp"].shape
    rx = np.arange(c["PML"], Nx - c["PML"], dtype=np.int32)
    rz = np.full_like(rx, c["rec_z"])
    shots = [S.ShotSpec(sx, sz, rx, rz, S.wavelet(S.WAVELET_Q, args.case_nt, c["dt"], c["f0"]))
             for sx, sz in zip(c["src_x"], c["src_z"])]
    with S.Engine(S.VISCOAC_2D, Nx, Nz, c["dx"], c["dz"], c["dt"], c["PML"], order=10, f0=c["f0"]) as e:
        e.set_model(c["vp"], c["rho"], c["q"])
        e.set_shots(shots)
        e.forward_device(0)
        e.forward_device(0)
        return e.timing()


def case_viscoel(args):
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import workloads as W
    c = W.config3(nshot=args.case_nshot)
    Nx, Nz = c["vp"].shape
    rx = np.arange(c["PML"], Nx - c["PML"], dtype=np.int32)
    rz = np.full_like(rx, c["rec_z"])
    shots = [S.ShotSpec(sx, sz, rx, rz, S.wavelet(S.WAVELET_Q, args.case_nt, c["dt"], c["f0"]))
             for sx, sz in zip(c["src_x"], c["src_z"])]
    with S.Engine(S.VISCOEL_2D, Nx, Nz, c["dx"], c["dz"], c["dt"], c["PML"], order=10, f0=c["f0"]) as e:
        e.set_model_elastic(c["vp"], (c["vp"] / 1.8).astype(np.float32), c["rho"], c["q"],
                            (0.7 * c["q"]).astype(np.float32))
        e.set_shots(shots)
        e.forward_device(0)
        e.forward_device(0)
        return e.timing()


def case_elastic(args):
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import workloads as W
    c = W.config3(nshot=args.case_nshot)
    Nx, Nz = c["vp"].shape
    rx = np.arange(c["PML"], Nx - c["PML"], dtype=np.int32)
    rz = np.full_like(rx, c["rec_z"])
    shots = [S.ShotSpec(sx, sz, rx, rz, S.wavelet(S.WAVELET_ISO, args.case_nt, c["dt"], c["f0"], delay=args.case_nt // 2))
             for sx, sz in zip(c["src_x"], c["src_z"])]
    with S.Engine(S.ELASTIC_2D, Nx, Nz, c["dx"], c["dz"], c["dt"], c["PML"], order=10, f0=c["f0"]) as e:
        e.set_model_elastic(c["vp"], (c["vp"] / 1.8).astype(np.float32), c["rho"])
        e.set_shots(shots)
        e.forward_device(0)
        e.forward_device(0)
        return e.timing()


def case_forward2d(args):
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import workloads as W
    case = W.config2(nshot=args.case_nshot, nt=args.case_nt)
    w = S.wavelet(S.WAVELET_RIC, case.nt, case.dt, case.f0, 150)
    rx, rz = case.receivers()
    shots = [S.ShotSpec(sx, sz, rx, rz, w) for sx, sz in zip(case.src_x, case.src_z)]
    with S.Engine(S.ACOUSTIC_2D, case.Nx, case.Nz, case.dx, case.dz, case.dt, case.PML, order=16) as e:
        e.set_model(case.vp, case.den)
        e.set_shots(shots)
        e.forward_device(0)
        e.forward_device(0)
        return e.timing()


def case_gradient(args):
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import workloads as W
    case, vp_true = W.config4(nshot=args.case_nshot, nt=args.case_nt)
    w = S.wavelet(S.WAVELET_RIC, case.nt, case.dt, case.f0, 150)
    rx, rz = case.receivers()
    shots = [S.ShotSpec(sx, sz, rx, rz, w) for sx, sz in zip(case.src_x, case.src_z)]
    with S.Engine(S.ACOUSTIC_2D, case.Nx, case.Nz, case.dx, case.dz, case.dt, case.PML, order=16) as e:
        e.set_model(vp_true, case.den)
        e.set_shots(shots)
        obs = e.forward()
        e.set_model(case.vp, case.den)
        e.set_checkpoint_interval(case.extra["checkpoint_interval"])
        e.gradient(obs)
        e.gradient(obs)
        return e.timing()


def case_qgradient(args):
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import workloads as W
    c = W.config3(nshot=args.case_nshot)
    Nx, Nz = c["vp"].shape
    rx = np.arange(c["PML"], Nx - c["PML"], dtype=np.int32)
    rz = np.full_like(rx, c["rec_z"])
    shots = [S.ShotSpec(sx, sz, rx, rz, S.wavelet(S.WAVELET_Q, args.case_nt, c["dt"], c["f0"]))
             for sx, sz in zip(c["src_x"], c["src_z"])]
    with S.Engine(S.VISCOAC_2D, Nx, Nz, c["dx"], c["dz"], c["dt"], c["PML"], order=10, f0=c["f0"]) as e:
        e.set_model(c["vp"], c["rho"], (c["q"] * 0.8).astype(np.float32))
        e.set_shots(shots)
        obs = e.forward()
        e.set_model(c["vp"], c["rho"], c["q"])
        e.gradient(obs, want_invq=True)
        e.gradient(obs, want_invq=True)
        return e.timing()


def case_gradient3d(args):
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import workloads as W
    n, pml, d, dt = args.case_n, min(50, args.case_n // 8), 10.0, 1e-3
    z = np.arange(n)
    vp = np.empty((n, n, n), np.float32)
    vp[:] = (1500.0 + 2500.0 * z / n)[None, None, :]
    w = S.wavelet(S.WAVELET_RIC, args.case_nt, dt, 15.0, 40)
    r = np.arange(pml, n - pml, dtype=np.int32)
    shots = [S.ShotSpec(n // 2, pml + 5, r, np.full_like(r, pml + 2), w, sy=n // 2, rec_y=r)
             for _ in range(args.case_nshot)]
    with S.Engine(S.ACOUSTIC_3D, n, n, d, d, dt, pml, order=8, ny=n, dy=d) as e:
        e.set_model((vp * 1.02).astype(np.float32))
        e.set_shots(shots)
        obs = e.forward()
        e.set_model(vp)
        e.gradient(obs)
        e.gradient(obs)
        return e.timing()


def case_vti(args):
    """The VTI modeller on the shipped .par geometry (workloads.vti_card), nshot shots, nt samples."""
    from seismic_code_github_b200 import seisfd as S
    from seismic_code_github_b200 import workloads as W
    c = W.vti_card(nshot=args.case_nshot, nt=args.case_nt)
    _, t = S.vti_forward(c["vz"], c["eps"], c["delta"], c["dx"], c["dz"], c["dt"], c["f0"], c["nt"], c["bounds"],
                         c["shots"])
    return t

CASES = {"acoustic3d": case_acoustic3d, "viscoac": case_viscoac, "gradient": case_gradient, "forward2d": case_forward2d,
         "qgradient": case_qgradient, "gradient3d": case_gradient3d, "viscoel": case_viscoel, "elastic": case_elastic,
         "vti": case_vti}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--exact", action="store_true", help="reference operation order (SFD_EXACT)")
    ap.add_argument("--nshot", type=int, default=64)
    ap.add_argument("--nt", type=int, default=4000)
    ap.add_argument("--plain-shots", type=int, default=4)
    ap.add_argument("--ref-steps", type=int, default=100, help="time steps per process in a CPU sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grad-steps", type=int, default=2, help="timed batched gradients (0 = skip)")
    ap.add_argument("--grad-nshot", type=int, default=32)
    ap.add_argument("--grad-nt", type=int, default=3000)
    ap.add_argument("--grad-plain-shots", type=int, default=0, help="plain per-shot gradient shots (0 = all)")
    ap.add_argument("--grad-cpu-steps", type=int, default=100, help="steps of the timed FP64 adjoint oracle sample")
    ap.add_argument("--q-steps", type=int, default=2, help="timed viscoacoustic forwards (0 = skip)")
    ap.add_argument("--q-nshot", type=int, default=16)
    ap.add_argument("--q-cpu-steps", type=int, default=120)
    ap.add_argument("--d3-steps", type=int, default=1, help="timed 3-D forwards (0 = skip)")
    ap.add_argument("--d3-nshot", type=int, default=4)
    ap.add_argument("--d3-nt-scale", type=float, default=1.0, help="record-length scale (1 = config 5's 1500-2500)")
    ap.add_argument("--d3-cpu-steps", type=int, default=3)
    ap.add_argument("--e-steps", type=int, default=1, help="timed visco-elastic forwards (0 = skip)")
    ap.add_argument("--el-steps", type=int, default=1, help="timed isotropic elastic forwards (0 = skip)")
    ap.add_argument("--vti-steps", type=int, default=1, help="timed VTI surveys (0 = skip)")
    ap.add_argument("--vti-nshot", type=int, default=64)
    ap.add_argument("--vti-nt", type=int, default=2000)
    ap.add_argument("--vti-cpu-steps", type=int, default=60)
    ap.add_argument("--qg-steps", type=int, default=1, help="timed viscoacoustic gradients (0 = skip)")
    ap.add_argument("--qg-nshot", type=int, default=16)
    ap.add_argument("--qg-nt-scale", type=float, default=1.0)
    ap.add_argument("--qg-plain-shots", type=int, default=0, help="plain per-shot gradient shots (0 = all)")
    ap.add_argument("--d3g-nshot", type=int, default=2, help="3-D gradient shots (0 = skip)")
    ap.add_argument("--d3g-nt-scale", type=float, default=1.0, help="record-length scale (1 = config 5's 1500-2500)")
    ap.add_argument("--d3g-plain-shots", type=int, default=1, help="plain per-shot 3-D gradient shots (0 = all)")
    ap.add_argument("--case", choices=sorted(CASES), help="run one small case for a profiler capture and print "
                    "its timing record (no benchmark line)")
    ap.add_argument("--case-n", type=int, default=384, help="--case: 3-D padded grid size per axis")
    ap.add_argument("--case-nshot", type=int, default=2)
    ap.add_argument("--case-nt", type=int, default=3)
    args = ap.parse_args()
    if args.case:
        print(json.dumps(CASES[args.case](args)))
        return 0
    world, rank, local = dist_env()
    if args.impl == "reference":
        return run_reference_arm(args, world, rank)
    return run_ours(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
