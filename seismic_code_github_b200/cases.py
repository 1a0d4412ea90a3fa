"""Small runs of each scheme with the benchmark geometries, for profiler captures.

    python -m seismic_code_github_b200.cases acoustic3d --n 384 --nshot 2 --nt 3
    python -m seismic_code_github_b200.cases viscoac --nshot 4 --nt 200
    python -m seismic_code_github_b200.cases gradient --nshot 4 --nt 300
    python -m seismic_code_github_b200.cases forward2d --nshot 16 --nt 40
    python -m seismic_code_github_b200.cases qgradient --nshot 4 --nt 100
    python -m seismic_code_github_b200.cases gradient3d --n 384 --nshot 2 --nt 6
    python -m seismic_code_github_b200.cases viscoel --nshot 4 --nt 60
    python -m seismic_code_github_b200.cases elastic --nshot 4 --nt 60

Each run builds a seeded synthetic model, runs one warm-up call and one timed call of the
batched path and prints the engine's timing record.  Sizes are chosen on the command line so
that a capture under a profiler stays small.
"""
import argparse
import json

import numpy as np

from . import seisfd as S
from . import workloads as W


def acoustic3d(args):
    n, pml, d, dt = args.n, min(50, args.n // 8), 10.0, 1e-3
    z = np.arange(n)
    vp = np.empty((n, n, n), np.float32)
    vp[:] = (1500.0 + 2500.0 * z / n)[None, None, :]
    w = S.wavelet(S.WAVELET_RIC, args.nt, dt, 15.0, 40)
    r = np.arange(pml, n - pml, dtype=np.int32)
    shots = [S.ShotSpec(n // 2, pml + 5, r, np.full_like(r, pml + 2), w, sy=n // 2, rec_y=r)
             for _ in range(args.nshot)]
    with S.Engine(S.ACOUSTIC_3D, n, n, d, d, dt, pml, order=8, ny=n, dy=d) as e:
        e.set_model(vp)
        e.set_shots(shots)
        e.forward_device(0)
        e.forward_device(0)
        return e.timing()


def viscoac(args):
    c = W.config3(nshot=args.nshot)
    Nx, Nz = c["vp"].shape
    rx = np.arange(c["PML"], Nx - c["PML"], dtype=np.int32)
    rz = np.full_like(rx, c["rec_z"])
    shots = [S.ShotSpec(sx, sz, rx, rz, S.wavelet(S.WAVELET_Q, args.nt, c["dt"], c["f0"]))
             for sx, sz in zip(c["src_x"], c["src_z"])]
    with S.Engine(S.VISCOAC_2D, Nx, Nz, c["dx"], c["dz"], c["dt"], c["PML"], order=10, f0=c["f0"]) as e:
        e.set_model(c["vp"], c["rho"], c["q"])
        e.set_shots(shots)
        e.forward_device(0)
        e.forward_device(0)
        return e.timing()


def viscoel(args):
    c = W.config3(nshot=args.nshot)
    Nx, Nz = c["vp"].shape
    rx = np.arange(c["PML"], Nx - c["PML"], dtype=np.int32)
    rz = np.full_like(rx, c["rec_z"])
    shots = [S.ShotSpec(sx, sz, rx, rz, S.wavelet(S.WAVELET_Q, args.nt, c["dt"], c["f0"]))
             for sx, sz in zip(c["src_x"], c["src_z"])]
    with S.Engine(S.VISCOEL_2D, Nx, Nz, c["dx"], c["dz"], c["dt"], c["PML"], order=10, f0=c["f0"]) as e:
        e.set_model_elastic(c["vp"], (c["vp"] / 1.8).astype(np.float32), c["rho"], c["q"],
                            (0.7 * c["q"]).astype(np.float32))
        e.set_shots(shots)
        e.forward_device(0)
        e.forward_device(0)
        return e.timing()


def elastic(args):
    c = W.config3(nshot=args.nshot)
    Nx, Nz = c["vp"].shape
    rx = np.arange(c["PML"], Nx - c["PML"], dtype=np.int32)
    rz = np.full_like(rx, c["rec_z"])
    shots = [S.ShotSpec(sx, sz, rx, rz, S.wavelet(S.WAVELET_ISO, args.nt, c["dt"], c["f0"], delay=args.nt // 2))
             for sx, sz in zip(c["src_x"], c["src_z"])]
    with S.Engine(S.ELASTIC_2D, Nx, Nz, c["dx"], c["dz"], c["dt"], c["PML"], order=10, f0=c["f0"]) as e:
        e.set_model_elastic(c["vp"], (c["vp"] / 1.8).astype(np.float32), c["rho"])
        e.set_shots(shots)
        e.forward_device(0)
        e.forward_device(0)
        return e.timing()


def forward2d(args):
    case = W.config2(nshot=args.nshot, nt=args.nt)
    w = S.wavelet(S.WAVELET_RIC, case.nt, case.dt, case.f0, 150)
    rx, rz = case.receivers()
    shots = [S.ShotSpec(sx, sz, rx, rz, w) for sx, sz in zip(case.src_x, case.src_z)]
    with S.Engine(S.ACOUSTIC_2D, case.Nx, case.Nz, case.dx, case.dz, case.dt, case.PML, order=16) as e:
        e.set_model(case.vp, case.den)
        e.set_shots(shots)
        e.forward_device(0)
        e.forward_device(0)
        return e.timing()


def gradient(args):
    case, vp_true = W.config4(nshot=args.nshot, nt=args.nt)
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


def qgradient(args):
    c = W.config3(nshot=args.nshot)
    Nx, Nz = c["vp"].shape
    rx = np.arange(c["PML"], Nx - c["PML"], dtype=np.int32)
    rz = np.full_like(rx, c["rec_z"])
    shots = [S.ShotSpec(sx, sz, rx, rz, S.wavelet(S.WAVELET_Q, args.nt, c["dt"], c["f0"]))
             for sx, sz in zip(c["src_x"], c["src_z"])]
    with S.Engine(S.VISCOAC_2D, Nx, Nz, c["dx"], c["dz"], c["dt"], c["PML"], order=10, f0=c["f0"]) as e:
        e.set_model(c["vp"], c["rho"], (c["q"] * 0.8).astype(np.float32))
        e.set_shots(shots)
        obs = e.forward()
        e.set_model(c["vp"], c["rho"], c["q"])
        e.gradient(obs, want_invq=True)
        e.gradient(obs, want_invq=True)
        return e.timing()


def gradient3d(args):
    n, pml, d, dt = args.n, min(50, args.n // 8), 10.0, 1e-3
    z = np.arange(n)
    vp = np.empty((n, n, n), np.float32)
    vp[:] = (1500.0 + 2500.0 * z / n)[None, None, :]
    w = S.wavelet(S.WAVELET_RIC, args.nt, dt, 15.0, 40)
    r = np.arange(pml, n - pml, dtype=np.int32)
    shots = [S.ShotSpec(n // 2, pml + 5, r, np.full_like(r, pml + 2), w, sy=n // 2, rec_y=r)
             for _ in range(args.nshot)]
    with S.Engine(S.ACOUSTIC_3D, n, n, d, d, dt, pml, order=8, ny=n, dy=d) as e:
        e.set_model((vp * 1.02).astype(np.float32))
        e.set_shots(shots)
        obs = e.forward()
        e.set_model(vp)
        e.gradient(obs)
        e.gradient(obs)
        return e.timing()


def vti(args):
    """The VTI modeller on the shipped .par geometry (workloads.vti_card), nshot shots, nt samples."""
    c = W.vti_card(nshot=args.nshot, nt=args.nt)
    _, t = S.vti_forward(c["vz"], c["eps"], c["delta"], c["dx"], c["dz"], c["dt"], c["f0"], c["nt"], c["bounds"],
                         c["shots"])
    return t


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["acoustic3d", "viscoac", "gradient", "forward2d", "qgradient", "gradient3d",
                                     "viscoel", "elastic", "vti"])
    ap.add_argument("--n", type=int, default=384, help="3-D padded grid size per axis")
    ap.add_argument("--nshot", type=int, default=2)
    ap.add_argument("--nt", type=int, default=3)
    args = ap.parse_args()
    cases = {"acoustic3d": acoustic3d, "viscoac": viscoac, "gradient": gradient, "forward2d": forward2d,
             "qgradient": qgradient, "gradient3d": gradient3d, "viscoel": viscoel, "elastic": elastic,
             "vti": vti}
    t = cases[args.case](args)
    print(json.dumps(t))


if __name__ == "__main__":
    main()
