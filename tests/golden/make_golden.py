"""Regenerates the committed fixtures in tests/golden/ (run in a container that has the
reference tree and the builds of oracle/ref_build.py; the GPU tests only read the outputs).

  afd_default/{record,Snap,Model}.dat  copied verbatim from
        forward/Acoustic_FD_by_ss/file/ -- the reference's own shipped outputs
        (NX=NZ=100, PML=20, Nt=2000, 16th order; record is 100 traces x 2000 samples).
  ric_trace255.f32   trace 255 of zero_offset_data.dat written by tools/ricker.cpp
        (built unmodified): the Ricker formula of tools/ricker.cpp:44, f0=35, dt=2 ms,
        delay 150 samples, 1024 samples.
  config1_record.f32 the patched reference (oracle/ref_build.py) run on the config-1 case of
        seismic_code_github_b200.workloads.config1(): 251 traces x 1000 samples.
  small_varden_record.f32  same for workloads.small_varden(): non-square grid, variable
        density, off-centre source (80 traces x 300 samples).
  afd_small/{record,Snap,Model,Pall}.dat  the patched reference with its own constant model and
        28 Hz wavelet on NX=NZ=40, PML=10, Nt=150, dt=1 ms, Snapshot at step 100 and the
        every-10-steps Pall.dat switched on: the outputs of the afd_fd program are pinned to it.
  manifest.json      sizes and sha256 of the above.

Usage: python tests/golden/make_golden.py [--reference DIR]   (default: $SFD_REFERENCE, else /root/reference)
"""
import argparse
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import ref_runner  # noqa: E402
from seismic_code_github_b200 import workloads  # noqa: E402


def ref_config(case: workloads.AcousticCase, wavelet: np.ndarray) -> ref_runner.AfdRefConfig:
    return ref_runner.AfdRefConfig(
        NX=case.NX, NZ=case.NZ, PML=case.PML, Nt=case.nt, dx=case.dx, dz=case.dz, dt=case.dt,
        vp=case.vp, den=case.den, wavelet=wavelet, sx=case.src_x[0], sz=case.src_z[0],
        rec_z=case.rec_z, snap=-1, pall=False)


def ric_wavelet(nt, dt, f0, delay=150):
    """tools/ricker.cpp:44 in numpy double arithmetic, rounded to float32 (fixture input)."""
    pi = 3.1415926
    j = np.arange(nt, dtype=np.float64)
    a = pi * float(f0) * (j - delay) * np.float64(np.float32(dt))
    return ((1 - 2 * a * a) * np.exp(-a * a)).astype(np.float32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("SFD_REFERENCE", "/root/reference"))
    args = ap.parse_args()
    ref = args.reference
    if not ref_runner.available():
        subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "ref_build.py"), "--reference", ref],
                       check=True)
    out = {}
    d = os.path.join(HERE, "afd_default")
    os.makedirs(d, exist_ok=True)
    for f in ("record.dat", "Snap.dat", "Model.dat"):
        shutil.copyfile(os.path.join(ref, "forward/Acoustic_FD_by_ss/file", f), os.path.join(d, f))
        out[f"afd_default/{f}"] = None

    tmp = tempfile.mkdtemp()
    try:
        subprocess.run([ref_runner.ref_binary("ricker")], cwd=tmp, check=True)
        sec = np.fromfile(os.path.join(tmp, "zero_offset_data.dat"), np.float32).reshape(512, 1024)
        sec[255].tofile(os.path.join(HERE, "ric_trace255.f32"))
        out["ric_trace255.f32"] = None
    finally:
        shutil.rmtree(tmp, ignore_errors=True)

    for case, fn in ((workloads.config1(), "config1_record.f32"),
                     (workloads.small_varden(), "small_varden_record.f32")):
        w = ric_wavelet(case.nt, case.dt, int(case.f0))
        res = ref_runner.run(ref_config(case, w))
        res["record"].astype(np.float32).tofile(os.path.join(HERE, fn))
        out[fn] = {"case": case.name, "wall_s": round(res["wall_s"], 3)}

    small = ref_runner.AfdRefConfig(NX=40, NZ=40, PML=10, Nt=150, dt=0.001, snap=100, pall=True)
    d = os.path.join(HERE, "afd_small")
    os.makedirs(d, exist_ok=True)
    work = tempfile.mkdtemp()
    try:
        ref_runner.run(small, keep=work)
        for f in ("record.dat", "Snap.dat", "Model.dat", "Pall.dat"):
            shutil.copyfile(os.path.join(work, "file", f), os.path.join(d, f))
            out[f"afd_small/{f}"] = {"case": "NX=NZ=40 PML=10 Nt=150 dt=1ms snap=100 pall"}
    finally:
        shutil.rmtree(work, ignore_errors=True)

    manifest = {}
    for k, meta in out.items():
        p = os.path.join(HERE, k)
        with open(p, "rb") as f:
            data = f.read()
        manifest[k] = {"bytes": len(data), "sha256": hashlib.sha256(data).hexdigest(), **(meta or {})}
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    print(json.dumps(manifest, indent=1))


if __name__ == "__main__":
    main()
