"""Builds the native library seismic_code_github_b200/libseisfd.so (sm_100a) and the host
programs in seismic_code_github_b200/bin/.

    python -m seismic_code_github_b200.build [--verbose-ptxas]

nvcc compiles every .cu/.cpp in csrc/ for sm_100a only (-gencode arch=compute_100a,code=sm_100a);
objects go to _build/ (git-ignored) and the shared library is placed in-tree so that it travels
with the source tree.
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(ROOT, "_build", "obj")
LIB = os.path.join(PKG, "libseisfd.so")
BIN = os.path.join(PKG, "bin")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-I", os.path.join(ROOT, "include"),
          "--expt-relaxed-constexpr", "-ccbin", "g++"]
LIB_SOURCES = ["api.cu", "acoustic2d.cu", "acoustic2d_fma.cu", "acoustic2d_march.cu", "adjoint2d.cu", "viscoac2d.cu", "viscoac2d_fast.cu", "q_adjoint2d.cu", "viscoel2d.cu", "elastic2d.cu", "vti2d.cu",
               "records.cu",
               "helpers.cpp", "noalloc.cu", "acoustic3d.cu", "snapshots.cu",
               "fileio.cpp"]
OPTIONAL_SOURCES = []
PROGRAMS = {"afd_fd": "cli_afd.cpp", "q_forward": "cli_qforward.cpp", "iso_forward": "cli_isoforward.cpp",
            "vti_forward": "cli_vtiforward.cpp"}


def _sources():
    srcs = [s for s in LIB_SOURCES]
    srcs += [s for s in OPTIONAL_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    return srcs


def _compile(src: str, ptxas_v: bool) -> str:
    out = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    deps = [path, os.path.join(CSRC, "sfd_internal.h"), os.path.join(ROOT, "include", "seisfd.h")]
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps if os.path.exists(d)) \
            and not ptxas_v:
        return out
    cmd = [NVCC] + ARCH + COMMON + ["-c", path, "-o", out]
    if ptxas_v and src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    if src.endswith(".cpp"):
        cmd = [NVCC] + COMMON + ["-x", "cu"] + ARCH + ["-c", path, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if ptxas_v:
        sys.stderr.write(r.stderr)
    return out


def build(ptxas_v: bool = False, programs: bool = True) -> str:
    if shutil.which(NVCC) is None and not os.path.exists(NVCC):
        raise RuntimeError("nvcc not found: the native library cannot be built")
    os.makedirs(OBJ, exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, ptxas_v), srcs))
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart", "-Xcompiler", "-fPIC"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    if programs:
        os.makedirs(BIN, exist_ok=True)
        for name, src in PROGRAMS.items():
            path = os.path.join(CSRC, src)
            if not os.path.exists(path):
                continue
            exe = os.path.join(BIN, name)
            cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), path, "-o", exe,
                   "-L", PKG, "-lseisfd", "-Wl,-rpath,$ORIGIN/.."]
            subprocess.run(cmd, check=True)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose_ptxas))


if __name__ == "__main__":
    main()
