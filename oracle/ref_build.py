"""Build recipe for the reference's own CPU code (test infrastructure only).

Compiles, with g++ -O3 and the flags of forward/Acoustic_FD_by_ss/src/Makefile:14-24,
straight from the reference tree:

  oracle/_ref/afd_orig    forward/Acoustic_FD_by_ss/src/Acoustic_1order_FD.cpp, unmodified.
                          Reproduces the shipped record.dat / Snap.dat / Model.dat bit-exactly.
  oracle/_ref/afd_ref     The same file with the declared minimal configuration patch below,
                          so that the reference's own time loop can run other grids, models,
                          wavelets, sources and receiver lines (driven by AFD_* environment
                          variables; every default is the original hard-coded value).
  oracle/_ref/ricker      tools/ricker.cpp, unmodified (pins the Ricker helper, RIC:44).

The patched source is written only into oracle/_ref/ (git-ignored); nothing of the reference
source is stored in this repository except the short anchor strings the patch must find.

Declared patch (each anchor must match exactly once, otherwise the build fails):
  AFD:13       add env helpers after the PI macro (no arithmetic changes)
  AFD:28-36    NX/NZ/PML/Nt/dx/dz/dt read from AFD_NX ... AFD_DT (defaults 100/100/20/2000/10/10/0.0005)
  AFD:137-142  optional AFD_VP_FILE / AFD_DEN_FILE (padded Nx*Nz f32, x-major) overwrite Vp/DEN
  AFD:190      bottom sponge loop bound j<Nx -> j<Nz (latent out-of-bounds write when Nx != Nz)
  AFD:199-209  optional AFD_WAVELET_FILE (Nt f32) overwrites signal[]
  AFD:215-216  source cell from AFD_SX / AFD_SZ (defaults Nx/2, Nz/2)
  AFD:344      snapshot step from AFD_SNAP (default 500)
  AFD:358      Pall.dat dump switchable by AFD_PALL (default 1) -- pure file output
  AFD:377      receiver line: AFD_REC_Z >= 0 records P1[i][AFD_REC_Z] (horizontal line);
               default keeps the original vertical line P1[nx_location][i]
Arithmetic, loop order and update semantics of the time loop (AFD:237-380) are untouched.

Usage: python oracle/ref_build.py [--reference DIR]   (default: $SFD_REFERENCE, else /root/reference)
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
AFD_REL = "forward/Acoustic_FD_by_ss/src/Acoustic_1order_FD.cpp"
RIC_REL = "tools/ricker.cpp"

CXX = ["g++", "-O3"]
CXXFLAGS = ["-Wno-unused-result", "-fmax-errors=5"]
LINK = ["-fopenmp", "-lm"]

ENV_HELPERS = r'''
/* ---- configuration patch helpers (oracle/ref_build.py) ---- */
static int sfd_env_i(const char *k, int d) { const char *v = getenv(k); return v ? atoi(v) : d; }
static double sfd_env_f(const char *k, double d) { const char *v = getenv(k); return v ? atof(v) : d; }
static void sfd_env_read2d(const char *k, float **a, int n1, int n2)
{
    const char *fn = getenv(k);
    if (!fn) return;
    FILE *f = fopen(fn, "rb");
    if (!f) { fprintf(stderr, "cannot open %s\n", fn); exit(3); }
    for (int i = 0; i < n1; i++)
        if (fread(a[i], sizeof(float), n2, f) != (size_t)n2) { fprintf(stderr, "short read %s\n", fn); exit(3); }
    fclose(f);
}
static void sfd_env_read1d(const char *k, float *a, int n)
{
    const char *fn = getenv(k);
    if (!fn) return;
    FILE *f = fopen(fn, "rb");
    if (!f) { fprintf(stderr, "cannot open %s\n", fn); exit(3); }
    if (fread(a, sizeof(float), n, f) != (size_t)n) { fprintf(stderr, "short read %s\n", fn); exit(3); }
    fclose(f);
}
static int sfd_cached(int *slot, const char *k, int d) { if (*slot == -7) *slot = sfd_env_i(k, d); return *slot; }
static int sfd_pall_slot = -7, sfd_recz_slot = -7;
#define SFD_PALL() sfd_cached(&sfd_pall_slot, "AFD_PALL", 1)
#define SFD_REC_Z() sfd_cached(&sfd_recz_slot, "AFD_REC_Z", -1)
'''

# (anchor, replacement) pairs; the anchor must occur exactly once in the reference file.
PATCH = [
    ("#define PI 3.1415926\n", "#define PI 3.1415926\n" + ENV_HELPERS),
    ("NX  = 100;", "NX  = sfd_env_i(\"AFD_NX\", 100);"),
    ("NZ  = 100;", "NZ  = sfd_env_i(\"AFD_NZ\", 100);"),
    ("PML = 20;", "PML = sfd_env_i(\"AFD_PML\", 20);"),
    ("Nt  = 2000;", "Nt  = sfd_env_i(\"AFD_NT\", 2000);"),
    ("dx  = 10.0;", "dx  = sfd_env_f(\"AFD_DX\", 10.0);"),
    ("dz  = 10.0;", "dz  = sfd_env_f(\"AFD_DZ\", 10.0);"),
    ("dt  = 0.0005;", "dt  = sfd_env_f(\"AFD_DT\", 0.0005);"),
    ("            DEN[i][j]=2400.0;\n        }\n",
     "            DEN[i][j]=2400.0;\n        }\n"
     "    sfd_env_read2d(\"AFD_VP_FILE\", Vp, Nx, Nz);\n"
     "    sfd_env_read2d(\"AFD_DEN_FILE\", DEN, Nx, Nz);\n"),
    ("for(j=0;j<Nx;j++)", "for(j=0;j<Nz;j++)"),
    ("                    *exp(-PI*PI*freq*freq*(t-t1)*(t-t1));\n    }\n",
     "                    *exp(-PI*PI*freq*freq*(t-t1)*(t-t1));\n    }\n"
     "    sfd_env_read1d(\"AFD_WAVELET_FILE\", signal, Nt);\n"),
    ("nx_location=Nx/2;", "nx_location=sfd_env_i(\"AFD_SX\", Nx/2);"),
    ("nz_location=Nz/2;", "nz_location=sfd_env_i(\"AFD_SZ\", Nz/2);"),
    ("Snapshot=500;", "Snapshot=sfd_env_i(\"AFD_SNAP\", 500);"),
    ("if(k%10==0)", "if(SFD_PALL() && k%10==0)"),
    ("record[i-PML][k]=P1[nx_location][i];",
     "record[i-PML][k]=(SFD_REC_Z() >= 0) ? P1[i][SFD_REC_Z()] : P1[nx_location][i];"),
]


def patched_source(src: str) -> str:
    for old, new in PATCH:
        n = src.count(old)
        if n != 1:
            raise RuntimeError(f"patch anchor found {n} times (expected 1): {old!r}")
        src = src.replace(old, new)
    return src


def run(cmd):
    print(" ".join(cmd))
    subprocess.run(cmd, check=True)


def build(reference: str) -> None:
    afd = os.path.join(reference, AFD_REL)
    ric = os.path.join(reference, RIC_REL)
    if not os.path.isfile(afd):
        raise FileNotFoundError(afd)
    os.makedirs(OUT, exist_ok=True)
    # 1) unmodified reference, compiled from where it lies
    run(CXX + ["-c", afd, "-o", os.path.join(OUT, "afd_orig.o")] + CXXFLAGS)
    run(CXX + [os.path.join(OUT, "afd_orig.o"), "-o", os.path.join(OUT, "afd_orig")] + LINK)
    # 2) declared configuration patch, written only into oracle/_ref
    with open(afd, "rb") as f:
        # the reference file has CRLF line endings; anchors are written with LF
        src = f.read().decode("latin-1").replace("\r\n", "\n")
    dst = os.path.join(OUT, "afd_ref_patched.cpp")
    with open(dst, "wb") as f:
        f.write(patched_source(src).encode("latin-1"))
    run(CXX + ["-c", dst, "-o", os.path.join(OUT, "afd_ref.o")] + CXXFLAGS)
    run(CXX + [os.path.join(OUT, "afd_ref.o"), "-o", os.path.join(OUT, "afd_ref")] + LINK)
    # 3) Ricker tool, unmodified
    run(CXX + [ric, "-o", os.path.join(OUT, "ricker")] + CXXFLAGS + ["-lm"])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("SFD_REFERENCE", "/root/reference"))
    a = ap.parse_args()
    build(a.reference)


if __name__ == "__main__":
    sys.exit(main())
