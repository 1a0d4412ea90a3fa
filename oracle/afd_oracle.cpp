// ORACLE -- test infrastructure only. CPU restatement of the reference's acoustic
// velocity-pressure staggered-grid time loop, used by tests/ and by bench.py's cpu_baseline
// leg as the checker. Never linked into, or called by, the product library.
//
// Follows forward/Acoustic_FD_by_ss/src/Acoustic_1order_FD.cpp (AFD):
//   coefficients            AFD:38-45 (radius 8); other radii use the staggered-grid Taylor
//                           coefficients of forward/Q_forward/..._subroutine_..._rotated.f90:9-28
//   sponge                  AFD:164-194 (with the bottom loop bound j<Nz, see AFD:190)
//   source injection        AFD:247-251
//   Vx, Vz, P updates       AFD:255-314 (same operation order and double promotions)
//   copy + sponge           AFD:317-340
//   snapshot / receivers    AFD:345-355, AFD:376-377 (receivers generalised to a cell list)
// Instantiated for T=float it is bit-exact with the reference built by g++ -O3 (no FMA);
// for T=double it is the FP64 oracle of the same discrete scheme (same float coefficients,
// model and wavelet, promoted).
// Build: oracle/Makefile (-O2 -ffp-contract=off).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace {

// AFD:38-45 (16th order, radius 8) and the Fortran `constant` module coefficients
// (QS:9-28) for radii 1, 2, 3, 4, 5. All are single-precision values, as in the reference.
int coeffs(int radius, float* c) {
    switch (radius) {
    case 8:
        c[0] = 1.2340911f; c[1] = -1.0664985e-1f; c[2] = 2.3036367e-2f; c[3] = -5.3423856e-3f;
        c[4] = 1.0772712e-3f; c[5] = -1.6641888e-4f; c[6] = 1.7021711e-5f; c[7] = -8.5234642e-7f;
        return 0;
    case 5:
        c[0] = 19845.0f / 16384.0f; c[1] = -735.0f / 8192.0f; c[2] = 567.0f / 40960.0f;
        c[3] = -405.0f / 229376.0f; c[4] = 35.0f / 294912.0f;
        return 0;
    case 4:
        c[0] = 1225.0f / 1024.0f; c[1] = -245.0f / 3072.0f; c[2] = 49.0f / 5120.0f; c[3] = -5.0f / 7168.0f;
        return 0;
    case 3:
        c[0] = 75.0f / 64.0f; c[1] = -25.0f / 384.0f; c[2] = 3.0f / 640.0f;
        return 0;
    case 2:
        c[0] = 9.0f / 8.0f; c[1] = -1.0f / 24.0f;
        return 0;
    case 1:
        c[0] = 1.0f;
        return 0;
    default:
        return -1;
    }
}

// AFD:164-194, sponge with overwrite semantics; the right/bottom loops use j<Nz.
void sponge(int Nx, int Nz, int PML, float* absorb) {
    for (int i = 0; i < Nx * Nz; i++) absorb[i] = 1.0f;
    for (int i = PML; i < Nx - PML; i++)
        for (int j = 0; j < PML; j++)
            absorb[i * Nz + j] = -0.38 * (PML - j - 1) * (PML - j - 1) / (1.0 * PML * PML) + 1;
    for (int i = PML; i < Nx - PML; i++)
        for (int j = Nz - PML; j < Nz; j++)
            absorb[i * Nz + j] = -0.38 * (j - Nz + PML) * (j - Nz + PML) / (1.0 * PML * PML) + 1;
    for (int i = 0; i < PML; i++)
        for (int j = 0; j < Nz; j++)
            absorb[i * Nz + j] = -0.38 * (PML - i - 1) * (PML - i - 1) / (1.0 * PML * PML) + 1;
    for (int i = Nx - PML; i < Nx; i++)
        for (int j = 0; j < Nz; j++)
            absorb[i * Nz + j] = -0.38 * (i - Nx + PML) * (i - Nx + PML) / (1.0 * PML * PML) + 1;
}

// Accumulation type of the stencil sums: float for the FP32 restatement (AFD sums in float),
// double for the FP64 oracle. The scale factors are double in both (AFD:259,276,293,302).
template <typename T>
int run_afd(const OracleAfdCfg* g, const float* vp, const float* den, const float* wavelet,
            T* record, T* snap_vx, T* final_state) {
    const int Nx = g->nx, Nz = g->nz, R = g->radius, Nt = g->nt;
    float cf[8];
    if (!g || Nx <= 2 * R || Nz <= 2 * R || Nt < 0 || coeffs(R, cf) != 0) return 1;
    if (g->sx < 0 || g->sx >= Nx || g->sz < 0 || g->sz >= Nz) return 1;
    const size_t n = (size_t)Nx * Nz;
    std::vector<T> P1(n, 0), P2(n, 0), Vx1(n, 0), Vx2(n, 0), Vz1(n, 0), Vz2(n, 0);
    std::vector<float> absorb(n);
    sponge(Nx, Nz, g->pml, absorb.data());
    T C[8];
    for (int m = 0; m < R; m++) C[m] = (T)cf[m];
    const float dt = g->dt, dx = g->dx, dz = g->dz;
    const int sidx = g->sx * Nz + g->sz;

    for (int k = 0; k < Nt; k++) {
        // AFD:247-251, float arithmetic: ((dt*DEN)*Vp)*signal
        P2[sidx] = P2[sidx] - (T)dt * (T)den[sidx] * (T)vp[sidx] * (T)wavelet[k];

        // AFD:255-269
#pragma omp parallel for schedule(static)
        for (int i = R; i < Nx - R; i++)
            for (int j = R; j < Nz - R; j++) {
                const size_t c = (size_t)i * Nz + j;
                T s = C[0] * (P2[c + Nz] - P2[c]);
                for (int m = 1; m < R; m++)
                    s = s + C[m] * (P2[c + (size_t)(m + 1) * Nz] - P2[c - (size_t)m * Nz]);
                Vx1[c] = (T)((double)Vx2[c] - (1.0 / (double)den[c]) * (double)(T)((T)dt / (T)dx) * (double)s);
            }
        // AFD:272-286
#pragma omp parallel for schedule(static)
        for (int i = R; i < Nx - R; i++)
            for (int j = R; j < Nz - R; j++) {
                const size_t c = (size_t)i * Nz + j;
                T s = C[0] * (P2[c + 1] - P2[c]);
                for (int m = 1; m < R; m++) s = s + C[m] * (P2[c + m + 1] - P2[c - m]);
                Vz1[c] = (T)((double)Vz2[c] - (1.0 / (double)den[c]) * (double)(T)((T)dt / (T)dz) * (double)s);
            }
        // AFD:289-314
#pragma omp parallel for schedule(static)
        for (int i = R; i < Nx - R; i++)
            for (int j = R; j < Nz - R; j++) {
                const size_t c = (size_t)i * Nz + j;
                T sx = C[0] * (Vx1[c] - Vx1[c - Nz]);
                for (int m = 1; m < R; m++)
                    sx = sx + C[m] * (Vx1[c + (size_t)m * Nz] - Vx1[c - (size_t)(m + 1) * Nz]);
                T sz = C[0] * (Vz1[c] - Vz1[c - 1]);
                for (int m = 1; m < R; m++) sz = sz + C[m] * (Vz1[c + m] - Vz1[c - m - 1]);
                const T kk = (T)den[c] * (T)vp[c] * (T)vp[c] * (T)dt;
                const double div = (1.0 / (double)dx) * (double)sx + (1.0 / (double)dz) * (double)sz;
                P1[c] = (T)((double)P2[c] - (double)kk * div);
            }
        // AFD:317-340: copy, then sponge all six arrays
        for (size_t c = 0; c < n; c++) {
            P2[c] = P1[c];
            Vx2[c] = Vx1[c];
            Vz2[c] = Vz1[c];
        }
        for (size_t c = 0; c < n; c++) {
            const T a = (T)absorb[c];
            Vx1[c] = Vx1[c] * a; Vx2[c] = Vx2[c] * a;
            Vz1[c] = Vz1[c] * a; Vz2[c] = Vz2[c] * a;
            P2[c] = P2[c] * a;   P1[c] = P1[c] * a;
        }
        // AFD:345-355
        if (snap_vx && k == g->snap_step)
            for (size_t c = 0; c < n; c++) snap_vx[c] = Vx1[c];
        // AFD:376-377, generalised to an arbitrary receiver list
        if (record)
            for (int r = 0; r < g->nrec; r++)
                record[(size_t)r * Nt + k] = P1[(size_t)g->rec_x[r] * Nz + g->rec_z[r]];
    }
    if (final_state) {
        std::memcpy(final_state, P1.data(), n * sizeof(T));
        std::memcpy(final_state + n, Vx1.data(), n * sizeof(T));
        std::memcpy(final_state + 2 * n, Vz1.data(), n * sizeof(T));
    }
    return 0;
}

}  // namespace

extern "C" {

int oracle_afd_sponge(int nx, int nz, int pml, float* absorb) {
    if (nx <= 0 || nz <= 0 || pml < 0) return 1;
    sponge(nx, nz, pml, absorb);
    return 0;
}

int oracle_afd_coeffs(int radius, float* c) { return coeffs(radius, c); }

int oracle_afd_f32(const OracleAfdCfg* g, const float* vp, const float* den, const float* wavelet,
                   float* record, float* snap_vx, float* final_state) {
    return run_afd<float>(g, vp, den, wavelet, record, snap_vx, final_state);
}

int oracle_afd_f64(const OracleAfdCfg* g, const float* vp, const float* den, const float* wavelet,
                   double* record, double* snap_vx, double* final_state) {
    return run_afd<double>(g, vp, den, wavelet, record, snap_vx, final_state);
}

// AFD:199-209: 50*(1-2 PI^2 f^2 (t-1/f)^2) exp(-PI^2 f^2 (t-1/f)^2), PI = 3.1415926 (AFD:13)
void oracle_wavelet_afd(int nt, float dt, float freq, float* out) {
    const double PI = 3.1415926;
    for (int i = 0; i < nt; i++) {
        float t = dt * i;
        float t1 = 1.0 / freq;
        out[i] = 50 * (1 - 2 * PI * PI * freq * freq * (t - t1) * (t - t1)) *
                 std::exp(-PI * PI * freq * freq * (t - t1) * (t - t1));
    }
}

// tools/ricker.cpp:44: (1-2(pi f0 (j-d) dt)^2) exp(-(pi f0 (j-d) dt)^2), pi = 3.1415926, f0 int
void oracle_wavelet_ric(int nt, float dt, int f0, int delay, float* out) {
    const double pi = 3.1415926;
    for (int j = 0; j < nt; j++)
        out[j] = (1 - 2 * (pi * f0 * (j - delay) * dt) * (pi * f0 * (j - delay) * dt)) *
                 std::exp(-(pi * f0 * (j - delay) * dt) * (pi * f0 * (j - delay) * dt));
}

}  // extern "C"
