// ORACLE -- test infrastructure only (tests/, bench.py cpu_baseline). Not part of the product.
// C ABI of the CPU restatements in oracle/*.cpp, loaded with ctypes by tests/oracle_lib.py.
#pragma once
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

// Acoustic v-p staggered grid, forward/Acoustic_FD_by_ss/src/Acoustic_1order_FD.cpp.
// Grid is the padded AFD grid (Nx = NX + 2 PML, Nz = NZ + 2 PML), arrays x-major, z fastest.
typedef struct {
    int nx, nz;      // padded grid
    int pml;         // sponge width (cells), AFD:30
    int nt;          // time steps
    float dx, dz, dt;
    int radius;      // stencil half-width: 8 = AFD's 16th order
    int sx, sz;      // source cell
    int nrec;        // receivers: record[r*nt + k] = P1[rec_x[r]][rec_z[r]] after the sponge
    const int* rec_x;
    const int* rec_z;
    int snap_step;   // step whose sponged Vx1 goes to snap_vx (AFD:345-355); -1 for none
} OracleAfdCfg;

int oracle_afd_sponge(int nx, int nz, int pml, float* absorb);
int oracle_afd_coeffs(int radius, float* c);
int oracle_afd_f32(const OracleAfdCfg* g, const float* vp, const float* den, const float* wavelet,
                   float* record, float* snap_vx, float* final_state);
int oracle_afd_f64(const OracleAfdCfg* g, const float* vp, const float* den, const float* wavelet,
                   double* record, double* snap_vx, double* final_state);
// FP64 misfit 0.5*sum (rec - obs)^2, its gradient w.r.t. Vp (padded grid) and w.r.t. the
// wavelet samples, and the FP64 records; obs and records are [nrec][nt].  Any output may be NULL.
int oracle_afd_gradient_f64(const OracleAfdCfg* g, const float* vp, const float* den, const float* wavelet,
                            const float* obs, double* misfit, double* grad_vp, double* dw, double* records);
void oracle_wavelet_afd(int nt, float dt, float freq, float* out);
void oracle_wavelet_ric(int nt, float dt, int f0, int delay, float* out);

#ifdef __cplusplus
}
#endif
