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
// Visco-elastic RSG modelling of one shot, forward/Q_forward (flat surface).  The model arrays
// are the interior (nz, nx) Fortran arrays (x-major, z fastest); records are [nxe][nt].
typedef struct {
    int nx, nz;                    // interior model size (nx_v, nz_v)
    float dx, dz, dt, f0;
    int nt;                        // record length (samples after the decay steps)
    int npxn, npxp, npzn, npzp;    // pad cells, nint(pml/d)+1 (QM:105-108)
    int ixmine, ixmaxe;            // aperture window (QM:128-129), 1-based model columns
    int isxe, isze;                // source cell in the padded grid, 1-based (QS:374-375)
    int nrz0;                      // receiver row offset, nint(rz0/dz)+1 (QM:112)
    int q_override;                // 1: Q = 1e5 everywhere (QM:418-419)
} OracleQCfg;
int oracle_q_f32(const OracleQCfg* c, const float* vp, const float* vs, const float* rho, const float* qp,
                 const float* qs, float* rec1, float* rec2, float* final_sxx);
int oracle_q_f64(const OracleQCfg* c, const float* vp, const float* vs, const float* rho, const float* qp,
                 const float* qs, double* rec1, double* rec2, double* final_sxx);
// Isotropic elastic standard staggered grid, 'abc' mode, flat surface (forward/yang_version_2016_2_2,
// oracle/iso_oracle.cpp).  Interior model (nz, nx) Fortran order = x-major float arrays; cells are
// 1-based as in the Fortran; records [nxe][nt], record1 = vx, record2 = vz.
typedef struct {
    int nx, nz;                    // interior model
    float dx, dz, dt, f0;
    int nt;                        // recorded samples (the loop runs nt + idecay steps)
    int npxn, npxp, npzn, npzp;    // sponge cells, nint(pp/dx) + 1 (YPRI:26-29)
    int ixmine, ixmaxe;            // window, 0-based model columns (i_ori = i + ixmine)
    int isxe, isze;                // source cell in the padded window, 1-based
    int nrz0;                      // receiver row offset below itopo, nint(rz0/dz) + 1
    int idecay;                    // nint(decay/dt): steps before the first recorded sample
    int rgau;                      // Gaussian window half-width (2 rgau - 1 cells), the .par's rgau
    int fsbc;                      // 0: 'abc' mode; 1: 'fsbc' mode, free surface at row itopo (1-based)
    const float* topo;             // surface depth (m) per model column (nx values), NULL: flat;
                                   // itopo = nint(topo/dz) + npzn per window column (YPUB:270-272)
} OracleIsoCfg;
// VTI pseudo-acoustic modeller (de-multiple/convolution_srm/vti_qa_2d_c3_demo1): the reference's
// parameters of one shot.  Model arrays [nx_v][nz_v] x-major; grid numbers 1-based as in the
// Fortran (nsx, nsz0 and nrz0 from VM:145-147, xmin / xmax the shot's aperture columns, VM:162-163);
// record[trace][nt] for the xmax - xmin + 1 traces.
typedef struct {
    int nx_v, nz_v, nt;
    float dx, dz, dt, f0;
    int nx_bound_l, nx_bound_r, nz_bound_u, nz_bound_d;  // PML cells (VM:136-141)
    int order_explicit, order_pml_1st, order_pml_2nd;    // 10, 9 or 10, 10
    int nsx, nsz0, nrz0, xmin, xmax;
} OracleVtiCfg;
// the FD coefficients of VS:1264-1472 (first = 0: coefficient_2nd(order), 1: coefficient_1st)
int oracle_vti_coef_f32(int order, int first, float* out);
int oracle_vti_coef_f64(int order, int first, double* out);
int oracle_vti_f32(const OracleVtiCfg* c, const float* vz, const float* eps, const float* delta, float* record);
int oracle_vti_f64(const OracleVtiCfg* c, const float* vz, const float* eps, const float* delta, double* record);
// the five arrays of the time loop after substagger and the PML smoothing (YPUB:323-634):
// busg2e, busg1e, lambmusg, lambsg, musge, each [NX][NZ] of the padded window
int oracle_iso_prepare_f32(const OracleIsoCfg* c, const float* vp, const float* vs, const float* rho, float* out);
int oracle_iso_f32(const OracleIsoCfg* c, const float* vp, const float* vs, const float* rho, float* rec1, float* rec2,
                   float* final_vx);
int oracle_iso_f64(const OracleIsoCfg* c, const float* vp, const float* vs, const float* rho, double* rec1,
                   double* rec2, double* final_vx);
// 3-D velocity-pressure staggered grid (the AFD scheme with a y axis; no reference counterpart).
// Arrays are [x][y][z], z fastest; record[r*nt + k] = P after step k's sponge at receiver r.
typedef struct {
    int nx, ny, nz, pml, nt, radius;
    float dx, dy, dz, dt;
    int sx, sy, sz;
    int nrec;
    const int* rec_x;
    const int* rec_y;
    const int* rec_z;
    float den_c;     // density where den is NULL
} OracleAfd3Cfg;
int oracle_afd3d_sponge(int nx, int ny, int nz, int pml, float* absorb);
int oracle_afd3d_f32(const OracleAfd3Cfg* g, const float* vp, const float* den, const float* wavelet, float* record,
                     float* final_p);
int oracle_afd3d_f64(const OracleAfd3Cfg* g, const float* vp, const float* den, const float* wavelet, double* record,
                     double* final_p);
// FP64 misfit, d misfit / d vp and d misfit / d wavelet of the 3-D scheme and its FP64 records
// ([nrec][nt]); obs NULL computes the records only.
int oracle_afd3d_gradient_f64(const OracleAfd3Cfg* g, const float* vp, const float* den, const float* wavelet,
                              const float* obs, double* misfit, double* grad_vp, double* dw, double* records);
// FP64 misfit gradient of the viscoacoustic (vs = 0) scheme on a padded grid (np sponge cells per
// side, arrays x-major): records [nrec][nt], d/dvp and d/d(1/Q) per cell, d/dw per sample.
typedef struct {
    int nx, nz, np;
    float dx, dz, dt, f0;
    int nt, sx, sz;        // steps, source cell (0-based)
    int nrec;
    const int* rec_x;
    const int* rec_z;
} OracleQGradCfg;
int oracle_q_gradient_f64(const OracleQGradCfg* c, const float* vp, const float* rho, const float* q,
                          const float* wavelet, const float* obs, double* misfit, double* grad_vp,
                          double* grad_invq, double* dw, double* records);
void oracle_wavelet_afd(int nt, float dt, float freq, float* out);
void oracle_wavelet_ric(int nt, float dt, int f0, int delay, float* out);

#ifdef __cplusplus
}
#endif
