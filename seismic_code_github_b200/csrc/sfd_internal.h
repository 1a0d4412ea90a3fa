// Internal definitions shared by the host library and the kernels.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/seisfd.h"

namespace sfd {

constexpr int kMaxRadius = 8;

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) once per device: the attribute belongs to the
// device, so a kernel first launched on a second GPU of the process needs it set there as well.
// `done` is the calling launcher's static table (one flag per device ordinal).
constexpr int kMaxDevices = 64;
inline cudaError_t smem_attr_once(const void* fn, int bytes, bool* done) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const bool tracked = dev >= 0 && dev < kMaxDevices;
    if (tracked && done[dev]) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess && tracked) done[dev] = true;
    return e;
}
// Both 2-D acoustic step kernels work on the same 64 x 64 tiles, so they share the field
// layout and the per-tile receiver tables.
constexpr int kTileX = 64;
constexpr int kTileZ = 64;

// Per-shot descriptor in device memory (one entry per shot, indexed by shot id).
struct ShotDev {
    int nx;            // shot-local padded width (aperture)
    int x0;            // model column of shot column 0
    int nt;            // steps
    int sx, sy, sz;    // source cell
    int nrec;
    long long rec_base;   // offset (floats) of this shot's [nt][nrec] block in the record buffer
    int rec_list;         // offset of this shot's receivers in rec_x/rec_z
    int wav_off;          // offset of this shot's wavelet
    int tile_rec_base;    // offset of this shot's per-tile receiver CSR (ntiles + 1 entries)
    float inj_scale;      // ((dt * den_src) * vp_src), float, AFD:250 order
    // viscoacoustic scheme: Gaussian source stamp (QS:1340-1444), box of non-zero weights
    int stamp_off;        // offset of the box's weights (x-major, z fastest) in the stamp array
    int stamp_x0, stamp_z0, stamp_w, stamp_h;
};

// Field storage of one 2-D scheme: per shot a (cols x pitch) slab, z fastest, with zero ghost
// margins of gx columns and gz rows so halo reads never leave the allocation.
struct Layout2D {
    int gx, gz;        // ghost margins
    int pitch;         // floats per column (multiple of 32)
    int cols;          // columns incl. ghosts
    long long shot_stride;  // floats per shot
    int ntx, ntz;      // tiles per shot along x and z
    int tx, tz;        // tile shape
};

// Arguments of the viscoacoustic kernels (viscoac2d.cu): in-place fields, no ping-pong.
struct QArgs {
    float* vx; float* vz;                 // QS vxx (= vx), vzz (= vz) for vs = 0
    float* sx; float* sz; float* sr;      // QS strxxx, strxxz, strxxr (= strzz parts for vs = 0)
    float* rx; float* rz; float* rr;      // QS rxxx, rxxz, rxxr
    Layout2D L;
    int nz, npx, npz;                     // grid depth, pad cells (QS npxn = npxp, npzn = npzp)
    const float* busg;                    // 1/averaged density (QS:434-469)
    const float* p1;                      // lambmu * taupstinss (QS:473-551)
    const float* p2;                      // lambmu * (taupstinss - 1)
    int mpitch, nx_model;
    float dt, f_mem;                      // f_mem = dt * (-1 * rtaustss)
    float hx, hz;                         // 0.5/dx, 0.5/dz
    float dz2;                            // dz*dz
    float a[5];                           // a100..a104
    const float* spg;                     // sponge tables: xn, xp, zn, zp, 1xn, 2xp, 1zn, 2zp
    int spg_stride;
    const ShotDev* shots;
    const int* slot_to_shot;
    const float* wavelets;
    const float* stamps;
    const int* rec_x; const int* rec_z;
    const int* tile_rec_ptr; const int* tile_rec_idx;
    float* records;                       // [nt][nrec] per shot: strzz (= strxx) at the receivers
    int step;
    float* d1_out;                        // optional: Dx1 vx of this step (field layout), for the gradient
    float* d4_out;                        // optional: Dz1 vz of this step
};
cudaError_t viscoac2d_launch_step(const QArgs& a, int active, cudaStream_t st);

// Default (fast, FMA) viscoacoustic step (viscoac2d_fast.cu): merged sigma and r everywhere,
// split parts in the sponge bands only (q.sx .. q.rr); q.vx / q.vz unused.
struct QFastArgs {
    CUtensorMap tm_s;                 // this step's input sigma (box of viscoac2d_fast_boxes)
    QArgs q;
    const float* s_in; float* s_out;  // merged stress, ping-pong
    const float* vx_in; float* vx_out;
    const float* vz_in; float* vz_out;
    float* r;                         // merged memory variable, in place
    float* e1; float* e4;             // 0.5/dx Dx1 vx and 0.5/dz Dz1 vz of the cells near the bands
    int* err_flag;                    // set by a CTA whose bounded wait ran out
};
// one step of the active shots: the step kernel (one CTA per shot, 64-wide z strip and segment of
// `seg` columns), then the band kernel (one CTA per shot and column, nx_max >= every active nx)
cudaError_t viscoac2d_fast_launch(const QFastArgs& a, int active, int seg, int nx_max, cudaStream_t st, bool pdl);
// TMA box extents (z, x) of the sigma loads
void viscoac2d_fast_boxes(int box_s[2]);

// Visco-elastic split fields (viscoel2d.cu), in the order of their slabs in the state buffer.
enum EField {
    E_VXX, E_VXZ, E_VZX, E_VZZ,
    E_SXXX, E_SXXZ, E_SXXR, E_SZZX, E_SZZZ, E_SZZR, E_SXZX, E_SXZZ, E_SXZR,
    E_RXXX, E_RXXZ, E_RXXR, E_RZZX, E_RZZZ, E_RZZR, E_RXZX, E_RXZZ, E_RXZR,
    E_NFIELDS
};

// Arguments of the visco-elastic kernels (viscoel2d.cu): 22 in-place split fields.
struct EArgs {
    float* f[E_NFIELDS];
    Layout2D L;
    int nz, npx, npz;
    const float* busg;                    // 1/averaged density (QS:434-469)
    const float* q1; const float* q2; const float* q3;  // lambda tau_p, lambda tau_p - 2 mu tau_s, mu tau_s
    const float* m1; const float* m2; const float* m3;  // the same with tau - 1 (memory variables)
    int mpitch, nx_model;
    float dt, f_mem, hx, hz, dz2;
    float a[5];
    const float* spg;
    int spg_stride;
    const ShotDev* shots;
    const int* slot_to_shot;
    const float* wavelets;
    const float* stamps;
    const int* rec_x; const int* rec_z;
    const int* tile_rec_ptr; const int* tile_rec_idx;
    float* records;                       // strzz (record1), [nt][nrec] per shot
    float* records2;                      // strxx (record2)
    int step;
};
cudaError_t viscoel2d_launch_step(const EArgs& a, int active, cudaStream_t st);
// QS:434-551 with vs: busg and the six stress coefficients on the padded grid, and rtaustss
void viscoel2d_prepare(int nx, int nz, const float* vp, const float* vs, const float* rho, const float* qp,
                       const float* qs, float f0, float* busg, float* q1, float* q2, float* q3, float* m1, float* m2,
                       float* m3, float* rtau_out);

// Isotropic elastic standard-staggered-grid split fields (elastic2d.cu), in slab order:
// forward/yang_version_2016_2_2 vxx vxz vzx vzz strxxx strxxz strzzx strzzz strxzx strxzz.
enum IField { I_VXX, I_VXZ, I_VZX, I_VZZ, I_SXXX, I_SXXZ, I_SZZX, I_SZZZ, I_SXZX, I_SXZZ, I_NFIELDS };

// Arguments of the isotropic elastic kernels (elastic2d.cu): ten in-place split fields.
struct IArgs {
    float* f[I_NFIELDS];
    Layout2D L;
    int nz, npx, npz;
    // prepared model (YPUB:323-634), row z = 0 of column 0: busg2e, busg1e, lambmusg, lambsg, musge
    const float* b2e; const float* b1e; const float* lm2; const float* lam; const float* mue;
    int mpitch, nx_model;
    float dt, dtdx, dtdz, dz2;
    float a[5];
    float cr[4][4];                       // M-term staggered coefficients, M = 1..4 (YMOD:7-20)
    int fs;                               // 1: free surface (fsbc mode), 0: abc mode
    const int* itopo;                     // per prepared-model column: the reference's itopo (1-based
                                          // surface row; abc updates from row itopo - npz - 1, 0-based)
    const float* spg;                     // spgxn spgxp spgzn spgzp spg1xn spg2xp spg1zn spg2zp
    int spg_stride;
    const ShotDev* shots;
    const int* slot_to_shot;
    const float* wavelets;
    const float* stamps;
    const int* rec_x; const int* rec_z;
    const int* tile_rec_ptr; const int* tile_rec_idx;
    float* records;                       // vx (record1), [nt][nrec] per shot
    float* records2;                      // vz (record2)
    int step;
};
// One step: the velocity and stress kernels, and in fsbc mode the surface kernel (YPUB:938-976
// calfsbcv, YPUB:1009-1024 calfsbcstrxz); *launches receives the kernel count.
cudaError_t elastic2d_launch_step(const IArgs& a, int active, int nx_max, cudaStream_t st, int* launches);
// YPUB:323-547 on one window (x-major, z fastest): substagger and the refill of the rows above
// itopo(x) (0-based rows < itopo - 1 take row itopo - 1); out: busg2e, busg1e, lambmusg, lambsg,
// musge.  Returns false on a zero density (YPUB:370, 400).
bool elastic2d_prepare(int nx, int nz, const float* vp, const float* vs, const float* rho, const int* itopo,
                       float* b2e, float* b1e, float* lm2, float* lam, float* mue);
// YPUB:1470-1501: the (2 rgau - 1)^2 Gaussian table (sigma 2 cells), normalised by its sum, in
// Fortran order gc(idx1, idx2) = out[(idx2 - 1) * w + idx1 - 1]; *lo / *hi: 0-based index range
// holding every non-zero weight (the same along both axes).
void elastic2d_gauss_table(int rgau, std::vector<float>* out, int* lo, int* hi);
// YPUB:1429-1466: the window of the source's Gaussian stamp clipped to the grid, box of
// non-zero weights (x0, z0, w, h) and the weights (x-major, z fastest).
void elastic2d_stamp(int nx, int nz, int sx, int sz, int rgau, const std::vector<float>& gc, int* box,
                     std::vector<float>* out);
// YPUB:592-634 on the device: the in-place Gaussian smoothing of rows z < itopo(x) of the five
// prepared arrays of every window (one sequential chain per array and window, serial order).
// arrays: five device pointers to row z = 0 of column 0 (column pitch mpitch, `ghost` replicated
// rows above z = 0, refreshed afterwards); itopo_dev: per prepared column; win: nwin (start
// column, width) pairs.
cudaError_t elastic2d_smooth(float* const arrays[5], int mpitch, int ghost, int nz, const int* itopo_dev,
                             const int* win_host, int nwin, const std::vector<float>& gc, int rgau, int lo, int hi,
                             cudaStream_t st);

// Arguments of the viscoacoustic adjoint kernels (q_adjoint2d.cu): adjoint fields in place.
struct QAdjArgs {
    float* avx; float* avz;               // adjoints of vx, vz
    float* asx; float* asz; float* asr;   // adjoints of sx, sz, sr
    float* arx; float* arz; float* arr;   // adjoints of rx, rz, rr
    float* qx; float* qz;                 // dt b vx^, dt b vz^ of the current step (halo exchange)
    const float* d1; const float* d4;     // Dx1 vx, Dz1 vz of the forward step being transposed
    float* g1; float* g2;                 // per-shot imaging sums for p1 and p2 (field layout)
    Layout2D L;
    int nz, npx, npz;
    const float* busg; const float* p1; const float* p2;  // prepared model (row z = 0 of column 0)
    int mpitch, nx_model;
    float dt, f_mem, hx, hz, dz2;
    float a[5];
    const float* spg;
    int spg_stride;
    const ShotDev* shots;
    const int* slot_to_shot;
    const float* stamps;
    const float* res;                     // residuals, [nt][nrec] per shot at ShotDev::rec_base
    const int* rec_x; const int* rec_z;
    const int* tile_rec_ptr; const int* tile_rec_idx;
    float* lam_src;                       // [shot][nt_max]: d misfit / d wavelet sample
    int nt_max;
    int step;
};
// adjoint of forward step a.step for the active shots (two launches)
cudaError_t q_adjoint_launch_step(const QAdjArgs& a, int active, cudaStream_t st);
// adjoint initial state: sx^, sz^, sr^ += residual of each shot's last step at its receivers
cudaError_t q_adjoint_launch_init(const QAdjArgs& a, int first_shot, int nshot, int nrec_max, cudaStream_t st);
// model-grid d misfit / d vp and d misfit / d (1/Q) from the per-shot double imaging sums
cudaError_t q_launch_gradient_reduce(const double* acc1, const double* acc2, const Layout2D& L, const ShotDev* shots,
                                     const int* ap_x0, int nshot, const float* vp, const float* p1, const float* p2,
                                     int mpitch, int nx_model, int nz, double dt, double f, double kappa,
                                     double* grad_vp, double* grad_invq, cudaStream_t st);
// host preparation, QS:434-551: busg, p1, p2 on the padded grid and rtaustss
void viscoac2d_prepare(int nx, int nz, const float* vp, const float* rho, const float* q, float f0, float* busg,
                       float* p1, float* p2, float* rtau);
// QS:555-605 cosine sponge tables (8 arrays of stride npx+1 / npz+1 packed with `stride`)
void viscoac2d_sponge_tables(int npx, int npz, float dx, float dz, int stride, float* out);
// QS:1398-1444 normalised Gaussian over an n1 x n2 grid, non-zero box around the source:
// returns the box (x0, z0, w, h) and appends its weights (x-major) to `out`
void viscoac2d_stamp(int nx, int nz, int sx, int sz, int* box, std::vector<float>* out);

// Arguments of the acoustic 2-D step kernels (passed by value; pointers are device memory).
struct Acou2DArgs {
    // TMA descriptors of this step's input fields (3-D: z, column, shot), used by the FMA kernel
    CUtensorMap tm_p, tm_vx, tm_vz;
    // the same fields with the boxes of the x-marching kernel (acoustic2d_march.cu)
    CUtensorMap tm_mp, tm_mvx, tm_mvz;
    int* err_flag;          // set to 1 by a CTA whose bounded wait ran out (SFD_ERR_TIMEOUT)
    // test hook of the bounded waits (sfd_test_wait_timeout): CTA test_cta of step test_step
    // issues no box loads and gives up its waits after test_wait_ns; test_cta < 0: off
    int test_cta, test_step;
    unsigned long long test_wait_ns;
    const float* p_in;  float* p_out;
    const float* vx_in; float* vx_out;
    const float* vz_in; float* vz_out;
    Layout2D L;
    int nz;                 // padded grid nz (same for every shot)
    int pml;
    const float* vp;        // model, (nx_model x mpitch)
    const float* den;       // NULL for constant density
    int mpitch;
    int nx_model;
    float den_c;            // constant density
    float dt;
    float dtdx, dtdz;       // float(dt/dx), float(dt/dz) (AFD:259, 276)
    double rdx_d, rdz_d;    // 1.0/dx, 1.0/dz in double (AFD:293, 302)
    double bx_d, bz_d;      // (1.0/den_c)*(dt/dx) in double, constant density
    float bx_f, bz_f;       // float versions for the fast path
    float rdx_f, rdz_f;
    float coef[kMaxRadius];
    float2 coef2[kMaxRadius];  // the same coefficients as (c, c) pairs: operands of paired FP32 math
    float sponge[256];      // sponge profile tab[q] = 1 - 0.38 q^2 / pml^2, q < pml (AFD:164-194)
    const ShotDev* shots;
    const int* slot_to_shot;   // active-slot -> shot id (shots sorted by nt, longest first)
    const float* wavelets;
    const int* rec_x; const int* rec_z;
    const int* tile_rec_ptr;   // per shot: ntiles + 1 offsets into tile_rec_idx
    const int* tile_rec_idx;   // receiver index within the shot
    // FMA kernel's CTA numbering: tile_major 0 = CTA t takes position k = t % T of slot t / T
    // (T tiles per shot), 1 = position k = t / active of slot t % active; position k is tile
    // tile_order[k] (tile k when tile_order is NULL)
    int tile_major;
    const int* tile_order;
    int l2_ahead;              // one-tile-per-CTA schedule: CTA t prefetches CTA t + l2_ahead's
                               // boxes into L2 (0: no prefetch)
    float* records;            // [nt][nrec] per shot at ShotDev::rec_base
    int step;
    float* div_out;            // optional: D = rdx S-x Vx + rdz S-z Vz of this step (field layout)
    float* src_pre;            // optional, per shot: P at the source cell before the next step's
                               // injection (the value AFD holds there after the sponge)
    // Adjoint mode of the FMA kernel (acoustic2d_fma_launch with adj = true): the P, Vx, Vz slots
    // hold the adjoint state nu = M K a Q (K = DEN Vp^2 dt, a the sponge, M the update mask),
    // X = a M X' and Z = a M Z' of adjoint step `step` (adjoint2d.cu states the recurrence).
    const float* adj_div;      // D_k of the forward step being transposed (field layout)
    float* adj_g;              // imaging sum, field layout: g += nu_old D_k
    const float* adj_res;      // residuals [nt][nrec] per shot at ShotDev::rec_base
    float* adj_lam;            // [shot][nt_max]: adjoint of P at the source cell
    int nt_max;
    float adj_cx, adj_cz;      // dtdx/den_c, dtdz/den_c (constant density), 1 with variable density
    float adj_xs, adj_zs;      // dx/dt, dz/dt: X = a den (dx/dt) (staged value) with variable density
};

// residual = pred - obs (both [nt][nrec] per shot), misfit += 0.5 sum residual^2 (double)
cudaError_t launch_residual(const float* pred, const float* obs, float* res, long long n, double* misfit,
                            cudaStream_t st);
// records [nrec][nt] per shot -> [nt][nrec] per shot
cudaError_t launch_records_transpose_in(const float* rec_nt, float* rec_tn, const ShotDev* shots, int nshot,
                                        int nrec_max, int nt_max, cudaStream_t st);
// adjoint initial state: nu(shot, buffer nt & 1) += M a K res[nt-1] at the receivers
cudaError_t launch_adjoint_init(float* q0, float* q1, const Acou2DArgs& a, int radius, int first_shot, int nshot,
                                int nrec_max, cudaStream_t st);
// acc (double) += seg (float) over n values
cudaError_t launch_accumulate(double* acc, const float* seg, long long n, cudaStream_t st);
// grad_model[x][z] = -(2 / vp) * sum over shots of acc_s(x - ap_x0_s, z)
cudaError_t launch_gradient_reduce(const double* acc, const Layout2D& L, const ShotDev* shots, int nshot,
                                   const float* vp, int mpitch, int nx_model, int nz, double* grad_model,
                                   cudaStream_t st);

// Host-side launchers (acoustic2d.cu).
struct Acou2DPlan {
    int radius;
    int tx, tz, threads;
    size_t smem_bytes;
    int gz;      // z ghost margin the step kernels need (multiple of 4)
    int stages;  // FMA tile kernel schedule (1 or 2)
    int seg;     // > 0: forward steps run the x-marching kernel with segments of `seg` columns
    bool forced; // seg set by SFD_MARCH_SEG: x-marching even where its grid does not fill the device
};
// Model arrays on the device carry this many replicated rows above z = 0 and below z = nz - 1
// so that vectorised halo reads stay inside the allocation and see finite values.
constexpr int kModelGhostZ = 16;
bool acoustic2d_plan(int radius, Acou2DPlan* plan);
cudaError_t acoustic2d_launch_step(const Acou2DPlan& plan, const Acou2DArgs& a, int active_shots,
                                   bool exact, bool varden, cudaStream_t st);
// stages: 1 = one tile per CTA, two CTAs per SM; 2 = persistent CTAs with double-buffered TMA.
// adj: run the adjoint of step a.step instead (the adj_* arguments).
cudaError_t acoustic2d_fma_launch(int radius, const Acou2DArgs& a, int active, bool varden, int stages,
                                 cudaStream_t st, bool adj = false);
int acoustic2d_fma_gz(int radius);
// Forward step of the FMA scheme on the x-marching kernel (bit-identical to the tile kernel):
// one CTA per (shot, 64-wide z strip, segment of seg_cols columns), seg_cols a multiple of 16.
// adj: the adjoint of step a.step (the adj_* arguments, as acoustic2d_fma_launch's adjoint mode).
cudaError_t acoustic2d_march_launch(int radius, const Acou2DArgs& a, int active, bool varden, int seg_cols,
                                   cudaStream_t st, bool pdl, bool adj = false);
// TMA box extents (z, x) of the x-marching kernel's P, Vx and Vz loads.
void acoustic2d_march_boxes(int box_p[2], int box_vx[2], int box_vz[2]);
// Whether an x-marching launch of `active` shots fills one wave of the device (four CTAs per SM);
// with fewer CTAs (one shot of the per-shot baseline, the last shots of an uneven batch) the tile
// kernel, which gives the same bits, runs instead.
bool acoustic2d_march_fills(const Layout2D& L, int active, int seg_cols);
inline bool acoustic2d_use_march(const Acou2DPlan& plan, const Layout2D& L, int active) {
    return plan.seg > 0 && (plan.forced || acoustic2d_march_fills(L, active, plan.seg));
}
// Forward step of the default (FMA) scheme with the plan's kernel: x-marching when plan.seg > 0
// and the launch fills the device, else the tile kernel with plan.stages.
cudaError_t acoustic2d_fwd_launch(const Acou2DPlan& plan, int radius, const Acou2DArgs& a, int active, bool varden,
                                  cudaStream_t st);
// Programmatic dependent launch of consecutive step kernels (SFD_PDL=0 turns it off).
bool pdl_enabled();
// TMA box extents (z, x) the FMA kernel loads for P, Vx and Vz at this radius.
void acoustic2d_fma_boxes(int radius, int box_p[2], int box_vx[2], int box_vz[2]);
cudaError_t acoustic2d_launch_inject0(const Acou2DArgs& a, int nshot, bool exact, cudaStream_t st);
cudaError_t launch_records_transpose(const float* rec_tn, float* rec_nt, const ShotDev* shots, int nshot,
                                     int nrec_max, int nt_max, cudaStream_t st);
cudaError_t launch_nan_scan(const float* rec, long long n, int* flag, cudaStream_t st);
// source cell of one shot for the gradient's source term: model index and -(dt) * DEN there
struct GradSrc {
    long long mi;
    double scale;
};
// grad[mi_s] += scale_s * sum_k lam[s][k] w_s[k] for every shot, in shot and sample order
cudaError_t launch_grad_source(double* grad, const GradSrc* src, const ShotDev* shots, int nshot, const float* lam,
                               int nt_max, const float* wav, cudaStream_t st);
// out[i] = (float) in[i]
cudaError_t launch_to_float(const double* in, float* out, long long n, cudaStream_t st);

// ---- wavefield snapshots (snapshots.cu) ----
struct SnapArgs {
    const float* f[3];          // split parts of the field, summed in order (nsum = 1, 2 or 3)
    int nsum;
    Layout2D L;
    int nz, pml;
    int ztop;                   // first interior row (pml; the free surface's top pad in fsbc mode)
    const ShotDev* shots;
    const int* slot_to_shot;
    const float* src_pre;       // acoustic P: value at the source cell before the next injection
    int step, index;            // step just completed, snapshot number
    float* out;                 // per shot at shot_off[shot]: [snapshot][nx_shot - 2 pml][nz - ztop - pml]
    const long long* shot_off;
};
cudaError_t launch_snapshot(const SnapArgs& a, int active, int nx_max, cudaStream_t st);

// ---- 3-D acoustic scheme (acoustic3d.cu) ----
// Field storage: per shot a dense [x][y][pitch] block, z fastest, pitch = nz rounded up to a
// multiple of 4 (16-byte rows for the TMA strides and float4 accesses).  No ghost cells: the
// tensor maps have the exact grid extents, so halo boxes read zeros outside the grid.
constexpr int kTile3Y = 32;
constexpr int kTile3Z = 32;
struct Layout3D {
    int nx, ny, nz;
    int pitch;
    long long xstride;      // ny * pitch
    long long shot_stride;  // nx * ny * pitch
    int nty, ntz;           // tiles per x-plane
};
struct Acou3DArgs {
    CUtensorMap tm_p, tm_vy, tm_vz;   // 4-D maps (z, y, x, shot) of this step's input P, Vy, Vz
    int* err_flag;
    Layout3D L;
    const float* p_in; const float* vx_in;
    float* p_out; float* vx_out; float* vy_out; float* vz_out;
    const float* vp; const float* den;  // model in the field layout (one shot); den NULL = constant
    float den_c, dt;
    float rdx, rdy, rdz;                // 1/dx, 1/dy, 1/dz
    float dtdx, dtdy, dtdz;             // dt/dx, dt/dy, dt/dz
    float coef[kMaxRadius];
    int pml;
    float sponge[256];                  // taper value at distance index q into the sponge
    const int* slot_to_shot;
    int slab_by_slot;                   // 0: shot s lives in field slab s; 1: in the slab of its launch
                                        // slot (the gradient's shot groups)
    float* div_out;                     // optional: D = sum_a rd_a S-a V_a' of this step (own points)
    // Adjoint mode (acoustic3d_launch_step with adj = true): the P, Vx, Vy, Vz slots hold the
    // adjoint state nu = M K a Q, X, Y, Z (the 2-D recurrence of adjoint2d.cu with a y axis)
    const ShotDev* shots;
    const float* adj_div;               // D_k of the forward step being transposed
    float* adj_g;                       // imaging sum: g += nu_old D_k
    float* adj_lam;                     // [shot][nt_max]: adjoint of P at the source cell
    int nt_max, step;
    int adj_radius;                     // R: the update mask of the receiver injection
    float adj_c[3];                     // dt / (d_a den_c) (constant density), 1 with variable density
};
// one time step of all active shots: velocities, then pressure, sponge (one launch); adj: the
// adjoint of step a.step instead
cudaError_t acoustic3d_launch_step(int radius, const Acou3DArgs& a, int active, bool varden, cudaStream_t st,
                                   bool adj = false);
// P_in[source] -= inj_scale * w[step] for the active shots (before the step)
cudaError_t acoustic3d_launch_inject(float* p, const Layout3D& L, const ShotDev* shots, const int* slot_to_shot,
                                     int active, const float* wavelets, int step, cudaStream_t st,
                                     int slab_by_slot = 0);
// records[rec_base + step * nrec + r] = P_out at receiver r (after the step)
cudaError_t acoustic3d_launch_gather(const float* p, const Layout3D& L, const ShotDev* shots,
                                     const int* slot_to_shot, int active, const int* rec_x, const int* rec_y,
                                     const int* rec_z, float* records, int nrec_max, int step, cudaStream_t st,
                                     int slab_by_slot = 0);
// adjoint: nu[receiver] += M a K res[step] (res [nt][nrec] per shot) before adjoint step `step`
cudaError_t acoustic3d_launch_adj_inject(float* nu, const Acou3DArgs& a, const int* rec_x, const int* rec_y,
                                         const int* rec_z, const float* res, int active, int nrec_max,
                                         cudaStream_t st);
// grad[x][y][z] += -(2 / vp) sum over the slabs [0, nslab) of acc (double, field layout)
cudaError_t acoustic3d_launch_gradient_reduce(const double* acc, int nslab, const Layout3D& L, const float* vp,
                                              double* grad, cudaStream_t st);
// TMA box extents (z, y) of the P, Vy and Vz boxes at this radius; false if unsupported
bool acoustic3d_boxes(int radius, int box_p[2], int box_vy[2], int box_vz[2]);

}  // namespace sfd
