/*
 * seisfd.h -- C ABI of the B200 finite-difference wave-propagation engine.
 *
 * The reference (stone0312/Seismic_code_github) has no in-process API: its hot path is two
 * standalone programs that talk through files.  Each entry point below replaces one step of
 * those programs; the reference location it replaces is cited beside it.
 *
 *   forward/Acoustic_FD_by_ss/src/Acoustic_1order_FD.cpp                    (AFD)
 *   forward/Q_forward/Q_multishot_fd_main_fsbc_zy_rotated.f90               (QM)
 *   forward/Q_forward/Q_multishot_fd_subroutine_fsbc_zy_rotated.f90         (QS)
 *   tools/ricker.cpp                                                        (RIC)
 *   forward/yang_version_2016_2_2/Iso_multishot_fd_subroutine_fsbc_zy_m2_{pub,pri}.f90 (YPUB, YPRI)
 *   forward/yang_version_2016_2_2/Iso_multishot_fd_main_fsbc_zy_m2.f90                 (YM)
 *   forward/yang_version_2016_2_2/Iso_multishot_fd_module_zy_m2.f90                    (YMOD)
 *
 * Conventions (the reference's in-memory and file layouts):
 *   - grids are x-major with z fastest: a[x * nz + z] (AFD:51-100 `P[i][j]`, i = x, j = z;
 *     QS:257 `vp(nz,nx)` column-major).  3-D grids are a[(x * ny + y) * nz + z].
 *   - all sizes are cells of the PADDED grid (interior + sponge), as AFD's Nx = NX + 2*PML.
 *   - records are trace-major, time fastest: rec[(shot_offset + r) * nt_shot + t]
 *     (AFD:385-393 `record.dat`; QM:456 `record1(nt, nxe)`).
 *   - float32 everywhere on the interface.
 * Errors: every call returns an int status (SFD_OK = 0).  Nothing calls exit/abort/trap; a
 * bounded device wait that runs out returns SFD_ERR_TIMEOUT; the last message is available
 * from sfd_last_error.  Threading: one context per host thread, one CUDA stream per context.
 */
#ifndef SEISFD_H
#define SEISFD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SFD_ABI_VERSION 1

/* ---- status codes (the reference stops the process instead: QS:463, QS:897, QS:960) ---- */
#define SFD_OK 0
#define SFD_ERR_ARG 1          /* invalid argument or configuration                        */
#define SFD_ERR_IO 2           /* file open/read/write failure                             */
#define SFD_ERR_CUDA 3         /* CUDA runtime error (message in sfd_last_error)           */
#define SFD_ERR_TIMEOUT 4      /* a bounded device-side wait gave up                       */
#define SFD_ERR_NAN 5          /* non-finite value detected in the receiver traces         */
#define SFD_ERR_NOMEM 6        /* device or host allocation failed                         */
#define SFD_ERR_UNSUPPORTED 7  /* valid request this build does not implement              */
#define SFD_ERR_STATE 8        /* call order (e.g. forward before set_model)               */

/* ---- schemes ---- */
#define SFD_ACOUSTIC_2D 0  /* velocity-pressure staggered grid, sponge: AFD:237-380          */
#define SFD_VISCOAC_2D 1   /* rotated staggered grid, 1 SLS memory variable, vs = 0:
                              QS:695-839 in its acoustic reduction                          */
#define SFD_ACOUSTIC_3D 2  /* 3-D velocity-pressure staggered grid (no reference counterpart) */
#define SFD_VISCOEL_2D 3   /* rotated staggered grid, P-SV visco-elastic with 1 SLS per stress
                              (vs > 0): QS:695-1337, the full Q_forward scheme              */
#define SFD_ELASTIC_2D 4   /* standard staggered grid, isotropic elastic P-SV, 10th order,
                              cosine sponge on four sides with the top sponge's moduli
                              Gaussian-smoothed: the 'abc' mode of forward/yang_version_2016_2_2
                              (YPRI:234-386), flat surface                                  */

/* ---- flags (sfd_grid.flags) ---- */
#define SFD_EXACT 0x1      /* reference operation order: every multiply and add rounded
                              separately, double-precision scale factors (AFD:259,276,293) */
#define SFD_NAN_CHECK 0x2  /* scan receiver traces for NaN/Inf after each forward           */

/* ---- wavelet conventions (sfd_wavelet) ---- */
#define SFD_WAVELET_AFD 0  /* AFD:199-209: 50(1-2pi^2f^2(t-1/f)^2)exp(-pi^2f^2(t-1/f)^2)    */
#define SFD_WAVELET_RIC 1  /* RIC:44: (1-2a^2)exp(-a^2), a = pi f0 (j-delay) dt, f0 integer  */
#define SFD_WAVELET_Q 2    /* QS:1376 (single precision): exp(-b^2)(1-2b^2),
                              b = pi f0 (it dt - 1.2/f0), it = j+1                           */
#define SFD_WAVELET_ISO 3  /* YPUB:1447-1448 (single precision): exp(-b^2)(1-2b^2),
                              b = pi f0 (it dt - delay dt), it = j+1, delay = nint(decay/dt) */

/* ---- wavefield selectors (sfd_get_wavefield) ---- */
#define SFD_FIELD_P 0      /* pressure (AFD P1) / stress sigma (QS strxx)                   */
#define SFD_FIELD_VX 1
#define SFD_FIELD_VZ 2
#define SFD_FIELD_VY 3
#define SFD_FIELD_R 4      /* memory variable r (QS rxx)                                     */
#define SFD_FIELD_SZZ 5    /* QS / YPUB strzz (elastic schemes; equals strxx when vs = 0)   */
#define SFD_FIELD_SXZ 6    /* QS / YPUB strxz (elastic schemes)                              */

typedef struct sfd_ctx sfd_ctx;

/* Grid and scheme.  Replaces the hard-coded block AFD:28-45 and the .par cards QS:162-231. */
typedef struct {
    int scheme;            /* SFD_ACOUSTIC_2D, SFD_VISCOAC_2D or SFD_ACOUSTIC_3D          */
    int nx, ny, nz;        /* padded grid; ny = 1 for 2-D                                   */
    int pml;               /* sponge width in cells (AFD:30 PML; QS: npxn = npxp = npzn = npzp) */
    float dx, dy, dz, dt;  /* metres, seconds                                              */
    int order;             /* spatial order 2R: 16 (AFD), 10 (QS), 8, 4 or 2               */
    int flags;             /* SFD_EXACT | SFD_NAN_CHECK                                     */
    float f0;              /* SLS reference frequency (QS:509 fup = 2.5 f0 2 pi); 0 = unused */
} sfd_grid;

/* One shot.  Replaces AFD:199-216 and AFD:376-377 (one source, one receiver line) and
 * QM:124-129 (per-shot source position, aperture window and record length). */
typedef struct {
    int sx, sy, sz;        /* source cell (shot-local padded coordinates)                  */
    int nt;                /* time steps of this shot (record length), >= 1               */
    int nrec;              /* receivers                                                     */
    const int* rec_x;      /* nrec cells, shot-local padded coordinates                     */
    const int* rec_y;      /* NULL for 2-D                                                   */
    const int* rec_z;
    const float* wavelet;  /* nt samples (host); injected as AFD:247-251 / QS:1376-1387       */
    int ap_x0;             /* aperture window: shot column i reads model column ap_x0 + i   */
    int ap_nx;             /* window width in cells; 0 = the whole model width              */
} sfd_shot;

/* Device timing of the last sfd_forward / sfd_gradient call (CUDA events on the context's
 * stream around the time loop) and the number of kernel launches it issued. */
typedef struct {
    double loop_ms;        /* device time of the time loop (all shots)                      */
    double device_ms;      /* device time of the whole call: state reset, loop, record transpose */
    double total_ms;       /* host wall time of the whole call incl. copies                  */
    double point_updates;  /* grid-point updates performed (padded points x steps x shots)   */
    long long launches;    /* kernels launched by the call                                   */
    long long h2d_bytes;
    long long d2h_bytes;
    int graph;             /* 1 if the time loop ran as a CUDA graph                          */
    int kernel_variant;    /* implementation detail: which step kernel ran                    */
} sfd_timing;

int sfd_abi_version(void);
const char* sfd_status_string(int status);

/* Context lifetime.  Replaces the allocation blocks AFD:51-132 and QM:283-409. */
int sfd_create(const sfd_grid* grid, int device, sfd_ctx** out);
int sfd_destroy(sfd_ctx* ctx);
int sfd_last_error(const sfd_ctx* ctx, char* buf, size_t len);

/* Model, padded grid (x-major, z fastest), host pointers, copied to the device.
 * Replaces AFD:137-142 (Vp, DEN) and QS:238-284 + QS:434-551 (read_data, substagger, pcalpas).
 * den may be NULL (constant 2400 kg/m^3, AFD:141); q (SFD_VISCOAC_2D only) may be NULL (no
 * attenuation: Q = 1e5, the QM:418-419 override). */
int sfd_set_model(sfd_ctx* ctx, const float* vp, const float* den, const float* q);

/* Visco-elastic model (SFD_VISCOEL_2D): P and S velocities, density and the P and S quality
 * factors on the padded grid.  Replaces QS:238-284 (read_data of vp, vs, rho, qfp, qfs) and
 * QS:434-551 (substagger, pcalpas).  den NULL = 2400 kg/m^3; qp / qs NULL = 1e5 (QM:418-419).
 * Elastic model (SFD_ELASTIC_2D): vp, vs, den; qp and qs must be NULL.  Replaces YPUB:148-184
 * (read_data) and YPUB:323-634 (substagger, then modipapml: the moduli and buoyancies of the top
 * sponge rows z < pml smoothed in place with the Gaussian of sfd_set_gauss_radius). */
int sfd_set_model_elastic(sfd_ctx* ctx, const float* vp, const float* vs, const float* den, const float* qp,
                          const float* qs);

/* Half-width rgau of the Gaussian (sigma 2 cells, window 2 rgau - 1 cells) that spreads the
 * source and smooths the top sponge of SFD_ELASTIC_2D (YPUB:1470-1501, the .par's "rad of gauss
 * smooth"; default 50).  Re-prepares the model and the source stamps if they are set. */
int sfd_set_gauss_radius(sfd_ctx* ctx, int rgau);

/* Boundary mode of SFD_ELASTIC_2D (YM:190-219 `molmod`).  top = 0: 'abc', the cosine sponge on
 * all four sides with the top sponge's moduli smoothed (YPRI:234-386; the default).  top >= 1:
 * 'fsbc', a flat free surface at padded row top - 1 (the reference's itopo = npzn = top,
 * YPRI:57-230): no top sponge, lower-order z derivatives on the five rows below the surface,
 * tau_zz = 0 on and above it, the tau_xz image and the extrapolated vz one row above it; the
 * rows above the surface are air.  Re-prepares the model if it is set. */
int sfd_set_free_surface(sfd_ctx* ctx, int top);

/* Topography of SFD_ELASTIC_2D: itopo[x] for every padded model column x, the reference's 1-based
 * surface row itopoe = nint(topo/dz) + npzn (YPUB:270-272); NULL restores the flat surface (pml in
 * abc mode, the sfd_set_free_surface row in fsbc mode).  In abc mode column x is updated from
 * padded row itopo[x] - pml - 1 down, with the top sponge on the pml + 1 rows from there
 * (YPUB:1095-1407, 851-897), and itopo[x] >= pml; in fsbc mode the free surface lies at row
 * itopo[x] - 1 of column x.  The smoothed rows (abc), the rows refilled by substagger and the
 * source condition (YPRI:163-168) follow it; receivers are placed by the caller.  Re-prepares
 * the model if it is set. */
int sfd_set_topography(sfd_ctx* ctx, const int* itopo);

/* Shots.  Replaces the shot loop QM:124-141 (one launch for all shots instead of one process
 * per shot).  Wavelets and receiver lists are copied; the caller keeps ownership. */
int sfd_set_shots(sfd_ctx* ctx, int nshot, const sfd_shot* shots);

/* Forward modelling of all shots in one batched time loop.  Replaces the time loop AFD:237-380
 * and QM:439-484.  records: host buffer of sum_s nrec_s * nt_s floats (trace-major per shot,
 * shots concatenated in order) or NULL. */
int sfd_forward(sfd_ctx* ctx, float* records);

/* Same, with the records left in device memory (caller-owned, same layout) and no host copy. */
int sfd_forward_device(sfd_ctx* ctx, float* records_dev);

/* Records of one component from the last forward, in the sfd_forward layout.  The
 * Q_forward programs record two (QM:452-459): record1 = strzz (SFD_FIELD_SZZ, what sfd_forward
 * returns for the viscoacoustic and visco-elastic schemes) and record2 = strxx (SFD_FIELD_P).
 * For SFD_VISCOAC_2D both are the same sigma.  SFD_ELASTIC_2D records vx (record1,
 * SFD_FIELD_VX, what sfd_forward returns) and vz (record2, SFD_FIELD_VZ), YPRI:361-367. */
int sfd_get_records(sfd_ctx* ctx, int field, float* records);

/* Plain per-shot path: shots one after another, one kernel launch per time step each, no
 * graph -- the unbatched baseline the batched loop is measured against. */
int sfd_forward_per_shot(sfd_ctx* ctx, float* records);

/* Final wavefield of one shot after the last forward step (after the sponge, as AFD stores
 * it at AFD:329-340), padded grid.  Replaces the snapshot writes AFD:343-355, QM:462-481. */
int sfd_get_wavefield(sfd_ctx* ctx, int shot, int field, float* out);

/* Full-waveform gradient: forward with checkpoints, adjoint of the discrete time loop,
 * zero-lag cross-correlation imaging (2-D acoustic, viscoacoustic and 3-D acoustic schemes).
 * obs: observed records in the sfd_forward layout.  misfit = 0.5 * sum (pred - obs)^2.  grad_vp: d misfit / d vp on the padded grid.
 * grad_invq: d misfit / d (1/Q) (SFD_VISCOAC_2D only; may be NULL).  No reference
 * counterpart (the reference has no adjoint). */
int sfd_gradient(sfd_ctx* ctx, const float* obs, float* misfit, float* grad_vp, float* grad_invq);

/* sfd_gradient with every buffer in the caller's device memory (zero-copy for torch and for a
 * device-side all-reduce of per-rank gradients): obs_dev (sfd_forward layout), misfit_dev (one
 * float), grad_vp_dev and grad_invq_dev (padded model grid; either may be NULL).  The results
 * equal sfd_gradient's bit for bit.  Pointers must be on the context's device. */
int sfd_gradient_device(sfd_ctx* ctx, const float* obs_dev, float* misfit_dev, float* grad_vp_dev,
                        float* grad_invq_dev);

/* Same gradient with the plain per-shot schedule: shots one after another, one kernel launch
 * per time step, no graph -- the baseline the batched gradient is measured against. */
int sfd_gradient_per_shot(sfd_ctx* ctx, const float* obs, float* misfit, float* grad_vp, float* grad_invq);

/* Gradient of the misfit of the last sfd_gradient call with respect to the wavelet samples of
 * one shot (nt_shot values).  With obs = F(w) - r this is F^T r, the adjoint of the
 * wavelet-to-records map, used by the dot-product test. */
int sfd_get_wavelet_gradient(sfd_ctx* ctx, int shot, float* out);

/* Test hook of the step kernels' bounded waits (no counterpart in the reference, which has no
 * device waits): in the forwards and gradients that follow, CTA `cta` of the 2-D acoustic FMA
 * step `step` issues none of its TMA box loads and gives up waiting for them after limit_s
 * seconds (0 < limit_s <= 10; every other wait keeps its limit of about one second).  That call
 * returns SFD_ERR_TIMEOUT and leaves the context usable.  cta < 0 removes the hook. */
int sfd_test_wait_timeout(sfd_ctx* ctx, int cta, int step, double limit_s);

/* Checkpoint interval of sfd_gradient in steps (0 = ceil(sqrt(nt))).  The forward state of
 * every shot is kept every `steps` steps; each segment is recomputed once during the
 * backward pass, so memory is O(nt/steps + steps) wavefields per shot. */
int sfd_set_checkpoint_interval(sfd_ctx* ctx, int steps);

/* Device-memory budget of sfd_gradient in bytes (0 = the free device memory).  The 3-D gradient
 * sizes its shot groups and checkpoint levels to the budget: every shot group keeps its
 * wavefields, adjoint fields and outer checkpoints; when one level of checkpoints does not fit,
 * segments are recomputed from inner checkpoints (two levels, four passes instead of three).
 * No reference counterpart (the reference has no adjoint). */
int sfd_set_memory_limit(sfd_ctx* ctx, long long bytes);

int sfd_get_timing(const sfd_ctx* ctx, sfd_timing* out);

/* Wavefield snapshots taken inside the forward time loop.  Replaces the Snap.dat / Pall.dat
 * writes of AFD:343-373 and the snapshot files of QM:462-481.  Stream id (0..3) records, after
 * every step k (0-based) with k >= first and (k - first) % every == 0, at most `count` times per
 * shot, the interior (pml <= x < nx_shot - pml, top <= z < nz - pml; top = pml, or the row
 * given to sfd_set_free_surface) of `field` as the reference
 * holds it after the step: SFD_FIELD_P (AFD P1 / QS strxx), SFD_FIELD_VX, SFD_FIELD_VZ, and
 * SFD_FIELD_R for the viscoacoustic scheme.  count = 0 removes the stream.  2-D schemes only. */
int sfd_set_snapshots(sfd_ctx* ctx, int id, int field, int first, int every, int count);
/* The snapshots of stream id for one shot from the last forward: n x (nx_shot - 2 pml) x
 * (nz - top - pml) floats, x-major, z fastest; *n_out receives n.  out may be NULL to query n. */
int sfd_get_snapshots(sfd_ctx* ctx, int id, int shot, float* out, int* n_out);

/* Single-shot 2-D acoustic forward that allocates no device memory.  No counterpart in the
 * reference: it is for callers that cannot allocate device memory when they model a shot (a
 * framework that has reserved the device memory for its own allocator, a process at its
 * device-memory quota, a real-time loop that forbids allocation after start-up).  Every working
 * buffer lives in a fixed 32 MiB device array inside the library; sizes that do not fit return
 * SFD_ERR_NOMEM.  vp_dev, den_dev (NULL = constant 2400), wavelet_dev (nt samples) and
 * records_dev (nrec x nt, trace-major) are device pointers owned by the caller; rec_x / rec_z
 * are host arrays.  Arithmetic is the reference order of SFD_EXACT.  The first call on a device
 * looks up the array's address (make it before any stream capture); calls that overlap on the
 * GPU race on the shared array.  stream may be NULL (the default stream); the call returns
 * after the stream has finished its work. */
int sfd_forward_noalloc(const sfd_grid* grid, const float* vp_dev, const float* den_dev, const float* wavelet_dev,
                        int nt, int sx, int sz, int nrec, const int* rec_x, const int* rec_z, float* records_dev,
                        void* stream);

/* Host helpers (no context). */
/* Source wavelet in one of the reference's conventions (AFD:199-209, RIC:44, QS:1376,
 * YPUB:1447-1448).  delay: in samples, RIC (RIC uses 150) and ISO (idecay) only. */
int sfd_wavelet(int convention, int nt, float dt, float f0, int delay, float* out);
/* AFD sponge factors absorb[x][z] (AFD:164-194; bottom loop bound j < Nz, see AFD:190). */
int sfd_afd_sponge(int nx, int nz, int pml, float* absorb);
/* Staggered first-derivative coefficients for order 2R (AFD:38-45 for 16, QS:9-28 otherwise). */
int sfd_fd_coeffs(int order, float* coeffs);
/* Edge-replicated padding of an interior model (QS:340-372): in (nx_in, nz_in) ->
 * out (nx_in + pxn + pxp, nz_in + pzn + pzp). */
int sfd_pad_model(const float* in, int nx_in, int nz_in, int pxn, int pxp, int pzn, int pzp, float* out);

/* ---- the reference programs' file contract (host only) ---- */
/* Q_forward parameter card (QS:121-234): pairs of a label line and a value line, in this order.
 * fdo2 / fdo1 are read and unused, as in the reference (the scheme is 10th order). */
typedef struct {
    char vp[256], vs[256], rho[256], qp[256], qs[256];     /* model files (nz x nx Fortran arrays) */
    char shot1[256], shot2[256], shot3[256], shot4[256];   /* per-shot / merged record prefixes  */
    int nshot;
    float offset_min, offset_max;                          /* metres, relative to the source     */
    float sx0, sz0, rz0;                                   /* first source x, source and receiver depth (m) */
    float dsx;                                             /* shot spacing (m)                   */
    int nx, nz;                                            /* model size (cells)                 */
    float dx, dz;
    int nt;                                                /* record length (samples)            */
    float dt, f0;
    float pml_xn, pml_xp, pml_zn, pml_zp;                  /* sponge thickness (m)               */
    int fdo2, fdo1;
} sfd_qpar;
int sfd_qpar_read(const char* path, sfd_qpar* out);
/* yang_version parameter card (YPUB:48-145): pairs of a label line and a value line, in this
 * order.  dtsnap: snapshot interval (s); decay: source delay (s), nint(decay/dt) steps before the
 * first recorded sample; rgau: Gaussian half-width (cells). */
typedef struct {
    char molmod[16];                                       /* "abc" or "fsbc" (YM:190-219)     */
    char vp[256], vs[256], rho[256], topo[256];            /* model files; topo: nx surface depths (m) */
    char snapx[256], snapz[256];                           /* vx / vz snapshot file prefixes     */
    char shot1[256], shot2[256], shot3[256], shot4[256];   /* vx parts / vx merged / vz parts / vz merged */
    int nshot;
    float offset_min, offset_max;
    float sx0, sz0, rz0;
    float dsx;
    int nx, nz;
    float dx, dz;
    int nt;
    float dt, dtsnap, f0, decay;
    float pml_xn, pml_xp, pml_zn, pml_zp;                  /* sponge thickness (m)               */
    int rgau;
} sfd_isopar;
int sfd_isopar_read(const char* path, sfd_isopar* out);
/* VTI modeller parameter card (VS:342-425, de-multiple/convolution_srm/vti_qa_2d_c3_demo1):
 * pairs of a label line and a value line, in this order. */
typedef struct {
    char vz[256], epsilon[256], delta[256];                /* model files (nz_v x nx_v Fortran arrays) */
    char shot1[256], shot2[256];                           /* per-shot SU prefix / merged SU prefix */
    int nshot;
    float offset_min, offset_max;                          /* m                                   */
    float sx0, sz0, rz0;                                   /* m                                   */
    float dsx;                                             /* m                                   */
    int nx_v, nz_v;
    float dx_v, dz_v;
    int nt;
    float dt, f0;
    float bound_x_l, bound_x_r, bound_z_u, bound_z_d;      /* PML thickness (m)                  */
    int order_explicit, order_pml_1st, order_pml_2nd;
} sfd_vtipar;
int sfd_vtipar_read(const char* path, sfd_vtipar* out);
/* Raw little-endian float32 files: models (x-major, z fastest: QS:238-284, tools/get_vel_model.cpp:
 * 50-58), AFD's record / snapshot outputs (AFD:343-393).  append = 1 opens for appending. */
int sfd_read_floats(const char* path, long long n, float* out);
int sfd_write_floats(const char* path, const float* data, long long n, int append);
/* One shot's SU file (QS:1476-1546): per trace a 240-byte SEG-Y header with fldr = shot_no,
 * trid = 1, sx = (isx - 1) dx, gx = (ixmin - 2 + i) dx for trace i = 1..ntr, offset = gx - sx,
 * cdp = nint((gx + sx) / dx) + 1, ns = nt, dt in microseconds (integer conversions as in the
 * Fortran), followed by the trace's nt float32 samples.  traces: [ntr][nt]. */
int sfd_su_write(const char* path, const float* traces, int ntr, int nt, int shot_no, int isx, int ixmin, float dx,
                 float dt);
/* The same with header options: SFD_SU_CDP sets cdp as QS:1535 does; yang_version's writer
 * (YPUB:1533-1604) leaves it 0. */
#define SFD_SU_CDP 0x1
/* SFD_SU_NO_OFFSET leaves offset 0, as the VTI modeller's writer does (VS:163-217) */
#define SFD_SU_NO_OFFSET 0x2
int sfd_su_write_ex(const char* path, const float* traces, int ntr, int nt, int shot_no, int isx, int ixmin, float dx,
                    float dt, int flags);
/* Concatenate per-shot SU files in order (QS:1550-1624); delete_inputs = 1 removes them as the
 * reference does. */
int sfd_su_merge(const char* out_path, const char* const* in_paths, int n, int delete_inputs);

/* ---- VTI pseudo-acoustic modeller (de-multiple/convolution_srm/vti_qa_2d_c3_demo1) ----
 * The coupled u / q second-order system with 10th-order second derivatives inside and split PML
 * fields on the four sides (VTI_multishot_qacoustic_fd_subroutine_c3.f90 = VS, main program VM).
 * One call runs every shot of a survey, batched in one launch per time step; it replaces the shot
 * loop of multi_shot_modelling (VM:12-180) and single_shot_modelling (VM:190-560), whose .par
 * card gives these fields (VS:342-425).  Grid numbers are the reference's, 1-based: nsx, nsz0 and
 * nrz0 as VM:145-147 and 158 compute them, xmin / xmax the shot's aperture columns (VM:162-163).
 * Model arrays are [nx_v][nz_v], x-major (z fastest), host pointers.  records (host) receives
 * [shot][xmax - xmin + 1][nt]: u on the receiver row (VM:446-453).  Every shot must have the same
 * xmax - xmin.  Orders: explicit 10, pml_1st 9 or 10, pml_2nd 10 (the stencils are written out
 * with five coefficients, VS:511-551); nx_bound_r and nz_bound_d >= 2 (VM:248-249). */
typedef struct {
    int nx_v, nz_v;        /* model grid                                                      */
    float dx, dz, dt, f0;  /* metres, seconds, Hz                                             */
    int nt;                /* record length                                                   */
    int nx_bound_l, nx_bound_r, nz_bound_u, nz_bound_d;  /* PML cells, nint(thickness / dx) (VM:136-141) */
    int order_explicit, order_pml_1st, order_pml_2nd;
    int flags;             /* SFD_EXACT: every operation rounded separately in the reference's order
                              (bit-exact with the restatement); 0: FMA contraction and approximate
                              divisions (relative L2 <= 1e-5 of it)                            */
} sfd_vti_par;

typedef struct {
    int nsx, nsz0, nrz0;   /* source column and row, receiver row                             */
    int xmin, xmax;        /* aperture: record columns xmin + 1 .. xmax + 1 of the model (VS:300) */
} sfd_vti_shot;

/* FD coefficients of coefficient_2nd (first = 0, order/2 values) or coefficient_1st (first = 1,
 * (order+1)/2 values), VS:1264-1472, as the modeller computes them in single precision. */
int sfd_vti_coefficients(int order, int first, float* out);
int sfd_vti_forward(const sfd_vti_par* par, const float* vz, const float* epsilon, const float* delta, int nshot,
                    const sfd_vti_shot* shots, int device, float* records, sfd_timing* timing);

#ifdef __cplusplus
}
#endif
#endif /* SEISFD_H */
