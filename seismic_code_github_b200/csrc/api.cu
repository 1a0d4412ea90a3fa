// C ABI implementation: context, model and shot upload, the batched time loop (one CUDA graph
// per shot set), the per-shot baseline path and read-back.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "sfd_internal.h"

using namespace sfd;

namespace sfd {
struct Engine2DState;  // scheme-specific device state (defined below)
}

struct sfd_ctx {
    sfd_grid g{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evs = nullptr, eve = nullptr;  // loop / whole call
    std::string err;
    int radius = 0;
    float coef[kMaxRadius] = {};

    // model (host copies are kept for the source scale factors and the gradient)
    bool have_model = false;
    std::vector<float> h_vp, h_den;
    bool varden = false;
    float den_c = 2400.0f;
    float* d_vp = nullptr;
    float* d_den = nullptr;
    float* d_q = nullptr;
    int mpitch = 0;

    // shots
    bool have_shots = false;
    int nshot = 0;
    int nt_max = 0;
    std::vector<ShotDev> h_shots;
    std::vector<int> h_rec_x, h_rec_z;
    std::vector<float> h_wav;
    std::vector<long long> rec_out_off;  // trace-major output offset per shot
    long long rec_total = 0;
    std::vector<int> order;              // shots sorted by nt, longest first
    std::vector<int> h_ident_order;      // 0, 1, ..., nshot - 1
    std::vector<int> active_at;          // not stored per step; computed on the fly

    // device buffers for the acoustic 2-D scheme
    Acou2DPlan plan{};
    Layout2D L{};
    ShotDev* d_shots = nullptr;
    int* d_slot = nullptr;     // sorted order
    int* d_ident = nullptr;    // identity (per-shot path)
    float* d_wav = nullptr;
    int* d_rec_x = nullptr;
    int* d_rec_z = nullptr;
    int* d_trp = nullptr;      // per-tile receiver CSR pointers
    int* d_tri = nullptr;      // per-tile receiver indices
    int* d_torder = nullptr;   // FMA kernel's forward tile order: interior tiles, then edge tiles
    int tile_major = 1;        // forward steps of the FMA kernel: tile-major over d_torder
    int test_cta = -1, test_step = 0;      // sfd_test_wait_timeout
    unsigned long long test_wait_ns = 0;
    int l2_ahead = 0;          // FMA kernel, one tile per CTA: L2 prefetch distance in CTAs
    float* d_rec_tn = nullptr; // [nt][nrec] per shot
    float* d_rec_nt = nullptr; // [nrec][nt] per shot (output layout)
    float* d_state = nullptr;  // 6 fields: p0 p1 vx0 vx1 vz0 vz1, each nshot * shot_stride
    size_t state_floats = 0;
    int* d_flag = nullptr;     // NaN watchdog
    int* d_err = nullptr;      // bounded-wait timeout flag written by the step kernels
    CUtensorMap tmaps[6];      // TMA descriptors: P0 P1 VX0 VX1 VZ0 VZ1
    CUtensorMap mtmaps[6];     // the same buffers with the x-marching kernel's boxes
    CUtensorMap qtmaps[2];     // default viscoacoustic step: sigma S0 S1 (viscoac2d_fast.cu box)

    // 3-D scheme: dense [x][y][pitch] slabs, 8 fields (P, Vx, Vy, Vz, two buffers each)
    Layout3D L3{};
    CUtensorMap tmaps3[6];     // TMA descriptors: P0 P1 VY0 VY1 VZ0 VZ1
    std::vector<int> h_rec_y;
    int* d_rec_y = nullptr;
    int nrec_max = 0;

    cudaGraphExec_t graph = nullptr;
    bool graph_valid = false;

    // wavefield snapshot streams (sfd_set_snapshots)
    struct Snap {
        int field = 0, first = 0, every = 1, count = 0;
        float* d_buf = nullptr;
        long long* d_off = nullptr;       // per shot offset (floats) into d_buf
        std::vector<long long> off;
        std::vector<int> taken;           // snapshots per shot
        long long total = 0;
        bool ready = false;               // filled by the last forward
    };
    Snap snaps[4];
    float* d_src_pre = nullptr;           // per shot: P at the source before the next injection

    // viscoacoustic scheme: prepared model (QS:434-551), sponge tables, source stamps
    float* q_busg = nullptr;
    float* q_p1 = nullptr;
    float* q_p2 = nullptr;
    float q_rtau = 0.0f;
    std::vector<float> h_q;        // quality factors as given (empty: Q = 1e5)
    std::vector<int> h_ap_x0;      // each shot's aperture start in the model as given
    int q_width = 0;               // columns of the prepared model (one block per shot window)
    float* d_spg = nullptr;
    int spg_stride = 0;
    float* d_stamps = nullptr;
    // visco-elastic scheme: the six stress coefficients (QS:473-551) and the strxx records
    float* e_q[6] = {};             // q1 q2 q3 m1 m2 m3 in the prepared-model layout
    std::vector<float> h_vs, h_qs;  // S velocity and S quality factor as given (empty: 0 / 1e5)
    float* d_rec2_tn = nullptr;     // strxx records [nt][nrec] per shot
    float* d_rec2_nt = nullptr;     // ... trace-major
    bool rec2_ready = false;
    bool elastic_call = false;      // sfd_set_model is running on behalf of sfd_set_model_elastic
    // isotropic elastic scheme (yang_version): Gaussian half-width, its table and non-zero range;
    // the prepared model lives in e_q[0..4] (busg2e, busg1e, lambmusg, lambsg, musge)
    int iso_rgau = 50;
    int iso_top = 0;                // 0: abc mode; >= 1: fsbc mode, top pad of iso_top rows (flat: itopo)
    std::vector<int> h_itopo;       // itopo per padded model column (sfd_set_topography); empty: flat
    int* d_itopo = nullptr;         // ... per prepared-model column
    long long topo_gen = 0;         // bumped by every sfd_set_topography
    std::vector<float> iso_gc;
    int iso_lo = 0, iso_hi = -1;
    long long model_gen = 0;        // bumped by every sfd_set_model
    // what the prepared model was built from (windows, model generation, rgau): a call with the
    // same inputs only re-targets the shots at the existing blocks
    std::vector<std::pair<int, int>> prep_wins;
    long long prep_gen = -1;
    int prep_rgau = -1;
    int prep_top = -1;
    long long prep_topo_gen = -1;

    // gradient (sized on first use for the current shot set)
    int ckpt_interval = 0;
    int grad_C = 0, grad_ncp = 0;
    int grad_keep = 0;          // first segment whose D_k the first forward keeps (no recomputation)
    float* d_ckpt = nullptr;    // [ncp][3 fields][nshot * shot_stride]
    float* d_div = nullptr;     // D_k slots: [C] of the segment being recomputed, then the kept tail
    float* d_adj = nullptr;     // adjoint state: nu0 nu1 x0 x1 z0 z1 (viscoacoustic: 8 adjoints + Qx Qz)
    CUtensorMap adj_tmaps[6];   // TMA descriptors of the acoustic adjoint buffers
    CUtensorMap adj_mtmaps[6];  // the same buffers with the x-marching kernel's boxes
    float* d_gseg = nullptr;    // per-segment imaging sum (float)
    double* d_gacc = nullptr;   // imaging sum over all segments (double)
    float* d_obs_nt = nullptr;  // observed records as given ([nrec][nt] per shot)
    float* d_obs_tn = nullptr;  // ... transposed to [nt][nrec]
    float* d_res = nullptr;     // residuals [nt][nrec]
    float* d_lam = nullptr;     // [nshot][nt_max] adjoint of P at the source cell
    double* d_misfit = nullptr;
    double* d_grad = nullptr;   // gradient on the model grid (double)
    double* d_grad2 = nullptr;  // viscoacoustic: d misfit / d (1/Q) on the model grid
    GradSrc* d_gsrc = nullptr;  // per shot: source cell and -dt DEN there (device-output gradient)
    int* d_apx0 = nullptr;      // viscoacoustic: each shot's aperture start in the model
    // 3-D gradient (shot groups of g3_G slabs, checkpoint levels g3_C1 / g3_C2)
    int state_slabs = 0;        // shot slabs per field held by d_state (3-D)
    float* g3_adj = nullptr;    // adjoint state nu0 nu1 X0 X1 Y0 Y1 Z0 Z1, g3_G slabs each
    CUtensorMap g3_tmaps[6];    // nu0 nu1 Y0 Y1 Z0 Z1
    float* g3_div = nullptr;    // D_k of the innermost segment [C][g3_G slabs]
    float* g3_ck1 = nullptr;    // outer checkpoints [n1][4 fields][g3_G slabs]
    float* g3_ck2 = nullptr;    // inner checkpoints [n2][4 fields][g3_G slabs] (two levels only)
    float* g3_gseg = nullptr;   // imaging sum of the segment (float)
    double* g3_gacc = nullptr;  // imaging sum of the group (double)
    int g3_G = 0, g3_C1 = 0, g3_C2 = 0, g3_n1 = 0, g3_n2 = 0;
    size_t mem_limit = 0;       // device-memory budget of the gradient (0: what is free)
    cudaGraphExec_t grad_graph = nullptr;
    bool grad_valid = false;
    bool have_grad = false;
    sfd_timing timing{};

    ~sfd_ctx();
};

namespace {

int set_err(sfd_ctx* c, int code, const char* fmt, ...) {
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        c->err = buf;
    }
    return code;
}

#define CK(call)                                                                               \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return set_err(ctx, e_ == cudaErrorMemoryAllocation ? SFD_ERR_NOMEM : SFD_ERR_CUDA, \
                           "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

template <typename T>
void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

int round_up(int v, int m) { return (v + m - 1) / m * m; }

// The viscoacoustic scheme runs the fused kernel (viscoac2d_fast.cu) unless SFD_EXACT is set.
// Its slabs: vx (2 parities), vz (2), sigma (2), r, and the six split parts of the sponge bands.
constexpr int kQVX = 0, kQVZ = 2, kQS = 4, kQR = 6, kQSplit = 7, kQE = 13, kQFastSlabs = 15;
constexpr int kQFastSeg = 256;  // columns per segment of the one-kernel step (SFD_QFAST_SEG overrides)
// Segment length of a step with `act` active shots: 256 columns, halved (down to 64) while the
// grid would not fill one wave of four CTAs per SM -- the last shots of an uneven batch get more,
// shorter segments (each pays a warm-up chunk; the results do not depend on the length).
int q_fast_seg(const sfd_ctx* c, int act) {
    const char* env = std::getenv("SFD_QFAST_SEG");
    const int v = env ? std::atoi(env) : 0;
    if (v >= 16 && v % 16 == 0) return v;
    static int nsm[kMaxDevices] = {};
    if (c->device >= 0 && c->device < kMaxDevices && nsm[c->device] == 0 &&
        cudaDeviceGetAttribute(&nsm[c->device], cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess)
        nsm[c->device] = 0;
    const int sms = (c->device >= 0 && c->device < kMaxDevices) ? nsm[c->device] : 0;
    const long long width = (long long)c->L.ntx * kTileX;
    int seg = kQFastSeg;
    while (seg > 64 && sms > 0 && (long long)act * c->L.ntz * ((width + seg - 1) / seg) < 4LL * sms) seg /= 2;
    return seg;
}
// The default viscoacoustic mode: the x-marching step kernel and the sponge-band kernel
// (viscoac2d_fast.cu; sigma, vx, vz ping-pong, r and the split parts of the bands in place);
// SFD_EXACT runs the reference-order pair of kernels (viscoac2d.cu, eight split fields in place).
bool q_fast(const sfd_ctx* c) { return c->g.scheme == SFD_VISCOAC_2D && !(c->g.flags & SFD_EXACT); }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// 3-D float32 tensor map over one field buffer: dims (pitch, cols, nshot), box (z, x, 1).
int encode_field_map(sfd_ctx* ctx, CUtensorMap* m, float* base, const Layout2D& L, int nshot, const int box[2]) {
    auto enc = tensor_map_encoder();
    if (!enc) return set_err(ctx, SFD_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const cuuint64_t dims[3] = {(cuuint64_t)L.pitch, (cuuint64_t)L.cols, (cuuint64_t)nshot};
    const cuuint64_t strides[2] = {(cuuint64_t)L.pitch * 4, (cuuint64_t)L.shot_stride * 4};
    const cuuint32_t bdim[3] = {(cuuint32_t)box[0], (cuuint32_t)box[1], 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, bdim, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_err(ctx, SFD_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return SFD_OK;
}

// 4-D float32 tensor map over one 3-D field buffer: dims (nz, ny, nx, nshot) with the exact grid
// extents (boxes read zeros outside the grid), box (z, y, 1, 1).
int encode_field_map3(sfd_ctx* ctx, CUtensorMap* m, float* base, const Layout3D& L, int nshot, const int box[2]) {
    auto enc = tensor_map_encoder();
    if (!enc) return set_err(ctx, SFD_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const cuuint64_t dims[4] = {(cuuint64_t)L.nz, (cuuint64_t)L.ny, (cuuint64_t)L.nx, (cuuint64_t)nshot};
    const cuuint64_t strides[3] = {(cuuint64_t)L.pitch * 4, (cuuint64_t)L.xstride * 4, (cuuint64_t)L.shot_stride * 4};
    const cuuint32_t bdim[4] = {(cuuint32_t)box[0], (cuuint32_t)box[1], 1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, dims, strides, bdim, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_err(ctx, SFD_ERR_CUDA, "cuTensorMapEncodeTiled (4-D) failed (%d)", (int)r);
    return SFD_OK;
}

// Sponge factor of the 3-D scheme at one cell: the AFD taper (AFD:164-194) of the x pad, else of
// the y pad, else of the z pad, else 1.
float sponge3(const sfd_grid& g, int x, int y, int z) {
    auto q = [&](int d, int n) { return d < g.pml ? g.pml - d - 1 : (d >= n - g.pml ? d - n + g.pml : -1); };
    int k = q(x, g.nx);
    if (k < 0) k = q(y, g.ny);
    if (k < 0) k = q(z, g.nz);
    return k < 0 ? 1.0f : (float)(-0.38 * k * k / (1.0 * g.pml * g.pml) + 1);
}

void free_shot_buffers(sfd_ctx* c) {
    dfree(c->d_shots); dfree(c->d_slot); dfree(c->d_ident); dfree(c->d_wav);
    dfree(c->d_rec_x); dfree(c->d_rec_z); dfree(c->d_trp); dfree(c->d_tri); dfree(c->d_torder); dfree(c->d_rec_y);
    dfree(c->d_rec_tn); dfree(c->d_rec_nt); dfree(c->d_state); dfree(c->d_stamps); dfree(c->d_src_pre);
    dfree(c->d_rec2_tn); dfree(c->d_rec2_nt);
    c->rec2_ready = false;
    for (auto& sn : c->snaps) {
        dfree(sn.d_buf);
        dfree(sn.d_off);
        sn.ready = false;
        sn.total = 0;
    }
    if (c->graph) cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
    c->graph_valid = false;
    dfree(c->d_ckpt); dfree(c->d_div); dfree(c->d_adj); dfree(c->d_gseg); dfree(c->d_gacc);
    dfree(c->d_obs_nt); dfree(c->d_obs_tn); dfree(c->d_res); dfree(c->d_lam); dfree(c->d_misfit);
    dfree(c->d_grad); dfree(c->d_grad2); dfree(c->d_apx0); dfree(c->d_gsrc);
    dfree(c->g3_adj); dfree(c->g3_div); dfree(c->g3_ck1); dfree(c->g3_ck2); dfree(c->g3_gseg); dfree(c->g3_gacc);
    c->g3_G = c->g3_C1 = c->g3_C2 = c->g3_n1 = c->g3_n2 = 0;
    c->state_slabs = 0;
    if (c->grad_graph) cudaGraphExecDestroy(c->grad_graph);
    c->grad_graph = nullptr;
    c->grad_valid = false;
    c->have_grad = false;
    c->grad_C = c->grad_ncp = 0;
}

}  // namespace

sfd_ctx::~sfd_ctx() {
    if (device >= 0) cudaSetDevice(device);
    free_shot_buffers(this);
    dfree(d_vp); dfree(d_den); dfree(d_q); dfree(d_flag); dfree(d_err);
    dfree(q_busg); dfree(q_p1); dfree(q_p2); dfree(d_spg); dfree(d_itopo);
    for (auto& p : e_q) dfree(p);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (evs) cudaEventDestroy(evs);
    if (eve) cudaEventDestroy(eve);
    if (stream) cudaStreamDestroy(stream);
}

namespace {
int alloc_state_3d(sfd_ctx* ctx, int nslab);
int full_state_3d(sfd_ctx* ctx);
int run_gradient_3d(sfd_ctx* ctx, const float* obs, float* misfit, float* grad_vp, bool batched, bool dev);
}  // namespace

namespace {

// Fill the kernel argument block for step `step`; buffers alternate each step.
Acou2DArgs make_args(const sfd_ctx* c, int step) {
    Acou2DArgs a{};
    const long long fs = (long long)c->nshot * c->L.shot_stride;
    float* P[2] = {c->d_state, c->d_state + fs};
    float* VX[2] = {c->d_state + 2 * fs, c->d_state + 3 * fs};
    float* VZ[2] = {c->d_state + 4 * fs, c->d_state + 5 * fs};
    const int i = step & 1, o = (step + 1) & 1;
    a.p_in = P[i]; a.p_out = P[o];
    a.vx_in = VX[i]; a.vx_out = VX[o];
    a.vz_in = VZ[i]; a.vz_out = VZ[o];
    a.L = c->L;
    a.nz = c->g.nz;
    a.pml = c->g.pml;
    a.vp = c->d_vp + kModelGhostZ;  // row z = 0 of column 0
    a.den = c->varden ? c->d_den + kModelGhostZ : nullptr;
    a.mpitch = c->mpitch;
    a.nx_model = c->g.nx;
    a.den_c = c->den_c;
    a.dt = c->g.dt;
    a.dtdx = c->g.dt / c->g.dx;
    a.dtdz = c->g.dt / c->g.dz;
    a.rdx_d = 1.0 / (double)c->g.dx;
    a.rdz_d = 1.0 / (double)c->g.dz;
    a.bx_d = (1.0 / (double)c->den_c) * (double)a.dtdx;
    a.bz_d = (1.0 / (double)c->den_c) * (double)a.dtdz;
    a.bx_f = (float)a.bx_d;
    a.bz_f = (float)a.bz_d;
    a.rdx_f = 1.0f / c->g.dx;
    a.rdz_f = 1.0f / c->g.dz;
    for (int m = 0; m < c->radius; m++) {
        a.coef[m] = c->coef[m];
        a.coef2[m] = make_float2(c->coef[m], c->coef[m]);
    }
    for (int q = 0; q < c->g.pml && q < 256; q++)
        a.sponge[q] = -0.38 * q * q / (1.0 * c->g.pml * c->g.pml) + 1;
    a.shots = c->d_shots;
    a.slot_to_shot = c->d_slot;
    a.wavelets = c->d_wav;
    a.rec_x = c->d_rec_x;
    a.rec_z = c->d_rec_z;
    a.tile_rec_ptr = c->d_trp;
    a.tile_rec_idx = c->d_tri;
    a.tile_major = c->tile_major;
    a.tile_order = c->tile_major ? c->d_torder : nullptr;
    a.l2_ahead = c->l2_ahead;
    a.records = c->d_rec_tn;
    a.tm_p = c->tmaps[i];
    a.tm_vx = c->tmaps[2 + i];
    a.tm_vz = c->tmaps[4 + i];
    a.tm_mp = c->mtmaps[i];
    a.tm_mvx = c->mtmaps[2 + i];
    a.tm_mvz = c->mtmaps[4 + i];
    a.err_flag = c->d_err;
    a.test_cta = c->test_cta;
    a.test_step = c->test_step;
    a.test_wait_ns = c->test_wait_ns;
    a.step = step;
    for (const auto& sn : c->snaps)
        if (sn.count > 0 && sn.field == SFD_FIELD_P) a.src_pre = c->d_src_pre;
    return a;
}

int active_shots(const sfd_ctx* c, int step) {
    int n = 0;
    for (int s : c->order)
        if (c->h_shots[s].nt > step) n++;
    return n;
}

// Arguments of the 3-D step: buffers alternate each step like the 2-D ones.
Acou3DArgs make_args3(const sfd_ctx* c, int step) {
    Acou3DArgs a{};
    const long long fs = (long long)c->state_slabs * c->L3.shot_stride;
    const int i = step & 1, o = (step + 1) & 1;
    float* F = c->d_state;
    a.p_in = F + i * fs; a.p_out = F + o * fs;
    a.vx_in = F + (2 + i) * fs; a.vx_out = F + (2 + o) * fs;
    a.vy_out = F + (4 + o) * fs;
    a.vz_out = F + (6 + o) * fs;
    a.tm_p = c->tmaps3[i];
    a.tm_vy = c->tmaps3[2 + i];
    a.tm_vz = c->tmaps3[4 + i];
    a.err_flag = c->d_err;
    a.L = c->L3;
    a.vp = c->d_vp;
    a.den = c->varden ? c->d_den : nullptr;
    a.den_c = c->den_c;
    a.dt = c->g.dt;
    a.rdx = 1.0f / c->g.dx; a.rdy = 1.0f / c->g.dy; a.rdz = 1.0f / c->g.dz;
    a.dtdx = c->g.dt / c->g.dx; a.dtdy = c->g.dt / c->g.dy; a.dtdz = c->g.dt / c->g.dz;
    for (int m = 0; m < c->radius; m++) a.coef[m] = c->coef[m];
    a.pml = c->g.pml;
    for (int q = 0; q < c->g.pml && q < 256; q++) a.sponge[q] = -0.38 * q * q / (1.0 * c->g.pml * c->g.pml) + 1;
    a.slot_to_shot = c->d_slot;
    return a;
}

// Arguments of the viscoacoustic step (fields in place, eight slabs per shot).
QArgs make_qargs(const sfd_ctx* c, int step);

// Arguments of the fused viscoacoustic step (default mode), step k: reads parity k & 1 of sigma,
// vx, vz and writes parity (k + 1) & 1; r and the split parts of the sponge bands in place.
QFastArgs make_qfast(const sfd_ctx* c, int step) {
    QFastArgs A{};
    A.q = make_qargs(c, step);
    const long long fs = (long long)c->nshot * c->L.shot_stride;
    float* F = c->d_state;
    const int i = step & 1, o = (step + 1) & 1;
    A.vx_in = F + (kQVX + i) * fs; A.vx_out = F + (kQVX + o) * fs;
    A.vz_in = F + (kQVZ + i) * fs; A.vz_out = F + (kQVZ + o) * fs;
    A.s_in = F + (kQS + i) * fs; A.s_out = F + (kQS + o) * fs;
    A.r = F + kQR * fs;
    A.q.vx = A.q.vz = nullptr;
    A.q.sx = F + (kQSplit + 0) * fs; A.q.sz = F + (kQSplit + 1) * fs; A.q.sr = F + (kQSplit + 2) * fs;
    A.q.rx = F + (kQSplit + 3) * fs; A.q.rz = F + (kQSplit + 4) * fs; A.q.rr = F + (kQSplit + 5) * fs;
    A.tm_s = c->qtmaps[i];
    A.e1 = F + kQE * fs;
    A.e4 = F + (kQE + 1) * fs;
    A.err_flag = c->d_err;
    return A;
}

QArgs make_qargs(const sfd_ctx* c, int step) {
    QArgs a{};
    const long long fs = (long long)c->nshot * c->L.shot_stride;
    float* f[8];
    for (int i = 0; i < 8; i++) f[i] = c->d_state + i * fs;
    a.vx = f[0]; a.vz = f[1]; a.sx = f[2]; a.sz = f[3]; a.sr = f[4]; a.rx = f[5]; a.rz = f[6]; a.rr = f[7];
    a.L = c->L;
    a.nz = c->g.nz;
    a.npx = a.npz = c->g.pml;
    a.busg = c->q_busg + kModelGhostZ;
    a.p1 = c->q_p1 + kModelGhostZ;
    a.p2 = c->q_p2 + kModelGhostZ;
    a.mpitch = c->mpitch;
    a.nx_model = c->q_width;
    a.dt = c->g.dt;
    a.f_mem = c->g.dt * (-1.0f * c->q_rtau);  // QS:1160 dt*(-1.0*rtaustss)
    a.hx = 0.5f / c->g.dx;
    a.hz = 0.5f / c->g.dz;
    a.dz2 = c->g.dz * c->g.dz;
    const float af[5] = {19845.0f / 16384.0f, -735.0f / 8192.0f, 567.0f / 40960.0f, -405.0f / 229376.0f,
                         35.0f / 294912.0f};
    std::memcpy(a.a, af, sizeof(af));
    a.spg = c->d_spg;
    a.spg_stride = c->spg_stride;
    a.shots = c->d_shots;
    a.slot_to_shot = c->d_slot;
    a.wavelets = c->d_wav;
    a.stamps = c->d_stamps;
    a.rec_x = c->d_rec_x;
    a.rec_z = c->d_rec_z;
    a.tile_rec_ptr = c->d_trp;
    a.tile_rec_idx = c->d_tri;
    a.records = c->d_rec_tn;
    a.step = step;
    return a;
}

// Arguments of the visco-elastic step (22 in-place split fields per shot).
EArgs make_eargs(const sfd_ctx* c, int step) {
    EArgs a{};
    const QArgs q = make_qargs(c, step);
    const long long fs = (long long)c->nshot * c->L.shot_stride;
    for (int i = 0; i < E_NFIELDS; i++) a.f[i] = c->d_state + i * fs;
    a.L = q.L;
    a.nz = q.nz; a.npx = q.npx; a.npz = q.npz;
    a.busg = q.busg;
    a.q1 = c->e_q[0] + kModelGhostZ; a.q2 = c->e_q[1] + kModelGhostZ; a.q3 = c->e_q[2] + kModelGhostZ;
    a.m1 = c->e_q[3] + kModelGhostZ; a.m2 = c->e_q[4] + kModelGhostZ; a.m3 = c->e_q[5] + kModelGhostZ;
    a.mpitch = q.mpitch; a.nx_model = q.nx_model;
    a.dt = q.dt; a.f_mem = q.f_mem; a.hx = q.hx; a.hz = q.hz; a.dz2 = q.dz2;
    std::memcpy(a.a, q.a, sizeof(a.a));
    a.spg = q.spg; a.spg_stride = q.spg_stride;
    a.shots = q.shots; a.slot_to_shot = q.slot_to_shot;
    a.wavelets = q.wavelets; a.stamps = q.stamps;
    a.rec_x = q.rec_x; a.rec_z = q.rec_z; a.tile_rec_ptr = q.tile_rec_ptr; a.tile_rec_idx = q.tile_rec_idx;
    a.records = c->d_rec_tn;
    a.records2 = c->d_rec2_tn;
    a.step = step;
    return a;
}

// Arguments of the isotropic elastic step (ten in-place split fields per shot).
IArgs make_iargs(const sfd_ctx* c, int step) {
    IArgs a{};
    const long long fs = (long long)c->nshot * c->L.shot_stride;
    for (int i = 0; i < I_NFIELDS; i++) a.f[i] = c->d_state + i * fs;
    a.L = c->L;
    a.nz = c->g.nz;
    a.npx = a.npz = c->g.pml;
    a.b2e = c->e_q[0] + kModelGhostZ; a.b1e = c->e_q[1] + kModelGhostZ; a.lm2 = c->e_q[2] + kModelGhostZ;
    a.lam = c->e_q[3] + kModelGhostZ; a.mue = c->e_q[4] + kModelGhostZ;
    a.mpitch = c->mpitch;
    a.nx_model = c->q_width;
    a.dt = c->g.dt;
    a.dtdx = c->g.dt / c->g.dx;  // YPUB:1113 (dt/dx)
    a.dtdz = c->g.dt / c->g.dz;
    a.dz2 = c->g.dz * c->g.dz;
    const float af[5] = {19845.0f / 16384.0f, -735.0f / 8192.0f, 567.0f / 40960.0f, -405.0f / 229376.0f,
                         35.0f / 294912.0f};  // YMOD:23-27
    std::memcpy(a.a, af, sizeof(af));
    // YMOD:7-20: the lower orders caluz uses next to the free surface
    const float cr[4][4] = {{1.0f, 0.0f, 0.0f, 0.0f},
                            {9.0f / 8.0f, -1.0f / 24.0f, 0.0f, 0.0f},
                            {75.0f / 64.0f, -25.0f / 384.0f, 3.0f / 640.0f, 0.0f},
                            {1225.0f / 1024.0f, -245.0f / 3072.0f, 49.0f / 5120.0f, -5.0f / 7168.0f}};
    std::memcpy(a.cr, cr, sizeof(cr));
    a.fs = c->iso_top > 0 ? 1 : 0;
    a.itopo = c->d_itopo;
    a.spg = c->d_spg;
    a.spg_stride = c->spg_stride;
    a.shots = c->d_shots;
    a.slot_to_shot = c->d_slot;
    a.wavelets = c->d_wav;
    a.stamps = c->d_stamps;
    a.rec_x = c->d_rec_x;
    a.rec_z = c->d_rec_z;
    a.tile_rec_ptr = c->d_trp;
    a.tile_rec_idx = c->d_tri;
    a.records = c->d_rec_tn;
    a.records2 = c->d_rec2_tn;
    a.step = step;
    return a;
}

// First row of the snapshot interior: the top pad (pml; the free surface's pad in fsbc mode).
int snap_top(const sfd_ctx* ctx) {
    return (ctx->g.scheme == SFD_ELASTIC_2D && ctx->iso_top > 0) ? ctx->iso_top : ctx->g.pml;
}

// Size the snapshot buffers for the current shot set; returns true if a buffer moved (the
// captured time loop holds their addresses).
bool snap_prepare(sfd_ctx* ctx, int* rc) {
    *rc = SFD_OK;
    bool moved = false;
    const int pml = ctx->g.pml, nzi = ctx->g.nz - snap_top(ctx) - pml;
    for (auto& sn : ctx->snaps) {
        sn.ready = false;
        if (sn.count <= 0) continue;
        sn.off.assign(ctx->nshot, 0);
        sn.taken.assign(ctx->nshot, 0);
        long long total = 0;
        for (int s = 0; s < ctx->nshot; s++) {
            const ShotDev& d = ctx->h_shots[s];
            const int t = d.nt > sn.first ? std::min(sn.count, (d.nt - 1 - sn.first) / sn.every + 1) : 0;
            sn.taken[s] = t;
            sn.off[s] = total;
            total += (long long)t * (d.nx - 2 * pml) * nzi;
        }
        if (!sn.d_buf || total != sn.total) {
            dfree(sn.d_buf);
            dfree(sn.d_off);
            if (cudaMalloc(&sn.d_buf, sizeof(float) * std::max<long long>(total, 1)) != cudaSuccess ||
                cudaMalloc(&sn.d_off, sizeof(long long) * ctx->nshot) != cudaSuccess) {
                cudaGetLastError();
                *rc = set_err(ctx, SFD_ERR_NOMEM, "snapshot buffer of %lld floats", total);
                return true;
            }
            moved = true;
        }
        sn.total = total;
        if (cudaMemcpy(sn.d_off, sn.off.data(), sizeof(long long) * ctx->nshot, cudaMemcpyHostToDevice) !=
            cudaSuccess) {
            *rc = set_err(ctx, SFD_ERR_CUDA, "snapshot offsets upload");
            return true;
        }
    }
    return moved;
}

// Snapshots due after step k for the shots in slots[0 .. act).
int snap_after_step(sfd_ctx* ctx, int k, const int* slots, int act, long long* launches) {
    for (auto& sn : ctx->snaps) {
        if (sn.count <= 0 || k < sn.first || (k - sn.first) % sn.every != 0) continue;
        const int j = (k - sn.first) / sn.every;
        if (j >= sn.count) continue;
        SnapArgs s{};
        const long long fs = (long long)ctx->nshot * ctx->L.shot_stride;
        const float* F = ctx->d_state;
        if (q_fast(ctx)) {
            const int o = (k + 1) & 1;  // parity written by step k
            s.nsum = 1;
            s.f[0] = F + (sn.field == SFD_FIELD_VX ? kQVX + o : sn.field == SFD_FIELD_VZ ? kQVZ + o
                          : sn.field == SFD_FIELD_P ? kQS + o : kQR) * fs;
        } else if (ctx->g.scheme == SFD_VISCOAC_2D) {
            const int f0 = sn.field == SFD_FIELD_VX ? 0 : sn.field == SFD_FIELD_VZ ? 1 : sn.field == SFD_FIELD_P ? 2 : 5;
            s.nsum = (sn.field == SFD_FIELD_P || sn.field == SFD_FIELD_R) ? 3 : 1;
            for (int i = 0; i < s.nsum; i++) s.f[i] = F + (f0 + i) * fs;
        } else if (ctx->g.scheme == SFD_ELASTIC_2D) {
            int f0;  // first of the field's two split parts
            switch (sn.field) {
            case SFD_FIELD_VX: f0 = I_VXX; break;
            case SFD_FIELD_VZ: f0 = I_VZX; break;
            case SFD_FIELD_P: f0 = I_SXXX; break;
            case SFD_FIELD_SZZ: f0 = I_SZZX; break;
            default: f0 = I_SXZX; break;
            }
            s.nsum = 2;
            for (int i = 0; i < 2; i++) s.f[i] = F + (f0 + i) * fs;
        } else if (ctx->g.scheme == SFD_VISCOEL_2D) {
            int f0;  // first split part; velocities have two, stresses and memory variables three
            switch (sn.field) {
            case SFD_FIELD_VX: f0 = E_VXX; break;
            case SFD_FIELD_VZ: f0 = E_VZX; break;
            case SFD_FIELD_P: f0 = E_SXXX; break;
            case SFD_FIELD_SZZ: f0 = E_SZZX; break;
            case SFD_FIELD_SXZ: f0 = E_SXZX; break;
            default: f0 = E_RXXX; break;
            }
            s.nsum = f0 < E_SXXX ? 2 : 3;
            for (int i = 0; i < s.nsum; i++) s.f[i] = F + (f0 + i) * fs;
        } else {
            const int o = (k + 1) & 1;  // buffer written by step k
            const int f0 = sn.field == SFD_FIELD_P ? 0 : sn.field == SFD_FIELD_VX ? 2 : 4;
            s.nsum = 1;
            s.f[0] = F + (f0 + o) * fs;
            if (sn.field == SFD_FIELD_P) s.src_pre = ctx->d_src_pre;
        }
        s.L = ctx->L;
        s.nz = ctx->g.nz;
        s.pml = ctx->g.pml;
        s.ztop = snap_top(ctx);
        s.shots = ctx->d_shots;
        s.slot_to_shot = slots;
        s.step = k;
        s.index = j;
        s.out = sn.d_buf;
        s.shot_off = sn.d_off;
        int nx_max = 0;
        for (const auto& d : ctx->h_shots) nx_max = std::max(nx_max, d.nx);
        CK(launch_snapshot(s, act, nx_max, ctx->stream));
        *launches += 1;
    }
    return SFD_OK;
}

int launch_one_step(sfd_ctx* ctx, int k, const int* slots, int act, long long* launches) {
    if (ctx->g.scheme == SFD_ACOUSTIC_3D) {
        Acou3DArgs a = make_args3(ctx, k);
        a.slot_to_shot = slots;
        float* p_in = const_cast<float*>(a.p_in);
        CK(acoustic3d_launch_inject(p_in, ctx->L3, ctx->d_shots, slots, act, ctx->d_wav, k, ctx->stream));
        CK(acoustic3d_launch_step(ctx->radius, a, act, ctx->varden, ctx->stream));
        CK(acoustic3d_launch_gather(a.p_out, ctx->L3, ctx->d_shots, slots, act, ctx->d_rec_x, ctx->d_rec_y,
                                    ctx->d_rec_z, ctx->d_rec_tn, ctx->nrec_max, k, ctx->stream));
        *launches += 2 + (ctx->nrec_max > 0 ? 1 : 0);
        return SFD_OK;
    }
    if (q_fast(ctx)) {
        QFastArgs q = make_qfast(ctx, k);
        q.q.slot_to_shot = slots;
        int nx_max = 0;
        for (const auto& d : ctx->h_shots) nx_max = std::max(nx_max, d.nx);
        CK(viscoac2d_fast_launch(q, act, q_fast_seg(ctx, act), nx_max, ctx->stream, pdl_enabled()));
        *launches += 2;
        return SFD_OK;
    }
    if (ctx->g.scheme == SFD_VISCOAC_2D) {
        QArgs q = make_qargs(ctx, k);
        q.slot_to_shot = slots;
        CK(viscoac2d_launch_step(q, act, ctx->stream));
        *launches += 2;
        return SFD_OK;
    }
    if (ctx->g.scheme == SFD_ELASTIC_2D) {
        IArgs e = make_iargs(ctx, k);
        e.slot_to_shot = slots;
        int n = 0;
        CK(elastic2d_launch_step(e, act, ctx->L.ntx * kTileX, ctx->stream, &n));
        *launches += n;
        return SFD_OK;
    }
    if (ctx->g.scheme == SFD_VISCOEL_2D) {
        EArgs e = make_eargs(ctx, k);
        e.slot_to_shot = slots;
        CK(viscoel2d_launch_step(e, act, ctx->stream));
        *launches += 2;
        return SFD_OK;
    }
    Acou2DArgs a = make_args(ctx, k);
    a.slot_to_shot = slots;
    CK(acoustic2d_launch_step(ctx->plan, a, act, (ctx->g.flags & SFD_EXACT) != 0, ctx->varden, ctx->stream));
    *launches += 1;
    return SFD_OK;
}

// Zero the wavefields and the record buffer, inject the step-0 source sample.
int prologue(sfd_ctx* ctx) {
    CK(cudaMemsetAsync(ctx->d_state, 0, ctx->state_floats * sizeof(float), ctx->stream));
    CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    CK(cudaMemsetAsync(ctx->d_rec_tn, 0, std::max<long long>(ctx->rec_total, 1) * sizeof(float), ctx->stream));
    if (ctx->d_rec2_tn)
        CK(cudaMemsetAsync(ctx->d_rec2_tn, 0, std::max<long long>(ctx->rec_total, 1) * sizeof(float), ctx->stream));
    // the viscoacoustic source is added inside every step, the 3-D one by its own launch
    if (ctx->g.scheme != SFD_ACOUSTIC_2D) return SFD_OK;
    Acou2DArgs a = make_args(ctx, -1);  // step -1 writes into buffer 0
    CK(acoustic2d_launch_inject0(a, ctx->nshot, (ctx->g.flags & SFD_EXACT) != 0, ctx->stream));
    return SFD_OK;
}

int enqueue_loop(sfd_ctx* ctx, long long* launches) {
    for (int k = 0; k < ctx->nt_max; k++) {
        const int act = active_shots(ctx, k);
        if (act == 0) break;
        int rc = launch_one_step(ctx, k, ctx->d_slot, act, launches);
        if (rc || (rc = snap_after_step(ctx, k, ctx->d_slot, act, launches))) return rc;
    }
    return SFD_OK;
}

int epilogue(sfd_ctx* ctx, float* out_dev) {
    CK(launch_records_transpose(ctx->d_rec_tn, out_dev, ctx->d_shots, ctx->nshot, ctx->nrec_max, ctx->nt_max,
                                ctx->stream));
    if (ctx->d_rec2_tn) {
        CK(launch_records_transpose(ctx->d_rec2_tn, ctx->d_rec2_nt, ctx->d_shots, ctx->nshot, ctx->nrec_max,
                                    ctx->nt_max, ctx->stream));
        ctx->rec2_ready = true;
    }
    if (ctx->g.flags & SFD_NAN_CHECK) {
        CK(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
        CK(launch_nan_scan(out_dev, ctx->rec_total, ctx->d_flag, ctx->stream));
    }
    return SFD_OK;
}

int check_ready(sfd_ctx* ctx) {
    if (!ctx) return SFD_ERR_ARG;
    if (!ctx->have_model) return set_err(ctx, SFD_ERR_STATE, "sfd_set_model has not been called");
    if (!ctx->have_shots) return set_err(ctx, SFD_ERR_STATE, "sfd_set_shots has not been called");
    CK(cudaSetDevice(ctx->device));
    return SFD_OK;
}

int finish_nan(sfd_ctx* ctx) {
    int err = 0;
    CK(cudaMemcpy(&err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return set_err(ctx, SFD_ERR_TIMEOUT, "a step kernel gave up waiting for its tile loads");
    if (ctx->g.flags & SFD_NAN_CHECK) {
        int flag = 0;
        CK(cudaMemcpy(&flag, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost));
        if (flag) return set_err(ctx, SFD_ERR_NAN, "non-finite value in the receiver traces");
    }
    return SFD_OK;
}

// Tuner for the forward step of the default (FMA) scheme.  Candidates: the tile kernel with one
// tile per CTA (two CTAs per SM), the persistent tile kernel with double-buffered TMA, and the
// x-marching kernel with segments of 128, 256 or 512 columns (segments longer than the shots are
// skipped).  Each runs a few steps on the real shot set, twice; the fastest is kept.  All
// candidates give bit-identical results.  SFD_FMA_STAGES=1|2 forces a tile schedule,
// SFD_MARCH_SEG=<columns> forces the x-marching kernel with that segment length.
int tune_schedule(sfd_ctx* ctx) {
    if ((ctx->g.flags & SFD_EXACT) || ctx->g.scheme != SFD_ACOUSTIC_2D) return SFD_OK;
    if (const char* env = std::getenv("SFD_FMA_STAGES")) {
        const int s = std::atoi(env);
        if (s == 1 || s == 2) {
            ctx->plan.stages = s;
            ctx->plan.seg = 0;
            ctx->plan.forced = false;
            return SFD_OK;
        }
    }
    if (const char* env = std::getenv("SFD_MARCH_SEG")) {
        const int s = std::atoi(env);
        if (s >= 16 && s % 16 == 0) {
            ctx->plan.stages = 1;
            ctx->plan.seg = s;
            ctx->plan.forced = true;
            return SFD_OK;
        }
    }
    struct Cand {
        int stages, seg;
    };
    std::vector<Cand> cands = {{1, 0}, {2, 0}};
    const int width = ctx->L.ntx * ctx->L.tx;
    for (int seg : {128, 256, 512})
        if (seg < width || seg == 128) cands.push_back({1, seg});
    const int act = active_shots(ctx, 0);
    const int steps = std::min(ctx->nt_max, 10);
    std::vector<float> best(cands.size(), 1e30f);
    for (int round = 0; round < 2; round++)  // two rounds, best of each candidate
        for (size_t ci = 0; ci < cands.size(); ci++) {
            ctx->plan.stages = cands[ci].stages;
            ctx->plan.seg = cands[ci].seg;
            ctx->plan.forced = false;
            int rc = prologue(ctx);
            if (rc) return rc;
            for (int k = 0; k < steps; k++) {
                if (k == 2) CK(cudaEventRecord(ctx->ev0, ctx->stream));
                CK(acoustic2d_launch_step(ctx->plan, make_args(ctx, k), act, false, ctx->varden, ctx->stream));
            }
            CK(cudaEventRecord(ctx->ev1, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            float ms = 0.0f;
            if (steps > 2) CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
            best[ci] = std::min(best[ci], ms);
        }
    size_t pick = 0;
    for (size_t ci = 1; ci < cands.size(); ci++)
        if (best[ci] < best[pick]) pick = ci;
    ctx->plan.stages = cands[pick].stages;
    ctx->plan.seg = cands[pick].seg;
    return SFD_OK;
}

int kernel_variant(const sfd_ctx* ctx) {
    if (ctx->g.scheme == SFD_ACOUSTIC_3D) return 30;
    if (ctx->g.scheme == SFD_VISCOAC_2D) return q_fast(ctx) ? 41 : 40;
    if (ctx->g.scheme == SFD_VISCOEL_2D) return 45;
    if (ctx->g.scheme == SFD_ELASTIC_2D) return 50;
    if (ctx->g.flags & SFD_EXACT) return 1;
    return acoustic2d_use_march(ctx->plan, ctx->L, active_shots(ctx, 0)) ? 13 : 10 + ctx->plan.stages;
}

int run_forward(sfd_ctx* ctx, float* out_dev) {
    int rc;
    long long launches = 0;
    if (ctx->g.scheme == SFD_ACOUSTIC_3D && (rc = full_state_3d(ctx))) return rc;
    if (snap_prepare(ctx, &rc)) ctx->graph_valid = false;
    if (rc) return rc;
    if (!ctx->graph_valid) {
        if ((rc = tune_schedule(ctx)) != SFD_OK) return rc;
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        rc = enqueue_loop(ctx, &launches);
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
        if (rc != SFD_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        CK(e);
        if (ctx->graph) cudaGraphExecDestroy(ctx->graph);
        e = cudaGraphInstantiate(&ctx->graph, g, 0);
        cudaGraphDestroy(g);
        CK(e);
        ctx->graph_valid = true;
    } else {
        for (int k = 0; k < ctx->nt_max && active_shots(ctx, k) > 0; k++) launches++;
        for (const auto& sn : ctx->snaps)
            for (int k = sn.first; sn.count > 0 && k < ctx->nt_max && (k - sn.first) / sn.every < sn.count;
                 k += sn.every)
                launches++;
    }
    CK(cudaEventRecord(ctx->evs, ctx->stream));
    if ((rc = prologue(ctx)) != SFD_OK) return rc;
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    CK(cudaGraphLaunch(ctx->graph, ctx->stream));
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    if ((rc = epilogue(ctx, out_dev)) != SFD_OK) return rc;
    CK(cudaEventRecord(ctx->eve, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.0f, dms = 0.0f;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    CK(cudaEventElapsedTime(&dms, ctx->evs, ctx->eve));
    ctx->timing.loop_ms = ms;
    ctx->timing.device_ms = dms;
    ctx->timing.launches = launches + 2 + ((ctx->g.flags & SFD_NAN_CHECK) ? 1 : 0);
    ctx->timing.graph = 1;
    for (auto& sn : ctx->snaps) sn.ready = sn.count > 0;
    ctx->timing.kernel_variant = kernel_variant(ctx);
    double pts = 0;
    for (const auto& s : ctx->h_shots) pts += (double)s.nx * ctx->g.ny * ctx->g.nz * s.nt;
    ctx->timing.point_updates = pts;
    return finish_nan(ctx);
}

// d tau_eps/tau_sigma / d (1/Q) of QS:473-551 (Blanch's tau: tau_p = (1/(0.9 Q)) (ln-ratio)
// / (atan-ratio)), in double, for the chain rule of the viscoacoustic gradient.
double q_kappa(float f0) {
    const double pi = 3.1415926, flow = 2.0 * 2.0 * pi, fup = 2.5 * (double)f0 * 2.0 * pi;
    const double tss = 1.0 / ((fup - flow) / 2.0);
    const double nlow = std::log(tss * tss * flow * flow + 1.0), nup = std::log(tss * tss * fup * fup + 1.0);
    const double dlow = std::atan(flow * tss) - flow * tss / (1.0 + tss * tss * flow * flow);
    const double dup = std::atan(fup * tss) - fup * tss / (1.0 + tss * tss * fup * fup);
    return (20.0 / 18.0) * (nup - nlow) / (dup - dlow);
}

// ---------------------------------------------------------------------------------------------
// Gradient: forward with checkpoints every C steps, residuals and misfit, then for each segment
// (last to first) restore its checkpoint, recompute its C forward steps keeping D_k, and run
// the C adjoint steps backwards accumulating the zero-lag imaging sum.
// ---------------------------------------------------------------------------------------------
// Per scheme: fields kept in a checkpoint, forward derivatives kept per recomputed step,
// adjoint fields, imaging sums.  Acoustic: P, Vx, Vz (one parity) / D / Q, X, Z ping-pong /
// g.  Viscoacoustic: the eight in-place fields / Dx1 vx, Dz1 vz / eight adjoints + Qx, Qz /
// g1, g2.
struct GradShape {
    int ckpt, div, adj, img;
};
GradShape grad_shape(const sfd_ctx* c) {
    return c->g.scheme == SFD_VISCOAC_2D ? GradShape{8, 2, 10, 2} : GradShape{3, 1, 6, 1};
}

int grad_alloc(sfd_ctx* ctx) {
    const int C = ctx->ckpt_interval > 0 ? std::min(ctx->ckpt_interval, ctx->nt_max)
                                         : (int)std::ceil(std::sqrt((double)ctx->nt_max));
    const int ncp = (ctx->nt_max + C - 1) / C;
    if (ctx->d_ckpt && C == ctx->grad_C && ncp == ctx->grad_ncp) return SFD_OK;
    dfree(ctx->d_ckpt); dfree(ctx->d_div);
    if (ctx->grad_graph) cudaGraphExecDestroy(ctx->grad_graph);
    ctx->grad_graph = nullptr;
    ctx->grad_valid = false;
    const GradShape gs = grad_shape(ctx);
    const size_t fs = (size_t)ctx->nshot * ctx->L.shot_stride;
    const size_t nrec = std::max<long long>(1, ctx->rec_total);
    CK(cudaMalloc(&ctx->d_ckpt, sizeof(float) * fs * gs.ckpt * ncp));
    if (!ctx->d_adj) {
        CK(cudaMalloc(&ctx->d_adj, sizeof(float) * fs * gs.adj));
        CK(cudaMalloc(&ctx->d_gseg, sizeof(float) * fs * gs.img));
        CK(cudaMalloc(&ctx->d_gacc, sizeof(double) * fs * gs.img));
        if (ctx->g.scheme == SFD_ACOUSTIC_2D) {
            int bp[2], bvx[2], bvz[2];
            acoustic2d_fma_boxes(ctx->radius, bp, bvx, bvz);
            const int* boxes[3] = {bp, bvx, bvz};
            int mp[2], mvx[2], mvz[2];
            acoustic2d_march_boxes(mp, mvx, mvz);
            const int* mboxes[3] = {mp, mvx, mvz};
            for (int b = 0; b < 6; b++) {
                int rc = encode_field_map(ctx, &ctx->adj_tmaps[b], ctx->d_adj + b * fs, ctx->L, ctx->nshot,
                                          boxes[b / 2]);
                if (!rc)
                    rc = encode_field_map(ctx, &ctx->adj_mtmaps[b], ctx->d_adj + b * fs, ctx->L, ctx->nshot,
                                          mboxes[b / 2]);
                if (rc) return rc;
            }
        }
        if (ctx->g.scheme == SFD_VISCOAC_2D) {
            CK(cudaMalloc(&ctx->d_grad2, sizeof(double) * (size_t)ctx->g.nx * ctx->g.nz));
            CK(cudaMalloc(&ctx->d_apx0, sizeof(int) * ctx->nshot));
            CK(cudaMemcpy(ctx->d_apx0, ctx->h_ap_x0.data(), sizeof(int) * ctx->nshot, cudaMemcpyHostToDevice));
        }
        CK(cudaMalloc(&ctx->d_obs_nt, sizeof(float) * nrec));
        CK(cudaMalloc(&ctx->d_obs_tn, sizeof(float) * nrec));
        CK(cudaMalloc(&ctx->d_res, sizeof(float) * nrec));
        CK(cudaMalloc(&ctx->d_lam, sizeof(float) * (size_t)ctx->nshot * ctx->nt_max));
        CK(cudaMalloc(&ctx->d_misfit, sizeof(double)));
        CK(cudaMalloc(&ctx->d_grad, sizeof(double) * (size_t)ctx->g.nx * ctx->g.nz));
    }
    // D_k slots: C for the segment being recomputed, plus as many tail steps as the memory budget
    // holds (whole segments from the last one back): the first forward keeps their D_k, and those
    // segments are transposed without recomputation
    const size_t slot = sizeof(float) * fs * gs.div;
    size_t freeb = 0, totb = 0;
    CK(cudaMemGetInfo(&freeb, &totb));
    double budget = 0.85 * (double)freeb - (double)(1ull << 30) - (double)slot * C;
    if (ctx->mem_limit > 0) budget = std::min(budget, (double)ctx->mem_limit - (double)slot * C);
    const long long extra = budget > 0 ? (long long)(budget / (double)slot) : 0;
    int keep = ncp;  // segments keep .. ncp-1 are kept
    while (keep > 0 && (long long)ctx->nt_max - (long long)(keep - 1) * C <= extra) keep--;
    const long long nslots = C + ((long long)ctx->nt_max - (long long)keep * C);
    if (cudaMalloc(&ctx->d_div, slot * nslots) != cudaSuccess) {
        cudaGetLastError();
        keep = ncp;
        CK(cudaMalloc(&ctx->d_div, slot * C));
    }
    ctx->grad_keep = keep;
    ctx->grad_C = C;
    ctx->grad_ncp = ncp;
    return SFD_OK;
}

// shots [first, first + count) as one schedule; `slots` maps launch slots to shots
struct GradRange {
    int first, count;
    const int* slots;
    bool batched;
};

// Kernel plan of the gradient's forward, recomputation and adjoint steps: the tile kernel with
// the tuned schedule (on config 4 it is 5% faster than the x-marching kernel over a whole
// gradient: 18.6 against 17.7 shots/s), x-marching only when SFD_MARCH_SEG forces it.
Acou2DPlan grad_plan(const sfd_ctx* ctx) {
    Acou2DPlan p = ctx->plan;
    if (!p.forced) p.seg = 0;
    return p;
}

int range_active(const sfd_ctx* ctx, const GradRange& r, int k) {
    if (r.batched) return active_shots(ctx, k);
    return ctx->h_shots[r.first].nt > k ? 1 : 0;
}

int grad_fwd_step(sfd_ctx* ctx, const GradRange& r, int k, int act, float* div_out) {
    if (ctx->g.scheme == SFD_VISCOAC_2D) {
        QArgs q = make_qargs(ctx, k);
        q.slot_to_shot = r.slots;
        if (div_out) {
            q.d1_out = div_out;
            q.d4_out = div_out + (size_t)ctx->nshot * ctx->L.shot_stride;
        }
        CK(viscoac2d_launch_step(q, act, ctx->stream));
        return SFD_OK;
    }
    Acou2DArgs a = make_args(ctx, k);
    a.slot_to_shot = r.slots;
    a.div_out = div_out;
    CK(acoustic2d_fwd_launch(grad_plan(ctx), ctx->radius, a, act, ctx->varden, ctx->stream));
    return SFD_OK;
}

// arguments of the viscoacoustic adjoint kernels (q_adjoint2d.cu) for forward step k
QAdjArgs make_qadj(const sfd_ctx* ctx, const GradRange& r, int k, const float* div) {
    const long long fs = (long long)ctx->nshot * ctx->L.shot_stride;
    const QArgs f = make_qargs(ctx, k);
    QAdjArgs a{};
    float* A = ctx->d_adj;
    a.avx = A; a.avz = A + fs; a.asx = A + 2 * fs; a.asz = A + 3 * fs; a.asr = A + 4 * fs;
    a.arx = A + 5 * fs; a.arz = A + 6 * fs; a.arr = A + 7 * fs; a.qx = A + 8 * fs; a.qz = A + 9 * fs;
    a.d1 = div;
    a.d4 = div ? div + fs : nullptr;
    a.g1 = ctx->d_gseg;
    a.g2 = ctx->d_gseg + fs;
    a.L = ctx->L;
    a.nz = f.nz; a.npx = f.npx; a.npz = f.npz;
    a.busg = f.busg; a.p1 = f.p1; a.p2 = f.p2;
    a.mpitch = f.mpitch; a.nx_model = f.nx_model;
    a.dt = f.dt; a.f_mem = f.f_mem; a.hx = f.hx; a.hz = f.hz; a.dz2 = f.dz2;
    std::memcpy(a.a, f.a, sizeof(a.a));
    a.spg = f.spg; a.spg_stride = f.spg_stride;
    a.shots = ctx->d_shots;
    a.slot_to_shot = r.slots;
    a.stamps = f.stamps;
    a.res = ctx->d_res;
    a.rec_x = ctx->d_rec_x; a.rec_z = ctx->d_rec_z;
    a.tile_rec_ptr = ctx->d_trp; a.tile_rec_idx = ctx->d_tri;
    a.lam_src = ctx->d_lam;
    a.nt_max = ctx->nt_max;
    a.step = k;
    return a;
}

int grad_adj_step_q(sfd_ctx* ctx, const GradRange& r, int k, int act, const float* div) {
    CK(q_adjoint_launch_step(make_qadj(ctx, r, k, div), act, ctx->stream));
    return SFD_OK;
}

// Arguments of the FMA kernel in adjoint mode for forward step k: reads buffer (k+1) & 1 of
// nu, X, Z and writes buffer k & 1.
Acou2DArgs make_adj_args(const sfd_ctx* ctx, const GradRange& r, int k, const float* div) {
    const long long fs = (long long)ctx->nshot * ctx->L.shot_stride;
    Acou2DArgs a = make_args(ctx, k);
    const int i = (k + 1) & 1, o = k & 1;
    float* A = ctx->d_adj;
    a.p_in = A + i * fs; a.p_out = A + o * fs;
    a.vx_in = A + (2 + i) * fs; a.vx_out = A + (2 + o) * fs;
    a.vz_in = A + (4 + i) * fs; a.vz_out = A + (4 + o) * fs;
    a.tm_p = ctx->adj_tmaps[i];
    a.tm_vx = ctx->adj_tmaps[2 + i];
    a.tm_vz = ctx->adj_tmaps[4 + i];
    a.tm_mp = ctx->adj_mtmaps[i];
    a.tm_mvx = ctx->adj_mtmaps[2 + i];
    a.tm_mvz = ctx->adj_mtmaps[4 + i];
    a.slot_to_shot = r.slots;
    a.tile_major = 0;
    a.tile_order = nullptr;
    a.records = nullptr;
    a.src_pre = nullptr;
    a.div_out = nullptr;
    a.adj_div = div;
    a.adj_g = ctx->d_gseg;
    a.adj_res = ctx->d_res;
    a.adj_lam = ctx->d_lam;
    a.nt_max = ctx->nt_max;
    a.adj_cx = ctx->varden ? 1.0f : a.dtdx / ctx->den_c;
    a.adj_cz = ctx->varden ? 1.0f : a.dtdz / ctx->den_c;
    a.adj_xs = ctx->g.dx / ctx->g.dt;
    a.adj_zs = ctx->g.dz / ctx->g.dt;
    return a;
}

int grad_adj_step(sfd_ctx* ctx, const GradRange& r, int k, int act, const float* div) {
    if (ctx->g.scheme == SFD_VISCOAC_2D) return grad_adj_step_q(ctx, r, k, act, div);
    if (acoustic2d_use_march(grad_plan(ctx), ctx->L, act))
        CK(acoustic2d_march_launch(ctx->radius, make_adj_args(ctx, r, k, div), act, ctx->varden, ctx->plan.seg,
                                   ctx->stream, pdl_enabled(), true));
    else
        CK(acoustic2d_fma_launch(ctx->radius, make_adj_args(ctx, r, k, div), act, ctx->varden, ctx->plan.stages,
                                 ctx->stream, true));
    return SFD_OK;
}

// copy the three forward fields of parity b for the shots of r between the state and a
// checkpoint slot (to_ckpt = save, else restore)
int grad_copy_state(sfd_ctx* ctx, const GradRange& r, int slot, int b, bool to_ckpt) {
    const size_t fs = (size_t)ctx->nshot * ctx->L.shot_stride;
    const size_t off = (size_t)r.first * ctx->L.shot_stride, len = (size_t)r.count * ctx->L.shot_stride;
    const bool visco = ctx->g.scheme == SFD_VISCOAC_2D;  // eight in-place fields, no parity
    const int nf = grad_shape(ctx).ckpt;
    for (int f = 0; f < nf; f++) {
        float* st = ctx->d_state + (visco ? f : 2 * f + b) * fs + off;
        float* ck = ctx->d_ckpt + ((size_t)slot * nf + f) * fs + off;
        CK(cudaMemcpyAsync(to_ckpt ? ck : st, to_ckpt ? st : ck, len * sizeof(float), cudaMemcpyDeviceToDevice,
                           ctx->stream));
    }
    return SFD_OK;
}

int enqueue_gradient_range(sfd_ctx* ctx, const GradRange& r, long long* launches) {
    int rc;
    const int C = ctx->grad_C, ncp = ctx->grad_ncp;
    const size_t fs = (size_t)ctx->nshot * ctx->L.shot_stride;
    const size_t off = (size_t)r.first * ctx->L.shot_stride, len = (size_t)r.count * ctx->L.shot_stride;
    const GradShape gs = grad_shape(ctx);
    const bool visco = ctx->g.scheme == SFD_VISCOAC_2D;
    const int per_step = visco ? 2 : 1;  // launches per forward or adjoint step
    int nrec_max = 0;
    for (int s = r.first; s < r.first + r.count; s++) nrec_max = std::max(nrec_max, ctx->h_shots[s].nrec);
    // D_k slot of step k: kept tail steps after the C recomputation slots
    const int kkeep = ctx->grad_keep * C;
    auto dslot = [&](int k, int k0) -> float* {
        const size_t i = k >= kkeep ? (size_t)C + (k - kkeep) : (size_t)(k - k0);
        return ctx->d_div + i * gs.div * fs;
    };
    // forward with checkpoints (and D_k of the kept tail)
    for (int k = 0; k < ctx->nt_max; k++) {
        const int act = range_active(ctx, r, k);
        if (act == 0) break;
        if (k % C == 0 && (rc = grad_copy_state(ctx, r, k / C, k & 1, true))) return rc;
        if ((rc = grad_fwd_step(ctx, r, k, act, k >= kkeep ? dslot(k, 0) : nullptr))) return rc;
        *launches += per_step;
    }
    // residuals of this range and the misfit
    const ShotDev& s0 = ctx->h_shots[r.first];
    const ShotDev& s1 = ctx->h_shots[r.first + r.count - 1];
    const long long rb = s0.rec_base, re = s1.rec_base + (long long)s1.nrec * s1.nt;
    CK(launch_residual(ctx->d_rec_tn + rb, ctx->d_obs_tn + rb, ctx->d_res + rb, re - rb, ctx->d_misfit, ctx->stream));
    if (visco) {
        CK(q_adjoint_launch_init(make_qadj(ctx, r, 0, nullptr), r.first, r.count, nrec_max, ctx->stream));
    } else {
        CK(launch_adjoint_init(ctx->d_adj, ctx->d_adj + fs, make_adj_args(ctx, r, 0, nullptr), ctx->radius, r.first,
                               r.count, nrec_max, ctx->stream));
    }
    *launches += 2;
    // segments, last to first
    for (int j = ncp - 1; j >= 0; j--) {
        const int k0 = j * C, k1 = std::min(k0 + C, ctx->nt_max);
        if (range_active(ctx, r, k0) == 0) continue;
        for (int i = 0; i < gs.img; i++)
            CK(cudaMemsetAsync(ctx->d_gseg + i * fs + off, 0, len * sizeof(float), ctx->stream));
        if (j < ctx->grad_keep) {  // recompute the segment from its checkpoint, keeping D_k
            if ((rc = grad_copy_state(ctx, r, j, k0 & 1, false))) return rc;
            for (int k = k0; k < k1; k++) {
                const int act = range_active(ctx, r, k);
                if (act == 0) break;
                if ((rc = grad_fwd_step(ctx, r, k, act, dslot(k, k0)))) return rc;
                *launches += per_step;
            }
        }
        for (int k = k1 - 1; k >= k0; k--) {
            const int act = range_active(ctx, r, k);
            if (act == 0) continue;
            if ((rc = grad_adj_step(ctx, r, k, act, dslot(k, k0)))) return rc;
            *launches += per_step;
        }
        for (int i = 0; i < gs.img; i++) {
            CK(launch_accumulate(ctx->d_gacc + i * fs + off, ctx->d_gseg + i * fs + off, (long long)len, ctx->stream));
            (*launches)++;
        }
    }
    return SFD_OK;
}

int enqueue_gradient(sfd_ctx* ctx, bool batched, long long* launches) {
    int rc;
    const size_t fs = (size_t)ctx->nshot * ctx->L.shot_stride;
    if ((rc = prologue(ctx))) return rc;
    CK(cudaMemsetAsync(ctx->d_misfit, 0, sizeof(double), ctx->stream));
    const GradShape gs = grad_shape(ctx);
    CK(cudaMemsetAsync(ctx->d_adj, 0, gs.adj * fs * sizeof(float), ctx->stream));
    CK(cudaMemsetAsync(ctx->d_gacc, 0, gs.img * fs * sizeof(double), ctx->stream));
    CK(cudaMemsetAsync(ctx->d_lam, 0, sizeof(float) * (size_t)ctx->nshot * ctx->nt_max, ctx->stream));
    int nrec_max = 0;
    for (const auto& s : ctx->h_shots) nrec_max = std::max(nrec_max, s.nrec);
    CK(launch_records_transpose_in(ctx->d_obs_nt, ctx->d_obs_tn, ctx->d_shots, ctx->nshot, nrec_max, ctx->nt_max,
                                   ctx->stream));
    *launches += 2;
    if (batched) {
        const GradRange r{0, ctx->nshot, ctx->d_slot, true};
        if ((rc = enqueue_gradient_range(ctx, r, launches))) return rc;
    } else {
        for (int s = 0; s < ctx->nshot; s++) {
            const GradRange r{s, 1, ctx->d_ident + s, false};
            if ((rc = enqueue_gradient_range(ctx, r, launches))) return rc;
        }
    }
    if (ctx->g.scheme == SFD_VISCOAC_2D) {
        const QArgs q = make_qargs(ctx, 0);
        CK(q_launch_gradient_reduce(ctx->d_gacc, ctx->d_gacc + fs, ctx->L, ctx->d_shots, ctx->d_apx0, ctx->nshot,
                                    ctx->d_vp + kModelGhostZ, q.p1, q.p2, ctx->mpitch, ctx->g.nx, ctx->g.nz,
                                    (double)q.dt, (double)q.f_mem, q_kappa(ctx->g.f0), ctx->d_grad, ctx->d_grad2,
                                    ctx->stream));
        (*launches)++;
        return SFD_OK;
    }
    CK(launch_gradient_reduce(ctx->d_gacc, ctx->L, ctx->d_shots, ctx->nshot, ctx->d_vp + kModelGhostZ, ctx->mpitch,
                              ctx->g.nx, ctx->g.nz, ctx->d_grad, ctx->stream));
    (*launches)++;
    return SFD_OK;
}

// Outputs to the caller's device memory: misfit (one float), grad_vp and grad_invq (model grid
// floats), converted from the double sums on the device, with the source term of d misfit / d vp
// added there in the host path's order (the results equal sfd_gradient's bit for bit).
int finish_gradient_device(sfd_ctx* ctx, float* misfit, float* grad_vp, float* grad_invq, bool source_term) {
    const bool is3d = ctx->g.scheme == SFD_ACOUSTIC_3D;
    const long long nm = (long long)ctx->g.nx * (is3d ? ctx->g.ny : 1) * ctx->g.nz;
    if (grad_vp && source_term) {
        std::vector<GradSrc> src(ctx->nshot);
        for (int s = 0; s < ctx->nshot; s++) {
            const ShotDev& sd = ctx->h_shots[s];
            const size_t mi = is3d ? ((size_t)sd.sx * ctx->g.ny + sd.sy) * ctx->g.nz + sd.sz
                                   : (size_t)(sd.x0 + sd.sx) * ctx->g.nz + sd.sz;
            const double den = ctx->varden ? ctx->h_den[mi] : ctx->den_c;
            src[s].mi = (long long)mi;
            src[s].scale = -(double)ctx->g.dt * den;
        }
        if (!ctx->d_gsrc) CK(cudaMalloc(&ctx->d_gsrc, sizeof(GradSrc) * ctx->nshot));
        CK(cudaMemcpyAsync(ctx->d_gsrc, src.data(), sizeof(GradSrc) * src.size(), cudaMemcpyHostToDevice, ctx->stream));
        CK(launch_grad_source(ctx->d_grad, ctx->d_gsrc, ctx->d_shots, ctx->nshot, ctx->d_lam, ctx->nt_max, ctx->d_wav,
                              ctx->stream));
    }
    if (grad_vp) CK(launch_to_float(ctx->d_grad, grad_vp, nm, ctx->stream));
    if (grad_invq) CK(launch_to_float(ctx->d_grad2, grad_invq, nm, ctx->stream));
    if (misfit) CK(launch_to_float(ctx->d_misfit, misfit, 1, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->timing.h2d_bytes = 0;
    ctx->timing.d2h_bytes = 0;
    return SFD_OK;
}

int run_gradient(sfd_ctx* ctx, const float* obs, float* misfit, float* grad_vp, float* grad_invq, bool batched,
                 bool dev = false) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (!obs) return set_err(ctx, SFD_ERR_ARG, "observed records are required");
    const bool visco = ctx->g.scheme == SFD_VISCOAC_2D;
    if (ctx->g.scheme == SFD_ACOUSTIC_3D) {
        if (grad_invq) return set_err(ctx, SFD_ERR_ARG, "grad_invq applies to the viscoacoustic scheme only");
        return run_gradient_3d(ctx, obs, misfit, grad_vp, batched, dev);
    }
    if (ctx->g.scheme != SFD_ACOUSTIC_2D && !visco)
        return set_err(ctx, SFD_ERR_UNSUPPORTED, "scheme %d has no gradient", ctx->g.scheme);
    if (grad_invq && !visco) return set_err(ctx, SFD_ERR_ARG, "grad_invq applies to the viscoacoustic scheme only");
    auto t0 = std::chrono::steady_clock::now();
    if ((rc = grad_alloc(ctx))) return rc;
    if (!ctx->graph_valid && (rc = tune_schedule(ctx))) return rc;
    CK(cudaMemcpyAsync(ctx->d_obs_nt, obs, sizeof(float) * ctx->rec_total,
                       dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
    long long launches = 0;
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    if (batched) {
        if (!ctx->grad_valid) {
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            rc = enqueue_gradient(ctx, true, &launches);
            cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            CK(e);
            if (ctx->grad_graph) cudaGraphExecDestroy(ctx->grad_graph);
            e = cudaGraphInstantiate(&ctx->grad_graph, g, 0);
            cudaGraphDestroy(g);
            CK(e);
            ctx->grad_valid = true;
            ctx->timing.launches = launches;
        }
        CK(cudaEventRecord(ctx->ev0, ctx->stream));
        CK(cudaGraphLaunch(ctx->grad_graph, ctx->stream));
    } else {
        if ((rc = enqueue_gradient(ctx, false, &launches))) return rc;
        ctx->timing.launches = launches;
    }
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    int err = 0;
    CK(cudaMemcpy(&err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return set_err(ctx, SFD_ERR_TIMEOUT, "a step kernel gave up waiting for its tile loads");
    ctx->timing.loop_ms = ms;
    ctx->timing.device_ms = ms;
    ctx->timing.graph = batched ? 1 : 0;
    ctx->timing.kernel_variant =
        visco ? 50 : (acoustic2d_use_march(grad_plan(ctx), ctx->L, batched ? active_shots(ctx, 0) : 1) ? 23
                                                                                             : 20 + ctx->plan.stages);
    // forward, recomputation of the segments before the kept tail, adjoint
    double pts = 0;
    const int kkeep = ctx->grad_keep * ctx->grad_C;
    for (const auto& s : ctx->h_shots) pts += (double)s.nx * ctx->g.nz * (2.0 * s.nt + std::min(s.nt, kkeep));
    ctx->timing.point_updates = pts;
    if (dev) {
        ctx->have_grad = true;
        rc = finish_gradient_device(ctx, misfit, grad_vp, grad_invq, !visco);
        ctx->timing.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return rc;
    }
    double mis = 0;
    CK(cudaMemcpy(&mis, ctx->d_misfit, sizeof(double), cudaMemcpyDeviceToHost));
    if (misfit) *misfit = (float)mis;
    ctx->have_grad = true;
    const size_t nm = (size_t)ctx->g.nx * ctx->g.nz;
    if (visco) {
        std::vector<double> g(nm);
        if (grad_vp) {
            CK(cudaMemcpy(g.data(), ctx->d_grad, nm * sizeof(double), cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < nm; i++) grad_vp[i] = (float)g[i];
        }
        if (grad_invq) {
            CK(cudaMemcpy(g.data(), ctx->d_grad2, nm * sizeof(double), cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < nm; i++) grad_invq[i] = (float)g[i];
        }
    } else if (grad_vp) {
        const size_t n = (size_t)ctx->g.nx * ctx->g.nz;
        std::vector<double> g(n);
        CK(cudaMemcpy(g.data(), ctx->d_grad, n * sizeof(double), cudaMemcpyDeviceToHost));
        // source scaling: P[src] -= (dt DEN Vp) w[k]  ->  -dt DEN sum_k lambda_k[src] w[k]
        std::vector<float> lam((size_t)ctx->nshot * ctx->nt_max);
        CK(cudaMemcpy(lam.data(), ctx->d_lam, lam.size() * sizeof(float), cudaMemcpyDeviceToHost));
        for (int s = 0; s < ctx->nshot; s++) {
            const ShotDev& sd = ctx->h_shots[s];
            const size_t mi = (size_t)(sd.x0 + sd.sx) * ctx->g.nz + sd.sz;
            const double den = ctx->varden ? ctx->h_den[mi] : ctx->den_c;
            double sw = 0;
            for (int j = 0; j < sd.nt; j++) sw += (double)lam[(size_t)s * ctx->nt_max + j] * ctx->h_wav[sd.wav_off + j];
            g[mi] += -(double)ctx->g.dt * den * sw;
        }
        for (size_t i = 0; i < n; i++) grad_vp[i] = (float)g[i];
    }
    ctx->timing.h2d_bytes = (long long)sizeof(float) * ctx->rec_total;
    ctx->timing.d2h_bytes = (long long)sizeof(float) * nm * ((grad_vp ? 1 : 0) + (grad_invq ? 1 : 0));
    ctx->timing.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return SFD_OK;
}

// Viscoacoustic model preparation, QS:434-551 (averaged density -> buoyancy, Lame and Blanch
// tau), done per shot window as QS does for each shot's padded grid: the 2 x 2 density average
// and its edge rule stop at the window's last row and column.  Every distinct window (aperture
// start and width) gets its own block of the prepared arrays; shot x0 becomes that block's start.
// Without shots the whole grid is one window.
int q_prepare(sfd_ctx* ctx) {
    const bool elastic = ctx->g.scheme == SFD_VISCOEL_2D;
    const bool iso = ctx->g.scheme == SFD_ELASTIC_2D;
    if ((ctx->g.scheme != SFD_VISCOAC_2D && !elastic && !iso) || !ctx->have_model) return SFD_OK;
    const int nz = ctx->g.nz;
    std::vector<std::pair<int, int>> wins;  // (x0, nx)
    std::vector<int> blk(ctx->have_shots ? ctx->nshot : 0);
    if (ctx->have_shots) {
        for (int s = 0; s < ctx->nshot; s++) {
            const std::pair<int, int> w(ctx->h_ap_x0[s], ctx->h_shots[s].nx);
            auto it = std::find(wins.begin(), wins.end(), w);
            blk[s] = (int)(it - wins.begin());
            if (it == wins.end()) wins.push_back(w);
        }
    } else {
        wins.emplace_back(0, ctx->g.nx);
    }
    int width = 0;
    std::vector<int> start(wins.size());
    for (size_t b = 0; b < wins.size(); b++) {
        start[b] = width;
        width += wins[b].second;
    }
    if (iso && wins == ctx->prep_wins && ctx->model_gen == ctx->prep_gen && ctx->iso_rgau == ctx->prep_rgau &&
        ctx->iso_top == ctx->prep_top && ctx->topo_gen == ctx->prep_topo_gen && width == ctx->q_width) {
        if (ctx->have_shots) {
            for (int s = 0; s < ctx->nshot; s++) ctx->h_shots[s].x0 = start[blk[s]];
            CK(cudaMemcpy(ctx->d_shots, ctx->h_shots.data(), sizeof(ShotDev) * ctx->nshot, cudaMemcpyHostToDevice));
        }
        return SFD_OK;
    }
    // yang_version surface rows per prepared column: the topography's itopo, or flat (the top pad:
    // pml in abc mode, the free surface's row in fsbc mode); YPUB:270-272
    std::vector<int> itopo(iso ? width : 0);
    if (iso) {
        const int flat = ctx->iso_top > 0 ? ctx->iso_top : ctx->g.pml;
        const int lo = ctx->iso_top > 0 ? 1 : ctx->g.pml, hi = nz - ctx->g.pml - 6;
        for (size_t b = 0; b < wins.size(); b++)
            for (int c = 0; c < wins[b].second; c++) {
                const int v = ctx->h_itopo.empty() ? flat : ctx->h_itopo[wins[b].first + c];
                if (v < lo || v > hi)
                    return set_err(ctx, SFD_ERR_ARG, "surface row %d of column %d outside [%d, %d]", v,
                                   wins[b].first + c, lo, hi);
                itopo[start[b] + c] = v;
            }
    }
    std::vector<float> busg((size_t)width * nz), p1((size_t)width * nz), p2((size_t)width * nz);
    std::vector<std::vector<float>> eq(elastic ? 6 : iso ? 5 : 0, std::vector<float>((size_t)width * nz));
    for (size_t b = 0; b < wins.size(); b++) {
        const size_t off = (size_t)wins[b].first * nz, len = (size_t)wins[b].second * nz;
        std::vector<float> rho(len, ctx->den_c);
        if (!ctx->h_den.empty()) rho.assign(ctx->h_den.begin() + off, ctx->h_den.begin() + off + len);
        const float* qw = ctx->h_q.empty() ? nullptr : ctx->h_q.data() + off;
        const size_t o = (size_t)start[b] * nz;
        if (iso) {  // YPUB:323-547 per window, flat surface: itopo = npzn (pml, or the free surface's row)
            std::vector<float> vs(len, 0.0f);
            if (!ctx->h_vs.empty()) vs.assign(ctx->h_vs.begin() + off, ctx->h_vs.begin() + off + len);
            if (!elastic2d_prepare(wins[b].second, nz, ctx->h_vp.data() + off, vs.data(), rho.data(),
                                   itopo.data() + start[b],
                                   eq[0].data() + o, eq[1].data() + o, eq[2].data() + o, eq[3].data() + o,
                                   eq[4].data() + o))
                return set_err(ctx, SFD_ERR_ARG, "zero density in the window at column %d", wins[b].first);
        } else if (elastic) {
            std::vector<float> vs(len, 0.0f);
            if (!ctx->h_vs.empty()) vs.assign(ctx->h_vs.begin() + off, ctx->h_vs.begin() + off + len);
            const float* qsw = ctx->h_qs.empty() ? nullptr : ctx->h_qs.data() + off;
            viscoel2d_prepare(wins[b].second, nz, ctx->h_vp.data() + off, vs.data(), rho.data(), qw, qsw, ctx->g.f0,
                              busg.data() + o, eq[0].data() + o, eq[1].data() + o, eq[2].data() + o,
                              eq[3].data() + o, eq[4].data() + o, eq[5].data() + o, &ctx->q_rtau);
        } else {
            viscoac2d_prepare(wins[b].second, nz, ctx->h_vp.data() + off, rho.data(), qw, ctx->g.f0, busg.data() + o,
                              p1.data() + o, p2.data() + o, &ctx->q_rtau);
        }
    }
    // upload with kModelGhostZ replicated rows (the layout of the other model arrays)
    const size_t mfloats = (size_t)width * ctx->mpitch;
    auto upload = [&](float** dst, const std::vector<float>& src) -> int {
        std::vector<float> staged(mfloats);
        for (int c = 0; c < width; c++)
            for (int k = 0; k < ctx->mpitch; k++)
                staged[(size_t)c * ctx->mpitch + k] = src[(size_t)c * nz + std::min(std::max(k - kModelGhostZ, 0), nz - 1)];
        if (width != ctx->q_width) {
            dfree(*dst);
            ctx->graph_valid = false;
        }
        if (!*dst) CK(cudaMalloc(dst, mfloats * sizeof(float)));
        CK(cudaMemcpy(*dst, staged.data(), mfloats * sizeof(float), cudaMemcpyHostToDevice));
        return SFD_OK;
    };
    int rc;
    if (iso) {
        for (int i = 0; i < 5; i++)
            if ((rc = upload(&ctx->e_q[i], eq[i]))) return rc;
        if (width != ctx->q_width) dfree(ctx->d_itopo);
        if (!ctx->d_itopo) CK(cudaMalloc(&ctx->d_itopo, sizeof(int) * width));
        CK(cudaMemcpy(ctx->d_itopo, itopo.data(), sizeof(int) * width, cudaMemcpyHostToDevice));
        // YPUB:549-634 modipapml on the device (abc mode only, YPRI:301-302): rows z < pml of the
        // five arrays, per window
        std::vector<int> win;
        if (ctx->iso_top == 0)
            for (size_t b = 0; b < wins.size(); b++) {
                win.push_back(start[b]);
                win.push_back(wins[b].second);
            }
        float* arrs[5];
        for (int i = 0; i < 5; i++) arrs[i] = ctx->e_q[i] + kModelGhostZ;
        CK(elastic2d_smooth(arrs, ctx->mpitch, kModelGhostZ, nz, ctx->d_itopo, win.data(), (int)win.size() / 2,
                            ctx->iso_gc, ctx->iso_rgau, ctx->iso_lo, ctx->iso_hi, ctx->stream));
    } else if ((rc = upload(&ctx->q_busg, busg))) {
        return rc;
    }
    if (elastic) {
        for (int i = 0; i < 6; i++)
            if ((rc = upload(&ctx->e_q[i], eq[i]))) return rc;
    } else if (!iso && ((rc = upload(&ctx->q_p1, p1)) || (rc = upload(&ctx->q_p2, p2)))) {
        return rc;
    }
    if (width != ctx->q_width) ctx->graph_valid = ctx->grad_valid = false;
    ctx->q_width = width;
    ctx->prep_wins = wins;
    ctx->prep_gen = ctx->model_gen;
    ctx->prep_rgau = ctx->iso_rgau;
    ctx->prep_top = ctx->iso_top;
    ctx->prep_topo_gen = ctx->topo_gen;
    if (ctx->have_shots) {
        for (int s = 0; s < ctx->nshot; s++) ctx->h_shots[s].x0 = start[blk[s]];
        CK(cudaMemcpy(ctx->d_shots, ctx->h_shots.data(), sizeof(ShotDev) * ctx->nshot, cudaMemcpyHostToDevice));
    }
    return SFD_OK;
}

// Gaussian source stamps of the current shots (QS:1340-1444; YPUB:1429-1466 with the context's
// rgau), uploaded with the shot descriptors.
int build_stamps(sfd_ctx* ctx) {
    const int nz = ctx->g.nz;
    std::vector<float> stamps;
    for (int s = 0; s < ctx->nshot; s++) {
        int box[4];
        ShotDev& d = ctx->h_shots[s];
        d.stamp_off = (int)stamps.size();
        if (ctx->g.scheme == SFD_ELASTIC_2D)
            elastic2d_stamp(d.nx, nz, d.sx, d.sz, ctx->iso_rgau, ctx->iso_gc, box, &stamps);
        else
            viscoac2d_stamp(d.nx, nz, d.sx, d.sz, box, &stamps);
        d.stamp_x0 = box[0];
        d.stamp_z0 = box[1];
        d.stamp_w = box[2];
        d.stamp_h = box[3];
    }
    dfree(ctx->d_stamps);
    CK(cudaMalloc(&ctx->d_stamps, sizeof(float) * std::max<size_t>(1, stamps.size())));
    if (!stamps.empty())
        CK(cudaMemcpy(ctx->d_stamps, stamps.data(), sizeof(float) * stamps.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_shots, ctx->h_shots.data(), sizeof(ShotDev) * ctx->nshot, cudaMemcpyHostToDevice));
    ctx->graph_valid = false;
    return SFD_OK;
}

// (Re)allocate the 3-D wavefields for `nslab` shot slabs per field (eight fields: P, Vx, Vy, Vz,
// two buffers each) and encode the TMA descriptors of the P, Vy and Vz buffers.  The forward
// holds every shot; the gradient may shrink the state to its shot-group size, and the next
// forward grows it back (the captured time loop is rebuilt because the buffers moved).
int alloc_state_3d(sfd_ctx* ctx, int nslab) {
    if (ctx->d_state && ctx->state_slabs == nslab) return SFD_OK;
    dfree(ctx->d_state);
    ctx->state_slabs = 0;
    ctx->graph_valid = false;
    const Layout3D& L = ctx->L3;
    ctx->state_floats = 8 * (size_t)nslab * L.shot_stride;
    if (cudaMalloc(&ctx->d_state, ctx->state_floats * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        ctx->d_state = nullptr;
        return set_err(ctx, SFD_ERR_NOMEM, "3-D wavefields of %d shots need %.1f GB of device memory", nslab,
                       ctx->state_floats * 4.0 / 1e9);
    }
    int bp[2], bvy[2], bvz[2];
    acoustic3d_boxes(ctx->radius, bp, bvy, bvz);
    const int* boxes[3] = {bp, bvy, bvz};
    const int field_of[3] = {0, 4, 6};  // P, Vy, Vz
    const long long fs = (long long)nslab * L.shot_stride;
    for (int f = 0; f < 3; f++)
        for (int b = 0; b < 2; b++) {
            const int rc = encode_field_map3(ctx, &ctx->tmaps3[2 * f + b], ctx->d_state + (field_of[f] + b) * fs, L,
                                             nslab, boxes[f]);
            if (rc) return rc;
        }
    ctx->state_slabs = nslab;
    return SFD_OK;
}

// The forward holds every shot's wavefields: release the gradient's buffers if the state was
// shrunk to a shot group, then grow it back.
int full_state_3d(sfd_ctx* ctx) {
    if (ctx->d_state && ctx->state_slabs == ctx->nshot) return SFD_OK;
    dfree(ctx->g3_adj); dfree(ctx->g3_div); dfree(ctx->g3_ck1); dfree(ctx->g3_ck2);
    dfree(ctx->g3_gseg); dfree(ctx->g3_gacc);
    ctx->g3_G = 0;
    return alloc_state_3d(ctx, ctx->nshot);
}

// sfd_set_shots for the 3-D scheme: every shot covers the whole grid (no aperture windows);
// sources must lie where the step updates P (R <= coordinate < n - R on every axis).
int set_shots_3d(sfd_ctx* ctx, int nshot, const sfd_shot* shots) {
    CK(cudaSetDevice(ctx->device));
    const sfd_grid& g = ctx->g;
    const int R = ctx->radius;
    std::vector<ShotDev> hs(nshot);
    std::vector<int> rx, ry, rz;
    std::vector<float> wav;
    std::vector<long long> out_off(nshot);
    long long rec_total = 0;
    int nt_max = 0, nrec_max = 0;
    for (int s = 0; s < nshot; s++) {
        const sfd_shot& sh = shots[s];
        if (sh.ap_x0 != 0 || (sh.ap_nx != 0 && sh.ap_nx != g.nx))
            return set_err(ctx, SFD_ERR_UNSUPPORTED, "shot %d: aperture windows are 2-D only", s);
        if (sh.nt < 1 || !sh.wavelet) return set_err(ctx, SFD_ERR_ARG, "shot %d: nt=%d or wavelet missing", s, sh.nt);
        if (sh.sx < R || sh.sx >= g.nx - R || sh.sy < R || sh.sy >= g.ny - R || sh.sz < R || sh.sz >= g.nz - R)
            return set_err(ctx, SFD_ERR_ARG, "shot %d: source (%d, %d, %d) outside the updated region", s, sh.sx,
                           sh.sy, sh.sz);
        if (sh.nrec < 0 || (sh.nrec > 0 && (!sh.rec_x || !sh.rec_y || !sh.rec_z)))
            return set_err(ctx, SFD_ERR_ARG, "shot %d: receiver list missing (3-D needs rec_y)", s);
        ShotDev d{};
        d.nx = g.nx; d.x0 = 0; d.nt = sh.nt; d.sx = sh.sx; d.sy = sh.sy; d.sz = sh.sz;
        d.nrec = sh.nrec;
        d.rec_base = rec_total;
        d.rec_list = (int)rx.size();
        d.wav_off = (int)wav.size();
        for (int r = 0; r < sh.nrec; r++) {
            if (sh.rec_x[r] < 0 || sh.rec_x[r] >= g.nx || sh.rec_y[r] < 0 || sh.rec_y[r] >= g.ny || sh.rec_z[r] < 0 ||
                sh.rec_z[r] >= g.nz)
                return set_err(ctx, SFD_ERR_ARG, "shot %d: receiver %d outside the grid", s, r);
            rx.push_back(sh.rec_x[r]);
            ry.push_back(sh.rec_y[r]);
            rz.push_back(sh.rec_z[r]);
        }
        wav.insert(wav.end(), sh.wavelet, sh.wavelet + sh.nt);
        out_off[s] = rec_total;
        rec_total += (long long)sh.nrec * sh.nt;
        nt_max = std::max(nt_max, sh.nt);
        nrec_max = std::max(nrec_max, sh.nrec);
        if (ctx->have_model) {
            const size_t mi = ((size_t)d.sx * g.ny + d.sy) * g.nz + d.sz;
            float sc = g.dt * (ctx->varden ? ctx->h_den[mi] : ctx->den_c);
            sc = sc * ctx->h_vp[mi];
            d.inj_scale = sc;
        }
        hs[s] = d;
    }
    free_shot_buffers(ctx);
    Layout3D L{};
    L.nx = g.nx; L.ny = g.ny; L.nz = g.nz;
    L.pitch = round_up(g.nz, 4);
    L.xstride = (long long)g.ny * L.pitch;
    L.shot_stride = (long long)g.nx * L.xstride;
    L.nty = (g.ny + kTile3Y - 1) / kTile3Y;
    L.ntz = (g.nz + kTile3Z - 1) / kTile3Z;
    ctx->L3 = L;
    std::vector<int> order(nshot), ident(nshot);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return hs[a].nt > hs[b].nt; });
    std::iota(ident.begin(), ident.end(), 0);
    ctx->h_shots = hs;
    ctx->h_rec_x = rx;
    ctx->h_rec_y = ry;
    ctx->h_rec_z = rz;
    ctx->h_wav = wav;
    ctx->rec_out_off = out_off;
    ctx->rec_total = rec_total;
    ctx->nshot = nshot;
    ctx->nt_max = nt_max;
    ctx->nrec_max = nrec_max;
    ctx->order = order;
    ctx->h_ident_order = ident;
    auto up = [&](auto** dst, const auto& v) -> int {
        using E = typename std::remove_reference<decltype(v)>::type::value_type;
        const size_t bytes = std::max<size_t>(1, v.size()) * sizeof(E);
        CK(cudaMalloc(dst, bytes));
        if (!v.empty()) CK(cudaMemcpy(*dst, v.data(), v.size() * sizeof(E), cudaMemcpyHostToDevice));
        return SFD_OK;
    };
    int rc;
    if ((rc = up(&ctx->d_shots, hs)) || (rc = up(&ctx->d_slot, order)) || (rc = up(&ctx->d_ident, ident)) ||
        (rc = up(&ctx->d_wav, wav)) || (rc = up(&ctx->d_rec_x, rx)) || (rc = up(&ctx->d_rec_y, ry)) ||
        (rc = up(&ctx->d_rec_z, rz)))
        return rc;
    const size_t rec_bytes = sizeof(float) * std::max<long long>(1, rec_total);
    CK(cudaMalloc(&ctx->d_rec_tn, rec_bytes));
    CK(cudaMalloc(&ctx->d_rec_nt, rec_bytes));
    const int rc3 = alloc_state_3d(ctx, nshot);
    if (rc3) return rc3;
    ctx->have_shots = true;
    ctx->graph_valid = false;
    return SFD_OK;
}

// ---------------------------------------------------------------------------------------------
// 3-D gradient.  Shots run in groups of G (launch slots 0..G-1 of a slot list, one field slab per
// slot).  Per group: the forward keeps outer checkpoints every C1 steps and the records; then,
// outer segment by outer segment from the last, either (one level, C2 = C1) the segment is
// recomputed keeping D_k and transposed, or (two levels) it is recomputed keeping inner
// checkpoints every C2 steps and each inner segment is recomputed keeping D_k and transposed.
// G, C1 and C2 are the largest group and the cheapest schedule that fit the memory budget.
// ---------------------------------------------------------------------------------------------
struct Plan3 {
    int G = 0, C1 = 0, C2 = 0, n1 = 0, n2 = 0;
};

// device bytes of a plan: wavefields and adjoint (8 + 8 slabs), imaging sums (1 float + 1 double),
// D of one inner segment and the checkpoints (4 fields each), per slot
double plan3_bytes(const sfd_ctx* c, const Plan3& p) {
    const double F = 4.0 * (double)c->L3.shot_stride;
    return F * p.G * (8.0 + 8.0 + 1.0 + 2.0 + p.C2 + 4.0 * (p.n1 + p.n2));
}

Plan3 plan3_make(int G, int C1, int C2, int nt) {
    Plan3 p;
    p.G = G;
    p.C1 = std::max(1, std::min(C1, nt));
    p.C2 = std::max(1, std::min(C2, p.C1));
    p.n1 = (nt + p.C1 - 1) / p.C1;
    p.n2 = p.C2 < p.C1 ? (p.C1 + p.C2 - 1) / p.C2 : 0;
    return p;
}

int plan3_choose(sfd_ctx* ctx, int Gmax, Plan3* out) {
    size_t freeb = 0, totb = 0;
    CK(cudaMemGetInfo(&freeb, &totb));
    // what this context holds and would release: the wavefields and the gradient buffers
    double held = (double)ctx->state_floats * 4.0;
    if (ctx->g3_G > 0) held += plan3_bytes(ctx, Plan3{ctx->g3_G, ctx->g3_C1, ctx->g3_C2, ctx->g3_n1, ctx->g3_n2});
    // model-sized gradient, observed / residual records, adjoint source traces
    const double fixed = 8.0 * (double)ctx->g.nx * ctx->g.ny * ctx->g.nz + 16.0 * (double)ctx->rec_total +
                         4.0 * (double)ctx->nshot * ctx->nt_max;
    double budget = 0.92 * ((double)freeb + held) - fixed - (double)(64u << 20);
    if (ctx->mem_limit > 0) budget = std::min(budget, (double)ctx->mem_limit - fixed);
    const int nt = ctx->nt_max;
    const int ci = ctx->ckpt_interval;
    for (int G = Gmax; G >= 1; G--) {
        // one level: C minimises 4 ceil(nt / C) + C (or the caller's interval)
        int best = ci > 0 ? ci : 1;
        if (ci <= 0) {
            double bm = 1e300;
            for (int C = 1; C <= nt; C++) {
                const double m = 4.0 * ((nt + C - 1) / C) + C;
                if (m < bm) bm = m, best = C;
            }
        }
        Plan3 p = plan3_make(G, best, best, nt);
        if (plan3_bytes(ctx, p) <= budget) {
            *out = p;
            return SFD_OK;
        }
        // two levels: inner interval C2 (the caller's, or sqrt(4 C1)), outer C1 by search
        Plan3 pb;
        double bb = 1e300;
        for (int C1 = 2; C1 <= nt; C1++) {
            const int C2 = ci > 0 ? std::min(ci, C1 - 1) : std::max(1, (int)std::ceil(std::sqrt(4.0 * C1)) - 1);
            if (C2 >= C1) continue;
            const Plan3 q = plan3_make(G, C1, C2, nt);
            const double m = plan3_bytes(ctx, q);
            if (m < bb) bb = m, pb = q;
        }
        if (pb.G > 0 && bb <= budget) {
            *out = pb;
            return SFD_OK;
        }
    }
    return set_err(ctx, SFD_ERR_NOMEM, "the 3-D gradient of one shot does not fit the memory budget (%.1f GB)",
                   budget / 1e9);
}

int g3_alloc(sfd_ctx* ctx, const Plan3& p) {
    int rc;
    const bool same = ctx->g3_adj && p.G == ctx->g3_G && p.C1 == ctx->g3_C1 && p.C2 == ctx->g3_C2 &&
                      ctx->state_slabs == p.G;
    if (!same) {
        dfree(ctx->g3_adj); dfree(ctx->g3_div); dfree(ctx->g3_ck1); dfree(ctx->g3_ck2);
        dfree(ctx->g3_gseg); dfree(ctx->g3_gacc);
        ctx->g3_G = 0;
        if ((rc = alloc_state_3d(ctx, p.G))) return rc;
        const size_t fsG = (size_t)p.G * ctx->L3.shot_stride;
        CK(cudaMalloc(&ctx->g3_adj, sizeof(float) * fsG * 8));
        CK(cudaMalloc(&ctx->g3_div, sizeof(float) * fsG * p.C2));
        CK(cudaMalloc(&ctx->g3_ck1, sizeof(float) * fsG * 4 * p.n1));
        if (p.n2 > 0) CK(cudaMalloc(&ctx->g3_ck2, sizeof(float) * fsG * 4 * p.n2));
        CK(cudaMalloc(&ctx->g3_gseg, sizeof(float) * fsG));
        CK(cudaMalloc(&ctx->g3_gacc, sizeof(double) * fsG));
        int bp[2], bvy[2], bvz[2];
        acoustic3d_boxes(ctx->radius, bp, bvy, bvz);
        const int* boxes[3] = {bp, bvy, bvz};
        const int field_of[3] = {0, 4, 6};  // nu, Y, Z
        for (int f = 0; f < 3; f++)
            for (int b = 0; b < 2; b++)
                if ((rc = encode_field_map3(ctx, &ctx->g3_tmaps[2 * f + b], ctx->g3_adj + (field_of[f] + b) * fsG,
                                            ctx->L3, p.G, boxes[f])))
                    return rc;
        ctx->g3_G = p.G; ctx->g3_C1 = p.C1; ctx->g3_C2 = p.C2; ctx->g3_n1 = p.n1; ctx->g3_n2 = p.n2;
    }
    if (!ctx->d_obs_nt) {
        const size_t nrec = std::max<long long>(1, ctx->rec_total);
        CK(cudaMalloc(&ctx->d_obs_nt, sizeof(float) * nrec));
        CK(cudaMalloc(&ctx->d_obs_tn, sizeof(float) * nrec));
        CK(cudaMalloc(&ctx->d_res, sizeof(float) * nrec));
        CK(cudaMalloc(&ctx->d_lam, sizeof(float) * (size_t)ctx->nshot * ctx->nt_max));
        CK(cudaMalloc(&ctx->d_misfit, sizeof(double)));
        CK(cudaMalloc(&ctx->d_grad, sizeof(double) * (size_t)ctx->g.nx * ctx->g.ny * ctx->g.nz));
    }
    return SFD_OK;
}

// one forward step of the group's active slots (source before, receivers after when `gather`)
int g3_fwd_step(sfd_ctx* ctx, const int* slots, int act, int k, float* div_out, bool gather, long long* launches) {
    Acou3DArgs a = make_args3(ctx, k);
    a.slot_to_shot = slots;
    a.slab_by_slot = 1;
    a.div_out = div_out;
    CK(acoustic3d_launch_inject(const_cast<float*>(a.p_in), ctx->L3, ctx->d_shots, slots, act, ctx->d_wav, k,
                                ctx->stream, 1));
    CK(acoustic3d_launch_step(ctx->radius, a, act, ctx->varden, ctx->stream));
    *launches += 2;
    if (gather) {
        CK(acoustic3d_launch_gather(a.p_out, ctx->L3, ctx->d_shots, slots, act, ctx->d_rec_x, ctx->d_rec_y,
                                    ctx->d_rec_z, ctx->d_rec_tn, ctx->nrec_max, k, ctx->stream, 1));
        (*launches)++;
    }
    return SFD_OK;
}

// adjoint of forward step k: residual of step k into nu, then the adjoint step
int g3_adj_step(sfd_ctx* ctx, const int* slots, int act, int k, const float* div, long long* launches) {
    Acou3DArgs a = make_args3(ctx, k);
    const long long fsA = (long long)ctx->g3_G * ctx->L3.shot_stride;
    const int i = (k + 1) & 1, o = k & 1;
    float* A = ctx->g3_adj;
    a.p_in = A + i * fsA; a.p_out = A + o * fsA;
    a.vx_in = A + (2 + i) * fsA; a.vx_out = A + (2 + o) * fsA;
    a.vy_out = A + (4 + o) * fsA;
    a.vz_out = A + (6 + o) * fsA;
    a.tm_p = ctx->g3_tmaps[i];
    a.tm_vy = ctx->g3_tmaps[2 + i];
    a.tm_vz = ctx->g3_tmaps[4 + i];
    a.slot_to_shot = slots;
    a.slab_by_slot = 1;
    a.shots = ctx->d_shots;
    a.adj_div = div;
    a.adj_g = ctx->g3_gseg;
    a.adj_lam = ctx->d_lam;
    a.nt_max = ctx->nt_max;
    a.step = k;
    a.adj_radius = ctx->radius;
    a.adj_c[0] = ctx->varden ? 1.0f : a.dtdx / ctx->den_c;
    a.adj_c[1] = ctx->varden ? 1.0f : a.dtdy / ctx->den_c;
    a.adj_c[2] = ctx->varden ? 1.0f : a.dtdz / ctx->den_c;
    CK(acoustic3d_launch_adj_inject(A + i * fsA, a, ctx->d_rec_x, ctx->d_rec_y, ctx->d_rec_z, ctx->d_res, act,
                                    ctx->nrec_max, ctx->stream));
    CK(acoustic3d_launch_step(ctx->radius, a, act, ctx->varden, ctx->stream, true));
    *launches += 2;
    return SFD_OK;
}

// P, Vx, Vy, Vz of parity b (G slabs) to or from checkpoint store `ck` slot j
int g3_copy_state(sfd_ctx* ctx, float* ck, int j, int b, bool save) {
    const size_t fsG = (size_t)ctx->g3_G * ctx->L3.shot_stride;
    const size_t fsS = (size_t)ctx->state_slabs * ctx->L3.shot_stride;
    for (int f = 0; f < 4; f++) {
        float* st = ctx->d_state + (2 * f + b) * fsS;
        float* cp = ck + ((size_t)j * 4 + f) * fsG;
        CK(cudaMemcpyAsync(save ? cp : st, save ? st : cp, sizeof(float) * fsG, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    return SFD_OK;
}

// the gradient of one group: shots h_slots[0..n) (launch slot order, longest record first),
// device slot list `slots`
int g3_group(sfd_ctx* ctx, const int* slots, const std::vector<int>& h_slots, long long* launches) {
    int rc;
    const int n = (int)h_slots.size();
    const int nt = ctx->h_shots[h_slots[0]].nt;
    auto act = [&](int k) {
        int a = 0;
        while (a < n && ctx->h_shots[h_slots[a]].nt > k) a++;
        return a;
    };
    const size_t fsG = (size_t)ctx->g3_G * ctx->L3.shot_stride;
    const int C1 = ctx->g3_C1, C2 = ctx->g3_C2;
    CK(cudaMemsetAsync(ctx->d_state, 0, ctx->state_floats * sizeof(float), ctx->stream));
    CK(cudaMemsetAsync(ctx->g3_adj, 0, sizeof(float) * fsG * 8, ctx->stream));
    CK(cudaMemsetAsync(ctx->g3_gseg, 0, sizeof(float) * fsG, ctx->stream));
    CK(cudaMemsetAsync(ctx->g3_gacc, 0, sizeof(double) * fsG, ctx->stream));
    // forward with outer checkpoints and the records
    for (int k = 0; k < nt; k++) {
        if (k % C1 == 0 && (rc = g3_copy_state(ctx, ctx->g3_ck1, k / C1, k & 1, true))) return rc;
        if ((rc = g3_fwd_step(ctx, slots, act(k), k, nullptr, true, launches))) return rc;
    }
    for (int s : h_slots) {
        const ShotDev& sd = ctx->h_shots[s];
        CK(launch_residual(ctx->d_rec_tn + sd.rec_base, ctx->d_obs_tn + sd.rec_base, ctx->d_res + sd.rec_base,
                           (long long)sd.nrec * sd.nt, ctx->d_misfit, ctx->stream));
        (*launches)++;
    }
    // innermost segment [a, b) restored from store ck slot j: recompute keeping D_k, transpose
    auto inner = [&](float* ck, int j, int a, int b) -> int {
        int r;
        if ((r = g3_copy_state(ctx, ck, j, a & 1, false))) return r;
        for (int k = a; k < b; k++)
            if ((r = g3_fwd_step(ctx, slots, act(k), k, ctx->g3_div + (size_t)(k - a) * fsG, false, launches)))
                return r;
        for (int k = b - 1; k >= a; k--)
            if ((r = g3_adj_step(ctx, slots, act(k), k, ctx->g3_div + (size_t)(k - a) * fsG, launches))) return r;
        CK(launch_accumulate(ctx->g3_gacc, ctx->g3_gseg, (long long)fsG, ctx->stream));
        CK(cudaMemsetAsync(ctx->g3_gseg, 0, sizeof(float) * fsG, ctx->stream));
        (*launches)++;
        return SFD_OK;
    };
    const int n1 = (nt + C1 - 1) / C1;
    for (int j1 = n1 - 1; j1 >= 0; j1--) {
        const int k0 = j1 * C1, k1 = std::min(k0 + C1, nt);
        if (C2 >= C1) {
            if ((rc = inner(ctx->g3_ck1, j1, k0, k1))) return rc;
            continue;
        }
        if ((rc = g3_copy_state(ctx, ctx->g3_ck1, j1, k0 & 1, false))) return rc;
        for (int k = k0; k < k1; k++) {
            if ((k - k0) % C2 == 0 && (rc = g3_copy_state(ctx, ctx->g3_ck2, (k - k0) / C2, k & 1, true))) return rc;
            if ((rc = g3_fwd_step(ctx, slots, act(k), k, nullptr, false, launches))) return rc;
        }
        for (int j2 = (k1 - k0 + C2 - 1) / C2 - 1; j2 >= 0; j2--) {
            const int a = k0 + j2 * C2, b = std::min(a + C2, k1);
            if ((rc = inner(ctx->g3_ck2, j2, a, b))) return rc;
        }
    }
    CK(acoustic3d_launch_gradient_reduce(ctx->g3_gacc, n, ctx->L3, ctx->d_vp, ctx->d_grad, ctx->stream));
    (*launches)++;
    return SFD_OK;
}

int run_gradient_3d(sfd_ctx* ctx, const float* obs, float* misfit, float* grad_vp, bool batched, bool dev) {
    int rc;
    auto t0 = std::chrono::steady_clock::now();
    Plan3 p;
    if ((rc = plan3_choose(ctx, batched ? ctx->nshot : 1, &p))) return rc;
    if ((rc = g3_alloc(ctx, p))) return rc;
    CK(cudaMemcpyAsync(ctx->d_obs_nt, obs, sizeof(float) * ctx->rec_total,
                       dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
    long long launches = 0;
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    CK(cudaMemsetAsync(ctx->d_misfit, 0, sizeof(double), ctx->stream));
    CK(cudaMemsetAsync(ctx->d_grad, 0, sizeof(double) * (size_t)ctx->g.nx * ctx->g.ny * ctx->g.nz, ctx->stream));
    CK(cudaMemsetAsync(ctx->d_lam, 0, sizeof(float) * (size_t)ctx->nshot * ctx->nt_max, ctx->stream));
    CK(cudaMemsetAsync(ctx->d_rec_tn, 0, sizeof(float) * std::max<long long>(1, ctx->rec_total), ctx->stream));
    CK(launch_records_transpose_in(ctx->d_obs_nt, ctx->d_obs_tn, ctx->d_shots, ctx->nshot, ctx->nrec_max, ctx->nt_max,
                                   ctx->stream));
    launches++;
    // groups: consecutive runs of the launch order (longest record first), or one shot each
    const std::vector<int>& ord = batched ? ctx->order : ctx->h_ident_order;
    const int* dslots = batched ? ctx->d_slot : ctx->d_ident;
    const int G = batched ? p.G : 1;
    for (int g0 = 0; g0 < ctx->nshot; g0 += G) {
        const std::vector<int> hs(ord.begin() + g0, ord.begin() + std::min(ctx->nshot, g0 + G));
        if ((rc = g3_group(ctx, dslots + g0, hs, &launches))) return rc;
    }
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    int err = 0;
    CK(cudaMemcpy(&err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return set_err(ctx, SFD_ERR_TIMEOUT, "a 3-D step kernel gave up waiting for its plane loads");
    ctx->timing.loop_ms = ms;
    ctx->timing.device_ms = ms;
    ctx->timing.launches = launches;
    ctx->timing.graph = 0;
    ctx->timing.kernel_variant = 60 + (p.C2 < p.C1 ? 2 : 1);
    double pts = 0;
    for (const auto& sd : ctx->h_shots) pts += (double)sd.nx * ctx->g.ny * ctx->g.nz * sd.nt;
    ctx->timing.point_updates = (p.C2 < p.C1 ? 4.0 : 3.0) * pts;  // forward, recomputation(s), adjoint
    if (dev) {
        ctx->have_grad = true;
        return finish_gradient_device(ctx, misfit, grad_vp, nullptr, true);
    }
    double mis = 0;
    CK(cudaMemcpy(&mis, ctx->d_misfit, sizeof(double), cudaMemcpyDeviceToHost));
    if (misfit) *misfit = (float)mis;
    ctx->have_grad = true;
    const size_t nm = (size_t)ctx->g.nx * ctx->g.ny * ctx->g.nz;
    if (grad_vp) {
        std::vector<double> g(nm);
        CK(cudaMemcpy(g.data(), ctx->d_grad, nm * sizeof(double), cudaMemcpyDeviceToHost));
        // source scaling: P[src] -= (dt DEN Vp) w[k]  ->  -dt DEN sum_k lambda_k[src] w[k]
        std::vector<float> lam((size_t)ctx->nshot * ctx->nt_max);
        CK(cudaMemcpy(lam.data(), ctx->d_lam, lam.size() * sizeof(float), cudaMemcpyDeviceToHost));
        for (int s = 0; s < ctx->nshot; s++) {
            const ShotDev& sd = ctx->h_shots[s];
            const size_t mi = ((size_t)sd.sx * ctx->g.ny + sd.sy) * ctx->g.nz + sd.sz;
            const double den = ctx->varden ? ctx->h_den[mi] : ctx->den_c;
            double sw = 0;
            for (int j = 0; j < sd.nt; j++) sw += (double)lam[(size_t)s * ctx->nt_max + j] * ctx->h_wav[sd.wav_off + j];
            g[mi] += -(double)ctx->g.dt * den * sw;
        }
        for (size_t i = 0; i < nm; i++) grad_vp[i] = (float)g[i];
    }
    ctx->timing.h2d_bytes = (long long)sizeof(float) * ctx->rec_total;
    ctx->timing.d2h_bytes = grad_vp ? (long long)sizeof(float) * nm : 0;
    ctx->timing.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return SFD_OK;
}

}  // namespace

extern "C" {

int sfd_abi_version(void) { return SFD_ABI_VERSION; }

const char* sfd_status_string(int s) {
    switch (s) {
    case SFD_OK: return "ok";
    case SFD_ERR_ARG: return "invalid argument";
    case SFD_ERR_IO: return "i/o error";
    case SFD_ERR_CUDA: return "cuda error";
    case SFD_ERR_TIMEOUT: return "device wait timed out";
    case SFD_ERR_NAN: return "non-finite values detected";
    case SFD_ERR_NOMEM: return "out of memory";
    case SFD_ERR_UNSUPPORTED: return "unsupported";
    case SFD_ERR_STATE: return "invalid call order";
    default: return "unknown status";
    }
}

int sfd_last_error(const sfd_ctx* ctx, char* buf, size_t len) {
    if (!ctx || !buf || len == 0) return SFD_ERR_ARG;
    std::snprintf(buf, len, "%s", ctx->err.c_str());
    return SFD_OK;
}

int sfd_create(const sfd_grid* g, int device, sfd_ctx** out) {
    if (!g || !out) return SFD_ERR_ARG;
    *out = nullptr;
    if (g->scheme != SFD_ACOUSTIC_2D && g->scheme != SFD_VISCOAC_2D && g->scheme != SFD_ACOUSTIC_3D &&
        g->scheme != SFD_VISCOEL_2D && g->scheme != SFD_ELASTIC_2D)
        return SFD_ERR_ARG;
    const bool is3d = g->scheme == SFD_ACOUSTIC_3D;
    if (g->nx <= 0 || g->nz <= 0 || (is3d ? g->ny <= 0 : g->ny > 1)) return SFD_ERR_ARG;
    if (!(g->dx > 0) || !(g->dz > 0) || !(g->dt > 0) || (is3d && !(g->dy > 0))) return SFD_ERR_ARG;
    if (g->pml < 0 || g->pml > 256 || 2 * g->pml > g->nx || 2 * g->pml > g->nz) return SFD_ERR_ARG;
    if (is3d && 2 * g->pml > g->ny) return SFD_ERR_ARG;
    float cf[8];
    if (sfd_fd_coeffs(g->order, cf) != SFD_OK) return SFD_ERR_ARG;
    const int R = g->order / 2;
    if (g->nx <= 2 * R || g->nz <= 2 * R || (is3d && g->ny <= 2 * R)) return SFD_ERR_ARG;
    std::unique_ptr<sfd_ctx> c(new sfd_ctx());
    c->g = *g;
    if (c->g.ny <= 0) c->g.ny = 1;
    c->device = device;
    c->radius = R;
    std::memcpy(c->coef, cf, sizeof(float) * R);
    sfd_ctx* ctx = c.get();
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&c->ev0));
    CK(cudaEventCreate(&c->ev1));
    CK(cudaEventCreate(&c->evs));
    CK(cudaEventCreate(&c->eve));
    CK(cudaMalloc(&c->d_flag, sizeof(int)));
    CK(cudaMalloc(&c->d_err, sizeof(int)));
    CK(cudaMemset(c->d_err, 0, sizeof(int)));
    if (g->scheme == SFD_ACOUSTIC_2D && !acoustic2d_plan(R, &c->plan))
        return set_err(ctx, SFD_ERR_UNSUPPORTED, "no kernel for radius %d", R);
    if (g->scheme == SFD_VISCOAC_2D || g->scheme == SFD_VISCOEL_2D) {
        // the rotated staggered grid of QS is 10th order only (a100..a104, QS:9-28)
        if (g->order != 10) return set_err(ctx, SFD_ERR_UNSUPPORTED, "the Q_forward schemes are 10th order");
        if (!(g->f0 > 0)) return set_err(ctx, SFD_ERR_ARG, "the Q_forward schemes need f0 > 0 (QS:509)");
        c->plan.radius = 5;
        c->plan.tx = kTileX;
        c->plan.tz = kTileZ;
        c->plan.gz = 8;  // RSG halo 5, rounded for float4 staging
        c->plan.stages = 1;
    }
    if (g->scheme == SFD_ELASTIC_2D) {
        // the staggered grid of yang_version is 10th order only (a100..a104, YMOD:23-27)
        if (g->order != 10) return set_err(ctx, SFD_ERR_UNSUPPORTED, "the yang_version scheme is 10th order");
        if (g->pml < 1) return set_err(ctx, SFD_ERR_ARG, "the yang_version sponge needs pml >= 1 (YPRI:26-29)");
        c->plan.radius = 5;
        c->plan.tx = kTileX;
        c->plan.tz = kTileZ;
        c->plan.gz = 8;  // staggered reach 5, rounded for float4 staging
        c->plan.stages = 1;
        elastic2d_gauss_table(c->iso_rgau, &c->iso_gc, &c->iso_lo, &c->iso_hi);
    }
    if (g->scheme == SFD_ACOUSTIC_3D) {
        int b0[2], b1[2], b2[2];
        if (!acoustic3d_boxes(R, b0, b1, b2))
            return set_err(ctx, SFD_ERR_UNSUPPORTED, "the 3-D kernel is built for orders 8 and 4, not %d", g->order);
        if (g->flags & SFD_EXACT)
            return set_err(ctx, SFD_ERR_UNSUPPORTED, "SFD_EXACT applies to the reference's 2-D schemes");
    }
    *out = c.release();
    return SFD_OK;
}

int sfd_destroy(sfd_ctx* ctx) {
    delete ctx;
    return SFD_OK;
}

int sfd_set_model(sfd_ctx* ctx, const float* vp, const float* den, const float* q) {
    if (!ctx || !vp) return SFD_ERR_ARG;
    const size_t n = (size_t)ctx->g.nx * ctx->g.ny * ctx->g.nz;
    for (size_t i = 0; i < n; i++)
        if (!(vp[i] > 0.0f) || !std::isfinite(vp[i]))
            return set_err(ctx, SFD_ERR_ARG, "vp[%zu] = %g is not a positive finite velocity", i, (double)vp[i]);
    if (den)
        for (size_t i = 0; i < n; i++)
            if (!(den[i] > 0.0f) || !std::isfinite(den[i]))
                return set_err(ctx, SFD_ERR_ARG, "den[%zu] = %g is not a positive finite density", i, (double)den[i]);
    CK(cudaSetDevice(ctx->device));
    ctx->model_gen++;
    ctx->h_vp.assign(vp, vp + n);
    ctx->varden = false;
    ctx->den_c = 2400.0f;
    ctx->h_den.clear();
    if (den) {
        ctx->h_den.assign(den, den + n);
        bool uniform = true;
        for (size_t i = 1; i < n && uniform; i++) uniform = den[i] == den[0];
        if (uniform) ctx->den_c = den[0];
        else ctx->varden = true;
    }
    const int cols = ctx->g.nx * ctx->g.ny;
    const int nz = ctx->g.nz;
    const bool is3d = ctx->g.scheme == SFD_ACOUSTIC_3D;
    // 2-D: kModelGhostZ replicated rows on both sides, tiles may read past nz; 3-D: the field
    // layout of one shot ([x][y][pitch], no ghost rows)
    const int ghost = is3d ? 0 : kModelGhostZ;
    const int nzt = (nz + kTileZ - 1) / kTileZ * kTileZ;
    ctx->mpitch = is3d ? round_up(nz, 4) : round_up(2 * kModelGhostZ + nzt, 32);
    const size_t mfloats = (size_t)cols * ctx->mpitch;
    // Buffers are allocated once per context and refilled in place, so a captured time loop
    // (which bakes these pointers and the density constant in) stays valid across model updates.
    const float den_c_old = ctx->have_model ? ctx->den_c : -1.0f;
    const bool varden_old = ctx->have_model && ctx->d_den != nullptr;
    // column-wise copy with kModelGhostZ replicated rows above and replicated rows below
    auto upload = [&](float** dst, const float* src) -> int {
        std::vector<float> staged(mfloats);
        for (int c = 0; c < cols; c++) {
            const float* s = src + (size_t)c * nz;
            float* d = staged.data() + (size_t)c * ctx->mpitch;
            for (int k = 0; k < ctx->mpitch; k++) {
                const int z = std::min(std::max(k - ghost, 0), nz - 1);
                d[k] = s[z];
            }
        }
        if (!*dst) CK(cudaMalloc(dst, mfloats * sizeof(float)));
        CK(cudaMemcpy(*dst, staged.data(), mfloats * sizeof(float), cudaMemcpyHostToDevice));
        return SFD_OK;
    };
    int urc = upload(&ctx->d_vp, vp);
    if (urc) return urc;
    if (ctx->varden) {
        if ((urc = upload(&ctx->d_den, den))) return urc;
    } else {
        dfree(ctx->d_den);
    }
    if (ctx->g.scheme == SFD_ELASTIC_2D) {
        // YPUB:323-634 per shot window: staggered moduli and buoyancies, smoothed top sponge
        if (q) return set_err(ctx, SFD_ERR_ARG, "the yang_version scheme has no quality factor");
        if (!ctx->elastic_call) ctx->h_vs.clear();  // no S waves: vs = 0
        ctx->have_model = true;
        if ((urc = q_prepare(ctx))) return urc;
    }
    if (ctx->g.scheme == SFD_VISCOAC_2D || ctx->g.scheme == SFD_VISCOEL_2D) {
        // QS:434-551 on the padded grid: averaged density -> buoyancy, Lame and Blanch tau
        if (q)
            for (size_t i = 0; i < n; i++)
                if (!(q[i] > 0.0f) || !std::isfinite(q[i]))
                    return set_err(ctx, SFD_ERR_ARG, "q[%zu] = %g is not a positive finite quality factor", i,
                                   (double)q[i]);
        if (q) ctx->h_q.assign(q, q + n);
        else ctx->h_q.clear();
        if (ctx->g.scheme == SFD_VISCOEL_2D && !ctx->elastic_call) {  // no S waves: vs = 0, Qs = Qp
            ctx->h_vs.clear();
            ctx->h_qs = ctx->h_q;
        }
        ctx->have_model = true;
        if ((urc = q_prepare(ctx))) return urc;
    }
    if (ctx->varden != varden_old || (!ctx->varden && ctx->den_c != den_c_old)) {
        ctx->graph_valid = false;
        ctx->grad_valid = false;
    }
    ctx->have_model = true;
    // source scale factors depend on the model (the viscoacoustic source is a stamp)
    if (ctx->have_shots && ctx->g.scheme != SFD_VISCOAC_2D && ctx->g.scheme != SFD_VISCOEL_2D &&
        ctx->g.scheme != SFD_ELASTIC_2D) {
        for (auto& s : ctx->h_shots) {
            const size_t mi = ((size_t)(s.x0 + s.sx) * ctx->g.ny + s.sy) * ctx->g.nz + s.sz;
            const float d = ctx->varden ? ctx->h_den[mi] : ctx->den_c;
            float sc = ctx->g.dt * d;
            sc = sc * ctx->h_vp[mi];
            s.inj_scale = sc;
        }
        CK(cudaMemcpy(ctx->d_shots, ctx->h_shots.data(), sizeof(ShotDev) * ctx->nshot, cudaMemcpyHostToDevice));
    }
    return SFD_OK;
}

int sfd_set_model_elastic(sfd_ctx* ctx, const float* vp, const float* vs, const float* den, const float* qp,
                          const float* qs) {
    if (!ctx || !vp || !vs) return SFD_ERR_ARG;
    if (ctx->g.scheme != SFD_VISCOEL_2D && ctx->g.scheme != SFD_ELASTIC_2D)
        return set_err(ctx, SFD_ERR_ARG, "sfd_set_model_elastic applies to SFD_VISCOEL_2D and SFD_ELASTIC_2D");
    if (ctx->g.scheme == SFD_ELASTIC_2D && (qp || qs))
        return set_err(ctx, SFD_ERR_ARG, "the yang_version scheme has no quality factors");
    const size_t n = (size_t)ctx->g.nx * ctx->g.nz;
    for (size_t i = 0; i < n; i++)
        if (!(vs[i] >= 0.0f) || !std::isfinite(vs[i]))
            return set_err(ctx, SFD_ERR_ARG, "vs[%zu] = %g is not a finite non-negative velocity", i, (double)vs[i]);
    if (qs)
        for (size_t i = 0; i < n; i++)
            if (!(qs[i] > 0.0f) || !std::isfinite(qs[i]))
                return set_err(ctx, SFD_ERR_ARG, "qs[%zu] = %g is not a positive finite quality factor", i,
                               (double)qs[i]);
    ctx->h_vs.assign(vs, vs + n);
    if (qs) ctx->h_qs.assign(qs, qs + n);
    else ctx->h_qs.clear();
    ctx->elastic_call = true;
    const int rc = sfd_set_model(ctx, vp, den, qp);
    ctx->elastic_call = false;
    return rc;
}

int sfd_set_shots(sfd_ctx* ctx, int nshot, const sfd_shot* shots) {
    if (!ctx || nshot <= 0 || !shots) return SFD_ERR_ARG;
    if (ctx->g.scheme == SFD_ACOUSTIC_3D) return set_shots_3d(ctx, nshot, shots);
    const bool elastic = ctx->g.scheme == SFD_VISCOEL_2D;
    const bool iso = ctx->g.scheme == SFD_ELASTIC_2D;
    // the Fortran schemes: in-place split fields, Gaussian source stamps, split cosine sponge
    const bool visco = ctx->g.scheme == SFD_VISCOAC_2D || elastic || iso;
    if (ctx->g.scheme != SFD_ACOUSTIC_2D && !visco)
        return set_err(ctx, SFD_ERR_UNSUPPORTED, "scheme %d is not implemented", ctx->g.scheme);
    CK(cudaSetDevice(ctx->device));
    const int nxm = ctx->g.nx, nz = ctx->g.nz;
    std::vector<ShotDev> hs(nshot);
    std::vector<int> rx, rz;
    std::vector<float> wav;
    std::vector<long long> out_off(nshot);
    long long rec_total = 0;
    int nx_max = 0, nt_max = 0;
    for (int s = 0; s < nshot; s++) {
        const sfd_shot& sh = shots[s];
        const int nxs = sh.ap_nx > 0 ? sh.ap_nx : nxm;
        if (sh.ap_x0 < 0 || sh.ap_x0 + nxs > nxm || nxs <= 2 * ctx->radius || 2 * ctx->g.pml > nxs)
            return set_err(ctx, SFD_ERR_ARG, "shot %d: aperture [%d, %d) outside the model (nx=%d)", s, sh.ap_x0,
                           sh.ap_x0 + nxs, nxm);
        if (sh.nt < 1 || !sh.wavelet)
            return set_err(ctx, SFD_ERR_ARG, "shot %d: nt=%d or wavelet missing", s, sh.nt);
        if (sh.sx < 0 || sh.sx >= nxs || sh.sz < 0 || sh.sz >= nz)
            return set_err(ctx, SFD_ERR_ARG, "shot %d: source (%d, %d) outside the grid", s, sh.sx, sh.sz);
        if (sh.nrec < 0 || (sh.nrec > 0 && (!sh.rec_x || !sh.rec_z)))
            return set_err(ctx, SFD_ERR_ARG, "shot %d: receiver list missing", s);
        ShotDev d{};
        d.nx = nxs; d.x0 = sh.ap_x0; d.nt = sh.nt; d.sx = sh.sx; d.sy = 0; d.sz = sh.sz;
        d.nrec = sh.nrec;
        d.rec_base = rec_total;
        d.rec_list = (int)rx.size();
        d.wav_off = (int)wav.size();
        for (int r = 0; r < sh.nrec; r++) {
            if (sh.rec_x[r] < 0 || sh.rec_x[r] >= nxs || sh.rec_z[r] < 0 || sh.rec_z[r] >= nz)
                return set_err(ctx, SFD_ERR_ARG, "shot %d: receiver %d (%d, %d) outside the grid", s, r,
                               sh.rec_x[r], sh.rec_z[r]);
            rx.push_back(sh.rec_x[r]);
            rz.push_back(sh.rec_z[r]);
        }
        wav.insert(wav.end(), sh.wavelet, sh.wavelet + sh.nt);
        out_off[s] = rec_total;
        rec_total += (long long)sh.nrec * sh.nt;
        nx_max = std::max(nx_max, nxs);
        nt_max = std::max(nt_max, sh.nt);
        hs[s] = d;
    }
    free_shot_buffers(ctx);
    // layout of the state slabs
    Layout2D L{};
    L.tx = ctx->plan.tx;
    L.tz = ctx->plan.tz;
    L.gx = visco ? 8 : 2 * ctx->radius;
    L.gz = ctx->plan.gz;
    L.ntx = (nx_max + L.tx - 1) / L.tx;
    L.ntz = (nz + L.tz - 1) / L.tz;
    L.pitch = round_up(L.gz + L.ntz * L.tz + L.gz, 32);
    L.cols = L.gx + L.ntx * L.tx + L.gx;
    L.shot_stride = (long long)L.cols * L.pitch;
    ctx->L = L;
    // per-tile receiver CSR
    const int ntiles = L.ntx * L.ntz;
    std::vector<int> trp, tri;
    for (int s = 0; s < nshot; s++) {
        hs[s].tile_rec_base = (int)trp.size();
        std::vector<std::vector<int>> bucket(ntiles);
        for (int r = 0; r < hs[s].nrec; r++) {
            const int x = rx[hs[s].rec_list + r], z = rz[hs[s].rec_list + r];
            bucket[(x / L.tx) * L.ntz + z / L.tz].push_back(r);
        }
        for (int t = 0; t < ntiles; t++) {
            trp.push_back((int)tri.size());
            tri.insert(tri.end(), bucket[t].begin(), bucket[t].end());
        }
        trp.push_back((int)tri.size());
    }
    // Tile order of the FMA kernel's forward steps: CTAs are numbered tile-major (the active
    // shots' copies of one tile are consecutive) over a tile order that puts the tiles whose
    // stencil reaches neither the sponge nor a grid edge (the kernel's interior body) first and
    // the edge tiles after them, so that nearly all CTAs resident at one time run the same code
    // path.  On 64 shots of 612 x 2148 this is 3% faster than shot-major numbering in natural
    // order; either change alone gains nothing.  The adjoint steps keep shot-major natural order,
    // and SFD_TILE_MAJOR=0 in the environment selects it for the forward steps too.
    std::vector<int> torder;
    {
        const int R = ctx->radius, RQ = (R + 3) & ~3, E = std::max(ctx->g.pml, R);
        int nxs = 0;
        for (const auto& d : hs) nxs = std::max(nxs, d.nx);
        for (int pass = 0; pass < 2; pass++)
            for (int t = 0; t < ntiles; t++) {
                const int x0 = (t / L.ntz) * L.tx, z0 = (t % L.ntz) * L.tz;
                const bool inner = x0 - R >= E && x0 + L.tx + R <= nxs - E && z0 - RQ >= E && z0 + L.tz + RQ <= nz - E;
                if (inner == (pass == 0)) torder.push_back(t);
            }
        ctx->tile_major = 1;
        if (const char* env = std::getenv("SFD_TILE_MAJOR")) ctx->tile_major = std::atoi(env) != 0;
    }
    // Each CTA of the one-tile-per-CTA schedule prefetches into L2 the boxes of the CTA that
    // starts one CTA per SM later, so that its TMA loads find them in L2 rather than in HBM.  On
    // 64 shots of 612 x 2148 the forward gains 1-2%; distances of 148, 222, 296, 370 and 444
    // CTAs measured 138.8, 138.2, 137.8, 137.0 and 134.3 Gpts/s on one B200 (no prefetch: about
    // 137).  SFD_L2_AHEAD in the environment sets another distance (0: no prefetch).
    {
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            sms = 148;
        ctx->l2_ahead = sms;
        if (const char* env = std::getenv("SFD_L2_AHEAD")) ctx->l2_ahead = std::max(0, std::atoi(env));
    }
    // source scale ((dt * DEN) * Vp) in float, AFD:250
    for (auto& d : hs) {
        if (ctx->have_model) {
            const size_t mi = (size_t)(d.x0 + d.sx) * nz + d.sz;
            const float den = ctx->varden ? ctx->h_den[mi] : ctx->den_c;
            float sc = ctx->g.dt * den;
            sc = sc * ctx->h_vp[mi];
            d.inj_scale = sc;
        }
    }
    std::vector<int> order(nshot);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return hs[a].nt > hs[b].nt; });
    std::vector<int> ident(nshot);
    std::iota(ident.begin(), ident.end(), 0);

    ctx->h_shots = hs;
    ctx->h_rec_x = rx;
    ctx->h_rec_z = rz;
    ctx->h_wav = wav;
    ctx->rec_out_off = out_off;
    ctx->rec_total = rec_total;
    ctx->nshot = nshot;
    ctx->nt_max = nt_max;
    ctx->order = order;
    ctx->nrec_max = 0;
    for (const auto& d : hs) ctx->nrec_max = std::max(ctx->nrec_max, d.nrec);

    auto up = [&](auto** dst, const auto& v) -> int {
        using E = typename std::remove_reference<decltype(v)>::type::value_type;
        const size_t bytes = std::max<size_t>(1, v.size()) * sizeof(E);
        CK(cudaMalloc(dst, bytes));
        if (!v.empty()) CK(cudaMemcpy(*dst, v.data(), v.size() * sizeof(E), cudaMemcpyHostToDevice));
        return SFD_OK;
    };
    int rc;
    if ((rc = up(&ctx->d_shots, hs)) || (rc = up(&ctx->d_slot, order)) || (rc = up(&ctx->d_ident, ident)) ||
        (rc = up(&ctx->d_wav, wav)) || (rc = up(&ctx->d_rec_x, rx)) || (rc = up(&ctx->d_rec_z, rz)) ||
        (rc = up(&ctx->d_trp, trp)) || (rc = up(&ctx->d_tri, tri)) || (rc = up(&ctx->d_torder, torder)))
        return rc;
    const size_t rec_bytes = sizeof(float) * std::max<long long>(1, rec_total);
    CK(cudaMalloc(&ctx->d_rec_tn, rec_bytes));
    CK(cudaMalloc(&ctx->d_rec_nt, rec_bytes));
    if (elastic || iso) {
        CK(cudaMalloc(&ctx->d_rec2_tn, rec_bytes));
        CK(cudaMalloc(&ctx->d_rec2_nt, rec_bytes));
    }
    ctx->state_floats = (iso ? I_NFIELDS : elastic ? E_NFIELDS : q_fast(ctx) ? kQFastSlabs : visco ? 8 : 6) *
                        (size_t)nshot * L.shot_stride;
    CK(cudaMalloc(&ctx->d_state, ctx->state_floats * sizeof(float)));
    CK(cudaMalloc(&ctx->d_src_pre, sizeof(float) * nshot));
    if (visco) {
        // Gaussian source stamps (QS:1340-1444, YPUB:1429-1466) and the split cosine sponge tables
        // (QS:555-605, YPUB:796-849)
        if ((rc = build_stamps(ctx))) return rc;
        ctx->spg_stride = ctx->g.pml + 1;
        std::vector<float> tab(8 * (size_t)ctx->spg_stride);
        viscoac2d_sponge_tables(ctx->g.pml, ctx->g.pml, ctx->g.dx, ctx->g.dz, ctx->spg_stride, tab.data());
        dfree(ctx->d_spg);
        if ((rc = up(&ctx->d_spg, tab))) return rc;
        if (q_fast(ctx)) {
            int bs[2];
            viscoac2d_fast_boxes(bs);
            const long long fs = (long long)nshot * L.shot_stride;
            for (int b = 0; b < 2; b++) {
                const int rc2 = encode_field_map(ctx, &ctx->qtmaps[b], ctx->d_state + (kQS + b) * fs, L, nshot, bs);
                if (rc2) return rc2;
            }
        }
    } else {
        // TMA descriptors of the six field buffers: 3-D (z, column, shot), one box per field
        int bp[2], bvx[2], bvz[2];
        acoustic2d_fma_boxes(ctx->radius, bp, bvx, bvz);
        const int* boxes[3] = {bp, bvx, bvz};
        const long long fs = (long long)nshot * L.shot_stride;
        int mp[2], mvx[2], mvz[2];
        acoustic2d_march_boxes(mp, mvx, mvz);
        const int* mboxes[3] = {mp, mvx, mvz};
        for (int b = 0; b < 6; b++) {
            int rc2 = encode_field_map(ctx, &ctx->tmaps[b], ctx->d_state + b * fs, L, nshot, boxes[b / 2]);
            if (!rc2) rc2 = encode_field_map(ctx, &ctx->mtmaps[b], ctx->d_state + b * fs, L, nshot, mboxes[b / 2]);
            if (rc2) return rc2;
        }
    }
    ctx->h_ap_x0.resize(nshot);
    for (int s = 0; s < nshot; s++) ctx->h_ap_x0[s] = shots[s].ap_x0;
    ctx->have_shots = true;
    ctx->graph_valid = false;
    if (visco) return q_prepare(ctx);
    return SFD_OK;
}

int sfd_forward_device(sfd_ctx* ctx, float* records_dev) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    auto t0 = std::chrono::steady_clock::now();
    rc = run_forward(ctx, records_dev ? records_dev : ctx->d_rec_nt);
    ctx->timing.h2d_bytes = 0;
    ctx->timing.d2h_bytes = 0;
    ctx->timing.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

int sfd_forward(sfd_ctx* ctx, float* records) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    auto t0 = std::chrono::steady_clock::now();
    rc = run_forward(ctx, ctx->d_rec_nt);
    if (rc) return rc;
    if (records && ctx->rec_total > 0)
        CK(cudaMemcpy(records, ctx->d_rec_nt, sizeof(float) * ctx->rec_total, cudaMemcpyDeviceToHost));
    ctx->timing.h2d_bytes = 0;
    ctx->timing.d2h_bytes = records ? (long long)sizeof(float) * ctx->rec_total : 0;
    ctx->timing.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return SFD_OK;
}

int sfd_forward_per_shot(sfd_ctx* ctx, float* records) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (ctx->g.scheme == SFD_ACOUSTIC_3D && (rc = full_state_3d(ctx))) return rc;
    auto t0 = std::chrono::steady_clock::now();
    CK(cudaEventRecord(ctx->evs, ctx->stream));
    if ((rc = prologue(ctx)) != SFD_OK) return rc;
    long long launches = 0;
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    snap_prepare(ctx, &rc);
    if (rc) return rc;
    for (int s = 0; s < ctx->nshot; s++)
        for (int k = 0; k < ctx->h_shots[s].nt; k++)
            if ((rc = launch_one_step(ctx, k, ctx->d_ident + s, 1, &launches)) ||
                (rc = snap_after_step(ctx, k, ctx->d_ident + s, 1, &launches)))
                return rc;
    for (auto& sn : ctx->snaps) sn.ready = sn.count > 0;
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    if ((rc = epilogue(ctx, ctx->d_rec_nt)) != SFD_OK) return rc;
    CK(cudaEventRecord(ctx->eve, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0, dms = 0;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    CK(cudaEventElapsedTime(&dms, ctx->evs, ctx->eve));
    ctx->timing.device_ms = dms;
    if (records && ctx->rec_total > 0)
        CK(cudaMemcpy(records, ctx->d_rec_nt, sizeof(float) * ctx->rec_total, cudaMemcpyDeviceToHost));
    ctx->timing.loop_ms = ms;
    ctx->timing.launches = launches + 2;
    ctx->timing.graph = 0;
    ctx->timing.kernel_variant = kernel_variant(ctx);
    double pts = 0;
    for (const auto& s : ctx->h_shots) pts += (double)s.nx * ctx->g.ny * ctx->g.nz * s.nt;
    ctx->timing.point_updates = pts;
    ctx->timing.h2d_bytes = 0;
    ctx->timing.d2h_bytes = records ? (long long)sizeof(float) * ctx->rec_total : 0;
    ctx->timing.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return finish_nan(ctx);
}

int sfd_get_wavefield(sfd_ctx* ctx, int shot, int field, float* out) {
    if (!ctx || !out) return SFD_ERR_ARG;
    if (!ctx->have_shots || shot < 0 || shot >= ctx->nshot) return set_err(ctx, SFD_ERR_ARG, "bad shot %d", shot);
    CK(cudaSetDevice(ctx->device));
    const ShotDev& sd = ctx->h_shots[shot];
    if (ctx->g.scheme == SFD_ACOUSTIC_3D) {
        // P is stored damped, the velocities before the sponge multiply (applied here)
        const int fidx = field == SFD_FIELD_P ? 0 : field == SFD_FIELD_VX ? 2 : field == SFD_FIELD_VY ? 4
                                                                          : field == SFD_FIELD_VZ ? 6 : -1;
        if (fidx < 0) return set_err(ctx, SFD_ERR_UNSUPPORTED, "field %d not available for this scheme", field);
        const Layout3D& L = ctx->L3;
        const int buf = sd.nt & 1;
        if (ctx->state_slabs != ctx->nshot)
            return set_err(ctx, SFD_ERR_STATE, "the 3-D wavefields of the last forward were released by the gradient");
        const long long fs = (long long)ctx->nshot * L.shot_stride;
        const float* base = ctx->d_state + (fidx + buf) * fs + (long long)shot * L.shot_stride;
        const int nz = ctx->g.nz;
        CK(cudaMemcpy2D(out, sizeof(float) * nz, base, sizeof(float) * L.pitch, sizeof(float) * nz,
                        (size_t)L.nx * L.ny, cudaMemcpyDeviceToHost));
        if (fidx != 0)
            for (int x = 0; x < L.nx; x++)
                for (int y = 0; y < L.ny; y++)
                    for (int z = 0; z < nz; z++) {
                        float& v = out[((size_t)x * L.ny + y) * nz + z];
                        v = v * sponge3(ctx->g, x, y, z);
                    }
        return SFD_OK;
    }
    if (ctx->g.scheme == SFD_VISCOAC_2D) {
        // vx, vz, sigma = (sx + sz) + sr (QS strxx), r = (rx + rz) + rr (QS rxx)
        const long long fs = (long long)ctx->nshot * ctx->L.shot_stride;
        const int nz = ctx->g.nz;
        auto fetch = [&](int f, float* dst) -> int {
            const float* base = ctx->d_state + f * fs + (long long)shot * ctx->L.shot_stride +
                                (long long)ctx->L.gx * ctx->L.pitch + ctx->L.gz;
            CK(cudaMemcpy2D(dst, sizeof(float) * nz, base, sizeof(float) * ctx->L.pitch, sizeof(float) * nz, sd.nx,
                            cudaMemcpyDeviceToHost));
            return SFD_OK;
        };
        const size_t n = (size_t)sd.nx * nz;
        int rc2;
        if (q_fast(ctx)) {  // merged fields; the shot's last step wrote parity nt & 1
            const int o = sd.nt & 1;
            if (field == SFD_FIELD_VX) return fetch(kQVX + o, out);
            if (field == SFD_FIELD_VZ) return fetch(kQVZ + o, out);
            if (field == SFD_FIELD_P) return fetch(kQS + o, out);
            if (field == SFD_FIELD_R) return fetch(kQR, out);
            return set_err(ctx, SFD_ERR_UNSUPPORTED, "field %d not available for this scheme", field);
        }
        if (field == SFD_FIELD_VX) return fetch(0, out);
        if (field == SFD_FIELD_VZ) return fetch(1, out);
        if (field != SFD_FIELD_P && field != SFD_FIELD_R)
            return set_err(ctx, SFD_ERR_UNSUPPORTED, "field %d not available for this scheme", field);
        std::vector<float> a(n), b(n), c(n);
        const int f0 = field == SFD_FIELD_P ? 2 : 5;
        if ((rc2 = fetch(f0, a.data())) || (rc2 = fetch(f0 + 1, b.data())) || (rc2 = fetch(f0 + 2, c.data())))
            return rc2;
        for (size_t i = 0; i < n; i++) out[i] = (a[i] + b[i]) + c[i];
        return SFD_OK;
    }
    if (ctx->g.scheme == SFD_VISCOEL_2D || ctx->g.scheme == SFD_ELASTIC_2D) {
        // sums of the split parts in the reference's order (QS:1273-1337, YPUB:1410-1426)
        const long long fs = (long long)ctx->nshot * ctx->L.shot_stride;
        const int nz = ctx->g.nz;
        const bool iso = ctx->g.scheme == SFD_ELASTIC_2D;
        int f0;
        if (iso) switch (field) {
        case SFD_FIELD_VX: f0 = I_VXX; break;
        case SFD_FIELD_VZ: f0 = I_VZX; break;
        case SFD_FIELD_P: f0 = I_SXXX; break;
        case SFD_FIELD_SZZ: f0 = I_SZZX; break;
        case SFD_FIELD_SXZ: f0 = I_SXZX; break;
        default: return set_err(ctx, SFD_ERR_UNSUPPORTED, "field %d not available for this scheme", field);
        }
        else switch (field) {
        case SFD_FIELD_VX: f0 = E_VXX; break;
        case SFD_FIELD_VZ: f0 = E_VZX; break;
        case SFD_FIELD_P: f0 = E_SXXX; break;
        case SFD_FIELD_SZZ: f0 = E_SZZX; break;
        case SFD_FIELD_SXZ: f0 = E_SXZX; break;
        case SFD_FIELD_R: f0 = E_RXXX; break;
        default: return set_err(ctx, SFD_ERR_UNSUPPORTED, "field %d not available for this scheme", field);
        }
        const int np = (iso || f0 < E_SXXX) ? 2 : 3;
        const size_t n = (size_t)sd.nx * nz;
        std::vector<float> part(n);
        for (int i = 0; i < np; i++) {
            const float* base = ctx->d_state + (f0 + i) * fs + (long long)shot * ctx->L.shot_stride +
                                (long long)ctx->L.gx * ctx->L.pitch + ctx->L.gz;
            CK(cudaMemcpy2D(i == 0 ? out : part.data(), sizeof(float) * nz, base, sizeof(float) * ctx->L.pitch,
                            sizeof(float) * nz, sd.nx, cudaMemcpyDeviceToHost));
            if (i > 0)
                for (size_t j = 0; j < n; j++) out[j] = out[j] + part[j];
        }
        return SFD_OK;
    }
    if (field != SFD_FIELD_P && field != SFD_FIELD_VX && field != SFD_FIELD_VZ)
        return set_err(ctx, SFD_ERR_UNSUPPORTED, "field %d not available for this scheme", field);
    const int buf = sd.nt & 1;  // state after nt steps lives in buffer nt % 2
    const long long fs = (long long)ctx->nshot * ctx->L.shot_stride;
    const int fidx = field == SFD_FIELD_P ? 0 : (field == SFD_FIELD_VX ? 2 : 4);
    const float* base = ctx->d_state + (fidx + buf) * fs + (long long)shot * ctx->L.shot_stride +
                        (long long)ctx->L.gx * ctx->L.pitch + ctx->L.gz;
    const int nz = ctx->g.nz;
    CK(cudaMemcpy2D(out, sizeof(float) * nz, base, sizeof(float) * ctx->L.pitch, sizeof(float) * nz, sd.nx,
                    cudaMemcpyDeviceToHost));
    if (field != SFD_FIELD_P) {
        // velocities are stored before the sponge multiply; return them as AFD holds them
        std::vector<float> a((size_t)sd.nx * nz);
        sfd_afd_sponge(sd.nx, nz, ctx->g.pml, a.data());
        for (size_t i = 0; i < a.size(); i++) out[i] = out[i] * a[i];
    }
    return SFD_OK;
}

int sfd_set_gauss_radius(sfd_ctx* ctx, int rgau) {
    if (!ctx || rgau < 1 || rgau > 4096) return SFD_ERR_ARG;
    if (ctx->g.scheme != SFD_ELASTIC_2D)
        return set_err(ctx, SFD_ERR_ARG, "the Gaussian radius applies to SFD_ELASTIC_2D");
    if (rgau == ctx->iso_rgau) return SFD_OK;
    CK(cudaSetDevice(ctx->device));
    ctx->iso_rgau = rgau;
    elastic2d_gauss_table(rgau, &ctx->iso_gc, &ctx->iso_lo, &ctx->iso_hi);
    int rc;
    if (ctx->have_shots && (rc = build_stamps(ctx))) return rc;
    return q_prepare(ctx);  // the top sponge's smoothing (no-op without a model)
}

int sfd_set_free_surface(sfd_ctx* ctx, int top) {
    if (!ctx || top < 0) return SFD_ERR_ARG;
    if (ctx->g.scheme != SFD_ELASTIC_2D)
        return set_err(ctx, SFD_ERR_ARG, "the free surface applies to SFD_ELASTIC_2D");
    if (top >= ctx->g.nz - ctx->g.pml - 5)
        return set_err(ctx, SFD_ERR_ARG, "free-surface row %d too deep for nz = %d", top, ctx->g.nz);
    if (top == ctx->iso_top) return SFD_OK;
    CK(cudaSetDevice(ctx->device));
    ctx->iso_top = top;
    ctx->graph_valid = false;
    for (auto& sn : ctx->snaps) sn.ready = false;  // the snapshot interior starts at the new top
    return q_prepare(ctx);  // substagger's refill row and the smoothing follow the mode
}

int sfd_set_topography(sfd_ctx* ctx, const int* itopo) {
    if (!ctx) return SFD_ERR_ARG;
    if (ctx->g.scheme != SFD_ELASTIC_2D) return set_err(ctx, SFD_ERR_ARG, "topography applies to SFD_ELASTIC_2D");
    if (itopo) {
        for (int x = 0; x < ctx->g.nx; x++)
            if (itopo[x] < 1 || itopo[x] > ctx->g.nz - ctx->g.pml - 6)
                return set_err(ctx, SFD_ERR_ARG, "itopo[%d] = %d outside [1, %d]", x, itopo[x],
                               ctx->g.nz - ctx->g.pml - 6);
        ctx->h_itopo.assign(itopo, itopo + ctx->g.nx);
    } else {
        ctx->h_itopo.clear();
    }
    CK(cudaSetDevice(ctx->device));
    ctx->topo_gen++;
    ctx->graph_valid = false;
    return q_prepare(ctx);  // the refill rows, the smoothing rows and the kernels follow the surface
}

int sfd_set_memory_limit(sfd_ctx* ctx, long long bytes) {
    if (!ctx || bytes < 0) return SFD_ERR_ARG;
    ctx->mem_limit = (size_t)bytes;
    return SFD_OK;
}

int sfd_set_checkpoint_interval(sfd_ctx* ctx, int steps) {
    if (!ctx || steps < 0) return SFD_ERR_ARG;
    ctx->ckpt_interval = steps;
    return SFD_OK;
}

int sfd_test_wait_timeout(sfd_ctx* ctx, int cta, int step, double limit_s) {
    if (!ctx || (cta >= 0 && (step < 0 || !(limit_s > 0.0) || limit_s > 10.0))) return SFD_ERR_ARG;
    ctx->test_cta = cta < 0 ? -1 : cta;
    ctx->test_step = step;
    ctx->test_wait_ns = cta < 0 ? 0ull : (unsigned long long)(limit_s * 1e9);
    ctx->graph_valid = false;  // the captured loop holds the step arguments
    ctx->grad_valid = false;
    return SFD_OK;
}

int sfd_gradient(sfd_ctx* ctx, const float* obs, float* misfit, float* grad_vp, float* grad_invq) {
    return run_gradient(ctx, obs, misfit, grad_vp, grad_invq, true);
}

int sfd_gradient_device(sfd_ctx* ctx, const float* obs_dev, float* misfit_dev, float* grad_vp_dev,
                        float* grad_invq_dev) {
    return run_gradient(ctx, obs_dev, misfit_dev, grad_vp_dev, grad_invq_dev, true, true);
}

int sfd_gradient_per_shot(sfd_ctx* ctx, const float* obs, float* misfit, float* grad_vp, float* grad_invq) {
    return run_gradient(ctx, obs, misfit, grad_vp, grad_invq, false);
}

int sfd_get_wavelet_gradient(sfd_ctx* ctx, int shot, float* out) {
    if (!ctx || !out) return SFD_ERR_ARG;
    if (!ctx->have_grad) return set_err(ctx, SFD_ERR_STATE, "sfd_gradient has not been called");
    if (shot < 0 || shot >= ctx->nshot) return set_err(ctx, SFD_ERR_ARG, "bad shot %d", shot);
    const ShotDev& sd = ctx->h_shots[shot];
    CK(cudaMemcpy(out, ctx->d_lam + (size_t)shot * ctx->nt_max, sizeof(float) * sd.nt, cudaMemcpyDeviceToHost));
    // acoustic: d misfit / d w[j] = -s lambda_j[src]; viscoacoustic: the kernels store the
    // stamp-weighted sum itself
    if (ctx->g.scheme != SFD_VISCOAC_2D)
        for (int j = 0; j < sd.nt; j++) out[j] = -sd.inj_scale * out[j];
    return SFD_OK;
}

int sfd_set_snapshots(sfd_ctx* ctx, int id, int field, int first, int every, int count) {
    if (!ctx || id < 0 || id >= 4 || count < 0 || first < 0 || (count > 0 && every < 1)) return SFD_ERR_ARG;
    if (ctx->g.scheme == SFD_ACOUSTIC_3D && count > 0)
        return set_err(ctx, SFD_ERR_UNSUPPORTED, "snapshots are taken for the 2-D schemes");
    const bool visco = ctx->g.scheme == SFD_VISCOAC_2D || ctx->g.scheme == SFD_VISCOEL_2D;
    const bool elastic = ctx->g.scheme == SFD_VISCOEL_2D || ctx->g.scheme == SFD_ELASTIC_2D;
    if (count > 0 && field != SFD_FIELD_P && field != SFD_FIELD_VX && field != SFD_FIELD_VZ &&
        !(visco && field == SFD_FIELD_R) && !(elastic && (field == SFD_FIELD_SZZ || field == SFD_FIELD_SXZ)))
        return set_err(ctx, SFD_ERR_ARG, "field %d cannot be recorded for this scheme", field);
    auto& sn = ctx->snaps[id];
    sn.field = field;
    sn.first = first;
    sn.every = every < 1 ? 1 : every;
    sn.count = count;
    sn.ready = false;
    ctx->graph_valid = false;
    return SFD_OK;
}

int sfd_get_records(sfd_ctx* ctx, int field, float* records) {
    if (!ctx || !records) return SFD_ERR_ARG;
    if (!ctx->have_shots) return set_err(ctx, SFD_ERR_STATE, "no shots");
    const bool q = ctx->g.scheme == SFD_VISCOAC_2D || ctx->g.scheme == SFD_VISCOEL_2D;
    const bool iso = ctx->g.scheme == SFD_ELASTIC_2D;
    if (!(q && (field == SFD_FIELD_SZZ || field == SFD_FIELD_P)) && !(iso && (field == SFD_FIELD_VX || field == SFD_FIELD_VZ)))
        return set_err(ctx, SFD_ERR_UNSUPPORTED, "records of field %d are not recorded for this scheme", field);
    CK(cudaSetDevice(ctx->device));
    // the time-major records of the last forward, transposed to the output layout: record1
    // (strzz; vx for the yang_version scheme) or record2 (strxx, which only the visco-elastic
    // scheme keeps apart -- for vs = 0 both are sigma; vz for the yang_version scheme)
    const bool sxx = (field == SFD_FIELD_P && ctx->g.scheme == SFD_VISCOEL_2D) || (iso && field == SFD_FIELD_VZ);
    if (sxx && !ctx->rec2_ready) return set_err(ctx, SFD_ERR_STATE, "no forward has run");
    float* tn = sxx ? ctx->d_rec2_tn : ctx->d_rec_tn;
    float* nt = sxx ? ctx->d_rec2_nt : ctx->d_rec_nt;
    CK(launch_records_transpose(tn, nt, ctx->d_shots, ctx->nshot, ctx->nrec_max, ctx->nt_max, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->rec_total > 0) CK(cudaMemcpy(records, nt, sizeof(float) * ctx->rec_total, cudaMemcpyDeviceToHost));
    return SFD_OK;
}

int sfd_get_snapshots(sfd_ctx* ctx, int id, int shot, float* out, int* n_out) {
    if (!ctx || id < 0 || id >= 4) return SFD_ERR_ARG;
    const auto& sn = ctx->snaps[id];
    if (!sn.ready) return set_err(ctx, SFD_ERR_STATE, "snapshot stream %d has not been filled by a forward", id);
    if (shot < 0 || shot >= ctx->nshot) return set_err(ctx, SFD_ERR_ARG, "bad shot %d", shot);
    if (n_out) *n_out = sn.taken[shot];
    if (out && sn.taken[shot] > 0) {
        CK(cudaSetDevice(ctx->device));
        const long long n = (long long)sn.taken[shot] * (ctx->h_shots[shot].nx - 2 * ctx->g.pml) *
                            (ctx->g.nz - snap_top(ctx) - ctx->g.pml);
        CK(cudaMemcpy(out, sn.d_buf + sn.off[shot], sizeof(float) * n, cudaMemcpyDeviceToHost));
    }
    return SFD_OK;
}

int sfd_get_timing(const sfd_ctx* ctx, sfd_timing* out) {
    if (!ctx || !out) return SFD_ERR_ARG;
    *out = ctx->timing;
    return SFD_OK;
}

}  // extern "C"
