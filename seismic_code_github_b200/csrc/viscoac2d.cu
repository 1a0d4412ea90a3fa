// Viscoacoustic (one standard-linear-solid memory variable) rotated-staggered-grid time step,
// the vs = 0 reduction of forward/Q_forward/Q_multishot_fd_subroutine_fsbc_zy_rotated.f90 (QS).
//
// With mu = 0, strxz and rxz stay exactly zero, so vxz = vzx = 0 and strxx = strzz (their
// split parts receive identical updates, sponges and sources).  The state per cell is
//   vx, vz                (QS vxx, vzz; vx is sponged in x only, vz in z only)
//   sx, sz, sr            (QS strxxx, strxxz, strxxr; sigma = (sx + sz) + sr)
//   rx, rz, rr            (QS rxxx, rxxz, rxxr;       r     = (rx + rz) + rr)
// and one step is two kernels:
//   velocity: d1 = Dx0(sigma), d2 = Dz0(sigma) (QS:843-966, xflag/zflag 0),
//             vx = (vx + dt b d1) * x-sponge, vz = (vz + dt b d2) * z-sponge   (QS:969-990, 609-654)
//   stress:   d1 = Dx1(vx), d4 = Dz1(vz) (flag 1),
//             sx = (sx + dt (p1 d1)) * x-sponge' + source, sz = (sz + dt (p1 d4)) * z-sponge',
//             sr = sr + dt r_old, rx = (rx + f (p2 d1)) * x-sponge', rz = (rz + f (p2 d4)) * z-sponge',
//             rr = rr + f r_old, f = dt (-1/tau_sigma)                       (QS:993-1337, 1340-1390)
// Every multiply and add is rounded separately in the reference's order, so the kernels agree
// bit for bit with the FP32 restatement in oracle/q_oracle.cpp.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "sfd_internal.h"

namespace sfd {
namespace {

constexpr int kThreads = 256;
constexpr int TX = kTileX, TZ = kTileZ;
constexpr int H = 5;                    // RSG halo (offsets -5..+5)
constexpr int HZ = 8;                   // z halo rounded for float4 staging
constexpr int SROWS = TX + 2 * H;       // 74
constexpr int SW = TZ + 2 * HZ;         // 80
constexpr int SMEM = SROWS * SW;        // floats per staged field
constexpr int kPer = TX * TZ / kThreads;  // cells per thread
constexpr int kNB = 4;    // cells per load batch
constexpr int kNBS = 2;  // cells per load batch of the stress kernel (three CTAs per SM)
static_assert(kPer % kNB == 0, "whole batches");

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }

// QS:843-966: 0.5/d * sum_m a_m t_m with t_m the rotated four-point difference
template <bool XDIR, int FLAG>
__device__ __forceinline__ float rsg(const float* s, int r, int c, const float* a, float h) {
    // s(row = x, col = z) with (r, c) the staged position of the output point
    auto u = [&](int dk, int di) { return s[(r + di) * SW + c + dk]; };
    float acc = 0.0f;
#pragma unroll
    for (int m = 0; m < 5; m++) {
        float t;
        if (FLAG == 0) {
            t = XDIR ? fs(fa(fs(u(m, m), u(-1 - m, -1 - m)), u(-1 - m, m)), u(m, -1 - m))
                     : fa(fs(fs(u(m, m), u(-1 - m, -1 - m)), u(-1 - m, m)), u(m, -1 - m));
        } else {
            t = XDIR ? fs(fa(fs(u(1 + m, 1 + m), u(-m, -m)), u(-m, 1 + m)), u(1 + m, -m))
                     : fa(fs(fs(u(1 + m, 1 + m), u(-m, -m)), u(-m, 1 + m)), u(1 + m, -m));
        }
        acc = (m == 0) ? fm(a[0], t) : fa(acc, fm(a[m], t));
    }
    return fm(h, acc);
}

struct TileRef {
    int shot, tile, x0, z0;
    ShotDev sd;
};

__device__ __forceinline__ bool tile_of(const QArgs& a, TileRef& t) {
    t.shot = a.slot_to_shot[blockIdx.y];
    t.sd = a.shots[t.shot];
    t.tile = blockIdx.x;
    const int tx_i = t.tile / a.L.ntz, tz_i = t.tile - tx_i * a.L.ntz;
    t.x0 = tx_i * TX;
    t.z0 = tz_i * TZ;
    return t.x0 < t.sd.nx;
}

__device__ __forceinline__ long long cell(const QArgs& a, int shot, int x, int z) {
    return (long long)shot * a.L.shot_stride + (long long)(x + a.L.gx) * a.L.pitch + a.L.gz + z;
}

// stage f0 (+ f1 + f2, summed in that order) on the tile plus halo
template <int NF>
__device__ __forceinline__ void stage(float* s, const QArgs& a, const TileRef& t, const float* f0, const float* f1,
                                      const float* f2) {
    constexpr int W4 = SW / 4;
#pragma unroll 3  // several rows' loads in flight before their shared-memory stores
    for (int i = threadIdx.x; i < SROWS * W4; i += kThreads) {
        const int r = i / W4, c = i - r * W4;
        const long long off = cell(a, t.shot, t.x0 - H + r, t.z0 - HZ + 4 * c);
        float4 v = __ldg(reinterpret_cast<const float4*>(f0 + off));
        if (NF == 3) {
            const float4 b = __ldg(reinterpret_cast<const float4*>(f1 + off));
            const float4 d = __ldg(reinterpret_cast<const float4*>(f2 + off));
            v = make_float4(fa(fa(v.x, b.x), d.x), fa(fa(v.y, b.y), d.y), fa(fa(v.z, b.z), d.z), fa(fa(v.w, b.w), d.w));
        }
        *reinterpret_cast<float4*>(s + r * SW + 4 * c) = v;
    }
}

// x / z factors of a split sponge: left/right (resp. top/bottom) tables, applied in QS order
__device__ __forceinline__ float xs(float u, int x, int nx, int np, const float* tn, const float* tp) {
    if (x <= np) u = fm(u, tn[x]);
    if (x >= nx - np - 1) u = fm(u, tp[nx - 1 - x]);
    return u;
}

__global__ void __launch_bounds__(kThreads) q_velocity_kernel(const __grid_constant__ QArgs a) {
    __shared__ __align__(16) float sS[SMEM];
    TileRef t;
    if (!tile_of(a, t)) return;
    stage<3>(sS, a, t, a.sx, a.sz, a.sr);  // sigma = (sx + sz) + sr  (QS:1294-1314)
    __syncthreads();
    const int nx = t.sd.nx, nz = a.nz;
    const float* tb = a.spg;
    const int st = a.spg_stride;
    // NB cells per batch: all global loads of a batch are issued before its arithmetic, so that
    // their latencies overlap (thread t handles column z = t % TZ of rows t / TZ + 4 j)
    for (int j0 = 0; j0 < kPer; j0 += kNB) {
        float vxo[kNB], vzo[kNB], bu[kNB];
        long long cc[kNB];
        bool ok[kNB];
#pragma unroll
        for (int u = 0; u < kNB; u++) {
            const int i = threadIdx.x + (j0 + u) * kThreads, r = i / TZ, z = i - r * TZ;
            const int gx = t.x0 + r, gz = t.z0 + z;
            ok[u] = gx < nx && gz < nz;
            cc[u] = cell(a, t.shot, gx, gz);
            if (ok[u]) {
                vxo[u] = a.vx[cc[u]];
                vzo[u] = a.vz[cc[u]];
                bu[u] = __ldg(a.busg + (long long)min(t.sd.x0 + gx, a.nx_model - 1) * a.mpitch + gz);
            }
        }
#pragma unroll
        for (int u = 0; u < kNB; u++) {
            if (!ok[u]) continue;
            const int i = threadIdx.x + (j0 + u) * kThreads, r = i / TZ, z = i - r * TZ;
            const int gx = t.x0 + r, gz = t.z0 + z;
            const float d1 = rsg<true, 0>(sS, r + H, z + HZ, a.a, a.hx);
            const float d2 = rsg<false, 0>(sS, r + H, z + HZ, a.a, a.hz);
            const float dtb = fm(a.dt, bu[u]);
            float vx = fa(vxo[u], fm(dtb, d1));
            float vz = fa(vzo[u], fm(dtb, d2));
            vx = xs(vx, gx, nx, a.npx, tb + 0 * st, tb + 1 * st);   // spgxn, spgxp
            vz = xs(vz, gz, nz, a.npz, tb + 2 * st, tb + 3 * st);   // spgzn, spgzp
            a.vx[cc[u]] = fa(vx, 0.0f);  // vx = vxx + vxz with vxz = 0
            a.vz[cc[u]] = fa(0.0f, vz);  // vz = vzx + vzz with vzx = 0
        }
    }
}

__global__ void __launch_bounds__(kThreads, 3) q_stress_kernel(const __grid_constant__ QArgs a) {
    __shared__ __align__(16) float sVx[SMEM];
    __shared__ __align__(16) float sVz[SMEM];
    TileRef t;
    if (!tile_of(a, t)) return;
    stage<1>(sVx, a, t, a.vx, nullptr, nullptr);
    stage<1>(sVz, a, t, a.vz, nullptr, nullptr);
    __syncthreads();
    const int nx = t.sd.nx, nz = a.nz;
    const float* tb = a.spg;
    const int st = a.spg_stride;
    const int step = a.step;
    const float wav = __ldg(a.wavelets + t.sd.wav_off + step);
    const ShotDev& sd = t.sd;
    for (int j0 = 0; j0 < kPer; j0 += kNBS) {
        float p1[kNBS], p2[kNBS], sx0[kNBS], sz0[kNBS], sr0[kNBS], rx0[kNBS], rz0[kNBS], rr0[kNBS];
        long long cc[kNBS];
        bool ok[kNBS];
#pragma unroll
        for (int u = 0; u < kNBS; u++) {
            const int i = threadIdx.x + (j0 + u) * kThreads, r = i / TZ, z = i - r * TZ;
            const int gx = t.x0 + r, gz = t.z0 + z;
            ok[u] = gx < nx && gz < nz;
            cc[u] = cell(a, t.shot, gx, gz);
            if (ok[u]) {
                const long long mi = (long long)min(sd.x0 + gx, a.nx_model - 1) * a.mpitch + gz;
                p1[u] = __ldg(a.p1 + mi);
                p2[u] = __ldg(a.p2 + mi);
                const long long c = cc[u];
                sx0[u] = a.sx[c]; sz0[u] = a.sz[c]; sr0[u] = a.sr[c];
                rx0[u] = a.rx[c]; rz0[u] = a.rz[c]; rr0[u] = a.rr[c];
            }
        }
#pragma unroll
        for (int u = 0; u < kNBS; u++) {
            if (!ok[u]) continue;
            const int i = threadIdx.x + (j0 + u) * kThreads, r = i / TZ, z = i - r * TZ;
            const int gx = t.x0 + r, gz = t.z0 + z;
            const long long c = cc[u];
            const float d1 = rsg<true, 1>(sVx, r + H, z + HZ, a.a, a.hx);
            const float d4 = rsg<false, 1>(sVz, r + H, z + HZ, a.a, a.hz);
            const float rold = fa(fa(rx0[u], rz0[u]), rr0[u]);  // QS rxx of the previous step
            // calpstrxx (QS:993-1020) with mu = 0, split sponge (QS:800), source (QS:801)
            float sx = fa(sx0[u], fm(a.dt, fm(p1[u], d1)));
            float sz = fa(sz0[u], fm(a.dt, fm(p1[u], d4)));
            const float sr = fa(sr0[u], fm(a.dt, rold));
            sx = xs(sx, gx, nx, a.npx, tb + 4 * st, tb + 5 * st);   // spg1xn, spg2xp
            sz = xs(sz, gz, nz, a.npz, tb + 6 * st, tb + 7 * st);   // spg1zn, spg2zp
            const int bx = gx - sd.stamp_x0, bz = gz - sd.stamp_z0;
            if (bx >= 0 && bx < sd.stamp_w && bz >= 0 && bz < sd.stamp_h) {
                const float g = __ldg(a.stamps + sd.stamp_off + bx * sd.stamp_h + bz);
                sx = fa(__fdiv_rn(fm(fm(wav, g), a.dt), a.dz2), sx);   // QS:1384
            }
            // calprxx (QS:1135-1170)
            float rx = fa(rx0[u], fm(a.f_mem, fm(p2[u], d1)));
            float rz = fa(rz0[u], fm(a.f_mem, fm(p2[u], d4)));
            const float rr = fa(rr0[u], fm(a.f_mem, rold));
            rx = xs(rx, gx, nx, a.npx, tb + 4 * st, tb + 5 * st);
            rz = xs(rz, gz, nz, a.npz, tb + 6 * st, tb + 7 * st);
            a.sx[c] = sx; a.sz[c] = sz; a.sr[c] = sr;
            a.rx[c] = rx; a.rz[c] = rz; a.rr[c] = rr;
            if (a.d1_out) {  // gradient recomputation keeps the derivatives for the imaging condition
                a.d1_out[c] = d1;
                a.d4_out[c] = d4;
            }
        }
    }
    // receivers: strzz (= strxx) = (sx + sz) + sr (QM:452-459)
    const int* trp = a.tile_rec_ptr + sd.tile_rec_base + t.tile;
    const int rb = trp[0], re = trp[1];
    if (re > rb) {
        __syncthreads();
        for (int j = rb + threadIdx.x; j < re; j += kThreads) {
            const int ridx = a.tile_rec_idx[j];
            const long long c = cell(a, t.shot, a.rec_x[sd.rec_list + ridx], a.rec_z[sd.rec_list + ridx]);
            a.records[sd.rec_base + (long long)step * sd.nrec + ridx] = fa(fa(a.sx[c], a.sz[c]), a.sr[c]);
        }
    }
}

}  // namespace

cudaError_t viscoac2d_launch_step(const QArgs& a, int active, cudaStream_t st) {
    dim3 grid(a.L.ntx * a.L.ntz, active);
    q_velocity_kernel<<<grid, kThreads, 0, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    q_stress_kernel<<<grid, kThreads, 0, st>>>(a);
    return cudaGetLastError();
}

// QS:434-469 (density averaged in place, then buoyancy) and QS:473-551 (Blanch's tau method),
// single precision in the reference's operation order.  q == nullptr: Q = 1e5 (QM:418-419).
void viscoac2d_prepare(int nx, int nz, const float* vp, const float* rho, const float* q, float f0, float* busg,
                       float* p1, float* p2, float* rtau_out) {
    std::vector<float> r(rho, rho + (size_t)nx * nz);
    auto R = [&](int k, int i) -> float& { return r[(size_t)i * nz + k]; };  // 0-based (z, x)
    for (int i = 0; i < nx - 1; i++)
        for (int k = 0; k < nz - 1; k++) R(k, i) = 0.25f * (R(k, i) + R(k + 1, i) + R(k + 1, i + 1) + R(k, i + 1));
    for (int i = 0; i < nx; i++) R(nz - 1, i) = R(nz - 2, i);
    for (int k = 0; k < nz; k++) R(k, nx - 1) = R(k, nx - 2);
    const float pi = 3.1415926f;
    const float flow = 2.0f * 2.0f * pi;
    const float fup = 2.5f * f0 * 2.0f * pi;
    const float tss = 1.0f / ((fup - flow) / 2.0f);
    const float nlow = std::log((tss * tss) * (flow * flow) + 1.0f);
    const float nup = std::log((tss * tss) * (fup * fup) + 1.0f);
    const float dlow = std::atan(flow * tss) - (flow * tss) / (1.0f + (tss * tss) * (flow * flow));
    const float dup = std::atan(fup * tss) - (fup * tss) / (1.0f + (tss * tss) * (fup * fup));
    for (size_t c = 0; c < (size_t)nx * nz; c++) {
        const float rr = r[c];
        busg[c] = 1.0f / rr;
        const float lambmu = rr * (vp[c] * vp[c]);
        const float qp = (q ? q[c] : 100000.0f) * (18.0f / 20.0f);
        float taup = 0.0f;
        if (dup - dlow != 0.0f) taup = 1.0f / qp * (nup - nlow) / (dup - dlow);
        const float tpe = taup * tss + tss;
        const float tpss = tpe / tss;
        p1[c] = lambmu * tpss;
        p2[c] = lambmu * (tpss - 1.0f);
    }
    *rtau_out = 1.0f / tss;
}

// QS:555-605 with R = 1e-3; tables xn, xp, zn, zp, 1xn, 2xp, 1zn, 2zp of `stride` entries
void viscoac2d_sponge_tables(int npx, int npz, float dx, float dz, int stride, float* out) {
    const float Rr = 1.0e-3f;
    const float fx = std::acos(Rr) / ((float)npx * dx), fz = std::acos(Rr) / ((float)npz * dz);
    for (int j = 0; j < 8 * stride; j++) out[j] = 1.0f;
    for (int i = 1; i <= npx + 1; i++) {
        out[0 * stride + i - 1] = std::cos(fx * (float)(npx - i + 1) * dx);
        out[1 * stride + i - 1] = std::cos(fx * (float)(npx - i + 1) * dx);
        out[4 * stride + i - 1] = (i == npx + 1) ? 1.0f : std::cos(fx * ((float)(npx - i + 1) * dx - dx / 2));
        out[5 * stride + i - 1] = std::cos(fx * ((float)(npx - i + 1) * dx + dx / 2));
    }
    for (int i = 1; i <= npz + 1; i++) {
        out[2 * stride + i - 1] = std::cos(fz * (float)(npz - i + 1) * dz);
        out[3 * stride + i - 1] = std::cos(fz * (float)(npz - i + 1) * dz);
        out[6 * stride + i - 1] = (i == npz + 1) ? 1.0f : std::cos(fz * ((float)(npz - i + 1) * dz - dz / 2));
        out[7 * stride + i - 1] = std::cos(fz * ((float)(npz - i + 1) * dz + dz / 2));
    }
}

// QS:1340-1444: the whole-grid Gaussian (sigma 1.5 cells) normalised by its single-precision
// sum, placed as the loop of QS:1378-1390 places it (centre offset by one cell for even sizes);
// the box of non-zero weights around the source.
void viscoac2d_stamp(int nx, int nz, int sx, int sz, int* box, std::vector<float>* out) {
    const int n1 = nz, n2 = nx;
    const int hw1 = (int)std::lround((n1 + 1) / 2.0), hw2 = (int)std::lround((n2 + 1) / 2.0);
    const int ixcen = (n1 + 1) / 2, izcen = (n2 + 1) / 2;
    const float pi = 3.1415926f, sigma2 = 1.5f * 1.5f;
    auto raw = [&](int i, int j) {  // g2c(i, j) before normalisation, 1-based
        const float dis = (float)((j - izcen) * (j - izcen) + (i - ixcen) * (i - ixcen));
        return 1.0f / (2.0f * pi * sigma2) * std::exp(-dis / (2.0f * sigma2));
    };
    float sum = 0.0f;
    for (int j = 1; j <= n2; j++)
        for (int i = 1; i <= n1; i++) sum = sum + raw(i, j);
    // 1-based source (isxe, isze) = (sx + 1, sz + 1); loop indices idx1 = m - (isze - hw1), idx2 likewise
    const int isxe = sx + 1, isze = sz + 1;
    int xlo = 1 << 30, xhi = -1, zlo = 1 << 30, zhi = -1;
    for (int n = isxe - (hw2 - 1); n <= isxe + (hw2 - 1); n++) {
        const int idx2 = n - (isxe - (hw2 - 1)) + 1;
        if (n < 1 || n > nx || idx2 > n2) continue;
        for (int m = isze - (hw1 - 1); m <= isze + (hw1 - 1); m++) {
            const int idx1 = m - (isze - (hw1 - 1)) + 1;
            if (m < 1 || m > nz || idx1 > n1) continue;
            if (raw(idx1, idx2) / sum != 0.0f) {
                xlo = std::min(xlo, n - 1); xhi = std::max(xhi, n - 1);
                zlo = std::min(zlo, m - 1); zhi = std::max(zhi, m - 1);
            }
        }
    }
    if (xhi < 0) {
        box[0] = box[1] = 0;
        box[2] = box[3] = 0;
        return;
    }
    box[0] = xlo; box[1] = zlo; box[2] = xhi - xlo + 1; box[3] = zhi - zlo + 1;
    for (int x = xlo; x <= xhi; x++)
        for (int z = zlo; z <= zhi; z++) {
            const int idx2 = (x + 1) - (isxe - (hw2 - 1)) + 1, idx1 = (z + 1) - (isze - (hw1 - 1)) + 1;
            out->push_back(raw(idx1, idx2) / sum);
        }
}

}  // namespace sfd
