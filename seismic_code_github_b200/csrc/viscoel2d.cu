// Visco-elastic (P-SV, one standard-linear-solid memory variable per stress) rotated-staggered-
// grid time step: the full scheme of forward/Q_forward/Q_multishot_fd_subroutine_fsbc_zy_rotated.f90
// (QS:695-1337) with vs > 0, flat surface.  Every field is kept in the reference's split form
// (x, z and memory parts), 22 per cell:
//   vxx vxz vzx vzz | sxxx sxxz sxxr | szzx szzz szzr | sxzx sxzz sxzr | rxxx rxxz rxxr |
//   rzzx rzzz rzzr | rxzx rxzz rxzr
// and one step is two kernels:
//   velocity: sxx, sxz, szz = sums of their parts (QS:1294-1337) on the tile plus halo;
//             vxx += dt b Dx0 sxx, vxz += dt b Dz0 sxz, vzx += dt b Dx0 sxz, vzz += dt b Dz0 szz,
//             x parts times the x sponge, z parts times the z sponge        (QS:713-748, 969-990)
//   stress:   vx = vxx + vxz, vz = vzx + vzz on the tile plus halo; d1 = Dx1 vx, d2 = Dx1 vz,
//             d3 = Dz1 vx, d4 = Dz1 vz; with r.. the memory sums of the previous step,
//             sxxx += dt (q1 d1), sxxz += dt (q2 d4), sxxr += dt rxx          (calpstrxx)
//             szzx += dt (q2 d1), szzz += dt (q1 d4), szzr += dt rzz          (calpstrzz)
//             sxzx += dt (q3 d2), sxzz += dt (q3 d3), sxzr += dt rxz          (calpstrxz)
//             rxxx += f (m1 d1), rxxz += f (m2 d4), rxxr += f rxx            (calprxx)
//             rzzz += f (m1 d4), rzzx += f (m2 d1), rzzr += f rzz            (calprzz)
//             rxzx += f (m3 d2), rxzz += f (m3 d3), rxzr += f rxz            (calprxz)
//             x parts times the x' sponge, z parts times the z' sponge, the source added to
//             sxxx and szzx after their sponge (QS:801, 1340-1390)
//   with q1 = lambda tau_p, q2 = lambda tau_p - 2 mu tau_s, q3 = mu tau_s, m1 = lambda (tau_p - 1),
//   m2 = lambda (tau_p - 1) - 2 mu (tau_s - 1), m3 = mu (tau_s - 1), f = dt (-1 / tau_sigma)
//   (QS:473-551), rounded in the reference's order.  Records: strzz (record1) and strxx (record2)
//   at the receivers after the step (QM:452-459).
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
constexpr int H = 5;                  // rotated-staggered reach
constexpr int HZ = 8;                 // z halo rounded for float4 staging
constexpr int SROWS = TX + 2 * H;     // 74
constexpr int SW = TZ + 2 * HZ;       // 80
constexpr int SMEM = SROWS * SW;      // floats per staged field
constexpr int kPer = TX * TZ / kThreads;
constexpr int kNB = 2;                // cells per load batch of the stress kernel

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }

// QS:843-966, the same rounding order as viscoac2d.cu
template <bool XDIR, int FLAG>
__device__ __forceinline__ float rsg(const float* s, int r, int c, const float* a, float h) {
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

__device__ __forceinline__ bool tile_of(const EArgs& a, TileRef& t) {
    t.shot = a.slot_to_shot[blockIdx.y];
    t.sd = a.shots[t.shot];
    t.tile = blockIdx.x;
    const int tx_i = t.tile / a.L.ntz, tz_i = t.tile - tx_i * a.L.ntz;
    t.x0 = tx_i * TX;
    t.z0 = tz_i * TZ;
    return t.x0 < t.sd.nx;
}

__device__ __forceinline__ long long cell(const EArgs& a, int shot, int x, int z) {
    return (long long)shot * a.L.shot_stride + (long long)(x + a.L.gx) * a.L.pitch + a.L.gz + z;
}

// stage (f0 + f1) + f2 (NF = 3) or f0 + f1 (NF = 2) on the tile plus halo
template <int NF>
__device__ __forceinline__ void stage(float* s, const EArgs& a, const TileRef& t, const float* f0, const float* f1,
                                      const float* f2) {
    constexpr int W4 = SW / 4;
#pragma unroll 3  // several rows' loads in flight before their shared-memory stores
    for (int i = threadIdx.x; i < SROWS * W4; i += kThreads) {
        const int r = i / W4, c = i - r * W4;
        const long long off = cell(a, t.shot, t.x0 - H + r, t.z0 - HZ + 4 * c);
        const float4 u = __ldg(reinterpret_cast<const float4*>(f0 + off));
        const float4 v = __ldg(reinterpret_cast<const float4*>(f1 + off));
        float4 w = make_float4(fa(u.x, v.x), fa(u.y, v.y), fa(u.z, v.z), fa(u.w, v.w));
        if (NF == 3) {
            const float4 d = __ldg(reinterpret_cast<const float4*>(f2 + off));
            w = make_float4(fa(w.x, d.x), fa(w.y, d.y), fa(w.z, d.z), fa(w.w, d.w));
        }
        *reinterpret_cast<float4*>(s + r * SW + 4 * c) = w;
    }
}

// one split-sponge factor applied in QS order (left table, then right table)
__device__ __forceinline__ float xs(float u, int x, int n, int np, const float* tn, const float* tp) {
    if (x <= np) u = fm(u, tn[x]);
    if (x >= n - np - 1) u = fm(u, tp[n - 1 - x]);
    return u;
}

__global__ void __launch_bounds__(kThreads) e_velocity_kernel(const __grid_constant__ EArgs a) {
    extern __shared__ __align__(16) float smem[];
    float* sSxx = smem;
    float* sSxz = smem + SMEM;
    float* sSzz = smem + 2 * SMEM;
    TileRef t;
    if (!tile_of(a, t)) return;
    stage<3>(sSxx, a, t, a.f[E_SXXX], a.f[E_SXXZ], a.f[E_SXXR]);
    stage<3>(sSxz, a, t, a.f[E_SXZX], a.f[E_SXZZ], a.f[E_SXZR]);
    stage<3>(sSzz, a, t, a.f[E_SZZX], a.f[E_SZZZ], a.f[E_SZZR]);
    __syncthreads();
    const int nx = t.sd.nx, nz = a.nz;
    const float* tb = a.spg;
    const int st = a.spg_stride;
    float* vxx = a.f[E_VXX];
    float* vxz = a.f[E_VXZ];
    float* vzx = a.f[E_VZX];
    float* vzz = a.f[E_VZZ];
    // four cells per batch: the batch's global loads are issued before its arithmetic
    for (int j0 = 0; j0 < kPer; j0 += 4) {
        float o[4][4], bu[4];
        long long cc[4];
        bool ok[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int i = threadIdx.x + (j0 + u) * kThreads, r = i / TZ, z = i - r * TZ;
            const int gx = t.x0 + r, gz = t.z0 + z;
            ok[u] = gx < nx && gz < nz;
            cc[u] = cell(a, t.shot, gx, gz);
            if (ok[u]) {
                o[u][0] = vxx[cc[u]]; o[u][1] = vxz[cc[u]]; o[u][2] = vzx[cc[u]]; o[u][3] = vzz[cc[u]];
                bu[u] = __ldg(a.busg + (long long)min(t.sd.x0 + gx, a.nx_model - 1) * a.mpitch + gz);
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            if (!ok[u]) continue;
            const int i = threadIdx.x + (j0 + u) * kThreads, r = i / TZ, z = i - r * TZ;
            const int gx = t.x0 + r, gz = t.z0 + z;
            const long long c = cc[u];
            const float dtb = fm(a.dt, bu[u]);
            float n_xx = fa(o[u][0], fm(dtb, rsg<true, 0>(sSxx, r + H, z + HZ, a.a, a.hx)));   // QS:713-720
            float n_xz = fa(o[u][1], fm(dtb, rsg<false, 0>(sSxz, r + H, z + HZ, a.a, a.hz)));  // QS:722-729
            n_xx = xs(n_xx, gx, nx, a.npx, tb + 0 * st, tb + 1 * st);
            n_xz = xs(n_xz, gz, nz, a.npz, tb + 2 * st, tb + 3 * st);
            float n_zx = fa(o[u][2], fm(dtb, rsg<true, 0>(sSxz, r + H, z + HZ, a.a, a.hx)));   // QS:733-740
            float n_zz = fa(o[u][3], fm(dtb, rsg<false, 0>(sSzz, r + H, z + HZ, a.a, a.hz)));  // QS:741-748
            n_zx = xs(n_zx, gx, nx, a.npx, tb + 0 * st, tb + 1 * st);
            n_zz = xs(n_zz, gz, nz, a.npz, tb + 2 * st, tb + 3 * st);
            vxx[c] = n_xx; vxz[c] = n_xz; vzx[c] = n_zx; vzz[c] = n_zz;
        }
    }
}

__global__ void __launch_bounds__(kThreads) e_stress_kernel(const __grid_constant__ EArgs a) {
    __shared__ __align__(16) float sVx[SMEM];
    __shared__ __align__(16) float sVz[SMEM];
    TileRef t;
    if (!tile_of(a, t)) return;
    stage<2>(sVx, a, t, a.f[E_VXX], a.f[E_VXZ], nullptr);  // vx = vxx + vxz (QS:1273-1291)
    stage<2>(sVz, a, t, a.f[E_VZX], a.f[E_VZZ], nullptr);  // vz = vzx + vzz
    __syncthreads();
    const int nx = t.sd.nx, nz = a.nz;
    const float* tb = a.spg;
    const int st = a.spg_stride;
    const ShotDev& sd = t.sd;
    const float wav = __ldg(a.wavelets + sd.wav_off + a.step);
    const float dt = a.dt, f = a.f_mem;
    for (int j0 = 0; j0 < kPer; j0 += kNB) {
        float v[kNB][18];
        float q1[kNB], q2[kNB], q3[kNB], m1[kNB], m2[kNB], m3[kNB];
        long long cc[kNB];
        bool ok[kNB];
#pragma unroll
        for (int u = 0; u < kNB; u++) {
            const int i = threadIdx.x + (j0 + u) * kThreads, r = i / TZ, z = i - r * TZ;
            const int gx = t.x0 + r, gz = t.z0 + z;
            ok[u] = gx < nx && gz < nz;
            cc[u] = cell(a, t.shot, gx, gz);
            if (ok[u]) {
#pragma unroll
                for (int k = 0; k < 18; k++) v[u][k] = a.f[E_SXXX + k][cc[u]];
                const long long mi = (long long)min(sd.x0 + gx, a.nx_model - 1) * a.mpitch + gz;
                q1[u] = __ldg(a.q1 + mi); q2[u] = __ldg(a.q2 + mi); q3[u] = __ldg(a.q3 + mi);
                m1[u] = __ldg(a.m1 + mi); m2[u] = __ldg(a.m2 + mi); m3[u] = __ldg(a.m3 + mi);
            }
        }
#pragma unroll
        for (int u = 0; u < kNB; u++) {
            if (!ok[u]) continue;
            const int i = threadIdx.x + (j0 + u) * kThreads, r = i / TZ, z = i - r * TZ;
            const int gx = t.x0 + r, gz = t.z0 + z;
            const float d1 = rsg<true, 1>(sVx, r + H, z + HZ, a.a, a.hx);   // Dx1 vx
            const float d2 = rsg<true, 1>(sVz, r + H, z + HZ, a.a, a.hx);   // Dx1 vz
            const float d3 = rsg<false, 1>(sVx, r + H, z + HZ, a.a, a.hz);  // Dz1 vx
            const float d4 = rsg<false, 1>(sVz, r + H, z + HZ, a.a, a.hz);  // Dz1 vz
            float* w = v[u];  // sxxx sxxz sxxr szzx szzz szzr sxzx sxzz sxzr rxxx rxxz rxxr rzzx rzzz rzzr rxzx rxzz rxzr
            const float rxx = fa(fa(w[9], w[10]), w[11]);   // memory sums of the previous step
            const float rzz = fa(fa(w[12], w[13]), w[14]);
            const float rxz = fa(fa(w[15], w[16]), w[17]);
            float src = 0.0f;
            const int bx = gx - sd.stamp_x0, bz = gz - sd.stamp_z0;
            const bool in_stamp = bx >= 0 && bx < sd.stamp_w && bz >= 0 && bz < sd.stamp_h;
            if (in_stamp)
                src = __fdiv_rn(fm(fm(wav, __ldg(a.stamps + sd.stamp_off + bx * sd.stamp_h + bz)), dt), a.dz2);
            // calpstrxx (QS:993-1020)
            w[0] = xs(fa(w[0], fm(dt, fm(q1[u], d1))), gx, nx, a.npx, tb + 4 * st, tb + 5 * st);
            w[1] = xs(fa(w[1], fm(dt, fm(q2[u], d4))), gz, nz, a.npz, tb + 6 * st, tb + 7 * st);
            w[2] = fa(w[2], fm(dt, rxx));
            if (in_stamp) w[0] = fa(src, w[0]);  // QS:801, 1384
            // calpstrzz (QS:1023-1050)
            w[3] = xs(fa(w[3], fm(dt, fm(q2[u], d1))), gx, nx, a.npx, tb + 4 * st, tb + 5 * st);
            w[4] = xs(fa(w[4], fm(dt, fm(q1[u], d4))), gz, nz, a.npz, tb + 6 * st, tb + 7 * st);
            w[5] = fa(w[5], fm(dt, rzz));
            if (in_stamp) w[3] = fa(src, w[3]);
            // calpstrxz (QS:1053-1132)
            w[6] = xs(fa(w[6], fm(dt, fm(q3[u], d2))), gx, nx, a.npx, tb + 4 * st, tb + 5 * st);
            w[7] = xs(fa(w[7], fm(dt, fm(q3[u], d3))), gz, nz, a.npz, tb + 6 * st, tb + 7 * st);
            w[8] = fa(w[8], fm(dt, rxz));
            // calprxx, calprzz, calprxz (QS:1135-1269)
            w[9] = xs(fa(w[9], fm(f, fm(m1[u], d1))), gx, nx, a.npx, tb + 4 * st, tb + 5 * st);
            w[10] = xs(fa(w[10], fm(f, fm(m2[u], d4))), gz, nz, a.npz, tb + 6 * st, tb + 7 * st);
            w[11] = fa(w[11], fm(f, rxx));
            w[12] = xs(fa(w[12], fm(f, fm(m2[u], d1))), gx, nx, a.npx, tb + 4 * st, tb + 5 * st);
            w[13] = xs(fa(w[13], fm(f, fm(m1[u], d4))), gz, nz, a.npz, tb + 6 * st, tb + 7 * st);
            w[14] = fa(w[14], fm(f, rzz));
            w[15] = xs(fa(w[15], fm(f, fm(m3[u], d2))), gx, nx, a.npx, tb + 4 * st, tb + 5 * st);
            w[16] = xs(fa(w[16], fm(f, fm(m3[u], d3))), gz, nz, a.npz, tb + 6 * st, tb + 7 * st);
            w[17] = fa(w[17], fm(f, rxz));
#pragma unroll
            for (int k = 0; k < 18; k++) a.f[E_SXXX + k][cc[u]] = w[k];
        }
    }
    // receivers: record1 = strzz, record2 = strxx after the step (QM:452-459)
    const int* trp = a.tile_rec_ptr + sd.tile_rec_base + t.tile;
    const int rb = trp[0], re = trp[1];
    if (re > rb) {
        __syncthreads();
        for (int j = rb + threadIdx.x; j < re; j += kThreads) {
            const int ridx = a.tile_rec_idx[j];
            const long long c = cell(a, t.shot, a.rec_x[sd.rec_list + ridx], a.rec_z[sd.rec_list + ridx]);
            const long long o = sd.rec_base + (long long)a.step * sd.nrec + ridx;
            a.records[o] = fa(fa(a.f[E_SZZX][c], a.f[E_SZZZ][c]), a.f[E_SZZR][c]);
            a.records2[o] = fa(fa(a.f[E_SXXX][c], a.f[E_SXXZ][c]), a.f[E_SXXR][c]);
        }
    }
}

}  // namespace

cudaError_t viscoel2d_launch_step(const EArgs& a, int active, cudaStream_t st) {
    dim3 grid(a.L.ntx * a.L.ntz, active);
    const size_t smem = sizeof(float) * 3 * SMEM;
    static bool attr[kMaxDevices] = {};
    if (cudaError_t e = smem_attr_once((const void*)e_velocity_kernel, (int)smem, attr)) return e;
    e_velocity_kernel<<<grid, kThreads, smem, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e_stress_kernel<<<grid, kThreads, 0, st>>>(a);
    return cudaGetLastError();
}

// QS:434-469 (density averaged in place, then buoyancy) and QS:473-551 (Blanch's tau for P and S),
// single precision in the reference's operation order, and the six stress-update coefficients.
// qp / qs == nullptr: Q = 1e5 (QM:418-419).
void viscoel2d_prepare(int nx, int nz, const float* vp, const float* vs, const float* rho, const float* qp,
                       const float* qs, float f0, float* busg, float* q1, float* q2, float* q3, float* m1, float* m2,
                       float* m3, float* rtau_out) {
    std::vector<float> r(rho, rho + (size_t)nx * nz);
    auto R = [&](int k, int i) -> float& { return r[(size_t)i * nz + k]; };
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
        const float mu = rr * (vs[c] * vs[c]);
        const float lambmu = rr * (vp[c] * vp[c]);
        const float qpv = (qp ? qp[c] : 100000.0f) * (18.0f / 20.0f);
        const float qsv = (qs ? qs[c] : 100000.0f) * (18.0f / 20.0f);
        float tp = 0.0f, ts = 0.0f;
        if (dup - dlow != 0.0f) {
            tp = 1.0f / qpv * (nup - nlow) / (dup - dlow);
            ts = 1.0f / qsv * (nup - nlow) / (dup - dlow);
        }
        const float taup = (tp * tss + tss) / tss;
        const float taus = (ts * tss + tss) / tss;
        q1[c] = lambmu * taup;
        q2[c] = lambmu * taup - 2.0f * mu * taus;
        q3[c] = mu * taus;
        m1[c] = lambmu * (taup - 1.0f);
        m2[c] = lambmu * (taup - 1.0f) - 2.0f * mu * (taus - 1.0f);
        m3[c] = mu * (taus - 1.0f);
    }
    *rtau_out = 1.0f / tss;
}

}  // namespace sfd
