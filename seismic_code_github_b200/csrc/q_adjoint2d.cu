// Adjoint of one time step of the viscoacoustic scheme (the vs = 0 reduction of
// forward/Q_forward/Q_multishot_fd_subroutine_fsbc_zy_rotated.f90, QS:695-1337, as the
// kernels of viscoac2d.cu implement it) and the zero-lag imaging conditions for the two
// model parameters of the stress update, p1 = lambda tau_eps/tau_sigma and
// p2 = lambda (tau_eps/tau_sigma - 1).  The reference has no adjoint.
//
// Forward step k (fields in place, eight per cell):
//   S  = sx + sz + sr
//   vx = Ax (vx + dt b Dx0 S),  vz = Az (vz + dt b Dz0 S)                 (velocity kernel)
//   d1 = Dx1 vx, d4 = Dz1 vz, R = rx + rz + rr (old)
//   sx = A'x (sx + dt p1 d1) + stamp w_k,  sz = A'z (sz + dt p1 d4),  sr += dt R
//   rx = A'x (rx + f p2 d1),  rz = A'z (rz + f p2 d4),  rr += f R            (stress kernel)
//   record = S at the receivers
// Adjoint step k (hatted fields hold d misfit / d state after step k, with the residual of
// step k already added at the receivers to sx^, sz^, sr^):
//   kernel A: T1 = A'x (dt p1 sx^ + f p2 rx^), T4 = A'z (dt p1 sz^ + f p2 rz^)   (on a halo)
//             vx^ = Ax (vx^ + Dx1^T T1),  vz^ = Az (vz^ + Dz1^T T4)
//             Qx = dt b vx^, Qz = dt b vz^;   dw_k = sum stamp sx^
//   kernel B: u1 = A'x sx^, u4 = A'z sz^, w1 = A'x rx^, w4 = A'z rz^, aR = f rr^ + dt sr^
//             aS = Dx0^T Qx + Dz0^T Qz
//             sx^ = u1 + aS, sz^ = u4 + aS, sr^ += aS, rx^ = w1 + aR, rz^ = w4 + aR, rr^ += aR
//             g1 += d1 u1 + d4 u4,  g2 += d1 w1 + d4 w4;   then sx^, sz^, sr^ += res_{k-1}
// so that d misfit / d p1 = dt sum g1 and d misfit / d p2 = f sum g2.  The transposed
// rotated-staggered derivatives gather from the mirrored taps of QS:843-966.  Kernel A reads
// the stress adjoints of its halo and writes only velocity adjoints and Qx, Qz; kernel B reads
// the Qx, Qz halo and writes only its own cells, so neither launch races with itself.
#include <cuda_runtime.h>

#include <algorithm>

#include "sfd_internal.h"

namespace sfd {
namespace {

constexpr int kThreads = 256;
constexpr int TX = kTileX, TZ = kTileZ;
constexpr int H = 5;               // rotated-staggered reach (offsets -5 .. +5)
constexpr int HZ = 8;              // z halo rounded for float4 staging
constexpr int SROWS = TX + 2 * H;  // staged rows x0-5 .. x0+TX+4
constexpr int SW = TZ + 2 * HZ;    // staged columns z0-8 .. z0+TZ+7
constexpr int SMEM = SROWS * SW;
constexpr int kPer = TX * TZ / kThreads;  // cells per thread
constexpr int kNB = 4;    // cells per load batch
constexpr int kNBS = 2;  // cells per load batch of the stress kernel (three CTAs per SM)

struct Tile {
    int shot, tile, x0, z0;
    ShotDev sd;
};

__device__ __forceinline__ bool tile_of(const QAdjArgs& a, Tile& t) {
    t.shot = a.slot_to_shot[blockIdx.y];
    t.sd = a.shots[t.shot];
    t.tile = blockIdx.x;
    const int tx_i = t.tile / a.L.ntz, tz_i = t.tile - tx_i * a.L.ntz;
    t.x0 = tx_i * TX;
    t.z0 = tz_i * TZ;
    return t.x0 < t.sd.nx;
}

__device__ __forceinline__ long long cell(const QAdjArgs& a, int shot, int x, int z) {
    return (long long)shot * a.L.shot_stride + (long long)(x + a.L.gx) * a.L.pitch + a.L.gz + z;
}

// product of the two split-sponge factors of a coordinate (left / right tables)
__device__ __forceinline__ float sp(int x, int n, int np, const float* tn, const float* tp) {
    float f = 1.0f;
    if (x <= np) f *= tn[x];
    if (x >= n - np - 1) f *= tp[n - 1 - x];
    return f;
}

__global__ void __launch_bounds__(kThreads) q_adj_velocity_kernel(const __grid_constant__ QAdjArgs a) {
    __shared__ __align__(16) float sT1[SMEM];
    __shared__ __align__(16) float sT4[SMEM];
    __shared__ float s_dw;
    Tile t;
    if (!tile_of(a, t)) return;
    const int nx = t.sd.nx, nz = a.nz;
    const float* tb = a.spg;
    const int st = a.spg_stride;
    const float dt = a.dt, f = a.f_mem;
    if (threadIdx.x == 0) s_dw = 0.0f;
    // T1, T4 on the tile plus halo (zero outside the grid: the forward never updates there)
    constexpr int W4 = SW / 4;
#pragma unroll 3  // several rows' loads in flight before their shared-memory stores
    for (int i = threadIdx.x; i < SROWS * W4; i += kThreads) {
        const int r = i / W4, c = i - r * W4;
        const int gx = t.x0 - H + r, gz0 = t.z0 - HZ + 4 * c;
        float4 o1 = make_float4(0.f, 0.f, 0.f, 0.f), o4 = o1;
        if (gx >= 0 && gx < nx && gz0 + 3 >= 0 && gz0 < nz) {
            const long long off = cell(a, t.shot, gx, gz0);
            const float4 SX = __ldg(reinterpret_cast<const float4*>(a.asx + off));
            const float4 RX = __ldg(reinterpret_cast<const float4*>(a.arx + off));
            const float4 SZ = __ldg(reinterpret_cast<const float4*>(a.asz + off));
            const float4 RZ = __ldg(reinterpret_cast<const float4*>(a.arz + off));
            const long long mi = (long long)min(t.sd.x0 + gx, a.nx_model - 1) * a.mpitch + gz0;
            const float4 P1 = __ldg(reinterpret_cast<const float4*>(a.p1 + mi));
            const float4 P2 = __ldg(reinterpret_cast<const float4*>(a.p2 + mi));
            const float ax = sp(gx, nx, a.npx, tb + 4 * st, tb + 5 * st);
            const float sx_[4] = {SX.x, SX.y, SX.z, SX.w}, rx_[4] = {RX.x, RX.y, RX.z, RX.w};
            const float sz_[4] = {SZ.x, SZ.y, SZ.z, SZ.w}, rz_[4] = {RZ.x, RZ.y, RZ.z, RZ.w};
            const float p1_[4] = {P1.x, P1.y, P1.z, P1.w}, p2_[4] = {P2.x, P2.y, P2.z, P2.w};
            float v1[4], v4[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int gz = gz0 + j;
                const bool ok = gz >= 0 && gz < nz;
                const float az = ok ? sp(gz, nz, a.npz, tb + 6 * st, tb + 7 * st) : 0.0f;
                const float d1 = dt * p1_[j], d2 = f * p2_[j];
                v1[j] = ok ? ax * fmaf(d1, sx_[j], d2 * rx_[j]) : 0.0f;
                v4[j] = ok ? az * fmaf(d1, sz_[j], d2 * rz_[j]) : 0.0f;
            }
            o1 = make_float4(v1[0], v1[1], v1[2], v1[3]);
            o4 = make_float4(v4[0], v4[1], v4[2], v4[3]);
        }
        *reinterpret_cast<float4*>(sT1 + r * SW + 4 * c) = o1;
        *reinterpret_cast<float4*>(sT4 + r * SW + 4 * c) = o4;
    }
    __syncthreads();
    float c[5];
#pragma unroll
    for (int m = 0; m < 5; m++) c[m] = a.a[m];
    // kNB cells per batch: the global loads of a batch are issued before its arithmetic
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
                vxo[u] = a.avx[cc[u]];
                vzo[u] = a.avz[cc[u]];
                bu[u] = __ldg(a.busg + (long long)min(t.sd.x0 + gx, a.nx_model - 1) * a.mpitch + gz);
            }
        }
#pragma unroll
        for (int u = 0; u < kNB; u++) {
            if (!ok[u]) continue;
            const int i = threadIdx.x + (j0 + u) * kThreads, r = i / TZ, z = i - r * TZ;
            const int gx = t.x0 + r, gz = t.z0 + z;
            const float* p1s = sT1 + (r + H) * SW + z + HZ;
            const float* p4s = sT4 + (r + H) * SW + z + HZ;
            auto T1 = [&](int dx, int dz) { return p1s[dx * SW + dz]; };
            auto T4 = [&](int dx, int dz) { return p4s[dx * SW + dz]; };
            float s1 = 0.0f, s4 = 0.0f;
#pragma unroll
            for (int m = 0; m < 5; m++) {
                // Dx1^T: t(x-1-m, z-1-m) - t(x+m, z+m) + t(x-1-m, z+m) - t(x+m, z-1-m); Dz1^T flips the cross terms
                const float a1 = T1(-1 - m, -1 - m) - T1(m, m), b1 = T1(-1 - m, m) - T1(m, -1 - m);
                const float a4 = T4(-1 - m, -1 - m) - T4(m, m), b4 = T4(-1 - m, m) - T4(m, -1 - m);
                s1 = fmaf(c[m], a1 + b1, s1);
                s4 = fmaf(c[m], a4 - b4, s4);
            }
            const float ax = sp(gx, nx, a.npx, tb + 0 * st, tb + 1 * st);
            const float az = sp(gz, nz, a.npz, tb + 2 * st, tb + 3 * st);
            const float vx = ax * fmaf(a.hx, s1, vxo[u]);
            const float vz = az * fmaf(a.hz, s4, vzo[u]);
            const float db = dt * bu[u];
            a.avx[cc[u]] = vx;
            a.avz[cc[u]] = vz;
            a.qx[cc[u]] = db * vx;
            a.qz[cc[u]] = db * vz;
        }
    }
    // wavelet gradient: dw_k = dt / dz^2 sum over the source stamp of sx^ (QS:1384 transposed)
    const ShotDev& sd = t.sd;
    const int bx0 = max(sd.stamp_x0, t.x0), bx1 = min(sd.stamp_x0 + sd.stamp_w, min(t.x0 + TX, nx));
    const int bz0 = max(sd.stamp_z0, t.z0), bz1 = min(sd.stamp_z0 + sd.stamp_h, min(t.z0 + TZ, nz));
    if (a.lam_src && bx1 > bx0 && bz1 > bz0) {
        const int w = bz1 - bz0;
        float part = 0.0f;
        for (int i = threadIdx.x; i < (bx1 - bx0) * w; i += kThreads) {
            const int x = bx0 + i / w, z = bz0 + i % w;
            const float g = __ldg(a.stamps + sd.stamp_off + (x - sd.stamp_x0) * sd.stamp_h + (z - sd.stamp_z0));
            part = fmaf(g, a.asx[cell(a, t.shot, x, z)], part);
        }
        for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) atomicAdd(&s_dw, part);
        __syncthreads();
        if (threadIdx.x == 0) atomicAdd(a.lam_src + (long long)t.shot * a.nt_max + a.step, s_dw * (dt / a.dz2));
    }
}

__global__ void __launch_bounds__(kThreads, 3) q_adj_stress_kernel(const __grid_constant__ QAdjArgs a) {
    __shared__ __align__(16) float sQx[SMEM];
    __shared__ __align__(16) float sQz[SMEM];
    Tile t;
    if (!tile_of(a, t)) return;
    const int nx = t.sd.nx, nz = a.nz;
    const float* tb = a.spg;
    const int st = a.spg_stride;
    constexpr int W4 = SW / 4;
#pragma unroll 3  // several rows' loads in flight before their shared-memory stores
    for (int i = threadIdx.x; i < SROWS * W4; i += kThreads) {
        const int r = i / W4, c = i - r * W4;
        const long long off = cell(a, t.shot, t.x0 - H + r, t.z0 - HZ + 4 * c);
        *reinterpret_cast<float4*>(sQx + r * SW + 4 * c) = __ldg(reinterpret_cast<const float4*>(a.qx + off));
        *reinterpret_cast<float4*>(sQz + r * SW + 4 * c) = __ldg(reinterpret_cast<const float4*>(a.qz + off));
    }
    __syncthreads();
    float c[5];
#pragma unroll
    for (int m = 0; m < 5; m++) c[m] = a.a[m];
    const float dt = a.dt, f = a.f_mem;
    for (int j0 = 0; j0 < kPer; j0 += kNBS) {
        float hsx[kNBS], hsz[kNBS], hsr[kNBS], hrx[kNBS], hrz[kNBS], hrr[kNBS], d1[kNBS], d4[kNBS], g1[kNBS], g2[kNBS];
        long long cc[kNBS];
        bool ok[kNBS];
#pragma unroll
        for (int u = 0; u < kNBS; u++) {
            const int i = threadIdx.x + (j0 + u) * kThreads, r = i / TZ, z = i - r * TZ;
            const int gx = t.x0 + r, gz = t.z0 + z;
            ok[u] = gx < nx && gz < nz;
            const long long c = cell(a, t.shot, gx, gz);
            cc[u] = c;
            if (ok[u]) {
                hsx[u] = a.asx[c]; hsz[u] = a.asz[c]; hsr[u] = a.asr[c];
                hrx[u] = a.arx[c]; hrz[u] = a.arz[c]; hrr[u] = a.arr[c];
                d1[u] = __ldg(a.d1 + c); d4[u] = __ldg(a.d4 + c);
                g1[u] = a.g1[c]; g2[u] = a.g2[c];
            }
        }
#pragma unroll
        for (int u = 0; u < kNBS; u++) {
            if (!ok[u]) continue;
            const int i = threadIdx.x + (j0 + u) * kThreads, r = i / TZ, z = i - r * TZ;
            const int gx = t.x0 + r, gz = t.z0 + z;
            const float* px = sQx + (r + H) * SW + z + HZ;
            const float* pz = sQz + (r + H) * SW + z + HZ;
            auto QX = [&](int dx, int dz) { return px[dx * SW + dz]; };
            auto QZ = [&](int dx, int dz) { return pz[dx * SW + dz]; };
            float sx = 0.0f, sz = 0.0f;
#pragma unroll
            for (int m = 0; m < 5; m++) {
                // Dx0^T: t(x-m, z-m) - t(x+1+m, z+1+m) + t(x-m, z+1+m) - t(x+1+m, z-m); Dz0^T flips the cross terms
                const float ax_ = QX(-m, -m) - QX(1 + m, 1 + m), bx_ = QX(-m, 1 + m) - QX(1 + m, -m);
                const float az_ = QZ(-m, -m) - QZ(1 + m, 1 + m), bz_ = QZ(-m, 1 + m) - QZ(1 + m, -m);
                sx = fmaf(c[m], ax_ + bx_, sx);
                sz = fmaf(c[m], az_ - bz_, sz);
            }
            const float aS = fmaf(a.hx, sx, a.hz * sz);
            const long long cu = cc[u];
            const float axs = sp(gx, nx, a.npx, tb + 4 * st, tb + 5 * st);
            const float azs = sp(gz, nz, a.npz, tb + 6 * st, tb + 7 * st);
            const float u1 = axs * hsx[u], u4 = azs * hsz[u];
            const float w1 = axs * hrx[u], w4 = azs * hrz[u];
            const float aR = fmaf(f, hrr[u], dt * hsr[u]);
            a.g1[cu] = g1[u] + fmaf(d1[u], u1, d4[u] * u4);
            a.g2[cu] = g2[u] + fmaf(d1[u], w1, d4[u] * w4);
            a.asx[cu] = u1 + aS;
            a.asz[cu] = u4 + aS;
            a.asr[cu] = hsr[u] + aS;
            a.arx[cu] = w1 + aR;
            a.arz[cu] = w4 + aR;
            a.arr[cu] = hrr[u] + aR;
        }
    }
    // residual of step k-1 at the receivers of this tile (QM:452-459 transposed): S^ -> sx^, sz^, sr^
    const ShotDev& sd = t.sd;
    const int* trp = a.tile_rec_ptr + sd.tile_rec_base + t.tile;
    const int rb = trp[0], re = trp[1];
    if (a.step >= 1 && re > rb) {
        __syncthreads();
        for (int j = rb + threadIdx.x; j < re; j += kThreads) {
            const int ridx = a.tile_rec_idx[j];
            const long long cc = cell(a, t.shot, a.rec_x[sd.rec_list + ridx], a.rec_z[sd.rec_list + ridx]);
            const float v = a.res[sd.rec_base + (long long)(a.step - 1) * sd.nrec + ridx];
            atomicAdd(a.asx + cc, v);
            atomicAdd(a.asz + cc, v);
            atomicAdd(a.asr + cc, v);
        }
    }
}

// sx^, sz^, sr^ of every shot in [first, first + n) += res of the shot's last step
__global__ void q_adjoint_init_kernel(QAdjArgs a, int first_shot) {
    const int s = first_shot + blockIdx.y;
    const ShotDev sd = a.shots[s];
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < sd.nrec; r += gridDim.x * blockDim.x) {
        const long long cc = cell(a, s, a.rec_x[sd.rec_list + r], a.rec_z[sd.rec_list + r]);
        const float v = a.res[sd.rec_base + (long long)(sd.nt - 1) * sd.nrec + r];
        atomicAdd(a.asx + cc, v);
        atomicAdd(a.asz + cc, v);
        atomicAdd(a.asr + cc, v);
    }
}

// Model-grid gradients.  Shot s's column x reads prepared-model column sd.x0 + x, which is
// model column ap_x0[s] + x.  dJ/dp1 = dt g1, dJ/dp2 = f g2 (sums over the shots covering the
// cell); p1 = lambda tpss, p2 = lambda (tpss - 1) with lambda = rho_avg vp^2 and
// tpss = 1 + kappa / Q (QS:473-551), so dp/dvp = 2 p / vp and dp1/d(1/Q) = dp2/d(1/Q) = lambda kappa.
__global__ void q_gradient_reduce_kernel(const double* __restrict__ acc1, const double* __restrict__ acc2, Layout2D L,
                                         const ShotDev* __restrict__ shots, const int* __restrict__ ap_x0, int nshot,
                                         const float* __restrict__ vp, const float* __restrict__ p1,
                                         const float* __restrict__ p2, int mpitch, int nx_model, int nz, double dt,
                                         double f, double kappa, double* grad_vp, double* grad_invq) {
    const long long n = (long long)nx_model * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int X = (int)(i / nz), z = (int)(i - (long long)X * nz);
        double gv = 0.0, gq = 0.0;
        for (int s = 0; s < nshot; s++) {
            const int x = X - ap_x0[s];
            if (x < 0 || x >= shots[s].nx) continue;
            const long long c = (long long)s * L.shot_stride + (long long)(x + L.gx) * L.pitch + L.gz + z;
            const double G1 = dt * acc1[c], G2 = f * acc2[c];
            const long long b = (long long)(shots[s].x0 + x) * mpitch + z;
            const double q1 = p1[b], q2 = p2[b];
            gv += 2.0 * (q1 * G1 + q2 * G2) / (double)vp[(long long)X * mpitch + z];
            gq += (q1 - q2) * kappa * (G1 + G2);
        }
        grad_vp[i] = gv;
        if (grad_invq) grad_invq[i] = gq;
    }
}

int grid_for(long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 16); }

}  // namespace

cudaError_t q_adjoint_launch_step(const QAdjArgs& a, int active, cudaStream_t st) {
    dim3 grid(a.L.ntx * a.L.ntz, active);
    q_adj_velocity_kernel<<<grid, kThreads, 0, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    q_adj_stress_kernel<<<grid, kThreads, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t q_adjoint_launch_init(const QAdjArgs& a, int first_shot, int nshot, int nrec_max, cudaStream_t st) {
    if (nrec_max <= 0 || nshot <= 0) return cudaSuccess;
    dim3 grid((nrec_max + 255) / 256, nshot);
    q_adjoint_init_kernel<<<grid, 256, 0, st>>>(a, first_shot);
    return cudaGetLastError();
}

cudaError_t q_launch_gradient_reduce(const double* acc1, const double* acc2, const Layout2D& L, const ShotDev* shots,
                                     const int* ap_x0, int nshot, const float* vp, const float* p1, const float* p2,
                                     int mpitch, int nx_model, int nz, double dt, double f, double kappa,
                                     double* grad_vp, double* grad_invq, cudaStream_t st) {
    const long long n = (long long)nx_model * nz;
    q_gradient_reduce_kernel<<<grid_for(n), 256, 0, st>>>(acc1, acc2, L, shots, ap_x0, nshot, vp, p1, p2, mpitch,
                                                           nx_model, nz, dt, f, kappa, grad_vp, grad_invq);
    return cudaGetLastError();
}

}  // namespace sfd
