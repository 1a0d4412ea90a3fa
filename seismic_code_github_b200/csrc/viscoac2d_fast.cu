// Default (fast) viscoacoustic step of SFD_VISCOAC_2D: the rotated-staggered-grid scheme of
// forward/Q_forward/Q_multishot_fd_subroutine_fsbc_zy_rotated.f90 (QS:751-835 and its leaves
// QS:843-1337) with vs = 0, FMA contraction, two kernels per time step.
//
// State.  Everywhere: vx, vz (ping-pong), the merged stress sigma = (sx + sz) + sr (QS strxx,
// ping-pong) and the merged memory variable r = (rx + rz) + rr (in place).  Away from the sponge
// bands the split parts only ever appear summed, so the step updates the sums:
//   sigma += dt (p1 (d1 + d4) + r_old) + source,   r += f (p2 (d1 + d4) + r_old),
// with f = -dt / tau_sigma, p1 = M tau_eps / tau_sigma, p2 = M (tau_eps / tau_sigma - 1),
// d1 = 0.5/dx Dx1 vx, d4 = 0.5/dz Dz1 vz.  In the bands (x <= npx, x >= nx - npx - 1, z <= npz,
// z >= nz - npz - 1) the split sponge of QS:609-654 multiplies the x and z parts separately, so
// there the split parts sx, sz, sr, rx, rz, rr are kept (in place) and updated in the reference's
// form by the band kernel, which overwrites sigma and r of those cells.
//
// Step kernel (viscoac2d_fast_kernel).  A CTA owns one 64-wide z strip of one shot over a segment
// of columns and walks down x in chunks of 16 columns.  Chunk xb:
//   phase V: the new velocities of columns [xb+5, xb+21) on z0-8 .. z0+72 from sigma(t-1) on
//            columns [xb, xb+25) (a TMA box, double-buffered one chunk ahead, no multicast), into a
//            32-column ring in shared memory (column x in row x & 31) and, for the strip's own
//            cells, to global memory;
//   phase S: sigma and r of columns [xb, xb+16) from the ring (columns xb-4 .. xb+21).
// Each velocity column is computed once per segment (a first chunk per segment only computes
// velocities), only the z halo of 8 on each side of the strip is recomputed.  The rotated
// stencils (QS:843-966, (0.5/d) sum_m a_m t_m over four-point differences t_m) are evaluated as
// sums of products, one input column at a time: a thread keeps one column's window of 20 values in
// registers and adds each tap with one FMA into the outputs of its column (ten z values in phase
// V, eight in phase S).  Chunks that touch a sponge band or the grid edge also apply the velocity
// sponges and zero the velocities outside the grid, and write d1 and d4 of their cells for the
// band kernel.
//
// Band kernel (viscoac2d_band_kernel), one CTA per (shot, column): the split update of the band
// cells of the column (QS:993-1020, 1135-1170 with the sponges of QS:800-834 and the source of
// QS:1340-1390), then the receivers of the column (QM:452-459: strzz = sigma).
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "sfd_internal.h"

namespace sfd {
namespace {

constexpr int kThreads = 128;
constexpr int TZ = 64;            // strip width
constexpr int CH = 16;            // chunk columns
constexpr int SH = 16;            // z halo of the staged sigma
// sigma row pitch = box width: z0-16 .. z0+96 (the stencils read z0-13 .. z0+76).  16 mod 32 words:
// a half-warp of phase V (two columns x eight 10-wide z groups, 8-byte loads) hits every bank once.
constexpr int SW = 112;
constexpr int SROWS = CH + 9;     // 25 sigma columns per chunk: [xb, xb + 25)
constexpr int VH = 8;             // z halo of the recomputed velocities
constexpr int NV = TZ + 2 * VH;   // 80 velocity values per column: z0-8 .. z0+72
// velocity ring row pitch, 16 mod 32 words: the ring stores of phase V hit every bank once
constexpr int VW = NV;
constexpr int VRING = 32;         // velocity ring rows: column x lives in row x & 31
constexpr int KV = NV / 8;        // 10 velocity values per thread

struct FL {
    // bytes; every TMA destination is 128-byte aligned
    static constexpr int SIGB = (SROWS * SW * 4 + 127) / 128 * 128;  // 11264
    static constexpr int VX = 2 * SIGB;
    static constexpr int VZ = VX + VRING * VW * 4;
    static constexpr int TAB = VZ + VRING * VW * 4;  // floats: in-grid flag [NV], vz sponge [NV] per velocity z
    static constexpr int BAR = TAB + 4 * 2 * NV;
    static constexpr int BYTES = BAR + 16;
    static constexpr unsigned TX = 4u * SROWS * SW;
    static_assert(SIGB % 128 == 0 && BAR % 8 == 0, "aligned boxes and barriers");
};

__device__ __forceinline__ unsigned sptr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(sptr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(sptr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(sptr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Split-sponge factors of coordinate c (QS:609-654): table n applies at c <= np, table p at
// c >= n - np - 1 (both in the product for a grid narrower than two bands)
__device__ __forceinline__ float sponge_factor(int c, int n, int np, const float* tn, const float* tp) {
    float f = 1.0f;
    if (c >= 0 && c <= np) f *= __ldg(tn + c);
    if (c >= n - np - 1 && c < n) f *= __ldg(tp + n - 1 - c);
    return f;
}

struct QFGeo {
    int seg, nseg, nstrip;
};

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ float2 ld2(const float* p) { return *reinterpret_cast<const float2*>(p); }

// Phase V of one thread: the ten velocities of column x = xb + 5 + r at z = zv .. zv + 9 (QS:843-990).
// w[i] = sigma(column, zv - 6 + i) (8-byte loads), sigma(z + d) = w[6 + j + d].
template <bool EDGE>
__device__ __forceinline__ void phase_v(const QFastArgs& A, const float* sS, float* sVx, float* sVz, const float* tZin,
                                        const float* tVz, const ShotDev& sd, long long soff, int xs, int xe, int xb,
                                        int z0, int r, int zb) {
    const QArgs& a = A.q;
    const int nx = sd.nx, nz = a.nz;
    const int x = xb + 5 + r;
    const int zv = z0 - VH + KV * zb;  // first velocity z of the thread
    const bool xin = x >= 0 && x < nx;
    const long long c = soff + (long long)(x + a.L.gx) * a.L.pitch + a.L.gz + zv;
    const long long mi = (long long)min(max(sd.x0 + x, 0), a.nx_model - 1) * a.mpitch + zv;
    // old velocities and buoyancy first: their latency is covered by the stencil
    float2 vxo[KV / 2], vzo[KV / 2], bu[KV / 2];
#pragma unroll
    for (int h = 0; h < KV / 2; h++) {
        vxo[h] = vzo[h] = make_float2(0.0f, 0.0f);
        if (!EDGE || xin) {
            vxo[h] = ld2(A.vx_in + c + 2 * h);
            vzo[h] = ld2(A.vz_in + c + 2 * h);
        }
        bu[h] = __ldg(reinterpret_cast<const float2*>(a.busg + mi + 2 * h));
    }
    const float am[5] = {a.a[0], a.a[1], a.a[2], a.a[3], a.a[4]};
    // d/dx = h (DE + DF), d/dz = h (DE - DF) with the main- and anti-diagonal sums
    //   DE = sum_m a_m [s(x+m, z+m) - s(x-1-m, z-1-m)],  DF = sum_m a_m [s(x+m, z-1-m) - s(x-1-m, z+m)];
    // staged column k (0..9) is x - 5 + k
    float de[KV], df[KV];
#pragma unroll
    for (int j = 0; j < KV; j++) de[j] = df[j] = 0.0f;
#pragma unroll
    for (int k = 0; k < 10; k++) {
        const float* row = sS + (r + k) * SW + SH - VH - 6 + KV * zb;
        float w[20];
#pragma unroll
        for (int i = 0; i < 10; i++) {
            const float2 v = ld2(row + 2 * i);
            w[2 * i] = v.x;
            w[2 * i + 1] = v.y;
        }
        const int m = k >= 5 ? k - 5 : 4 - k;
#pragma unroll
        for (int j = 0; j < KV; j++) {
            if (k >= 5) {  // column x + m
                de[j] = fmaf(am[m], w[6 + j + m], de[j]);
                df[j] = fmaf(am[m], w[5 + j - m], df[j]);
            } else {       // column x - 1 - m
                de[j] = fmaf(-am[m], w[5 + j - m], de[j]);
                df[j] = fmaf(-am[m], w[6 + j + m], df[j]);
            }
        }
    }
    float fx = 1.0f, fi = 1.0f;
    if (EDGE) {
        fx = xin ? sponge_factor(x, nx, a.npx, a.spg, a.spg + a.spg_stride) : 0.0f;  // spgxn, spgxp
        fi = xin ? 1.0f : 0.0f;
    }
    const float cx = a.dt * a.hx, cz = a.dt * a.hz;
    float2 vxn[KV / 2], vzn[KV / 2];
    float* vxr = sVx + (x & (VRING - 1)) * VW + KV * zb;
    float* vzr = sVz + (x & (VRING - 1)) * VW + KV * zb;
#pragma unroll
    for (int h = 0; h < KV / 2; h++) {
        const int j = 2 * h;
        float2 vx, vz;
        vx.x = fmaf(bu[h].x * cx, de[j] + df[j], vxo[h].x);
        vx.y = fmaf(bu[h].y * cx, de[j + 1] + df[j + 1], vxo[h].y);
        vz.x = fmaf(bu[h].x * cz, de[j] - df[j], vzo[h].x);
        vz.y = fmaf(bu[h].y * cz, de[j + 1] - df[j + 1], vzo[h].y);
        if (EDGE) {  // sponges (QS:609-654: vx in x, vz in z), and zero outside the grid
            const float2 zi = ld2(tZin + KV * zb + j), zs = ld2(tVz + KV * zb + j);
            vx.x *= fx * zi.x;
            vx.y *= fx * zi.y;
            vz.x *= fi * zs.x;
            vz.y *= fi * zs.y;
        }
        *reinterpret_cast<float2*>(vxr + j) = vx;
        *reinterpret_cast<float2*>(vzr + j) = vz;
        vxn[h] = vx;
        vzn[h] = vz;
    }
    // the strip's own cells of the columns this segment owns
    if (x >= xs && x < xe && xin) {
#pragma unroll
        for (int h = 0; h < KV / 2; h++) {
            const int gz = zv + 2 * h;
            if (gz < z0 || gz >= z0 + TZ || gz >= nz) continue;
            if (gz + 1 < nz) {
                *reinterpret_cast<float2*>(A.vx_out + c + 2 * h) = vxn[h];
                *reinterpret_cast<float2*>(A.vz_out + c + 2 * h) = vzn[h];
            } else {
                A.vx_out[c + 2 * h] = vxn[h].x;
                A.vz_out[c + 2 * h] = vzn[h].x;
            }
        }
    }
}

template <bool EDGE>
__device__ __forceinline__ void chunk_body(const QFastArgs& A, unsigned char* smem, int set, const ShotDev& sd,
                                           int shot, int strip, int xs, int xe, int xb, bool first) {
    const QArgs& a = A.q;
    const float* sS = reinterpret_cast<const float*>(smem + set * FL::SIGB);
    float* sVx = reinterpret_cast<float*>(smem + FL::VX);
    float* sVz = reinterpret_cast<float*>(smem + FL::VZ);
    const float* tZin = reinterpret_cast<const float*>(smem + FL::TAB);  // 1 / 0: velocity z inside the grid
    const float* tVz = tZin + NV;                                        // vz sponge per velocity z (0 outside)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nx = sd.nx, nz = a.nz;
    const int z0 = strip * TZ;
    const long long soff = (long long)shot * a.L.shot_stride;

    // ---- phase V: velocities of columns xb+5 .. xb+21 on z0-8 .. z0+72; thread = column x 10 z
    // (a half-warp = two columns x eight z groups hits every bank once with the 16-mod-32 pitches) ----
    phase_v<EDGE>(A, sS, sVx, sVz, tZin, tVz, sd, soff, xs, xe, xb, z0, threadIdx.x >> 3, threadIdx.x & 7);
    if (first) return;
    __syncthreads();  // velocities of columns xb-4 .. xb+21 are in the ring

    // ---- phase S: sigma and r of columns xb .. xb+16 (QS:993-1337); thread = two columns x 4 z
    // (a quarter-warp reads 128 contiguous bytes of a ring row) ----
    {
        const int x = xb + 2 * (2 * warp + (lane >> 4)), zq = lane & 15;
        const int gz0 = z0 + 4 * zq;
        const float am[5] = {a.a[0], a.a[1], a.a[2], a.a[3], a.a[4]};
        // model and memory variable first: their latency is covered by the stencils
        float4 p1v[2], p2v[2], rov[2];
        long long cc[2];
        bool own[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            cc[u] = soff + (long long)(x + u + a.L.gx) * a.L.pitch + a.L.gz + gz0;
            own[u] = x + u < nx && gz0 < nz;
            const long long mi = (long long)min(max(sd.x0 + x + u, 0), a.nx_model - 1) * a.mpitch + gz0;
            p1v[u] = __ldg(reinterpret_cast<const float4*>(a.p1 + mi));
            p2v[u] = __ldg(reinterpret_cast<const float4*>(a.p2 + mi));
            rov[u] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (!EDGE || own[u]) rov[u] = ld4(A.r + cc[u]);
        }
        // d/dx of vx: sum_m a_m [(A(z+1+m) + A(z-m)) - (B(z-m) + B(z+1+m))], d/dz of vz:
        // sum_m a_m [(A(z+1+m) - A(z-m)) + (B(z+1+m) - B(z-m))], A = column x+1+m, B = column x-m.
        // Ring column k (0..10) is x - 4 + k: for output column x it is A with m = k - 5 or B with
        // m = 4 - k, for x + 1 A with m = k - 6 or B with m = 5 - k.  Window w[i] = v(., gz0 - 4 + i):
        // v(z + d) = w[4 + j + d]
        float d1[2][4], d4[2][4];
#pragma unroll
        for (int u = 0; u < 2; u++)
#pragma unroll
            for (int j = 0; j < 4; j++) d1[u][j] = d4[u][j] = 0.0f;
#pragma unroll
        for (int f = 0; f < 2; f++) {
            const float* ring = f == 0 ? sVx : sVz;
#pragma unroll
            for (int k = 0; k < 11; k++) {
                const float* row = ring + ((x - 4 + k) & (VRING - 1)) * VW + 4 + 4 * zq;
                float w[16];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const float4 v = ld4(row + 4 * i);
                    w[4 * i] = v.x; w[4 * i + 1] = v.y; w[4 * i + 2] = v.z; w[4 * i + 3] = v.w;
                }
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    const int kk = k - u;  // position of the ring column relative to output column x + u
                    if (kk < 0 || kk > 9) continue;
                    const int m = kk >= 5 ? kk - 5 : 4 - kk;
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        const float hi = w[5 + j + m], lo = w[4 + j - m];
                        if (f == 0) {  // A: +(hi + lo), B: -(lo + hi)
                            const float sg = kk >= 5 ? am[m] : -am[m];
                            d1[u][j] = fmaf(sg, hi, fmaf(sg, lo, d1[u][j]));
                        } else {       // A and B: +hi - lo
                            d4[u][j] = fmaf(am[m], hi, fmaf(-am[m], lo, d4[u][j]));
                        }
                    }
                }
            }
        }
        const float wav = __ldg(a.wavelets + sd.wav_off + a.step);
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const float4 so = ld4(sS + (x + u - xb) * SW + SH + 4 * zq);  // sigma(t-1) of the cells
            const float4 ro = rov[u], p1 = p1v[u], p2 = p2v[u];
            const float sof[4] = {so.x, so.y, so.z, so.w}, rof[4] = {ro.x, ro.y, ro.z, ro.w};
            const float p1f[4] = {p1.x, p1.y, p1.z, p1.w}, p2f[4] = {p2.x, p2.y, p2.z, p2.w};
            float sn[4], rn[4], e1[4], e4[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                e1[j] = a.hx * d1[u][j];
                e4[j] = a.hz * d4[u][j];
                const float dv = e1[j] + e4[j];
                sn[j] = fmaf(a.dt, fmaf(p1f[j], dv, rof[j]), sof[j]);
                rn[j] = fmaf(a.f_mem, fmaf(p2f[j], dv, rof[j]), rof[j]);
            }
            // source: the Gaussian stamp into strxx (QS:1340-1390); the band kernel adds it again
            // to the split part where the stamp reaches a band cell
            const int bx = x + u - sd.stamp_x0;
            if (bx >= 0 && bx < sd.stamp_w && gz0 + 4 > sd.stamp_z0 && gz0 < sd.stamp_z0 + sd.stamp_h) {
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int bz = gz0 + j - sd.stamp_z0;
                    if (bz >= 0 && bz < sd.stamp_h) {
                        const float g = __ldg(a.stamps + sd.stamp_off + bx * sd.stamp_h + bz);
                        sn[j] += (wav * g * a.dt) / a.dz2;
                    }
                }
            }
            const long long c = cc[u];
            if (EDGE && !own[u]) continue;
            if (!EDGE || gz0 + 4 <= nz) {
                *reinterpret_cast<float4*>(A.s_out + c) = make_float4(sn[0], sn[1], sn[2], sn[3]);
                *reinterpret_cast<float4*>(A.r + c) = make_float4(rn[0], rn[1], rn[2], rn[3]);
                if (EDGE) {
                    *reinterpret_cast<float4*>(A.e1 + c) = make_float4(e1[0], e1[1], e1[2], e1[3]);
                    *reinterpret_cast<float4*>(A.e4 + c) = make_float4(e4[0], e4[1], e4[2], e4[3]);
                }
            } else {
#pragma unroll
                for (int j = 0; j < 4; j++)
                    if (gz0 + j < nz) {
                        A.s_out[c + j] = sn[j];
                        A.r[c + j] = rn[j];
                        A.e1[c + j] = e1[j];
                        A.e4[c + j] = e4[j];
                    }
            }
        }
    }
}

__global__ void __launch_bounds__(kThreads, 4) viscoac2d_fast_kernel(const __grid_constant__ QFastArgs A, int active,
                                                                     QFGeo geo) {
    extern __shared__ __align__(128) unsigned char smem[];
    const QArgs& a = A.q;
    const int tid = threadIdx.x;
    const int slot = blockIdx.x % active;
    const int rest = blockIdx.x / active;
    const int strip = rest % geo.nstrip;
    const int seg = rest / geo.nstrip;
    const int shot = a.slot_to_shot[slot];
    const ShotDev sd = a.shots[shot];
    const int nx = sd.nx, nz = a.nz;
    const int xs = seg * geo.seg;
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (xs >= nx) {
        asm volatile("griddepcontrol.wait;" ::: "memory");
        return;
    }
    const int xe = min(xs + geo.seg, (nx + CH - 1) / CH * CH);
    const int nch = (xe - xs) / CH;
    const int z0 = strip * TZ;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + FL::BAR);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sptr(bars)) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sptr(bars + 1)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // z tables of the strip: in-grid flag and vz sponge (0 outside the grid) per velocity z
    {
        float* tZin = reinterpret_cast<float*>(smem + FL::TAB);
        float* tVz = tZin + NV;
        const float* tb = a.spg;
        const int st = a.spg_stride;
        for (int i = tid; i < NV; i += kThreads) {
            const int z = z0 - VH + i;
            const bool in = z >= 0 && z < nz;
            tZin[i] = in ? 1.0f : 0.0f;
            tVz[i] = in ? sponge_factor(z, nz, a.npz, tb + 2 * st, tb + 3 * st) : 0.0f;  // spgzn, spgzp
        }
    }
    __syncthreads();
    asm volatile("griddepcontrol.wait;" ::: "memory");

    auto issue = [&](int i) {  // sigma box of chunk i - 1 into buffer set i & 1
        const int s = i & 1;
        const int xb = xs + (i - 1) * CH;
        uint64_t* bar = bars + s;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sptr(bar)), "r"(FL::TX) : "memory");
        tma_load_3d(smem + s * FL::SIGB, &A.tm_s, a.L.gz + z0 - SH, a.L.gx + xb, shot, bar);
    };
    if (tid == 0) issue(0);

    // chunks whose velocity columns (xb-11 .. xb+21), z range and stress cells avoid the sponge
    // bands and the grid edges run without tables
    const bool zedge = !(z0 - VH > a.npz && z0 + TZ + VH < nz - a.npz - 1);
    for (int i = 0; i <= nch; i++) {
        const int s = i & 1;
        const unsigned par = (i >> 1) & 1;
        auto bounded_wait = [&]() {
            bool ok = mbar_try_wait(bars + s, par);
            if (!ok) {
                const uint64_t t0 = global_ns();
                while (!(ok = mbar_try_wait(bars + s, par)) && global_ns() - t0 < 1000000000ull) {
                }
            }
            return ok;
        };
        bool done = true;
        if (tid == 0) done = bounded_wait();
        // also: every thread is done with chunk i - 2's sigma box (the set refilled below) and with
        // the ring columns that chunk i - 1's stress phase read
        if (__syncthreads_or(!done)) {
            if (tid == 0) {
                atomicExch(A.err_flag, 1);
                bounded_wait();
            }
            return;
        }
        if (tid != 0) mbar_try_wait(bars + s, par);
        if (tid == 0 && i < nch) issue(i + 1);
        const int xb = xs + (i - 1) * CH;
        const bool xedge = !(xb - 2 * CH > a.npx && xb + 2 * CH < nx - a.npx - 1);
        if (zedge || xedge) chunk_body<true>(A, smem, s, sd, shot, strip, xs, xe, xb, i == 0);
        else chunk_body<false>(A, smem, s, sd, shot, strip, xs, xe, xb, i == 0);
    }
}

// One CTA per (column, active shot): the band cells of the column, then its receivers.
__global__ void __launch_bounds__(kThreads) viscoac2d_band_kernel(const __grid_constant__ QFastArgs A) {
    asm volatile("griddepcontrol.wait;" ::: "memory");  // the step kernel's fields are complete
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const QArgs& a = A.q;
    const int shot = a.slot_to_shot[blockIdx.y];
    const ShotDev& sd = a.shots[shot];
    const int x = blockIdx.x;
    const int nx = sd.nx, nz = a.nz;
    if (x >= nx) return;
    const long long soff = (long long)shot * a.L.shot_stride;
    const long long col = soff + (long long)(x + a.L.gx) * a.L.pitch + a.L.gz;
    const long long mcol = (long long)min(max(sd.x0 + x, 0), a.nx_model - 1) * a.mpitch;
    const float* tb = a.spg;
    const int st = a.spg_stride;
    const bool xband = x <= a.npx || x >= nx - a.npx - 1;
    const float fxs = sponge_factor(x, nx, a.npx, tb + 4 * st, tb + 5 * st);  // spgxn1, spgxp2
    const float wav = __ldg(a.wavelets + sd.wav_off + a.step);
    const int bx = x - sd.stamp_x0;
    const bool stamp_col = bx >= 0 && bx < sd.stamp_w;
    // band z of the column: all of it in an x band, else [0, npz] and [nz - npz - 1, nz)
    const int top = min(a.npz + 1, nz), bot = max(nz - a.npz - 1, top);
    const int n = xband ? nz : top + (nz - bot);
    for (int i = threadIdx.x; i < n; i += kThreads) {
        const int z = xband ? i : (i < top ? i : bot + (i - top));
        const long long c = col + z;
        const float e1 = A.e1[c], e4 = A.e4[c];
        const float p1 = __ldg(a.p1 + mcol + z), p2 = __ldg(a.p2 + mcol + z);
        const float fz = sponge_factor(z, nz, a.npz, tb + 6 * st, tb + 7 * st);  // spgzn1, spgzp2
        const float sx = a.sx[c], sz = a.sz[c], sr = a.sr[c], rx = a.rx[c], rz = a.rz[c], rr = a.rr[c];
        // the reference's split update (QS:993-1020, 1135-1170) and sponges (QS:800-834)
        const float rold = (rx + rz) + rr;
        float sxv = fmaf(a.dt, p1 * e1, sx) * fxs;
        const float szv = fmaf(a.dt, p1 * e4, sz) * fz;
        const float srv = fmaf(a.dt, rold, sr);
        const float rxv = fmaf(a.f_mem, p2 * e1, rx) * fxs;
        const float rzv = fmaf(a.f_mem, p2 * e4, rz) * fz;
        const float rrv = fmaf(a.f_mem, rold, rr);
        float sn = (sxv + szv) + srv;
        if (stamp_col) {  // the source stamp, after the sponge (QS:1340-1390)
            const int bz = z - sd.stamp_z0;
            if (bz >= 0 && bz < sd.stamp_h) {
                const float add = (wav * __ldg(a.stamps + sd.stamp_off + bx * sd.stamp_h + bz) * a.dt) / a.dz2;
                sn += add;
                sxv += add;
            }
        }
        a.sx[c] = sxv; a.sz[c] = szv; a.sr[c] = srv;
        a.rx[c] = rxv; a.rz[c] = rzv; a.rr[c] = rrv;
        A.s_out[c] = sn;
        A.r[c] = (rxv + rzv) + rrv;
    }
    // receivers of the column: strzz = sigma (QM:452-459), from the tiles of its 64-column band
    const int* trp = a.tile_rec_ptr + sd.tile_rec_base + (x / kTileX) * a.L.ntz;
    const int rb = __ldg(trp), re = __ldg(trp + a.L.ntz);
    if (re > rb) {
        __syncthreads();  // this column's band cells are stored
        for (int j = rb + threadIdx.x; j < re; j += kThreads) {
            const int ridx = a.tile_rec_idx[j];
            if (a.rec_x[sd.rec_list + ridx] != x) continue;
            const int rz = a.rec_z[sd.rec_list + ridx];
            a.records[sd.rec_base + (long long)a.step * sd.nrec + ridx] = A.s_out[col + rz];
        }
    }
}

cudaError_t launch_pdl(const void* fn, dim3 grid, int smem, cudaStream_t st, bool pdl, void** args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = pdl ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, fn, args);
}

}  // namespace

cudaError_t viscoac2d_fast_launch(const QFastArgs& A, int active, int seg, int nx_max, cudaStream_t st, bool pdl) {
    if (seg < CH || seg % CH != 0 || A.q.L.tz != TZ || nx_max <= 0) return cudaErrorInvalidValue;
    static bool attr[kMaxDevices] = {};
    if (cudaError_t e = smem_attr_once((const void*)viscoac2d_fast_kernel, FL::BYTES, attr)) return e;
    QFGeo geo;
    geo.seg = seg;
    geo.nstrip = A.q.L.ntz;
    geo.nseg = (A.q.L.ntx * kTileX + seg - 1) / seg;
    QFastArgs a = A;
    void* args[3] = {&a, &active, &geo};
    if (cudaError_t e = launch_pdl((const void*)viscoac2d_fast_kernel, dim3((unsigned)(active * geo.nstrip * geo.nseg)),
                                   FL::BYTES, st, pdl, args))
        return e;
    void* bargs[1] = {&a};
    return launch_pdl((const void*)viscoac2d_band_kernel, dim3((unsigned)nx_max, (unsigned)active), 0, st, pdl, bargs);
}

void viscoac2d_fast_boxes(int box_s[2]) {
    box_s[0] = SW; box_s[1] = SROWS;
}

}  // namespace sfd
