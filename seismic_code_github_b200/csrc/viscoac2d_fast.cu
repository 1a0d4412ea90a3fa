// Fused viscoacoustic step (default mode of SFD_VISCOAC_2D): the rotated-staggered-grid scheme of
// forward/Q_forward/Q_multishot_fd_subroutine_fsbc_zy_rotated.f90 (QS:751-835 and its leaves
// QS:843-1337) with vs = 0, one kernel per time step, FMA contraction.
//
// State.  Everywhere: vx, vz (ping-pong), the merged stress sigma = (sx + sz) + sr (QS strxx,
// ping-pong) and the merged memory variable r = (rx + rz) + rr (in place).  In the sponge bands
// (x <= npx, x >= nx - npx - 1, z <= npz, z >= nz - npz - 1) the split sponge of QS:609-654
// multiplies the x and z parts separately, so there the split parts sx, sz, sr, rx, rz, rr are
// kept as well (in place) and updated in the reference's form; sigma and r are written from
// them.  Away from the bands the parts only ever appear summed, and the kernel updates the sums:
//   sigma += dt (p1 (d1 + d4) + r_old) + source,   r += f (p2 (d1 + d4) + r_old),
// with f = -dt / tau_sigma, p1 = M tau_eps / tau_sigma, p2 = M (tau_eps / tau_sigma - 1).
//
// Staging (as the x-marching acoustic kernel): a CTA owns one 64-wide z strip of one shot over a
// segment of columns and walks down x in chunks of 16 columns with two shared-memory buffer
// sets; the three TMA boxes of chunk c+1 (sigma on columns [xb, xb+25), z halo 16; vx and vz on
// [xb+5, xb+21), z halo 8; no multicast) are issued while chunk c computes.  The stress of
// columns [xb, xb+16) needs the new velocities on [xb-4, xb+21) (the stencil reaches -4 .. +5):
// the chunk computes them on [xb+5, xb+21) and carries the last 9 columns into the next chunk's
// buffer, so each velocity column is computed once per segment (only a z halo of 8 is
// recomputed).  The first chunk of a segment (c = -1) only computes velocities.
// Stencils: QS:843-966, (0.5/d) sum_m a_m t_m over the rotated four-point differences t_m.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "sfd_internal.h"

namespace sfd {
namespace {

constexpr int kThreads = 128;
constexpr int TZ = 64;           // strip width
constexpr int CH = 16;           // chunk columns
constexpr int SH = 16;           // z halo of the staged sigma
constexpr int SW = TZ + 2 * SH;  // 96: sigma row pitch = box width
constexpr int SROWS = CH + 9;    // 25: sigma columns per chunk
constexpr int VH = 8;            // z halo of the recomputed velocities
constexpr int VW = TZ + 2 * VH;  // 80: velocity row pitch = box width
constexpr int CARRY = 9;         // velocity columns carried into the next chunk
constexpr int VROWS = CARRY + CH;  // 25
constexpr int KV = VW / 8;       // 10: velocity values per thread
constexpr int KS = TZ / 8;       // 8: stress values per thread

struct FL {
    // bytes; the TMA destinations (SIG, VX + CARRY rows, VZ + CARRY rows) are 128-byte aligned
    static constexpr int SIG = 0;
    static constexpr int VX = SROWS * SW * 4 + 64;       // 9664
    static constexpr int VZ = VX + VROWS * VW * 4 + 64;  // 17728
    static constexpr int SET = VZ + VROWS * VW * 4;      // 25728
    static constexpr int TAB = 2 * SET;                  // floats: vz sponge [VW], in-grid [VW], stress z sponge' [TZ]
    static constexpr int BAR = TAB + 4 * (2 * VW + TZ);
    static constexpr int BYTES = BAR + 16;
    static constexpr unsigned TX = 4u * (SROWS * SW + 2 * CH * VW);
    static_assert((VX + CARRY * VW * 4) % 128 == 0 && (VZ + CARRY * VW * 4) % 128 == 0, "TMA destinations");
    static_assert(SET % 128 == 0 && BAR % 8 == 0, "buffer sets and barriers stay aligned");
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

__device__ __forceinline__ bool in_band(int c, int n, int np) { return c <= np || c >= n - np - 1; }

struct QFGeo {
    int seg, nseg, nstrip;
};

// Term m of the rotated differences for NOUT consecutive outputs of one thread.  Rows A and B of
// a staged field (A = x + m or x + 1 + m, B = x - 1 - m or x - m); output j's taps are at
// staged columns cb + j + P (a = A, d = B) and cb + j + Q (c = A, b = B) with (P, Q) = (m, -1-m)
// for sigma (QS FLAG 0) and (1+m, -m) for the velocities (FLAG 1); cb is even.
//   tX = ((a - b) + c) - d,  tZ = ((a - b) - c) + d;  acc = a_m t (m = 0) or fma(a_m, t, acc)
template <int NOUT, int P, int Q, bool FIRST, bool WX, bool WZ>
__device__ __forceinline__ void rsg_term(const float* rowA, const float* rowB, int cb, float am, float* accx,
                                         float* accz) {
    constexpr int LO = (Q < P ? Q : P);
    constexpr int HI = NOUT - 1 + (Q < P ? P : Q);
    constexpr int L = LO >= 0 ? (LO & ~1) : -((1 - LO) & ~1);  // even, <= LO
    constexpr int NW = ((HI - L + 2) & ~1);                     // even count covering [L, HI]
    float wa[NW], wb[NW];
#pragma unroll
    for (int i = 0; i < NW; i += 2) {
        const float2 va = *reinterpret_cast<const float2*>(rowA + cb + L + i);
        const float2 vb = *reinterpret_cast<const float2*>(rowB + cb + L + i);
        wa[i] = va.x; wa[i + 1] = va.y;
        wb[i] = vb.x; wb[i + 1] = vb.y;
    }
#pragma unroll
    for (int j = 0; j < NOUT; j++) {
        const float a = wa[j + P - L], c = wa[j + Q - L], b = wb[j + Q - L], d = wb[j + P - L];
        const float ab = a - b;
        if (WX) {
            const float t = (ab + c) - d;
            accx[j] = FIRST ? am * t : fmaf(am, t, accx[j]);
        }
        if (WZ) {
            const float t = (ab - c) + d;
            accz[j] = FIRST ? am * t : fmaf(am, t, accz[j]);
        }
    }
}

// all five terms of one rotated stencil (rows 5 + r + m and 4 + r - m of a staged field of pitch W)
template <int NOUT, int FLAG, int W, bool WX, bool WZ>
__device__ __forceinline__ void rsg_all(const float* s, int r, int cb, const float* coef, float* accx, float* accz) {
#define SFD_TERM(M, FIRST)                                                                              \
    rsg_term<NOUT, (FLAG == 0 ? (M) : 1 + (M)), (FLAG == 0 ? -1 - (M) : -(M)), FIRST, WX, WZ>(          \
        s + (5 + r + (M)) * W, s + (4 + r - (M)) * W, cb, coef[M], accx, accz)
    SFD_TERM(0, true);
    SFD_TERM(1, false);
    SFD_TERM(2, false);
    SFD_TERM(3, false);
    SFD_TERM(4, false);
#undef SFD_TERM
}

template <bool EDGE>
__device__ __forceinline__ void chunk_body(const QFastArgs& A, unsigned char* smem, int set, const ShotDev& sd,
                                           int shot, int strip, int xs, int xe, int xb, bool first) {
    const QArgs& a = A.q;
    const float* sS = reinterpret_cast<const float*>(smem + set * FL::SET + FL::SIG);
    float* sVx = reinterpret_cast<float*>(smem + set * FL::SET + FL::VX);
    float* sVz = reinterpret_cast<float*>(smem + set * FL::SET + FL::VZ);
    float* nVx = reinterpret_cast<float*>(smem + (set ^ 1) * FL::SET + FL::VX);
    float* nVz = reinterpret_cast<float*>(smem + (set ^ 1) * FL::SET + FL::VZ);
    const float* tVz = reinterpret_cast<const float*>(smem + FL::TAB);  // vz sponge per velocity z (0 outside the grid)
    const float* tZin = tVz + VW;                                        // 1 / 0: velocity z inside the grid
    const float* tSz = tZin + VW;                                        // z sponge' per stress z
    const int tid = threadIdx.x;
    const int nx = sd.nx, nz = a.nz;
    const int z0 = strip * TZ;
    const long long soff = (long long)shot * a.L.shot_stride;
    auto cell = [&](int x, int z) -> long long { return soff + (long long)(x + a.L.gx) * a.L.pitch + a.L.gz + z; };
    auto midx = [&](int x, int z) -> long long {
        return (long long)min(max(sd.x0 + x, 0), a.nx_model - 1) * a.mpitch + z;
    };
    const float* tb = a.spg;
    const int st = a.spg_stride;

    // ---- velocities on columns xb+5 .. xb+21, z0-8 .. z0+72 (QS:843-990); thread = column x 10 z ----
    {
        const int r = tid >> 3, zb = tid & 7;
        const int x = xb + 5 + r;
        const int cb = 8 + KV * zb;  // sigma column of the first output
        // buoyancy first: its latency is covered by the stencil
        float2 bu[KV / 2];
        {
            const long long mi = midx(x, z0 - VH + KV * zb);
#pragma unroll
            for (int j = 0; j < KV; j += 2) bu[j / 2] = __ldg(reinterpret_cast<const float2*>(a.busg + mi + j));
        }
        float d1[KV], d2[KV];
        rsg_all<KV, 0, SW, true, true>(sS, r, cb, a.a, d1, d2);
        const bool xin = x >= 0 && x < nx;
        float fx = 1.0f;
        if (EDGE) fx = xin ? sponge_factor(x, nx, a.npx, tb + 0 * st, tb + 1 * st) : 0.0f;
        float* vxr = sVx + (CARRY + r) * VW + KV * zb;
        float* vzr = sVz + (CARRY + r) * VW + KV * zb;
#pragma unroll
        for (int j = 0; j < KV; j += 2) {
            float2 vx = *reinterpret_cast<const float2*>(vxr + j);
            float2 vz = *reinterpret_cast<const float2*>(vzr + j);
            const float db0 = a.dt * bu[j / 2].x, db1 = a.dt * bu[j / 2].y;
            vx.x = fmaf(db0, a.hx * d1[j], vx.x);
            vx.y = fmaf(db1, a.hx * d1[j + 1], vx.y);
            vz.x = fmaf(db0, a.hz * d2[j], vz.x);
            vz.y = fmaf(db1, a.hz * d2[j + 1], vz.y);
            if (EDGE) {  // sponges (QS:609-654: vx in x, vz in z), and zero outside the grid
                const float xi = xin ? 1.0f : 0.0f;
                vx.x *= fx * tZin[KV * zb + j];
                vx.y *= fx * tZin[KV * zb + j + 1];
                vz.x *= xi * tVz[KV * zb + j];
                vz.y *= xi * tVz[KV * zb + j + 1];
            }
            *reinterpret_cast<float2*>(vxr + j) = vx;
            *reinterpret_cast<float2*>(vzr + j) = vz;
            // the next chunk needs the last CARRY columns
            if (CARRY + r >= CH) {
                *reinterpret_cast<float2*>(nVx + (CARRY + r - CH) * VW + KV * zb + j) = vx;
                *reinterpret_cast<float2*>(nVz + (CARRY + r - CH) * VW + KV * zb + j) = vz;
            }
        }
        // store the columns this segment owns (the grid part of the strip)
        if (x >= xs && x < xe && xin) {
#pragma unroll
            for (int j = 0; j < KV; j++) {
                const int gz = z0 - VH + KV * zb + j;
                if (gz >= z0 && gz < z0 + TZ && gz < nz) {
                    const long long c = cell(x, gz);
                    A.vx_out[c] = vxr[j];
                    A.vz_out[c] = vzr[j];
                }
            }
        }
    }
    if (first) return;
    __syncthreads();  // velocities of columns xb-4 .. xb+21 are staged

    // ---- stress and memory variable on columns xb .. xb+16 (QS:993-1337); thread = column x 8 z ----
    const int step = a.step;
    {
        const int r = tid >> 3, zq = tid & 7;
        const int x = xb + r;
        const int gz0 = z0 + KS * zq;
        const int cb = VH + KS * zq;  // velocity column of the first output
        // model and (away from the bands) the merged state first: their latency is covered by the
        // stencils
        const long long mi = midx(x, gz0);
        const long long c0 = cell(x, gz0);
        float4 p1v[KS / 4], p2v[KS / 4], sov[KS / 4], rov[KS / 4];
#pragma unroll
        for (int h = 0; h < KS / 4; h++) {
            p1v[h] = __ldg(reinterpret_cast<const float4*>(a.p1 + mi + 4 * h));
            p2v[h] = __ldg(reinterpret_cast<const float4*>(a.p2 + mi + 4 * h));
            if (!EDGE) {
                sov[h] = *reinterpret_cast<const float4*>(A.s_in + c0 + 4 * h);
                rov[h] = *reinterpret_cast<const float4*>(A.r + c0 + 4 * h);
            }
        }
        float d1[KS], d4[KS];
        rsg_all<KS, 1, VW, true, false>(sVx, r, cb, a.a, d1, nullptr);
        rsg_all<KS, 1, VW, false, true>(sVz, r, cb, a.a, nullptr, d4);
        float p1[KS], p2[KS];
#pragma unroll
        for (int h = 0; h < KS / 4; h++) {
            p1[4 * h] = p1v[h].x; p1[4 * h + 1] = p1v[h].y; p1[4 * h + 2] = p1v[h].z; p1[4 * h + 3] = p1v[h].w;
            p2[4 * h] = p2v[h].x; p2[4 * h + 1] = p2v[h].y; p2[4 * h + 2] = p2v[h].z; p2[4 * h + 3] = p2v[h].w;
        }
        const float wav = __ldg(a.wavelets + sd.wav_off + step);
        const bool xin = x < nx;
        const bool xband = EDGE && in_band(x, nx, a.npx);
        const float fxs = EDGE ? sponge_factor(x, nx, a.npx, tb + 4 * st, tb + 5 * st) : 1.0f;
        // the strip's outputs: contiguous cells c0 .. c0 + 7 of column x
        float sn[KS], rn[KS];
        if (!EDGE) {
            float so[KS], ro[KS];
#pragma unroll
            for (int h = 0; h < KS / 4; h++) {
                const float4 s4 = sov[h], r4 = rov[h];
                so[4 * h] = s4.x; so[4 * h + 1] = s4.y; so[4 * h + 2] = s4.z; so[4 * h + 3] = s4.w;
                ro[4 * h] = r4.x; ro[4 * h + 1] = r4.y; ro[4 * h + 2] = r4.z; ro[4 * h + 3] = r4.w;
            }
#pragma unroll
            for (int j = 0; j < KS; j++) {
                const float dv = fmaf(a.hx, d1[j], a.hz * d4[j]);
                sn[j] = fmaf(a.dt, fmaf(p1[j], dv, ro[j]), so[j]);
                rn[j] = fmaf(a.f_mem, fmaf(p2[j], dv, ro[j]), ro[j]);
            }
        } else {
#pragma unroll
            for (int j = 0; j < KS; j++) {
                const int gz = gz0 + j;
                sn[j] = rn[j] = 0.0f;
                if (!xin || gz >= nz) continue;
                const long long c = c0 + j;
                const float e1 = a.hx * d1[j], e4 = a.hz * d4[j];
                if (xband || in_band(gz, nz, a.npz)) {
                    // the reference's split update (QS:993-1020, 1135-1170), sponges (QS:800-834)
                    const float rold = (A.q.rx[c] + A.q.rz[c]) + A.q.rr[c];
                    const float fz = tSz[KS * zq + j];
                    const float sxv = fmaf(a.dt, p1[j] * e1, A.q.sx[c]) * fxs;
                    const float szv = fmaf(a.dt, p1[j] * e4, A.q.sz[c]) * fz;
                    const float srv = fmaf(a.dt, rold, A.q.sr[c]);
                    const float rxv = fmaf(a.f_mem, p2[j] * e1, A.q.rx[c]) * fxs;
                    const float rzv = fmaf(a.f_mem, p2[j] * e4, A.q.rz[c]) * fz;
                    const float rrv = fmaf(a.f_mem, rold, A.q.rr[c]);
                    A.q.sx[c] = sxv; A.q.sz[c] = szv; A.q.sr[c] = srv;
                    A.q.rx[c] = rxv; A.q.rz[c] = rzv; A.q.rr[c] = rrv;
                    sn[j] = (sxv + szv) + srv;
                    rn[j] = (rxv + rzv) + rrv;
                } else {
                    const float ro = A.r[c];
                    const float dv = e1 + e4;
                    sn[j] = fmaf(a.dt, fmaf(p1[j], dv, ro), A.s_in[c]);
                    rn[j] = fmaf(a.f_mem, fmaf(p2[j], dv, ro), ro);
                }
            }
        }
        // source: the Gaussian stamp into strxx (QS:1340-1390), after the sponge
        const int bx = x - sd.stamp_x0;
        if (bx >= 0 && bx < sd.stamp_w && gz0 + KS > sd.stamp_z0 && gz0 < sd.stamp_z0 + sd.stamp_h) {
#pragma unroll
            for (int j = 0; j < KS; j++) {
                const int bz = gz0 + j - sd.stamp_z0;
                if (bz >= 0 && bz < sd.stamp_h && xin && gz0 + j < nz) {
                    const float g = __ldg(a.stamps + sd.stamp_off + bx * sd.stamp_h + bz);
                    const float add = (wav * g * a.dt) / a.dz2;
                    sn[j] += add;
                    if (EDGE && (xband || in_band(gz0 + j, nz, a.npz))) A.q.sx[c0 + j] += add;
                }
            }
        }
        if (xin) {
            if (gz0 + KS <= nz) {
#pragma unroll
                for (int h = 0; h < KS; h += 4) {
                    *reinterpret_cast<float4*>(A.s_out + c0 + h) = make_float4(sn[h], sn[h + 1], sn[h + 2], sn[h + 3]);
                    *reinterpret_cast<float4*>(A.r + c0 + h) = make_float4(rn[h], rn[h + 1], rn[h + 2], rn[h + 3]);
                }
            } else {
#pragma unroll
                for (int j = 0; j < KS; j++)
                    if (gz0 + j < nz) {
                        A.s_out[c0 + j] = sn[j];
                        A.r[c0 + j] = rn[j];
                    }
            }
        }
    }
    // ---- receivers: strzz = sigma (QM:452-459) ----
    const int* trp = a.tile_rec_ptr + sd.tile_rec_base + (xb / kTileX) * a.L.ntz + strip;
    const int rb = __ldg(trp), re = __ldg(trp + 1);
    if (re > rb) {
        __syncthreads();  // this chunk's sigma is in global memory (written by this CTA)
        for (int j = rb + tid; j < re; j += kThreads) {
            const int ridx = a.tile_rec_idx[j];
            const int rx = a.rec_x[sd.rec_list + ridx];
            if (rx < xb || rx >= xb + CH) continue;
            const int rz = a.rec_z[sd.rec_list + ridx];
            a.records[sd.rec_base + (long long)step * sd.nrec + ridx] = A.s_out[cell(rx, rz)];
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
    if (xs >= nx) return;
    const int xe = min(xs + geo.seg, (nx + CH - 1) / CH * CH);
    const int nch = (xe - xs) / CH;
    const int z0 = strip * TZ;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + FL::BAR);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sptr(bars)) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sptr(bars + 1)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // z tables of the strip: vz sponge (0 outside the grid) and in-grid flag per velocity z,
    // z sponge' per stress z
    {
        float* tVz = reinterpret_cast<float*>(smem + FL::TAB);
        float* tZin = tVz + VW;
        float* tSz = tZin + VW;
        const float* tb = a.spg;
        const int st = a.spg_stride;
        for (int i = tid; i < VW; i += kThreads) {
            const int z = z0 - VH + i;
            const bool in = z >= 0 && z < nz;
            tVz[i] = in ? sponge_factor(z, nz, a.npz, tb + 2 * st, tb + 3 * st) : 0.0f;
            tZin[i] = in ? 1.0f : 0.0f;
        }
        for (int i = tid; i < TZ; i += kThreads) {
            const int z = z0 + i;
            tSz[i] = z < nz ? sponge_factor(z, nz, a.npz, tb + 6 * st, tb + 7 * st) : 1.0f;
        }
    }
    __syncthreads();
    asm volatile("griddepcontrol.wait;" ::: "memory");

    auto issue = [&](int i) {
        const int s = i & 1;
        const int xb = xs + (i - 1) * CH;
        unsigned char* base = smem + s * FL::SET;
        uint64_t* bar = bars + s;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sptr(bar)), "r"(FL::TX) : "memory");
        const int gx = a.L.gx, gz = a.L.gz;
        tma_load_3d(base + FL::SIG, &A.tm_s, gz + z0 - SH, gx + xb, shot, bar);
        tma_load_3d(base + FL::VX + CARRY * VW * 4, &A.tm_vx, gz + z0 - VH, gx + xb + 5, shot, bar);
        tma_load_3d(base + FL::VZ + CARRY * VW * 4, &A.tm_vz, gz + z0 - VH, gx + xb + 5, shot, bar);
    };
    if (tid == 0) issue(0);

    // chunks whose velocity columns (xb-4 .. xb+21), z range and stress cells avoid the sponge
    // bands and the grid edges run the merged update without tables
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
        const bool xedge = !(xb - 4 > a.npx && xb + CH + 5 < nx - a.npx - 1);
        if (zedge || xedge) chunk_body<true>(A, smem, s, sd, shot, strip, xs, xe, xb, i == 0);
        else chunk_body<false>(A, smem, s, sd, shot, strip, xs, xe, xb, i == 0);
    }
}

}  // namespace

cudaError_t viscoac2d_fast_launch(const QFastArgs& A, int active, int seg, cudaStream_t st, bool pdl) {
    if (seg < CH || seg % CH != 0 || A.q.L.tz != TZ) return cudaErrorInvalidValue;
    static bool attr[kMaxDevices] = {};
    if (cudaError_t e = smem_attr_once((const void*)viscoac2d_fast_kernel, FL::BYTES, attr)) return e;
    QFGeo geo;
    geo.seg = seg;
    geo.nstrip = A.q.L.ntz;
    geo.nseg = (A.q.L.ntx * kTileX + seg - 1) / seg;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(active * geo.nstrip * geo.nseg));
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = FL::BYTES;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = pdl ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, viscoac2d_fast_kernel, A, active, geo);
}

void viscoac2d_fast_boxes(int box_s[2], int box_v[2]) {
    box_s[0] = SW; box_s[1] = SROWS;
    box_v[0] = VW; box_v[1] = CH;
}

}  // namespace sfd
