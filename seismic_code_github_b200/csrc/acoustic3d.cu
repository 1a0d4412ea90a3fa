// 3-D velocity-pressure staggered-grid step for sm_100a (no reference counterpart: the 2-D
// scheme of forward/Acoustic_FD_by_ss/src/Acoustic_1order_FD.cpp:237-380 with a y axis).
//
// One launch per time step does the whole update of every active shot: Vx, Vy, Vz from P, then
// P from the new velocities, the sponge, and the frozen rim.  Each CTA owns a 32 x 32 (y, z)
// column of one shot and marches along x, the slowest axis of the [x][y][z] layout:
//   * P, Vy and Vz of plane s arrive by three TMA bulk-tensor loads (cp.async.bulk.tensor.4d,
//     no multicast) into one of two shared-memory stages while plane s-1 is computed; the boxes
//     carry the y / z halos and read zeros outside the grid (exact tensor-map extents), so the
//     field buffers need no ghost cells.  The wait on the stage's mbarrier is bounded.
//   * the x-derivatives need no halo exchange: each thread keeps its own points' P of planes
//     s .. s+2R-1 and the new Vx of planes s-R .. s+R-1 in register queues (coalesced float4
//     loads one plane ahead), so P is read from DRAM once per step and Vx never leaves the CTA
//     until it is stored;
//   * Vy and Vz are recomputed on the R-wide y / z halo of the column (from the staged P) so
//     that the pressure update needs no second pass.
// Velocities are stored before the sponge multiply (the next step applies it on load); the
// pressure update uses the undamped new velocities and P is stored damped -- the order of
// AFD:289-340.  The source (before the step) and the receivers (after it) are separate small
// launches.
//
// The same kernel runs the adjoint step (ADJ = true), the 2-D recurrence of adjoint2d.cu with a
// y axis: the P slot holds nu = M K a Q, the velocity slots X, Y, Z; the velocity phases form
// X' = X + rd S+ nu and stage B M X' (B = dt / (d den)) for the pressure phase, which forms
// nu' = M a K (nu / K + sum_a S-a(B M X_a')) and the imaging sum g += nu D_k; the velocity
// outputs are a M X'.  Every model factor is needed at the updated point only.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <algorithm>
#include <type_traits>

#include "sfd_internal.h"

namespace sfd {
namespace {

constexpr int kThreads = 256;
constexpr int TY = kTile3Y, TZ = kTile3Z;

__host__ __device__ constexpr int r4(int v) { return (v + 3) & ~3; }
__host__ __device__ constexpr int r32(int v) { return (v + 31) & ~31; }
__host__ __device__ constexpr int cdiv4(int v) { return (v + 3) / 4; }

template <int R>
struct K3 {
    static constexpr int RQ = r4(R);          // z halo of the Vz region (16-byte TMA coordinate)
    static constexpr int HY = 2 * R;          // y halo of the staged pressure
    static constexpr int HZ = r4(RQ + R);     // z halo of the staged pressure
    static constexpr int PY = TY + 2 * HY, PZ = TZ + 2 * HZ;
    static constexpr int VYR = TY + 2 * R;    // rows of the Vy region (y0-R .. y0+TY+R-1)
    static constexpr int VZW = TZ + 2 * RQ;   // columns of the Vz region (z0-RQ .. z0+TZ+RQ-1)
    static constexpr int NVY2 = (VYR / 2) * (TZ / 4);  // Vy tasks: two rows x one float4
    static constexpr int NVZ = TY * (VZW / 4);         // Vz tasks: one float4
    // Vz tasks: threads from NVY2 on take up to three, the rest go to the last Vy threads
    static constexpr int HVZ = kThreads - NVY2;
    static constexpr int RVZ = NVZ > 3 * HVZ ? NVZ - 3 * HVZ : 0;
    // Vz window: P columns 4u + B4 .. of the staged box, BR = first needed column - B4
    static constexpr int B = HZ - RQ + 1 - R, B4 = B & ~3, BR = B - B4, NFZ = cdiv4(BR + 2 * R + 3);
    // d/dz of the new Vz at the own points: columns zr + D4 .. of the Vz region
    static constexpr int D = RQ - R, D4 = D & ~3, DR = D - D4, NFD = cdiv4(DR + 2 * R + 3);
    static constexpr int NQ = 2 * R;  // planes held in the P (registers) and Vx (shared) queues
    // shared layout (floats): two TMA stages {P box, Vy box, Vz box}, two buffers of the new
    // Vy / Vz regions, the per-thread Vx ring, the sponge tables and two mbarriers
    static constexpr int OFF_VY = r32(PY * PZ);
    static constexpr int OFF_VZ = OFF_VY + r32(VYR * TZ);
    static constexpr int STAGE = r32(OFF_VZ + TY * VZW);
    static constexpr int NB_NZ = r32(VYR * TZ);           // within a new-velocity buffer
    static constexpr int NBUF = NB_NZ + r32(TY * VZW);
    static constexpr int OFF_NB = 2 * STAGE;
    static constexpr int OFF_VQ = OFF_NB + 2 * NBUF;           // [NQ][kThreads] float4
    static constexpr int NTAB = VYR * VZW;                      // positions of the CTA's region
    static constexpr int OFF_FA = OFF_VQ + NQ * kThreads * 4;  // y/z damping factor per position
    static constexpr int OFF_FK = OFF_FA + r32(NTAB);          // 1 where y and z are updated, else 0
    static constexpr int OFF_BAR = OFF_FK + r32(NTAB);
    static constexpr int SMEM_FLOATS = OFF_BAR + 4;
    static constexpr unsigned TX_BYTES = 4u * (PY * PZ + VYR * TZ + TY * VZW);
    static_assert(TY * TZ / 4 == kThreads, "one float4 of own points per thread");
    static_assert(VYR % 2 == 0 && NVY2 <= kThreads && RVZ <= NVY2, "halo task split");
    static_assert(B >= 0 && D >= 0, "halo windows start inside the staged boxes");
    static_assert(SMEM_FLOATS * 4 <= 227 * 1024, "shared memory of one CTA");
};

__device__ __forceinline__ unsigned sptr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tma_load_4d(float* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(sptr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(sptr(bar))
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

// bounded wait on an mbarrier phase: about one second of wall time, then give up
__device__ __forceinline__ bool bounded_wait(uint64_t* bar, unsigned parity) {
    bool done = mbar_try_wait(bar, parity);
    if (!done) {
        const uint64_t t0 = global_ns();
        while (!(done = mbar_try_wait(bar, parity)) && global_ns() - t0 < 1000000000ull) {
        }
    }
    return done;
}

__device__ __forceinline__ float4 ld4s(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4s(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float2 lo2(const float4& v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4& v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ float4 cat4(float2 a, float2 b) { return make_float4(a.x, a.y, b.x, b.y); }
__device__ __forceinline__ float2 bc2(float c) { return make_float2(c, c); }
__device__ __forceinline__ float4 mul4(float4 a, float4 b) {
    return cat4(__fmul2_rn(lo2(a), lo2(b)), __fmul2_rn(hi2(a), hi2(b)));
}

// Every stencil sum is written with explicit roundings in one fixed order, so a halo value a CTA
// recomputes is bit-identical to the value the owning CTA stores.
// sum_m C_m (hi_m - lo_m), m = 1..R, one point (z stencils) ...
struct Acc {
    float v;
    __device__ __forceinline__ void add(int m, float c, float hi, float lo) {
        const float d = __fsub_rn(hi, lo);
        v = (m == 1) ? __fmul_rn(c, d) : __fmaf_rn(c, d, v);
    }
};
// ... and two neighbouring z points per paired FP32 instruction (x and y stencils); cc = (c, c)
struct Acc2 {
    float2 v;
    __device__ __forceinline__ void add(int m, float2 cc, float2 hi, float2 lo) {
        const float2 d = __ffma2_rn(lo, make_float2(-1.0f, -1.0f), hi);  // hi - lo, one rounding
        v = (m == 1) ? __fmul2_rn(cc, d) : __ffma2_rn(cc, d, v);
    }
};

// Taper factor of a position along one axis: the sponge value if d lies in the pad, else 1.
__device__ __forceinline__ float axis_taper(const Acou3DArgs& a, int d, int n, bool* in_pad) {
    const int q = d < a.pml ? a.pml - d - 1 : (d >= n - a.pml ? d - n + a.pml : -1);
    *in_pad = q >= 0;
    return (q >= 0 && q < a.pml) ? a.sponge[q] : 1.0f;
}

// new velocity on four points: (v_old * f - b * sum) * k, with f the damping factors of the old
// value and k the rim mask (EDGE), else v_old - b * sum
template <bool EDGE>
__device__ __forceinline__ float4 vel_update(float4 vo, float4 b, float2 s01, float2 s23, float4 f, float4 k) {
    float2 v01 = lo2(vo), v23 = hi2(vo);
    if (EDGE) {
        v01 = __fmul2_rn(v01, lo2(f));
        v23 = __fmul2_rn(v23, hi2(f));
    }
    v01 = __ffma2_rn(make_float2(-b.x, -b.y), s01, v01);
    v23 = __ffma2_rn(make_float2(-b.z, -b.w), s23, v23);
    if (EDGE) {
        v01 = __fmul2_rn(v01, lo2(k));
        v23 = __fmul2_rn(v23, hi2(k));
    }
    return cat4(v01, v23);
}

// adjoint velocity update on four points: staged B M (X + rd sum), output a M (X + rd sum)
template <bool EDGE, bool VARDEN>
__device__ __forceinline__ float4 adj_vel(float4 xo, float rd, float2 s01, float2 s23, float4 f, float4 k, float4 b,
                                          float4* out) {
    float2 v01 = __ffma2_rn(make_float2(rd, rd), s01, lo2(xo));
    float2 v23 = __ffma2_rn(make_float2(rd, rd), s23, hi2(xo));
    if (EDGE) {
        v01 = __fmul2_rn(v01, lo2(k));
        v23 = __fmul2_rn(v23, hi2(k));
        *out = cat4(__fmul2_rn(v01, lo2(f)), __fmul2_rn(v23, hi2(f)));
    } else {
        *out = cat4(v01, v23);
    }
    if (VARDEN) {
        v01 = __fmul2_rn(v01, lo2(b));
        v23 = __fmul2_rn(v23, hi2(b));
    }
    return cat4(v01, v23);
}

template <int R, bool VARDEN, bool ADJ>
__global__ void __launch_bounds__(kThreads, 2) acoustic3d_step_kernel(const __grid_constant__ Acou3DArgs a) {
    using K = K3<R>;
    extern __shared__ __align__(128) float smem[];
    const int tid = threadIdx.x;
    const Layout3D& L = a.L;
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const int shot = a.slot_to_shot[blockIdx.y];
    const int ty_i = blockIdx.x / L.ntz;
    const int y0 = ty_i * TY, z0 = (blockIdx.x - ty_i * L.ntz) * TZ;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + K::OFF_BAR);
    float4* sVq = reinterpret_cast<float4*>(smem + K::OFF_VQ) + tid;  // this thread's Vx ring
    const float* sFA = smem + K::OFF_FA;
    const float* sFK = smem + K::OFF_FK;

    // own points: one row y, four consecutive z
    const int yl = tid >> 3, zr = (tid & 7) * 4;
    const int yo = y0 + yl, zo = z0 + zr;
    const bool own_ok = yo < ny && zo < L.pitch;  // the float4 lies inside the allocation
    const long long own_off = (long long)min(yo, ny - 1) * L.pitch + min(zo, L.pitch - 4);
    const int slab = a.slab_by_slot ? (int)blockIdx.y : shot;
    const long long shot_off = (long long)slab * L.shot_stride;
    const float* p_in = a.p_in + shot_off;
    const float* vx_in = a.vx_in + shot_off;

    // Damping factor (y pad wins over z pad; 1 outside the pads) and rim mask of every position
    // (y0-R+i, z0-RQ+j) of the CTA's region; the x pad is applied per plane.
    for (int i = tid; i < K::NTAB; i += kThreads) {
        const int y = y0 - R + i / K::VZW, z = z0 - K::RQ + i % K::VZW;
        bool py, pz;
        const float fy = axis_taper(a, y, ny, &py);
        const float fz = axis_taper(a, z, nz, &pz);
        smem[K::OFF_FA + i] = py ? fy : fz;
        smem[K::OFF_FK + i] = (y >= R && y < ny - R && z >= R && z < nz - R) ? 1.0f : 0.0f;
    }
    const int E = a.pml > R ? a.pml : R;
    const bool yz_int = y0 - R >= E && y0 + TY + R <= ny - E && z0 - K::RQ >= E && z0 + TZ + K::RQ <= nz - E;
    const float bxc = a.dtdx / a.den_c, byc = a.dtdy / a.den_c, bzc = a.dtdz / a.den_c, kc = a.den_c * a.dt;
    float2 cc[R];
#pragma unroll
    for (int m = 0; m < R; m++) cc[m] = bc2(a.coef[m]);

    auto ld_own = [&](const float* base, int x) -> float4 {
        if (!own_ok || x >= nx) return make_float4(0.f, 0.f, 0.f, 0.f);
        return __ldg(reinterpret_cast<const float4*>(base + (long long)x * L.xstride + own_off));
    };
    auto ld_model = [&](const float* base, int x, int y, int z) -> float4 {
        y = min(max(y, 0), ny - 1);
        z = min(max(z, 0), L.pitch - 4);
        return __ldg(reinterpret_cast<const float4*>(base + (long long)x * L.xstride + (long long)y * L.pitch + z));
    };
    auto issue = [&](int s) {
        const int stg = s & 1;
        float* st = smem + stg * K::STAGE;
        uint64_t* bar = bars + stg;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sptr(bar)), "r"(K::TX_BYTES)
                     : "memory");
        tma_load_4d(st, &a.tm_p, z0 - K::HZ, y0 - K::HY, s, slab, bar);
        tma_load_4d(st + K::OFF_VY, &a.tm_vy, z0, y0 - R, s, slab, bar);
        tma_load_4d(st + K::OFF_VZ, &a.tm_vz, z0 - K::RQ, y0, s, slab, bar);
    };

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sptr(bars)) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sptr(bars + 1)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // iteration s: new Vx on plane s+R-1 (own points), then, for s >= R, new Vy / Vz on plane s
    // (column + halo) and new P on plane s.  Planes below R and from nx-R on are the frozen rim.
    // The boxes of plane s+2 are requested once every thread is done with those of plane s.
    const int s_begin = 1, s_end = nx - R;
    if (tid == 0) {
        issue(s_begin);
        if (s_begin + 1 < s_end) issue(s_begin + 1);
    }
    float4 Pq[K::NQ];
#pragma unroll
    for (int j = 0; j < K::NQ; j++) {
        Pq[j] = ld_own(p_in, s_begin + j);
        sVq[j * kThreads] = make_float4(0.f, 0.f, 0.f, 0.f);  // planes below R: rim
    }
    float4 Pn = ld_own(p_in, s_begin + K::NQ);
    float4 Vxo = ld_own(vx_in, s_begin + R - 1);
    float4 vpn = ld_own(a.vp, s_begin);
    unsigned phase = 0;

    for (int s = s_begin; s < s_end; s++) {
        const int stg = s & 1;
        const bool got = bounded_wait(bars + stg, (phase >> stg) & 1u);
        phase ^= 1u << stg;
        const float* st = smem + stg * K::STAGE;
        float* nby = smem + K::OFF_NB + stg * K::NBUF;  // new Vy region of this plane
        float* nbz = nby + K::NB_NZ;                     // new Vz region of this plane
        // adjoint: D_k and the imaging sum of the own points of plane s, requested before the
        // velocity phases so that their latency is covered
        float4 adk = make_float4(0.f, 0.f, 0.f, 0.f), agk = adk;
        if (ADJ && s >= R && own_ok) {
            const long long pofs = shot_off + (long long)s * L.xstride + own_off;
            adk = __ldg(reinterpret_cast<const float4*>(a.adj_div + pofs));
            agk = *reinterpret_cast<const float4*>(a.adj_g + pofs);
        }
        // the loads of the next plane's own values are issued as soon as this plane's are used
        const int xv = s + R - 1;  // plane of this iteration's new Vx
        const bool edge = !yz_int || !(s >= E && xv < nx - E);
        bool xpad_s, xpad_v;
        const float fx_s = axis_taper(a, s, nx, &xpad_s);
        const float fx_v = axis_taper(a, xv, nx, &xpad_v);
        const float kx_s = (s >= R && s < nx - R) ? 1.0f : 0.0f, kx_v = (xv >= R && xv < nx - R) ? 1.0f : 0.0f;
        // damping factors and masks of four points of the region at table index i, plane s
        auto edge_f = [&](int i, bool xpad, float fx) {
            return xpad ? make_float4(fx, fx, fx, fx) : ld4s(sFA + i);
        };
        auto edge_k = [&](int i, float kx) {
            const float4 k = ld4s(sFK + i);
            return make_float4(k.x * kx, k.y * kx, k.z * kx, k.w * kx);
        };

        if (s >= R) {
            const long long plane_off = shot_off + (long long)s * L.xstride;
            // ---- new Vy on the Vy region: rows y0-R .. y0+TY+R-1, two rows x float4 per task ----
            if (tid < K::NVY2) {
                const int r0 = (tid >> 3) * 2, zt = (tid & 7) * 4;
                // P rows r0+R+1-m (lo, row r0) ... r0+R+1+m (hi, row r0+1), center row shared
                const float* pc = st + K::HZ + zt;
                Acc2 a01, a23, b01, b23;  // rows r0 and r0+1
                float4 hi_a = ld4s(pc + (r0 + R + 1) * K::PZ), lo_b = hi_a;
#pragma unroll
                for (int m = 1; m <= R; m++) {
                    const float4 lo_a = ld4s(pc + (r0 + R + 1 - m) * K::PZ);
                    const float4 hi_b = ld4s(pc + (r0 + R + 1 + m) * K::PZ);
                    a01.add(m, cc[m - 1], lo2(hi_a), lo2(lo_a));
                    a23.add(m, cc[m - 1], hi2(hi_a), hi2(lo_a));
                    b01.add(m, cc[m - 1], lo2(hi_b), lo2(lo_b));
                    b23.add(m, cc[m - 1], hi2(hi_b), hi2(lo_b));
                    hi_a = hi_b;
                    lo_b = lo_a;
                }
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int row = r0 + h;
                    float4 b = make_float4(byc, byc, byc, byc);
                    if (VARDEN) {
                        const float4 d = ld_model(a.den, s, y0 - R + row, z0 + zt);
                        b = make_float4(a.dtdy / d.x, a.dtdy / d.y, a.dtdy / d.z, a.dtdy / d.w);
                    }
                    const float4 vo = ld4s(st + K::OFF_VY + row * TZ + zt);
                    const float2 s01 = h ? b01.v : a01.v, s23 = h ? b23.v : a23.v;
                    float4 vn, vout;
                    const int i = row * K::VZW + K::RQ + zt;
                    if (ADJ) {
                        if (edge)
                            vn = adj_vel<true, VARDEN>(vo, a.rdy, s01, s23, edge_f(i, xpad_s, fx_s), edge_k(i, kx_s), b,
                                                       &vout);
                        else
                            vn = adj_vel<false, VARDEN>(vo, a.rdy, s01, s23, vo, vo, b, &vout);
                    } else {
                        if (edge)
                            vn = vel_update<true>(vo, b, s01, s23, edge_f(i, xpad_s, fx_s), edge_k(i, kx_s));
                        else
                            vn = vel_update<false>(vo, b, s01, s23, vo, vo);
                        vout = vn;
                    }
                    st4s(nby + row * TZ + zt, vn);
                    const int y = y0 - R + row;
                    if (row >= R && row < R + TY && y < ny && z0 + zt < L.pitch)
                        st4s(a.vy_out + plane_off + (long long)y * L.pitch + z0 + zt, vout);
                }
            }
            // ---- new Vz on the Vz region: rows y0 .. y0+TY-1, z0-RQ .. z0+TZ+RQ-1 ----
            auto vz_task = [&](int t) {
                const int row = t / (K::VZW / 4), u = t % (K::VZW / 4);
                float w[4 * K::NFZ];
#pragma unroll
                for (int f = 0; f < K::NFZ; f++) {
                    const float4 v = ld4s(st + (row + K::HY) * K::PZ + 4 * u + K::B4 + 4 * f);
                    w[4 * f] = v.x; w[4 * f + 1] = v.y; w[4 * f + 2] = v.z; w[4 * f + 3] = v.w;
                }
                Acc acc[4];
#pragma unroll
                for (int c = 0; c < 4; c++)
#pragma unroll
                    for (int m = 1; m <= R; m++)
                        acc[c].add(m, a.coef[m - 1], w[K::BR + R - 1 + c + m], w[K::BR + R + c - m]);
                float4 b = make_float4(bzc, bzc, bzc, bzc);
                if (VARDEN) {
                    const float4 d = ld_model(a.den, s, y0 + row, z0 - K::RQ + 4 * u);
                    b = make_float4(a.dtdz / d.x, a.dtdz / d.y, a.dtdz / d.z, a.dtdz / d.w);
                }
                const float4 vo = ld4s(st + K::OFF_VZ + row * K::VZW + 4 * u);
                const float2 s01 = make_float2(acc[0].v, acc[1].v), s23 = make_float2(acc[2].v, acc[3].v);
                float4 vn, vout;
                const int i = (row + R) * K::VZW + 4 * u;
                if (ADJ) {
                    if (edge)
                        vn = adj_vel<true, VARDEN>(vo, a.rdz, s01, s23, edge_f(i, xpad_s, fx_s), edge_k(i, kx_s), b,
                                                   &vout);
                    else
                        vn = adj_vel<false, VARDEN>(vo, a.rdz, s01, s23, vo, vo, b, &vout);
                } else {
                    if (edge)
                        vn = vel_update<true>(vo, b, s01, s23, edge_f(i, xpad_s, fx_s), edge_k(i, kx_s));
                    else
                        vn = vel_update<false>(vo, b, s01, s23, vo, vo);
                    vout = vn;
                }
                st4s(nbz + row * K::VZW + 4 * u, vn);
                const int y = y0 + row, z = z0 - K::RQ + 4 * u;
                if (4 * u >= K::RQ && 4 * u < K::RQ + TZ && y < ny && z < L.pitch)
                    st4s(a.vz_out + plane_off + (long long)y * L.pitch + z, vout);
            };
            if (tid >= K::NVY2) {
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    const int j = (tid - K::NVY2) + k * K::HVZ;
                    if (j < K::NVZ) vz_task(j);
                }
            } else if (K::RVZ > 0 && tid >= K::NVY2 - K::RVZ) {
                vz_task(3 * K::HVZ + tid - (K::NVY2 - K::RVZ));
            }
        }
        const int io = (yl + R) * K::VZW + K::RQ + zr;  // table index of the own points
        // ---- new Vx on plane xv (own points, P from the register queue) ----
        {
            Acc2 s01, s23;
#pragma unroll
            for (int m = 1; m <= R; m++) {
                s01.add(m, cc[m - 1], lo2(Pq[R - 1 + m]), lo2(Pq[R - m]));
                s23.add(m, cc[m - 1], hi2(Pq[R - 1 + m]), hi2(Pq[R - m]));
            }
            float4 b = make_float4(bxc, bxc, bxc, bxc);
            if (VARDEN) {
                const float4 d = ld_model(a.den, xv, yo, zo);
                b = make_float4(a.dtdx / d.x, a.dtdx / d.y, a.dtdx / d.z, a.dtdx / d.w);
            }
            float4 vn, vout;
            if (ADJ) {
                vn = edge ? adj_vel<true, VARDEN>(Vxo, a.rdx, s01.v, s23.v, edge_f(io, xpad_v, fx_v), edge_k(io, kx_v),
                                                  b, &vout)
                          : adj_vel<false, VARDEN>(Vxo, a.rdx, s01.v, s23.v, Vxo, Vxo, b, &vout);
            } else {
                vn = edge ? vel_update<true>(Vxo, b, s01.v, s23.v, edge_f(io, xpad_v, fx_v), edge_k(io, kx_v))
                          : vel_update<false>(Vxo, b, s01.v, s23.v, Vxo, Vxo);
                vout = vn;
            }
            Vxo = ld_own(vx_in, s + R);
            if (own_ok) st4s(a.vx_out + shot_off + (long long)xv * L.xstride + own_off, vout);
            sVq[((unsigned)xv % K::NQ) * kThreads] = vn;
        }
        // every thread is done with this stage and with the new-velocity buffer of plane s-1
        if (__syncthreads_or(!got)) {
            if (tid == 0) {
                atomicExch(a.err_flag, 1);
                // let the copies still in flight land before the CTA's shared memory is released
                bounded_wait(bars + stg, ((phase >> stg) & 1u) ^ 1u);
                if (s + 1 < s_end) bounded_wait(bars + (stg ^ 1), (phase >> (stg ^ 1)) & 1u);
            }
            return;
        }
        if (tid == 0 && s + 2 < s_end) issue(s + 2);
        if (s >= R) {
            // ---- new P on plane s (own points) ----
            float wz[4 * K::NFD];
#pragma unroll
            for (int f = 0; f < K::NFD; f++) {
                const float4 v = ld4s(nbz + yl * K::VZW + zr + K::D4 + 4 * f);
                wz[4 * f] = v.x; wz[4 * f + 1] = v.y; wz[4 * f + 2] = v.z; wz[4 * f + 3] = v.w;
            }
            Acc2 ax01, ax23, ay01, ay23;
#pragma unroll
            for (int m = 1; m <= R; m++) {
                const float4 xhi = sVq[((unsigned)(s + m - 1) % K::NQ) * kThreads];
                const float4 xlo = sVq[((unsigned)(s - m) % K::NQ) * kThreads];
                ax01.add(m, cc[m - 1], lo2(xhi), lo2(xlo));
                ax23.add(m, cc[m - 1], hi2(xhi), hi2(xlo));
                const float4 yhi = ld4s(nby + (yl + R + m - 1) * TZ + zr);
                const float4 ylo = ld4s(nby + (yl + R - m) * TZ + zr);
                ay01.add(m, cc[m - 1], lo2(yhi), lo2(ylo));
                ay23.add(m, cc[m - 1], hi2(yhi), hi2(ylo));
            }
            Acc az[4];
#pragma unroll
            for (int c = 0; c < 4; c++)
#pragma unroll
                for (int m = 1; m <= R; m++)
                    az[c].add(m, a.coef[m - 1], wz[K::DR + R + c + m - 1], wz[K::DR + R + c - m]);
            // div = ((Sx / dx) + Sy / dy) + Sz / dz, then P = P - (den dt vp vp) div; the adjoint
            // weighs the sums by B (constant density) instead
            const float2 rdx = bc2(ADJ ? a.adj_c[0] : a.rdx), rdy = bc2(ADJ ? a.adj_c[1] : a.rdy),
                         rdz = bc2(ADJ ? a.adj_c[2] : a.rdz);
            float2 d01 = __fmul2_rn(ax01.v, rdx), d23 = __fmul2_rn(ax23.v, rdx);
            d01 = __ffma2_rn(ay01.v, rdy, d01);
            d23 = __ffma2_rn(ay23.v, rdy, d23);
            d01 = __ffma2_rn(make_float2(az[0].v, az[1].v), rdz, d01);
            d23 = __ffma2_rn(make_float2(az[2].v, az[3].v), rdz, d23);
            float4 kk;
            if (VARDEN) {
                const float4 d = ld_model(a.den, s, yo, zo);
                kk = make_float4(d.x * a.dt, d.y * a.dt, d.z * a.dt, d.w * a.dt);
            } else {
                kk = make_float4(kc, kc, kc, kc);
            }
            const float2 k01 = __fmul2_rn(__fmul2_rn(lo2(kk), lo2(vpn)), lo2(vpn));
            const float2 k23 = __fmul2_rn(__fmul2_rn(hi2(kk), hi2(vpn)), hi2(vpn));
            const long long pofs = shot_off + (long long)s * L.xstride + own_off;
            if (ADJ) {
                // bracket = nu / K + sum (= M a Q_old + ...), nu' = M a K bracket, g += nu D_k
                const float4 po = Pq[0];
                const float2 b01 = __fadd2_rn(d01, make_float2(__fdividef(po.x, k01.x), __fdividef(po.y, k01.y)));
                const float2 b23 = __fadd2_rn(d23, make_float2(__fdividef(po.z, k23.x), __fdividef(po.w, k23.y)));
                float4 pn = cat4(__fmul2_rn(b01, k01), __fmul2_rn(b23, k23));
                if (edge) pn = mul4(mul4(pn, edge_f(io, xpad_s, fx_s)), edge_k(io, kx_s));
                if (own_ok) {
                    st4s(a.p_out + pofs, pn);
                    const float4 dk = adk;
                    float4 g = agk;
                    g = make_float4(fmaf(po.x, dk.x, g.x), fmaf(po.y, dk.y, g.y), fmaf(po.z, dk.z, g.z),
                                    fmaf(po.w, dk.w, g.w));
                    st4s(a.adj_g + pofs, g);
                    const ShotDev& sd = a.shots[shot];
                    if (s == sd.sx && yo == sd.sy && sd.sz >= zo && sd.sz < zo + 4) {
                        const float bq[4] = {b01.x, b01.y, b23.x, b23.y};
                        for (int c = 0; c < 4; c++)
                            if (sd.sz == zo + c) a.adj_lam[(long long)shot * a.nt_max + a.step] = bq[c];
                    }
                }
            } else {
                float4 pn = cat4(__ffma2_rn(make_float2(-k01.x, -k01.y), d01, lo2(Pq[0])),
                                 __ffma2_rn(make_float2(-k23.x, -k23.y), d23, hi2(Pq[0])));
                if (edge) pn = mul4(mul4(pn, edge_f(io, xpad_s, fx_s)), edge_k(io, kx_s));
                if (own_ok) {
                    st4s(a.p_out + pofs, pn);
                    if (a.div_out) st4s(a.div_out + pofs, cat4(d01, d23));  // recomputation for the adjoint
                }
            }
        }
        vpn = ld_own(a.vp, s + 1);
#pragma unroll
        for (int j = 0; j + 1 < K::NQ; j++) Pq[j] = Pq[j + 1];
        Pq[K::NQ - 1] = Pn;
        Pn = ld_own(p_in, s + K::NQ + 1);
    }
}

__global__ void inject3d_kernel(float* p, Layout3D L, const ShotDev* shots, const int* slot_to_shot, int active,
                                const float* wavelets, int step, int by_slot) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= active) return;
    const ShotDev sd = shots[slot_to_shot[i]];
    if (step >= sd.nt) return;
    const long long o = (long long)(by_slot ? i : slot_to_shot[i]) * L.shot_stride + (long long)sd.sx * L.xstride +
                        (long long)sd.sy * L.pitch + sd.sz;
    // P[s] -= (dt * den * vp) * w[k], AFD:250 (separate roundings)
    p[o] = __fsub_rn(p[o], __fmul_rn(sd.inj_scale, wavelets[sd.wav_off + step]));
}

__global__ void gather3d_kernel(const float* p, Layout3D L, const ShotDev* shots, const int* slot_to_shot,
                                const int* rec_x, const int* rec_y, const int* rec_z, float* records, int step,
                                int by_slot) {
    const int shot = slot_to_shot[blockIdx.y];
    const ShotDev sd = shots[shot];
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= sd.nrec || step >= sd.nt) return;
    const int q = sd.rec_list + r;
    const long long o = (long long)(by_slot ? (int)blockIdx.y : shot) * L.shot_stride + (long long)rec_x[q] * L.xstride +
                        (long long)rec_y[q] * L.pitch + rec_z[q];
    records[sd.rec_base + (long long)step * sd.nrec + r] = p[o];
}

// adjoint of the receiver gather: nu[receiver] += M a K res[step] (M = 1 where the step updates P)
__global__ void adj_inject3d_kernel(float* nu, const Acou3DArgs a, const int* rec_x, const int* rec_y,
                                    const int* rec_z, const float* res) {
    const int shot = a.slot_to_shot[blockIdx.y];
    const ShotDev sd = a.shots[shot];
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= sd.nrec || a.step >= sd.nt) return;
    const Layout3D& L = a.L;
    const int q = sd.rec_list + r;
    const int x = rec_x[q], y = rec_y[q], z = rec_z[q];
    if (x < a.adj_radius || x >= L.nx - a.adj_radius || y < a.adj_radius || y >= L.ny - a.adj_radius ||
        z < a.adj_radius || z >= L.nz - a.adj_radius)
        return;
    const long long m = (long long)x * L.xstride + (long long)y * L.pitch + z;
    const float vp = a.vp[m], den = a.den ? a.den[m] : a.den_c;
    bool pad;
    float f = axis_taper(a, x, L.nx, &pad);
    if (!pad) {
        f = axis_taper(a, y, L.ny, &pad);
        if (!pad) f = axis_taper(a, z, L.nz, &pad);
    }
    const float v = res[sd.rec_base + (long long)a.step * sd.nrec + r];
    const int slab = a.slab_by_slot ? (int)blockIdx.y : shot;
    atomicAdd(nu + (long long)slab * L.shot_stride + m, den * a.dt * vp * vp * f * v);
}

__global__ void reduce3d_kernel(const double* __restrict__ acc, int nslab, Layout3D L, const float* __restrict__ vp,
                                double* grad) {
    const long long n = (long long)L.nx * L.ny * L.nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long xy = i / L.nz;
        const int z = (int)(i - xy * L.nz);
        const long long m = xy * L.pitch + z;
        double s = 0.0;
        for (int k = 0; k < nslab; k++) s += acc[(long long)k * L.shot_stride + m];
        grad[i] += -2.0 * s / (double)vp[m];
    }
}

template <int R, bool VARDEN, bool ADJ>
cudaError_t launch_t(const Acou3DArgs& a, int active, cudaStream_t st) {
    const size_t smem = sizeof(float) * K3<R>::SMEM_FLOATS;
    auto k = acoustic3d_step_kernel<R, VARDEN, ADJ>;
    static bool attr[kMaxDevices] = {};
    if (cudaError_t e = smem_attr_once((const void*)k, (int)smem, attr)) return e;
    const dim3 grid(a.L.nty * a.L.ntz, active);
    k<<<grid, kThreads, smem, st>>>(a);
    return cudaGetLastError();
}

template <int R>
void boxes_t(int bp[2], int bvy[2], int bvz[2]) {
    using K = K3<R>;
    bp[0] = K::PZ; bp[1] = K::PY;
    bvy[0] = TZ; bvy[1] = K::VYR;
    bvz[0] = K::VZW; bvz[1] = TY;
}

}  // namespace

template <int R>
cudaError_t launch_r(const Acou3DArgs& a, int active, bool varden, bool adj, cudaStream_t st) {
    if (adj) return varden ? launch_t<R, true, true>(a, active, st) : launch_t<R, false, true>(a, active, st);
    return varden ? launch_t<R, true, false>(a, active, st) : launch_t<R, false, false>(a, active, st);
}

cudaError_t acoustic3d_launch_step(int radius, const Acou3DArgs& a, int active, bool varden, cudaStream_t st,
                                   bool adj) {
    if (active <= 0) return cudaSuccess;
    switch (radius) {
    case 2: return launch_r<2>(a, active, varden, adj, st);
    case 4: return launch_r<4>(a, active, varden, adj, st);
    default: return cudaErrorInvalidValue;
    }
}

bool acoustic3d_boxes(int radius, int bp[2], int bvy[2], int bvz[2]) {
    switch (radius) {
    case 2: boxes_t<2>(bp, bvy, bvz); return true;
    case 4: boxes_t<4>(bp, bvy, bvz); return true;
    default: return false;
    }
}

cudaError_t acoustic3d_launch_inject(float* p, const Layout3D& L, const ShotDev* shots, const int* slot_to_shot,
                                     int active, const float* wavelets, int step, cudaStream_t st, int slab_by_slot) {
    if (active <= 0) return cudaSuccess;
    inject3d_kernel<<<(active + 63) / 64, 64, 0, st>>>(p, L, shots, slot_to_shot, active, wavelets, step,
                                                       slab_by_slot);
    return cudaGetLastError();
}

cudaError_t acoustic3d_launch_gather(const float* p, const Layout3D& L, const ShotDev* shots,
                                     const int* slot_to_shot, int active, const int* rec_x, const int* rec_y,
                                     const int* rec_z, float* records, int nrec_max, int step, cudaStream_t st,
                                     int slab_by_slot) {
    if (active <= 0 || nrec_max <= 0) return cudaSuccess;
    const dim3 grid((nrec_max + 255) / 256, active);
    gather3d_kernel<<<grid, 256, 0, st>>>(p, L, shots, slot_to_shot, rec_x, rec_y, rec_z, records, step,
                                          slab_by_slot);
    return cudaGetLastError();
}

cudaError_t acoustic3d_launch_adj_inject(float* nu, const Acou3DArgs& a, const int* rec_x, const int* rec_y,
                                         const int* rec_z, const float* res, int active, int nrec_max,
                                         cudaStream_t st) {
    if (active <= 0 || nrec_max <= 0) return cudaSuccess;
    const dim3 grid((nrec_max + 255) / 256, active);
    adj_inject3d_kernel<<<grid, 256, 0, st>>>(nu, a, rec_x, rec_y, rec_z, res);
    return cudaGetLastError();
}

cudaError_t acoustic3d_launch_gradient_reduce(const double* acc, int nslab, const Layout3D& L, const float* vp,
                                              double* grad, cudaStream_t st) {
    const long long n = (long long)L.nx * L.ny * L.nz;
    const int grid = (int)std::min<long long>((n + 255) / 256, 148 * 16);
    reduce3d_kernel<<<grid, 256, 0, st>>>(acc, nslab, L, vp, grad);
    return cudaGetLastError();
}

}  // namespace sfd
