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
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

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
    static constexpr int VYR = TY + 2 * R;    // rows of the Vy region
    static constexpr int VZW = TZ + 2 * RQ;   // width of the Vz region
    static constexpr int NVY = VYR * (TZ / 4);  // float4 tasks of the Vy region
    static constexpr int NVZ = TY * (VZW / 4);  // float4 tasks of the Vz region
    // Vz window: P columns 4u + B4 .. of the staged box, BR = first needed column - B4
    static constexpr int B = HZ - RQ + 1 - R, B4 = B & ~3, BR = B - B4, NFZ = cdiv4(BR + 2 * R + 3);
    // d/dz of the new Vz at the own points: columns zr + D4 .. of the Vz region
    static constexpr int D = RQ - R, D4 = D & ~3, DR = D - D4, NFD = cdiv4(DR + 2 * R + 3);
    static constexpr int OFF_VY = r32(PY * PZ);
    static constexpr int OFF_VZ = OFF_VY + r32(VYR * TZ);
    static constexpr int STAGE = r32(OFF_VZ + TY * VZW);
    static constexpr int OFF_NY = 2 * STAGE;              // new Vy on the Vy region
    static constexpr int OFF_NZ = OFF_NY + r32(VYR * TZ);  // new Vz on the Vz region
    static constexpr int OFF_TY = OFF_NZ + r32(TY * VZW);  // float2 per Vy-region row
    static constexpr int OFF_TZ = OFF_TY + r32(2 * VYR);    // float2 per Vz-region column
    static constexpr int OFF_BAR = OFF_TZ + r32(2 * VZW);
    static constexpr int SMEM_FLOATS = OFF_BAR + 4;
    static constexpr unsigned TX_BYTES = 4u * (PY * PZ + VYR * TZ + TY * VZW);
    static constexpr int NQ = 2 * R;  // planes held in each register queue
    static_assert(TY * TZ / 4 == kThreads, "one float4 of own points per thread");
    static_assert(NVY <= 2 * kThreads && NVZ <= 2 * kThreads, "at most two halo tasks per thread");
    static_assert(B >= 0 && D >= 0, "halo windows start inside the staged boxes");
    static_assert(VYR <= 64 && VZW <= kThreads - 64, "table fill: one thread per entry");
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

__device__ __forceinline__ float c4(const float4& v, int i) {
    return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}
__device__ __forceinline__ float& r4f(float4& v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w)); }
__device__ __forceinline__ float4 ld4s(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4s(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }

// Every stencil sum is written with explicit roundings in one fixed order, so a halo value a CTA
// recomputes is bit-identical to the value the owning CTA stores.
// sum_m C_m (hi_m - lo_m), m = 1..R
template <int R>
struct Acc {
    float v;
    __device__ __forceinline__ void add(int m, float c, float hi, float lo) {
        const float d = __fsub_rn(hi, lo);
        v = (m == 1) ? __fmul_rn(c, d) : __fmaf_rn(c, d, v);
    }
};

// Taper factor of a position along one axis: the sponge value if d lies in the pad, else 1.
__device__ __forceinline__ float axis_taper(const Acou3DArgs& a, int d, int n, bool* in_pad) {
    const int q = d < a.pml ? a.pml - d - 1 : (d >= n - a.pml ? d - n + a.pml : -1);
    *in_pad = q >= 0;
    return (q >= 0 && q < a.pml) ? a.sponge[q] : 1.0f;
}
// y/z part of the sponge (the y factor wins over the z factor where the pads overlap)
__device__ __forceinline__ float taper_yz(const Acou3DArgs& a, int y, int z) {
    bool py, pz;
    const float fy = axis_taper(a, y, a.L.ny, &py);
    const float fz = axis_taper(a, z, a.L.nz, &pz);
    return py ? fy : fz;
}
template <int R>
__device__ __forceinline__ bool in_yz(const Acou3DArgs& a, int y, int z) {
    return y >= R && y < a.L.ny - R && z >= R && z < a.L.nz - R;
}

template <int R, bool VARDEN>
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
    float* sNY = smem + K::OFF_NY;
    float* sNZ = smem + K::OFF_NZ;

    // own points: one row y, four consecutive z
    const int yl = tid >> 3, zr = (tid & 7) * 4;
    const int yo = y0 + yl, zo = z0 + zr;
    const bool own_ok = yo < ny && zo < L.pitch;  // the float4 lies inside the allocation
    const long long own_off = (long long)min(yo, ny - 1) * L.pitch + min(zo, L.pitch - 4);
    const long long shot_off = (long long)shot * L.shot_stride;
    const float* p_in = a.p_in + shot_off;
    const float* vx_in = a.vx_in + shot_off;

    // Per-CTA tables of the y / z sponge factors and rim masks (read on edge iterations only):
    // tY[i] for y = y0 - R + i: (taper if y lies in a y pad else -1, 1 if R <= y < ny-R else 0),
    // tZ[i] for z = z0 - RQ + i: (taper or 1, 1 if R <= z < nz-R else 0).
    float2* tY = reinterpret_cast<float2*>(smem + K::OFF_TY);
    float2* tZ = reinterpret_cast<float2*>(smem + K::OFF_TZ);
    if (tid < K::VYR) {
        const int y = y0 - R + tid;
        bool py;
        const float f = axis_taper(a, y, ny, &py);
        tY[tid] = make_float2(py ? f : -1.0f, (y >= R && y < ny - R) ? 1.0f : 0.0f);
    } else if (tid >= 64 && tid < 64 + K::VZW) {
        const int z = z0 - K::RQ + (tid - 64);
        bool pz;
        const float f = axis_taper(a, z, nz, &pz);
        tZ[tid - 64] = make_float2(f, (z >= R && z < nz - R) ? 1.0f : 0.0f);
    }
    const int E = a.pml > R ? a.pml : R;
    const bool yz_int = y0 - R >= E && y0 + TY + R <= ny - E && z0 - K::RQ >= E && z0 + TZ + K::RQ <= nz - E;
    const float bxc = a.dtdx / a.den_c, byc = a.dtdy / a.den_c, bzc = a.dtdz / a.den_c, kc = a.den_c * a.dt;

    auto own_tables = [&](float2& fy, float2* fz) {
        fy = tY[yl + R];
        const float4 z01 = ld4s(reinterpret_cast<const float*>(tZ + K::RQ + zr));
        const float4 z23 = ld4s(reinterpret_cast<const float*>(tZ + K::RQ + zr + 2));
        fz[0] = make_float2(z01.x, z01.y); fz[1] = make_float2(z01.z, z01.w);
        fz[2] = make_float2(z23.x, z23.y); fz[3] = make_float2(z23.z, z23.w);
    };
    auto ld_own = [&](const float* base, int x) -> float4 {
        if (!own_ok || x >= nx) return make_float4(0.f, 0.f, 0.f, 0.f);
        return __ldg(reinterpret_cast<const float4*>(base + (long long)x * L.xstride + own_off));
    };
    auto ld_model = [&](const float* base, int x, int y, int z) -> float4 {
        y = min(max(y, 0), ny - 1);
        z = min(max(z, 0), L.pitch - 4);
        return __ldg(reinterpret_cast<const float4*>(base + (long long)x * L.xstride + (long long)y * L.pitch + z));
    };
    auto issue = [&](int s, int stg) {
        float* st = smem + stg * K::STAGE;
        uint64_t* bar = bars + stg;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sptr(bar)), "r"(K::TX_BYTES)
                     : "memory");
        tma_load_4d(st, &a.tm_p, z0 - K::HZ, y0 - K::HY, s, shot, bar);
        tma_load_4d(st + K::OFF_VY, &a.tm_vy, z0, y0 - R, s, shot, bar);
        tma_load_4d(st + K::OFF_VZ, &a.tm_vz, z0 - K::RQ, y0, s, shot, bar);
    };

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sptr(bars)) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sptr(bars + 1)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // iteration s: new Vx on plane s+R-1 (own points), then, for s >= R, new Vy / Vz on plane s
    // (column + halo) and new P on plane s.  Planes below R and from nx-R on are the frozen rim.
    const int s_begin = 1, s_end = nx - R;
    if (tid == 0) issue(s_begin, s_begin & 1);

    float4 Pq[K::NQ], Vq[K::NQ];
#pragma unroll
    for (int j = 0; j < K::NQ; j++) {
        Pq[j] = ld_own(p_in, s_begin + j);
        Vq[j] = make_float4(0.f, 0.f, 0.f, 0.f);  // planes s_begin - R .. R - 1: rim
    }
    float4 Pn = ld_own(p_in, s_begin + K::NQ);
    float4 Vxo = ld_own(vx_in, s_begin + R - 1);
    float4 vpn = ld_own(a.vp - 0, s_begin);
    unsigned phase = 0;

    for (int s = s_begin; s < s_end; s++) {
        const int stg = s & 1;
        const unsigned par = (phase >> stg) & 1u;
        bool done = mbar_try_wait(bars + stg, par);
        if (!done) {
            const uint64_t t0 = global_ns();
            while (!(done = mbar_try_wait(bars + stg, par)) && global_ns() - t0 < 1000000000ull) {
            }
        }
        if (__syncthreads_or(!done)) {  // also: every thread is done with iteration s-1
            if (tid == 0) atomicExch(a.err_flag, 1);
            return;
        }
        phase ^= 1u << stg;
        if (tid == 0 && s + 1 < s_end) issue(s + 1, stg ^ 1);
        const float* st = smem + stg * K::STAGE;
        const float4 vxo = Vxo, vpc = vpn, pnext = Pn;
        Pn = ld_own(p_in, s + K::NQ + 1);
        Vxo = ld_own(vx_in, s + R);
        vpn = ld_own(a.vp, s + 1);

        const int xv = s + R - 1;  // plane of this iteration's new Vx
        const bool edge = !yz_int || !(s >= E && xv < nx - E);
        // x-plane factors (uniform): sponge value where the plane lies in an x pad, rim masks
        bool xpad_s, xpad_v;
        const float fx_s = axis_taper(a, s, nx, &xpad_s);
        const float fx_v = axis_taper(a, xv, nx, &xpad_v);
        const bool xin_s = s >= R && s < nx - R, xin_v = xv >= R && xv < nx - R;

        if (s >= R) {
            // ---- new Vy on the Vy region: rows y0-R .. y0+TY+R-1, float4 along z ----
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const int t = tid + k * kThreads;
                if (k == 1 && t >= K::NVY) break;
                const int row = t >> 3, zt = (t & 7) * 4;
                float4 sum;
                {
                    Acc<R> acc[4];
#pragma unroll
                    for (int m = 1; m <= R; m++) {
                        const float4 hi = ld4s(st + (row + R + m) * K::PZ + K::HZ + zt);
                        const float4 lo = ld4s(st + (row + R - m + 1) * K::PZ + K::HZ + zt);
#pragma unroll
                        for (int c = 0; c < 4; c++) acc[c].add(m, a.coef[m - 1], c4(hi, c), c4(lo, c));
                    }
                    sum = make_float4(acc[0].v, acc[1].v, acc[2].v, acc[3].v);
                }
                float4 vo = ld4s(st + K::OFF_VY + row * TZ + zt);
                float4 b = make_float4(byc, byc, byc, byc);
                if (VARDEN) {
                    const float4 d = ld_model(a.den, s, y0 - R + row, z0 + zt);
                    b = make_float4(a.dtdy / d.x, a.dtdy / d.y, a.dtdy / d.z, a.dtdy / d.w);
                }
                float4 vn;
                float2 fy, fz[4];
                if (edge) {
                    fy = tY[row];
                    const float4 z01 = ld4s(reinterpret_cast<const float*>(tZ + K::RQ + zt));
                    const float4 z23 = ld4s(reinterpret_cast<const float*>(tZ + K::RQ + zt + 2));
                    fz[0] = make_float2(z01.x, z01.y); fz[1] = make_float2(z01.z, z01.w);
                    fz[2] = make_float2(z23.x, z23.y); fz[3] = make_float2(z23.z, z23.w);
                }
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    float v = c4(vo, c);
                    if (edge) v = __fmul_rn(v, xpad_s ? fx_s : (fy.x >= 0.0f ? fy.x : fz[c].x));
                    v = __fmaf_rn(-c4(b, c), c4(sum, c), v);
                    if (edge) v = (xin_s && fy.y != 0.0f && fz[c].y != 0.0f) ? v : 0.0f;
                    r4f(vn, c) = v;
                }
                st4s(sNY + row * TZ + zt, vn);
            }
            // ---- new Vz on the Vz region: rows y0 .. y0+TY-1, z0-RQ .. z0+TZ+RQ-1 ----
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const int t = tid + k * kThreads;
                if (k == 1 && t >= K::NVZ) break;
                const int row = t / (K::VZW / 4), u = t % (K::VZW / 4);
                float w[4 * K::NFZ];
#pragma unroll
                for (int f = 0; f < K::NFZ; f++) {
                    const float4 v = ld4s(st + (row + K::HY) * K::PZ + 4 * u + K::B4 + 4 * f);
                    w[4 * f] = v.x; w[4 * f + 1] = v.y; w[4 * f + 2] = v.z; w[4 * f + 3] = v.w;
                }
                float4 vo = ld4s(st + K::OFF_VZ + row * K::VZW + 4 * u);
                float4 b = make_float4(bzc, bzc, bzc, bzc);
                if (VARDEN) {
                    const float4 d = ld_model(a.den, s, y0 + row, z0 - K::RQ + 4 * u);
                    b = make_float4(a.dtdz / d.x, a.dtdz / d.y, a.dtdz / d.z, a.dtdz / d.w);
                }
                float4 vn;
                float2 fy, fz[4];
                if (edge) {
                    fy = tY[row + R];
                    const float4 z01 = ld4s(reinterpret_cast<const float*>(tZ + 4 * u));
                    const float4 z23 = ld4s(reinterpret_cast<const float*>(tZ + 4 * u + 2));
                    fz[0] = make_float2(z01.x, z01.y); fz[1] = make_float2(z01.z, z01.w);
                    fz[2] = make_float2(z23.x, z23.y); fz[3] = make_float2(z23.z, z23.w);
                }
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    Acc<R> acc;
#pragma unroll
                    for (int m = 1; m <= R; m++)
                        acc.add(m, a.coef[m - 1], w[K::BR + R - 1 + c + m], w[K::BR + R + c - m]);
                    float v = c4(vo, c);
                    if (edge) v = __fmul_rn(v, xpad_s ? fx_s : (fy.x >= 0.0f ? fy.x : fz[c].x));
                    v = __fmaf_rn(-c4(b, c), acc.v, v);
                    if (edge) v = (xin_s && fy.y != 0.0f && fz[c].y != 0.0f) ? v : 0.0f;
                    r4f(vn, c) = v;
                }
                st4s(sNZ + row * K::VZW + 4 * u, vn);
            }
        }
        // ---- new Vx on plane xv (own points, register queue) ----
        {
            float4 b = make_float4(bxc, bxc, bxc, bxc);
            if (VARDEN) {
                const float4 d = ld_model(a.den, xv, yo, zo);
                b = make_float4(a.dtdx / d.x, a.dtdx / d.y, a.dtdx / d.z, a.dtdx / d.w);
            }
            float4 vn;
            float2 fy, fz[4];
            if (edge) own_tables(fy, fz);
#pragma unroll
            for (int c = 0; c < 4; c++) {
                Acc<R> acc;
#pragma unroll
                for (int m = 1; m <= R; m++) acc.add(m, a.coef[m - 1], c4(Pq[R - 1 + m], c), c4(Pq[R - m], c));
                float v = c4(vxo, c);
                if (edge) v = __fmul_rn(v, xpad_v ? fx_v : (fy.x >= 0.0f ? fy.x : fz[c].x));
                v = __fmaf_rn(-c4(b, c), acc.v, v);
                if (edge) v = (xin_v && fy.y != 0.0f && fz[c].y != 0.0f) ? v : 0.0f;
                r4f(vn, c) = v;
            }
            if (own_ok) st4s(a.vx_out + shot_off + (long long)xv * L.xstride + own_off, vn);
#pragma unroll
            for (int j = 0; j + 1 < K::NQ; j++) Vq[j] = Vq[j + 1];
            Vq[K::NQ - 1] = vn;
        }
        __syncthreads();  // new Vy / Vz of the column and its halo are in shared memory
        if (s >= R) {
            // ---- new P on plane s (own points) ----
            float wz[4 * K::NFD];
#pragma unroll
            for (int f = 0; f < K::NFD; f++) {
                const float4 v = ld4s(sNZ + yl * K::VZW + zr + K::D4 + 4 * f);
                wz[4 * f] = v.x; wz[4 * f + 1] = v.y; wz[4 * f + 2] = v.z; wz[4 * f + 3] = v.w;
            }
            Acc<R> ay_acc[4];
#pragma unroll
            for (int m = 1; m <= R; m++) {
                const float4 hi = ld4s(sNY + (yl + R + m - 1) * TZ + zr);
                const float4 lo = ld4s(sNY + (yl + R - m) * TZ + zr);
#pragma unroll
                for (int c = 0; c < 4; c++) ay_acc[c].add(m, a.coef[m - 1], c4(hi, c), c4(lo, c));
            }
            float4 kk;
            if (VARDEN) {
                const float4 d = ld_model(a.den, s, yo, zo);
                kk = make_float4(d.x * a.dt, d.y * a.dt, d.z * a.dt, d.w * a.dt);
            } else {
                kk = make_float4(kc, kc, kc, kc);
            }
            const float4 pold = Pq[0];
            float4 pn;
            float2 fy, fz[4];
            if (edge) own_tables(fy, fz);
#pragma unroll
            for (int c = 0; c < 4; c++) {
                Acc<R> ax, az_;
#pragma unroll
                for (int m = 1; m <= R; m++) {
                    ax.add(m, a.coef[m - 1], c4(Vq[R + m - 1], c), c4(Vq[R - m], c));
                    az_.add(m, a.coef[m - 1], wz[K::DR + R + c + m - 1], wz[K::DR + R + c - m]);
                }
                float div = __fmul_rn(ax.v, a.rdx);
                div = __fmaf_rn(ay_acc[c].v, a.rdy, div);
                div = __fmaf_rn(az_.v, a.rdz, div);
                const float v = c4(vpc, c);
                const float k = __fmul_rn(__fmul_rn(c4(kk, c), v), v);
                float p = __fmaf_rn(-k, div, c4(pold, c));
                if (edge)
                    p = (xin_s && fy.y != 0.0f && fz[c].y != 0.0f)
                            ? __fmul_rn(p, xpad_s ? fx_s : (fy.x >= 0.0f ? fy.x : fz[c].x))
                            : 0.0f;
                r4f(pn, c) = p;
            }
            if (own_ok) {
                const long long o = shot_off + (long long)s * L.xstride + own_off;
                st4s(a.p_out + o, pn);
                st4s(a.vy_out + o, ld4s(sNY + (yl + R) * TZ + zr));
                st4s(a.vz_out + o, ld4s(sNZ + yl * K::VZW + zr + K::RQ));
            }
        }
#pragma unroll
        for (int j = 0; j + 1 < K::NQ; j++) Pq[j] = Pq[j + 1];
        Pq[K::NQ - 1] = pnext;
    }
}

__global__ void inject3d_kernel(float* p, Layout3D L, const ShotDev* shots, const int* slot_to_shot, int active,
                                const float* wavelets, int step) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= active) return;
    const ShotDev sd = shots[slot_to_shot[i]];
    if (step >= sd.nt) return;
    const long long o = (long long)slot_to_shot[i] * L.shot_stride + (long long)sd.sx * L.xstride +
                        (long long)sd.sy * L.pitch + sd.sz;
    // P[s] -= (dt * den * vp) * w[k], AFD:250 (separate roundings)
    p[o] = __fsub_rn(p[o], __fmul_rn(sd.inj_scale, wavelets[sd.wav_off + step]));
}

__global__ void gather3d_kernel(const float* p, Layout3D L, const ShotDev* shots, const int* slot_to_shot,
                                const int* rec_x, const int* rec_y, const int* rec_z, float* records, int step) {
    const int shot = slot_to_shot[blockIdx.y];
    const ShotDev sd = shots[shot];
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= sd.nrec || step >= sd.nt) return;
    const int q = sd.rec_list + r;
    const long long o = (long long)shot * L.shot_stride + (long long)rec_x[q] * L.xstride +
                        (long long)rec_y[q] * L.pitch + rec_z[q];
    records[sd.rec_base + (long long)step * sd.nrec + r] = p[o];
}

template <int R, bool VARDEN>
cudaError_t launch_t(const Acou3DArgs& a, int active, cudaStream_t st) {
    const size_t smem = sizeof(float) * K3<R>::SMEM_FLOATS;
    auto k = acoustic3d_step_kernel<R, VARDEN>;
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
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

cudaError_t acoustic3d_launch_step(int radius, const Acou3DArgs& a, int active, bool varden, cudaStream_t st) {
    if (active <= 0) return cudaSuccess;
    switch (radius) {
    case 2: return varden ? launch_t<2, true>(a, active, st) : launch_t<2, false>(a, active, st);
    case 4: return varden ? launch_t<4, true>(a, active, st) : launch_t<4, false>(a, active, st);
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
                                     int active, const float* wavelets, int step, cudaStream_t st) {
    if (active <= 0) return cudaSuccess;
    inject3d_kernel<<<(active + 63) / 64, 64, 0, st>>>(p, L, shots, slot_to_shot, active, wavelets, step);
    return cudaGetLastError();
}

cudaError_t acoustic3d_launch_gather(const float* p, const Layout3D& L, const ShotDev* shots,
                                     const int* slot_to_shot, int active, const int* rec_x, const int* rec_y,
                                     const int* rec_z, float* records, int nrec_max, int step, cudaStream_t st) {
    if (active <= 0 || nrec_max <= 0) return cudaSuccess;
    const dim3 grid((nrec_max + 255) / 256, active);
    gather3d_kernel<<<grid, 256, 0, st>>>(p, L, shots, slot_to_shot, rec_x, rec_y, rec_z, records, step);
    return cudaGetLastError();
}

}  // namespace sfd
