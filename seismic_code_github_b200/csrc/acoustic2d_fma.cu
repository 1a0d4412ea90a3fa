// FMA step kernel of the 2-D acoustic velocity-pressure scheme (AFD:237-380) for sm_100a.
//
// Same tile (64 x 64), update semantics and outputs as the reference-order kernel in
// acoustic2d.cu; staging and arithmetic are organised for Blackwell:
//   * the three input fields of a tile (P with a 2R halo, Vx with an R x-halo, Vz with an
//     R z-halo) arrive by three TMA bulk-tensor loads (cp.async.bulk.tensor.3d, no multicast)
//     completing on one mbarrier; the wait is bounded and reports a timeout through a flag;
//   * every stencil sum runs on paired FP32 instructions (FFMA2 / FMUL2), two grid points per
//     instruction, from register windows (each staged value is read from shared memory about
//     once per thread instead of 2R times);
//   * x-stencils (Vx update, d/dx of Vx) pair two neighbouring z: the float4 layout of a row;
//   * z-stencils (Vz update, d/dz of Vz) pair two neighbouring x rows: P (rows of the tile) and
//     the new Vz are copied into an x-pair-interleaved buffer so that every shifted operand is
//     an aligned register pair;
//   * tiles whose working set is inside the sponge-free, fully updated interior skip the
//     sponge and mask multiplies (a CTA-uniform branch).
// Two CTAs share an SM, so one CTA's loads overlap the other's arithmetic.  The divergence
// sx + sz is formed with scalar round-to-nearest adds (never fused with the products before
// them), as in the x-marching kernel (acoustic2d_march.cu), so that the two give the same bits.
//
// The same kernel runs the adjoint step (ADJ = true; the recurrence is stated in adjoint2d.cu):
// the P, Vx, Vz slots then hold the adjoint state nu = M K a Q (halo 2R), X and Z; phase A forms
// X' = X + rdx S+x nu, phase B Z' = Z + rdz S+z nu, phase C the new nu from S-x and S-z of the
// density-scaled, masked X' and Z', plus the imaging sum g += nu_old D_k.  Every model factor is
// needed at the tile's own cells only, which is why the adjoint carries nu rather than Q.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>

#include "sfd_internal.h"

namespace sfd {
namespace {

constexpr int kThreads = 256;

__host__ __device__ constexpr int r4(int v) { return (v + 3) & ~3; }
__host__ __device__ constexpr int r2(int v) { return (v + 1) & ~1; }
__host__ __device__ constexpr int r32(int v) { return (v + 31) & ~31; }
__host__ __device__ constexpr int odd_pairs(int w) { return ((w / 2) % 2 == 1) ? w : w + 2; }
// smallest w >= v with w = 8 (mod 16): 8-byte loads of 16 lanes spread over rows two apart
// then cover all 16 eight-byte bank slots
__host__ __device__ constexpr int pitch8(int v) { return v + ((8 - v % 16) + 16) % 16; }

template <int R, int NST>
struct TP {
    static constexpr int TX = kTileX, TZ = kTileZ;
    static constexpr int RQ = r4(R);         // z halo of the velocity region
    static constexpr int HZ = 2 * RQ;        // z halo of the staged pressure
    static constexpr int HX = 2 * R;         // x halo of the staged pressure
    // TMA boxes land densely: row pitch = box width
    static constexpr int SP_ROWS = TX + 2 * HX, SP_W = TZ + 2 * HZ, SP_P = SP_W;
    // Vx rows are padded to TZ + 4 floats (the TMA box is 4 floats wider than the tile) so that
    // rows four apart fall on different shared-memory banks in phase C
    static constexpr int SVX_ROWS = TX + 2 * R, SVX_P = TZ + 4;
    static constexpr int NZV = TZ + 2 * RQ, SVZ_P = pitch8(NZV);
    static constexpr int NXV = TX + 2 * R;
    static constexpr int NPAIR = TX / 2;
    static constexpr int IW = odd_pairs(SP_W);   // z entries per interleaved pair row
    // phase A (Vx): one z-vector x KX rows per thread
    static constexpr int KX = 5, VX_BLOCKS = (SVX_ROWS + KX - 1) / KX, NA = (TZ / 4) * VX_BLOCKS;
    // phase B (Vz): one x pair x KZB z per thread; NPAIR * NZB = 256 threads
    static constexpr int NZB = kThreads / NPAIR;
    static constexpr int KZB = r2((NZV + NZB - 1) / NZB);
    static constexpr int OFFB = (R % 2 == 0) ? R : R - 1;
    static constexpr int NWB = r2(KZB + OFFB + R);
    // phase C (P): 4 rows x one z-vector per thread
    static constexpr int OFFC = (R % 2 == 0) ? R : R + 1;
    static constexpr int NWC = r2(OFFC + R + 3);
    // shared layout (floats): two stages of TMA destinations (128-byte aligned), each holding
    // P, Vx and Vz of one tile, then the interleave buffer, the sponge tables and two
    // mbarriers.  Slack after each array absorbs window over-reads of the last thread blocks
    // at small radii.
    static constexpr int PAD = 256;
    static constexpr int OFF_VX = r32(SP_ROWS * SP_P + PAD);           // within a stage
    static constexpr int OFF_VZ = r32(OFF_VX + SVX_ROWS * SVX_P + PAD);  // within a stage
    static constexpr int STAGE = r32(OFF_VZ + TX * SVZ_P + PAD);
    static constexpr int OFF_I = NST * STAGE;
    static constexpr int OFF_AX = r32(OFF_I + NPAIR * IW * 2 + PAD);
    static constexpr int OFF_MX = OFF_AX + r4(NXV);
    static constexpr int OFF_AZ = OFF_MX + r4(NXV);
    static constexpr int OFF_MZ = OFF_AZ + r4(NZV);
    static constexpr int OFF_BAR = r4(OFF_MZ + r4(NZV));  // two mbarriers (8 bytes each)
    static constexpr int SMEM_FLOATS = OFF_BAR + 4;
    static constexpr unsigned TX_BYTES = 4u * (SP_ROWS * SP_W + SVX_ROWS * SVX_P + TX * SVZ_P);
    static_assert(NPAIR * NZB == kThreads, "phase B covers the block");
    static_assert(TX * TZ == 16 * kThreads, "phase C: 16 points per thread");
    static_assert(NZB * KZB >= NZV, "phase B covers the velocity region");
};

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float2 ld2(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ void st2(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }
__device__ __forceinline__ float2 lo(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi(float4 v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ float4 cat(float2 a, float2 b) { return make_float4(a.x, a.y, b.x, b.y); }
__device__ __forceinline__ float2 bc(float c) { return make_float2(c, c); }
// a - b, exactly rounded once (fma with a -1 factor)
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float comp(float4 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w)); }
__device__ __forceinline__ float cmp2(float2 v, int i) { return i == 0 ? v.x : v.y; }

__device__ __forceinline__ unsigned sptr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tma_load_3d(float* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(sptr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(sptr(bar))
        : "memory");
}

// L2 prefetch of a box (no shared-memory destination, no completion to wait for); the
// coordinates follow the rules of tma_load_3d
__device__ __forceinline__ void tma_prefetch_3d(const CUtensorMap* map, int c0, int c1, int c2) {
    asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];"
                 ::"l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2)
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

// One tile.  EDGE = some point of the tile's working set lies in the sponge or the frozen rim.
template <int R, int NST, bool VARDEN, bool EDGE, bool ADJ>
__device__ __forceinline__ void tile_body(const Acou2DArgs& a, float* smem, float* stage, const ShotDev& sd, int shot,
                                          int tile, int x0, int z0) {
    using T = TP<R, NST>;
    float* sP = stage;
    float* sVx = stage + T::OFF_VX;
    float* sVz = stage + T::OFF_VZ;
    float* sI = smem + T::OFF_I;
    const float* sAx = smem + T::OFF_AX;
    const float* sMx = smem + T::OFF_MX;
    const float* sAz = smem + T::OFF_AZ;
    const float* sMz = smem + T::OFF_MZ;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nx = sd.nx, nz = a.nz;
    const long long soff = (long long)shot * a.L.shot_stride;
    const int pitch = a.L.pitch;
    auto cell = [&](int x, int z) -> long long { return soff + (long long)(x + a.L.gx) * pitch + a.L.gz + z; };

    float C[R];
#pragma unroll
    for (int m = 0; m < R; m++) C[m] = a.coef[m];

    // Model values of this thread's phase-C points and the tile's receiver range: the global
    // loads are issued now so that their latency is covered by phases A and B.
    float4 vpre[4], dpre[4];
    {
        const int zgv = (lane & 3) + 4 * (lane >> 3), xbv = ((lane >> 2) & 1) + 2 * warp;  // phase C's mapping
        const int gz = z0 + 4 * zgv;
#pragma unroll
        for (int o = 0; o < 4; o++) {
            const long long mi = (long long)min(sd.x0 + x0 + 4 * xbv + o, a.nx_model - 1) * a.mpitch + gz;
            vpre[o] = __ldg(reinterpret_cast<const float4*>(a.vp + mi));
            dpre[o] = VARDEN ? __ldg(reinterpret_cast<const float4*>(a.den + mi))
                             : make_float4(a.den_c, a.den_c, a.den_c, a.den_c);
        }
    }
    const int* trp = a.tile_rec_ptr + sd.tile_rec_base + tile;
    const int rb = __ldg(trp), re = __ldg(trp + 1);

    // ---- interleave the tile's P rows in x pairs: sI[(p*IW + z)*2 + {0,1}] = P[x0+2p+{0,1}][z] ----
    // (each item moves two z of a pair: 8-byte loads and 16-byte stores, both contiguous across
    // consecutive lanes, so neither side has bank conflicts)
    {
        constexpr int Q = T::SP_W / 2, N = T::NPAIR * Q, IT = (N + kThreads - 1) / kThreads;
#pragma unroll
        for (int it = 0; it < IT; it++) {
            const int i = tid + it * kThreads;
            if (i < N) {
                const int p = i / Q, q = i - p * Q;
                const float2 u = ld2(sP + (2 * p + T::HX) * T::SP_P + 2 * q);
                const float2 v = ld2(sP + (2 * p + 1 + T::HX) * T::SP_P + 2 * q);
                st4(sI + (p * T::IW + 2 * q) * 2, make_float4(u.x, v.x, u.y, v.y));
            }
        }
    }

    // ---- phase A: Vx(t) on rows x0-R .. x0+TX+R (AFD:255-269) ----
#pragma unroll
    for (int it = 0; it < (T::NA + kThreads - 1) / kThreads; it++) {
        const int blk = tid + it * kThreads;
        if (blk >= T::NA) break;
        // 8 consecutive lanes -> 8 consecutive z-vectors of one row
        const int zgv = (blk & 7) + 8 * ((blk >> 3) / T::VX_BLOCKS);
        const int r0 = ((blk >> 3) % T::VX_BLOCKS) * T::KX;
        const int zo = 4 * zgv;
        const float* wbase = sP + (r0 + 1) * T::SP_P + T::HZ + zo;
        float4 w[T::KX + 2 * R - 1];
#pragma unroll
        for (int j = 0; j < T::KX + 2 * R - 1; j++) w[j] = ld4(wbase + j * T::SP_P);
        float4 az = make_float4(1.f, 1.f, 1.f, 1.f), mz = az;
        if (EDGE) {
            az = ld4(sAz + T::RQ + zo);
            mz = ld4(sMz + T::RQ + zo);
        }
#pragma unroll
        for (int o = 0; o < T::KX; o++) {
            const int row = r0 + o;
            if (row < T::SVX_ROWS) {
                float2 sl = mul2(bc(C[0]), sub2(lo(w[o + R]), lo(w[o + R - 1])));
                float2 sh = mul2(bc(C[0]), sub2(hi(w[o + R]), hi(w[o + R - 1])));
#pragma unroll
                for (int m = 1; m < R; m++) {
                    sl = fma2(bc(C[m]), sub2(lo(w[o + R + m]), lo(w[o + R - 1 - m])), sl);
                    sh = fma2(bc(C[m]), sub2(hi(w[o + R + m]), hi(w[o + R - 1 - m])), sh);
                }
                float* vrow = sVx + row * T::SVX_P + zo;
                const float4 vo = ld4(vrow);
                float2 bl = bc(-a.bx_f), bh = bl;
                if (VARDEN) {
                    const int gx = min(max(sd.x0 + x0 - R + row, 0), a.nx_model - 1);
                    const float4 d = __ldg(reinterpret_cast<const float4*>(a.den + (long long)gx * a.mpitch + z0 + zo));
                    bl = make_float2(-a.dtdx / d.x, -a.dtdx / d.y);
                    bh = make_float2(-a.dtdx / d.z, -a.dtdx / d.w);
                }
                float2 vl = lo(vo), vh = hi(vo);
                if (ADJ) {  // staged X'' = B M (X + rdx S+x nu), B = dt/(dx den) (1 here for constant density)
                    vl = fma2(bc(a.rdx_f), sl, vl);
                    vh = fma2(bc(a.rdx_f), sh, vh);
                    if (EDGE) {
                        const float mx = sMx[row];
                        vl = mul2(vl, mul2(bc(mx), lo(mz)));
                        vh = mul2(vh, mul2(bc(mx), hi(mz)));
                    }
                    if (VARDEN) {
                        vl = mul2(vl, make_float2(-bl.x, -bl.y));
                        vh = mul2(vh, make_float2(-bh.x, -bh.y));
                    }
                } else if (EDGE) {
                    const float ax = sAx[row], mx = sMx[row];
                    const float4 sa = ax >= 0.0f ? make_float4(ax, ax, ax, ax) : az;
                    vl = mul2(vl, lo(sa));
                    vh = mul2(vh, hi(sa));
                    vl = mul2(fma2(bl, sl, vl), mul2(bc(mx), lo(mz)));
                    vh = mul2(fma2(bh, sh, vh), mul2(bc(mx), hi(mz)));
                } else {
                    vl = fma2(bl, sl, vl);
                    vh = fma2(bh, sh, vh);
                }
                st4(vrow, cat(vl, vh));
            }
        }
    }

    __syncthreads();  // sI holds interleaved P

    // ---- phase B: Vz(t) on x pairs of the tile, z0-RQ .. z0+TZ+RQ (AFD:272-286) ----
    // lanes 0-7 of a group take 8 consecutive z blocks of one x pair: the window loads of those
    // lanes start 2*KZB floats apart, which spreads them over all 16-byte bank groups
    float2 outz[T::KZB];
    const int pB = tid / T::NZB, zbB = tid % T::NZB;
    {
        const float* wsrc = sI + (pB * T::IW + zbB * T::KZB + T::RQ - T::OFFB) * 2;
        float2 wp[T::NWB];
#pragma unroll
        for (int j = 0; j < T::NWB; j += 2) {
            const float4 v = ld4(wsrc + 2 * j);
            wp[j] = lo(v);
            wp[j + 1] = hi(v);
        }
        const int xr0 = 2 * pB;  // tile-relative rows xr0, xr0+1
        float ax0 = 1.f, ax1 = 1.f, mx0 = 1.f, mx1 = 1.f;
        if (EDGE) {
            ax0 = sAx[xr0 + R]; ax1 = sAx[xr0 + 1 + R];
            mx0 = sMx[xr0 + R]; mx1 = sMx[xr0 + 1 + R];
        }
        const float* vo0p = sVz + xr0 * T::SVZ_P + zbB * T::KZB;
        const float* vo1p = vo0p + T::SVZ_P;
#pragma unroll
        for (int k = 0; k < T::KZB; k += 2) {
            const int zi = zbB * T::KZB + k;  // Vz-region index, z = z0 - RQ + zi
            if (zi < T::NZV) {
                const float2 o0 = ld2(vo0p + k), o1 = ld2(vo1p + k);  // (row, z..z+1)
#pragma unroll
                for (int kk = 0; kk < 2; kk++) {
                    const int kq = k + kk;
                    float2 s = mul2(bc(C[0]), sub2(wp[kq + T::OFFB + 1], wp[kq + T::OFFB]));
#pragma unroll
                    for (int m = 1; m < R; m++)
                        s = fma2(bc(C[m]), sub2(wp[kq + T::OFFB + m + 1], wp[kq + T::OFFB - m]), s);
                    float vo0 = cmp2(o0, kk), vo1 = cmp2(o1, kk);
                    float b0 = a.bz_f, b1 = a.bz_f;
                    if (VARDEN) {
                        const int zg = z0 - T::RQ + zi + kk;
                        const int g0 = min(sd.x0 + x0 + xr0, a.nx_model - 1);
                        const int g1 = min(sd.x0 + x0 + xr0 + 1, a.nx_model - 1);
                        b0 = a.dtdz / __ldg(a.den + (long long)g0 * a.mpitch + zg);
                        b1 = a.dtdz / __ldg(a.den + (long long)g1 * a.mpitch + zg);
                    }
                    if (ADJ) {  // staged Z'' = B M (Z + rdz S+z nu)
                        const float mz = EDGE ? sMz[zi + kk] : 1.0f;
                        const float c0 = VARDEN ? b0 : 1.0f, c1 = VARDEN ? b1 : 1.0f;
                        outz[kq] = make_float2(fmaf(a.rdz_f, s.x, vo0) * (mx0 * mz) * c0,
                                               fmaf(a.rdz_f, s.y, vo1) * (mx1 * mz) * c1);
                    } else if (EDGE) {
                        const float az = sAz[zi + kk], mz = sMz[zi + kk];
                        vo0 *= (ax0 >= 0.0f ? ax0 : az);
                        vo1 *= (ax1 >= 0.0f ? ax1 : az);
                        outz[kq] = make_float2(fmaf(-b0, s.x, vo0) * (mx0 * mz), fmaf(-b1, s.y, vo1) * (mx1 * mz));
                    } else {
                        outz[kq] = make_float2(fmaf(-b0, s.x, vo0), fmaf(-b1, s.y, vo1));
                    }
                }
            }
        }
    }
    __syncthreads();  // everyone is done reading interleaved P
    {
        // interleaved new Vz, two z per 16-byte store: the eight lanes of a quarter warp share
        // one x pair and start 2*KZB entries apart, which spreads them over all banks
        float* dst = sI + (pB * T::IW + zbB * T::KZB) * 2;
#pragma unroll
        for (int k = 0; k < T::KZB; k += 2)
            if (zbB * T::KZB + k < T::NZV) st4(dst + 2 * k, cat(outz[k], outz[k + 1]));
    }
    __syncthreads();

    // ---- phase C: P(t) on the tile, 4 rows x one z-vector per thread (AFD:289-314, 337-338) ----
    const int step = a.step;
    // a quarter warp = 4 consecutive z-vectors x 2 consecutive x blocks: with the padded Vx rows
    // and odd x blocks taking their two x pairs in reverse order, the Vx and interleaved-Vz
    // window loads of the eight lanes fall on distinct banks
    const int zgv = (lane & 3) + 4 * (lane >> 3);
    const int xbv = ((lane >> 2) & 1) + 2 * warp;
    const int zo = 4 * zgv, r0 = 4 * xbv;
    float4 sx[4];
    {
        const float* vbase = sVx + r0 * T::SVX_P + zo;
        float4 vw[2 * R + 3];
#pragma unroll
        for (int j = 0; j < 2 * R + 3; j++) vw[j] = ld4(vbase + j * T::SVX_P);
#pragma unroll
        for (int o = 0; o < 4; o++) {
            float2 sl = mul2(bc(C[0]), sub2(lo(vw[o + R]), lo(vw[o + R - 1])));
            float2 sh = mul2(bc(C[0]), sub2(hi(vw[o + R]), hi(vw[o + R - 1])));
#pragma unroll
            for (int m = 1; m < R; m++) {
                sl = fma2(bc(C[m]), sub2(lo(vw[o + R + m]), lo(vw[o + R - m - 1])), sl);
                sh = fma2(bc(C[m]), sub2(hi(vw[o + R + m]), hi(vw[o + R - m - 1])), sh);
            }
            const float cx = ADJ ? a.adj_cx : a.rdx_f;
            sx[o] = cat(mul2(sl, bc(cx)), mul2(sh, bc(cx)));
        }
        const int gz = z0 + zo;
        if (!ADJ && gz < nz) {
            float* vxo = a.vx_out + cell(x0 + r0, gz);
#pragma unroll
            for (int o = 0; o < 4; o++) {
                if (x0 + r0 + o < nx) {
                    const float4 v = vw[o + R];
                    if (gz + 3 < nz) *reinterpret_cast<float4*>(vxo + (long long)o * pitch) = v;
                    else for (int q = 0; q < 4 && gz + q < nz; q++) vxo[(long long)o * pitch + q] = comp(v, q);
                }
            }
        }
    }
    float4 az = make_float4(1.f, 1.f, 1.f, 1.f), mz = az;
    if (EDGE) {
        az = ld4(sAz + T::RQ + zo);
        mz = ld4(sMz + T::RQ + zo);
    }
    const int gz = z0 + zo;
#pragma unroll
    for (int qi = 0; qi < 2; qi++) {
        const int q = (xbv & 1) ? 1 - qi : qi;
        const int p = 2 * xbv + q;  // x pair: tile rows 2p, 2p+1 = r0 + 2q, r0 + 2q + 1
        // adjoint: D_k and the imaging sum of the pair's cells, loaded before the z-stencil so
        // that their latency is covered
        float4 dpf[2], gpf[2];
        if (ADJ) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int gx = x0 + r0 + 2 * q + h;
                dpf[h] = gpf[h] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (gx < nx && gz + 3 < nz) {
                    const long long c = cell(gx, gz);
                    dpf[h] = __ldg(reinterpret_cast<const float4*>(a.adj_div + c));
                    gpf[h] = *reinterpret_cast<const float4*>(a.adj_g + c);
                }
            }
        }
        const float* zsrc = sI + (p * T::IW + zo + T::RQ - T::OFFC) * 2;
        float2 vz[T::NWC];
#pragma unroll
        for (int j = 0; j < T::NWC; j += 2) {
            const float4 v = ld4(zsrc + 2 * j);
            vz[j] = lo(v);
            vz[j + 1] = hi(v);
        }
        float2 sz[4];  // (row 2p, row 2p+1) at z = zo + c, scaled by 1/dz
#pragma unroll
        for (int c = 0; c < 4; c++) {
            float2 s = mul2(bc(C[0]), sub2(vz[c + T::OFFC], vz[c + T::OFFC - 1]));
#pragma unroll
            for (int m = 1; m < R; m++) s = fma2(bc(C[m]), sub2(vz[c + T::OFFC + m], vz[c + T::OFFC - m - 1]), s);
            sz[c] = mul2(s, bc(ADJ ? a.adj_cz : a.rdz_f));
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int o = 2 * q + h, row = r0 + o, gx = x0 + row;
            float* pc = sP + (row + T::HX) * T::SP_P + T::HZ + zo;
            const float4 po = ld4(pc);
            // q depends on the thread: pick the register arrays' entries by selects
            const float4 vp4 = q ? vpre[2 + h] : vpre[h];
            const float4 dn4 = q ? dpre[2 + h] : dpre[h];
            const float4 sxo = q ? sx[2 + h] : sx[h];
            if (ADJ) {
                // bracket = nu_old / K + S-x(B M X') + S-z(B M Z') (= M a Q_old + ...), nu_new = M a K bracket
                const float2 kl = mul2(mul2(mul2(lo(dn4), lo(vp4)), lo(vp4)), bc(a.dt));
                const float2 kh = mul2(mul2(mul2(hi(dn4), hi(vp4)), hi(vp4)), bc(a.dt));
                const float2 dl = make_float2(cmp2(sz[0], h), cmp2(sz[1], h));
                const float2 dh = make_float2(cmp2(sz[2], h), cmp2(sz[3], h));
                const float2 bl = make_float2(__fadd_rn(__fadd_rn(sxo.x, dl.x), __fdividef(po.x, kl.x)),
                                              __fadd_rn(__fadd_rn(sxo.y, dl.y), __fdividef(po.y, kl.y)));
                const float2 bh = make_float2(__fadd_rn(__fadd_rn(sxo.z, dh.x), __fdividef(po.z, kh.x)),
                                              __fadd_rn(__fadd_rn(sxo.w, dh.y), __fdividef(po.w, kh.y)));
                float4 fa4 = make_float4(1.f, 1.f, 1.f, 1.f), fm4 = fa4;  // sponge a and mask M of the own cells
                if (EDGE) {
                    const float ax = sAx[row + R], mx = sMx[row + R];
                    fa4 = ax >= 0.0f ? make_float4(ax, ax, ax, ax) : az;
                    fm4 = make_float4(mx * mz.x, mx * mz.y, mx * mz.z, mx * mz.w);
                }
                const float2 nl = mul2(mul2(bl, kl), mul2(lo(fa4), lo(fm4)));
                const float2 nh = mul2(mul2(bh, kh), mul2(hi(fa4), hi(fm4)));
                if (gx < nx && gz < nz) {
                    const long long c = cell(gx, gz);
                    // X = a M X' and Z = a M Z' from the staged B M X', B M Z'
                    float4 xf = fa4, zf = fa4;
                    if (VARDEN) {
                        xf = make_float4(fa4.x * dn4.x * a.adj_xs, fa4.y * dn4.y * a.adj_xs, fa4.z * dn4.z * a.adj_xs,
                                         fa4.w * dn4.w * a.adj_xs);
                        zf = make_float4(fa4.x * dn4.x * a.adj_zs, fa4.y * dn4.y * a.adj_zs, fa4.z * dn4.z * a.adj_zs,
                                         fa4.w * dn4.w * a.adj_zs);
                    }
                    const float4 xs = ld4(sVx + (row + R) * T::SVX_P + zo);
                    const float4 xo = make_float4(xs.x * xf.x, xs.y * xf.y, xs.z * xf.z, xs.w * xf.w);
                    const float4 zo4 = make_float4(cmp2(vz[T::OFFC], h) * zf.x, cmp2(vz[T::OFFC + 1], h) * zf.y,
                                                   cmp2(vz[T::OFFC + 2], h) * zf.z, cmp2(vz[T::OFFC + 3], h) * zf.w);
                    const float bq[4] = {bl.x, bl.y, bh.x, bh.y};
                    if (gx == sd.sx && sd.sz >= gz && sd.sz < gz + 4)
                        for (int cc = 0; cc < 4; cc++)
                            if (sd.sz == gz + cc) a.adj_lam[(long long)shot * a.nt_max + step] = bq[cc];
                    const float4 nn = cat(nl, nh);
                    if (gz + 3 < nz) {
                        const float4 d4 = dpf[h];
                        float4 g4 = gpf[h];
                        g4 = make_float4(fmaf(po.x, d4.x, g4.x), fmaf(po.y, d4.y, g4.y), fmaf(po.z, d4.z, g4.z),
                                         fmaf(po.w, d4.w, g4.w));
                        *reinterpret_cast<float4*>(a.adj_g + c) = g4;
                        *reinterpret_cast<float4*>(a.p_out + c) = nn;
                        *reinterpret_cast<float4*>(a.vx_out + c) = xo;
                        *reinterpret_cast<float4*>(a.vz_out + c) = zo4;
                    } else {
                        for (int qq = 0; qq < 4 && gz + qq < nz; qq++) {
                            a.adj_g[c + qq] = fmaf(comp(po, qq), __ldg(a.adj_div + c + qq), a.adj_g[c + qq]);
                            a.p_out[c + qq] = comp(nn, qq);
                            a.vx_out[c + qq] = comp(xo, qq);
                            a.vz_out[c + qq] = comp(zo4, qq);
                        }
                    }
                }
                continue;
            }
            // -kk = -DEN * Vp * Vp * dt (AFD:293)
            const float2 kl = mul2(mul2(mul2(lo(dn4), lo(vp4)), lo(vp4)), bc(-a.dt));
            const float2 kh = mul2(mul2(mul2(hi(dn4), hi(vp4)), hi(vp4)), bc(-a.dt));
            const float2 dl = make_float2(cmp2(sz[0], h), cmp2(sz[1], h));
            const float2 dh = make_float2(cmp2(sz[2], h), cmp2(sz[3], h));
            const float2 divl = make_float2(__fadd_rn(sxo.x, dl.x), __fadd_rn(sxo.y, dl.y));
            const float2 divh = make_float2(__fadd_rn(sxo.z, dh.x), __fadd_rn(sxo.w, dh.y));
            float2 pl = fma2(kl, divl, lo(po));
            float2 ph = fma2(kh, divh, hi(po));
            if (a.div_out != nullptr && gx < nx && gz < nz) {  // recomputation for the adjoint
                float* dp = a.div_out + cell(gx, gz);
                if (gz + 3 < nz) *reinterpret_cast<float4*>(dp) = cat(divl, divh);
                else for (int qq = 0; qq < 4 && gz + qq < nz; qq++) dp[qq] = comp(cat(divl, divh), qq);
            }
            if (EDGE) {
                const float ax = sAx[row + R], mx = sMx[row + R];
                const float4 sa = ax >= 0.0f ? make_float4(ax, ax, ax, ax) : az;
                pl = mul2(mul2(pl, lo(sa)), mul2(bc(mx), lo(mz)));
                ph = mul2(mul2(ph, hi(sa)), mul2(bc(mx), hi(mz)));
            }
            float pn[4] = {pl.x, pl.y, ph.x, ph.y};
            st4(pc, make_float4(pn[0], pn[1], pn[2], pn[3]));  // receivers read the recorded value here
            if (gx < nx && gz < nz) {
                if (gx == sd.sx && sd.sz >= gz && sd.sz < gz + 4 && step + 1 < sd.nt) {
                    const float inj = sd.inj_scale * __ldg(a.wavelets + sd.wav_off + step + 1);
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        if (sd.sz == gz + c) {
                            if (a.src_pre) a.src_pre[shot] = pn[c];
                            pn[c] -= inj;
                        }
                }
                const long long c = cell(gx, gz);
                const float4 vzc = make_float4(cmp2(vz[T::OFFC], h), cmp2(vz[T::OFFC + 1], h),
                                               cmp2(vz[T::OFFC + 2], h), cmp2(vz[T::OFFC + 3], h));
                if (gz + 3 < nz) {
                    *reinterpret_cast<float4*>(a.p_out + c) = make_float4(pn[0], pn[1], pn[2], pn[3]);
                    *reinterpret_cast<float4*>(a.vz_out + c) = vzc;
                } else {
                    for (int qq = 0; qq < 4 && gz + qq < nz; qq++) {
                        a.p_out[c + qq] = pn[qq];
                        a.vz_out[c + qq] = comp(vzc, qq);
                    }
                }
            }
        }
    }
    // ---- adjoint: residual of step k-1 at the receivers of this tile (AFD:376-377 transposed),
    // nu += M a K res; several receivers may share a cell, so the adds are atomic ----
    if (ADJ) {
        if (step >= 1 && re > rb) {
            __syncthreads();
            for (int j = rb + tid; j < re; j += kThreads) {
                const int ridx = a.tile_rec_idx[j];
                const int rx = a.rec_x[sd.rec_list + ridx], rz = a.rec_z[sd.rec_list + ridx];
                if (rx < R || rx >= nx - R || rz < R || rz >= nz - R) continue;  // M = 0
                const long long mi = (long long)min(sd.x0 + rx, a.nx_model - 1) * a.mpitch + rz;
                const float vpv = __ldg(a.vp + mi), dnv = VARDEN ? __ldg(a.den + mi) : a.den_c;
                float sa = 1.0f;
                if (rx < a.pml) sa = a.sponge[a.pml - 1 - rx];
                else if (rx >= nx - a.pml) sa = a.sponge[rx - (nx - a.pml)];
                else if (rz < a.pml) sa = a.sponge[a.pml - 1 - rz];
                else if (rz >= nz - a.pml) sa = a.sponge[rz - (nz - a.pml)];
                const float v = a.adj_res[sd.rec_base + (long long)(step - 1) * sd.nrec + ridx];
                atomicAdd(a.p_out + cell(rx, rz), dnv * vpv * vpv * a.dt * sa * v);
            }
        }
        return;
    }
    // ---- receivers (AFD:376-377) ----
    if (re > rb) {
        __syncthreads();
        for (int j = rb + tid; j < re; j += kThreads) {
            const int ridx = a.tile_rec_idx[j];
            const int rx = a.rec_x[sd.rec_list + ridx], rz = a.rec_z[sd.rec_list + ridx];
            a.records[sd.rec_base + (long long)step * sd.nrec + ridx] =
                sP[(rx - x0 + T::HX) * T::SP_P + (rz - z0) + T::HZ];
        }
    }
}

// Sponge / update-mask tables of one tile (AFD:164-194; AFD updates only R <= i,j < N-R).
template <int R, int NST>
__device__ __forceinline__ void build_tables(const Acou2DArgs& a, float* smem, int x0, int z0, int nx) {
    using T = TP<R, NST>;
    const int nz = a.nz, pml = a.pml, tid = threadIdx.x;
    float* sAx = smem + T::OFF_AX;
    float* sMx = smem + T::OFF_MX;
    float* sAz = smem + T::OFF_AZ;
    float* sMz = smem + T::OFF_MZ;
    for (int i = tid; i < T::NXV; i += kThreads) {
        const int x = x0 - R + i;
        float ax = -1.0f, mx = 0.0f;
        if (x >= 0 && x < nx) {
            if (x < pml) ax = a.sponge[pml - 1 - x];
            else if (x >= nx - pml) ax = a.sponge[x - (nx - pml)];
            mx = (x >= R && x < nx - R) ? 1.0f : 0.0f;
        }
        sAx[i] = ax;
        sMx[i] = mx;
    }
    for (int i = tid; i < T::NZV; i += kThreads) {
        const int z = z0 - T::RQ + i;
        float az = 1.0f, mz = 0.0f;
        if (z >= 0 && z < nz) {
            if (z < pml) az = a.sponge[pml - 1 - z];
            else if (z >= nz - pml) az = a.sponge[z - (nz - pml)];
            mz = (z >= R && z < nz - R) ? 1.0f : 0.0f;
        }
        sAz[i] = az;
        sMz[i] = mz;
    }
}

// Persistent kernel: CTA b processes tiles b, b+G, b+2G, ... of all active shots.  While a tile
// is computed out of one shared-memory stage, the TMA unit fills the other stage with the next
// tile's P, Vx and Vz boxes (one mbarrier per stage, expect_tx accounting).
template <int R, int NST, bool VARDEN, bool ADJ>
__global__ void __launch_bounds__(kThreads, NST == 1 ? 2 : 1)
acoustic2d_step_fma_kernel(const __grid_constant__ Acou2DArgs a, int active) {
    using T = TP<R, NST>;
    extern __shared__ __align__(128) float smem[];
    const int tid = threadIdx.x;
    const int per_shot = a.L.ntx * a.L.ntz;
    const int total = active * per_shot;
    const int G = gridDim.x;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + T::OFF_BAR);

    // which tile t is: shot, tile index within the shot, origin; false if beyond the aperture
    auto locate = [&](int t, int& shot, int& tile, int& x0, int& z0) -> bool {
        int slot, k;
        if (a.tile_major) {
            k = t / active;
            slot = t - k * active;
        } else {
            slot = t / per_shot;
            k = t - slot * per_shot;
        }
        tile = a.tile_order ? __ldg(a.tile_order + k) : k;
        shot = a.slot_to_shot[slot];
        const int tx_i = tile / a.L.ntz;
        x0 = tx_i * T::TX;
        z0 = (tile - tx_i * a.L.ntz) * T::TZ;
        return x0 < a.shots[shot].nx;
    };
    // the test hook: this CTA issues no loads and waits test_wait_ns instead of about one second
    const bool probed = (int)blockIdx.x == a.test_cta && a.step == a.test_step;
    const unsigned long long wait_ns = probed ? a.test_wait_ns : 1000000000ull;
    // thread 0: start the three box loads of tile t into stage stg
    auto issue = [&](int t, int stg) {
        int shot, tile, x0, z0;
        if (probed || !locate(t, shot, tile, x0, z0)) return;
        float* st = smem + stg * T::STAGE;
        uint64_t* bar = bars + stg;
        // order this thread's view of earlier generic-proxy writes to the stage before the
        // async-proxy writes that follow
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sptr(bar)), "r"(T::TX_BYTES)
                     : "memory");
        const int gx = a.L.gx, gz = a.L.gz;
        tma_load_3d(st, &a.tm_p, gz + z0 - T::HZ, gx + x0 - T::HX, shot, bar);
        tma_load_3d(st + T::OFF_VX, &a.tm_vx, gz + z0, gx + x0 - R, shot, bar);
        tma_load_3d(st + T::OFF_VZ, &a.tm_vz, gz + z0 - T::RQ, gx + x0, shot, bar);
    };
    // thread 0: prefetch the three boxes of tile t into L2 (for the CTA that will take tile t)
    auto prefetch = [&](int t) {
        int shot, tile, x0, z0;
        if (!locate(t, shot, tile, x0, z0)) return;
        const int gx = a.L.gx, gz = a.L.gz;
        tma_prefetch_3d(&a.tm_p, gz + z0 - T::HZ, gx + x0 - T::HX, shot);
        tma_prefetch_3d(&a.tm_vx, gz + z0, gx + x0 - R, shot);
        tma_prefetch_3d(&a.tm_vz, gz + z0 - T::RQ, gx + x0, shot);
    };

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sptr(bars)) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sptr(bars + 1)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // Programmatic dependent launch (the step kernels are launched with programmatic stream
    // serialisation): the next step's CTAs may be scheduled once every CTA of this grid has
    // started, so they fill the SMs that this step's last wave leaves idle.  Every thread waits
    // here until the previous grid in the stream has completed and its writes are visible; all
    // reads of wavefields, imaging sums and records follow this point.
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (tid == 0 && (int)blockIdx.x < total) issue(blockIdx.x, 0);
    if (NST == 1 && tid == 0 && a.l2_ahead > 0 && (int)blockIdx.x + a.l2_ahead < total)
        prefetch(blockIdx.x + a.l2_ahead);

    unsigned phase = 0;  // bit s: parity of the next completion of stage s's barrier
    for (int i = 0;; i++) {
        const int t = blockIdx.x + i * G;
        if (t >= total) break;
        const int stg = NST == 1 ? 0 : (i & 1);
        if (NST == 2 && tid == 0 && t + G < total) issue(t + G, stg ^ 1);  // prefetch into the other stage
        int shot, tile, x0, z0;
        if (!locate(t, shot, tile, x0, z0)) continue;  // uniform: no load was issued for it
        const ShotDev sd = a.shots[shot];
        const int nx = sd.nx, nz = a.nz;
        const int E = a.pml > R ? a.pml : R;
        const bool edge =
            !(x0 - R >= E && x0 + T::TX + R <= nx - E && z0 - T::RQ >= E && z0 + T::TZ + T::RQ <= nz - E);
        if (edge) build_tables<R, NST>(a, smem, x0, z0, nx);
        __syncthreads();  // tables written
        // bounded wait for this tile's boxes (about one second of wall time, then give up).  One
        // thread polls while the others sleep in the barrier, so that a waiting CTA takes no issue
        // slots from the CTA computing beside it; after the barrier every thread observes the
        // completed phase itself, which orders the TMA writes before its shared-memory reads.
        const unsigned par = (phase >> stg) & 1u;
        auto bounded_wait = [&](int b, unsigned pa) {
            bool ok = mbar_try_wait(bars + b, pa);
            if (!ok) {
                const uint64_t t0 = global_ns();
                while (!(ok = mbar_try_wait(bars + b, pa)) && global_ns() - t0 < wait_ns) {
                }
            }
            return ok;
        };
        bool done = true;
        if (tid == 0) done = bounded_wait(stg, par);
        if (__syncthreads_or(!done)) {
            if (tid == 0) {
                atomicExch(a.err_flag, 1);
                // let copies still in flight land before the CTA's shared memory is released
                bounded_wait(stg, par);
                if (NST == 2 && t + G < total) bounded_wait(stg ^ 1, (phase >> (stg ^ 1)) & 1u);
            }
            return;
        }
        if (tid != 0) mbar_try_wait(bars + stg, par);  // completed: returns at once
        phase ^= 1u << stg;
        float* st = smem + stg * T::STAGE;
        if (edge) tile_body<R, NST, VARDEN, true, ADJ>(a, smem, st, sd, shot, tile, x0, z0);
        else tile_body<R, NST, VARDEN, false, ADJ>(a, smem, st, sd, shot, tile, x0, z0);
        __syncthreads();  // stage, interleave buffer and tables are free again
    }
}

int sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    }
    return n;
}

template <int R, int NST, bool VARDEN, bool ADJ>
cudaError_t launch_t(const Acou2DArgs& a, int active, cudaStream_t st) {
    const size_t smem = sizeof(float) * TP<R, NST>::SMEM_FLOATS;
    auto k = acoustic2d_step_fma_kernel<R, NST, VARDEN, ADJ>;
    static bool attr[kMaxDevices] = {};
    if (cudaError_t e = smem_attr_once((const void*)k, (int)smem, attr)) return e;
    const int total = a.L.ntx * a.L.ntz * active;
    // one stage: one tile per CTA, two CTAs per SM; two stages: one persistent CTA per SM
    const int grid = NST == 1 ? total : (total < sm_count() ? total : sm_count());
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, a, active);
}

template <int R, bool ADJ>
cudaError_t launch_r(const Acou2DArgs& a, int active, bool varden, int stages, cudaStream_t st) {
    if (stages == 2)
        return varden ? launch_t<R, 2, true, ADJ>(a, active, st) : launch_t<R, 2, false, ADJ>(a, active, st);
    return varden ? launch_t<R, 1, true, ADJ>(a, active, st) : launch_t<R, 1, false, ADJ>(a, active, st);
}

template <int R>
void boxes_t(int bp[2], int bvx[2], int bvz[2]) {
    using T = TP<R, 1>;
    bp[0] = T::SP_W; bp[1] = T::SP_ROWS;
    bvx[0] = T::SVX_P; bvx[1] = T::SVX_ROWS;
    bvz[0] = T::SVZ_P; bvz[1] = T::TX;
}

}  // namespace

// Programmatic dependent launch of consecutive step kernels (SFD_PDL=0 in the environment
// turns it off; the kernels' griddepcontrol.wait is then a no-op)
bool pdl_enabled() {
    static int on = -1;
    if (on < 0) {
        const char* env = std::getenv("SFD_PDL");
        on = (env && std::atoi(env) == 0) ? 0 : 1;
    }
    return on == 1;
}

cudaError_t acoustic2d_fwd_launch(const Acou2DPlan& plan, int radius, const Acou2DArgs& a, int active, bool varden,
                                  cudaStream_t st) {
    if (acoustic2d_use_march(plan, a.L, active))
        return acoustic2d_march_launch(radius, a, active, varden, plan.seg, st, pdl_enabled());
    return acoustic2d_fma_launch(radius, a, active, varden, plan.stages, st);
}

cudaError_t acoustic2d_fma_launch(int radius, const Acou2DArgs& a, int active, bool varden, int stages,
                                 cudaStream_t st, bool adj) {
    switch (radius) {
#define SFD_CASE(RR) \
    case RR: return adj ? launch_r<RR, true>(a, active, varden, stages, st) \
                        : launch_r<RR, false>(a, active, varden, stages, st);
        SFD_CASE(1) SFD_CASE(2) SFD_CASE(4) SFD_CASE(5) SFD_CASE(8)
#undef SFD_CASE
    default: return cudaErrorInvalidValue;
    }
}

int acoustic2d_fma_gz(int radius) { return 2 * r4(radius); }

void acoustic2d_fma_boxes(int radius, int bp[2], int bvx[2], int bvz[2]) {
    switch (radius) {
    case 1: boxes_t<1>(bp, bvx, bvz); break;
    case 2: boxes_t<2>(bp, bvx, bvz); break;
    case 4: boxes_t<4>(bp, bvx, bvz); break;
    case 5: boxes_t<5>(bp, bvx, bvz); break;
    default: boxes_t<8>(bp, bvx, bvz); break;
    }
}

}  // namespace sfd
