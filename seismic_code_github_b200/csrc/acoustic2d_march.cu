// x-marching step kernel of the 2-D acoustic velocity-pressure scheme (AFD:237-380) for sm_100a.
//
// Same update semantics, arithmetic and outputs as the FMA tile kernel (acoustic2d_fma.cu); the
// records and wavefields are bit-identical.  Only the staging differs:
//   * a CTA owns one 64-wide z strip of one shot over a segment [xs, xe) of columns and walks
//     down x in chunks of 16 columns;
//   * chunk c needs P(t-1) on columns [xb, xb+32) (z halo 16), Vx(t-1) on [xb+R, xb+R+16) and
//     Vz(t-1) on [xb, xb+16) (z halo 8): three TMA boxes (cp.async.bulk.tensor.3d, no
//     multicast) into one of two shared-memory buffer sets, issued one chunk ahead so that the
//     copies of chunk c+1 land while chunk c computes;
//   * Vx(t) is computed once per column: chunk c computes columns [xb+R, xb+R+16) and passes the
//     last 2R of them to the next chunk's buffer, which needs Vx(t) on [xb+16-R, xb+16+R) for
//     the x-derivative of P; only Vz(t) is recomputed on a z halo (8 on each side of the strip);
//   * a first chunk per segment (c = -1) only computes Vx(t) on [xs-R, xs+R).
// Per chunk: phase A (Vx, x-stencil from a register window of P rows), phase B (Vz, z-stencil),
// phase C1 (rdx S-x Vx into a scratch block of shared memory), phase C2 (rdz S-z Vz, the P
// update, sponge, source injection and all global stores), then the receivers.  Stencil sums
// use paired FP32 instructions (FFMA2) over neighbouring z; in the z-stencils every other tap's
// operand pair straddles an 8-byte boundary and is assembled from the aligned window.  The
// divergence sx + sz is formed with scalar round-to-nearest adds, which the compiler never fuses
// with the products before them (a paired multiply feeding a paired add was fused into one FFMA2,
// which rounds once where the tile kernel rounds twice).
// With ADJ the same kernel runs the adjoint step, as the tile kernel's adjoint mode does: the P,
// Vx and Vz slots hold nu, X and Z, phase A stages B M (X + rdx S+x nu), phase B B M (Z + rdz S+z nu),
// phase C2 forms the new nu and the imaging sum g += nu_old D_k, and the receivers' residuals of
// the previous step are added at the end of the chunk.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "sfd_internal.h"

namespace sfd {
namespace {

constexpr int kThreads = 128;  // four warps
constexpr int TZ = 64;         // strip width (z)
constexpr int CH = 16;         // chunk (x columns)
constexpr int HZ = 16;         // z halo of the staged P
constexpr int VH = 8;          // z halo of the recomputed Vz
// P row pitch = box width: the z range z0-16 .. z0+80 plus 4 columns that are never read, so that
// in phase C2 (a quarter-warp = two neighbouring columns x four 8-wide z groups, 16-byte loads)
// the two columns fall on disjoint banks (pitch = 4 mod 8 words)
constexpr int PW = TZ + 2 * HZ + 4;    // 100
constexpr int PROWS = 2 * CH;          // 32: P columns per chunk (needs 2R <= CH)
constexpr int VXROWS = CH + 2 * 8;     // 32: Vx columns per buffer (R <= 8)
constexpr int NZV = TZ + 2 * VH;       // 80: Vz values per column
constexpr int ZW = NZV + 4;            // 84: Vz row pitch = box width (staggers rows over banks)
constexpr int KZB = NZV / 8;           // 10: phase B values per thread

struct ML {
    // floats; every TMA destination is 128-byte aligned
    static constexpr int P = 0;
    static constexpr int VX = P + PROWS * PW;          // 3200
    static constexpr int VZ = VX + VXROWS * TZ;        // 5120
    static constexpr int SET = VZ + CH * ZW;           // 6592 floats = 26368 bytes = 206 x 128
    static constexpr int TAB = 2 * SET;                // az[NZV], mz[NZV]
    static constexpr int BAR = TAB + 2 * NZV;          // two mbarriers (8 bytes each)
    static constexpr int FLOATS = BAR + 4;
    static constexpr unsigned TX_FULL = 4u * (PROWS * PW + CH * TZ + CH * ZW);
    static constexpr unsigned TX_FIRST = 4u * (PROWS * PW + CH * TZ);  // chunk -1: no Vz box
    static_assert((SET * 4) % 128 == 0, "buffer sets stay 128-byte aligned");
    static_assert((VX * 4) % 128 == 0 && (VZ * 4) % 128 == 0, "TMA destinations are 128-byte aligned");
};

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float2 ld2(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ void st2(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }
__device__ __forceinline__ float2 bc(float c) { return make_float2(c, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ unsigned sptr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }


__device__ __forceinline__ void tma_load_3d(float* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
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

// Sponge factor and update mask of column x (AFD:164-194; AFD updates only R <= i < N-R).
// ax < 0: the column is outside the x sponge (the z sponge or 1 applies).
template <int R>
__device__ __forceinline__ void col_tables(const Acou2DArgs& a, int x, int nx, float& ax, float& mx) {
    ax = -1.0f;
    mx = 0.0f;
    if (x >= 0 && x < nx) {
        if (x < a.pml) ax = a.sponge[a.pml - 1 - x];
        else if (x >= nx - a.pml) ax = a.sponge[x - (nx - a.pml)];
        mx = (x >= R && x < nx - R) ? 1.0f : 0.0f;
    }
}

// Segment geometry of one launch.
struct MarchGeo {
    int seg;      // columns per segment (multiple of CH)
    int nseg;     // segments per shot
    int nstrip;   // z strips per shot
};

template <int R, bool VARDEN, bool EDGE, bool ADJ>
__device__ __forceinline__ void chunk_body(const Acou2DArgs& a, float* smem, int set, const ShotDev& sd, int shot,
                                           int strip, int xs, int xe, int xb, bool first) {
    float* sP = smem + set * ML::SET + ML::P;
    float* sVx = smem + set * ML::SET + ML::VX;
    float* sVz = smem + set * ML::SET + ML::VZ;
    float* sVxNext = smem + (set ^ 1) * ML::SET + ML::VX;
    float* sX = sP + CH * PW + HZ;  // rdx S-x Vx of the chunk (P columns xb+16.. are dead after phase A)
    const float* sAz = smem + ML::TAB;
    const float* sMz = smem + ML::TAB + NZV;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nx = sd.nx, nz = a.nz;
    const int z0 = strip * TZ;
    const long long soff = (long long)shot * a.L.shot_stride;
    const int pitch = a.L.pitch;
    auto cell = [&](int x, int z) -> long long { return soff + (long long)(x + a.L.gx) * pitch + a.L.gz + z; };
    auto midx = [&](int x, int z) -> long long {
        return (long long)min(max(sd.x0 + x, 0), a.nx_model - 1) * a.mpitch + z;
    };

    // ---- phase A: Vx(t) on columns xb+R .. xb+R+16 (AFD:255-269); thread = z pair x 4 columns ----
    {
        const int zo = 2 * lane;
        const int r0 = 4 * warp;  // output o is Vx buffer column 2R + r0 + o, x = xb + R + r0 + o
        float2 w[2 * R + 3];      // P columns xb + r0 + 1 + j
#pragma unroll
        for (int j = 0; j < 2 * R + 3; j++) w[j] = ld2(sP + (r0 + 1 + j) * PW + HZ + zo);
        float2 az = bc(1.0f), mz = bc(1.0f);
        if (EDGE) {
            az = ld2(sAz + VH + zo);
            mz = ld2(sMz + VH + zo);
        }
#pragma unroll
        for (int o = 0; o < 4; o++) {
            const int x = xb + R + r0 + o;
            float2 s = mul2(a.coef2[0], sub2(w[o + R], w[o + R - 1]));
#pragma unroll
            for (int m = 1; m < R; m++) s = fma2(a.coef2[m], sub2(w[o + R + m], w[o + R - 1 - m]), s);
            float* vrow = sVx + (2 * R + r0 + o) * TZ + zo;
            float2 v = ld2(vrow);
            float2 b = bc(-a.bx_f), d = bc(a.den_c);
            if (VARDEN) {
                d = __ldg(reinterpret_cast<const float2*>(a.den + midx(x, z0 + zo)));
                b = make_float2(-a.dtdx / d.x, -a.dtdx / d.y);
            }
            float ax = -1.0f, mx = 1.0f;
            if (EDGE) col_tables<R>(a, x, nx, ax, mx);
            const float2 sa = EDGE ? (ax >= 0.0f ? bc(ax) : az) : bc(1.0f);
            float2 out = v;  // the value stored in the Vx (adjoint: X) field
            if (ADJ) {
                // staged X'' = B M (X + rdx S+x nu), B = dt / (dx den) (applied in phase C1 for
                // constant density); stored X = a M X' = a (den dx / dt) X'' (a alone for constant
                // density, where X'' = M X')
                v = fma2(bc(a.rdx_f), s, v);
                if (EDGE) v = mul2(v, mul2(bc(mx), mz));
                if (VARDEN) v = mul2(v, make_float2(-b.x, -b.y));
                out = VARDEN ? mul2(v, make_float2(sa.x * d.x * a.adj_xs, sa.y * d.y * a.adj_xs)) : mul2(v, sa);
            } else {
                if (EDGE) {
                    v = mul2(v, sa);
                    v = mul2(fma2(b, s, v), mul2(bc(mx), mz));
                } else {
                    v = fma2(b, s, v);
                }
                out = v;
            }
            st2(vrow, v);
            // the next chunk's buffer holds Vx(t) from column xb + 16 - R on
            if (2 * R + r0 + o >= CH) st2(sVxNext + (2 * R + r0 + o - CH) * TZ + zo, v);
            const int gz = z0 + zo;
            if (x >= xs && x < xe && x < nx && gz < nz) {
                float* dst = a.vx_out + cell(x, gz);
                if (gz + 1 < nz) st2(dst, out);
                else dst[0] = out.x;
            }
        }
    }
    if (first) return;  // chunk -1: only the Vx columns the first chunk needs

    // ---- phase B: Vz(t) on columns xb .. xb+16, z0-8 .. z0+72 (AFD:272-286); thread = column x 10 z ----
    {
        const int r = tid >> 3, zb = tid & 7;
        const int x = xb + r;
        const int c0 = KZB * zb;  // Vz column index: z = z0 - VH + c0 + j
        // window u[i] = P(x, z0 - HZ + c0 + i): P(z + 1 + m) = u[9 + j + m], P(z - m) = u[8 + j - m]
        constexpr int NW = KZB + 16;
        float2 u[NW / 2];
#pragma unroll
        for (int i = 0; i < NW / 2; i++) u[i] = ld2(sP + r * PW + c0 + 2 * i);
        auto uf = [&](int i) -> float { return (i & 1) ? u[i >> 1].y : u[i >> 1].x; };
        auto pr = [&](int i) -> float2 {  // (u[i], u[i+1]) as a register pair
            return (i & 1) ? make_float2(u[i >> 1].y, u[(i >> 1) + 1].x) : u[i >> 1];
        };
        float ax = -1.0f, mx = 1.0f;
        if (EDGE) col_tables<R>(a, x, nx, ax, mx);
        float* vrow = sVz + r * ZW + c0;
#pragma unroll
        for (int j = 0; j < KZB; j += 2) {
            float2 s = mul2(a.coef2[0], sub2(pr(9 + j), pr(8 + j)));
#pragma unroll
            for (int m = 1; m < R; m++) s = fma2(a.coef2[m], sub2(pr(9 + j + m), pr(8 + j - m)), s);
            float2 v = ld2(vrow + j);
            float2 nb = bc(-a.bz_f);
            if (VARDEN) {
                const int gz = z0 - VH + c0 + j;
                const long long mi = midx(x, gz);
                nb = make_float2(-(a.dtdz / __ldg(a.den + mi)), -(a.dtdz / __ldg(a.den + mi + 1)));
            }
            if (ADJ) {  // staged Z'' = B M (Z + rdz S+z nu)
                const float2 mz = EDGE ? make_float2(sMz[c0 + j], sMz[c0 + j + 1]) : bc(1.0f);
                const float2 cb = VARDEN ? make_float2(-nb.x, -nb.y) : bc(1.0f);
                v = make_float2(fmaf(a.rdz_f, s.x, v.x) * (mx * mz.x) * cb.x, fmaf(a.rdz_f, s.y, v.y) * (mx * mz.y) * cb.y);
            } else if (EDGE) {
                const float2 az = make_float2(sAz[c0 + j], sAz[c0 + j + 1]);
                const float2 mz = make_float2(sMz[c0 + j], sMz[c0 + j + 1]);
                v.x *= (ax >= 0.0f ? ax : az.x);
                v.y *= (ax >= 0.0f ? ax : az.y);
                v = make_float2(fmaf(nb.x, s.x, v.x) * (mx * mz.x), fmaf(nb.y, s.y, v.y) * (mx * mz.y));
            } else {
                v = make_float2(fmaf(nb.x, s.x, v.x), fmaf(nb.y, s.y, v.y));
            }
            st2(vrow + j, v);
        }
        (void)uf;
    }
    __syncthreads();  // Vx(t) and Vz(t) of the chunk are staged; P columns xb+16.. are free

    // ---- phase C1: rdx S-x Vx on columns xb .. xb+16 (AFD:289-297); thread = z pair x 4 columns ----
    {
        const int zo = 2 * lane, r0 = 4 * warp;
        float2 w[2 * R + 3];  // Vx buffer columns r0 + j, x = xb - R + r0 + j
#pragma unroll
        for (int j = 0; j < 2 * R + 3; j++) w[j] = ld2(sVx + (r0 + j) * TZ + zo);
#pragma unroll
        for (int o = 0; o < 4; o++) {
            float2 s = mul2(a.coef2[0], sub2(w[o + R], w[o + R - 1]));
#pragma unroll
            for (int m = 1; m < R; m++) s = fma2(a.coef2[m], sub2(w[o + R + m], w[o + R - m - 1]), s);
            st2(sX + (r0 + o) * PW + zo, mul2(s, bc(ADJ ? a.adj_cx : a.rdx_f)));
        }
    }
    __syncthreads();

    // ---- phase C2: P(t) on columns xb .. xb+16 (AFD:289-314, 337-338); thread = column x 8 z ----
    const int step = a.step;
    {
        // lane bits b4..b0: column 2 b4 + b2 of the warp's four, z group b1 b0 + 4 b3 (a quarter-warp
        // reads two columns whose rows sit 100 or 84 words apart: no bank is hit twice)
        const int r = 4 * warp + 2 * (lane >> 4) + ((lane >> 2) & 1), zq = (lane & 3) + 4 * ((lane >> 3) & 1);
        const int x = xb + r, zo = 8 * zq, gz = z0 + zo;
        // model values first: their latency is covered by the z-stencil
        float4 vp4[2], dn4[2];
        {
            const long long mi = midx(x, gz);
#pragma unroll
            for (int h = 0; h < 2; h++) {
                vp4[h] = __ldg(reinterpret_cast<const float4*>(a.vp + mi + 4 * h));
                dn4[h] = VARDEN ? __ldg(reinterpret_cast<const float4*>(a.den + mi + 4 * h))
                                : make_float4(a.den_c, a.den_c, a.den_c, a.den_c);
            }
        }
        // window u[i] = Vz(x, z0 + zo - 8 + i): Vz(z + m) = u[8 + j + m], Vz(z - m - 1) = u[7 + j - m]
        float2 u[12];
#pragma unroll
        for (int i = 0; i < 6; i++) {
            const float4 v = ld4(sVz + r * ZW + zo + 4 * i);
            u[2 * i] = make_float2(v.x, v.y);
            u[2 * i + 1] = make_float2(v.z, v.w);
        }
        auto pr = [&](int i) -> float2 {
            return (i & 1) ? make_float2(u[i >> 1].y, u[(i >> 1) + 1].x) : u[i >> 1];
        };
        float2 sz[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int j = 2 * q;
            float2 s = mul2(a.coef2[0], sub2(pr(8 + j), pr(7 + j)));
#pragma unroll
            for (int m = 1; m < R; m++) s = fma2(a.coef2[m], sub2(pr(8 + j + m), pr(7 + j - m)), s);
            sz[q] = s;  // scaled by rdz (adjoint: adj_cz) where it is added to the x part
        }
        float* pc = sP + r * PW + HZ + zo;
        const float* xc = sX + r * PW + zo;
        float pn[8], divv[8];
        float ax = -1.0f, mx = 1.0f;
        if (EDGE) col_tables<R>(a, x, nx, ax, mx);
        if (ADJ) {
            // the adjoint recurrence (stated in adjoint2d.cu): bracket = nu_old / K + S-x(B M X') +
            // S-z(B M Z'), nu_new = M a K bracket, g += nu_old D_k; stored Z = a M Z'
            const bool own = x < nx && gz < nz;
            const long long c = cell(x, gz);
            float4 dk[2], gk[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                dk[h] = gk[h] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (own && gz + 7 < nz) {
                    dk[h] = __ldg(reinterpret_cast<const float4*>(a.adj_div + c + 4 * h));
                    gk[h] = ld4(a.adj_g + c + 4 * h);
                }
            }
            float nn[8], zo8[8], po8[8], br8[8];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const float4 po = ld4(pc + 4 * h);
                const float4 sx4 = ld4(xc + 4 * h);
                const float4 vp = vp4[h], dn = dn4[h];
                const float2 kl = mul2(mul2(mul2(make_float2(dn.x, dn.y), make_float2(vp.x, vp.y)),
                                            make_float2(vp.x, vp.y)), bc(a.dt));
                const float2 kh = mul2(mul2(mul2(make_float2(dn.z, dn.w), make_float2(vp.z, vp.w)),
                                            make_float2(vp.z, vp.w)), bc(a.dt));
                const float cz = a.adj_cz;
                const float2 bl = make_float2(
                    __fadd_rn(__fadd_rn(sx4.x, __fmul_rn(sz[2 * h].x, cz)), __fdividef(po.x, kl.x)),
                    __fadd_rn(__fadd_rn(sx4.y, __fmul_rn(sz[2 * h].y, cz)), __fdividef(po.y, kl.y)));
                const float2 bh = make_float2(
                    __fadd_rn(__fadd_rn(sx4.z, __fmul_rn(sz[2 * h + 1].x, cz)), __fdividef(po.z, kh.x)),
                    __fadd_rn(__fadd_rn(sx4.w, __fmul_rn(sz[2 * h + 1].y, cz)), __fdividef(po.w, kh.y)));
                float4 fa4 = make_float4(1.f, 1.f, 1.f, 1.f), fm4 = fa4;  // sponge a and mask M of the cells
                if (EDGE) {
                    const float4 az = ld4(sAz + VH + zo + 4 * h), mz = ld4(sMz + VH + zo + 4 * h);
                    fa4 = ax >= 0.0f ? make_float4(ax, ax, ax, ax) : az;
                    fm4 = make_float4(mx * mz.x, mx * mz.y, mx * mz.z, mx * mz.w);
                }
                const float2 nl = mul2(mul2(bl, kl), mul2(make_float2(fa4.x, fa4.y), make_float2(fm4.x, fm4.y)));
                const float2 nh = mul2(mul2(bh, kh), mul2(make_float2(fa4.z, fa4.w), make_float2(fm4.z, fm4.w)));
                float4 zf = fa4;
                if (VARDEN)
                    zf = make_float4(fa4.x * dn.x * a.adj_zs, fa4.y * dn.y * a.adj_zs, fa4.z * dn.z * a.adj_zs,
                                     fa4.w * dn.w * a.adj_zs);
                const float4 zs = ld4(sVz + r * ZW + VH + zo + 4 * h);
                const float fzf[4] = {zf.x, zf.y, zf.z, zf.w}, fzs[4] = {zs.x, zs.y, zs.z, zs.w};
                const float fn[4] = {nl.x, nl.y, nh.x, nh.y}, fb[4] = {bl.x, bl.y, bh.x, bh.y};
                const float fp[4] = {po.x, po.y, po.z, po.w};
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    nn[4 * h + q] = fn[q];
                    zo8[4 * h + q] = fzs[q] * fzf[q];
                    po8[4 * h + q] = fp[q];
                    br8[4 * h + q] = fb[q];
                }
            }
            if (own) {
                if (x == sd.sx && sd.sz >= gz && sd.sz < gz + 8)
                    for (int q = 0; q < 8; q++)
                        if (sd.sz == gz + q) a.adj_lam[(long long)shot * a.nt_max + step] = br8[q];
                if (gz + 7 < nz) {
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const float4 d4 = dk[h], g4 = gk[h];
                        st4(a.adj_g + c + 4 * h, make_float4(fmaf(po8[4 * h], d4.x, g4.x), fmaf(po8[4 * h + 1], d4.y, g4.y),
                                                           fmaf(po8[4 * h + 2], d4.z, g4.z),
                                                           fmaf(po8[4 * h + 3], d4.w, g4.w)));
                        st4(a.p_out + c + 4 * h, make_float4(nn[4 * h], nn[4 * h + 1], nn[4 * h + 2], nn[4 * h + 3]));
                        st4(a.vz_out + c + 4 * h,
                            make_float4(zo8[4 * h], zo8[4 * h + 1], zo8[4 * h + 2], zo8[4 * h + 3]));
                    }
                } else {
                    for (int q = 0; q < 8 && gz + q < nz; q++) {
                        a.adj_g[c + q] = fmaf(po8[q], __ldg(a.adj_div + c + q), a.adj_g[c + q]);
                        a.p_out[c + q] = nn[q];
                        a.vz_out[c + q] = zo8[q];
                    }
                }
            }
        }
#pragma unroll
        for (int h = 0; h < 2 && !ADJ; h++) {
            const float4 po = ld4(pc + 4 * h);
            const float4 sx4 = ld4(xc + 4 * h);
            const float4 vp = vp4[h], dn = dn4[h];
            // -kk = -DEN * Vp * Vp * dt (AFD:293)
            const float2 kl = mul2(mul2(mul2(make_float2(dn.x, dn.y), make_float2(vp.x, vp.y)), make_float2(vp.x, vp.y)),
                                   bc(-a.dt));
            const float2 kh = mul2(mul2(mul2(make_float2(dn.z, dn.w), make_float2(vp.z, vp.w)), make_float2(vp.z, vp.w)),
                                   bc(-a.dt));
            const float cz = a.rdz_f;
            const float2 divl = make_float2(__fadd_rn(sx4.x, __fmul_rn(sz[2 * h].x, cz)),
                                            __fadd_rn(sx4.y, __fmul_rn(sz[2 * h].y, cz)));
            const float2 divh = make_float2(__fadd_rn(sx4.z, __fmul_rn(sz[2 * h + 1].x, cz)),
                                            __fadd_rn(sx4.w, __fmul_rn(sz[2 * h + 1].y, cz)));
            float2 pl = fma2(kl, divl, make_float2(po.x, po.y));
            float2 ph = fma2(kh, divh, make_float2(po.z, po.w));
            if (EDGE) {
                const float4 az = ld4(sAz + VH + zo + 4 * h), mz = ld4(sMz + VH + zo + 4 * h);
                const float4 sa = ax >= 0.0f ? make_float4(ax, ax, ax, ax) : az;
                pl = mul2(mul2(pl, make_float2(sa.x, sa.y)), mul2(bc(mx), make_float2(mz.x, mz.y)));
                ph = mul2(mul2(ph, make_float2(sa.z, sa.w)), mul2(bc(mx), make_float2(mz.z, mz.w)));
            }
            pn[4 * h] = pl.x; pn[4 * h + 1] = pl.y; pn[4 * h + 2] = ph.x; pn[4 * h + 3] = ph.y;
            divv[4 * h] = divl.x; divv[4 * h + 1] = divl.y; divv[4 * h + 2] = divh.x; divv[4 * h + 3] = divh.y;
            st4(pc + 4 * h, make_float4(pl.x, pl.y, ph.x, ph.y));  // receivers read the recorded value here
        }
        if (!ADJ && x < nx && gz < nz) {
            if (x == sd.sx && sd.sz >= gz && sd.sz < gz + 8 && step + 1 < sd.nt) {
                const float inj = sd.inj_scale * __ldg(a.wavelets + sd.wav_off + step + 1);
#pragma unroll
                for (int c = 0; c < 8; c++)
                    if (sd.sz == gz + c) {
                        if (a.src_pre) a.src_pre[shot] = pn[c];
                        pn[c] -= inj;
                    }
            }
            const long long c = cell(x, gz);
            const float4 vz0 = ld4(sVz + r * ZW + VH + zo), vz1 = ld4(sVz + r * ZW + VH + zo + 4);
            if (gz + 7 < nz) {
                st4(a.p_out + c, make_float4(pn[0], pn[1], pn[2], pn[3]));
                st4(a.p_out + c + 4, make_float4(pn[4], pn[5], pn[6], pn[7]));
                st4(a.vz_out + c, vz0);
                st4(a.vz_out + c + 4, vz1);
                if (a.div_out) {
                    st4(a.div_out + c, make_float4(divv[0], divv[1], divv[2], divv[3]));
                    st4(a.div_out + c + 4, make_float4(divv[4], divv[5], divv[6], divv[7]));
                }
            } else {
                const float vzs[8] = {vz0.x, vz0.y, vz0.z, vz0.w, vz1.x, vz1.y, vz1.z, vz1.w};
#pragma unroll
                for (int q = 0; q < 8; q++)
                    if (gz + q < nz) {
                        a.p_out[c + q] = pn[q];
                        a.vz_out[c + q] = vzs[q];
                        if (a.div_out) a.div_out[c + q] = divv[q];
                    }
            }
        }
    }
    const int* trp = a.tile_rec_ptr + sd.tile_rec_base + (xb / kTileX) * a.L.ntz + strip;
    const int rb = __ldg(trp), re = __ldg(trp + 1);
    // ---- adjoint: residual of step k-1 at the receivers of this chunk (AFD:376-377 transposed),
    // nu += M a K res; several receivers may share a cell, so the adds are atomic ----
    if (ADJ) {
        if (step >= 1 && re > rb) {
            __syncthreads();  // nu_new of the chunk is stored
            for (int j = rb + tid; j < re; j += kThreads) {
                const int ridx = a.tile_rec_idx[j];
                const int rx = a.rec_x[sd.rec_list + ridx];
                if (rx < xb || rx >= xb + CH) continue;
                const int rz = a.rec_z[sd.rec_list + ridx];
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
    // ---- receivers (AFD:376-377) of this chunk ----
    if (re > rb) {
        __syncthreads();
        for (int j = rb + tid; j < re; j += kThreads) {
            const int ridx = a.tile_rec_idx[j];
            const int rx = a.rec_x[sd.rec_list + ridx];
            if (rx < xb || rx >= xb + CH) continue;
            const int rz = a.rec_z[sd.rec_list + ridx];
            a.records[sd.rec_base + (long long)step * sd.nrec + ridx] = sP[(rx - xb) * PW + HZ + (rz - z0)];
        }
    }
}

template <int R, bool VARDEN, bool ADJ>
__global__ void __launch_bounds__(kThreads, 4)
acoustic2d_march_kernel(const __grid_constant__ Acou2DArgs a, int active, MarchGeo geo) {
    static_assert(2 * R <= CH && R <= 8, "one chunk carries the 2R columns of Vx the next one needs");
    extern __shared__ __align__(128) float smem[];
    const int tid = threadIdx.x;
    // CTA order: the active shots' copies of one (segment, strip) are consecutive
    const int slot = blockIdx.x % active;
    const int rest = blockIdx.x / active;
    const int strip = rest % geo.nstrip;
    const int seg = rest / geo.nstrip;
    const int shot = a.slot_to_shot[slot];
    const ShotDev sd = a.shots[shot];
    const int nx = sd.nx, nz = a.nz;
    const int xs = seg * geo.seg;
    // the launch also lets the next step's CTAs be scheduled; returning early counts as done
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (xs >= nx) return;
    const int xe = min(xs + geo.seg, (nx + CH - 1) / CH * CH);
    const int nch = (xe - xs) / CH;
    const int z0 = strip * TZ;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + ML::BAR);

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sptr(bars)) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sptr(bars + 1)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // z sponge and mask of the strip's Vz range z0-8 .. z0+72
    for (int i = tid; i < NZV; i += kThreads) {
        const int z = z0 - VH + i;
        float az = 1.0f, mz = 0.0f;
        if (z >= 0 && z < nz) {
            if (z < a.pml) az = a.sponge[a.pml - 1 - z];
            else if (z >= nz - a.pml) az = a.sponge[z - (nz - a.pml)];
            mz = (z >= R && z < nz - R) ? 1.0f : 0.0f;
        }
        smem[ML::TAB + i] = az;
        smem[ML::TAB + NZV + i] = mz;
    }
    __syncthreads();
    // every read of this step's inputs follows the previous step's completion
    asm volatile("griddepcontrol.wait;" ::: "memory");

    // the test hook: this CTA issues no loads and waits test_wait_ns instead of about one second
    const bool probed = (int)blockIdx.x == a.test_cta && a.step == a.test_step;
    const unsigned long long wait_ns = probed ? a.test_wait_ns : 1000000000ull;
    // thread 0: the boxes of chunk i - 1 (i = 0 is the first chunk, c = -1) into buffer set i & 1
    auto issue = [&](int i) {
        if (probed) return;
        const int set = i & 1;
        const int xb = xs + (i - 1) * CH;
        float* base = smem + set * ML::SET;
        uint64_t* bar = bars + set;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sptr(bar)),
                     "r"(i == 0 ? ML::TX_FIRST : ML::TX_FULL)
                     : "memory");
        const int gx = a.L.gx, gz = a.L.gz;
        tma_load_3d(base + ML::P, &a.tm_mp, gz + z0 - HZ, gx + xb, shot, bar);
        tma_load_3d(base + ML::VX + 2 * R * TZ, &a.tm_mvx, gz + z0, gx + xb + R, shot, bar);
        if (i > 0) tma_load_3d(base + ML::VZ, &a.tm_mvz, gz + z0 - VH, gx + xb, shot, bar);
    };
    if (tid == 0) issue(0);

    const int E = a.pml > R ? a.pml : R;
    const bool zedge = !(z0 - VH >= E && z0 + TZ + VH <= nz - E);
    for (int i = 0; i <= nch; i++) {
        const int set = i & 1;
        const unsigned par = (i >> 1) & 1;
        // bounded wait for this chunk's boxes (about one second of wall time, then give up): one
        // thread polls while the others wait in the barrier, which also ends the previous chunk
        auto bounded_wait = [&]() {
            bool ok = mbar_try_wait(bars + set, par);
            if (!ok) {
                const uint64_t t0 = global_ns();
                while (!(ok = mbar_try_wait(bars + set, par)) && global_ns() - t0 < wait_ns) {
                }
            }
            return ok;
        };
        bool done = true;
        if (tid == 0) done = bounded_wait();
        if (__syncthreads_or(!done)) {
            if (tid == 0) {
                atomicExch(a.err_flag, 1);
                bounded_wait();  // let copies still in flight land before the CTA's shared memory is released
            }
            return;
        }
        if (tid != 0) mbar_try_wait(bars + set, par);  // completed: observes the TMA writes
        // the other buffer set is free (chunk i - 1 has finished): start the next chunk's copies
        if (tid == 0 && i < nch) issue(i + 1);
        const int xb = xs + (i - 1) * CH;
        const bool xedge = !(xb >= E && xb + CH + R <= nx - E);
        if (zedge || xedge) chunk_body<R, VARDEN, true, ADJ>(a, smem, set, sd, shot, strip, xs, xe, xb, i == 0);
        else chunk_body<R, VARDEN, false, ADJ>(a, smem, set, sd, shot, strip, xs, xe, xb, i == 0);
    }
}

template <int R, bool VARDEN, bool ADJ>
cudaError_t launch_t(const Acou2DArgs& a, int active, int seg, cudaStream_t st, bool pdl) {
    const size_t smem = sizeof(float) * ML::FLOATS;
    auto k = acoustic2d_march_kernel<R, VARDEN, ADJ>;
    static bool attr[kMaxDevices] = {};
    if (cudaError_t e = smem_attr_once((const void*)k, (int)smem, attr)) return e;
    MarchGeo geo;
    geo.seg = seg;
    geo.nstrip = a.L.ntz;
    geo.nseg = (a.L.ntx * kTileX + seg - 1) / seg;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(active * geo.nstrip * geo.nseg));
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = pdl ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, a, active, geo);
}

template <int R>
cudaError_t launch_r(const Acou2DArgs& a, int active, bool varden, int seg, cudaStream_t st, bool pdl, bool adj) {
    if (adj)
        return varden ? launch_t<R, true, true>(a, active, seg, st, pdl) : launch_t<R, false, true>(a, active, seg, st, pdl);
    return varden ? launch_t<R, true, false>(a, active, seg, st, pdl) : launch_t<R, false, false>(a, active, seg, st, pdl);
}

}  // namespace

cudaError_t acoustic2d_march_launch(int radius, const Acou2DArgs& a, int active, bool varden, int seg_cols,
                                   cudaStream_t st, bool pdl, bool adj) {
    if (seg_cols < CH || seg_cols % CH != 0) return cudaErrorInvalidValue;
    if (a.L.tz != TZ || a.L.tx % CH != 0) return cudaErrorInvalidValue;
    switch (radius) {
    case 1: return launch_r<1>(a, active, varden, seg_cols, st, pdl, adj);
    case 2: return launch_r<2>(a, active, varden, seg_cols, st, pdl, adj);
    case 4: return launch_r<4>(a, active, varden, seg_cols, st, pdl, adj);
    case 5: return launch_r<5>(a, active, varden, seg_cols, st, pdl, adj);
    case 8: return launch_r<8>(a, active, varden, seg_cols, st, pdl, adj);
    default: return cudaErrorInvalidValue;
    }
}

bool acoustic2d_march_fills(const Layout2D& L, int active, int seg_cols) {
    static int nsm[kMaxDevices] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return true;
    if (nsm[dev] == 0 && cudaDeviceGetAttribute(&nsm[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        nsm[dev] = 0;
        return true;
    }
    const long long ctas = (long long)active * L.ntz * ((L.ntx * kTileX + seg_cols - 1) / seg_cols);
    return ctas >= 4LL * nsm[dev];  // one wave at four CTAs per SM
}

void acoustic2d_march_boxes(int box_p[2], int box_vx[2], int box_vz[2]) {
    box_p[0] = PW; box_p[1] = PROWS;
    box_vx[0] = TZ; box_vx[1] = CH;
    box_vz[0] = ZW; box_vz[1] = CH;
}

}  // namespace sfd
