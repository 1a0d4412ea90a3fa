// Fused time-step kernel of the 2-D acoustic velocity-pressure staggered-grid scheme of
// forward/Acoustic_FD_by_ss/src/Acoustic_1order_FD.cpp (AFD:237-380), batched over shots.
//
// One launch = one time step of every active shot.  A CTA owns a TX x TZ tile of one shot:
//   1. stage P(t) on the tile plus a 2R halo (a cross in x and z), Vx(t-1) on the tile plus
//      an R halo in x and Vz(t-1) plus an R halo in z into shared memory (float4 loads);
//   2. Vx(t) on tile+x-halo and Vz(t) on tile+z-halo (AFD:255-286), reading the old velocity
//      through the sponge (the lazy form of AFD:329-336, see below);
//   3. P(t) on the tile from the unsponged new velocities (AFD:289-314), sponge (AFD:337-338),
//      receiver extraction (AFD:376-377) and the source injection of step t+1 (AFD:247-251);
//   4. store P (sponged), Vx and Vz (unsponged) for the tile.
// Velocities are stored *before* the sponge multiply.  AFD multiplies Vx1 (and its copy
// Vx2) by absorb after P has been computed (AFD:329-336), so the next step's Vx2 equals
// stored * absorb, which step 2 computes with the same single rounding.  With EXACT the
// kernel keeps AFD's operation order (no FMA contraction, double-precision scale factors) and
// reproduces the reference bit for bit; without it the sums use FMA.
#include <cuda_runtime.h>

#include "sfd_internal.h"

namespace sfd {
namespace {

constexpr int kThreads = 256;

__host__ __device__ constexpr int round4(int v) { return (v + 3) & ~3; }


template <int R>
struct Tile {
    static constexpr int TX = kTileX;         // columns (x)
    static constexpr int TZ = kTileZ;         // rows (z, contiguous)
    static constexpr int HX = 2 * R;          // P halo along x
    static constexpr int HZ = round4(2 * R);  // P / Vz halo along z, rounded for float4
    static constexpr int SP_ROWS = TX + 2 * HX;
    static constexpr int SP_W = TZ + 2 * HZ;
    static constexpr int SVX_ROWS = TX + 2 * R;
    static constexpr int SVX_W = TZ;
    static constexpr int SVZ_ROWS = TX;
    static constexpr int SVZ_W = TZ + 2 * HZ;
    static constexpr int SMEM_FLOATS = SP_ROWS * SP_W + SVX_ROWS * SVX_W + SVZ_ROWS * SVZ_W + 256;
};

// AFD:164-194 sponge with overwrite semantics: the x edges win in the corners.
__device__ __forceinline__ float sponge_at(int x, int z, int nx, int nz, int pml, const float* tab) {
    if (x < pml) return tab[pml - 1 - x];
    if (x >= nx - pml) return tab[x - (nx - pml)];
    if (z < pml) return tab[pml - 1 - z];
    if (z >= nz - pml) return tab[z - (nz - pml)];
    return 1.0f;
}

template <int R, bool EXACT, bool VARDEN>
__global__ void __launch_bounds__(kThreads)
acoustic2d_step_kernel(const __grid_constant__ Acou2DArgs a) {
    using T = Tile<R>;
    extern __shared__ __align__(16) float smem[];
    float* sP = smem;                                // [SP_ROWS][SP_W]
    float* sVx = sP + T::SP_ROWS * T::SP_W;          // [SVX_ROWS][SVX_W]
    float* sVz = sVx + T::SVX_ROWS * T::SVX_W;       // [SVZ_ROWS][SVZ_W]
    float* sTab = sVz + T::SVZ_ROWS * T::SVZ_W;      // sponge profile

    const int shot = a.slot_to_shot[blockIdx.y];
    const ShotDev sd = a.shots[shot];
    const int tile = blockIdx.x;
    const int tx_i = tile / a.L.ntz, tz_i = tile - tx_i * a.L.ntz;
    if (tx_i * T::TX >= sd.nx) return;  // tile beyond this shot's aperture
    const int x0 = tx_i * T::TX, z0 = tz_i * T::TZ;
    const int nx = sd.nx, nz = a.nz, pml = a.pml;
    const int tid = threadIdx.x;

    const long long soff = (long long)shot * a.L.shot_stride;
    const int pitch = a.L.pitch;
    // address of cell (x, z) inside this shot's slab
    auto cell = [&](int x, int z) -> long long { return soff + (long long)(x + a.L.gx) * pitch + a.L.gz + z; };

    for (int i = tid; i < pml && i < 256; i += kThreads) sTab[i] = a.sponge[i];

    // ---- stage P(t): rows x0-HX .. x0+TX+HX, z0-HZ .. z0+TZ+HZ ----
    {
        constexpr int W4 = T::SP_W / 4;
        for (int i = tid; i < T::SP_ROWS * W4; i += kThreads) {
            const int r = i / W4, c = i - r * W4;
            const float4 v = __ldg(reinterpret_cast<const float4*>(a.p_in + cell(x0 - T::HX + r, z0 - T::HZ + 4 * c)));
            *reinterpret_cast<float4*>(sP + r * T::SP_W + 4 * c) = v;
        }
    }
    // ---- stage Vx(t-1): rows x0-R .. x0+TX+R, z0 .. z0+TZ ----
    {
        constexpr int W4 = T::SVX_W / 4;
        for (int i = tid; i < T::SVX_ROWS * W4; i += kThreads) {
            const int r = i / W4, c = i - r * W4;
            const float4 v = __ldg(reinterpret_cast<const float4*>(a.vx_in + cell(x0 - R + r, z0 + 4 * c)));
            *reinterpret_cast<float4*>(sVx + r * T::SVX_W + 4 * c) = v;
        }
    }
    // ---- stage Vz(t-1): rows x0 .. x0+TX, z0-HZ .. z0+TZ+HZ ----
    {
        constexpr int W4 = T::SVZ_W / 4;
        for (int i = tid; i < T::SVZ_ROWS * W4; i += kThreads) {
            const int r = i / W4, c = i - r * W4;
            const float4 v = __ldg(reinterpret_cast<const float4*>(a.vz_in + cell(x0 + r, z0 - T::HZ + 4 * c)));
            *reinterpret_cast<float4*>(sVz + r * T::SVZ_W + 4 * c) = v;
        }
    }
    __syncthreads();

    float C[R];
#pragma unroll
    for (int m = 0; m < R; m++) C[m] = a.coef[m];

    // ---- Vx(t) on rows x0-R .. x0+TX+R (AFD:255-269) ----
    for (int i = tid; i < T::SVX_ROWS * T::TZ; i += kThreads) {
        const int r = i / T::TZ, z = i - r * T::TZ;
        const int gx = x0 - R + r, gz = z0 + z;
        float vnew = 0.0f;
        if (gx >= R && gx < nx - R && gz >= R && gz < nz - R) {
            const float* pr = sP + (r + R) * T::SP_W + z + T::HZ;  // P row of gx
            const float sa = sponge_at(gx, gz, nx, nz, pml, sTab);
            const float vold = sVx[r * T::SVX_W + z];
            if (EXACT) {
                float s = __fmul_rn(C[0], __fsub_rn(pr[T::SP_W], pr[0]));
#pragma unroll
                for (int m = 1; m < R; m++)
                    s = __fadd_rn(s, __fmul_rn(C[m], __fsub_rn(pr[(m + 1) * T::SP_W], pr[-m * T::SP_W])));
                double b = a.bx_d;
                if (VARDEN) {
                    const float d = __ldg(a.den + (long long)min(sd.x0 + gx, a.nx_model - 1) * a.mpitch + gz);
                    b = __dmul_rn(__drcp_rn((double)d), (double)a.dtdx);
                }
                vnew = __double2float_rn(__dsub_rn((double)__fmul_rn(vold, sa), __dmul_rn(b, (double)s)));
            } else {
                float s = C[0] * (pr[T::SP_W] - pr[0]);
#pragma unroll
                for (int m = 1; m < R; m++) s = fmaf(C[m], pr[(m + 1) * T::SP_W] - pr[-m * T::SP_W], s);
                float b = a.bx_f;
                if (VARDEN) {
                    const float d = __ldg(a.den + (long long)min(sd.x0 + gx, a.nx_model - 1) * a.mpitch + gz);
                    b = a.dtdx / d;
                }
                vnew = fmaf(-b, s, vold * sa);
            }
        }
        sVx[r * T::SVX_W + z] = vnew;
    }
    // ---- Vz(t) on columns x0 .. x0+TX, rows z0-R .. z0+TZ+R (AFD:272-286) ----
    for (int i = tid; i < T::TX * (T::TZ + 2 * R); i += kThreads) {
        const int r = i / (T::TZ + 2 * R), zz = i - r * (T::TZ + 2 * R);
        const int gx = x0 + r, gz = z0 - R + zz;
        const int zs = zz - R + T::HZ;  // index within the staged rows
        float vnew = 0.0f;
        if (gx >= R && gx < nx - R && gz >= R && gz < nz - R) {
            const float* pc = sP + (r + T::HX) * T::SP_W + zs;
            const float sa = sponge_at(gx, gz, nx, nz, pml, sTab);
            const float vold = sVz[r * T::SVZ_W + zs];
            if (EXACT) {
                float s = __fmul_rn(C[0], __fsub_rn(pc[1], pc[0]));
#pragma unroll
                for (int m = 1; m < R; m++) s = __fadd_rn(s, __fmul_rn(C[m], __fsub_rn(pc[m + 1], pc[-m])));
                double b = a.bz_d;
                if (VARDEN) {
                    const float d = __ldg(a.den + (long long)min(sd.x0 + gx, a.nx_model - 1) * a.mpitch + gz);
                    b = __dmul_rn(__drcp_rn((double)d), (double)a.dtdz);
                }
                vnew = __double2float_rn(__dsub_rn((double)__fmul_rn(vold, sa), __dmul_rn(b, (double)s)));
            } else {
                float s = C[0] * (pc[1] - pc[0]);
#pragma unroll
                for (int m = 1; m < R; m++) s = fmaf(C[m], pc[m + 1] - pc[-m], s);
                float b = a.bz_f;
                if (VARDEN) {
                    const float d = __ldg(a.den + (long long)min(sd.x0 + gx, a.nx_model - 1) * a.mpitch + gz);
                    b = a.dtdz / d;
                }
                vnew = fmaf(-b, s, vold * sa);
            }
        }
        sVz[r * T::SVZ_W + zs] = vnew;
    }
    __syncthreads();

    // ---- P(t) on the tile (AFD:289-314), sponge (AFD:337-338), stores ----
    const int step = a.step;
    for (int i = tid; i < T::TX * T::TZ; i += kThreads) {
        const int r = i / T::TZ, z = i - r * T::TZ;
        const int gx = x0 + r, gz = z0 + z;
        float* pcell = sP + (r + T::HX) * T::SP_W + z + T::HZ;
        const float* vxr = sVx + (r + R) * T::SVX_W + z;
        const float* vzc = sVz + r * T::SVZ_W + z + T::HZ;
        float pn = 0.0f;
        if (gx >= R && gx < nx - R && gz >= R && gz < nz - R) {
            const long long mi = (long long)min(sd.x0 + gx, a.nx_model - 1) * a.mpitch + gz;
            const float vp = __ldg(a.vp + mi);
            const float den = VARDEN ? __ldg(a.den + mi) : a.den_c;
            const float sa = sponge_at(gx, gz, nx, nz, pml, sTab);
            const float pold = *pcell;
            if (EXACT) {
                float sx = __fmul_rn(C[0], __fsub_rn(vxr[0], vxr[-T::SVX_W]));
                float sz = __fmul_rn(C[0], __fsub_rn(vzc[0], vzc[-1]));
#pragma unroll
                for (int m = 1; m < R; m++) {
                    sx = __fadd_rn(sx, __fmul_rn(C[m], __fsub_rn(vxr[m * T::SVX_W], vxr[-(m + 1) * T::SVX_W])));
                    sz = __fadd_rn(sz, __fmul_rn(C[m], __fsub_rn(vzc[m], vzc[-(m + 1)])));
                }
                const float kk = __fmul_rn(__fmul_rn(__fmul_rn(den, vp), vp), a.dt);
                const double div = __dadd_rn(__dmul_rn(a.rdx_d, (double)sx), __dmul_rn(a.rdz_d, (double)sz));
                const float p1 = __double2float_rn(__dsub_rn((double)pold, __dmul_rn((double)kk, div)));
                pn = __fmul_rn(p1, sa);
            } else {
                float sx = C[0] * (vxr[0] - vxr[-T::SVX_W]);
                float sz = C[0] * (vzc[0] - vzc[-1]);
#pragma unroll
                for (int m = 1; m < R; m++) {
                    sx = fmaf(C[m], vxr[m * T::SVX_W] - vxr[-(m + 1) * T::SVX_W], sx);
                    sz = fmaf(C[m], vzc[m] - vzc[-(m + 1)], sz);
                }
                const float kk = den * vp * vp * a.dt;
                pn = fmaf(-kk, fmaf(sx, a.rdx_f, sz * a.rdz_f), pold) * sa;
            }
        }
        *pcell = pn;  // receivers read the recorded (pre-injection) value from here
        if (gx < nx && gz < nz) {
            float pw = pn;
            if (gx == sd.sx && gz == sd.sz && step + 1 < sd.nt) {
                const float w = __ldg(a.wavelets + sd.wav_off + step + 1);
                pw = EXACT ? __fsub_rn(pn, __fmul_rn(sd.inj_scale, w)) : pn - sd.inj_scale * w;
            }
            const long long c = cell(gx, gz);
            a.p_out[c] = pw;
            a.vx_out[c] = vxr[0];
            a.vz_out[c] = vzc[0];
        }
    }
    // ---- receivers (AFD:376-377) ----
    const int* trp = a.tile_rec_ptr + sd.tile_rec_base + tile;
    const int rb = trp[0], re = trp[1];
    if (re > rb) {
        __syncthreads();
        for (int j = rb + tid; j < re; j += kThreads) {
            const int ridx = a.tile_rec_idx[j];
            const int rx = a.rec_x[sd.rec_list + ridx], rz = a.rec_z[sd.rec_list + ridx];
            a.records[sd.rec_base + (long long)step * sd.nrec + ridx] =
                sP[(rx - x0 + T::HX) * T::SP_W + (rz - z0) + T::HZ];
        }
    }
}

// ------------------------------------------------------------------------------------------
// FMA step kernel with register micro-tiles.
//
// Same tile, same staging and the same update semantics as the kernel above, but every thread
// computes a small block of outputs from a sliding window of float4 z-vectors held in
// registers, so each staged value is read from shared memory a few times instead of 2R times:
//   Vx  (x stencil): 1 z-vector x 5 rows,  window of 2R+4 rows        (lanes along z)
//   Vz  (z stencil): 1 row x 20 z,         window of 20+2RQ z          (lanes along x)
//   P   (both):      4 rows x 1 z-vector,  windows of 2R+3 rows of Vx and 4+2RQ z of Vz
// Row pitches are chosen with pitch/4 odd so that 8 lanes reading 16-byte vectors from 8
// different rows hit 8 different bank groups.
// ------------------------------------------------------------------------------------------
__host__ __device__ constexpr int odd_quads(int w) { return ((w / 4) % 2 == 1) ? w : w + 4; }

template <int R>
struct Tile2 {
    static constexpr int TX = kTileX, TZ = kTileZ;
    static constexpr int RQ = round4(R);        // z halo of the velocity region
    static constexpr int HZ = 2 * RQ;           // z halo of the staged pressure
    static constexpr int HX = 2 * R;            // x halo of the staged pressure
    static constexpr int SP_ROWS = TX + 2 * HX, SP_W = TZ + 2 * HZ, SP_P = odd_quads(SP_W);
    static constexpr int SVX_ROWS = TX + 2 * R, SVX_P = odd_quads(TZ);
    static constexpr int SVZ_W = TZ + 2 * RQ, SVZ_P = odd_quads(SVZ_W);
    static constexpr int NXV = TX + 2 * R;      // rows of the Vx region (sponge/mask tables)
    static constexpr int NZV = TZ + 2 * RQ;     // z of the Vz region (sponge/mask tables)
    static constexpr int KX = 5;                // Vx rows per thread
    static constexpr int VX_BLOCKS = (SVX_ROWS + KX - 1) / KX;
    static constexpr int KZ4 = 5;               // Vz z-vectors per thread
    static constexpr int VZ_BLOCKS = (NZV / 4 + KZ4 - 1) / KZ4;
    static constexpr int PAD = 64;              // slack after each array for clamped window reads
    static constexpr int OFF_VX = SP_ROWS * SP_P + PAD;
    static constexpr int OFF_VZ = OFF_VX + SVX_ROWS * SVX_P + PAD;
    static constexpr int OFF_AX = OFF_VZ + TX * SVZ_P + PAD;
    static constexpr int OFF_MX = OFF_AX + round4(NXV);
    static constexpr int OFF_AZ = OFF_MX + round4(NXV);
    static constexpr int OFF_MZ = OFF_AZ + round4(NZV);
    static constexpr int SMEM_FLOATS = OFF_MZ + round4(NZV);
};

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float4 sub4(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
__device__ __forceinline__ float4 mul4(float c, float4 a) { return make_float4(c * a.x, c * a.y, c * a.z, c * a.w); }
__device__ __forceinline__ float4 fma4(float c, float4 a, float4 b) {
    return make_float4(fmaf(c, a.x, b.x), fmaf(c, a.y, b.y), fmaf(c, a.z, b.z), fmaf(c, a.w, b.w));
}
__device__ __forceinline__ float comp(float4 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w)); }

// Asynchronous global -> shared copy of a ROWS x (4*W4) block (rows `gpitch` floats apart in
// global memory, SPITCH floats apart in shared memory), 16 bytes per copy, L2-only caching.
template <int ROWS, int W4, int SPITCH>
__device__ __forceinline__ void stage_async(float* dst, const float* src, int gpitch, int tid) {
    constexpr int N = ROWS * W4;
#pragma unroll 4
    for (int i = tid; i < N; i += kThreads) {
        const int r = i / W4, c = i - r * W4;
        const unsigned saddr = (unsigned)__cvta_generic_to_shared(dst + r * SPITCH + 4 * c);
        const float* g = src + (long long)r * gpitch + 4 * c;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(g) : "memory");
    }
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <int R, bool VARDEN>
__global__ void __launch_bounds__(kThreads, 2)
acoustic2d_step_fma_kernel(const __grid_constant__ Acou2DArgs a) {
    using T = Tile2<R>;
    extern __shared__ __align__(16) float smem[];
    float* sP = smem;
    float* sVx = smem + T::OFF_VX;
    float* sVz = smem + T::OFF_VZ;
    float* sAx = smem + T::OFF_AX;   // x sponge value for x edges, -1 elsewhere; index x - (x0 - R)
    float* sMx = smem + T::OFF_MX;   // 1 where the column is updated (R <= x < nx - R)
    float* sAz = smem + T::OFF_AZ;   // z sponge value (1 inside); index z - (z0 - RQ)
    float* sMz = smem + T::OFF_MZ;

    const int shot = a.slot_to_shot[blockIdx.y];
    const ShotDev sd = a.shots[shot];
    const int tile = blockIdx.x;
    const int tx_i = tile / a.L.ntz, tz_i = tile - tx_i * a.L.ntz;
    if (tx_i * T::TX >= sd.nx) return;
    const int x0 = tx_i * T::TX, z0 = tz_i * T::TZ;
    const int nx = sd.nx, nz = a.nz, pml = a.pml;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long soff = (long long)shot * a.L.shot_stride;
    const int pitch = a.L.pitch;
    auto cell = [&](int x, int z) -> long long { return soff + (long long)(x + a.L.gx) * pitch + a.L.gz + z; };

    // ---- sponge / update-mask tables (AFD:164-194; AFD updates only R <= i,j < N-R) ----
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
    // ---- stage P(t), Vx(t-1), Vz(t-1): 16-byte asynchronous copies, all in flight at once ----
    stage_async<T::SP_ROWS, T::SP_W / 4, T::SP_P>(sP, a.p_in + cell(x0 - T::HX, z0 - T::HZ), pitch, tid);
    stage_async<T::SVX_ROWS, T::TZ / 4, T::SVX_P>(sVx, a.vx_in + cell(x0 - R, z0), pitch, tid);
    stage_async<T::TX, T::SVZ_W / 4, T::SVZ_P>(sVz, a.vz_in + cell(x0, z0 - T::RQ), pitch, tid);
    cp_async_wait_all();
    __syncthreads();

    float C[R];
#pragma unroll
    for (int m = 0; m < R; m++) C[m] = a.coef[m];

    // ---- Vx(t) on rows x0-R .. x0+TX+R, one z-vector x KX rows per thread (AFD:255-269) ----
    for (int blk = tid; blk < 16 * T::VX_BLOCKS; blk += kThreads) {
        // 8 consecutive lanes -> 8 consecutive z-vectors of one row (conflict-free 16-byte loads)
        const int zgv = (blk & 7) + 8 * ((blk >> 3) / T::VX_BLOCKS);
        const int xbb = (blk >> 3) % T::VX_BLOCKS;
        const int r0 = xbb * T::KX;
        const int zo = 4 * zgv;  // z offset inside the tile
        float4 w[T::KX + 2 * R - 1];
#pragma unroll
        for (int j = 0; j < T::KX + 2 * R - 1; j++) {
            const int row = min(r0 + 1 + j, T::SP_ROWS - 1);
            w[j] = ld4(sP + row * T::SP_P + T::HZ + zo);
        }
        const float4 az = ld4(sAz + T::RQ + zo), mz = ld4(sMz + T::RQ + zo);
        float4 dz4 = make_float4(a.den_c, a.den_c, a.den_c, a.den_c);
#pragma unroll
        for (int o = 0; o < T::KX; o++) {
            const int row = r0 + o;
            if (row < T::SVX_ROWS) {
                float4 s = mul4(C[0], sub4(w[o + R], w[o + R - 1]));
#pragma unroll
                for (int m = 1; m < R; m++) s = fma4(C[m], sub4(w[o + R + m], w[o + R - 1 - m]), s);
                const float ax = sAx[row], mx = sMx[row];
                const float4 sa = ax >= 0.0f ? make_float4(ax, ax, ax, ax) : az;
                const float4 vo = ld4(sVx + row * T::SVX_P + zo);
                float4 b4 = make_float4(a.bx_f, a.bx_f, a.bx_f, a.bx_f);
                if (VARDEN) {
                    const int gx = min(max(sd.x0 + x0 - R + row, 0), a.nx_model - 1);
                    dz4 = __ldg(reinterpret_cast<const float4*>(a.den + (long long)gx * a.mpitch + z0 + zo));
                    b4 = make_float4(a.dtdx / dz4.x, a.dtdx / dz4.y, a.dtdx / dz4.z, a.dtdx / dz4.w);
                }
                float4 vn;
                vn.x = fmaf(-b4.x, s.x, vo.x * sa.x) * (mx * mz.x);
                vn.y = fmaf(-b4.y, s.y, vo.y * sa.y) * (mx * mz.y);
                vn.z = fmaf(-b4.z, s.z, vo.z * sa.z) * (mx * mz.z);
                vn.w = fmaf(-b4.w, s.w, vo.w * sa.w) * (mx * mz.w);
                st4(sVx + row * T::SVX_P + zo, vn);
            }
        }
    }
    // ---- Vz(t) on columns x0 .. x0+TX, z0-RQ .. z0+TZ+RQ, one row x 4*KZ4 z per thread ----
    for (int blk = tid; blk < T::TX * T::VZ_BLOCKS; blk += kThreads) {
        const int xr = blk % T::TX;          // consecutive lanes -> consecutive rows
        const int zb = blk / T::TX;
        const int zs = 4 * T::KZ4 * zb;      // first output, index into the Vz region
        constexpr int NW = T::KZ4 + T::RQ / 2;  // float4 in the window
        float wf[4 * NW];
#pragma unroll
        for (int j = 0; j < NW; j++) {
            // window starts RQ before the first output: sP z index HZ - 2RQ + zs + 4j = zs + 4j
            const float4 v = ld4(sP + (xr + T::HX) * T::SP_P + min(zs + 4 * j, T::SP_P - 4));
            wf[4 * j] = v.x; wf[4 * j + 1] = v.y; wf[4 * j + 2] = v.z; wf[4 * j + 3] = v.w;
        }
        const float ax = sAx[xr + R], mx = sMx[xr + R];
        float bz = a.bz_f;
#pragma unroll
        for (int g = 0; g < T::KZ4; g++) {
            const int zi = zs + 4 * g;       // index into the Vz region (z = z0 - RQ + zi)
            if (zi < T::NZV) {
                const float4 vo = ld4(sVz + xr * T::SVZ_P + zi);
                const float4 az = ld4(sAz + zi), mz = ld4(sMz + zi);
                float4 dz4 = make_float4(a.den_c, a.den_c, a.den_c, a.den_c);
                if (VARDEN) {
                    const int gx = min(sd.x0 + x0 + xr, a.nx_model - 1);
                    dz4 = __ldg(reinterpret_cast<const float4*>(a.den + (long long)gx * a.mpitch + z0 - T::RQ + zi));
                }
                float out[4];
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const int k = 4 * g + c;  // output index; P[z + d] = wf[RQ + k + d]
                    float s = C[0] * (wf[T::RQ + k + 1] - wf[T::RQ + k]);
#pragma unroll
                    for (int m = 1; m < R; m++) s = fmaf(C[m], wf[T::RQ + k + m + 1] - wf[T::RQ + k - m], s);
                    const float sa = ax >= 0.0f ? ax : comp(az, c);
                    if (VARDEN) bz = a.dtdz / comp(dz4, c);
                    out[c] = fmaf(-bz, s, comp(vo, c) * sa) * (mx * comp(mz, c));
                }
                st4(sVz + xr * T::SVZ_P + zi, make_float4(out[0], out[1], out[2], out[3]));
            }
        }
    }
    __syncthreads();

    // ---- P(t) on the tile, 4 rows x one z-vector per thread (AFD:289-314, 337-338) ----
    const int step = a.step;
    {
        const int zgv = (tid & 7) + 8 * (warp & 1);      // z-vector (lanes 0-7 consecutive)
        const int xbv = (lane >> 3) + 4 * (warp >> 1);   // block of 4 rows
        const int zo = 4 * zgv, r0 = 4 * xbv;  // tile-relative
        float4 sx[4];
        {
            float4 vw[2 * R + 3];
#pragma unroll
            for (int j = 0; j < 2 * R + 3; j++) vw[j] = ld4(sVx + (r0 + j) * T::SVX_P + zo);
#pragma unroll
            for (int o = 0; o < 4; o++) {
                float4 s = mul4(C[0], sub4(vw[o + R], vw[o + R - 1]));
#pragma unroll
                for (int m = 1; m < R; m++) s = fma4(C[m], sub4(vw[o + R + m], vw[o + R - m - 1]), s);
                sx[o] = s;
            }
#pragma unroll
            for (int o = 0; o < 4; o++) {
                const int gx = x0 + r0 + o, gz = z0 + zo;
                if (gx < nx && gz < nz) {
                    const float4 v = vw[o + R];
                    const long long c = cell(gx, gz);
                    if (gz + 3 < nz) *reinterpret_cast<float4*>(a.vx_out + c) = v;
                    else for (int q = 0; q < 4 && gz + q < nz; q++) a.vx_out[c + q] = comp(v, q);
                }
            }
        }
        const float4 az = ld4(sAz + T::RQ + zo), mz = ld4(sMz + T::RQ + zo);
#pragma unroll
        for (int o = 0; o < 4; o++) {
            const int row = r0 + o, gx = x0 + row, gz = z0 + zo;
            constexpr int NW = 1 + T::RQ / 2;
            float zf[4 * NW];
#pragma unroll
            for (int j = 0; j < NW; j++) {
                const float4 v = ld4(sVz + row * T::SVZ_P + zo + 4 * j);
                zf[4 * j] = v.x; zf[4 * j + 1] = v.y; zf[4 * j + 2] = v.z; zf[4 * j + 3] = v.w;
            }
            float* pc = sP + (row + T::HX) * T::SP_P + T::HZ + zo;
            const float4 po = ld4(pc);
            const float ax = sAx[row + R], mx = sMx[row + R];
            const int gxm = min(sd.x0 + gx, a.nx_model - 1);
            const float4 vp4 = __ldg(reinterpret_cast<const float4*>(a.vp + (long long)gxm * a.mpitch + gz));
            float4 dn4 = make_float4(a.den_c, a.den_c, a.den_c, a.den_c);
            if (VARDEN) dn4 = __ldg(reinterpret_cast<const float4*>(a.den + (long long)gxm * a.mpitch + gz));
            float pn[4];
#pragma unroll
            for (int c = 0; c < 4; c++) {
                float sz = C[0] * (zf[T::RQ + c] - zf[T::RQ + c - 1]);
#pragma unroll
                for (int m = 1; m < R; m++) sz = fmaf(C[m], zf[T::RQ + c + m] - zf[T::RQ + c - m - 1], sz);
                const float vp = comp(vp4, c);
                const float kk = comp(dn4, c) * vp * vp * a.dt;
                const float sa = ax >= 0.0f ? ax : comp(az, c);
                pn[c] = fmaf(-kk, fmaf(comp(sx[o], c), a.rdx_f, sz * a.rdz_f), comp(po, c)) * sa * (mx * comp(mz, c));
            }
            st4(pc, make_float4(pn[0], pn[1], pn[2], pn[3]));  // receivers read the recorded value here
            if (gx < nx && gz < nz) {
                if (gx == sd.sx && sd.sz >= gz && sd.sz < gz + 4 && step + 1 < sd.nt) {
                    const float inj = sd.inj_scale * __ldg(a.wavelets + sd.wav_off + step + 1);
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        if (sd.sz == gz + c) pn[c] -= inj;
                }
                const long long c = cell(gx, gz);
                const float4 vzc = make_float4(zf[T::RQ], zf[T::RQ + 1], zf[T::RQ + 2], zf[T::RQ + 3]);
                if (gz + 3 < nz) {
                    *reinterpret_cast<float4*>(a.p_out + c) = make_float4(pn[0], pn[1], pn[2], pn[3]);
                    *reinterpret_cast<float4*>(a.vz_out + c) = vzc;
                } else {
                    for (int q = 0; q < 4 && gz + q < nz; q++) {
                        a.p_out[c + q] = pn[q];
                        a.vz_out[c + q] = comp(vzc, q);
                    }
                }
            }
        }
    }
    // ---- receivers (AFD:376-377) ----
    const int* trp = a.tile_rec_ptr + sd.tile_rec_base + tile;
    const int rb = trp[0], re = trp[1];
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

// Step-0 source injection into the zeroed P(0): P2[src] = 0 - ((dt*DEN)*Vp)*signal[0].
__global__ void inject0_kernel(const __grid_constant__ Acou2DArgs a, int nshot, bool exact) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nshot) return;
    const ShotDev sd = a.shots[s];
    const float w = a.wavelets[sd.wav_off];
    const long long c = (long long)s * a.L.shot_stride + (long long)(sd.sx + a.L.gx) * a.L.pitch + a.L.gz + sd.sz;
    a.p_out[c] = exact ? __fsub_rn(0.0f, __fmul_rn(sd.inj_scale, w)) : -(sd.inj_scale * w);
}

template <int R, bool EXACT, bool VARDEN>
cudaError_t launch_t(const Acou2DArgs& a, int active, cudaStream_t st) {
    // the reference-order path keeps the plain kernel; the FMA path uses register micro-tiles
    const size_t smem = sizeof(float) * (EXACT ? Tile<R>::SMEM_FLOATS : Tile2<R>::SMEM_FLOATS);
    auto k = EXACT ? acoustic2d_step_kernel<R, true, VARDEN> : acoustic2d_step_fma_kernel<R, VARDEN>;
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    dim3 grid(a.L.ntx * a.L.ntz, active);
    k<<<grid, kThreads, smem, st>>>(a);
    return cudaGetLastError();
}

template <int R>
cudaError_t launch_r(const Acou2DArgs& a, int active, bool exact, bool varden, cudaStream_t st) {
    if (exact) return varden ? launch_t<R, true, true>(a, active, st) : launch_t<R, true, false>(a, active, st);
    return varden ? launch_t<R, false, true>(a, active, st) : launch_t<R, false, false>(a, active, st);
}

}  // namespace

bool acoustic2d_plan(int radius, Acou2DPlan* plan) {
    switch (radius) {
#define SFD_PLAN(RR)                                                  \
    case RR:                                                          \
        plan->radius = RR;                                            \
        plan->tx = Tile<RR>::TX;                                      \
        plan->tz = Tile<RR>::TZ;                                      \
        plan->threads = kThreads;                                     \
        plan->smem_bytes = sizeof(float) * Tile2<RR>::SMEM_FLOATS;    \
        plan->gz = Tile2<RR>::HZ;                                     \
        return true;
        SFD_PLAN(1) SFD_PLAN(2) SFD_PLAN(4) SFD_PLAN(5) SFD_PLAN(8)
#undef SFD_PLAN
    default:
        return false;
    }
}

cudaError_t acoustic2d_launch_step(const Acou2DPlan& plan, const Acou2DArgs& a, int active, bool exact,
                                   bool varden, cudaStream_t st) {
    switch (plan.radius) {
    case 1: return launch_r<1>(a, active, exact, varden, st);
    case 2: return launch_r<2>(a, active, exact, varden, st);
    case 4: return launch_r<4>(a, active, exact, varden, st);
    case 5: return launch_r<5>(a, active, exact, varden, st);
    case 8: return launch_r<8>(a, active, exact, varden, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t acoustic2d_launch_inject0(const Acou2DArgs& a, int nshot, bool exact, cudaStream_t st) {
    inject0_kernel<<<(nshot + 127) / 128, 128, 0, st>>>(a, nshot, exact);
    return cudaGetLastError();
}

}  // namespace sfd
