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
                if (a.src_pre) a.src_pre[shot] = pn;
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
    // the reference-order kernel; the FMA path lives in acoustic2d_fma.cu
    const size_t smem = sizeof(float) * Tile<R>::SMEM_FLOATS;
    auto k = acoustic2d_step_kernel<R, EXACT, VARDEN>;
    static bool attr[kMaxDevices] = {};
    if (cudaError_t e = smem_attr_once((const void*)k, (int)smem, attr)) return e;
    dim3 grid(a.L.ntx * a.L.ntz, active);
    k<<<grid, kThreads, smem, st>>>(a);
    return cudaGetLastError();
}

template <int R>
cudaError_t launch_r(const Acou2DPlan& plan, const Acou2DArgs& a, int active, bool exact, bool varden,
                     cudaStream_t st) {
    if (exact) return varden ? launch_t<R, true, true>(a, active, st) : launch_t<R, true, false>(a, active, st);
    return acoustic2d_fwd_launch(plan, R, a, active, varden, st);
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
        plan->smem_bytes = sizeof(float) * Tile<RR>::SMEM_FLOATS;     \
        plan->gz = acoustic2d_fma_gz(RR);                             \
        plan->stages = 1;                                             \
        plan->seg = 0;                                                \
        plan->forced = false;                                         \
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
    case 1: return launch_r<1>(plan, a, active, exact, varden, st);
    case 2: return launch_r<2>(plan, a, active, exact, varden, st);
    case 4: return launch_r<4>(plan, a, active, exact, varden, st);
    case 5: return launch_r<5>(plan, a, active, exact, varden, st);
    case 8: return launch_r<8>(plan, a, active, exact, varden, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t acoustic2d_launch_inject0(const Acou2DArgs& a, int nshot, bool exact, cudaStream_t st) {
    inject0_kernel<<<(nshot + 127) / 128, 128, 0, st>>>(a, nshot, exact);
    return cudaGetLastError();
}

}  // namespace sfd
