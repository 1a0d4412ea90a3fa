// Adjoint of one time step of the 2-D acoustic scheme (AFD:237-380) and the zero-lag imaging
// condition.  The reference has no adjoint; this is the exact transpose of the forward step as
// the forward kernels implement it (velocities stored before the sponge, receivers after it):
//   mu = Q + R^T res[k],  l1 = a mu,  nu = M K l1,  K = DEN Vp^2 dt
//   X' = X + rdx S+x nu,  Z' = Z + rdz S+z nu
//   Q  <- M l1 + S-x(B_x M X') + S-z(B_z M Z'),   X <- a M X',   Z <- a M Z'
//   g  += l1 M D_k    (D_k = rdx S-x Vx + rdz S-z Vz of forward step k)
// with S+ q(i) = sum_m C_m (q[i+m+1] - q[i-m]) and S- q(i) = sum_m C_m (q[i+m] - q[i-m-1]);
// (S+)^T = -S- and (S-)^T = -S+.  Q arrives with the residual of step k already added (the
// previous adjoint step, or the initial state, injects it), and this step adds the residual of
// step k-1 at the receivers of its tile.  d misfit / d Vp = -2 DEN Vp dt sum_k g.
#include <cuda_runtime.h>

#include <algorithm>

#include "sfd_internal.h"

namespace sfd {
namespace {

constexpr int kThreads = 256;

__host__ __device__ constexpr int r4(int v) { return (v + 3) & ~3; }

template <int R>
struct TA {
    static constexpr int TX = kTileX, TZ = kTileZ;
    static constexpr int HX = 2 * R;
    static constexpr int HZ = r4(2 * R);
    static constexpr int SQ_ROWS = TX + 2 * HX, SQ_W = TZ + 2 * HZ;   // Q, then nu
    static constexpr int SX_ROWS = TX + 2 * R, SX_W = TZ;            // X, then B_x M X'
    static constexpr int SZ_W = TZ + 2 * HZ;                         // Z, then B_z M Z' (TX rows)
    static constexpr int OFF_QC = SQ_ROWS * SQ_W;                    // tile copy of Q, then Q_new
    static constexpr int OFF_X = OFF_QC + TX * TZ;
    static constexpr int OFF_Z = OFF_X + SX_ROWS * SX_W;
    static constexpr int OFF_T = OFF_Z + TX * SZ_W;
    static constexpr int SMEM_FLOATS = OFF_T + 256;
};

__device__ __forceinline__ float sponge_at(int x, int z, int nx, int nz, int pml, const float* tab) {
    if (x < pml) return tab[pml - 1 - x];
    if (x >= nx - pml) return tab[x - (nx - pml)];
    if (z < pml) return tab[pml - 1 - z];
    if (z >= nz - pml) return tab[z - (nz - pml)];
    return 1.0f;
}

template <int R, bool VARDEN>
__global__ void __launch_bounds__(kThreads, 2) adjoint2d_step_kernel(const __grid_constant__ Adj2DArgs a) {
    using T = TA<R>;
    extern __shared__ __align__(16) float smem[];
    float* sQ = smem;
    float* sQc = smem + T::OFF_QC;
    float* sX = smem + T::OFF_X;
    float* sZ = smem + T::OFF_Z;
    float* sTab = smem + T::OFF_T;

    const int shot = a.slot_to_shot[blockIdx.y];
    const ShotDev sd = a.shots[shot];
    const int tile = blockIdx.x;
    const int tx_i = tile / a.L.ntz, tz_i = tile - tx_i * a.L.ntz;
    if (tx_i * T::TX >= sd.nx) return;
    const int x0 = tx_i * T::TX, z0 = tz_i * T::TZ;
    const int nx = sd.nx, nz = a.nz, pml = a.pml;
    const int tid = threadIdx.x;
    const long long soff = (long long)shot * a.L.shot_stride;
    const int pitch = a.L.pitch;
    auto cell = [&](int x, int z) -> long long { return soff + (long long)(x + a.L.gx) * pitch + a.L.gz + z; };
    auto inside = [&](int x, int z) { return x >= R && x < nx - R && z >= R && z < nz - R; };
    auto model = [&](const float* m, int x, int z) {
        return __ldg(m + (long long)min(max(sd.x0 + x, 0), a.nx_model - 1) * a.mpitch + z);
    };

    for (int i = tid; i < pml && i < 256; i += kThreads) sTab[i] = a.sponge[i];
    {
        constexpr int W4 = T::SQ_W / 4;
        for (int i = tid; i < T::SQ_ROWS * W4; i += kThreads) {
            const int r = i / W4, c = i - r * W4;
            *reinterpret_cast<float4*>(sQ + r * T::SQ_W + 4 * c) =
                __ldg(reinterpret_cast<const float4*>(a.q_in + cell(x0 - T::HX + r, z0 - T::HZ + 4 * c)));
        }
    }
    {
        constexpr int W4 = T::SX_W / 4;
        for (int i = tid; i < T::SX_ROWS * W4; i += kThreads) {
            const int r = i / W4, c = i - r * W4;
            *reinterpret_cast<float4*>(sX + r * T::SX_W + 4 * c) =
                __ldg(reinterpret_cast<const float4*>(a.x_in + cell(x0 - R + r, z0 + 4 * c)));
        }
    }
    {
        constexpr int W4 = T::SZ_W / 4;
        for (int i = tid; i < T::TX * W4; i += kThreads) {
            const int r = i / W4, c = i - r * W4;
            *reinterpret_cast<float4*>(sZ + r * T::SZ_W + 4 * c) =
                __ldg(reinterpret_cast<const float4*>(a.z_in + cell(x0 + r, z0 - T::HZ + 4 * c)));
        }
    }
    __syncthreads();

    // keep Q of the tile, turn the staged Q into nu = M K a Q
    for (int i = tid; i < T::TX * T::TZ; i += kThreads) {
        const int r = i / T::TZ, z = i - r * T::TZ;
        sQc[i] = sQ[(r + T::HX) * T::SQ_W + z + T::HZ];
    }
    __syncthreads();
    for (int i = tid; i < T::SQ_ROWS * T::SQ_W; i += kThreads) {
        const int r = i / T::SQ_W, zz = i - r * T::SQ_W;
        const int gx = x0 - T::HX + r, gz = z0 - T::HZ + zz;
        float nu = 0.0f;
        if (inside(gx, gz)) {
            const float vp = model(a.vp, gx, gz);
            const float den = VARDEN ? model(a.den, gx, gz) : a.den_c;
            nu = den * vp * vp * a.dt * sponge_at(gx, gz, nx, nz, pml, sTab) * sQ[i];
        }
        sQ[i] = nu;
    }
    __syncthreads();

    float C[R];
#pragma unroll
    for (int m = 0; m < R; m++) C[m] = a.coef[m];

    // X' = X + rdx S+x nu on rows x0-R .. x0+TX+R
    for (int i = tid; i < T::SX_ROWS * T::TZ; i += kThreads) {
        const int r = i / T::TZ, z = i - r * T::TZ;
        const int gx = x0 - R + r, gz = z0 + z;
        const float* nr = sQ + (r + R) * T::SQ_W + z + T::HZ;  // nu row of gx
        float s = C[0] * (nr[T::SQ_W] - nr[0]);
#pragma unroll
        for (int m = 1; m < R; m++) s = fmaf(C[m], nr[(m + 1) * T::SQ_W] - nr[-m * T::SQ_W], s);
        const float xp = fmaf(a.rdx, s, sX[r * T::SX_W + z]);
        const float msk = inside(gx, gz) ? 1.0f : 0.0f;
        if (r >= R && r < R + T::TX && gx < nx && gz < nz)
            a.x_out[cell(gx, gz)] = sponge_at(gx, gz, nx, nz, pml, sTab) * msk * xp;
        float b = a.dtdx / a.den_c;
        if (VARDEN && msk != 0.0f) b = a.dtdx / model(a.den, gx, gz);
        sX[r * T::SX_W + z] = b * msk * xp;
    }
    // Z' = Z + rdz S+z nu on columns x0 .. x0+TX, z0-R .. z0+TZ+R
    for (int i = tid; i < T::TX * (T::TZ + 2 * R); i += kThreads) {
        const int r = i / (T::TZ + 2 * R), zz = i - r * (T::TZ + 2 * R);
        const int gx = x0 + r, gz = z0 - R + zz;
        const int zs = zz - R + T::HZ;
        const float* nc = sQ + (r + T::HX) * T::SQ_W + zs;
        float s = C[0] * (nc[1] - nc[0]);
#pragma unroll
        for (int m = 1; m < R; m++) s = fmaf(C[m], nc[m + 1] - nc[-m], s);
        const float zp = fmaf(a.rdz, s, sZ[r * T::SZ_W + zs]);
        const float msk = inside(gx, gz) ? 1.0f : 0.0f;
        if (zz >= R && zz < R + T::TZ && gx < nx && gz < nz)
            a.z_out[cell(gx, gz)] = sponge_at(gx, gz, nx, nz, pml, sTab) * msk * zp;
        float b = a.dtdz / a.den_c;
        if (VARDEN && msk != 0.0f) b = a.dtdz / model(a.den, gx, gz);
        sZ[r * T::SZ_W + zs] = b * msk * zp;
    }
    __syncthreads();

    // Q_new = M a Q + S-x(B M X') + S-z(B M Z') on the tile (every cell: the transpose reaches
    // the frozen rim); imaging g += a Q M D
    const int step = a.step;
    for (int i = tid; i < T::TX * T::TZ; i += kThreads) {
        const int r = i / T::TZ, z = i - r * T::TZ;
        const int gx = x0 + r, gz = z0 + z;
        const float* xr = sX + (r + R) * T::SX_W + z;
        const float* zc = sZ + r * T::SZ_W + z + T::HZ;
        float sx = C[0] * (xr[0] - xr[-T::SX_W]);
        float sz = C[0] * (zc[0] - zc[-1]);
#pragma unroll
        for (int m = 1; m < R; m++) {
            sx = fmaf(C[m], xr[m * T::SX_W] - xr[-(m + 1) * T::SX_W], sx);
            sz = fmaf(C[m], zc[m] - zc[-(m + 1)], sz);
        }
        float qn = 0.0f;
        if (gx < nx && gz < nz) {
            const float aq = sponge_at(gx, gz, nx, nz, pml, sTab) * sQc[i];
            const bool in = inside(gx, gz);
            qn = (in ? aq : 0.0f) + sx + sz;
            const long long c = cell(gx, gz);
            if (in) a.g_seg[c] = fmaf(aq, __ldg(a.div + c), a.g_seg[c]);
            a.q_out[c] = qn;
            if (gx == sd.sx && gz == sd.sz) a.lam_src[(long long)shot * a.nt_max + step] = qn;
        }
        sQc[i] = qn;
    }
    // residual of step k-1 at the receivers of this tile (AFD:376-377 transposed)
    const int* trp = a.tile_rec_ptr + sd.tile_rec_base + tile;
    const int rb = trp[0], re = trp[1];
    if (step >= 1 && re > rb) {
        __syncthreads();
        for (int j = rb + tid; j < re; j += kThreads) {
            const int ridx = a.tile_rec_idx[j];
            const int rx = a.rec_x[sd.rec_list + ridx], rz = a.rec_z[sd.rec_list + ridx];
            const float v = a.res[sd.rec_base + (long long)(step - 1) * sd.nrec + ridx];
            // several receivers may share a cell: accumulate atomically on the stored value
            atomicAdd(&a.q_out[cell(rx, rz)], v);
        }
    }
}

template <int R, bool VARDEN>
cudaError_t launch_t(const Adj2DArgs& a, int active, cudaStream_t st) {
    const size_t smem = sizeof(float) * TA<R>::SMEM_FLOATS;
    auto k = adjoint2d_step_kernel<R, VARDEN>;
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

__global__ void residual_kernel(const float* __restrict__ pred, const float* __restrict__ obs, float* __restrict__ res,
                                long long n, double* misfit) {
    double acc = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float r = pred[i] - obs[i];
        res[i] = r;
        acc += 0.5 * (double)r * (double)r;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(misfit, acc);
}

__global__ void transpose_in_kernel(const float* __restrict__ in, float* __restrict__ out,
                                    const ShotDev* __restrict__ shots) {
    __shared__ float tile[32][33];
    const ShotDev sd = shots[blockIdx.z];
    const int t0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    if (r0 >= sd.nrec || t0 >= sd.nt) return;
    const float* src = in + sd.rec_base;  // [nrec][nt]
    float* dst = out + sd.rec_base;       // [nt][nrec]
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = r0 + j, t = t0 + threadIdx.x;
        if (t < sd.nt && r < sd.nrec) tile[j][threadIdx.x] = src[(long long)r * sd.nt + t];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int t = t0 + j, r = r0 + threadIdx.x;
        if (t < sd.nt && r < sd.nrec) dst[(long long)t * sd.nrec + r] = tile[threadIdx.x][j];
    }
}

__global__ void adjoint_init_kernel(float* q0, float* q1, Layout2D L, const ShotDev* __restrict__ shots,
                                    int first_shot, const float* __restrict__ res, const int* __restrict__ rec_x,
                                    const int* __restrict__ rec_z) {
    const int s = first_shot + blockIdx.y;
    const ShotDev sd = shots[s];
    float* q = (sd.nt & 1) ? q1 : q0;  // the first adjoint step (k = nt-1) reads buffer nt & 1
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < sd.nrec; r += gridDim.x * blockDim.x) {
        const int x = rec_x[sd.rec_list + r], z = rec_z[sd.rec_list + r];
        atomicAdd(q + (long long)s * L.shot_stride + (long long)(x + L.gx) * L.pitch + L.gz + z,
                  res[sd.rec_base + (long long)(sd.nt - 1) * sd.nrec + r]);
    }
}

__global__ void accumulate_kernel(double* __restrict__ acc, const float* __restrict__ seg, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        acc[i] += (double)seg[i];
}

__global__ void gradient_reduce_kernel(const double* __restrict__ acc, Layout2D L, const ShotDev* __restrict__ shots,
                                       int nshot, const float* __restrict__ vp, const float* __restrict__ den,
                                       float den_c, int mpitch, int nx_model, int nz, float dt, double* grad) {
    const long long n = (long long)nx_model * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int X = (int)(i / nz), z = (int)(i - (long long)X * nz);
        double s = 0.0;
        for (int sh = 0; sh < nshot; sh++) {
            const int x = X - shots[sh].x0;
            if (x >= 0 && x < shots[sh].nx)
                s += acc[(long long)sh * L.shot_stride + (long long)(x + L.gx) * L.pitch + L.gz + z];
        }
        const double v = vp[(long long)X * mpitch + z];
        const double d = den ? (double)den[(long long)X * mpitch + z] : (double)den_c;
        grad[i] = -2.0 * d * v * (double)dt * s;
    }
}

int grid_for(long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 16); }

}  // namespace

cudaError_t adjoint2d_launch_step(int radius, const Adj2DArgs& a, int active, bool varden, cudaStream_t st) {
    switch (radius) {
#define SFD_CASE(RR) \
    case RR: return varden ? launch_t<RR, true>(a, active, st) : launch_t<RR, false>(a, active, st);
        SFD_CASE(1) SFD_CASE(2) SFD_CASE(4) SFD_CASE(5) SFD_CASE(8)
#undef SFD_CASE
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_residual(const float* pred, const float* obs, float* res, long long n, double* misfit,
                            cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    residual_kernel<<<grid_for(n), 256, 0, st>>>(pred, obs, res, n, misfit);
    return cudaGetLastError();
}

cudaError_t launch_records_transpose_in(const float* rec_nt, float* rec_tn, const ShotDev* shots, int nshot,
                                        int nrec_max, int nt_max, cudaStream_t st) {
    if (nrec_max <= 0 || nt_max <= 0) return cudaSuccess;
    dim3 grid((nt_max + 31) / 32, (nrec_max + 31) / 32, nshot);
    transpose_in_kernel<<<grid, dim3(32, 8), 0, st>>>(rec_nt, rec_tn, shots);
    return cudaGetLastError();
}

cudaError_t launch_adjoint_init(float* q0, float* q1, const Layout2D& L, const ShotDev* shots, int first_shot,
                                int nshot, const float* res, const int* rec_x, const int* rec_z, int nrec_max,
                                cudaStream_t st) {
    if (nrec_max <= 0) return cudaSuccess;
    dim3 grid((nrec_max + 255) / 256, nshot);
    adjoint_init_kernel<<<grid, 256, 0, st>>>(q0, q1, L, shots, first_shot, res, rec_x, rec_z);
    return cudaGetLastError();
}

cudaError_t launch_accumulate(double* acc, const float* seg, long long n, cudaStream_t st) {
    accumulate_kernel<<<grid_for(n), 256, 0, st>>>(acc, seg, n);
    return cudaGetLastError();
}

cudaError_t launch_gradient_reduce(const double* acc, const Layout2D& L, const ShotDev* shots, int nshot,
                                   const float* vp, const float* den, float den_c, int mpitch, int nx_model,
                                   int nz, float dt, double* grad_model, cudaStream_t st) {
    const long long n = (long long)nx_model * nz;
    gradient_reduce_kernel<<<grid_for(n), 256, 0, st>>>(acc, L, shots, nshot, vp, den, den_c, mpitch, nx_model, nz,
                                                        dt, grad_model);
    return cudaGetLastError();
}

}  // namespace sfd
