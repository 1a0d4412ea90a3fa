// Adjoint of one time step of the 2-D acoustic scheme (AFD:237-380) and the zero-lag imaging
// condition.  The reference has no adjoint; this is the exact transpose of the forward step as
// the forward kernels implement it (velocities stored before the sponge, receivers after it):
//   mu = Q + R^T res[k],  l1 = a mu,  nu = M K l1,  K = DEN Vp^2 dt
//   X' = X + rdx S+x nu,  Z' = Z + rdz S+z nu
//   Q  <- M l1 + S-x(B_x M X') + S-z(B_z M Z'),   X <- a M X',   Z <- a M Z'
//   g  += l1 M D_k    (D_k = rdx S-x Vx + rdz S-z Vz of forward step k)
// with S+ q(i) = sum_m C_m (q[i+m+1] - q[i-m]) and S- q(i) = sum_m C_m (q[i+m] - q[i-m-1]);
// (S+)^T = -S- and (S-)^T = -S+, a the sponge, M the update mask (R <= x < nx-R, R <= z < nz-R),
// B = dt / (d DEN).  d misfit / d Vp = -2 DEN Vp dt sum_k g.
//
// The step itself runs in the FMA step kernel (acoustic2d_fma.cu, adjoint mode), which carries
// nu = M K a Q instead of Q: then M l1 = nu / K, the new state is nu' = M a K (nu / K + S-x(..)
// + S-z(..)), the receivers add M a K res, and the imaging sum becomes sum_k nu D_k, so that
// d misfit / d Vp = -(2 / Vp) sum_k nu D_k.  Every model factor is then needed at the updated
// cell only.  This file holds the kernels around the step: residuals and misfit, the record
// transpose, the initial adjoint state, the double-precision accumulation and the reduction to
// the model grid.
#include <cuda_runtime.h>

#include <algorithm>

#include "sfd_internal.h"

namespace sfd {
namespace {

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

// nu of every shot in [first, first + n), buffer nt & 1 (read by the first adjoint step,
// k = nt - 1), += M a K res of the shot's last step at its receivers
__global__ void adjoint_init_kernel(float* q0, float* q1, const Acou2DArgs a, int first_shot, int R) {
    const int s = first_shot + blockIdx.y;
    const ShotDev sd = a.shots[s];
    float* q = (sd.nt & 1) ? q1 : q0;
    const int nx = sd.nx, nz = a.nz, pml = a.pml;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < sd.nrec; r += gridDim.x * blockDim.x) {
        const int x = a.rec_x[sd.rec_list + r], z = a.rec_z[sd.rec_list + r];
        if (x < R || x >= nx - R || z < R || z >= nz - R) continue;  // M = 0
        const long long mi = (long long)min(sd.x0 + x, a.nx_model - 1) * a.mpitch + z;
        const float vp = a.vp[mi], den = a.den ? a.den[mi] : a.den_c;
        float sa = 1.0f;
        if (x < pml) sa = a.sponge[pml - 1 - x];
        else if (x >= nx - pml) sa = a.sponge[x - (nx - pml)];
        else if (z < pml) sa = a.sponge[pml - 1 - z];
        else if (z >= nz - pml) sa = a.sponge[z - (nz - pml)];
        const float v = a.adj_res[sd.rec_base + (long long)(sd.nt - 1) * sd.nrec + r];
        atomicAdd(q + (long long)s * a.L.shot_stride + (long long)(x + a.L.gx) * a.L.pitch + a.L.gz + z,
                  den * vp * vp * a.dt * sa * v);
    }
}

__global__ void accumulate_kernel(double* __restrict__ acc, const float* __restrict__ seg, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        acc[i] += (double)seg[i];
}

__global__ void gradient_reduce_kernel(const double* __restrict__ acc, Layout2D L, const ShotDev* __restrict__ shots,
                                       int nshot, const float* __restrict__ vp, int mpitch, int nx_model, int nz,
                                       double* grad) {
    const long long n = (long long)nx_model * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int X = (int)(i / nz), z = (int)(i - (long long)X * nz);
        double s = 0.0;
        for (int sh = 0; sh < nshot; sh++) {
            const int x = X - shots[sh].x0;
            if (x >= 0 && x < shots[sh].nx)
                s += acc[(long long)sh * L.shot_stride + (long long)(x + L.gx) * L.pitch + L.gz + z];
        }
        grad[i] = -2.0 * s / (double)vp[(long long)X * mpitch + z];
    }
}

int grid_for(long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 16); }

}  // namespace

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

cudaError_t launch_adjoint_init(float* q0, float* q1, const Acou2DArgs& a, int radius, int first_shot, int nshot,
                                int nrec_max, cudaStream_t st) {
    if (nrec_max <= 0) return cudaSuccess;
    dim3 grid((nrec_max + 255) / 256, nshot);
    adjoint_init_kernel<<<grid, 256, 0, st>>>(q0, q1, a, first_shot, radius);
    return cudaGetLastError();
}

cudaError_t launch_accumulate(double* acc, const float* seg, long long n, cudaStream_t st) {
    accumulate_kernel<<<grid_for(n), 256, 0, st>>>(acc, seg, n);
    return cudaGetLastError();
}

cudaError_t launch_gradient_reduce(const double* acc, const Layout2D& L, const ShotDev* shots, int nshot,
                                   const float* vp, int mpitch, int nx_model, int nz, double* grad_model,
                                   cudaStream_t st) {
    const long long n = (long long)nx_model * nz;
    gradient_reduce_kernel<<<grid_for(n), 256, 0, st>>>(acc, L, shots, nshot, vp, mpitch, nx_model, nz, grad_model);
    return cudaGetLastError();
}

}  // namespace sfd
