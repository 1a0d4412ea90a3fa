// Record post-processing: the time loop writes each shot's samples time-major ([nt][nrec], one
// coalesced row per step); the interface layout is trace-major ([nrec][nt], AFD:385-393), so a
// tiled transpose runs once after the loop.  Also the NaN/Inf watchdog on the traces.
#include <cuda_runtime.h>

#include <algorithm>

#include "sfd_internal.h"

namespace sfd {
namespace {

__global__ void transpose_kernel(const float* __restrict__ in, float* __restrict__ out,
                                 const ShotDev* __restrict__ shots) {
    __shared__ float tile[32][33];
    const ShotDev sd = shots[blockIdx.z];
    const int r0 = blockIdx.x * 32, t0 = blockIdx.y * 32;
    if (r0 >= sd.nrec || t0 >= sd.nt) return;
    const float* src = in + sd.rec_base;
    float* dst = out + sd.rec_base;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int t = t0 + j, r = r0 + threadIdx.x;
        if (t < sd.nt && r < sd.nrec) tile[j][threadIdx.x] = src[(long long)t * sd.nrec + r];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = r0 + j, t = t0 + threadIdx.x;
        if (t < sd.nt && r < sd.nrec) dst[(long long)r * sd.nt + t] = tile[threadIdx.x][j];
    }
}

__global__ void nan_scan_kernel(const float* __restrict__ v, long long n, int* flag) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (!isfinite(v[i])) {
            atomicExch(flag, 1);
            return;
        }
}

// d misfit / d vp at the source cells: the source term P[src] -= (dt DEN Vp) w[k] gives
// -dt DEN sum_k lambda_k w[k].  One thread, shots and samples in order, double precision with
// explicitly rounded operations: the same sums, in the same order, as the host path of
// sfd_gradient, so both give the same bits.
__global__ void grad_source_kernel(double* grad, const GradSrc* src, const ShotDev* shots, int nshot, const float* lam,
                                   int nt_max, const float* wav) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int s = 0; s < nshot; s++) {
        const ShotDev sd = shots[s];
        double sw = 0.0;
        for (int j = 0; j < sd.nt; j++)
            sw = __dadd_rn(sw, __dmul_rn((double)lam[(long long)s * nt_max + j], (double)wav[sd.wav_off + j]));
        grad[src[s].mi] = __dadd_rn(grad[src[s].mi], __dmul_rn(src[s].scale, sw));
    }
}

__global__ void to_float_kernel(const double* __restrict__ in, float* __restrict__ out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = __double2float_rn(in[i]);
}

}  // namespace

cudaError_t launch_grad_source(double* grad, const GradSrc* src, const ShotDev* shots, int nshot, const float* lam,
                               int nt_max, const float* wav, cudaStream_t st) {
    if (nshot <= 0) return cudaSuccess;
    grad_source_kernel<<<1, 32, 0, st>>>(grad, src, shots, nshot, lam, nt_max, wav);
    return cudaGetLastError();
}

cudaError_t launch_to_float(const double* in, float* out, long long n, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 16);
    to_float_kernel<<<blocks, 256, 0, st>>>(in, out, n);
    return cudaGetLastError();
}

cudaError_t launch_records_transpose(const float* rec_tn, float* rec_nt, const ShotDev* shots, int nshot,
                                     int nrec_max, int nt_max, cudaStream_t st) {
    if (nrec_max <= 0 || nt_max <= 0 || nshot <= 0) return cudaSuccess;
    dim3 grid((nrec_max + 31) / 32, (nt_max + 31) / 32, nshot);
    transpose_kernel<<<grid, dim3(32, 8), 0, st>>>(rec_tn, rec_nt, shots);
    return cudaGetLastError();
}

cudaError_t launch_nan_scan(const float* rec, long long n, int* flag, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 8);
    nan_scan_kernel<<<blocks, 256, 0, st>>>(rec, n, flag);
    return cudaGetLastError();
}

}  // namespace sfd
