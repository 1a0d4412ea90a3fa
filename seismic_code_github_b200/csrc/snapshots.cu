// Wavefield snapshots taken inside the time loop: the interior of one field after a step, the
// way AFD writes Snap.dat and Pall.dat (forward/Acoustic_FD_by_ss/src/Acoustic_1order_FD.cpp:
// 343-373), Q_forward writes its snapshot files (forward/Q_forward/
// Q_multishot_fd_main_fsbc_zy_rotated.f90:462-481) and yang_version its vx / vz files (YPUB:20-44).
// The interior (pml <= x < nx - pml, ztop <= z < nz - pml, ztop = pml except below a free
// surface's top pad) carries no sponge factor, so the undamped velocities the step kernels
// store are the values the reference holds there.
#include <cuda_runtime.h>

#include "sfd_internal.h"

namespace sfd {
namespace {

__global__ void snapshot_kernel(const __grid_constant__ SnapArgs a) {
    const int shot = a.slot_to_shot[blockIdx.y];
    const ShotDev sd = a.shots[shot];
    if (a.step >= sd.nt) return;
    const int nxi = sd.nx - 2 * a.pml, nzi = a.nz - a.ztop - a.pml;
    const long long n = (long long)nxi * nzi;
    const long long base = (long long)shot * a.L.shot_stride + (long long)a.L.gx * a.L.pitch + a.L.gz;
    float* out = a.out + a.shot_off[shot] + (long long)a.index * n;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int xi = (int)(i / nzi), zi = (int)(i - (long long)xi * nzi);
        const int x = a.pml + xi, z = a.ztop + zi;
        const long long c = base + (long long)x * a.L.pitch + z;
        float v = a.f[0][c];
        if (a.nsum >= 2) v = __fadd_rn(v, a.f[1][c]);  // split parts summed in order: x + z (QS, YPUB calu)
        if (a.nsum == 3) v = __fadd_rn(v, a.f[2][c]);  // (sx + sz) + sr, QS calsum
        if (a.src_pre && x == sd.sx && z == sd.sz && a.step + 1 < sd.nt) v = a.src_pre[shot];
        out[i] = v;
    }
}

}  // namespace

cudaError_t launch_snapshot(const SnapArgs& a, int active, int nx_max, cudaStream_t st) {
    if (active <= 0) return cudaSuccess;
    const long long n = (long long)(nx_max - 2 * a.pml) * (a.nz - a.ztop - a.pml);
    const int blocks = (int)((n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024);
    snapshot_kernel<<<dim3(blocks > 0 ? blocks : 1, active), 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace sfd
