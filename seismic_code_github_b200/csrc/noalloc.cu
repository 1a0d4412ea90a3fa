// sfd_forward_noalloc: a single-shot 2-D acoustic forward that allocates no device memory.
//
// Some callers cannot allocate device memory when they want to model a shot: a service whose
// framework has already reserved the device memory for its own caching allocator, a process
// running under a device-memory quota its pools have used up, or a real-time loop that forbids
// allocation after start-up (cudaMalloc and cudaFree synchronise the device).  This entry point
// serves them: the caller passes its inputs and output in device memory, and every working
// buffer -- the wavefields, the one-shot descriptor, the receiver tables and the time-major
// records -- lives in one file-scope device array of fixed size, kNoAllocBytes (32 MiB), that
// each GPU loading the library holds until the process exits.  It runs the same
// reference-order step kernel as sfd_forward with SFD_EXACT.
//
// The first call on a device looks up the array's device address (cudaGetSymbolAddress, with
// that device current); make that first call before any stream capture.  All calls share the
// array: each call clears the parts that must start at zero, and calls that overlap on the GPU
// (several host threads, or several streams) race on it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "sfd_internal.h"

namespace sfd {
namespace {

constexpr size_t kNoAllocBytes = 32u << 20;  // stated maximum of the scratch array

// The scratch array.  In host code this name is only a stand-in for the symbol: its device
// address comes from cudaGetSymbolAddress (once per device, with that device current).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_mu;
void* g_scratch_addr[64] = {};  // per device ordinal

// One-shot descriptor and active-slot table, written on the device (no host copy needed).
__global__ void noalloc_init_kernel(ShotDev* shot, int* slot, ShotDev sd, const float* vp, const float* den,
                                    float den_c, int nz, float dt) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const long long si = (long long)sd.sx * nz + sd.sz;
    const float d = den ? den[si] : den_c;
    sd.inj_scale = __fmul_rn(__fmul_rn(dt, d), vp[si]);  // ((dt * DEN) * Vp), AFD:250
    *shot = sd;
    *slot = 0;
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace
}  // namespace sfd

using namespace sfd;

extern "C" int sfd_forward_noalloc(const sfd_grid* g, const float* vp_dev, const float* den_dev,
                                   const float* wavelet_dev, int nt, int sx, int sz, int nrec, const int* rec_x,
                                   const int* rec_z, float* records_dev, void* stream) {
    if (!g || !vp_dev || !wavelet_dev || nt < 1 || nrec < 0 || (nrec > 0 && (!rec_x || !rec_z || !records_dev)))
        return SFD_ERR_ARG;
    // an error left pending by earlier work of the caller's thread is not this call's: drop it so
    // that the launch checks below report only this call's launches
    (void)cudaGetLastError();
    if (g->scheme != SFD_ACOUSTIC_2D || g->ny > 1) return SFD_ERR_UNSUPPORTED;
    float cf[8];
    if (sfd_fd_coeffs(g->order, cf) != SFD_OK) return SFD_ERR_ARG;
    const int R = g->order / 2, nx = g->nx, nz = g->nz, pml = g->pml;
    if (nx <= 2 * R || nz <= 2 * R || pml < 0 || pml > 256 || 2 * pml > nx || 2 * pml > nz) return SFD_ERR_ARG;
    if (!(g->dx > 0) || !(g->dz > 0) || !(g->dt > 0)) return SFD_ERR_ARG;
    if (sx < 0 || sx >= nx || sz < 0 || sz >= nz) return SFD_ERR_ARG;
    for (int r = 0; r < nrec; r++)
        if (rec_x[r] < 0 || rec_x[r] >= nx || rec_z[r] < 0 || rec_z[r] >= nz) return SFD_ERR_ARG;
    Acou2DPlan plan{};
    if (!acoustic2d_plan(R, &plan)) return SFD_ERR_UNSUPPORTED;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // layout of the wavefields (as sfd_set_shots builds it for one shot)
    Layout2D L{};
    L.tx = plan.tx;
    L.tz = plan.tz;
    L.gx = 2 * R;
    L.gz = plan.gz;
    L.ntx = (nx + L.tx - 1) / L.tx;
    L.ntz = (nz + L.tz - 1) / L.tz;
    L.pitch = (L.gz + L.ntz * L.tz + L.gz + 31) / 32 * 32;
    L.cols = L.gx + L.ntx * L.tx + L.gx;
    L.shot_stride = (long long)L.cols * L.pitch;
    const int ntiles = L.ntx * L.ntz;

    // per-tile receiver tables on the host (small), copied into the scratch array
    std::vector<int> trp(ntiles + 1, 0), tri;
    tri.reserve(nrec);
    {
        std::vector<std::vector<int>> bucket(ntiles);
        for (int r = 0; r < nrec; r++) bucket[(rec_x[r] / L.tx) * L.ntz + rec_z[r] / L.tz].push_back(r);
        for (int t = 0; t < ntiles; t++) {
            trp[t] = (int)tri.size();
            tri.insert(tri.end(), bucket[t].begin(), bucket[t].end());
        }
        trp[ntiles] = (int)tri.size();
    }

    // carve the scratch array: shot, slot, tables, receivers, records (time-major), 6 fields
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align256(off + bytes);
        return o;
    };
    const size_t o_shot = take(sizeof(ShotDev));
    const size_t o_slot = take(sizeof(int));
    const size_t o_trp = take(sizeof(int) * trp.size());
    const size_t o_tri = take(sizeof(int) * std::max<size_t>(1, tri.size()));
    const size_t o_rx = take(sizeof(int) * std::max(1, nrec));
    const size_t o_rz = take(sizeof(int) * std::max(1, nrec));
    const size_t o_rec = take(sizeof(float) * std::max<long long>(1, (long long)nrec * nt));
    const size_t state_floats = 6 * (size_t)L.shot_stride;
    const size_t o_state = take(sizeof(float) * state_floats);
    if (off > kNoAllocBytes) return SFD_ERR_NOMEM;  // the grid and record do not fit the stated maximum

    // scratch address on the current device (set-up on the first call per device)
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return SFD_ERR_CUDA;
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_scratch_addr[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return SFD_ERR_CUDA;
            g_scratch_addr[dev] = p;
        }
        base = static_cast<unsigned char*>(g_scratch_addr[dev]);
    }
    ShotDev* d_shot = reinterpret_cast<ShotDev*>(base + o_shot);
    int* d_slot = reinterpret_cast<int*>(base + o_slot);
    int* d_trp = reinterpret_cast<int*>(base + o_trp);
    int* d_tri = reinterpret_cast<int*>(base + o_tri);
    int* d_rx = reinterpret_cast<int*>(base + o_rx);
    int* d_rz = reinterpret_cast<int*>(base + o_rz);
    float* d_rec = reinterpret_cast<float*>(base + o_rec);
    float* d_state = reinterpret_cast<float*>(base + o_state);

    // the array keeps the previous call's contents: clear what must start at zero
    if (cudaMemsetAsync(d_state, 0, state_floats * sizeof(float), st) != cudaSuccess) return SFD_ERR_CUDA;
    if (cudaMemsetAsync(d_rec, 0, sizeof(float) * std::max<long long>(1, (long long)nrec * nt), st) != cudaSuccess)
        return SFD_ERR_CUDA;
    if (cudaMemcpyAsync(d_trp, trp.data(), sizeof(int) * trp.size(), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        (!tri.empty() &&
         cudaMemcpyAsync(d_tri, tri.data(), sizeof(int) * tri.size(), cudaMemcpyHostToDevice, st) != cudaSuccess) ||
        (nrec > 0 && (cudaMemcpyAsync(d_rx, rec_x, sizeof(int) * nrec, cudaMemcpyHostToDevice, st) != cudaSuccess ||
                      cudaMemcpyAsync(d_rz, rec_z, sizeof(int) * nrec, cudaMemcpyHostToDevice, st) != cudaSuccess)))
        return SFD_ERR_CUDA;

    ShotDev sd{};
    sd.nx = nx; sd.x0 = 0; sd.nt = nt; sd.sx = sx; sd.sz = sz; sd.nrec = nrec;
    sd.rec_base = 0; sd.rec_list = 0; sd.wav_off = 0; sd.tile_rec_base = 0;
    const float den_c = 2400.0f;
    noalloc_init_kernel<<<1, 32, 0, st>>>(d_shot, d_slot, sd, vp_dev, den_dev, den_c, nz, g->dt);
    if (cudaGetLastError() != cudaSuccess) return SFD_ERR_CUDA;

    // step arguments: the model and wavelet are read in place from the caller's buffers
    Acou2DArgs a{};
    a.test_cta = -1;  // no test hook
    const long long fs = L.shot_stride;
    a.L = L;
    a.nz = nz;
    a.pml = pml;
    a.vp = vp_dev;
    a.den = den_dev;
    a.mpitch = nz;  // the reference-order kernel reads the model only inside the updated region
    a.nx_model = nx;
    a.den_c = den_c;
    a.dt = g->dt;
    a.dtdx = g->dt / g->dx;
    a.dtdz = g->dt / g->dz;
    a.rdx_d = 1.0 / (double)g->dx;
    a.rdz_d = 1.0 / (double)g->dz;
    a.bx_d = (1.0 / (double)den_c) * (double)a.dtdx;
    a.bz_d = (1.0 / (double)den_c) * (double)a.dtdz;
    a.bx_f = (float)a.bx_d;
    a.bz_f = (float)a.bz_d;
    a.rdx_f = 1.0f / g->dx;
    a.rdz_f = 1.0f / g->dz;
    std::memcpy(a.coef, cf, sizeof(float) * R);
    for (int q = 0; q < pml; q++) a.sponge[q] = -0.38 * q * q / (1.0 * pml * pml) + 1;
    a.shots = d_shot;
    a.slot_to_shot = d_slot;
    a.wavelets = wavelet_dev;
    a.rec_x = d_rx;
    a.rec_z = d_rz;
    a.tile_rec_ptr = d_trp;
    a.tile_rec_idx = d_tri;
    a.records = d_rec;
    auto set_step = [&](int step) {
        const int i = step & 1, o = (step + 1) & 1;
        a.p_in = d_state + i * fs; a.p_out = d_state + o * fs;
        a.vx_in = d_state + (2 + i) * fs; a.vx_out = d_state + (2 + o) * fs;
        a.vz_in = d_state + (4 + i) * fs; a.vz_out = d_state + (4 + o) * fs;
        a.step = step;
    };
    set_step(-1);
    if (acoustic2d_launch_inject0(a, 1, true, st) != cudaSuccess) return SFD_ERR_CUDA;
    const bool varden = den_dev != nullptr;
    for (int k = 0; k < nt; k++) {
        set_step(k);
        if (acoustic2d_launch_step(plan, a, 1, /*exact*/ true, varden, st) != cudaSuccess) return SFD_ERR_CUDA;
    }
    if (nrec > 0 && launch_records_transpose(d_rec, records_dev, d_shot, 1, nrec, nt, st) != cudaSuccess)
        return SFD_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return SFD_ERR_CUDA;
    return SFD_OK;
}
