// ORACLE -- test infrastructure only (tests/, smoke(), bench.py cpu_baseline). Not part of the
// product.
//
// Restatement of the 3-D velocity-pressure staggered-grid scheme.  The reference has no 3-D
// modeller, so this scheme is the 2-D one of forward/Acoustic_FD_by_ss/src/Acoustic_1order_FD.cpp
// extended by a y axis, step for step:
//   AFD:247-251  source:   P[s] -= (dt * den[s] * vp[s]) * w[k]           (before the update)
//   AFD:255-286  velocity: V_a = V_a - dt / (den * d_a) * sum_m C_m (P[i+m] - P[i-m+1])  (a = x, y, z)
//   AFD:289-314  pressure: P = P - den vp^2 dt sum_a (1/d_a) sum_m C_m (V_a[i+m-1] - V_a[i-m])
//                          (with the new, not yet damped velocities)
//   AFD:317-340  sponge:   every field times absorb (after the pressure update)
//   AFD:376-377  record:   P at each receiver after the sponge
// Cells within R of any face are never updated (AFD's loops run over [R, N-R)).  The sponge is
// AFD's quadratic taper 1 - 0.38 q^2 / PML^2 per axis; where pads overlap, the x factor wins over
// y and y over z (AFD:164-194 writes the z edges first and lets the x edges overwrite them).
// Parity unpinned: there is no reference output for this scheme; the tests compare the CUDA
// kernel with the FP64 instance of this file.
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace {

// AFD:164-194 taper value at distance index q into a sponge of width pml (double, stored float)
float taper(int q, int pml) { return (float)(-0.38 * q * q / (1.0 * pml * pml) + 1); }

// -1 if d is not in a pad of the axis of length n, else the distance index q
int pad_q(int d, int n, int pml) {
    if (d < pml) return pml - d - 1;
    if (d >= n - pml) return d - n + pml;
    return -1;
}

float absorb3(int x, int y, int z, int nx, int ny, int nz, int pml) {
    int q = pad_q(x, nx, pml);
    if (q >= 0) return taper(q, pml);
    q = pad_q(y, ny, pml);
    if (q >= 0) return taper(q, pml);
    q = pad_q(z, nz, pml);
    if (q >= 0) return taper(q, pml);
    return 1.0f;
}

template <typename T>
int run(const OracleAfd3Cfg* g, const float* vp, const float* den, const float* wav, T* record, T* final_p) {
    const int nx = g->nx, ny = g->ny, nz = g->nz, R = g->radius, pml = g->pml;
    if (nx <= 2 * R || ny <= 2 * R || nz <= 2 * R || R < 1 || R > 8) return 1;
    if (2 * pml > nx || 2 * pml > ny || 2 * pml > nz || pml < 0) return 1;
    float cf[8];
    if (oracle_afd_coeffs(R, cf)) return 1;
    const size_t n = (size_t)nx * ny * nz;
    const long long SX = (long long)ny * nz, SY = nz;
    std::vector<T> P(n, 0), Vx(n, 0), Vy(n, 0), Vz(n, 0);
    std::vector<float> ab(n);
#pragma omp parallel for schedule(static)
    for (int x = 0; x < nx; x++)
        for (int y = 0; y < ny; y++)
            for (int z = 0; z < nz; z++) ab[(x * SX) + y * SY + z] = absorb3(x, y, z, nx, ny, nz, pml);
    auto D = [&](size_t i) -> T { return den ? (T)den[i] : (T)g->den_c; };
    const size_t si = (size_t)g->sx * SX + (size_t)g->sy * SY + g->sz;
    // (dt * den) * vp in float, AFD:250
    float sc = g->dt * (den ? den[si] : g->den_c);
    sc = sc * vp[si];
    const T dt = (T)g->dt, dx = (T)g->dx, dy = (T)g->dy, dz = (T)g->dz;
    for (int k = 0; k < g->nt; k++) {
        P[si] -= (T)sc * (T)wav[k];
#pragma omp parallel for schedule(static)
        for (int x = R; x < nx - R; x++)
            for (int y = R; y < ny - R; y++)
                for (int z = R; z < nz - R; z++) {
                    const size_t i = x * SX + y * SY + z;
                    T sx = 0, sy = 0, sz = 0;
                    for (int m = 1; m <= R; m++) {
                        sx += (T)cf[m - 1] * (P[i + m * SX] - P[i - (m - 1) * SX]);
                        sy += (T)cf[m - 1] * (P[i + m * SY] - P[i - (m - 1) * SY]);
                        sz += (T)cf[m - 1] * (P[i + m] - P[i - (m - 1)]);
                    }
                    const T d = D(i);
                    Vx[i] -= dt / (d * dx) * sx;
                    Vy[i] -= dt / (d * dy) * sy;
                    Vz[i] -= dt / (d * dz) * sz;
                }
#pragma omp parallel for schedule(static)
        for (int x = R; x < nx - R; x++)
            for (int y = R; y < ny - R; y++)
                for (int z = R; z < nz - R; z++) {
                    const size_t i = x * SX + y * SY + z;
                    T sx = 0, sy = 0, sz = 0;
                    for (int m = 1; m <= R; m++) {
                        sx += (T)cf[m - 1] * (Vx[i + (m - 1) * SX] - Vx[i - m * SX]);
                        sy += (T)cf[m - 1] * (Vy[i + (m - 1) * SY] - Vy[i - m * SY]);
                        sz += (T)cf[m - 1] * (Vz[i + (m - 1)] - Vz[i - m]);
                    }
                    const T v = (T)vp[i];
                    P[i] -= D(i) * v * v * dt * (sx / dx + sy / dy + sz / dz);
                }
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < (long long)n; i++) {
            const T a = (T)ab[i];
            P[i] *= a;
            Vx[i] *= a;
            Vy[i] *= a;
            Vz[i] *= a;
        }
        if (record)
            for (int r = 0; r < g->nrec; r++)
                record[(size_t)r * g->nt + k] = P[(size_t)g->rec_x[r] * SX + (size_t)g->rec_y[r] * SY + g->rec_z[r]];
    }
    if (final_p) std::memcpy(final_p, P.data(), n * sizeof(T));
    return 0;
}

}  // namespace

extern "C" {

int oracle_afd3d_sponge(int nx, int ny, int nz, int pml, float* a) {
    if (!a || 2 * pml > nx || 2 * pml > ny || 2 * pml > nz || pml < 0) return 1;
    for (int x = 0; x < nx; x++)
        for (int y = 0; y < ny; y++)
            for (int z = 0; z < nz; z++) a[((size_t)x * ny + y) * nz + z] = absorb3(x, y, z, nx, ny, nz, pml);
    return 0;
}

int oracle_afd3d_f32(const OracleAfd3Cfg* g, const float* vp, const float* den, const float* wavelet, float* record,
                     float* final_p) {
    return run<float>(g, vp, den, wavelet, record, final_p);
}

int oracle_afd3d_f64(const OracleAfd3Cfg* g, const float* vp, const float* den, const float* wavelet, double* record,
                     double* final_p) {
    return run<double>(g, vp, den, wavelet, record, final_p);
}

}  // extern "C"
