// ORACLE -- test infrastructure only (tests/, smoke(), bench.py cpu_baseline). Not part of the
// product.  CPU restatement of the 2-D VTI pseudo-acoustic modeller of
// de-multiple/convolution_srm/vti_qa_2d_c3_demo1 (VS = VTI_multishot_qacoustic_fd_subroutine_c3.f90,
// VM = VTI_multishot_qacoustic_fd_main_c3.f90): the coupled u / q second-order system with
// 10th-order second derivatives inside and split PML fields on the left, right, top and bottom.
//
// Parity unpinned: the shipped main program does not compile (the second extrapolation_one_step_2
// call ends its argument list with an empty argument, VM:462-463), no Fortran compiler is present,
// and the folder ships no record of its output.  The restatement follows the subroutines in their
// written operation order (every multiply and add rounded separately in float; the time loop of
// VM:413-505 with that trailing comma removed); it is checked by FP32 against FP64, symmetry and
// the isotropic limit in tests/test_vti_oracle.py.
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace {

// VS:1264-1363 coefficient_2nd and VS:1366-1472 coefficient_1st: the matrix a(i,j) = i^p / p!
// (p = 2j or 2j-1) inverted by successive Sherman-Morrison updates of the identity, one row of a
// at a time; coefficient(i) = (inv(a) (0.5 e_i))(1).
template <class T>
int coefs(int order, int first, T* out) {
    const int k = first ? (order + 1) / 2 : order / 2;
    if (k < 1 || k > 8) return 1;
    std::vector<T> a(k * k), inv(k * k, T(0)), temp(k), f4(k), f2(k * k), f3(k * k);
    for (int i = 1; i <= k; i++)
        for (int j = 1; j <= k; j++) {
            const int p = first ? 2 * j - 1 : 2 * j;
            T num = 1, fact = 1;
            for (int m = 0; m < p; m++) num = num * T(i);      // i**p (exact for these sizes)
            for (int m = 1; m <= p; m++) fact = fact * T(m);   // factorical(p, 1.0)
            a[(i - 1) * k + (j - 1)] = num / fact;
        }
    for (int d = 0; d < k; d++) inv[d * k + d] = 1;
    for (int i = 0; i < k; i++) {
        for (int c = 0; c < k; c++) temp[c] = a[i * k + c];
        temp[i] = temp[i] - 1;
        T f1 = 0;
        for (int r = 0; r < k; r++) f1 = f1 + temp[r] * inv[r * k + i];
        f1 = f1 + 1;
        for (int r = 0; r < k; r++) f4[r] = inv[r * k + i];
        for (int j1 = 0; j1 < k; j1++)
            for (int i1 = 0; i1 < k; i1++) f2[j1 * k + i1] = f4[j1] * temp[i1];
        for (int j = 0; j < k; j++)
            for (int l = 0; l < k; l++) {
                T s = 0;
                for (int m = 0; m < k; m++) s = s + f2[j * k + m] * inv[m * k + l];
                f3[j * k + l] = s;
            }
        for (int j = 0; j < k; j++)
            for (int l = 0; l < k; l++) f3[j * k + l] = f3[j * k + l] / f1;
        for (int q = 0; q < k * k; q++) inv[q] = inv[q] - f3[q];
    }
    for (int i = 0; i < k; i++) {
        T s = 0;  // matmul(inv_a, b)(1) with b = 0.5 e_i
        for (int m = 0; m < k; m++) s = s + inv[m] * (m == i ? T(0.5) : T(0));
        out[i] = s;
    }
    return 0;
}

template <class T>
struct Grid {
    int nx, nz, nxl, nxr, nzu, nzd;
    int NXH;  // nx + 10: the fields are u(-4:nx+5, -4:nz+5), i fastest
    std::vector<T> f[4];  // u1 u2 q1 q2
    // split PML fields, pairs (_1, _2): x strips (nxl+nxr, nz) of u1, u2, u2_tmp, u3 for u and q;
    // z strips (nx, nzu+nzd) of u1, u2, u2_tmp, u3 for u
    std::vector<T> ux[4][2], uz[4][2], qx[4][2];
    long long F(int i, int j) const { return (long long)(j + 4) * NXH + (i + 4); }
    long long X(int is, int j) const { return (long long)(j - 1) * (nxl + nxr) + (is - 1); }
    long long Z(int i, int js) const { return (long long)(js - 1) * nx + (i - 1); }
};

template <class T>
int run(const OracleVtiCfg* c, const float* vz_m, const float* eps_m, const float* del_m, T* record) {
    const int range = c->xmax - c->xmin + 1;
    if (range < 1 || c->nx_bound_r < 2 || c->nz_bound_d < 2 || c->nx_bound_l < 0 || c->nz_bound_u < 0) return 1;
    if (c->order_explicit != 10 || c->order_pml_2nd != 10 || (c->order_pml_1st != 9 && c->order_pml_1st != 10))
        return 1;  // the stencils are written out with five coefficients (VS:511-551)
    Grid<T> g;
    g.nxl = c->nx_bound_l; g.nxr = c->nx_bound_r; g.nzu = c->nz_bound_u; g.nzd = c->nz_bound_d;
    const int nx = range + g.nxl + g.nxr - 2, nz = c->nz_v + g.nzu + g.nzd - 2;  // VM:248-249
    g.nx = nx; g.nz = nz; g.NXH = nx + 10;
    const size_t nf = (size_t)(nx + 10) * (nz + 10);
    for (auto& v : g.f) v.assign(nf, T(0));
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 2; b++) {
            g.ux[a][b].assign((size_t)(g.nxl + g.nxr) * nz, T(0));
            g.qx[a][b].assign((size_t)(g.nxl + g.nxr) * nz, T(0));
            g.uz[a][b].assign((size_t)nx * (g.nzu + g.nzd), T(0));
        }
    T cE[5], c2[5], c1[5];
    if (coefs<T>(10, 0, cE) || coefs<T>(10, 0, c2) || coefs<T>(c->order_pml_1st, 1, c1)) return 1;

    // get_currshot_parameters (VS:268-338): the window with edge-replicated vz pads; epsilon and
    // delta only inside the window, then zero on rows 1 .. nsz0 + nzu + 6 (VM:405-408)
    std::vector<T> vz((size_t)nx * nz, T(0)), ep((size_t)nx * nz, T(0)), de((size_t)nx * nz, T(0));
    auto M = [&](int i, int j) { return (size_t)(j - 1) * nx + (i - 1); };
    for (int i = 1; i <= range; i++) {
        int io = i + c->xmin;
        io = io < 1 ? 1 : (io > c->nx_v ? c->nx_v : io);
        for (int j = 1; j <= c->nz_v; j++) {
            const size_t src = (size_t)(io - 1) * c->nz_v + (j - 1);
            vz[M(i + g.nxl, g.nzu + j)] = (T)vz_m[src];
            ep[M(i + g.nxl, g.nzu + j)] = (T)eps_m[src];
            de[M(i + g.nxl, g.nzu + j)] = (T)del_m[src];
        }
    }
    for (int j = 1; j <= g.nzu; j++)
        for (int i = 1; i <= nx; i++) vz[M(i, j)] = vz[M(i, g.nzu + 1)];
    for (int j = g.nzu + c->nz_v + 1; j <= nz; j++)
        for (int i = 1; i <= nx; i++) vz[M(i, j)] = vz[M(i, g.nzu + c->nz_v)];
    for (int j = 1; j <= nz; j++)
        for (int i = 1; i <= g.nxl; i++) vz[M(i, j)] = vz[M(g.nxl + 1, j)];
    for (int j = 1; j <= nz; j++)
        for (int i = g.nxl + range + 1; i <= nx; i++) vz[M(i, j)] = vz[M(g.nxl + range, j)];
    for (int j = 1; j <= c->nsz0 + g.nzu + 6 && j <= nz; j++)
        for (int i = 1; i <= nx; i++) ep[M(i, j)] = de[M(i, j)] = T(0);
    const int snx = c->nsx - c->xmin + g.nxl, snz = c->nsz0 + g.nzu;
    if (snx < 1 || snx > nx || snz < 1 || snz > nz) return 1;

    const T dx = (T)c->dx, dz = (T)c->dz, dt = (T)c->dt, f0 = (T)c->f0;
    const T Rr = (T)1.0e-3, pi = (T)3.1415926;
    const T L = std::log(T(1) / Rr);
    const T two = 2, one = 1, three = 3;
    const int nwt = (int)std::lround((double)((T(2.0) * T(0.07)) / dt)) + 1;  // VM:250 nint(2*0.07/dt)+1
    const int half = (int)std::lround((double)(nwt - 1) / 2.0);
    int rrow = c->nrz0 + g.nzu;
    const bool low = rrow < 6;
    if (low) rrow = 6;
    if (rrow > nz) return 1;

    // sums of VS:511-551 (second derivative, fd_coe) and VS:565-630 (PML first / second)
    auto d2 = [&](const std::vector<T>& u, int i, int j, int di, int dj, const T* cf, T h) {
        const T u0 = u[g.F(i, j)];
        T s = cf[0] * ((u[g.F(i + di, j + dj)] + u[g.F(i - di, j - dj)]) - two * u0);
        for (int m = 2; m <= 5; m++)
            s = s + cf[m - 1] * ((u[g.F(i + m * di, j + m * dj)] + u[g.F(i - m * di, j - m * dj)]) - two * u0);
        return s / (h * h);
    };
    auto d1 = [&](const std::vector<T>& u, int i, int j, int di, int dj, T h) {
        T s = c1[0] * (u[g.F(i + di, j + dj)] - u[g.F(i - di, j - dj)]);
        for (int m = 2; m <= 5; m++) s = s + c1[m - 1] * (u[g.F(i + m * di, j + m * dj)] - u[g.F(i - m * di, j - m * dj)]);
        return s / h;
    };
    for (int it = 1; it <= c->nt + half; it++) {
        const int cu = (it % 2 == 1) ? 1 : 0, ou = 1 - cu;  // current and new slots (VM:417-505)
        std::vector<T>& U = g.f[cu];
        std::vector<T>& Un = g.f[ou];
        std::vector<T>& Q = g.f[2 + cu];
        std::vector<T>& Qn = g.f[2 + ou];
        if (it <= nwt) {  // VM:420-424 / VM:468-472
            const T b = ((pi * f0) * ((T)it - (T(0.07) / dt))) * dt;
            U[g.F(snx, snz)] = U[g.F(snx, snz)] + std::exp(-(b * b)) * (one - two * (b * b));
        }
        // extrapolation_one_step_1 (VS:432-960): new u into the slot of the old one
#pragma omp parallel for schedule(static)
        for (int j = 1; j <= nz; j++)
            for (int i = 1; i <= nx; i++) {
                const size_t m = M(i, j);
                const T v = vz[m];
                if (i > g.nxl && i < nx - g.nxr + 1 && j > g.nzu && j < nz - g.nzd + 1) {
                    const T sxu = d2(U, i, j, 1, 0, cE, dx), szu = d2(U, i, j, 0, 1, cE, dz), sxq = d2(Q, i, j, 1, 0, cE, dx);
                    Un[g.F(i, j)] = ((two * U[g.F(i, j)]) - Un[g.F(i, j)]) +
                                    ((dt * dt) * (v * v)) * (((one + two * de[m]) * (sxu + sxq)) + szu);
                } else if (i <= g.nxl || i >= nx - g.nxr + 1) {
                    const bool left = i <= g.nxl;
                    const T vn = v * std::sqrt(one + two * de[m]);
                    const T vx = v * std::sqrt(one + two * ep[m]);
                    T s1 = d1(U, i, j, 1, 0, dx);
                    const T s1q = d1(Q, i, j, 1, 0, dx);
                    T s2 = d2(U, i, j, 1, 0, c2, dx);
                    const T sz2 = d2(U, i, j, 0, 1, c2, dz);
                    const T s2q = d2(Q, i, j, 1, 0, c2, dx);
                    s1 = s1 + s1q;
                    s2 = s2 + s2q;
                    const T axis = (T)(left ? i - (g.nxl + 1) : i - (nx - g.nxr)) * dx;
                    const T thick = (T)(left ? g.nxl : g.nxr) * dx;
                    const int is = left ? i : i - (nx - g.nxr) + g.nxl;
                    const T A = (three * vx) / (two * thick);
                    const T d = (A * ((axis / thick) * (axis / thick))) * L;
                    const T dd = (A * ((two * axis) / (thick * thick))) * L;
                    const long long x = g.X(is, j);
                    T* a1 = g.ux[0][ou].data(); const T* a1o = g.ux[0][cu].data();
                    T* a2 = g.ux[1][ou].data(); const T* a2o = g.ux[1][cu].data();
                    T* t2 = g.ux[2][ou].data(); const T* t2o = g.ux[2][cu].data();
                    T* a3 = g.ux[3][ou].data(); const T* a3o = g.ux[3][cu].data();
                    const T h2 = dx * dx;
                    const T P = ((two * h2) + (((two * d) * dt) * h2)) - (((d * d) * h2) * (dt * dt));
                    const T Den = h2 + (((two * d) * dt) * h2);
                    a1[x] = (((a1o[x] * P) - (h2 * a1[x])) + (((vn * vn) * (dt * dt)) * (s2 * h2))) / Den;
                    const T P2 = ((two * dx) + (((two * d) * dt) * dx)) - (((dt * dt) * dx) * (d * d));
                    const T Den2 = dx + (((two * d) * dt) * dx);
                    t2[x] = (((t2o[x] * P2) - (dx * t2[x])) - ((((vn * vn) * (dt * dt)) * dd) * (s1 * dx))) / Den2;
                    a2[x] = (a2o[x] * (one - (d * dt))) + (t2[x] * dt);
                    a3[x] = ((two * a3o[x]) - a3[x]) + ((((v * v) * (dt * dt)) * (sz2 * (dz * dz))) / (dz * dz));
                    Un[g.F(i, j)] = (a1[x] + a2[x]) + a3[x];
                } else {
                    const bool top = j <= g.nzu;
                    const T vn = v * std::sqrt(one + two * de[m]);
                    const T sz1 = d1(U, i, j, 0, 1, dx);  // divided by dx as written (VS:796, 880)
                    const T sx2 = d2(U, i, j, 1, 0, c2, dx);
                    const T sz2 = d2(U, i, j, 0, 1, c2, dz);
                    const T sx2q = d2(Q, i, j, 1, 0, c2, dx);
                    const T axis = (T)(top ? j - (g.nzu + 1) : j - (nz - g.nzd)) * dz;
                    const T thick = (T)(top ? g.nzu : g.nzd) * dz;
                    const int js = top ? j : j - (nz - g.nzd) + g.nzu;
                    const T A = (three * v) / (two * thick);
                    const T d = (A * ((axis / thick) * (axis / thick))) * L;
                    const T dd = (A * ((two * axis) / (thick * thick))) * L;
                    const long long z = g.Z(i, js);
                    T* a1 = g.uz[0][ou].data(); const T* a1o = g.uz[0][cu].data();
                    T* a2 = g.uz[1][ou].data(); const T* a2o = g.uz[1][cu].data();
                    T* t2 = g.uz[2][ou].data(); const T* t2o = g.uz[2][cu].data();
                    T* a3 = g.uz[3][ou].data(); const T* a3o = g.uz[3][cu].data();
                    const T h2 = dz * dz;
                    const T P = ((two * h2) + (((two * d) * dt) * h2)) - (((d * d) * h2) * (dt * dt));
                    const T Den = h2 + (((two * d) * dt) * h2);
                    a1[z] = (((a1o[z] * P) - (h2 * a1[z])) + (((v * v) * (dt * dt)) * (sz2 * h2))) / Den;
                    const T P2 = ((two * dz) + (((two * d) * dt) * dz)) - (((dt * dt) * dz) * (d * d));
                    const T Den2 = dz + (((two * d) * dt) * dz);
                    t2[z] = (((t2o[z] * P2) - (dz * t2[z])) - ((((v * v) * (dt * dt)) * dd) * (sz1 * dz))) / Den2;
                    a2[z] = (a2o[z] * (one - (d * dt))) + (t2[z] * dt);
                    a3[z] = ((two * a3o[z]) - a3[z]) + (((vn * vn) * (dt * dt)) * (sx2 + sx2q));
                    Un[g.F(i, j)] = (a1[z] + a2[z]) + a3[z];
                }
            }
        // extrapolation_one_step_2 (VS:965-1258): new q from the current u (not the new one)
#pragma omp parallel for schedule(static)
        for (int j = 1; j <= nz; j++)
            for (int i = 1; i <= nx; i++) {
                const size_t m = M(i, j);
                const T v = vz[m];
                if (i > g.nxl && i < nx - g.nxr + 1) {
                    const T sxu = d2(U, i, j, 1, 0, cE, dx), sxq = d2(Q, i, j, 1, 0, cE, dx);
                    Qn[g.F(i, j)] = ((two * Q[g.F(i, j)]) - Qn[g.F(i, j)]) +
                                    ((dt * dt) * (v * v)) * ((two * (ep[m] - de[m])) * (sxq + sxu));
                } else {
                    const bool left = i <= g.nxl;
                    const T vn = v * std::sqrt(one + two * de[m]);
                    const T vx = v * std::sqrt(one + two * ep[m]);
                    T s1 = d1(Q, i, j, 1, 0, dx);
                    const T s1u = d1(U, i, j, 1, 0, dx);
                    T s2 = d2(Q, i, j, 1, 0, c2, dx);
                    const T s2u = d2(U, i, j, 1, 0, c2, dx);
                    s1 = s1 + s1u;
                    s2 = s2 + s2u;
                    const T axis = (T)(left ? i - (g.nxl + 1) : i - (nx - g.nxr)) * dx;
                    const T thick = (T)(left ? g.nxl : g.nxr) * dx;
                    const int is = left ? i : i - (nx - g.nxr) + g.nxl;
                    const T A = (three * vx) / (two * thick);
                    const T d = (A * ((axis / thick) * (axis / thick))) * L;
                    const T dd = (A * ((two * axis) / (thick * thick))) * L;
                    const T k2 = (vx * vx) - (vn * vn);
                    const long long x = g.X(is, j);
                    T* a1 = g.qx[0][ou].data(); const T* a1o = g.qx[0][cu].data();
                    T* a2 = g.qx[1][ou].data(); const T* a2o = g.qx[1][cu].data();
                    T* t2 = g.qx[2][ou].data(); const T* t2o = g.qx[2][cu].data();
                    const T h2 = dx * dx;
                    const T P = ((two * h2) + (((two * d) * dt) * h2)) - (((d * d) * h2) * (dt * dt));
                    const T Den = h2 + (((two * d) * dt) * h2);
                    a1[x] = (((a1o[x] * P) - (h2 * a1[x])) + ((k2 * (dt * dt)) * (s2 * h2))) / Den;
                    const T P2 = ((two * dx) + (((two * d) * dt) * dx)) - (((dt * dt) * dx) * (d * d));
                    const T Den2 = dx + (((two * d) * dt) * dx);
                    t2[x] = (((t2o[x] * P2) - (dx * t2[x])) - (((k2 * (dt * dt)) * dd) * (s1 * dx))) / Den2;
                    a2[x] = (a2o[x] * (one - (d * dt))) + (t2[x] * dt);
                    Qn[g.F(i, j)] = a1[x] + a2[x];
                }
            }
        // recording (VM:446-453 / VM:494-501): the new u on the receiver row, traces nxl+1 ..
        const int iit = it - half;
        if ((!low && iit >= 1) || (low && iit > 1))
            for (int ix = 1; ix <= range && iit <= c->nt; ix++)
                record[(size_t)(ix - 1) * c->nt + (iit - 1)] = Un[g.F(g.nxl + ix, rrow)];
    }
    return 0;
}

}  // namespace

extern "C" {

int oracle_vti_coef_f32(int order, int first, float* out) { return coefs<float>(order, first, out); }
int oracle_vti_coef_f64(int order, int first, double* out) { return coefs<double>(order, first, out); }

int oracle_vti_f32(const OracleVtiCfg* c, const float* vz, const float* eps, const float* delta, float* record) {
    if (!c || !vz || !eps || !delta || !record) return 1;
    std::memset(record, 0, sizeof(float) * (size_t)(c->xmax - c->xmin + 1) * c->nt);
    return run<float>(c, vz, eps, delta, record);
}

int oracle_vti_f64(const OracleVtiCfg* c, const float* vz, const float* eps, const float* delta, double* record) {
    if (!c || !vz || !eps || !delta || !record) return 1;
    std::memset(record, 0, sizeof(double) * (size_t)(c->xmax - c->xmin + 1) * c->nt);
    return run<double>(c, vz, eps, delta, record);
}

}  // extern "C"
