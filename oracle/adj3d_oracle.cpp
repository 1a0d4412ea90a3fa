// ORACLE -- test infrastructure only. FP64 CPU adjoint of the 3-D velocity-pressure scheme
// restated in oracle/afd3d_oracle.cpp (the 2-D scheme of
// forward/Acoustic_FD_by_ss/src/Acoustic_1order_FD.cpp, AFD:237-380, with a y axis), used by
// tests/ to check the GPU 3-D gradient.  No reference adjoint exists; this file states the exact
// transpose of the discrete forward operator, axis by axis as oracle/adj_oracle.cpp does in 2-D:
//   forward   P <- P - s w[k] e_src (before the step),  U_a' = M (a U_a - B_a S+a P)  (a = x, y, z)
//             D = sum_a rd_a S-a U_a',  P' = a M (P - K D),  record = P' at the receivers
//   adjoint   mu = Q + R^T res[k],  l1 = a mu,  nu = M K l1
//             X_a' = X_a + rd_a S+a nu,  Q <- M l1 + sum_a S-a(B_a M X_a'),  X_a <- a M X_a'
//             g += l1 M D_k
// with U the velocities before the sponge (the restatement multiplies them by the sponge after
// the step), M = 1 on [R, N-R)^3, K = DEN Vp^2 dt, B_a = dt / (DEN d_a), s = dt DEN Vp at the
// source.  d misfit / d Vp = -2 DEN Vp dt g, plus -dt DEN sum_j Q_j[src] w[j] at the source.
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace {

struct G3 {
    int nx, ny, nz, R;
    size_t n() const { return (size_t)nx * ny * nz; }
    size_t at(int x, int y, int z) const { return ((size_t)x * ny + y) * nz + z; }
    size_t stride(int dir) const { return dir == 0 ? (size_t)ny * nz : (dir == 1 ? (size_t)nz : 1); }
};

// S+ along axis dir at every updated cell, other cells 0
void splus3(const G3& g, const double* C, const std::vector<double>& q, std::vector<double>& out, int dir) {
    const size_t st = g.stride(dir);
    std::fill(out.begin(), out.end(), 0.0);
#pragma omp parallel for schedule(static)
    for (int x = g.R; x < g.nx - g.R; x++)
        for (int y = g.R; y < g.ny - g.R; y++)
            for (int z = g.R; z < g.nz - g.R; z++) {
                const size_t c = g.at(x, y, z);
                double s = 0;
                for (int m = 0; m < g.R; m++) s += C[m] * (q[c + (m + 1) * st] - q[c - m * st]);
                out[c] = s;
            }
}

// S- along axis dir; full = true evaluates it at every cell with q = 0 outside the grid (the
// transpose of S+ restricted to the updated cells)
void sminus3(const G3& g, const double* C, const std::vector<double>& q, std::vector<double>& out, int dir,
             bool full) {
    std::fill(out.begin(), out.end(), 0.0);
    const int lo = full ? 0 : g.R;
    const int n[3] = {g.nx, g.ny, g.nz};
#pragma omp parallel for schedule(static)
    for (int x = lo; x < g.nx - lo; x++)
        for (int y = lo; y < g.ny - lo; y++)
            for (int z = lo; z < g.nz - lo; z++) {
                int p[3] = {x, y, z};
                double s = 0;
                for (int m = 0; m < g.R; m++) {
                    int pa[3] = {p[0], p[1], p[2]}, pb[3] = {p[0], p[1], p[2]};
                    pa[dir] += m;
                    pb[dir] -= m + 1;
                    const double qa = pa[dir] < n[dir] ? q[g.at(pa[0], pa[1], pa[2])] : 0.0;
                    const double qb = pb[dir] >= 0 ? q[g.at(pb[0], pb[1], pb[2])] : 0.0;
                    s += C[m] * (qa - qb);
                }
                out[g.at(x, y, z)] = s;
            }
}

}  // namespace

extern "C" int oracle_afd3d_gradient_f64(const OracleAfd3Cfg* cfg, const float* vp, const float* den,
                                         const float* wavelet, const float* obs, double* misfit, double* grad_vp,
                                         double* dw, double* records) {
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz, R = cfg->radius, nt = cfg->nt;
    float cf[8];
    if (nx <= 2 * R || ny <= 2 * R || nz <= 2 * R || nt < 1 || R < 1 || R > 8 || oracle_afd_coeffs(R, cf) != 0)
        return 1;
    double C[8];
    for (int m = 0; m < R; m++) C[m] = cf[m];
    const G3 g{nx, ny, nz, R};
    const size_t n = g.n();
    std::vector<float> absf(n);
    if (oracle_afd3d_sponge(nx, ny, nz, cfg->pml, absf.data())) return 1;
    const double dt = cfg->dt, d[3] = {cfg->dx, cfg->dy, cfg->dz};
    std::vector<double> a(n), M(n, 0.0), K(n), B[3] = {std::vector<double>(n), std::vector<double>(n),
                                                       std::vector<double>(n)};
    for (size_t c = 0; c < n; c++) {
        const double dn = den ? (double)den[c] : (double)cfg->den_c;
        a[c] = absf[c];
        K[c] = dn * vp[c] * vp[c] * dt;
        for (int ax = 0; ax < 3; ax++) B[ax][c] = dt / (dn * d[ax]);
    }
    for (int x = R; x < nx - R; x++)
        for (int y = R; y < ny - R; y++)
            for (int z = R; z < nz - R; z++) M[g.at(x, y, z)] = 1.0;
    const size_t src = g.at(cfg->sx, cfg->sy, cfg->sz);
    // (dt * den) * vp rounded to float, as the restatement and the GPU inject it (AFD:250)
    float s_f = cfg->dt * (den ? den[src] : cfg->den_c);
    s_f = s_f * vp[src];
    const double s_src = s_f;

    // ---- forward, keeping D_k ----
    std::vector<double> P(n, 0.0), t(n), acc(n);
    std::vector<std::vector<double>> U(3, std::vector<double>(n, 0.0));
    std::vector<double> D((size_t)nt * n), rec((size_t)cfg->nrec * nt);
    for (int k = 0; k < nt; k++) {
        P[src] -= s_src * wavelet[k];
        for (int ax = 0; ax < 3; ax++) {
            splus3(g, C, P, t, ax);
            for (size_t c = 0; c < n; c++) U[ax][c] = M[c] * (a[c] * U[ax][c] - B[ax][c] * t[c]);
        }
        double* Dk = D.data() + (size_t)k * n;
        std::fill(Dk, Dk + n, 0.0);
        for (int ax = 0; ax < 3; ax++) {
            sminus3(g, C, U[ax], t, ax, false);
            for (size_t c = 0; c < n; c++) Dk[c] += t[c] / d[ax];
        }
        for (size_t c = 0; c < n; c++) P[c] = a[c] * (M[c] * (P[c] - K[c] * Dk[c]));
        for (int r = 0; r < cfg->nrec; r++)
            rec[(size_t)r * nt + k] = P[g.at(cfg->rec_x[r], cfg->rec_y[r], cfg->rec_z[r])];
    }
    double J = 0.0;
    if (obs)
        for (size_t i = 0; i < rec.size(); i++) {
            const double rr = rec[i] - (double)obs[i];
            J += 0.5 * rr * rr;
        }
    if (misfit) *misfit = J;
    if (records) std::memcpy(records, rec.data(), rec.size() * sizeof(double));
    if (!obs || (!grad_vp && !dw)) return 0;

    // ---- adjoint ----
    std::vector<double> Q(n, 0.0), gacc(n, 0.0), l1(n), nu(n), qsrc(nt);
    std::vector<std::vector<double>> X(3, std::vector<double>(n, 0.0));
    for (int k = nt - 1; k >= 0; k--) {
        for (int r = 0; r < cfg->nrec; r++)
            Q[g.at(cfg->rec_x[r], cfg->rec_y[r], cfg->rec_z[r])] +=
                rec[(size_t)r * nt + k] - (double)obs[(size_t)r * nt + k];
        for (size_t c = 0; c < n; c++) {
            l1[c] = a[c] * Q[c];
            nu[c] = M[c] * K[c] * l1[c];
        }
        for (size_t c = 0; c < n; c++) acc[c] = M[c] * l1[c];
        for (int ax = 0; ax < 3; ax++) {
            splus3(g, C, nu, t, ax);
            for (size_t c = 0; c < n; c++) X[ax][c] += t[c] / d[ax];  // X'
            std::vector<double> bm(n);
            for (size_t c = 0; c < n; c++) bm[c] = B[ax][c] * M[c] * X[ax][c];
            sminus3(g, C, bm, t, ax, true);
            for (size_t c = 0; c < n; c++) {
                acc[c] += t[c];
                X[ax][c] = a[c] * M[c] * X[ax][c];
            }
        }
        const double* Dk = D.data() + (size_t)k * n;
        for (size_t c = 0; c < n; c++) {
            gacc[c] += l1[c] * M[c] * Dk[c];
            Q[c] = acc[c];
        }
        qsrc[k] = Q[src];
    }
    if (grad_vp) {
        for (size_t c = 0; c < n; c++)
            grad_vp[c] = -2.0 * (den ? (double)den[c] : (double)cfg->den_c) * vp[c] * dt * gacc[c];
        double sw = 0.0;
        for (int j = 0; j < nt; j++) sw += qsrc[j] * wavelet[j];
        grad_vp[src] += -dt * (den ? (double)den[src] : (double)cfg->den_c) * sw;
    }
    if (dw)
        for (int j = 0; j < nt; j++) dw[j] = -s_src * qsrc[j];
    return 0;
}
