// ORACLE -- test infrastructure only. FP64 CPU adjoint of the acoustic velocity-pressure
// time loop of forward/Acoustic_FD_by_ss/src/Acoustic_1order_FD.cpp (AFD:237-380), used by
// tests/ to check the GPU gradient.  The reference has no adjoint; this file states the exact
// transpose of its discrete forward operator.
//
// Forward (same as AFD, written with the unsponged velocities U, W of the previous step, so
// that AFD's "Vx2 = sponged Vx1" is a*U):
//   U' = M (a U - B_x S+x P),  W' = M (a W - B_z S+z P)             AFD:255-286, 329-336
//   D  = rdx S-x U' + rdz S-z W'                                    AFD:293-311
//   P1 = M (P - K D),  K = DEN Vp^2 dt                              AFD:289-314
//   Phat = a P1;  record = Phat at receivers;  P <- Phat - s w[k+1] e_src   AFD:247-251,337-338,376
// with S+ q(i) = sum_m C_m (q[i+m+1] - q[i-m]),  S- q(i) = sum_m C_m (q[i+m] - q[i-m-1]),
// M = 1 on the updated interior [R, N-R)^2, a = AFD sponge, B = dt/(DEN d), s = dt DEN Vp at
// the source.  Since (S+)^T = -S- and (S-)^T = -S+, one adjoint step is
//   mu = Q + R^T res[k],  l1 = a mu,  nu = M K l1
//   X' = X + rdx S+x nu,  Z' = Z + rdz S+z nu
//   Q  <- M l1 + S-x(B_x M X') + S-z(B_z M Z'),  X <- a M X',  Z <- a M Z'
//   g  += l1 M D_k
// and d misfit / d Vp = -2 DEN Vp dt g, plus -dt DEN sum_j Q_j[src] w[j] at the source cell.
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace {

int coeffs(int radius, double* c) {
    float f[8];
    if (oracle_afd_coeffs(radius, f) != 0) return -1;
    for (int m = 0; m < radius; m++) c[m] = (double)f[m];
    return 0;
}

struct Grid {
    int nx, nz, R;
    size_t n() const { return (size_t)nx * nz; }
};

// S+ along x (dir 0) or z (dir 1) at every updated cell; other cells 0
void splus(const Grid& g, const double* C, const std::vector<double>& q, std::vector<double>& out, int dir) {
    const int nx = g.nx, nz = g.nz, R = g.R;
    const size_t st = dir == 0 ? (size_t)nz : 1;
    std::fill(out.begin(), out.end(), 0.0);
#pragma omp parallel for schedule(static)
    for (int i = R; i < nx - R; i++)
        for (int j = R; j < nz - R; j++) {
            const size_t c = (size_t)i * nz + j;
            double s = 0;
            for (int m = 0; m < R; m++) s += C[m] * (q[c + (m + 1) * st] - q[c - m * st]);
            out[c] = s;
        }
}

// S- along x or z.  full = false: at the updated cells (forward use).  full = true: at every
// cell, q taken as zero outside the grid -- the transpose of S+ restricted to updated cells
// reaches into the frozen rim, which matters for a source placed there.
void sminus(const Grid& g, const double* C, const std::vector<double>& q, std::vector<double>& out, int dir,
            bool full = false) {
    const int nx = g.nx, nz = g.nz, R = g.R;
    std::fill(out.begin(), out.end(), 0.0);
    const int lo = full ? 0 : R;
#pragma omp parallel for schedule(static)
    for (int i = lo; i < nx - lo; i++)
        for (int j = lo; j < nz - lo; j++) {
            double s = 0;
            for (int m = 0; m < R; m++) {
                const int ia = dir == 0 ? i + m : i, ja = dir == 0 ? j : j + m;
                const int ib = dir == 0 ? i - m - 1 : i, jb = dir == 0 ? j : j - m - 1;
                const double qa = (ia < nx && ja < nz) ? q[(size_t)ia * nz + ja] : 0.0;
                const double qb = (ib >= 0 && jb >= 0) ? q[(size_t)ib * nz + jb] : 0.0;
                s += C[m] * (qa - qb);
            }
            out[(size_t)i * nz + j] = s;
        }
}

}  // namespace

extern "C" int oracle_afd_gradient_f64(const OracleAfdCfg* cfg, const float* vp, const float* den,
                                       const float* wavelet, const float* obs, double* misfit, double* grad_vp,
                                       double* dw, double* records) {
    const int nx = cfg->nx, nz = cfg->nz, R = cfg->radius, nt = cfg->nt;
    double C[8];
    if (nx <= 2 * R || nz <= 2 * R || nt < 1 || coeffs(R, C) != 0) return 1;
    const Grid g{nx, nz, R};
    const size_t n = g.n();
    std::vector<float> absf(n);
    oracle_afd_sponge(nx, nz, cfg->pml, absf.data());
    std::vector<double> a(n), M(n, 0.0), K(n), Bx(n), Bz(n);
    const double dt = cfg->dt, rdx = 1.0 / (double)cfg->dx, rdz = 1.0 / (double)cfg->dz;
    for (size_t c = 0; c < n; c++) {
        a[c] = absf[c];
        K[c] = (double)den[c] * vp[c] * vp[c] * dt;
        Bx[c] = dt / ((double)den[c] * cfg->dx);
        Bz[c] = dt / ((double)den[c] * cfg->dz);
    }
    for (int i = R; i < nx - R; i++)
        for (int j = R; j < nz - R; j++) M[(size_t)i * nz + j] = 1.0;
    const size_t src = (size_t)cfg->sx * nz + cfg->sz;
    const double s_src = dt * (double)den[src] * vp[src];

    // ---- forward, keeping D_k for the imaging condition ----
    std::vector<double> P(n, 0.0), U(n, 0.0), W(n, 0.0), t1(n), t2(n), t3(n);
    std::vector<double> D((size_t)nt * n);
    std::vector<double> rec((size_t)cfg->nrec * nt);
    P[src] -= s_src * wavelet[0];
    for (int k = 0; k < nt; k++) {
        splus(g, C, P, t1, 0);
        splus(g, C, P, t2, 1);
        for (size_t c = 0; c < n; c++) {
            U[c] = M[c] * (a[c] * U[c] - Bx[c] * t1[c]);
            W[c] = M[c] * (a[c] * W[c] - Bz[c] * t2[c]);
        }
        sminus(g, C, U, t1, 0);
        sminus(g, C, W, t2, 1);
        double* Dk = D.data() + (size_t)k * n;
        for (size_t c = 0; c < n; c++) {
            Dk[c] = rdx * t1[c] + rdz * t2[c];
            P[c] = a[c] * (M[c] * (P[c] - K[c] * Dk[c]));
        }
        for (int r = 0; r < cfg->nrec; r++) rec[(size_t)r * nt + k] = P[(size_t)cfg->rec_x[r] * nz + cfg->rec_z[r]];
        if (k + 1 < nt) P[src] -= s_src * wavelet[k + 1];
    }
    double J = 0.0;
    for (size_t i = 0; i < rec.size(); i++) {
        const double rr = rec[i] - (double)obs[i];
        J += 0.5 * rr * rr;
    }
    if (misfit) *misfit = J;
    if (records) std::memcpy(records, rec.data(), rec.size() * sizeof(double));

    // ---- adjoint ----
    std::vector<double> Q(n, 0.0), X(n, 0.0), Z(n, 0.0), gacc(n, 0.0), l1(n), nu(n);
    std::vector<double> qsrc(nt);
    for (int k = nt - 1; k >= 0; k--) {
        for (int r = 0; r < cfg->nrec; r++) {
            const size_t c = (size_t)cfg->rec_x[r] * nz + cfg->rec_z[r];
            Q[c] += rec[(size_t)r * nt + k] - (double)obs[(size_t)r * nt + k];
        }
        for (size_t c = 0; c < n; c++) {
            l1[c] = a[c] * Q[c];
            nu[c] = M[c] * K[c] * l1[c];
        }
        splus(g, C, nu, t1, 0);
        splus(g, C, nu, t2, 1);
        for (size_t c = 0; c < n; c++) {
            X[c] = X[c] + rdx * t1[c];  // X'
            Z[c] = Z[c] + rdz * t2[c];  // Z'
            t3[c] = Bx[c] * M[c] * X[c];
        }
        sminus(g, C, t3, t1, 0, true);
        for (size_t c = 0; c < n; c++) t3[c] = Bz[c] * M[c] * Z[c];
        sminus(g, C, t3, t2, 1, true);
        const double* Dk = D.data() + (size_t)k * n;
        for (size_t c = 0; c < n; c++) {
            gacc[c] += l1[c] * M[c] * Dk[c];
            Q[c] = M[c] * l1[c] + t1[c] + t2[c];
            X[c] = a[c] * M[c] * X[c];
            Z[c] = a[c] * M[c] * Z[c];
        }
        qsrc[k] = Q[src];
    }
    if (grad_vp) {
        for (size_t c = 0; c < n; c++) grad_vp[c] = -2.0 * (double)den[c] * vp[c] * dt * gacc[c];
        double sw = 0.0;
        for (int j = 0; j < nt; j++) sw += qsrc[j] * wavelet[j];
        grad_vp[src] += -dt * (double)den[src] * sw;
    }
    if (dw)  // d misfit / d wavelet[j] = -s Q_j[src]
        for (int j = 0; j < nt; j++) dw[j] = -s_src * qsrc[j];
    return 0;
}
