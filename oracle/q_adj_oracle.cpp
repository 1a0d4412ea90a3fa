// ORACLE -- test infrastructure only. FP64 gradient of the viscoacoustic (vs = 0) scheme: the
// checker of the GPU d misfit / d vp and d misfit / d (1/Q).
//
// The forward is the vs = 0 reduction of the Q_forward step (forward/Q_forward/
// Q_multishot_fd_subroutine_fsbc_zy_rotated.f90, QS) on an already padded grid, held in the
// eight fields the GPU kernels hold:
//   velocity  vx = Ax (vx + dt b Dx0 S),  vz = Az (vz + dt b Dz0 S),  S = sx + sz + sr   (QS:969-990)
//   stress    sx = A'x (sx + dt p1 Dx1 vx) + stamp w_k dt / dz^2,  sz = A'z (sz + dt p1 Dz1 vz),
//             sr = sr + dt R,   rx = A'x (rx + f p2 Dx1 vx),  rz = A'z (rz + f p2 Dz1 vz),
//             rr = rr + f R,    R = rx + rz + rr (old), f = -dt / tau_sigma       (QS:993-1337)
//   record    S at the receivers after the step                                  (QM:452-459)
// with the rotated-staggered derivatives of QS:843-966, the split cosine sponges of QS:555-654,
// the density average and buoyancy of QS:434-469 and Blanch's tau of QS:473-551 (p1 = lambda
// tau_eps/tau_sigma, p2 = lambda (tau_eps/tau_sigma - 1), lambda = rho_avg vp^2, tau_eps/tau_sigma
// = 1 + kappa / Q), all in double.  The gradient is the exact adjoint of this discrete map
// (every forward step stored, no checkpoints): adjoint fields run backwards through the stress
// update, the transposed derivatives and the velocity update; the zero-lag correlation of the
// adjoint stresses with the forward derivatives gives d/dp1 and d/dp2, and the chain rule gives
// d/dvp and d/d(1/Q).  A separate restatement from the GPU code: plain loops, double precision.
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace {

struct Grid {
    int nx, nz, m;  // padded grid and zero margin around it
    int w, h;       // allocated width / height
    Grid(int nx_, int nz_) : nx(nx_), nz(nz_), m(6), w(nx_ + 12), h(nz_ + 12) {}
    size_t at(int x, int z) const { return (size_t)(x + m) * h + (z + m); }
    size_t size() const { return (size_t)w * h; }
};

const double kA[5] = {19845.0 / 16384.0, -735.0 / 8192.0, 567.0 / 40960.0, -405.0 / 229376.0, 35.0 / 294912.0};

// rotated-staggered derivative (QS:843-966) of u at (x, z): flag 0 / 1, x or z direction
double rsg(const Grid& g, const std::vector<double>& u, int x, int z, int flag, bool xdir, double hh) {
    double s = 0;
    for (int m = 0; m < 5; m++) {
        const int p = flag == 0 ? m : 1 + m, q = flag == 0 ? -1 - m : -m;  // the two offsets
        const double a = u[g.at(x + p, z + p)], b = u[g.at(x + q, z + q)];
        const double c = u[g.at(x + p, z + q)], d = u[g.at(x + q, z + p)];  // (z+q, x+p), (z+p, x+q)
        s += kA[m] * (xdir ? (a - b + c - d) : (a - b - c + d));
    }
    return hh * s;
}

// transpose of rsg: scatter-gather form, out(x', z') = sum over taps of sign * t(x' - dx, z' - dz)
double rsg_t(const Grid& g, const std::vector<double>& t, int x, int z, int flag, bool xdir, double hh) {
    double s = 0;
    for (int m = 0; m < 5; m++) {
        const int p = flag == 0 ? m : 1 + m, q = flag == 0 ? -1 - m : -m;
        // forward taps: +(x+p, z+p), -(x+q, z+q), (x+p, z+q) with sign c, (x+q, z+p) with sign -c
        const double cs = xdir ? 1.0 : -1.0;
        s += kA[m] * (t[g.at(x - p, z - p)] - t[g.at(x - q, z - q)] + cs * t[g.at(x - p, z - q)] - cs * t[g.at(x - q, z - p)]);
    }
    return hh * s;
}

}  // namespace

extern "C" int oracle_q_gradient_f64(const OracleQGradCfg* c, const float* vp, const float* rho, const float* q,
                                     const float* wavelet, const float* obs, double* misfit, double* grad_vp,
                                     double* grad_invq, double* dw, double* records) {
    const int nx = c->nx, nz = c->nz, np = c->np, nt = c->nt, nrec = c->nrec;
    if (nx < 12 || nz < 12 || np < 1 || 2 * np > nx || 2 * np > nz || nt < 1) return 1;
    Grid g(nx, nz);
    const size_t n = (size_t)nx * nz, N = g.size();
    auto mi = [&](int x, int z) { return (size_t)x * nz + z; };
    // QS:434-469 density average within the grid, then buoyancy; QS:473-551 Blanch's tau
    std::vector<double> r(n), busg(n), lam(n), tpss(n), p1(n), p2(n);
    for (size_t i = 0; i < n; i++) r[i] = rho[i];
    for (int x = 0; x < nx - 1; x++)
        for (int z = 0; z < nz - 1; z++)
            r[mi(x, z)] = 0.25 * (r[mi(x, z)] + r[mi(x, z + 1)] + r[mi(x + 1, z + 1)] + r[mi(x + 1, z)]);
    for (int x = 0; x < nx; x++) r[mi(x, nz - 1)] = r[mi(x, nz - 2)];
    for (int z = 0; z < nz; z++) r[mi(nx - 1, z)] = r[mi(nx - 2, z)];
    const double pi = 3.1415926, flow = 2.0 * 2.0 * pi, fup = 2.5 * c->f0 * 2.0 * pi;
    const double tss = 1.0 / ((fup - flow) / 2.0);
    const double nlow = std::log(tss * tss * flow * flow + 1.0), nup = std::log(tss * tss * fup * fup + 1.0);
    const double dlow = std::atan(flow * tss) - flow * tss / (1.0 + tss * tss * flow * flow);
    const double dup = std::atan(fup * tss) - fup * tss / (1.0 + tss * tss * fup * fup);
    const double kappa = (20.0 / 18.0) * (nup - nlow) / (dup - dlow);  // tau_p = kappa / Q
    std::vector<double> invq(n);
    for (size_t i = 0; i < n; i++) {
        busg[i] = 1.0 / r[i];
        lam[i] = r[i] * (double)vp[i] * (double)vp[i];
        invq[i] = 1.0 / (q ? (double)q[i] : 100000.0);
        tpss[i] = 1.0 + kappa * invq[i];
        p1[i] = lam[i] * tpss[i];
        p2[i] = lam[i] * (tpss[i] - 1.0);
    }
    const double dt = c->dt, f = dt * (-1.0 / tss), hx = 0.5 / c->dx, hz = 0.5 / c->dz;
    // QS:555-605 split cosine sponges: per x (resp. z) the factor of the v-grid and of the s-grid
    std::vector<double> axv(nx, 1.0), axs(nx, 1.0), azv(nz, 1.0), azs(nz, 1.0);
    {
        const double R = 1.0e-3, fx = std::acos(R) / (np * c->dx), fz = std::acos(R) / (np * c->dz);
        for (int i = 1; i <= np + 1; i++) {
            const double cv = std::cos(fx * (np - i + 1) * c->dx);
            const double c1 = (i == np + 1) ? 1.0 : std::cos(fx * ((np - i + 1) * c->dx - c->dx / 2));
            const double c2 = std::cos(fx * ((np - i + 1) * c->dx + c->dx / 2));
            axv[i - 1] *= cv;  axv[nx - i] *= cv;
            axs[i - 1] *= c1;  axs[nx - i] *= c2;
            const double zv = std::cos(fz * (np - i + 1) * c->dz);
            const double z1 = (i == np + 1) ? 1.0 : std::cos(fz * ((np - i + 1) * c->dz - c->dz / 2));
            const double z2 = std::cos(fz * ((np - i + 1) * c->dz + c->dz / 2));
            azv[i - 1] *= zv;  azv[nz - i] *= zv;
            azs[i - 1] *= z1;  azs[nz - i] *= z2;
        }
    }
    // QS:1398-1444: a Gaussian (sigma 1.5 cells) over an nz x nx window centred at
    // ((nz+1)/2, (nx+1)/2) (integer division), normalised by its sum over the window and placed
    // with its index hw = nint((n+1)/2) on the source cell (one cell off centre for even sizes);
    // dt / dz^2 applied (QS:1384)
    std::vector<double> stamp(n, 0.0);
    {
        const int n1 = nz, n2 = nx, ic1 = (n1 + 1) / 2, ic2 = (n2 + 1) / 2;
        const int hw1 = (int)std::lround((n1 + 1) / 2.0), hw2 = (int)std::lround((n2 + 1) / 2.0);
        auto raw = [&](int i, int j) {  // 1-based (z index i, x index j)
            const double d2 = (double)(j - ic2) * (j - ic2) + (double)(i - ic1) * (i - ic1);
            return std::exp(-d2 / (2 * 2.25)) / (2 * pi * 2.25);
        };
        double sum = 0;
        for (int j = 1; j <= n2; j++)
            for (int i = 1; i <= n1; i++) sum += raw(i, j);
        for (int x = 0; x < nx; x++)
            for (int z = 0; z < nz; z++) {
                const int i = z - c->sz + hw1, j = x - c->sx + hw2;
                if (i >= 1 && i <= n1 && j >= 1 && j <= n2 && std::abs(x - c->sx) <= hw2 - 1 &&
                    std::abs(z - c->sz) <= hw1 - 1)
                    stamp[mi(x, z)] = raw(i, j) / sum * dt / ((double)c->dz * c->dz);
            }
    }
    // forward, keeping Dx1 vx and Dz1 vz of every step
    enum { VX, VZ, SX, SZ, SR, RX, RZ, RR, NF };
    std::vector<std::vector<double>> u(NF, std::vector<double>(N, 0.0));
    std::vector<double> S(N, 0.0), D1((size_t)nt * n), D4((size_t)nt * n), rec((size_t)nrec * nt);
    for (int k = 0; k < nt; k++) {
        for (int x = 0; x < nx; x++)
            for (int z = 0; z < nz; z++) S[g.at(x, z)] = u[SX][g.at(x, z)] + u[SZ][g.at(x, z)] + u[SR][g.at(x, z)];
        for (int x = 0; x < nx; x++)
            for (int z = 0; z < nz; z++) {
                const size_t a = g.at(x, z);
                u[VX][a] = axv[x] * (u[VX][a] + dt * busg[mi(x, z)] * rsg(g, S, x, z, 0, true, hx));
                u[VZ][a] = azv[z] * (u[VZ][a] + dt * busg[mi(x, z)] * rsg(g, S, x, z, 0, false, hz));
            }
        for (int x = 0; x < nx; x++)
            for (int z = 0; z < nz; z++) {
                const size_t a = g.at(x, z), b = mi(x, z);
                const double d1 = rsg(g, u[VX], x, z, 1, true, hx), d4 = rsg(g, u[VZ], x, z, 1, false, hz);
                D1[(size_t)k * n + b] = d1;
                D4[(size_t)k * n + b] = d4;
                const double R = u[RX][a] + u[RZ][a] + u[RR][a];
                u[SX][a] = axs[x] * (u[SX][a] + dt * p1[b] * d1) + stamp[b] * wavelet[k];
                u[SZ][a] = azs[z] * (u[SZ][a] + dt * p1[b] * d4);
                u[SR][a] = u[SR][a] + dt * R;
                u[RX][a] = axs[x] * (u[RX][a] + f * p2[b] * d1);
                u[RZ][a] = azs[z] * (u[RZ][a] + f * p2[b] * d4);
                u[RR][a] = u[RR][a] + f * R;
            }
        for (int i = 0; i < nrec; i++) {
            const size_t a = g.at(c->rec_x[i], c->rec_z[i]);
            rec[(size_t)i * nt + k] = u[SX][a] + u[SZ][a] + u[SR][a];
        }
    }
    if (records) std::memcpy(records, rec.data(), sizeof(double) * rec.size());
    std::vector<double> res((size_t)nrec * nt, 0.0);
    double J = 0;
    if (obs)
        for (size_t i = 0; i < res.size(); i++) {
            res[i] = rec[i] - (double)obs[i];
            J += 0.5 * res[i] * res[i];
        }
    if (misfit) *misfit = J;
    if (!obs || (!grad_vp && !grad_invq && !dw)) return 0;
    // adjoint, last step first
    std::vector<std::vector<double>> A(NF, std::vector<double>(N, 0.0));
    std::vector<double> T1(N, 0.0), T4(N, 0.0), Qx(N, 0.0), Qz(N, 0.0);
    std::vector<double> g1(n, 0.0), g2(n, 0.0);
    for (int k = nt - 1; k >= 0; k--) {
        for (int i = 0; i < nrec; i++) {  // the record of step k reads S after the step
            const size_t a = g.at(c->rec_x[i], c->rec_z[i]);
            const double rr = res[(size_t)i * nt + k];
            A[SX][a] += rr;
            A[SZ][a] += rr;
            A[SR][a] += rr;
        }
        if (dw) {
            double s = 0;
            for (int x = 0; x < nx; x++)
                for (int z = 0; z < nz; z++) s += A[SX][g.at(x, z)] * stamp[mi(x, z)];
            dw[k] = s;
        }
        // stress and memory-variable update, transposed (cell-local)
        for (int x = 0; x < nx; x++)
            for (int z = 0; z < nz; z++) {
                const size_t a = g.at(x, z), b = mi(x, z);
                const double u1 = axs[x] * A[SX][a], u4 = azs[z] * A[SZ][a];
                const double w1 = axs[x] * A[RX][a], w4 = azs[z] * A[RZ][a];
                const double aR = f * A[RR][a] + dt * A[SR][a];
                T1[a] = dt * p1[b] * u1 + f * p2[b] * w1;
                T4[a] = dt * p1[b] * u4 + f * p2[b] * w4;
                g1[b] += D1[(size_t)k * n + b] * u1 + D4[(size_t)k * n + b] * u4;
                g2[b] += D1[(size_t)k * n + b] * w1 + D4[(size_t)k * n + b] * w4;
                A[SX][a] = u1;
                A[SZ][a] = u4;
                A[RX][a] = w1 + aR;
                A[RZ][a] = w4 + aR;
                A[RR][a] = A[RR][a] + aR;
            }
        // d1 = Dx1 vx, d4 = Dz1 vz transposed; velocity update transposed
        for (int x = 0; x < nx; x++)
            for (int z = 0; z < nz; z++) {
                const size_t a = g.at(x, z), b = mi(x, z);
                const double vxa = A[VX][a] + rsg_t(g, T1, x, z, 1, true, hx);
                const double vza = A[VZ][a] + rsg_t(g, T4, x, z, 1, false, hz);
                A[VX][a] = axv[x] * vxa;
                A[VZ][a] = azv[z] * vza;
                Qx[a] = dt * busg[b] * axv[x] * vxa;
                Qz[a] = dt * busg[b] * azv[z] * vza;
            }
        for (int x = 0; x < nx; x++)
            for (int z = 0; z < nz; z++) {
                const size_t a = g.at(x, z);
                const double aS = rsg_t(g, Qx, x, z, 0, true, hx) + rsg_t(g, Qz, x, z, 0, false, hz);
                A[SX][a] += aS;
                A[SZ][a] += aS;
                A[SR][a] += aS;
            }
    }
    for (size_t i = 0; i < n; i++) {
        const double Gp1 = dt * g1[i], Gp2 = f * g2[i];
        if (grad_vp) grad_vp[i] = 2.0 * r[i] * (double)vp[i] * (tpss[i] * Gp1 + (tpss[i] - 1.0) * Gp2);
        if (grad_invq) grad_invq[i] = lam[i] * kappa * (Gp1 + Gp2);
    }
    return 0;
}
