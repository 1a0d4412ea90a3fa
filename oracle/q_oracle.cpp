// ORACLE -- test infrastructure only. CPU restatement of the reference's visco-elastic
// rotated-staggered-grid modelling of one shot, used by tests/ as the checker of the
// viscoacoustic GPU path.  The reference is Fortran 90 + MPI + OpenMP and cannot be compiled in
// this environment (no Fortran compiler), so this restatement is not pinned by a run of the
// reference: "parity unpinned" for this scheme; it is checked by physics properties instead
// (tests/test_q_oracle.py).
//
// Follows forward/Q_forward/Q_multishot_fd_subroutine_fsbc_zy_rotated.f90 (QS) and
// Q_multishot_fd_main_fsbc_zy_rotated.f90 (QM) for a flat surface (topo = 0):
//   QS:9-28     coefficients a100..a104 (10th order)      QS:288-428 window + edge padding
//   QS:434-469  density averaging and buoyancy (in place) QS:473-551 Lame, Blanch tau
//   QS:555-605  cosine sponge profiles                    QS:609-654 split sponge
//   QS:695-839  one step: velocities, stresses, memory variables (split x / z / r parts)
//   QS:843-966  RSG diagonal derivatives                  QS:969-1337 updates and sums
//   QS:1340-1444 Gaussian-spread Ricker source           QM:279-280 nwt, decay
//   QM:418-419  optional Q override (1e5)                 QM:439-459 time loop, recording
// Fortran (k, i) with k = z (1..nz) and i = x (1..nx) maps to C index (i-1)*nz + (k-1).
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace {

template <typename T>
struct Field {  // (lo_k:hi_k, lo_i:hi_i), Fortran order
    int lk, hk, li, hi, nk;
    std::vector<T> d;
    Field() {}
    Field(int lk_, int hk_, int li_, int hi_) : lk(lk_), hk(hk_), li(li_), hi(hi_), nk(hk_ - lk_ + 1) {
        d.assign((size_t)nk * (hi_ - li_ + 1), T(0));
    }
    T& operator()(int k, int i) { return d[(size_t)(i - li) * nk + (k - lk)]; }
    T operator()(int k, int i) const { return d[(size_t)(i - li) * nk + (k - lk)]; }
};

template <typename T>
struct QSolver {
    int nx, nz, npxn, npxp, npzn, npzp;
    T dx, dz, dt, f0;
    T a[5];
    // halo fields (-4:nz+5, -4:nx+5)
    Field<T> vx, vz, sxx, szz, sxz;
    // memory variables (nz, nx)
    Field<T> rxx, rzz, rxz;
    // split parts (0:nz, nx)
    Field<T> vxx, vxz, vzx, vzz, sxxx, sxxz, sxxr, szzx, szzz, szzr, sxzx, sxzz, sxzr;
    Field<T> rxxx, rxxz, rxxr, rzzx, rzzz, rzzr, rxzx, rxzz, rxzr;
    Field<T> d1, d2, d3, d4;
    // parameters (nz, nx)
    Field<T> busg, lambmu, mu, taup, taus, rtau;
    std::vector<T> spgxn, spgxp, spgzn, spgzp, spg1xn, spg2xp, spg1zn, spg2zp;

    void alloc() {
        auto H = [&] { return Field<T>(-4, nz + 5, -4, nx + 5); };
        auto N = [&] { return Field<T>(1, nz, 1, nx); };
        auto S = [&] { return Field<T>(0, nz, 1, nx); };
        vx = H(); vz = H(); sxx = H(); szz = H(); sxz = H();
        rxx = N(); rzz = N(); rxz = N();
        for (auto* f : {&vxx, &vxz, &vzx, &vzz, &sxxx, &sxxz, &sxxr, &szzx, &szzz, &szzr, &sxzx, &sxzz, &sxzr,
                        &rxxx, &rxxz, &rxxr, &rzzx, &rzzz, &rzzr, &rxzx, &rxzz, &rxzr})
            *f = S();
        d1 = N(); d2 = N(); d3 = N(); d4 = N();
        busg = N(); lambmu = N(); mu = N(); taup = N(); taus = N(); rtau = N();
    }

    // QS:843-903 (xflag 0 / 1)
    void derx(int flag, const Field<T>& u, Field<T>& der) {
        const T h = T(0.5) / dx;
#pragma omp parallel for schedule(static)
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= nz; k++) {
                T s = 0;
                for (int m = 0; m < 5; m++) {
                    T t;
                    if (flag == 0)
                        t = u(k + m, i + m) - u(k - 1 - m, i - 1 - m) + u(k - 1 - m, i + m) - u(k + m, i - 1 - m);
                    else
                        t = u(k + 1 + m, i + 1 + m) - u(k - m, i - m) + u(k - m, i + 1 + m) - u(k + 1 + m, i - m);
                    s = (m == 0) ? a[0] * t : s + a[m] * t;
                }
                der(k, i) = h * s;
            }
    }
    // QS:906-966
    void derz(int flag, const Field<T>& u, Field<T>& der) {
        const T h = T(0.5) / dz;
#pragma omp parallel for schedule(static)
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= nz; k++) {
                T s = 0;
                for (int m = 0; m < 5; m++) {
                    T t;
                    if (flag == 0)
                        t = u(k + m, i + m) - u(k - 1 - m, i - 1 - m) - u(k - 1 - m, i + m) + u(k + m, i - 1 - m);
                    else
                        t = u(k + 1 + m, i + 1 + m) - u(k - m, i - m) - u(k - m, i + 1 + m) + u(k + 1 + m, i - m);
                    s = (m == 0) ? a[0] * t : s + a[m] * t;
                }
                der(k, i) = h * s;
            }
    }
    // QS:609-654, flat surface: itopo(i) - npzn = 1
    void sponge(Field<T>& ux, Field<T>& uz, const std::vector<T>& sxn, const std::vector<T>& sxp,
                const std::vector<T>& szn, const std::vector<T>& szp) {
        for (int i = 1; i <= npxn + 1; i++)
            for (int k = 1; k <= nz; k++) ux(k, i) = ux(k, i) * sxn[i - 1];
        for (int i = 1; i <= npxp + 1; i++)
            for (int k = 1; k <= nz; k++) ux(k, nx - i + 1) = ux(k, nx - i + 1) * sxp[i - 1];
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= npzn + 1; k++) uz(k, i) = uz(k, i) * szn[k - 1];
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= npzp + 1; k++) uz(nz - k + 1, i) = uz(nz - k + 1, i) * szp[k - 1];
    }
    void sum2(Field<T>& v, const Field<T>& a_, const Field<T>& b_) {
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= nz; k++) v(k, i) = a_(k, i) + b_(k, i);
    }
    void sum3(Field<T>& v, const Field<T>& a_, const Field<T>& b_, const Field<T>& c_) {
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= nz; k++) v(k, i) = a_(k, i) + b_(k, i) + c_(k, i);
    }

    // QS:695-839 (the source is added by the caller through `src`)
    template <typename Src>
    void step(Src&& src) {
        // velocities
        derx(0, sxx, d1);
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= nz; k++) vxx(k, i) = vxx(k, i) + dt * busg(k, i) * d1(k, i);
        derz(0, sxz, d2);
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= nz; k++) vxz(k, i) = vxz(k, i) + dt * busg(k, i) * d2(k, i);
        sponge(vxx, vxz, spgxn, spgxp, spgzn, spgzp);
        sum2(vx, vxx, vxz);
        derx(0, sxz, d1);
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= nz; k++) vzx(k, i) = vzx(k, i) + dt * busg(k, i) * d1(k, i);
        derz(0, szz, d2);
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= nz; k++) vzz(k, i) = vzz(k, i) + dt * busg(k, i) * d2(k, i);
        sponge(vzx, vzz, spgxn, spgxp, spgzn, spgzp);
        sum2(vz, vzx, vzz);
        // stresses
        derx(1, vx, d1);
        derx(1, vz, d2);
        derz(1, vx, d3);
        derz(1, vz, d4);
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= nz; k++) {  // calpstrxx
                sxxx(k, i) = sxxx(k, i) + dt * (lambmu(k, i) * taup(k, i) * d1(k, i));
                sxxz(k, i) = sxxz(k, i) + dt * ((lambmu(k, i) * taup(k, i) - T(2.0) * mu(k, i) * taus(k, i)) * d4(k, i));
                sxxr(k, i) = sxxr(k, i) + dt * rxx(k, i);
            }
        sponge(sxxx, sxxz, spg1xn, spg2xp, spg1zn, spg2zp);
        src(sxxx);
        sum3(sxx, sxxx, sxxz, sxxr);
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= nz; k++) {  // calpstrzz
                szzx(k, i) = szzx(k, i) + dt * ((lambmu(k, i) * taup(k, i) - T(2.0) * mu(k, i) * taus(k, i)) * d1(k, i));
                szzz(k, i) = szzz(k, i) + dt * (lambmu(k, i) * taup(k, i) * d4(k, i));
                szzr(k, i) = szzr(k, i) + dt * rzz(k, i);
            }
        sponge(szzx, szzz, spg1xn, spg2xp, spg1zn, spg2zp);
        src(szzx);
        sum3(szz, szzx, szzz, szzr);
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= nz; k++) {  // calpstrxz
                sxzx(k, i) = sxzx(k, i) + dt * (mu(k, i) * taus(k, i) * d2(k, i));
                sxzz(k, i) = sxzz(k, i) + dt * (mu(k, i) * taus(k, i) * d3(k, i));
                sxzr(k, i) = sxzr(k, i) + dt * rxz(k, i);
            }
        sponge(sxzx, sxzz, spg1xn, spg2xp, spg1zn, spg2zp);
        sum3(sxz, sxzx, sxzz, sxzr);
        // memory variables
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= nz; k++) {  // calprxx
                const T f = dt * (T(-1.0) * rtau(k, i));
                rxxx(k, i) = rxxx(k, i) + f * (lambmu(k, i) * (taup(k, i) - 1) * d1(k, i));
                rxxz(k, i) = rxxz(k, i) +
                             f * ((lambmu(k, i) * (taup(k, i) - 1) - T(2.0) * mu(k, i) * (taus(k, i) - 1)) * d4(k, i));
                rxxr(k, i) = rxxr(k, i) + f * rxx(k, i);
            }
        sponge(rxxx, rxxz, spg1xn, spg2xp, spg1zn, spg2zp);
        sum3(rxx, rxxx, rxxz, rxxr);
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= nz; k++) {  // calprzz
                const T f = dt * (T(-1.0) * rtau(k, i));
                rzzz(k, i) = rzzz(k, i) + f * (lambmu(k, i) * (taup(k, i) - 1) * d4(k, i));
                rzzx(k, i) = rzzx(k, i) +
                             f * ((lambmu(k, i) * (taup(k, i) - 1) - T(2.0) * mu(k, i) * (taus(k, i) - 1)) * d1(k, i));
                rzzr(k, i) = rzzr(k, i) + f * rzz(k, i);
            }
        sponge(rzzx, rzzz, spg1xn, spg2xp, spg1zn, spg2zp);
        sum3(rzz, rzzx, rzzz, rzzr);
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= nz; k++) {  // calprxz
                const T f = dt * (T(-1.0) * rtau(k, i));
                rxzx(k, i) = rxzx(k, i) + f * (mu(k, i) * (taus(k, i) - 1) * d2(k, i));
                rxzz(k, i) = rxzz(k, i) + f * (mu(k, i) * (taus(k, i) - 1) * d3(k, i));
                rxzr(k, i) = rxzr(k, i) + f * rxz(k, i);
            }
        sponge(rxzx, rxzz, spg1xn, spg2xp, spg1zn, spg2zp);
        sum3(rxz, rxzx, rxzz, rxzr);
    }
};

template <typename T>
int run_q(const OracleQCfg* c, const float* vp_in, const float* vs_in, const float* rho_in, const float* qp_in,
          const float* qs_in, T* rec1, T* rec2, T* snap_p) {
    const int nx_m = c->nx, nz_m = c->nz;  // interior model (nz, nx)
    const int nxe = c->ixmaxe - c->ixmine + 1, nze = nz_m;
    QSolver<T> S;
    S.npxn = c->npxn; S.npxp = c->npxp; S.npzn = c->npzn; S.npzp = c->npzp;
    S.nx = nxe + c->npxn + c->npxp;
    S.nz = nze + c->npzn + c->npzp;
    S.dx = c->dx; S.dz = c->dz; S.dt = c->dt; S.f0 = c->f0;
    // QS:9-28, single precision constants
    const float af[5] = {19845.0f / 16384.0f, -735.0f / 8192.0f, 567.0f / 40960.0f, -405.0f / 229376.0f,
                         35.0f / 294912.0f};
    for (int m = 0; m < 5; m++) S.a[m] = (T)af[m];
    if (S.nx < 12 || S.nz < 12) return 1;
    S.alloc();
    const int NX = S.nx, NZ = S.nz;
    // QS:288-372 window and edge padding (vpe..qfse), flat topography
    Field<T> vpe(1, NZ, 1, NX), vse(1, NZ, 1, NX), rhoe(1, NZ, 1, NX), qpe(1, NZ, 1, NX), qse(1, NZ, 1, NX);
    auto in = [&](const float* m, int k, int i) { return (T)m[(size_t)(i - 1) * nz_m + (k - 1)]; };
    for (int i = 1; i <= nxe; i++) {
        int io = i + c->ixmine;
        if (io < 1) io = 1;
        if (io > nx_m) io = nx_m;
        for (int k = 1; k <= nze; k++) {
            vpe(k + c->npzn, i + c->npxn) = in(vp_in, k, io);
            vse(k + c->npzn, i + c->npxn) = in(vs_in, k, io);
            rhoe(k + c->npzn, i + c->npxn) = in(rho_in, k, io);
            qpe(k + c->npzn, i + c->npxn) = in(qp_in, k, io);
            qse(k + c->npzn, i + c->npxn) = in(qs_in, k, io);
        }
    }
    for (auto* f : {&vpe, &vse, &rhoe, &qpe, &qse}) {
        for (int k = 1; k <= c->npzn; k++)
            for (int i = 1; i <= NX; i++) (*f)(k, i) = (*f)(c->npzn + 1, i);
        for (int k = c->npzn + nze + 1; k <= NZ; k++)
            for (int i = 1; i <= NX; i++) (*f)(k, i) = (*f)(c->npzn + nz_m, i);
        for (int k = 1; k <= NZ; k++)
            for (int i = 1; i <= c->npxn; i++) (*f)(k, i) = (*f)(k, c->npxn + 1);
        for (int k = 1; k <= NZ; k++)
            for (int i = c->npxn + nxe + 1; i <= NX; i++) (*f)(k, i) = (*f)(k, c->npxn + nxe);
    }
    if (c->q_override) {  // QM:418-419
        for (auto& v : qpe.d) v = (T)100000.0f;
        for (auto& v : qse.d) v = (T)100000.0f;
    }
    // QS:434-469 staggered density (in place) and buoyancy
    for (int i = 1; i <= NX - 1; i++)
        for (int k = 1; k <= NZ - 1; k++)
            rhoe(k, i) = T(0.25) * (rhoe(k, i) + rhoe(k + 1, i) + rhoe(k + 1, i + 1) + rhoe(k, i + 1));
    for (int i = 1; i <= NX; i++) rhoe(NZ, i) = rhoe(NZ - 1, i);
    for (int k = 1; k <= NZ; k++) rhoe(k, NX) = rhoe(k, NX - 1);
    for (int i = 1; i <= NX; i++)
        for (int k = 1; k <= NZ; k++) {
            if (rhoe(k, i) == T(0)) return 2;  // QS:463 stops here
            S.busg(k, i) = T(1.0) / rhoe(k, i);
        }
    // QS:473-551 (Blanch's tau method), with the averaged density
    const T pi = (T)3.1415926f;
    for (int i = 1; i <= NX; i++)
        for (int k = 1; k <= NZ; k++) {
            const T r = rhoe(k, i);
            S.mu(k, i) = r * (vse(k, i) * vse(k, i));       // rhoe*vse**2
            S.lambmu(k, i) = r * (vpe(k, i) * vpe(k, i));   // rhoe*vpe**2
            const T flow = T(2) * T(2) * pi;
            const T fup = T(2.5) * S.f0 * T(2) * pi;
            const T qp = qpe(k, i) * (T(18.0) / T(20.0));
            const T qs = qse(k, i) * (T(18.0) / T(20.0));
            const T tss = T(1.0) / ((fup - flow) / T(2.0));
            const T nlow = std::log((tss * tss) * (flow * flow) + T(1));  // tss**2*flow**2+1
            const T nup = std::log((tss * tss) * (fup * fup) + T(1));
            const T dlow = std::atan(flow * tss) - (flow * tss) / (T(1) + (tss * tss) * (flow * flow));
            const T dup = std::atan(fup * tss) - (fup * tss) / (T(1) + (tss * tss) * (fup * fup));
            T tp = 0, ts = 0;
            if (dup - dlow != T(0)) {
                tp = T(1.0) / qp * (nup - nlow) / (dup - dlow);
                ts = T(1.0) / qs * (nup - nlow) / (dup - dlow);
            }
            const T tpe = tp * tss + tss, tse = ts * tss + tss;
            S.rtau(k, i) = T(1.0) / tss;
            S.taup(k, i) = tpe / tss;
            S.taus(k, i) = tse / tss;
        }
    // QS:555-605 cosine sponge, R = 1e-3
    {
        const T Rr = (T)1.0e-3f;
        const T fxn = std::acos(Rr) / (T(c->npxn) * S.dx), fxp = std::acos(Rr) / (T(c->npxp) * S.dx);
        const T fzn = std::acos(Rr) / (T(c->npzn) * S.dz), fzp = std::acos(Rr) / (T(c->npzp) * S.dz);
        S.spgxn.resize(c->npxn + 1); S.spg1xn.resize(c->npxn + 1);
        S.spgzn.resize(c->npzn + 1); S.spg1zn.resize(c->npzn + 1);
        S.spgxp.resize(c->npxp + 1); S.spg2xp.resize(c->npxp + 1);
        S.spgzp.resize(c->npzp + 1); S.spg2zp.resize(c->npzp + 1);
        for (int i = 1; i <= c->npxn + 1; i++) {
            S.spgxn[i - 1] = std::cos(fxn * T(c->npxn - i + 1) * S.dx);
            S.spg1xn[i - 1] = (i == c->npxn + 1) ? T(1) : std::cos(fxn * (T(c->npxn - i + 1) * S.dx - S.dx / 2));
        }
        for (int i = 1; i <= c->npzn + 1; i++) {
            S.spgzn[i - 1] = std::cos(fzn * T(c->npzn - i + 1) * S.dz);
            S.spg1zn[i - 1] = (i == c->npzn + 1) ? T(1) : std::cos(fzn * (T(c->npzn - i + 1) * S.dz - S.dz / 2));
        }
        for (int i = 1; i <= c->npxp + 1; i++) {
            S.spgxp[i - 1] = std::cos(fxp * T(c->npxp - i + 1) * S.dx);
            S.spg2xp[i - 1] = std::cos(fxp * (T(c->npxp - i + 1) * S.dx + S.dx / 2));
        }
        for (int i = 1; i <= c->npzp + 1; i++) {
            S.spgzp[i - 1] = std::cos(fzp * T(c->npzp - i + 1) * S.dz);
            S.spg2zp[i - 1] = std::cos(fzp * (T(c->npzp - i + 1) * S.dz + S.dz / 2));
        }
    }
    // QS:1340-1444 Gaussian stamp over the whole grid (n1 = NZ, n2 = NX), normalised by its sum
    const int n1 = NZ, n2 = NX;
    const int hw1 = (int)std::lround((n1 + 1) / 2.0), hw2 = (int)std::lround((n2 + 1) / 2.0);
    const int ixcen = (n1 + 1) / 2, izcen = (n2 + 1) / 2;
    const T sigma2 = T(1.5) * T(1.5);
    Field<T> g2c(1, n1, 1, n2);
    T sum_tmp = 0;
    for (int j = 1; j <= n2; j++)
        for (int i = 1; i <= n1; i++) {
            const T dis = (T)((j - izcen) * (j - izcen) + (i - ixcen) * (i - ixcen));
            g2c(i, j) = T(1) / (T(2) * pi * sigma2) * std::exp(-dis / (T(2) * sigma2));
        }
    for (int j = 1; j <= n2; j++)
        for (int i = 1; i <= n1; i++) sum_tmp = sum_tmp + g2c(i, j);
    for (auto& v : g2c.d) v = v / sum_tmp;
    const int isxe = c->isxe, isze = c->isze;
    // cells the whole-grid loop of QS:1378-1390 touches with a non-zero weight (adding an exact
    // zero elsewhere leaves u unchanged), in the loop's order
    struct Tap { int m, n; T g; };
    std::vector<Tap> taps;
    {
        int idx2 = 1;
        for (int n = isxe - (hw2 - 1); n <= isxe + (hw2 - 1); n++) {
            int idx1 = 1;
            for (int m = isze - (hw1 - 1); m <= isze + (hw1 - 1); m++) {
                if (n >= 1 && n <= NX && m >= 1 && m <= NZ && idx2 <= n2 && idx1 <= n1 && g2c(idx1, idx2) != T(0))
                    taps.push_back({m, n, g2c(idx1, idx2)});
                idx1++;
            }
            idx2++;
        }
    }
    int it_cur = 0;
    auto addsrc = [&](Field<T>& u) {
        const T b = pi * S.f0 * (T(it_cur) * S.dt - T(1.2f) / S.f0);  // 1.2 is a REAL literal
        const T wav = std::exp(-(b * b)) * (T(1) - T(2) * (b * b));
        for (const Tap& t : taps) u(t.m, t.n) = wav * t.g * S.dt / (S.dz * S.dz) + u(t.m, t.n);
    };
    // QM:439-459
    const int nwt = 2 * (int)std::lround(1.2f / (c->f0 * c->dt));  // single precision, QM:279
    const int decay = (int)std::lround(nwt / 2.0);
    const int nt = c->nt;
    for (int it = 1; it <= nt + decay; it++) {
        it_cur = it;
        S.step(addsrc);
        const int iit = it - decay;
        if (iit >= 1) {
            const int kr = c->npzn + 1 + c->nrz0;
            for (int i = 1; i <= nxe; i++) {
                if (rec1) rec1[(size_t)(i - 1) * nt + (iit - 1)] = S.szz(kr, i + c->npxn);
                if (rec2) rec2[(size_t)(i - 1) * nt + (iit - 1)] = S.sxx(kr, i + c->npxn);
            }
        }
    }
    if (snap_p)
        for (int i = 1; i <= NX; i++)
            for (int k = 1; k <= NZ; k++) snap_p[(size_t)(i - 1) * NZ + (k - 1)] = S.sxx(k, i);
    return 0;
}

}  // namespace

extern "C" {

int oracle_q_f32(const OracleQCfg* c, const float* vp, const float* vs, const float* rho, const float* qp,
                 const float* qs, float* rec1, float* rec2, float* final_sxx) {
    return run_q<float>(c, vp, vs, rho, qp, qs, rec1, rec2, final_sxx);
}

int oracle_q_f64(const OracleQCfg* c, const float* vp, const float* vs, const float* rho, const float* qp,
                 const float* qs, double* rec1, double* rec2, double* final_sxx) {
    return run_q<double>(c, vp, vs, rho, qp, qs, rec1, rec2, final_sxx);
}

}  // extern "C"
