// ORACLE -- test infrastructure only. CPU restatement of the reference's isotropic elastic
// standard-staggered-grid modelling of one shot (forward/yang_version_2016_2_2, both modes:
// 'abc', cosine sponge on all four sides, and 'fsbc', free surface on top), flat or with
// topography, used by tests/ as the checker of the SFD_ELASTIC_2D GPU path.  The reference is Fortran 90 + MPI + OpenMP and cannot be compiled in
// this environment (no Fortran compiler), so this restatement is not pinned by a run of the
// reference: "parity unpinned" for this scheme; it is checked by physics properties instead
// (tests/test_iso_oracle.py).
//
// Files of forward/yang_version_2016_2_2: YMOD = Iso_multishot_fd_module_zy_m2.f90,
// YPRI = Iso_multishot_fd_subroutine_fsbc_zy_m2_pri.f90, YPUB = Iso_multishot_fd_subroutine_fsbc_zy_m2_pub.f90
//   YMOD:23-27     coefficients a100..a104 (10th order)
//   YPUB:188-313   window, edge padding, itopoe = nint(topo/dz) + npzn, source cell, gc2d (sigma 2)
//   YPUB:323-547   substagger: Lame moduli, staggered buoyancies and moduli, rows above itopoe
//                  refilled from row itopoe
//   YPUB:549-634   modipapml / gauss_filter_2d: rows k <= itopoe(i) replaced IN PLACE by the
//                  gc2d-weighted sum of their window.  The reference runs this loop under an
//                  OpenMP DO while it overwrites u, so with several threads its result depends on
//                  the schedule; the restatement takes the serial (one-thread) order.
//   YPUB:796-849   csponge                        YPUB:851-897 calpmlbclrtb (split sponge)
//   YPUB:1095-1157 caluxabs    YPUB:1347-1407 caluzabs    YPUB:1410-1426 calu (sums)
//   YPUB:1429-1466 addsrc      YPUB:1470-1501 get_gauss_filter_coe
//   YPRI:234-386   isoewm2dabc (time loop)     YPUB:2-16 get_record (record1 = vx, record2 = vz)
//   YPRI:57-230    isoewm2dfsbc (time loop, free surface): YPUB:1026-1092 calux and
//                  YPUB:1160-1343 caluz (rows from itopo; z derivatives of order 8, 6, 4, 2 on the
//                  five rows nearest the surface, YMOD:7-20), YPUB:901-934 calpmlbclrb (no top
//                  sponge), YPUB:938-976 calfsbcv, YPUB:978-1007 calfsbcstrzz,
//                  YPUB:1009-1024 calfsbcstrxz; no smoothing
//   The free-surface velocity vz(itopo - 1) = vz(itopo) + lambda/(lambda + 2 mu) dx vx is written
//   into the split parts after calu has summed them (YPRI:141-150), so the stress update reads
//   it one step later.
// Topography: itopo(i) = nint(topo/dz) + npzn per window column (YPUB:270-272); every loop
// bound, sponge row, surface row, the source condition and the receiver row follow it.
// The split fields also hold a row k = 0 (YPUB:1095 `ux(0:nz,nx)`, abc loops from itopo - npzn,
// which is 0 for a flat surface); calu and get_record never read it, so it is not kept here.  Fortran (k, i), k = z, i = x,
// maps to C index (i-1)*nz + (k-1).
#include <algorithm>
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
struct IsoSolver {
    int nx, nz, npxn, npxp, npzn, npzp;
    T dx, dz, dt;
    T a[5];
    bool fs = false;   // free surface (fsbc mode)
    std::vector<int> itopo;  // itopo(i), i = 1..nx: surface row (1-based) per column
    T cr[6][5] = {};   // cr[M]: coefficients of the M-term staggered derivative (YMOD:7-27)
    Field<T> vx, vz, sxx, szz, sxz;                                     // (-4:nz+5, -4:nx+5)
    Field<T> vxx, vxz, vzx, vzz, sxxx, sxxz, szzx, szzz, sxzx, sxzz;    // (1:nz, 1:nx)
    Field<T> busg1e, busg2e, lambsg, lambmusg, musge;                   // (1:nz, 1:nx)
    std::vector<T> spgxn, spgxp, spgzn, spgzp, spg1xn, spg2xp, spg1zn, spg2zp;

    void alloc() {
        auto H = [&] { return Field<T>(-4, nz + 5, -4, nx + 5); };
        auto N = [&] { return Field<T>(1, nz, 1, nx); };
        vx = H(); vz = H(); sxx = H(); szz = H(); sxz = H();
        for (auto* f : {&vxx, &vxz, &vzx, &vzz, &sxxx, &sxxz, &szzx, &szzz, &sxzx, &sxzz}) *f = N();
    }

    // YPUB:1095-1157 (x) and YPUB:1347-1407 (z); flag 0: u(i) - u(i-1) ..., flag 1: u(i+1) - u(i) ...;
    // M terms (5 = 10th order; fewer near the free surface, YPUB:1183-1251, 1275-1335)
    T der(const Field<T>& u, int k, int i, bool xdir, int flag, int M = 5) const {
        auto U = [&](int o) { return xdir ? u(k, i + o) : u(k + o, i); };
        T s = 0;
        for (int m = 0; m < M; m++) {
            const T t = flag == 0 ? U(m) - U(-1 - m) : U(1 + m) - U(-m);
            s = (m == 0) ? cr[M][0] * t : s + cr[M][m] * t;
        }
        return s;
    }
    // terms of caluz's derivative at row k of column i (YPUB:1160-1343): d rows below the surface
    int zterms(int k, int i, int flag) const {
        if (!fs) return 5;
        const int d = k - itopo[i];
        return flag == 0 ? (d >= 5 ? 5 : (d < 1 ? 1 : d)) : (d >= 4 ? 5 : d + 1);
    }
    // first updated row of column i: itopo (calux / caluz) or itopo - npzn (caluxabs /
    // caluzabs; row 0 is not kept)
    int krow(int i) const { return fs ? itopo[i] : std::max(itopo[i] - npzn, 1); }
    // ux(k,i) = ux(k,i) + (dt/dh)*pa(k,i)*(...)
    void update(Field<T>& ux, const Field<T>& u, const Field<T>& pa, bool xdir, int flag) {
        const T c = xdir ? dt / dx : dt / dz;
#pragma omp parallel for schedule(static)
        for (int i = 1; i <= nx; i++)
            for (int k = krow(i); k <= nz; k++)
                ux(k, i) = ux(k, i) + c * pa(k, i) * der(u, k, i, xdir, flag, xdir ? 5 : zterms(k, i, flag));
    }
    // YPUB:851-897: left and right from the first updated row; the top loop runs
    // k = itopo - npzn .. itopo with factor spgzn(k - (itopo - npzn) + 1) (rows >= 1 kept here).
    // fsbc: YPUB:901-934 calpmlbclrb, left and right from row itopo, no top sponge
    void sponge(Field<T>& ux, Field<T>& uz, const std::vector<T>& sxn, const std::vector<T>& sxp,
                const std::vector<T>& szn, const std::vector<T>& szp) {
        for (int i = 1; i <= npxn + 1; i++)
            for (int k = krow(i); k <= nz; k++) ux(k, i) = ux(k, i) * sxn[i - 1];
        for (int i = 1; i <= npxp + 1; i++)
            for (int k = krow(nx - i + 1); k <= nz; k++) ux(k, nx - i + 1) = ux(k, nx - i + 1) * sxp[i - 1];
        for (int i = 1; i <= nx && !fs; i++)
            for (int k = std::max(itopo[i] - npzn, 1); k <= itopo[i]; k++)
                uz(k, i) = uz(k, i) * szn[k - (itopo[i] - npzn)];
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= npzp + 1; k++) uz(nz - k + 1, i) = uz(nz - k + 1, i) * szp[k - 1];
    }
    void sum2(Field<T>& v, const Field<T>& a_, const Field<T>& b_) {  // YPUB:1410-1426
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= nz; k++) v(k, i) = a_(k, i) + b_(k, i);
    }

    // YPUB:938-976 calfsbcv on one pair of split parts: vz(izh-1) from vz(izh) and dx vx(izh),
    // izh = itopo(ix) for both columns ix and ix + 1 (row 0 of the split parts is never read)
    void fsbcv(const Field<T>& vxp, Field<T>& vzp) {
        for (int i = 1; i <= nx - 1; i++) {
            const int h = itopo[i];
            if (h - 1 < 1) continue;
            vzp(h - 1, i) = vzp(h, i) + (lambsg(h, i) / lambmusg(h, i)) * (vxp(h, i + 1) - vxp(h, i));
        }
    }
    // YPUB:978-1007 calfsbcstrzz: rows 0..itopo zero
    void fsbczz(Field<T>& t) {
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= itopo[i]; k++) t(k, i) = T(0.0);
    }
    // YPUB:1009-1024 calfsbcstrxz: image row above the surface
    void fsbcxz(Field<T>& t) {
        for (int i = 1; i <= nx; i++)
            if (itopo[i] - 1 >= 1) t(itopo[i] - 1, i) = -t(itopo[i], i);
    }

    // YPRI:305-359 (isoewm2dabc) or YPRI:121-196 (isoewm2dfsbc), one step; `src` adds the source
    // to a split stress
    template <typename Src>
    void step(Src&& src, bool src_xx) {
        update(vxx, sxx, busg2e, true, 0);     // xflag 0, strxx
        update(vxz, sxz, busg2e, false, 0);    // zflag 0, strxz
        sponge(vxx, vxz, spgxn, spgxp, spgzn, spgzp);
        sum2(vx, vxx, vxz);
        update(vzx, sxz, busg1e, true, 1);     // xflag 1, strxz
        update(vzz, szz, busg1e, false, 1);    // zflag 1, strzz
        sponge(vzx, vzz, spg1xn, spg2xp, spg1zn, spg2zp);
        sum2(vz, vzx, vzz);
        if (fs) {
            fsbcv(vxx, vzx);
            fsbcv(vxz, vzz);
        }
        update(sxxx, vx, lambmusg, true, 1);
        update(sxxz, vz, lambsg, false, 0);
        sponge(sxxx, sxxz, spg1xn, spg2xp, spgzn, spgzp);
        if (src_xx) src(sxxx);
        sum2(sxx, sxxx, sxxz);
        update(szzx, vx, lambsg, true, 1);
        update(szzz, vz, lambmusg, false, 0);
        sponge(szzx, szzz, spg1xn, spg2xp, spgzn, spgzp);
        if (fs) {
            fsbczz(szzz);
            fsbczz(szzx);
        }
        src(szzx);
        sum2(szz, szzx, szzz);
        update(sxzx, vz, musge, true, 0);
        update(sxzz, vx, musge, false, 1);
        sponge(sxzx, sxzz, spgxn, spgxp, spg1zn, spg2zp);
        if (fs) {
            fsbcxz(sxzx);
            fsbcxz(sxzz);
        }
        sum2(sxz, sxzx, sxzz);
    }
};

// YPUB:592-634, serial order: rows k = 1..itopo(i) of every column, each replaced by the
// weighted sum of its (2 rgau - 1)^2 window as it stands at that moment
template <typename T>
void gauss_filter(Field<T>& u, int nx, int nz, int rgau, const std::vector<int>& itopo, const Field<T>& gc) {
    const int w = 2 * rgau - 1;
    for (int i = 1; i <= nx; i++)
        for (int k = 1; k <= itopo[i]; k++) {
            T s = 0;
            int idx2 = 1;
            for (int n = i - (rgau - 1); n <= i + (rgau - 1); n++) {
                int idx1 = 1;
                for (int m = k - (rgau - 1); m <= k + (rgau - 1); m++) {
                    if (n >= 1 && n <= nx && m >= 1 && m <= nz && idx2 <= w && idx1 <= w) s = s + u(m, n) * gc(idx1, idx2);
                    idx1++;
                }
                idx2++;
            }
            u(k, i) = s;
        }
}

// Model preparation of one shot window (YPUB:188-634) into S; the Gaussian table into gc.
template <typename T>
int prepare(const OracleIsoCfg* c, const float* vp_in, const float* vs_in, const float* rho_in, IsoSolver<T>& S,
            Field<T>& gc) {
    const int nx_m = c->nx, nz_m = c->nz;
    const int nxe = c->ixmaxe - c->ixmine + 1, nze = nz_m;
    if (c->rgau < 1 || c->npxn < 1 || c->npxp < 1 || c->npzn < 1 || c->npzp < 1) return 1;
    S.npxn = c->npxn; S.npxp = c->npxp; S.npzn = c->npzn; S.npzp = c->npzp;
    S.nx = nxe + c->npxn + c->npxp;
    S.nz = nze + c->npzn + c->npzp;
    S.dx = c->dx; S.dz = c->dz; S.dt = c->dt;
    // YMOD:23-27, single precision constants
    const float af[5] = {19845.0f / 16384.0f, -735.0f / 8192.0f, 567.0f / 40960.0f, -405.0f / 229376.0f,
                         35.0f / 294912.0f};
    for (int m = 0; m < 5; m++) S.a[m] = S.cr[5][m] = (T)af[m];
    // YMOD:7-20 lower orders
    const float a8[4] = {1225.0f / 1024.0f, -245.0f / 3072.0f, 49.0f / 5120.0f, -5.0f / 7168.0f};
    const float a6[3] = {75.0f / 64.0f, -25.0f / 384.0f, 3.0f / 640.0f};
    const float a4[2] = {9.0f / 8.0f, -1.0f / 24.0f};
    for (int m = 0; m < 4; m++) S.cr[4][m] = (T)a8[m];
    for (int m = 0; m < 3; m++) S.cr[3][m] = (T)a6[m];
    for (int m = 0; m < 2; m++) S.cr[2][m] = (T)a4[m];
    S.cr[1][0] = (T)1.0f;
    S.fs = c->fsbc != 0;
    if (S.nx < 12 || S.nz < 12) return 1;
    S.alloc();
    const int NX = S.nx, NZ = S.nz;

    // YPUB:210-266 window and edge padding
    Field<T> vpe(1, NZ, 1, NX), vse(1, NZ, 1, NX), rhoe(1, NZ, 1, NX);
    auto in = [&](const float* m, int k, int i) { return (T)m[(size_t)(i - 1) * nz_m + (k - 1)]; };
    for (int i = 1; i <= nxe; i++) {
        int io = i + c->ixmine;
        if (io < 1) io = 1;
        if (io > nx_m) io = nx_m;
        for (int k = 1; k <= nze; k++) {
            vpe(k + c->npzn, i + c->npxn) = in(vp_in, k, io);
            vse(k + c->npzn, i + c->npxn) = in(vs_in, k, io);
            rhoe(k + c->npzn, i + c->npxn) = in(rho_in, k, io);
        }
    }
    for (auto* f : {&vpe, &vse, &rhoe}) {
        for (int k = 1; k <= c->npzn; k++)
            for (int i = 1; i <= NX; i++) (*f)(k, i) = (*f)(c->npzn + 1, i);
        for (int k = c->npzn + nze + 1; k <= NZ; k++)
            for (int i = 1; i <= NX; i++) (*f)(k, i) = (*f)(c->npzn + nz_m, i);
        for (int k = 1; k <= NZ; k++)
            for (int i = 1; i <= c->npxn; i++) (*f)(k, i) = (*f)(k, c->npxn + 1);
        for (int k = 1; k <= NZ; k++)
            for (int i = c->npxn + nxe + 1; i <= NX; i++) (*f)(k, i) = (*f)(k, c->npxn + nxe);
    }
    // YPUB:216-272 surface: topoe of the window (edge columns repeated), itopoe = nint(topoe/dz) + npzn
    {
        std::vector<float> topoe(NX + 1, 0.0f);
        for (int i = 1; i <= nxe; i++) {
            int io = i + c->ixmine;
            if (io < 1) io = 1;
            if (io > nx_m) io = nx_m;
            topoe[i + c->npxn] = c->topo ? c->topo[io - 1] : 0.0f;
        }
        for (int i = 1; i <= c->npxn; i++) topoe[i] = topoe[c->npxn + 1];
        for (int i = c->npxn + nxe + 1; i <= NX; i++) topoe[i] = topoe[c->npxn + nxe];
        S.itopo.assign(NX + 1, 0);
        for (int i = 1; i <= NX; i++) {
            S.itopo[i] = (int)std::lround(topoe[i] / (float)c->dz) + c->npzn;
            if (S.itopo[i] < (S.fs ? 1 : c->npzn) || S.itopo[i] > NZ - c->npzp - 6) return 3;
        }
    }
    // YPUB:1470-1501 Gaussian coefficients, sigma = 2.0 cells, (2 rgau - 1)^2 window, normalised
    const T pi = (T)3.1415926f;
    const int w = 2 * c->rgau - 1;
    gc = Field<T>(1, w, 1, w);
    {
        const T sigma2 = T(2.0) * T(2.0);
        const int cen = (w + 1) / 2;
        T sum_tmp = 0;
        for (int j = 1; j <= w; j++)
            for (int i = 1; i <= w; i++) {
                const T dis = (T)((j - cen) * (j - cen) + (i - cen) * (i - cen));
                gc(i, j) = T(1) / (T(2) * pi * sigma2) * std::exp(-(dis / (T(2) * sigma2)));
            }
        for (int j = 1; j <= w; j++)
            for (int i = 1; i <= w; i++) sum_tmp = sum_tmp + gc(i, j);
        for (auto& v : gc.d) v = v / sum_tmp;
    }
    // YPUB:323-547 substagger
    Field<T> mu(1, NZ, 1, NX), lamb(1, NZ, 1, NX), busg1(1, NZ, 1, NX), busg2(1, NZ, 1, NX), musg(1, NZ, 1, NX);
    S.busg1e = Field<T>(1, NZ, 1, NX); S.busg2e = Field<T>(1, NZ, 1, NX); S.musge = Field<T>(1, NZ, 1, NX);
    S.lambsg = Field<T>(1, NZ, 1, NX); S.lambmusg = Field<T>(1, NZ, 1, NX);
    for (int i = 1; i <= NX; i++)
        for (int k = 1; k <= NZ; k++) {
            mu(k, i) = rhoe(k, i) * vse(k, i) * vse(k, i);
            lamb(k, i) = rhoe(k, i) * vpe(k, i) * vpe(k, i) - T(2.0) * mu(k, i);
        }
    for (int i = 1; i <= NX - 1; i++)
        for (int k = 1; k <= NZ - 1; k++)
            busg1(k, i) = T(0.25) * (rhoe(k, i) + rhoe(k + 1, i) + rhoe(k + 1, i + 1) + rhoe(k, i + 1));
    for (int i = 1; i <= NX; i++) busg1(NZ, i) = busg1(NZ - 1, i);
    for (int k = 1; k <= NZ; k++) busg1(k, NX) = busg1(k, NX - 1);
    for (int i = 1; i <= NX; i++)
        for (int k = 1; k <= NZ; k++) {
            if (busg1(k, i) == T(0)) return 2;  // YPUB:370 stops here
            busg1(k, i) = T(1.0) / busg1(k, i);
        }
    for (int i = 1; i <= NX; i++)
        for (int k = 2; k <= NZ; k++) S.busg1e(k, i) = T(0.5) * (busg1(k, i) + busg1(k - 1, i));
    for (int i = 1; i <= NX; i++) S.busg1e(1, i) = busg1(1, i);
    for (int i = 1; i <= NX; i++)
        for (int k = 1; k <= NZ; k++) {
            if (rhoe(k, i) == T(0)) return 2;
            busg2(k, i) = T(1.0) / rhoe(k, i);
        }
    for (int i = 1; i <= NX - 1; i++)
        for (int k = 1; k <= NZ; k++) S.busg2e(k, i) = T(0.5) * (busg2(k, i) + busg2(k, i + 1));
    for (int k = 1; k <= NZ; k++) S.busg2e(k, NX) = busg2(k, NX);
    for (int i = 1; i <= NX; i++)
        for (int k = 1; k <= NZ - 1; k++) musg(k, i) = T(0.5) * (mu(k + 1, i) + mu(k, i));
    for (int i = 1; i <= NX; i++) musg(NZ, i) = mu(NZ, i);
    for (int i = 1; i <= NX - 1; i++)
        for (int k = 2; k <= NZ; k++) {
            if (musg(k, i) != T(0) && musg(k - 1, i) != T(0) && musg(k, i + 1) != T(0) && musg(k - 1, i + 1) != T(0))
                S.musge(k, i) = T(4.0) / (T(1.0) / musg(k, i) + T(1.0) / musg(k, i + 1) + T(1.0) / musg(k - 1, i + 1) +
                                          T(1.0) / musg(k - 1, i));
            else
                S.musge(k, i) = T(0);
        }
    for (int i = 1; i <= NX; i++) S.musge(1, i) = musg(1, i);
    for (int k = 1; k <= NZ; k++) S.musge(k, NX) = musg(k, NX);
    for (int k = 1; k <= NZ; k++)
        for (int i = 1; i <= NX - 1; i++) S.lambsg(k, i) = T(0.5) * (lamb(k, i + 1) + lamb(k, i));
    for (int k = 1; k <= NZ; k++) S.lambsg(k, NX) = lamb(k, NX);
    for (int i = 1; i <= NX - 1; i++)
        for (int k = 1; k <= NZ; k++)
            S.lambmusg(k, i) = T(0.5) * (lamb(k, i) + T(2) * mu(k, i) + lamb(k, i + 1) + T(2) * mu(k, i + 1));
    for (int k = 1; k <= NZ; k++) S.lambmusg(k, NX) = lamb(k, NX) + T(2) * mu(k, NX);
    // YPUB:484-501 rows above itopo take row itopo's values (only the time loop's five arrays
    // are carried further)
    for (auto* f : {&S.lambsg, &S.lambmusg, &S.musge, &S.busg1e, &S.busg2e})
        for (int i = 1; i <= NX; i++)
            for (int k = S.itopo[i]; k >= 2; k--) (*f)(k - 1, i) = (*f)(k, i);
    // YPRI:301-302 modipapml, abc mode only
    if (!S.fs)
        for (auto* f : {&S.lambsg, &S.musge, &S.lambmusg, &S.busg1e, &S.busg2e})
            gauss_filter(*f, NX, NZ, c->rgau, S.itopo, gc);
    // YPUB:796-849 cosine sponge, R = 1e-3
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
    return 0;
}

template <typename T>
int run_iso(const OracleIsoCfg* c, const float* vp_in, const float* vs_in, const float* rho_in, T* rec1, T* rec2,
            T* final_vx) {
    IsoSolver<T> S;
    Field<T> gc;
    const int rc = prepare(c, vp_in, vs_in, rho_in, S, gc);
    if (rc) return rc;
    const int NX = S.nx, NZ = S.nz, nxe = c->ixmaxe - c->ixmine + 1;
    const T pi = (T)3.1415926f;
    // YPUB:1429-1466 addsrc: the (2 rgau - 1)^2 window around the source; cells with an exact zero
    // weight are left out (adding a zero leaves u unchanged)
    const int isxe = c->isxe, isze = c->isze;
    struct Tap { int m, n; T g; };
    std::vector<Tap> taps;
    {
        int idx2 = 1;
        for (int n = isxe - (c->rgau - 1); n <= isxe + (c->rgau - 1); n++) {
            int idx1 = 1;
            for (int m = isze - (c->rgau - 1); m <= isze + (c->rgau - 1); m++) {
                if (n >= 1 && n <= NX && m >= 1 && m <= NZ && gc(idx1, idx2) != T(0)) taps.push_back({m, n, gc(idx1, idx2)});
                idx1++;
            }
            idx2++;
        }
    }
    int it_cur = 0;
    const T f0 = c->f0;
    auto addsrc = [&](Field<T>& u) {
        const T b = pi * f0 * (T(it_cur) * S.dt - T(c->idecay) * S.dt);
        const T wav = std::exp(-(b * b)) * (T(1) - T(2) * (b * b));
        for (const Tap& t : taps) u(t.m, t.n) = wav * t.g * S.dt / (S.dz * S.dz) + u(t.m, t.n);
    };
    // YPRI:305-367
    const int nt = c->nt;

    // YPRI:163-168: in fsbc mode strxx takes the source only below the surface
    const bool src_xx = !S.fs || isze > S.itopo[isxe];
    for (int it = 1; it <= nt + c->idecay; it++) {
        it_cur = it;
        S.step(addsrc, src_xx);
        const int iit = it - c->idecay;
        if (iit >= 1) {
            for (int i = 1; i <= nxe; i++) {
                const int kr = S.itopo[i + c->npxn] + c->nrz0;  // YPUB:13 itopo(i+npxn)+nrz0
                if (rec1) rec1[(size_t)(i - 1) * nt + (iit - 1)] = S.vx(kr, i + c->npxn);
                if (rec2) rec2[(size_t)(i - 1) * nt + (iit - 1)] = S.vz(kr, i + c->npxn);
            }
        }
    }
    if (final_vx)
        for (int i = 1; i <= NX; i++)
            for (int k = 1; k <= NZ; k++) final_vx[(size_t)(i - 1) * NZ + (k - 1)] = S.vx(k, i);
    return 0;
}

}  // namespace

extern "C" {

int oracle_iso_prepare_f32(const OracleIsoCfg* c, const float* vp, const float* vs, const float* rho, float* out) {
    IsoSolver<float> S;
    Field<float> gc;
    const int rc = prepare(c, vp, vs, rho, S, gc);
    if (rc) return rc;
    const size_t n = (size_t)S.nx * S.nz;
    const Field<float>* arrs[5] = {&S.busg2e, &S.busg1e, &S.lambmusg, &S.lambsg, &S.musge};
    for (int a = 0; a < 5; a++) std::memcpy(out + a * n, arrs[a]->d.data(), n * sizeof(float));
    return 0;
}

int oracle_iso_f32(const OracleIsoCfg* c, const float* vp, const float* vs, const float* rho, float* rec1, float* rec2,
                   float* final_vx) {
    return run_iso<float>(c, vp, vs, rho, rec1, rec2, final_vx);
}

int oracle_iso_f64(const OracleIsoCfg* c, const float* vp, const float* vs, const float* rho, double* rec1,
                   double* rec2, double* final_vx) {
    return run_iso<double>(c, vp, vs, rho, rec1, rec2, final_vx);
}

}  // extern "C"
