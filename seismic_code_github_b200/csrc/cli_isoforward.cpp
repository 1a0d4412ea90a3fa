// iso_forward: drop-in for the forward/yang_version_2016_2_2 program
// (Iso_multishot_fd_main_fsbc_zy_m2.f90, YM) on one GPU: isotropic elastic P-SV modelling on the
// standard staggered grid, in the card's mode ('abc' or 'fsbc').
//
//   iso_forward PARFILE [--snapshots DIR] [--keep-parts] [--device N]
//
// Reads the parameter card (YPUB:48-145) and the model files vp, vs, rho (nz x nx Fortran arrays,
// i.e. x-major with z fastest) and the topography (nx values, YPUB:148-184).  Lays out the shots
// as YM:71-81 and YPRI:2-53 do: isx = isx0 + nint((i-1) dsx/dx), aperture [ixmine, ixmaxe] from
// the offsets, sponge cells np = nint(pp/dx) + 1 per side, decay nint(decay/dt) steps.  Pads every
// shot's window by edge replication (YPUB:188-313).  Models all shots in one batched time loop of
// nt + decay steps (YPRI:57-386).  Writes each shot's records as SU files, <shot_fn1>N.su from vx
// and <shot_fn3>N.su from vz (YPUB:1533-1604, no cdp), and merges them into <shot_fn2>.su and
// <shot_fn4>.su (YPUB:1607-1684), deleting the per-shot files unless --keep-parts.
//
// --snapshots DIR writes the interior vx / vz every dtsnap of the last shot as DIR/<name><it>,
// where <name> is the last path component of the card's snapx / snapz prefix (YPRI:212-224,
// YPUB:20-44).  The reference writes them for the shots of MPI rank 0 into the card's
// directories.
// The topography file gives each model column's surface depth; every window column gets
// itopoe = nint(topoe/dz) + npzn (YPUB:216-272, pads repeat the window's edge columns), the
// source sits at isz + itopoe(isxe) and trace i records row itopoe(i + npxn) + nrz0 (YPUB:2-16).
// Limit of this engine, reported as an error: one sponge width for the left, right and bottom
// sides (and the top in abc mode).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "seisfd.h"

namespace {

int fail(const char* what, int rc, sfd_ctx* ctx) {
    char msg[512] = "";
    if (ctx) sfd_last_error(ctx, msg, sizeof(msg));
    std::fprintf(stderr, "iso_forward: %s: %s%s%s\n", what, sfd_status_string(rc), msg[0] ? ": " : "", msg);
    if (ctx) sfd_destroy(ctx);
    return 1;
}

int nint(float v) { return (int)std::lround(v); }  // Fortran nint: halves away from zero

std::string strip(const char* s) {
    std::string t(s);
    size_t a = t.find_first_not_of(" \t");
    size_t b = t.find_last_not_of(" \t");
    return a == std::string::npos ? std::string() : t.substr(a, b - a + 1);
}

std::string basename_of(const std::string& p) {
    const size_t k = p.find_last_of('/');
    return k == std::string::npos ? p : p.substr(k + 1);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: iso_forward PARFILE [--snapshots DIR] [--keep-parts] [--device N]\n");
        return 2;
    }
    const char* par_fn = argv[1];
    bool keep = false;
    std::string snap_dir;
    int device = 0;
    for (int i = 2; i < argc; i++) {
        const std::string a = argv[i];
        if (a == "--keep-parts") keep = true;
        else if (a == "--snapshots" && i + 1 < argc) snap_dir = argv[++i];
        else if (a == "--device" && i + 1 < argc) device = std::atoi(argv[++i]);
        else {
            std::fprintf(stderr, "iso_forward: unknown option %s\n", a.c_str());
            return 2;
        }
    }
    sfd_isopar p{};
    int rc = sfd_isopar_read(par_fn, &p);
    if (rc) return fail(par_fn, rc, nullptr);
    const int nx = p.nx, nz = p.nz;
    if (nx < 1 || nz < 1 || p.nt < 1 || p.nshot < 1 || !(p.dx > 0) || !(p.dz > 0) || !(p.dt > 0) || !(p.f0 > 0) ||
        p.rgau < 1)
        return fail("parameter card", SFD_ERR_ARG, nullptr);
    const std::string mode = strip(p.molmod);
    const bool fsbc = mode == "fsbc";
    if (!fsbc && mode != "abc") return fail("modelling mode (YM:190-219: abc or fsbc)", SFD_ERR_ARG, nullptr);
    // YPRI:26-38: sponge cells, steps, source / receiver rows (1-based)
    const int npxn = nint(p.pml_xn / p.dx) + 1, npxp = nint(p.pml_xp / p.dx) + 1;
    const int npzn = nint(p.pml_zn / p.dz) + 1, npzp = nint(p.pml_zp / p.dz) + 1;
    if (npxn != npxp || npxn != npzp || (!fsbc && npxn != npzn))
        return fail("sponge widths (the engine uses one width on the left, right and bottom, and the top in abc mode)",
                    SFD_ERR_UNSUPPORTED, nullptr);
    const int np = npxn, top = npzn;
    const int idtsnap = nint(p.dtsnap / p.dt), idecay = nint(p.decay / p.dt);
    const int isx0 = nint(p.sx0 / p.dx) + 1, isz0 = nint(p.sz0 / p.dz) + 1, irz0 = nint(p.rz0 / p.dz) + 1;
    // YPUB:148-184: models and topography
    const size_t nm = (size_t)nx * nz;
    std::vector<float> vp(nm), vs(nm), rho(nm), topo(nx);
    const char* files[3] = {p.vp, p.vs, p.rho};
    std::vector<float>* arrays[3] = {&vp, &vs, &rho};
    for (int f = 0; f < 3; f++)
        if ((rc = sfd_read_floats(strip(files[f]).c_str(), (long long)nm, arrays[f]->data())))
            return fail(files[f], rc, nullptr);
    if ((rc = sfd_read_floats(strip(p.topo).c_str(), nx, topo.data()))) return fail(p.topo, rc, nullptr);
    const int nt_run = p.nt + idecay;
    std::vector<float> w(nt_run);
    if ((rc = sfd_wavelet(SFD_WAVELET_ISO, nt_run, p.dt, p.f0, idecay, w.data()))) return fail("wavelet", rc, nullptr);

    // shots (YM:71-81, YPRI:40-45) and their padded windows (YPUB:210-266), identical windows shared
    struct ShotInfo {
        int isx, ixmine, ixmaxe, nxe, block;
    };
    std::vector<ShotInfo> shots(p.nshot);
    std::map<std::pair<int, int>, int> block_of;
    std::vector<std::pair<int, int>> blocks;  // (ixmine, nxe)
    for (int i = 1; i <= p.nshot; i++) {
        ShotInfo s{};
        s.isx = isx0 + nint((i - 1) * p.dsx / p.dx);
        s.ixmine = s.isx + nint(p.offset_min / p.dx);
        s.ixmaxe = s.isx + nint(p.offset_max / p.dx);
        s.nxe = s.ixmaxe - s.ixmine + 1;
        if (s.nxe < 1) return fail("offset range", SFD_ERR_ARG, nullptr);
        auto key = std::make_pair(s.ixmine, s.nxe);
        auto it = block_of.find(key);
        if (it == block_of.end()) {
            it = block_of.emplace(key, (int)blocks.size()).first;
            blocks.push_back(key);
        }
        s.block = it->second;
        shots[i - 1] = s;
    }
    const int nzea = nz + top + np;
    std::vector<int> block_x0(blocks.size());
    int width = 0;
    for (size_t b = 0; b < blocks.size(); b++) {
        block_x0[b] = width;
        width += blocks[b].second + 2 * np;
    }
    const size_t nme = (size_t)width * nzea;
    std::vector<float> vpe(nme), vse(nme), rhoe(nme);
    std::vector<int> itopoe(width);  // YPUB:270-272 per padded window column
    for (size_t b = 0; b < blocks.size(); b++) {
        const int ixmine = blocks[b].first, nxe = blocks[b].second, nxea = nxe + 2 * np;
        for (int c = 0; c < nxea; c++) {
            // window column i = 1..nxe reads model column i + ixmine (YPUB:216-228, clamped); pad
            // columns repeat the window's edge columns, pad rows its first and last row
            const int i = c < np ? 1 : (c >= np + nxe ? nxe : c - np + 1);
            int i_ori = i + ixmine;
            i_ori = i_ori < 1 ? 1 : (i_ori > nx ? nx : i_ori);
            itopoe[block_x0[b] + c] = nint(topo[i_ori - 1] / p.dz) + top;
            for (int k = 0; k < nzea; k++) {
                const int kz = k < top ? 0 : (k >= top + nz ? nz - 1 : k - top);
                const size_t src = (size_t)(i_ori - 1) * nz + kz, dst = (size_t)(block_x0[b] + c) * nzea + k;
                vpe[dst] = vp[src];
                vse[dst] = vs[src];
                rhoe[dst] = rho[src];
            }
        }
    }

    sfd_grid g{};
    g.scheme = SFD_ELASTIC_2D;
    g.nx = width;
    g.ny = 1;
    g.nz = nzea;
    g.pml = np;
    g.dx = p.dx;
    g.dz = p.dz;
    g.dt = p.dt;
    g.order = 10;
    g.f0 = p.f0;
    sfd_ctx* ctx = nullptr;
    if ((rc = sfd_create(&g, device, &ctx))) return fail("sfd_create", rc, ctx);
    if ((rc = sfd_set_gauss_radius(ctx, p.rgau))) return fail("sfd_set_gauss_radius", rc, ctx);
    if (fsbc && (rc = sfd_set_free_surface(ctx, top))) return fail("sfd_set_free_surface", rc, ctx);
    if ((rc = sfd_set_topography(ctx, itopoe.data()))) return fail("sfd_set_topography", rc, ctx);
    if ((rc = sfd_set_model_elastic(ctx, vpe.data(), vse.data(), rhoe.data(), nullptr, nullptr)))
        return fail("sfd_set_model_elastic", rc, ctx);
    std::vector<sfd_shot> desc(p.nshot);
    std::vector<std::vector<int>> rx(p.nshot), rz(p.nshot);
    for (int i = 0; i < p.nshot; i++) {
        const ShotInfo& s = shots[i];
        // YPUB:276-277: isxe = isx - ixmine + npxn + 1, isze = isz + itopoe(isxe)
        const int* it = itopoe.data() + block_x0[s.block];
        desc[i].sx = s.isx - s.ixmine + np;
        desc[i].sz = isz0 + it[desc[i].sx] - 1;
        desc[i].nt = nt_run;
        // YPUB:2-16: receivers at row itopoe(i + npxn) + irz0 of every window column
        rx[i].resize(s.nxe);
        rz[i].resize(s.nxe);
        for (int c = 0; c < s.nxe; c++) {
            rx[i][c] = np + c;
            rz[i][c] = it[np + c] + irz0 - 1;
        }
        desc[i].nrec = s.nxe;
        desc[i].rec_x = rx[i].data();
        desc[i].rec_z = rz[i].data();
        desc[i].wavelet = w.data();
        desc[i].ap_x0 = block_x0[s.block];
        desc[i].ap_nx = s.nxe + 2 * np;
    }
    if ((rc = sfd_set_shots(ctx, p.nshot, desc.data()))) return fail("sfd_set_shots", rc, ctx);
    const int nsnap = idtsnap > 0 ? nt_run / idtsnap : 0;
    // YPRI:212-224: vx and vz after every step it with mod(it, idtsnap) = 0
    if (!snap_dir.empty() && nsnap > 0 &&
        ((rc = sfd_set_snapshots(ctx, 0, SFD_FIELD_VX, idtsnap - 1, idtsnap, nsnap)) ||
         (rc = sfd_set_snapshots(ctx, 1, SFD_FIELD_VZ, idtsnap - 1, idtsnap, nsnap))))
        return fail("sfd_set_snapshots", rc, ctx);
    long long total = 0;
    for (const auto& s : shots) total += (long long)s.nxe * nt_run;
    std::vector<float> recx(total), recz(total);
    if ((rc = sfd_forward(ctx, recx.data()))) return fail("sfd_forward", rc, ctx);  // record1: vx
    if ((rc = sfd_get_records(ctx, SFD_FIELD_VZ, recz.data()))) return fail("sfd_get_records", rc, ctx);

    // SU output per shot (vx -> shot_fn1, vz -> shot_fn3), then the merge
    const std::string f1 = strip(p.shot1), f2 = strip(p.shot2), f3 = strip(p.shot3), f4 = strip(p.shot4);
    std::vector<std::string> parts1, parts3;
    long long off = 0;
    for (int i = 0; i < p.nshot; i++) {
        const ShotInfo& s = shots[i];
        std::vector<float> tx((size_t)s.nxe * p.nt), tz((size_t)s.nxe * p.nt);
        for (int r = 0; r < s.nxe; r++) {
            std::memcpy(tx.data() + (size_t)r * p.nt, recx.data() + off + (long long)r * nt_run + idecay,
                        sizeof(float) * p.nt);
            std::memcpy(tz.data() + (size_t)r * p.nt, recz.data() + off + (long long)r * nt_run + idecay,
                        sizeof(float) * p.nt);
        }
        off += (long long)s.nxe * nt_run;
        const std::string n1 = f1 + std::to_string(i + 1) + ".su", n3 = f3 + std::to_string(i + 1) + ".su";
        if ((rc = sfd_su_write_ex(n1.c_str(), tx.data(), s.nxe, p.nt, i + 1, s.isx, s.ixmine, p.dx, p.dt, 0)) ||
            (rc = sfd_su_write_ex(n3.c_str(), tz.data(), s.nxe, p.nt, i + 1, s.isx, s.ixmine, p.dx, p.dt, 0)))
            return fail("SU write", rc, ctx);
        parts1.push_back(n1);
        parts3.push_back(n3);
    }
    auto merge = [&](const std::string& out, const std::vector<std::string>& parts) {
        std::vector<const char*> v;
        for (const auto& s : parts) v.push_back(s.c_str());
        return sfd_su_merge(out.c_str(), v.data(), (int)v.size(), keep ? 0 : 1);
    };
    if ((rc = merge(f2 + ".su", parts1)) || (rc = merge(f4 + ".su", parts3))) return fail("SU merge", rc, ctx);
    if (!snap_dir.empty() && nsnap > 0) {
        const int last = p.nshot - 1;
        const long long nf = (long long)shots[last].nxe * nz;
        std::vector<float> fx((size_t)nsnap * nf), fz((size_t)nsnap * nf);
        int got = 0, gotz = 0;
        if ((rc = sfd_get_snapshots(ctx, 0, last, fx.data(), &got)) ||
            (rc = sfd_get_snapshots(ctx, 1, last, fz.data(), &gotz)))
            return fail("snapshots", rc, ctx);
        const std::string nxn = basename_of(strip(p.snapx)), nzn = basename_of(strip(p.snapz));
        for (int j = 0; j < got && j < gotz; j++) {
            const std::string it = std::to_string(idtsnap * (j + 1));
            if ((rc = sfd_write_floats((snap_dir + "/" + nxn + it).c_str(), fx.data() + j * nf, nf, 0)) ||
                (rc = sfd_write_floats((snap_dir + "/" + nzn + it).c_str(), fz.data() + j * nf, nf, 0)))
                return fail("snapshot files", rc, ctx);
        }
    }
    sfd_destroy(ctx);
    std::printf("2D isotropic elastic-wave modelling ends\n");
    return 0;
}
