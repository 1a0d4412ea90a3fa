// q_forward: drop-in for the forward/Q_forward program (Q_multishot_fd_main_fsbc_zy_rotated.f90,
// QM) on one GPU: the viscoacoustic scheme when the vs file is zero everywhere, the full
// visco-elastic P-SV scheme otherwise.
//
//   q_forward PARFILE [--use-q] [--snapshots DIR] [--keep-parts] [--device N]
//
// Reads the parameter card (QS:121-234) and the five model files (QS:238-284), lays out the
// shots as QM:124-141 does (isx = isx0 + nint((i-1) dsx/dx), aperture [ixmine, ixmaxe] from the
// offsets), pads every shot's window by edge replication (QS:288-428), models all shots in one
// batched time loop of nt + decay steps (QM:439-459), writes each shot's records as SU files
// (QS:1476-1546: <shot_fn1>N.su from strzz, <shot_fn3>N.su from strxx; for vs = 0 both are the
// pressure sigma) and merges them into <shot_fn2>.su and <shot_fn4>.su (QS:1550-1624), deleting
// the per-shot files unless --keep-parts.
//
// The stock program overrides the quality factors with 1e5 before modelling (QM:418-419), so by
// default Q is ignored as there; --use-q models with the qfp file.  --snapshots DIR writes the
// interior strxx / strzz every 50 steps (QM:462-481) of the last shot, named
// iso_vx_elastic_<it> / iso_vz_elastic_<it>.  The per-shot model dumps of QS:377-425 (vpe_test
// ...) are debugging output and are not written.
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
    std::fprintf(stderr, "q_forward: %s: %s%s%s\n", what, sfd_status_string(rc), msg[0] ? ": " : "", msg);
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

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: q_forward PARFILE [--use-q] [--snapshots DIR] [--keep-parts] [--device N]\n");
        return 2;
    }
    const char* par_fn = argv[1];
    bool use_q = false, keep = false;
    std::string snap_dir;
    int device = 0;
    for (int i = 2; i < argc; i++) {
        const std::string a = argv[i];
        if (a == "--use-q") use_q = true;
        else if (a == "--keep-parts") keep = true;
        else if (a == "--snapshots" && i + 1 < argc) snap_dir = argv[++i];
        else if (a == "--device" && i + 1 < argc) device = std::atoi(argv[++i]);
        else {
            std::fprintf(stderr, "q_forward: unknown option %s\n", a.c_str());
            return 2;
        }
    }
    sfd_qpar p{};
    int rc = sfd_qpar_read(par_fn, &p);
    if (rc) return fail(par_fn, rc, nullptr);
    const int nx = p.nx, nz = p.nz;
    if (nx < 1 || nz < 1 || p.nt < 1 || p.nshot < 1 || !(p.dx > 0) || !(p.dz > 0) || !(p.dt > 0) || !(p.f0 > 0))
        return fail("parameter card", SFD_ERR_ARG, nullptr);
    // QM:104-112: pads in cells, source / receiver positions (1-based)
    const int npxn = nint(p.pml_xn / p.dx) + 1, npxp = nint(p.pml_xp / p.dx) + 1;
    const int npzn = nint(p.pml_zn / p.dz) + 1, npzp = nint(p.pml_zp / p.dz) + 1;
    if (npxn != npxp || npxn != npzn || npxn != npzp)
        return fail("sponge widths (the engine uses one width on all four sides)", SFD_ERR_UNSUPPORTED, nullptr);
    const int np = npxn;
    const int isx0 = nint(p.sx0 / p.dx) + 1, nsz0 = nint(p.sz0 / p.dz) + 1, nrz0 = nint(p.rz0 / p.dz) + 1;
    // QS:238-284: model arrays (nz, nx), i.e. x-major with z fastest
    const size_t nm = (size_t)nx * nz;
    std::vector<float> vp(nm), vs(nm), rho(nm), qp(nm), qs(nm);
    const char* files[5] = {p.vp, p.vs, p.rho, p.qp, p.qs};
    std::vector<float>* arrays[5] = {&vp, &vs, &rho, &qp, &qs};
    for (int f = 0; f < 5; f++)
        if ((rc = sfd_read_floats(strip(files[f]).c_str(), (long long)nm, arrays[f]->data())))
            return fail(files[f], rc, nullptr);
    bool elastic = false;  // any shear velocity: the full P-SV scheme (QS:751-835)
    for (size_t i = 0; i < nm; i++) elastic = elastic || vs[i] != 0.0f;
    // QS:1364-1366 (single precision): wavelet length and the decay steps before recording
    const int nwt = 2 * nint(1.2f / (p.f0 * p.dt));
    const int decay = nint(nwt / 2.0f);
    const int nt_run = p.nt + decay;
    std::vector<float> w(nt_run);
    if ((rc = sfd_wavelet(SFD_WAVELET_Q, nt_run, p.dt, p.f0, 0, w.data()))) return fail("wavelet", rc, nullptr);

    // shots (QM:124-129) and their padded windows (QS:288-372), identical windows shared
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
    const int nzea = nz + 2 * np;
    std::vector<int> block_x0(blocks.size());
    int width = 0;
    for (size_t b = 0; b < blocks.size(); b++) {
        block_x0[b] = width;
        width += blocks[b].second + 2 * np;
    }
    const size_t nme = (size_t)width * nzea;
    std::vector<float> vpe(nme), rhoe(nme), qpe(nme), vse(elastic ? nme : 0), qse(elastic ? nme : 0);
    for (size_t b = 0; b < blocks.size(); b++) {
        const int ixmine = blocks[b].first, nxe = blocks[b].second, nxea = nxe + 2 * np;
        for (int c = 0; c < nxea; c++) {
            // window column i = 1..nxe reads model column i + ixmine (QS:310-313, clamped);
            // pad columns repeat the window's edge columns (QS:351-372)
            const int i = c < np ? 1 : (c >= np + nxe ? nxe : c - np + 1);
            int i_ori = i + ixmine;
            i_ori = i_ori < 1 ? 1 : (i_ori > nx ? nx : i_ori);
            for (int k = 0; k < nzea; k++) {
                const int kz = k < np ? 0 : (k >= np + nz ? nz - 1 : k - np);  // QS:326-347
                const size_t src = (size_t)(i_ori - 1) * nz + kz, dst = (size_t)(block_x0[b] + c) * nzea + k;
                vpe[dst] = vp[src];
                rhoe[dst] = rho[src];
                qpe[dst] = qp[src];
                if (elastic) {
                    vse[dst] = vs[src];
                    qse[dst] = qs[src];
                }
            }
        }
    }

    sfd_grid g{};
    g.scheme = elastic ? SFD_VISCOEL_2D : SFD_VISCOAC_2D;
    g.nx = width;
    g.ny = 1;
    g.nz = nzea;
    g.pml = np;
    g.dx = p.dx;
    g.dz = p.dz;
    g.dt = p.dt;
    g.order = 10;
    g.f0 = p.f0;
    g.flags = SFD_EXACT;  // the reference's operation order: the outputs equal the reference program's
    sfd_ctx* ctx = nullptr;
    if ((rc = sfd_create(&g, device, &ctx))) return fail("sfd_create", rc, ctx);
    if (elastic) {
        if ((rc = sfd_set_model_elastic(ctx, vpe.data(), vse.data(), rhoe.data(), use_q ? qpe.data() : nullptr,
                                        use_q ? qse.data() : nullptr)))
            return fail("sfd_set_model_elastic", rc, ctx);
    } else if ((rc = sfd_set_model(ctx, vpe.data(), rhoe.data(), use_q ? qpe.data() : nullptr))) {
        return fail("sfd_set_model", rc, ctx);
    }
    std::vector<sfd_shot> desc(p.nshot);
    std::vector<std::vector<int>> rx(p.nshot), rz(p.nshot);
    for (int i = 0; i < p.nshot; i++) {
        const ShotInfo& s = shots[i];
        // QS:374-375: isxe = isx - ixmine + npxn + 1, isze = isz + itopoe (flat surface: npzn + 1)
        desc[i].sx = s.isx - s.ixmine + np;
        desc[i].sz = nsz0 + np;
        desc[i].nt = nt_run;
        // QM:452-459: receivers at row itopoe + nrz0 of every window column
        rx[i].resize(s.nxe);
        rz[i].assign(s.nxe, np + nrz0);
        for (int c = 0; c < s.nxe; c++) rx[i][c] = np + c;
        desc[i].nrec = s.nxe;
        desc[i].rec_x = rx[i].data();
        desc[i].rec_z = rz[i].data();
        desc[i].wavelet = w.data();
        desc[i].ap_x0 = block_x0[s.block];
        desc[i].ap_nx = s.nxe + 2 * np;
    }
    if ((rc = sfd_set_shots(ctx, p.nshot, desc.data()))) return fail("sfd_set_shots", rc, ctx);
    const int nsnap = nt_run / 50;
    // QM:462-481: strxx (snapx) and strzz (snapz) every 50 steps
    if (!snap_dir.empty() && nsnap > 0 &&
        ((rc = sfd_set_snapshots(ctx, 0, SFD_FIELD_P, 49, 50, nsnap)) ||
         (elastic && (rc = sfd_set_snapshots(ctx, 1, SFD_FIELD_SZZ, 49, 50, nsnap)))))
        return fail("sfd_set_snapshots", rc, ctx);
    long long total = 0;
    for (const auto& s : shots) total += (long long)s.nxe * nt_run;
    std::vector<float> rec(total), rec2;
    if ((rc = sfd_forward(ctx, rec.data()))) return fail("sfd_forward", rc, ctx);  // record1: strzz
    if (elastic) {  // record2: strxx (for vs = 0 the same sigma)
        rec2.resize(total);
        if ((rc = sfd_get_records(ctx, SFD_FIELD_P, rec2.data()))) return fail("sfd_get_records", rc, ctx);
    }
    const std::vector<float>& recx = elastic ? rec2 : rec;

    // SU output per shot (record1 -> shot_fn1, record2 -> shot_fn3), then the merge
    const std::string f1 = strip(p.shot1), f2 = strip(p.shot2), f3 = strip(p.shot3), f4 = strip(p.shot4);
    std::vector<std::string> parts1, parts3;
    long long off = 0;
    for (int i = 0; i < p.nshot; i++) {
        const ShotInfo& s = shots[i];
        std::vector<float> tr((size_t)s.nxe * p.nt), tx((size_t)s.nxe * p.nt);
        for (int r = 0; r < s.nxe; r++) {
            std::memcpy(tr.data() + (size_t)r * p.nt, rec.data() + off + (long long)r * nt_run + decay,
                        sizeof(float) * p.nt);
            std::memcpy(tx.data() + (size_t)r * p.nt, recx.data() + off + (long long)r * nt_run + decay,
                        sizeof(float) * p.nt);
        }
        off += (long long)s.nxe * nt_run;
        const std::string n1 = f1 + std::to_string(i + 1) + ".su", n3 = f3 + std::to_string(i + 1) + ".su";
        if ((rc = sfd_su_write(n1.c_str(), tr.data(), s.nxe, p.nt, i + 1, s.isx, s.ixmine, p.dx, p.dt)) ||
            (rc = sfd_su_write(n3.c_str(), tx.data(), s.nxe, p.nt, i + 1, s.isx, s.ixmine, p.dx, p.dt)))
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
        std::vector<float> frames((size_t)nsnap * nf), framez;
        int got = 0, gotz = 0;
        if ((rc = sfd_get_snapshots(ctx, 0, last, frames.data(), &got))) return fail("snapshots", rc, ctx);
        if (elastic) {
            framez.resize(frames.size());
            if ((rc = sfd_get_snapshots(ctx, 1, last, framez.data(), &gotz))) return fail("snapshots", rc, ctx);
        }
        const std::vector<float>& fz = elastic ? framez : frames;  // strzz (= strxx for vs = 0)
        for (int j = 0; j < got; j++) {
            const std::string it = std::to_string(50 * (j + 1));
            if ((rc = sfd_write_floats((snap_dir + "/iso_vx_elastic_" + it).c_str(), frames.data() + j * nf, nf, 0)) ||
                (rc = sfd_write_floats((snap_dir + "/iso_vz_elastic_" + it).c_str(), fz.data() + j * nf, nf, 0)))
                return fail("snapshot files", rc, ctx);
        }
    }
    sfd_destroy(ctx);
    std::printf("==========2D_Iso_acoustic_modelling end==========\n");
    return 0;
}
