// afd_fd: drop-in for the forward/Acoustic_FD_by_ss program (Acoustic_1order_FD.cpp).
//
// With no options it runs the reference's hard-coded case (AFD:28-45: NX = NZ = 100, PML = 20,
// Nt = 2000, dx = dz = 10 m, dt = 0.5 ms, Vp = 2000, DEN = 2400, 28 Hz wavelet of AFD:199-209,
// source at (Nx/2, Nz/2), receivers on the vertical line x = Nx/2) and writes the same files into
// ../file: Model.dat (interior Vp), Snap.dat (interior Vx after step 500), Pall.dat (interior P
// after every 10th step, appended) and record.dat (trace-major).  The reference-order arithmetic
// (SFD_EXACT) is the default, so the outputs equal the reference's bit for bit; --fast selects the
// FMA kernel.  The options override the hard-coded values; grid indices are padded-grid cells.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "seisfd.h"

namespace {

void usage() {
    std::fprintf(stderr,
                 "usage: afd_fd [--nx 100] [--nz 100] [--pml 20] [--nt 2000] [--dx 10] [--dz 10] [--dt 0.0005]\n"
                 "              [--f0 28] [--vp FILE | --vp-const 2000] [--den FILE | --den-const 2400]\n"
                 "              [--wavelet FILE] [--sx X] [--sz Z] [--rec-z Z] [--snap K] [--pall-every N]\n"
                 "              [--out DIR] [--fast] [--device N]\n"
                 "  FILE arrays are the padded Nx x Nz grid (Nx = NX + 2 PML), float32, x-major; --rec-z puts the\n"
                 "  receivers on the horizontal line z = Z instead of AFD's vertical line x = Nx/2;\n"
                 "  --snap -1 and --pall-every 0 switch those outputs off.\n");
}

int fail(const char* what, int rc, sfd_ctx* ctx) {
    char msg[512] = "";
    if (ctx) sfd_last_error(ctx, msg, sizeof(msg));
    std::fprintf(stderr, "afd_fd: %s: %s%s%s\n", what, sfd_status_string(rc), msg[0] ? ": " : "", msg);
    if (ctx) sfd_destroy(ctx);
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    int NX = 100, NZ = 100, PML = 20, Nt = 2000, sx = -1, sz = -1, rec_z = -1, snap = 500, pall = 10, device = 0;
    float dx = 10.0f, dz = 10.0f, dt = 0.0005f, f0 = 28.0f, vp_c = 2000.0f, den_c = 2400.0f;
    std::string vp_file, den_file, wav_file, out = "../file";
    bool fast = false;
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        auto val = [&]() -> const char* {
            if (i + 1 >= argc) {
                usage();
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "--nx") NX = std::atoi(val());
        else if (a == "--nz") NZ = std::atoi(val());
        else if (a == "--pml") PML = std::atoi(val());
        else if (a == "--nt") Nt = std::atoi(val());
        else if (a == "--dx") dx = std::strtof(val(), nullptr);
        else if (a == "--dz") dz = std::strtof(val(), nullptr);
        else if (a == "--dt") dt = std::strtof(val(), nullptr);
        else if (a == "--f0") f0 = std::strtof(val(), nullptr);
        else if (a == "--vp") vp_file = val();
        else if (a == "--vp-const") vp_c = std::strtof(val(), nullptr);
        else if (a == "--den") den_file = val();
        else if (a == "--den-const") den_c = std::strtof(val(), nullptr);
        else if (a == "--wavelet") wav_file = val();
        else if (a == "--sx") sx = std::atoi(val());
        else if (a == "--sz") sz = std::atoi(val());
        else if (a == "--rec-z") rec_z = std::atoi(val());
        else if (a == "--snap") snap = std::atoi(val());
        else if (a == "--pall-every") pall = std::atoi(val());
        else if (a == "--out") out = val();
        else if (a == "--fast") fast = true;
        else if (a == "--device") device = std::atoi(val());
        else {
            usage();
            return 2;
        }
    }
    const int Nx = NX + 2 * PML, Nz = NZ + 2 * PML;
    if (NX < 1 || NZ < 1 || PML < 0 || Nt < 1) {
        usage();
        return 2;
    }
    if (sx < 0) sx = Nx / 2;  // AFD:215-216
    if (sz < 0) sz = Nz / 2;
    const size_t n = (size_t)Nx * Nz;
    std::vector<float> vp(n, vp_c), den(n, den_c), w(Nt);
    int rc;
    if (!vp_file.empty() && (rc = sfd_read_floats(vp_file.c_str(), (long long)n, vp.data())))
        return fail(vp_file.c_str(), rc, nullptr);
    if (!den_file.empty() && (rc = sfd_read_floats(den_file.c_str(), (long long)n, den.data())))
        return fail(den_file.c_str(), rc, nullptr);
    if (!wav_file.empty()) {
        if ((rc = sfd_read_floats(wav_file.c_str(), Nt, w.data()))) return fail(wav_file.c_str(), rc, nullptr);
    } else if ((rc = sfd_wavelet(SFD_WAVELET_AFD, Nt, dt, f0, 0, w.data()))) {
        return fail("wavelet", rc, nullptr);
    }
    // receivers: AFD:376-377 records P1[nx_location][i] for i = PML .. Nx-PML-1 (a vertical line
    // at the source column); --rec-z gives the horizontal line P1[i][rec_z] instead
    std::vector<int> rx(NX), rz(NX);
    for (int i = 0; i < NX; i++) {
        rx[i] = rec_z >= 0 ? PML + i : sx;
        rz[i] = rec_z >= 0 ? rec_z : PML + i;
    }
    sfd_grid g{};
    g.scheme = SFD_ACOUSTIC_2D;
    g.nx = Nx;
    g.ny = 1;
    g.nz = Nz;
    g.pml = PML;
    g.dx = dx;
    g.dz = dz;
    g.dt = dt;
    g.order = 16;
    g.flags = fast ? 0 : SFD_EXACT;
    sfd_ctx* ctx = nullptr;
    if ((rc = sfd_create(&g, device, &ctx))) return fail("sfd_create", rc, ctx);
    if ((rc = sfd_set_model(ctx, vp.data(), den.data(), nullptr))) return fail("sfd_set_model", rc, ctx);
    sfd_shot shot{};
    shot.sx = sx;
    shot.sz = sz;
    shot.nt = Nt;
    shot.nrec = NX;
    shot.rec_x = rx.data();
    shot.rec_z = rz.data();
    shot.wavelet = w.data();
    if ((rc = sfd_set_shots(ctx, 1, &shot))) return fail("sfd_set_shots", rc, ctx);
    if (snap >= 0 && snap < Nt && (rc = sfd_set_snapshots(ctx, 0, SFD_FIELD_VX, snap, 1, 1)))
        return fail("sfd_set_snapshots", rc, ctx);
    if (pall > 0 && (rc = sfd_set_snapshots(ctx, 1, SFD_FIELD_P, 0, pall, (Nt - 1) / pall + 1)))
        return fail("sfd_set_snapshots", rc, ctx);
    std::vector<float> rec((size_t)NX * Nt);
    if ((rc = sfd_forward(ctx, rec.data()))) return fail("sfd_forward", rc, ctx);

    // outputs, AFD:144-158 (Model.dat), AFD:343-373 (Snap.dat, Pall.dat), AFD:385-393 (record.dat)
    const std::string dir = out + "/";
    std::vector<float> interior((size_t)NX * NZ);
    for (int i = 0; i < NX; i++)
        for (int j = 0; j < NZ; j++) interior[(size_t)i * NZ + j] = vp[(size_t)(i + PML) * Nz + j + PML];
    if ((rc = sfd_write_floats((dir + "Model.dat").c_str(), interior.data(), (long long)interior.size(), 0)))
        return fail("Model.dat", rc, ctx);
    int nsnap = 0;
    if (snap >= 0 && snap < Nt) {
        if ((rc = sfd_get_snapshots(ctx, 0, 0, interior.data(), &nsnap))) return fail("snapshot", rc, ctx);
        if ((rc = sfd_write_floats((dir + "Snap.dat").c_str(), interior.data(), (long long)interior.size(), 0)))
            return fail("Snap.dat", rc, ctx);
    }
    if (pall > 0) {
        std::vector<float> frames((size_t)((Nt - 1) / pall + 1) * NX * NZ);
        if ((rc = sfd_get_snapshots(ctx, 1, 0, frames.data(), &nsnap))) return fail("snapshots", rc, ctx);
        std::remove((dir + "Pall.dat").c_str());  // AFD:221, then appended frame by frame
        if ((rc = sfd_write_floats((dir + "Pall.dat").c_str(), frames.data(), (long long)nsnap * NX * NZ, 1)))
            return fail("Pall.dat", rc, ctx);
    }
    if ((rc = sfd_write_floats((dir + "record.dat").c_str(), rec.data(), (long long)rec.size(), 0)))
        return fail("record.dat", rc, ctx);
    sfd_destroy(ctx);
    std::printf("\nEnd of Calculation!!\n");
    return 0;
}
