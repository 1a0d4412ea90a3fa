// vti_forward: drop-in for the VTI pseudo-acoustic modelling program of
// de-multiple/convolution_srm/vti_qa_2d_c3_demo1 (VTI_multishot_qacoustic_fd_main_c3.f90, VM;
// subroutines VS) on one GPU.
//
//   vti_forward [PARFILE] [--fast] [--keep-parts] [--device N] [--batch N]
//
// PARFILE defaults to ./vti_qa_2d_modelling_new.par as VM:8-9 does.  Reads the card (VS:342-425)
// and the model files (VS:104-157: nz_v x nx_v Fortran arrays, one record of nz_v floats per model
// column, i.e. x-major with z fastest).  read_data then sets epsilon and delta to zero
// (VS:147-148), so the shipped program models an isotropic medium whatever those files hold;
// this program does the same.  The shots follow VM:136-163: PML cells nint(bound/dx) per side,
// nsx0 = nint(sx0/dx) + 1, nsz0 and nrz0 likewise, nsx = nsx0 + nint((i-1) dsx/dx), aperture
// [nsx + nint(offset_min/dx), nsx + nint(offset_max/dx)].  All shots run batched in one time loop
// per group of --batch shots (default all; every shot has the same aperture width).  The
// reference's operation order is kept (SFD_EXACT) unless --fast.  Each shot is written as
// <shot_fn1>N.su (VS:163-217: fldr, trid, sx, gx, ns, dt; no offset, no cdp) and the parts are
// merged into <shot_fn2>.su (VS:220-264), deleted unless --keep-parts.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "seisfd.h"

namespace {

int nint(float v) { return (int)std::lround(v); }  // Fortran nint: halves away from zero

std::string strip(const char* s) {
    std::string t(s);
    size_t a = t.find_first_not_of(" \t");
    size_t b = t.find_last_not_of(" \t");
    return a == std::string::npos ? std::string() : t.substr(a, b - a + 1);
}

int fail(const char* what, int rc) {
    std::fprintf(stderr, "vti_forward: %s: %s\n", what, sfd_status_string(rc));
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    std::string par_fn = "./vti_qa_2d_modelling_new.par";
    bool fast = false, keep = false;
    int device = 0, batch = 0;
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        if (a == "--fast") fast = true;
        else if (a == "--keep-parts") keep = true;
        else if (a == "--device" && i + 1 < argc) device = std::atoi(argv[++i]);
        else if (a == "--batch" && i + 1 < argc) batch = std::atoi(argv[++i]);
        else if (!a.empty() && a[0] != '-') par_fn = a;
        else {
            std::fprintf(stderr, "usage: vti_forward [PARFILE] [--fast] [--keep-parts] [--device N] [--batch N]\n");
            return 2;
        }
    }
    sfd_vtipar p;
    int rc = sfd_vtipar_read(par_fn.c_str(), &p);
    if (rc) return fail(par_fn.c_str(), rc);
    if (p.nshot < 1 || p.nx_v < 1 || p.nz_v < 1 || p.nt < 1 || !(p.dx_v > 0) || !(p.dz_v > 0))
        return fail("parameter card", SFD_ERR_ARG);

    const size_t nm = (size_t)p.nx_v * p.nz_v;
    std::vector<float> vz(nm), eps(nm), del(nm);
    if ((rc = sfd_read_floats(strip(p.vz).c_str(), (long long)nm, vz.data()))) return fail(p.vz, rc);
    if ((rc = sfd_read_floats(strip(p.epsilon).c_str(), (long long)nm, eps.data()))) return fail(p.epsilon, rc);
    if ((rc = sfd_read_floats(strip(p.delta).c_str(), (long long)nm, del.data()))) return fail(p.delta, rc);
    std::fill(eps.begin(), eps.end(), 0.0f);  // VS:147-148
    std::fill(del.begin(), del.end(), 0.0f);

    sfd_vti_par vp{};
    vp.nx_v = p.nx_v;
    vp.nz_v = p.nz_v;
    vp.dx = p.dx_v;
    vp.dz = p.dz_v;
    vp.dt = p.dt;
    vp.f0 = p.f0;
    vp.nt = p.nt;
    vp.nx_bound_l = nint(p.bound_x_l / p.dx_v);  // VM:136-141
    vp.nx_bound_r = nint(p.bound_x_r / p.dx_v);
    vp.nz_bound_u = nint(p.bound_z_u / p.dz_v);
    vp.nz_bound_d = nint(p.bound_z_d / p.dz_v);
    vp.order_explicit = p.order_explicit;
    vp.order_pml_1st = p.order_pml_1st;
    vp.order_pml_2nd = p.order_pml_2nd;
    vp.flags = fast ? 0 : SFD_EXACT;
    const int nsx0 = nint(p.sx0 / p.dx_v) + 1, nsz0 = nint(p.sz0 / p.dz_v) + 1, nrz0 = nint(p.rz0 / p.dz_v) + 1;
    std::vector<sfd_vti_shot> shots(p.nshot);
    for (int i = 1; i <= p.nshot; i++) {  // VM:158-163
        sfd_vti_shot& s = shots[i - 1];
        s.nsx = nsx0 + nint((float)(i - 1) * p.dsx / p.dx_v);
        s.nsz0 = nsz0;
        s.nrz0 = nrz0;
        s.xmin = s.nsx + nint(p.offset_min / p.dx_v);
        s.xmax = s.nsx + nint(p.offset_max / p.dx_v);
    }
    const int range = shots[0].xmax - shots[0].xmin + 1;
    if (batch <= 0 || batch > p.nshot) batch = p.nshot;
    std::vector<float> rec((size_t)batch * range * p.nt);
    const std::string prefix1 = strip(p.shot1), prefix2 = strip(p.shot2);
    std::vector<std::string> parts;
    for (int b0 = 0; b0 < p.nshot; b0 += batch) {
        const int nb = std::min(batch, p.nshot - b0);
        if ((rc = sfd_vti_forward(&vp, vz.data(), eps.data(), del.data(), nb, shots.data() + b0, device, rec.data(),
                                  nullptr)))
            return fail("sfd_vti_forward", rc);
        for (int k = 0; k < nb; k++) {
            const int i = b0 + k + 1;
            const std::string name = prefix1 + std::to_string(i) + ".su";
            if ((rc = sfd_su_write_ex(name.c_str(), rec.data() + (size_t)k * range * p.nt, range, p.nt, i,
                                      shots[i - 1].nsx, shots[i - 1].xmin, p.dx_v, p.dt, SFD_SU_NO_OFFSET)))
                return fail(name.c_str(), rc);
            parts.push_back(name);
        }
    }
    std::vector<const char*> v;
    for (const auto& s : parts) v.push_back(s.c_str());
    const std::string out = prefix2 + ".su";
    if ((rc = sfd_su_merge(out.c_str(), v.data(), (int)v.size(), keep ? 0 : 1))) return fail(out.c_str(), rc);
    std::printf("vti_forward: %d shots of %d traces x %d samples -> %s\n", p.nshot, range, p.nt, out.c_str());
    return 0;
}
