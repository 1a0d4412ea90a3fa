// The reference programs' file contract: the Q_forward and yang_version parameter cards, binary
// model files and the SU shot records with their merge step.  Used by the afd_fd / q_forward programs and
// exported through the C ABI so that other callers can read and write the same files.
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "sfd_internal.h"

namespace {

// one line without the end-of-line characters (LF or CRLF); false at end of file
bool read_line(FILE* f, std::string* out) {
    out->clear();
    int c;
    bool any = false;
    while ((c = std::fgetc(f)) != EOF) {
        any = true;
        if (c == '\n') break;
        out->push_back((char)c);
    }
    while (!out->empty() && (out->back() == '\r' || out->back() == ' ' || out->back() == '\t')) out->pop_back();
    return any;
}

// list-directed numeric fields of one line: separated by blanks or commas (Fortran `read(u,*)`,
// and the width-less `(F)` / `(I)` edit descriptors of QS:190-222)
std::vector<double> numbers(const std::string& line) {
    std::vector<double> v;
    std::string tok;
    auto flush = [&]() {
        if (tok.empty()) return;
        for (auto& ch : tok)
            if (ch == 'd' || ch == 'D') ch = 'e';  // Fortran double-precision exponent
        char* end = nullptr;
        const double x = std::strtod(tok.c_str(), &end);
        if (end && *end == '\0') v.push_back(x);
        tok.clear();
    };
    for (char ch : line) {
        if (ch == ' ' || ch == '\t' || ch == ',') flush();
        else tok.push_back(ch);
    }
    flush();
    return v;
}

std::string strip(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && (s[a] == ' ' || s[a] == '\t')) a++;
    while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t')) b--;
    return s.substr(a, b - a);
}

void put16(unsigned char* h, int off, int v) {
    const int16_t x = (int16_t)v;
    std::memcpy(h + off, &x, 2);
}
void put32(unsigned char* h, int off, int v) {
    const int32_t x = (int32_t)v;
    std::memcpy(h + off, &x, 4);
}

}  // namespace

extern "C" {

int sfd_qpar_read(const char* path, sfd_qpar* p) {
    if (!path || !p) return SFD_ERR_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return SFD_ERR_IO;
    std::memset(p, 0, sizeof(*p));
    std::string label, line;
    // QS:162-222: nine file names, then the numeric cards, each after one label line
    char* names[9] = {p->vp, p->vs, p->rho, p->qp, p->qs, p->shot1, p->shot2, p->shot3, p->shot4};
    int rc = SFD_OK;
    for (int i = 0; i < 9 && rc == SFD_OK; i++) {
        if (!read_line(f, &label) || !read_line(f, &line)) rc = SFD_ERR_IO;
        else std::snprintf(names[i], sizeof(p->vp), "%s", strip(line).c_str());
    }
    struct Card {
        int n;
        double* d[4];
    };
    double nshot, omin, omax, sx0, sz0, rz0, dsx, nx, nz, dx, dz, nt, dt, f0, pxn, pxp, pzn, pzp, fdo2, fdo1;
    const Card cards[] = {{1, {&nshot}}, {2, {&omin, &omax}}, {3, {&sx0, &sz0, &rz0}}, {1, {&dsx}},
                          {2, {&nx, &nz}}, {2, {&dx, &dz}},     {1, {&nt}},             {1, {&dt}},
                          {1, {&f0}},    {2, {&pxn, &pxp}},    {2, {&pzn, &pzp}},      {1, {&fdo2}},
                          {1, {&fdo1}}};
    for (const Card& c : cards) {
        if (rc != SFD_OK) break;
        if (!read_line(f, &label) || !read_line(f, &line)) {
            rc = SFD_ERR_IO;
            break;
        }
        const std::vector<double> v = numbers(line);
        if ((int)v.size() < c.n) {
            rc = SFD_ERR_ARG;
            break;
        }
        for (int i = 0; i < c.n; i++) *c.d[i] = v[i];
    }
    std::fclose(f);
    if (rc != SFD_OK) return rc;
    p->nshot = (int)nshot;
    p->offset_min = (float)omin;
    p->offset_max = (float)omax;
    p->sx0 = (float)sx0;
    p->sz0 = (float)sz0;
    p->rz0 = (float)rz0;
    p->dsx = (float)dsx;
    p->nx = (int)nx;
    p->nz = (int)nz;
    p->dx = (float)dx;
    p->dz = (float)dz;
    p->nt = (int)nt;
    p->dt = (float)dt;
    p->f0 = (float)f0;
    p->pml_xn = (float)pxn;
    p->pml_xp = (float)pxp;
    p->pml_zn = (float)pzn;
    p->pml_zp = (float)pzp;
    p->fdo2 = (int)fdo2;
    p->fdo1 = (int)fdo1;
    return SFD_OK;
}

int sfd_vtipar_read(const char* path, sfd_vtipar* p) {
    if (!path || !p) return SFD_ERR_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return SFD_ERR_IO;
    std::memset(p, 0, sizeof(*p));
    std::string label, line;
    // VS:383-392: five file names, then the numeric cards (VS:393-421), each after one label line
    int rc = SFD_OK;
    char* names[5] = {p->vz, p->epsilon, p->delta, p->shot1, p->shot2};
    for (int i = 0; i < 5 && rc == SFD_OK; i++) {
        if (!read_line(f, &label) || !read_line(f, &line)) rc = SFD_ERR_IO;
        else std::snprintf(names[i], sizeof(p->vz), "%s", strip(line).c_str());
    }
    struct Card {
        int n;
        double* d[3];
    };
    double nshot, omin, omax, sx0, sz0, rz0, dsx, nx, nz, dx, dz, nt, dt, f0, bxl, bxr, bzu, bzd, oe, o1, o2;
    const Card cards[] = {{1, {&nshot}}, {2, {&omin, &omax}}, {3, {&sx0, &sz0, &rz0}}, {1, {&dsx}},
                          {2, {&nx, &nz}}, {2, {&dx, &dz}},   {1, {&nt}},             {1, {&dt}},
                          {1, {&f0}},    {2, {&bxl, &bxr}},   {2, {&bzu, &bzd}},      {1, {&oe}},
                          {1, {&o1}},    {1, {&o2}}};
    for (const Card& c : cards) {
        if (rc != SFD_OK) break;
        if (!read_line(f, &label) || !read_line(f, &line)) {
            rc = SFD_ERR_IO;
            break;
        }
        const std::vector<double> v = numbers(line);
        if ((int)v.size() < c.n) {
            rc = SFD_ERR_ARG;
            break;
        }
        for (int i = 0; i < c.n; i++) *c.d[i] = v[i];
    }
    std::fclose(f);
    if (rc != SFD_OK) return rc;
    p->nshot = (int)nshot;
    p->offset_min = (float)omin;
    p->offset_max = (float)omax;
    p->sx0 = (float)sx0;
    p->sz0 = (float)sz0;
    p->rz0 = (float)rz0;
    p->dsx = (float)dsx;
    p->nx_v = (int)nx;
    p->nz_v = (int)nz;
    p->dx_v = (float)dx;
    p->dz_v = (float)dz;
    p->nt = (int)nt;
    p->dt = (float)dt;
    p->f0 = (float)f0;
    p->bound_x_l = (float)bxl;
    p->bound_x_r = (float)bxr;
    p->bound_z_u = (float)bzu;
    p->bound_z_d = (float)bzd;
    p->order_explicit = (int)oe;
    p->order_pml_1st = (int)o1;
    p->order_pml_2nd = (int)o2;
    return SFD_OK;
}

int sfd_isopar_read(const char* path, sfd_isopar* p) {
    if (!path || !p) return SFD_ERR_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return SFD_ERR_IO;
    std::memset(p, 0, sizeof(*p));
    std::string label, line;
    // YPUB:94-115: the mode, ten file names, then the numeric cards, each after one label line
    int rc = SFD_OK;
    if (!read_line(f, &label) || !read_line(f, &line)) rc = SFD_ERR_IO;
    else std::snprintf(p->molmod, sizeof(p->molmod), "%s", strip(line).c_str());
    char* names[10] = {p->vp, p->vs, p->rho, p->topo, p->snapx, p->snapz, p->shot1, p->shot2, p->shot3, p->shot4};
    for (int i = 0; i < 10 && rc == SFD_OK; i++) {
        if (!read_line(f, &label) || !read_line(f, &line)) rc = SFD_ERR_IO;
        else std::snprintf(names[i], sizeof(p->vp), "%s", strip(line).c_str());
    }
    struct Card {
        int n;
        double* d[3];
    };
    double nshot, omin, omax, sx0, sz0, rz0, dsx, nx, nz, dx, dz, nt, dt, dtsnap, f0, decay, pxn, pxp, pzn, pzp, rgau;
    // YPUB:116-141
    const Card cards[] = {{1, {&nshot}},      {2, {&omin, &omax}}, {3, {&sx0, &sz0, &rz0}}, {1, {&dsx}},
                          {2, {&nx, &nz}},    {2, {&dx, &dz}},     {1, {&nt}},             {2, {&dt, &dtsnap}},
                          {1, {&f0}},         {1, {&decay}},       {2, {&pxn, &pxp}},      {2, {&pzn, &pzp}},
                          {1, {&rgau}}};
    for (const Card& c : cards) {
        if (rc != SFD_OK) break;
        if (!read_line(f, &label) || !read_line(f, &line)) {
            rc = SFD_ERR_IO;
            break;
        }
        const std::vector<double> v = numbers(line);
        if ((int)v.size() < c.n) {
            rc = SFD_ERR_ARG;
            break;
        }
        for (int i = 0; i < c.n; i++) *c.d[i] = v[i];
    }
    std::fclose(f);
    if (rc != SFD_OK) return rc;
    p->nshot = (int)nshot;
    p->offset_min = (float)omin;
    p->offset_max = (float)omax;
    p->sx0 = (float)sx0;
    p->sz0 = (float)sz0;
    p->rz0 = (float)rz0;
    p->dsx = (float)dsx;
    p->nx = (int)nx;
    p->nz = (int)nz;
    p->dx = (float)dx;
    p->dz = (float)dz;
    p->nt = (int)nt;
    p->dt = (float)dt;
    p->dtsnap = (float)dtsnap;
    p->f0 = (float)f0;
    p->decay = (float)decay;
    p->pml_xn = (float)pxn;
    p->pml_xp = (float)pxp;
    p->pml_zn = (float)pzn;
    p->pml_zp = (float)pzp;
    p->rgau = (int)rgau;
    return SFD_OK;
}

int sfd_read_floats(const char* path, long long n, float* out) {
    if (!path || !out || n < 0) return SFD_ERR_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return SFD_ERR_IO;
    const size_t got = std::fread(out, sizeof(float), (size_t)n, f);
    std::fclose(f);
    return got == (size_t)n ? SFD_OK : SFD_ERR_IO;
}

int sfd_write_floats(const char* path, const float* data, long long n, int append) {
    if (!path || (!data && n > 0) || n < 0) return SFD_ERR_ARG;
    FILE* f = std::fopen(path, append ? "ab" : "wb");
    if (!f) return SFD_ERR_IO;
    const size_t put = n > 0 ? std::fwrite(data, sizeof(float), (size_t)n, f) : 0;
    const int rc = std::fclose(f);
    return (put == (size_t)n && rc == 0) ? SFD_OK : SFD_ERR_IO;
}

int sfd_su_write(const char* path, const float* traces, int ntr, int nt, int shot_no, int isx, int ixmin, float dx,
                 float dt) {
    return sfd_su_write_ex(path, traces, ntr, nt, shot_no, isx, ixmin, dx, dt, SFD_SU_CDP);
}

int sfd_su_write_ex(const char* path, const float* traces, int ntr, int nt, int shot_no, int isx, int ixmin, float dx,
                    float dt, int flags) {
    if (!path || (!traces && ntr > 0) || ntr < 0 || nt < 1 || nt > 32767 || !(dx > 0) || !(dt > 0))
        return SFD_ERR_ARG;
    FILE* f = std::fopen(path, "wb");
    if (!f) return SFD_ERR_IO;
    // QS:1502-1545.  Header arithmetic follows the Fortran: real(4) products, conversion to
    // integer by truncation on assignment, nint for the cdp.
    unsigned char h[240];
    std::memset(h, 0, sizeof(h));
    const int sx = (int)((float)(isx - 1) * dx);
    put32(h, 8, shot_no);                       // fldr
    put16(h, 28, 1);                            // trid
    put32(h, 72, sx);                           // sx
    put16(h, 114, nt);                          // ns
    put16(h, 116, (int)(dt * 1.0E6f));          // dt in microseconds
    int rc = SFD_OK;
    for (int i = 1; i <= ntr && rc == SFD_OK; i++) {
        const int gx = (int)((float)(ixmin - 1 + i - 1) * dx);
        put32(h, 80, gx);                                            // gx
        if (!(flags & SFD_SU_NO_OFFSET)) put32(h, 36, gx - sx);      // offset
        if (flags & SFD_SU_CDP) put32(h, 20, (int)std::lround((float)(gx + sx) / dx) + 1);  // cdp
        if (std::fwrite(h, 1, 240, f) != 240 ||
            std::fwrite(traces + (size_t)(i - 1) * nt, sizeof(float), (size_t)nt, f) != (size_t)nt)
            rc = SFD_ERR_IO;
    }
    if (std::fclose(f) != 0) rc = SFD_ERR_IO;
    return rc;
}

int sfd_su_merge(const char* out_path, const char* const* in_paths, int n, int delete_inputs) {
    if (!out_path || n < 0 || (n > 0 && !in_paths)) return SFD_ERR_ARG;
    FILE* o = std::fopen(out_path, "wb");
    if (!o) return SFD_ERR_IO;
    std::vector<unsigned char> buf(1 << 20);
    int rc = SFD_OK;
    for (int i = 0; i < n && rc == SFD_OK; i++) {
        FILE* f = std::fopen(in_paths[i], "rb");
        if (!f) {
            rc = SFD_ERR_IO;
            break;
        }
        size_t got;
        while ((got = std::fread(buf.data(), 1, buf.size(), f)) > 0)
            if (std::fwrite(buf.data(), 1, got, o) != got) {
                rc = SFD_ERR_IO;
                break;
            }
        std::fclose(f);
    }
    if (std::fclose(o) != 0) rc = SFD_ERR_IO;
    if (rc == SFD_OK && delete_inputs)
        for (int i = 0; i < n; i++) std::remove(in_paths[i]);  // QS:1582 close(status='delete')
    return rc;
}

}  // extern "C"
