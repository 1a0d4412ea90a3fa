// Host helpers of the C ABI that need no device: wavelets, sponge, coefficients, padding.
#include <cmath>
#include <cstring>

#include "sfd_internal.h"

extern "C" {

// Staggered first-derivative coefficients: AFD:38-45 (order 16) and the single-precision
// `constant` module of forward/Q_forward/Q_multishot_fd_subroutine_fsbc_zy_rotated.f90:9-28.
int sfd_fd_coeffs(int order, float* c) {
    if (!c) return SFD_ERR_ARG;
    switch (order) {
    case 16: {
        const float v[8] = {1.2340911f, -1.0664985e-1f, 2.3036367e-2f, -5.3423856e-3f,
                            1.0772712e-3f, -1.6641888e-4f, 1.7021711e-5f, -8.5234642e-7f};
        std::memcpy(c, v, sizeof(v));
        return SFD_OK;
    }
    case 10:
        c[0] = 19845.0f / 16384.0f; c[1] = -735.0f / 8192.0f; c[2] = 567.0f / 40960.0f;
        c[3] = -405.0f / 229376.0f; c[4] = 35.0f / 294912.0f;
        return SFD_OK;
    case 8:
        c[0] = 1225.0f / 1024.0f; c[1] = -245.0f / 3072.0f; c[2] = 49.0f / 5120.0f; c[3] = -5.0f / 7168.0f;
        return SFD_OK;
    case 4:
        c[0] = 9.0f / 8.0f; c[1] = -1.0f / 24.0f;
        return SFD_OK;
    case 2:
        c[0] = 1.0f;
        return SFD_OK;
    default:
        return SFD_ERR_ARG;
    }
}

// AFD:164-194.  absorb = 1 - 0.38 q^2 / PML^2 with q the distance index into the sponge,
// evaluated in double and stored as float; x edges overwrite z edges in the corners.
int sfd_afd_sponge(int nx, int nz, int pml, float* a) {
    if (!a || nx <= 0 || nz <= 0 || pml < 0 || 2 * pml > nx || 2 * pml > nz) return SFD_ERR_ARG;
    for (int i = 0; i < nx * nz; i++) a[i] = 1.0f;
    for (int i = pml; i < nx - pml; i++)
        for (int j = 0; j < pml; j++) a[i * nz + j] = -0.38 * (pml - j - 1) * (pml - j - 1) / (1.0 * pml * pml) + 1;
    for (int i = pml; i < nx - pml; i++)
        for (int j = nz - pml; j < nz; j++) a[i * nz + j] = -0.38 * (j - nz + pml) * (j - nz + pml) / (1.0 * pml * pml) + 1;
    for (int i = 0; i < pml; i++)
        for (int j = 0; j < nz; j++) a[i * nz + j] = -0.38 * (pml - i - 1) * (pml - i - 1) / (1.0 * pml * pml) + 1;
    for (int i = nx - pml; i < nx; i++)
        for (int j = 0; j < nz; j++) a[i * nz + j] = -0.38 * (i - nx + pml) * (i - nx + pml) / (1.0 * pml * pml) + 1;
    return SFD_OK;
}

int sfd_wavelet(int convention, int nt, float dt, float f0, int delay, float* out) {
    if (!out || nt < 0 || !(f0 > 0.0f)) return SFD_ERR_ARG;
    if (convention == SFD_WAVELET_AFD) {
        // AFD:199-209 (PI = 3.1415926, AFD:13; t and t1 are float)
        const double PI = 3.1415926;
        const float freq = f0;
        for (int i = 0; i < nt; i++) {
            const float t = dt * i;
            const float t1 = 1.0 / freq;
            out[i] = 50 * (1 - 2 * PI * PI * freq * freq * (t - t1) * (t - t1)) *
                     std::exp(-PI * PI * freq * freq * (t - t1) * (t - t1));
        }
        return SFD_OK;
    }
    if (convention == SFD_WAVELET_RIC) {
        // tools/ricker.cpp:44 (pi = 3.1415926, f0 an int, arithmetic in double)
        const double pi = 3.1415926;
        const int fi = (int)f0;
        for (int j = 0; j < nt; j++) {
            const double a = pi * fi * (j - delay) * dt;
            out[j] = (1 - 2 * a * a) * std::exp(-a * a);
        }
        return SFD_OK;
    }
    if (convention == SFD_WAVELET_Q) {
        // QS:1376, Fortran default reals: it*dt - 1.2/f0 in single precision, it = 1..nt
        const float pi = 3.1415926f;
        for (int j = 0; j < nt; j++) {
            const float b = pi * f0 * ((float)(j + 1) * dt - 1.2f / f0);
            out[j] = std::exp(-(b * b)) * (1.0f - 2.0f * (b * b));
        }
        return SFD_OK;
    }
    if (convention == SFD_WAVELET_ISO) {
        // YPUB:1447-1448, Fortran default reals: it*dt - idecay*dt in single precision, it = 1..nt
        if (delay < 0) return SFD_ERR_ARG;
        const float pi = 3.1415926f;
        for (int j = 0; j < nt; j++) {
            const float b = pi * f0 * ((float)(j + 1) * dt - (float)delay * dt);
            out[j] = std::exp(-(b * b)) * (1.0f - 2.0f * (b * b));
        }
        return SFD_OK;
    }
    return SFD_ERR_ARG;
}

// Edge-replicated padding, QS:340-372 (top/bottom rows first, then left/right columns).
int sfd_pad_model(const float* in, int nx, int nz, int pxn, int pxp, int pzn, int pzp, float* out) {
    if (!in || !out || nx <= 0 || nz <= 0 || pxn < 0 || pxp < 0 || pzn < 0 || pzp < 0) return SFD_ERR_ARG;
    const int NX = nx + pxn + pxp, NZ = nz + pzn + pzp;
    for (int i = 0; i < NX; i++) {
        int si = i - pxn;
        si = si < 0 ? 0 : (si >= nx ? nx - 1 : si);
        for (int k = 0; k < NZ; k++) {
            int sk = k - pzn;
            sk = sk < 0 ? 0 : (sk >= nz ? nz - 1 : sk);
            out[(size_t)i * NZ + k] = in[(size_t)si * nz + sk];
        }
    }
    return SFD_OK;
}

}  // extern "C"
