// 2-D VTI pseudo-acoustic modelling for sm_100a: the coupled u / q second-order system of
// de-multiple/convolution_srm/vti_qa_2d_c3_demo1 (VS = VTI_multishot_qacoustic_fd_subroutine_c3.f90,
// VM = VTI_multishot_qacoustic_fd_main_c3.f90), every shot of a call in one launch per time step.
//
// Per time step the reference calls extrapolation_one_step_1 (new u from the current u and q,
// VS:432-960) and then extrapolation_one_step_2 (new q from the current u and q, VS:965-1258).
// Neither reads what the other writes -- step 2 takes the current u, not the new one -- so one
// kernel does both.  A CTA stages the current u and q of a 32 x 8 tile with its 5-cell halo in
// shared memory; each thread owns one cell of one shot, forms the stencil sums that both
// subroutines share once, updates the split PML fields of its cell in place and writes the new
// u and q into the slots of the old ones.  All global loads of a thread are issued before the
// tile barrier, and the registers are bounded for five CTAs per SM (the kernel is bound by the
// latency of those loads and of the IEEE divisions the reference order requires).  The
// operation order is the reference's as written, every multiply, add and divide rounded
// separately (__fmul_rn, __fadd_rn, __fdiv_rn, __fsqrt_rn), so the records equal the FP32
// restatement in oracle/vti_oracle.cpp bit for bit.  A one-thread-per-shot kernel adds the source
// to the current u before each step (VM:420-424, 468-472); the receiver row is written by the
// step kernel's threads on that row.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "seisfd.h"

namespace {

constexpr int kBX = 32, kBZ = 8;             // threads per CTA (x, z)
constexpr int kTX = 32, kH = 5;               // cells per CTA tile in x, stencil halo
constexpr int kSX = kTX + 2 * kH;
// One cell per thread and registers bounded for five CTAs per SM.  Measured on the .par geometry
// (64 shots of 348 x 698): 1, 2 and 4 cells per thread 36.9, 35.3 and 28.6 Gpts/s at four CTAs per
// SM; one cell at five and six CTAs per SM 39.3 and 39.2 Gpts/s (the latter spills).
constexpr int kCPT = 1, kMinBlocks = 5;

// E = true: every operation rounded separately in the reference's order (bit-exact with the
// restatement); E = false: multiplies and adds may contract into FMAs and divisions are the
// approximate __fdividef (records within relative L2 1e-5 of the restatement)
template <bool E> __device__ __forceinline__ float fm(float a, float b) { return E ? __fmul_rn(a, b) : a * b; }
template <bool E> __device__ __forceinline__ float fa(float a, float b) { return E ? __fadd_rn(a, b) : a + b; }
template <bool E> __device__ __forceinline__ float fs(float a, float b) { return E ? __fsub_rn(a, b) : a - b; }
template <bool E> __device__ __forceinline__ float fd(float a, float b) { return E ? __fdiv_rn(a, b) : __fdividef(a, b); }
template <bool E> __device__ __forceinline__ float fsq(float a) { return E ? __fsqrt_rn(a) : sqrtf(a); }

struct VtiDev {
    // per shot: fields u[2], q[2] (pitch x (nz + 10), cell (i, j) 1-based at (j+4)*pitch + i+4),
    // model vz, eps, delta in the same layout, x-strip PML fields (nxl+nxr) x nz of u (4 pairs)
    // and q (3 pairs), z-strip PML fields nx x (nzu+nzd) of u (4 pairs)
    float* base;
    long long field, shot_stride;  // floats per field slab, per shot
    long long xs, zs;              // floats per x strip, per z strip
    int pitch, nx, nz, nxl, nxr, nzu, nzd, range, nt;
    float dx, dz, dt, L;
    float cE[5], c1[5];    // coefficient_2nd(10) (fd_coe and fd_coe_pml_2nd alike), coefficient_1st
    const int* src;        // per shot: source cell i, j
    const int* rrow;       // per shot: receiver row and whether it is the row-6 fallback
    float* records;        // [shot][range][nt]
};

// one shot's arrays, by arithmetic on VtiDev::base (no pointer tables: the slot indices are
// run-time values)
struct VtiSlab {
    float* p;
    long long field, xs, zs;
    __device__ float* u(int b) const { return p + b * field; }
    __device__ float* q(int b) const { return p + (2 + b) * field; }
    __device__ const float* vz() const { return p + 4 * field; }
    __device__ const float* ep() const { return p + 5 * field; }
    __device__ const float* de() const { return p + 6 * field; }
    __device__ float* ux(int k, int b) const { return p + 7 * field + (2 * k + b) * xs; }
    __device__ float* qx(int k, int b) const { return p + 7 * field + (8 + 2 * k + b) * xs; }
    __device__ float* uz(int k, int b) const { return p + 7 * field + 14 * xs + (2 * k + b) * zs; }
};

__device__ __forceinline__ VtiSlab slab(const VtiDev& a, int s) {
    return VtiSlab{a.base + (long long)s * a.shot_stride, a.field, a.xs, a.zs};
}

// second-derivative sum of VS:511-525: (c1 (f+1 + f-1 - 2 f0) + ... + c5 (...)) / h**2
template <bool E>
__device__ __forceinline__ float d2(const float* f, int c, int st, const float* cf, float h) {
    const float two_f0 = fm<E>(2.0f, f[c]);
    float s = fm<E>(cf[0], fs<E>(fa<E>(f[c + st], f[c - st]), two_f0));
#pragma unroll
    for (int m = 2; m <= 5; m++) s = fa<E>(s, fm<E>(cf[m - 1], fs<E>(fa<E>(f[c + m * st], f[c - m * st]), two_f0)));
    return fd<E>(s, fm<E>(h, h));
}
// first-derivative sum of VS:567-578: (p1 (f+1 - f-1) + ... + p5 (...)) / h
template <bool E>
__device__ __forceinline__ float d1(const float* f, int c, int st, const float* cf, float h) {
    float s = fm<E>(cf[0], fs<E>(f[c + st], f[c - st]));
#pragma unroll
    for (int m = 2; m <= 5; m++) s = fa<E>(s, fm<E>(cf[m - 1], fs<E>(f[c + m * st], f[c - m * st])));
    return fd<E>(s, h);
}

// the split PML recurrences of one boundary cell (VS:651-663, 840-858): a1 (second-derivative
// part), t2 (first-derivative part with the damping derivative), a2; k2s2 = speed^2 dt^2 (s2 h^2)
// and k2dd = speed^2 dt^2 dd (s1 h), both formed by the caller in the reference's order
template <bool E>
__device__ __forceinline__ void pml_cell(float d, float dt, float h, float* a1, const float* a1o, float* t2,
                                         const float* t2o, float* a2, const float* a2o, long long x, float k2s2,
                                         float k2dd) {
    const float h2 = fm<E>(h, h);
    const float d2dt = fm<E>(fm<E>(2.0f, d), dt);
    const float P = fs<E>(fa<E>(fm<E>(2.0f, h2), fm<E>(d2dt, h2)), fm<E>(fm<E>(fm<E>(d, d), h2), fm<E>(dt, dt)));
    const float Den = fa<E>(h2, fm<E>(d2dt, h2));
    const float n1 = fd<E>(fa<E>(fs<E>(fm<E>(a1o[x], P), fm<E>(h2, a1[x])), k2s2), Den);
    const float P2 = fs<E>(fa<E>(fm<E>(2.0f, h), fm<E>(d2dt, h)), fm<E>(fm<E>(fm<E>(dt, dt), h), fm<E>(d, d)));
    const float Den2 = fa<E>(h, fm<E>(d2dt, h));
    const float nt = fd<E>(fs<E>(fs<E>(fm<E>(t2o[x], P2), fm<E>(h, t2[x])), k2dd), Den2);
    a1[x] = n1;
    t2[x] = nt;
    a2[x] = fa<E>(fm<E>(a2o[x], fs<E>(1.0f, fm<E>(d, dt))), fm<E>(nt, dt));
}

__global__ void vti_inject_kernel(VtiDev a, int cu, float w) {
    const int s = blockIdx.x;
    if (threadIdx.x != 0) return;
    const VtiSlab p = slab(a, s);
    const long long c = (long long)(a.src[2 * s + 1] + 4) * a.pitch + (a.src[2 * s] + 4);
    p.u(cu)[c] = __fadd_rn(p.u(cu)[c], w);
}

// one cell (i, j) of shot s: U and Q are the shared-memory tiles of the current u and q, sc the
// cell's tile index, P the tile's row stride; c indexes the cell in the field layout
// (v, de, ep: the cell's model; uo, qo: its old u and q, loaded by the caller ahead of time)
template <bool E>
__device__ __forceinline__ void vti_cell(const VtiDev& a, const VtiSlab& p, const float* U, const float* Q, int sc,
                                         int P, int i, int j, int s, int cu, int iit, float v, float de, float ep,
                                         float uo, float qo) {
    const int ou = 1 - cu;
    const int c = sc;
    const long long g = (long long)(j + 4) * a.pitch + (i + 4);
    const float dt = a.dt, dx = a.dx, dz = a.dz, L = a.L;
    const int nx = a.nx, nz = a.nz, nxl = a.nxl, nxr = a.nxr, nzu = a.nzu, nzd = a.nzd;
    const bool xin = i > nxl && i < nx - nxr + 1;
    float un, qn;

    // The sums of the current u and q that both subroutines form: coefficient_2nd(10) is both
    // fd_coe and fd_coe_pml_2nd, the x sums of u and q appear in step 1 and step 2 (added in the
    // other order there, which IEEE addition does not distinguish), the z sum of u in every
    // region of step 1.  Each is formed once.
    const float sxu = d2<E>(U, c, 1, a.cE, dx), sxq = d2<E>(Q, c, 1, a.cE, dx), szu = d2<E>(U, c, P, a.cE, dz);

    // ---- extrapolation_one_step_1 (VS:432-960): new u; step 2's PML cells share its terms ----
    if (xin && j > nzu && j < nz - nzd + 1) {
        un = fa<E>(fs<E>(fm<E>(2.0f, U[c]), uo), fm<E>(fm<E>(fm<E>(dt, dt), fm<E>(v, v)), fa<E>(fm<E>(fa<E>(1.0f, fm<E>(2.0f, de)), fa<E>(sxu, sxq)), szu)));
    } else if (!xin) {
        const bool left = i <= nxl;
        const float vn = fm<E>(v, fsq<E>(fa<E>(1.0f, fm<E>(2.0f, de))));
        const float vx = fm<E>(v, fsq<E>(fa<E>(1.0f, fm<E>(2.0f, ep))));
        const float s1 = fa<E>(d1<E>(U, c, 1, a.c1, dx), d1<E>(Q, c, 1, a.c1, dx));
        const float s2 = fa<E>(sxu, sxq);
        const float axis = fm<E>((float)(left ? i - (nxl + 1) : i - (nx - nxr)), dx);
        const float thick = fm<E>((float)(left ? nxl : nxr), dx);
        const int is = left ? i : i - (nx - nxr) + nxl;
        const float A = fd<E>(fm<E>(3.0f, vx), fm<E>(2.0f, thick));
        const float d = fm<E>(fm<E>(A, fm<E>(fd<E>(axis, thick), fd<E>(axis, thick))), L);
        const float dd = fm<E>(fm<E>(A, fd<E>(fm<E>(2.0f, axis), fm<E>(thick, thick))), L);
        const long long x = (long long)(j - 1) * (nxl + nxr) + (is - 1);
        const float k2 = fm<E>(fm<E>(vn, vn), fm<E>(dt, dt));
        pml_cell<E>(d, dt, dx, p.ux(0, ou), p.ux(0, cu), p.ux(2, ou), p.ux(2, cu), p.ux(1, ou), p.ux(1, cu), x,
                 fm<E>(k2, fm<E>(s2, fm<E>(dx, dx))), fm<E>(fm<E>(k2, dd), fm<E>(s1, dx)));
        float* a3 = p.ux(3, ou);
        const float* a3o = p.ux(3, cu);
        const float n3 = fa<E>(fs<E>(fm<E>(2.0f, a3o[x]), a3[x]), fd<E>(fm<E>(fm<E>(fm<E>(v, v), fm<E>(dt, dt)), fm<E>(szu, fm<E>(dz, dz))), fm<E>(dz, dz)));
        a3[x] = n3;
        un = fa<E>(fa<E>(p.ux(0, ou)[x], p.ux(1, ou)[x]), n3);
        // extrapolation_one_step_2's PML cell (VS:1073-1150): the same s1, s2, d and dd
        const float kq = fm<E>(fs<E>(fm<E>(vx, vx), fm<E>(vn, vn)), fm<E>(dt, dt));
        pml_cell<E>(d, dt, dx, p.qx(0, ou), p.qx(0, cu), p.qx(2, ou), p.qx(2, cu), p.qx(1, ou), p.qx(1, cu), x,
                 fm<E>(kq, fm<E>(s2, fm<E>(dx, dx))), fm<E>(fm<E>(kq, dd), fm<E>(s1, dx)));
        qn = fa<E>(p.qx(0, ou)[x], p.qx(1, ou)[x]);
    } else {
        const bool top = j <= nzu;
        const float vn = fm<E>(v, fsq<E>(fa<E>(1.0f, fm<E>(2.0f, de))));
        const float sz1 = d1<E>(U, c, P, a.c1, dx);  // divided by dx as written (VS:796, 880)
        const float axis = fm<E>((float)(top ? j - (nzu + 1) : j - (nz - nzd)), dz);
        const float thick = fm<E>((float)(top ? nzu : nzd), dz);
        const int js = top ? j : j - (nz - nzd) + nzu;
        const float A = fd<E>(fm<E>(3.0f, v), fm<E>(2.0f, thick));
        const float d = fm<E>(fm<E>(A, fm<E>(fd<E>(axis, thick), fd<E>(axis, thick))), L);
        const float dd = fm<E>(fm<E>(A, fd<E>(fm<E>(2.0f, axis), fm<E>(thick, thick))), L);
        const long long z = (long long)(js - 1) * nx + (i - 1);
        const float k2 = fm<E>(fm<E>(v, v), fm<E>(dt, dt));
        pml_cell<E>(d, dt, dz, p.uz(0, ou), p.uz(0, cu), p.uz(2, ou), p.uz(2, cu), p.uz(1, ou), p.uz(1, cu), z,
                 fm<E>(k2, fm<E>(szu, fm<E>(dz, dz))), fm<E>(fm<E>(k2, dd), fm<E>(sz1, dz)));
        float* a3 = p.uz(3, ou);
        const float* a3o = p.uz(3, cu);
        const float n3 = fa<E>(fs<E>(fm<E>(2.0f, a3o[z]), a3[z]), fm<E>(fm<E>(fm<E>(vn, vn), fm<E>(dt, dt)), fa<E>(sxu, sxq)));
        a3[z] = n3;
        un = fa<E>(fa<E>(p.uz(0, ou)[z], p.uz(1, ou)[z]), n3);
    }

    // ---- extrapolation_one_step_2 (VS:965-1072): new q inside, from the current u ----
    if (xin)
        qn = fa<E>(fs<E>(fm<E>(2.0f, Q[c]), qo), fm<E>(fm<E>(fm<E>(dt, dt), fm<E>(v, v)), fm<E>(fm<E>(2.0f, fs<E>(ep, de)), fa<E>(sxq, sxu))));
    p.u(ou)[g] = un;
    p.q(ou)[g] = qn;

    // ---- recording (VM:446-453, 494-501): new u on the receiver row ----
    const int rr = a.rrow[2 * s], low = a.rrow[2 * s + 1];
    if (j == rr && i > nxl && i <= nxl + a.range && iit <= a.nt && ((!low && iit >= 1) || (low && iit > 1)))
        a.records[((long long)s * a.range + (i - nxl - 1)) * a.nt + (iit - 1)] = un;
}

// Tiles of 32 x (8 CPT) cells per CTA (32 x 8 threads, CPT cells per thread): the current u and
// q of the tile and its 5-cell halo are staged in shared memory once, every stencil reads them
// there.
template <int CPT, int MINB, bool E>
__global__ void __launch_bounds__(kBX * kBZ, MINB) vti_step_kernel(VtiDev a, int cu, int iit) {
    constexpr int kTZ = kBZ * CPT, kSZ = kTZ + 2 * kH;
    __shared__ float sU[kSX * kSZ], sQ[kSX * kSZ];
    const int s = blockIdx.z, tx = threadIdx.x, ty = threadIdx.y, tid = ty * kBX + tx;
    const int i0 = blockIdx.x * kTX + 1, j0 = blockIdx.y * kTZ + 1;
    const VtiSlab p = slab(a, s);
    const float* U = p.u(cu);
    const float* Q = p.q(cu);
    // tile cell (lx, lz) is field cell (i0 - 5 + lx, j0 - 5 + lz), array column i + 4 >= 0 and row
    // j + 4 >= 0; columns past the pitch and rows past nz + 5 (only reached by the tile's own cells
    // beyond the grid, which store nothing) read as zero.  All of the thread's global loads -- its
    // share of the tiles and its cells' model and old u, q -- are issued before the first use.
    constexpr int NE = kSX * kSZ, IT = (NE + kBX * kBZ - 1) / (kBX * kBZ);
    float ru[IT], rq[IT];
#pragma unroll
    for (int t = 0; t < IT; t++) {
        const int e = tid + t * kBX * kBZ;
        const int lz = e / kSX, lx = e - lz * kSX;
        const int gi = i0 - kH + lx + 4, gj = j0 - kH + lz + 4;
        ru[t] = 0.0f;
        rq[t] = 0.0f;
        if (e < NE && gi < a.pitch && gj < a.nz + 10) {
            const long long gg = (long long)gj * a.pitch + gi;
            ru[t] = U[gg];
            rq[t] = Q[gg];
        }
    }
    const int i = i0 + tx, ou = 1 - cu;
    float mv[CPT], md[CPT], me[CPT], mu[CPT], mq[CPT];
#pragma unroll
    for (int k = 0; k < CPT; k++) {
        const int j = j0 + ty + kBZ * k;
        mv[k] = md[k] = me[k] = mu[k] = mq[k] = 0.0f;
        if (i <= a.nx && j <= a.nz) {
            const long long g = (long long)(j + 4) * a.pitch + (i + 4);
            mv[k] = p.vz()[g];
            md[k] = p.de()[g];
            me[k] = p.ep()[g];
            mu[k] = p.u(ou)[g];
            mq[k] = p.q(ou)[g];
        }
    }
#pragma unroll
    for (int t = 0; t < IT; t++) {
        const int e = tid + t * kBX * kBZ;
        if (e < NE) {
            sU[e] = ru[t];
            sQ[e] = rq[t];
        }
    }
    __syncthreads();
    if (i > a.nx) return;
#pragma unroll
    for (int k = 0; k < CPT; k++) {
        const int lz = ty + kBZ * k, j = j0 + lz;
        if (j > a.nz) break;
        vti_cell<E>(a, p, sU, sQ, (lz + kH) * kSX + tx + kH, kSX, i, j, s, cu, iit, mv[k], md[k], me[k], mu[k], mq[k]);
    }
}

// coefficient_2nd / coefficient_1st (VS:1264-1472): a(i,j) = i^p / p! (p = 2j or 2j-1) inverted
// by successive Sherman-Morrison updates of the identity; coefficient(i) = 0.5 inv(a)(1, i)
int coefficients(int order, int first, float* out) {
    const int k = first ? (order + 1) / 2 : order / 2;
    if (k < 1 || k > 8) return SFD_ERR_ARG;
    float a[64], inv[64], temp[8], col[8], outer[64], upd[64];
    for (int i = 1; i <= k; i++)
        for (int j = 1; j <= k; j++) {
            const int pw = first ? 2 * j - 1 : 2 * j;
            float num = 1.0f, fact = 1.0f;
            for (int m = 0; m < pw; m++) num = num * (float)i;
            for (int m = 1; m <= pw; m++) fact = fact * (float)m;
            a[(i - 1) * k + (j - 1)] = num / fact;
        }
    for (int q = 0; q < k * k; q++) inv[q] = 0.0f;
    for (int d = 0; d < k; d++) inv[d * k + d] = 1.0f;
    for (int i = 0; i < k; i++) {
        for (int c = 0; c < k; c++) temp[c] = a[i * k + c];
        temp[i] = temp[i] - 1.0f;
        float den = 0.0f;
        for (int r = 0; r < k; r++) den = den + temp[r] * inv[r * k + i];
        den = den + 1.0f;
        for (int r = 0; r < k; r++) col[r] = inv[r * k + i];
        for (int r = 0; r < k; r++)
            for (int c = 0; c < k; c++) outer[r * k + c] = col[r] * temp[c];
        for (int r = 0; r < k; r++)
            for (int c = 0; c < k; c++) {
                float s = 0.0f;
                for (int m = 0; m < k; m++) s = s + outer[r * k + m] * inv[m * k + c];
                upd[r * k + c] = s / den;
            }
        for (int q = 0; q < k * k; q++) inv[q] = inv[q] - upd[q];
    }
    for (int i = 0; i < k; i++) {
        float s = 0.0f;
        for (int m = 0; m < k; m++) s = s + inv[m] * (m == i ? 0.5f : 0.0f);
        out[i] = s;
    }
    return SFD_OK;
}

template <class T>
struct DevBuf {
    T* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, std::max<size_t>(1, n) * sizeof(T)); }
};

}  // namespace

extern "C" {

int sfd_vti_coefficients(int order, int first, float* out) {
    if (!out) return SFD_ERR_ARG;
    return coefficients(order, first, out);
}

int sfd_vti_forward(const sfd_vti_par* par, const float* vz, const float* epsilon, const float* delta, int nshot,
                    const sfd_vti_shot* shots, int device, float* records, sfd_timing* timing) {
    const auto t_start = std::chrono::steady_clock::now();
    if (!par || !vz || !epsilon || !delta || !shots || !records || nshot < 1) return SFD_ERR_ARG;
    const sfd_vti_par& c = *par;
    if (c.nx_v < 1 || c.nz_v < 1 || c.nt < 1 || !(c.dx > 0) || !(c.dz > 0) || !(c.dt > 0)) return SFD_ERR_ARG;
    if (c.order_explicit != 10 || c.order_pml_2nd != 10 || (c.order_pml_1st != 9 && c.order_pml_1st != 10))
        return SFD_ERR_UNSUPPORTED;  // the stencils are written out with five coefficients (VS:511-551)
    if (c.nx_bound_l < 0 || c.nz_bound_u < 0 || c.nx_bound_r < 2 || c.nz_bound_d < 2) return SFD_ERR_ARG;
    const int range = shots[0].xmax - shots[0].xmin + 1;
    if (range < 1) return SFD_ERR_ARG;
    for (int s = 0; s < nshot; s++)
        if (shots[s].xmax - shots[s].xmin + 1 != range) return SFD_ERR_ARG;  // one grid for the batch
    const int nxl = c.nx_bound_l, nxr = c.nx_bound_r, nzu = c.nz_bound_u, nzd = c.nz_bound_d;
    const int nx = range + nxl + nxr - 2, nz = c.nz_v + nzu + nzd - 2;  // VM:248-249
    if (nx <= 10 || nz <= 10) return SFD_ERR_ARG;

    VtiDev a{};
    a.nx = nx; a.nz = nz; a.nxl = nxl; a.nxr = nxr; a.nzu = nzu; a.nzd = nzd; a.range = range; a.nt = c.nt;
    a.dx = c.dx; a.dz = c.dz; a.dt = c.dt;
    a.L = std::log(1.0f / 1.0e-3f);  // log(1/R), R = 1.0E-3 (VS:14)
    if (coefficients(10, 0, a.cE) || coefficients(c.order_pml_1st, 1, a.c1))
        return SFD_ERR_ARG;
    a.pitch = (nx + 10 + 31) / 32 * 32;
    a.field = (long long)a.pitch * (nz + 10);
    a.xs = (long long)(nxl + nxr) * nz;
    a.zs = (long long)nx * (nzu + nzd);
    a.shot_stride = 7 * a.field + 14 * a.xs + 8 * a.zs;
    a.shot_stride = (a.shot_stride + 31) / 32 * 32;

    // per-shot windows (get_currshot_parameters, VS:268-338, and VM:405-408), source cells and
    // receiver rows
    std::vector<float> host((size_t)nshot * 3 * a.field, 0.0f);
    std::vector<int> src(2 * nshot), rrow(2 * nshot);
    for (int s = 0; s < nshot; s++) {
        const sfd_vti_shot& sh = shots[s];
        float* hv = host.data() + (size_t)s * 3 * a.field;
        float* he = hv + a.field;
        float* hd = he + a.field;
        auto C = [&](int i, int j) { return (size_t)(j + 4) * a.pitch + (i + 4); };
        for (int i = 1; i <= range; i++) {
            int io = i + sh.xmin;
            io = io < 1 ? 1 : (io > c.nx_v ? c.nx_v : io);
            for (int j = 1; j <= c.nz_v; j++) {
                const size_t m = (size_t)(io - 1) * c.nz_v + (j - 1);
                hv[C(i + nxl, nzu + j)] = vz[m];
                he[C(i + nxl, nzu + j)] = epsilon[m];
                hd[C(i + nxl, nzu + j)] = delta[m];
            }
        }
        for (int j = 1; j <= nzu; j++)
            for (int i = 1; i <= nx; i++) hv[C(i, j)] = hv[C(i, nzu + 1)];
        for (int j = nzu + c.nz_v + 1; j <= nz; j++)
            for (int i = 1; i <= nx; i++) hv[C(i, j)] = hv[C(i, nzu + c.nz_v)];
        for (int j = 1; j <= nz; j++)
            for (int i = 1; i <= nxl; i++) hv[C(i, j)] = hv[C(nxl + 1, j)];
        for (int j = 1; j <= nz; j++)
            for (int i = nxl + range + 1; i <= nx; i++) hv[C(i, j)] = hv[C(nxl + range, j)];
        for (int j = 1; j <= sh.nsz0 + nzu + 6 && j <= nz; j++)
            for (int i = 1; i <= nx; i++) he[C(i, j)] = hd[C(i, j)] = 0.0f;
        for (int j = 1; j <= nz; j++)
            for (int i = 1; i <= nx; i++)
                if (!(hv[C(i, j)] > 0.0f) || !std::isfinite(hv[C(i, j)]) || !std::isfinite(he[C(i, j)]) ||
                    !std::isfinite(hd[C(i, j)]) || !(1.0f + 2.0f * he[C(i, j)] >= 0.0f) ||
                    !(1.0f + 2.0f * hd[C(i, j)] >= 0.0f))
                    return SFD_ERR_ARG;
        src[2 * s] = sh.nsx - sh.xmin + nxl;  // VS:294-295
        src[2 * s + 1] = sh.nsz0 + nzu;
        if (src[2 * s] < 1 || src[2 * s] > nx || src[2 * s + 1] < 1 || src[2 * s + 1] > nz) return SFD_ERR_ARG;
        const int r = sh.nrz0 + nzu;
        rrow[2 * s] = r >= 6 ? r : 6;
        rrow[2 * s + 1] = r >= 6 ? 0 : 1;
        if (rrow[2 * s] > nz) return SFD_ERR_ARG;
    }

    // source samples (VM:420-424): exp(-(pi f0 (it - 0.07/dt) dt)^2) (1 - 2 (...)^2), it <= nwt
    const int nwt = (int)std::lround((double)((2.0f * 0.07f) / c.dt)) + 1;
    const int half = (int)std::lround((double)(nwt - 1) / 2.0);
    const int NT = c.nt + half;
    std::vector<float> w(nwt + 1, 0.0f);
    for (int it = 1; it <= nwt; it++) {
        const float b = ((3.1415926f * c.f0) * ((float)it - (0.07f / c.dt))) * c.dt;
        w[it] = std::exp(-(b * b)) * (1.0f - 2.0f * (b * b));
    }

    if (cudaSetDevice(device) != cudaSuccess) return SFD_ERR_CUDA;
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return SFD_ERR_CUDA;
    struct StreamGuard { cudaStream_t s; ~StreamGuard() { cudaStreamDestroy(s); } } sg{st};
    DevBuf<float> state, recs;
    DevBuf<int> dsrc, drow;
    const size_t total = (size_t)nshot * a.shot_stride;
    const size_t rec_n = (size_t)nshot * range * c.nt;
    if (state.alloc(total) != cudaSuccess || recs.alloc(rec_n) != cudaSuccess || dsrc.alloc(2 * nshot) != cudaSuccess ||
        drow.alloc(2 * nshot) != cudaSuccess) {
        cudaGetLastError();
        return SFD_ERR_NOMEM;
    }
    long long h2d = 0;
    if (cudaMemsetAsync(state.p, 0, total * sizeof(float), st) != cudaSuccess ||
        cudaMemsetAsync(recs.p, 0, rec_n * sizeof(float), st) != cudaSuccess)
        return SFD_ERR_CUDA;
    for (int s = 0; s < nshot; s++) {
        if (cudaMemcpyAsync(state.p + (size_t)s * a.shot_stride + 4 * a.field, host.data() + (size_t)s * 3 * a.field,
                            3 * a.field * sizeof(float), cudaMemcpyHostToDevice, st) != cudaSuccess)
            return SFD_ERR_CUDA;
        h2d += 3 * a.field * (long long)sizeof(float);
    }
    if (cudaMemcpyAsync(dsrc.p, src.data(), 2 * nshot * sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(drow.p, rrow.data(), 2 * nshot * sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return SFD_ERR_CUDA;
    a.base = state.p; a.src = dsrc.p; a.rrow = drow.p; a.records = recs.p;

    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const bool exact = (c.flags & SFD_EXACT) != 0;
    const int tz = kBZ * kCPT;
    const dim3 grid((nx + kTX - 1) / kTX, (nz + tz - 1) / tz, nshot), block(kBX, kBZ);
    long long launches = 0;
    cudaEventRecord(e0, st);
    for (int it = 1; it <= NT; it++) {
        const int cu = (it % 2 == 1) ? 1 : 0;  // odd steps: u2 / q2 current (VM:417-505)
        if (it <= nwt) {
            vti_inject_kernel<<<nshot, 32, 0, st>>>(a, cu, w[it]);
            launches++;
        }
        if (exact) vti_step_kernel<kCPT, kMinBlocks, true><<<grid, block, 0, st>>>(a, cu, it - half);
        else vti_step_kernel<kCPT, kMinBlocks, false><<<grid, block, 0, st>>>(a, cu, it - half);
        launches++;
    }
    cudaEventRecord(e1, st);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(records, recs.p, rec_n * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    float ms = 0.0f;
    if (err == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err != cudaSuccess) return SFD_ERR_CUDA;
    if (timing) {
        std::memset(timing, 0, sizeof(*timing));
        timing->loop_ms = ms;
        timing->device_ms = ms;
        timing->total_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
        timing->point_updates = (double)nx * nz * NT * nshot;
        timing->launches = launches;
        timing->h2d_bytes = h2d;
        timing->d2h_bytes = (long long)(rec_n * sizeof(float));
        timing->graph = 0;
        timing->kernel_variant = exact ? 71 : 70;
    }
    return SFD_OK;
}

}  // extern "C"
