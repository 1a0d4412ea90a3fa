// Isotropic elastic (P-SV) standard-staggered-grid time step, 10th order: the two modes of
// forward/yang_version_2016_2_2 for a flat surface -- 'abc' (YPRI:234-386, cosine sponge on all
// four sides) and 'fsbc' (YPRI:57-230, free surface at row zs, no top sponge).  Every field is kept in the reference's split form (x and z parts), ten per cell:
//   vxx vxz vzx vzz | strxxx strxxz | strzzx strzzz | strxzx strxzz
// and one step is two kernels (YPUB = Iso_multishot_fd_subroutine_fsbc_zy_m2_pub.f90):
//   velocity: strxx, strxz, strzz = sums of their parts (YPUB:1410-1426) on the tile plus halo;
//             vxx += (dt/dx) busg2e Dx0 strxx, vxz += (dt/dz) busg2e Dz0 strxz,
//             vzx += (dt/dx) busg1e Dx1 strxz, vzz += (dt/dz) busg1e Dz1 strzz
//             (caluxabs / caluzabs, YPUB:1095-1157, 1347-1407), each part times its sponge
//   stress:   vx = vxx + vxz, vz = vzx + vzz on the tile plus halo;
//             strxxx += (dt/dx) lambmusg Dx1 vx, strxxz += (dt/dz) lambsg Dz0 vz,
//             strzzx += (dt/dx) lambsg Dx1 vx,   strzzz += (dt/dz) lambmusg Dz0 vz,
//             strxzx += (dt/dx) musge Dx0 vz,    strxzz += (dt/dz) musge Dz1 vx,
//             each part times its sponge, the Gaussian source added to strxxx and strzzx after
//             their sponge (YPRI:331-359, YPUB:1429-1466); records vx, vz at the receivers
// Dx0 u(i) = sum_m a_m (u(i+m) - u(i-1-m)), Dx1 u(i) = sum_m a_m (u(i+1+m) - u(i-m)), m = 0..4.
// Every multiply and add is rounded separately in the reference's order, so the kernels agree
// bit for bit with the FP32 restatement in oracle/iso_oracle.cpp.
//
// The surface row is per column: itopo(x) (1-based, the reference's itopoe), from a topography or
// flat.  abc mode updates the rows from t0 = itopo - npz - 1 (0-based) down, with the top sponge
// on rows t0 .. t0 + npz taking spgzn(z - t0 + 1) (YPUB:851-897); a flat surface has t0 = -1.
// Free surface (fsbc, zs = itopo - 1): rows above zs keep their values; the z derivatives of the five rows from
// zs down drop to 8th, 6th, 4th and 2nd order (YPUB:1160-1343); left and right sponges act from
// zs down, the bottom sponge everywhere, no top sponge (YPUB:901-934); strzz parts are zero on
// rows <= zs after their sponge and before the source (YPUB:978-1007), which enters strxx only for
// sources below the surface (YPRI:163-168).  After the stress kernel the surface kernel writes
// the image strxz(zs - 1) = -strxz(zs) (YPUB:1009-1024) and vz(zs - 1) from vz(zs) and dx vx(zs)
// (YPUB:938-976).  The reference writes that vz after summing the split parts, so its stress
// update reads it one step later; running the surface kernel after the stress kernel gives the
// same order.
//
// Model preparation (host, per shot window): substagger (YPUB:323-547); then, in abc mode, on the
// device the PML smoothing of modipapml (YPUB:549-634), which overwrites each top-sponge cell with the
// Gaussian-weighted sum of its window while later cells read the already smoothed ones: a
// sequential chain, run as one thread per array and window in the reference's serial order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "sfd_internal.h"

namespace sfd {
namespace {

constexpr int kThreads = 256;
constexpr int TX = kTileX, TZ = kTileZ;
constexpr int H = 5;                  // staggered reach: Dx0 reads i-5..i+4, Dx1 i-4..i+5
constexpr int HZ = 8;                 // z halo rounded for float4 staging
constexpr int SROWS = TX + 2 * H;     // 74
constexpr int SW = TZ + 2 * HZ;       // 80
constexpr int SMEM = SROWS * SW;      // floats per staged field

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }

struct TileRef {
    int shot, tile, x0, z0;
    ShotDev sd;
};

__device__ __forceinline__ bool tile_of(const IArgs& a, TileRef& t) {
    t.shot = a.slot_to_shot[blockIdx.y];
    t.sd = a.shots[t.shot];
    t.tile = blockIdx.x;
    const int tx_i = t.tile / a.L.ntz, tz_i = t.tile - tx_i * a.L.ntz;
    t.x0 = tx_i * TX;
    t.z0 = tz_i * TZ;
    return t.x0 < t.sd.nx;
}

__device__ __forceinline__ long long cell(const IArgs& a, int shot, int x, int z) {
    return (long long)shot * a.L.shot_stride + (long long)(x + a.L.gx) * a.L.pitch + a.L.gz + z;
}

// stage f0 + f1 (YPUB:1410-1426) on the tile plus halo
__device__ __forceinline__ void stage(float* s, const IArgs& a, const TileRef& t, const float* f0, const float* f1) {
    constexpr int W4 = SW / 4;
#pragma unroll 3  // several rows' loads in flight before their shared-memory stores
    for (int i = threadIdx.x; i < SROWS * W4; i += kThreads) {
        const int r = i / W4, c = i - r * W4;
        const long long off = cell(a, t.shot, t.x0 - H + r, t.z0 - HZ + 4 * c);
        const float4 u = __ldg(reinterpret_cast<const float4*>(f0 + off));
        const float4 v = __ldg(reinterpret_cast<const float4*>(f1 + off));
        *reinterpret_cast<float4*>(s + r * SW + 4 * c) = make_float4(fa(u.x, v.x), fa(u.y, v.y), fa(u.z, v.z), fa(u.w, v.w));
    }
}

// one split-sponge factor in YPUB:851-897's order (near-side table, then far-side table)
__device__ __forceinline__ float xs(float u, int x, int n, int np, const float* tn, const float* tp) {
    if (x <= np) u = fm(u, tn[x]);
    if (x >= n - np - 1) u = fm(u, tp[n - 1 - x]);
    return u;
}

// Work items: thread t takes the z-vector zv = t % 16 (cells z0 + 4 zv .. + 3) of the rows
// t / 16 + 16 j, j = 0..3; a warp covers two whole tile rows, so every field access is one
// coalesced 16-byte load or store per lane.  The stencils read float4 windows from shared
// memory: an x derivative of four cells is ten 16-byte loads, a z derivative four.
constexpr int kItems = TX * TZ / 4 / kThreads;  // 4

__device__ __forceinline__ float4 lds4(const float* s, int r, int c) { return *reinterpret_cast<const float4*>(s + r * SW + c); }
__device__ __forceinline__ float cmp(const float4& v, int q) { return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w)); }
__device__ __forceinline__ float& cmpr(float4& v, int q) { return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w)); }

// x derivative (YPUB:1095-1157) of the four cells (row r, columns c..c+3) of a staged field
template <int FLAG>
__device__ __forceinline__ float4 dx4(const float* s, int r, int c, const float* a) {
    float4 acc;
#pragma unroll
    for (int m = 0; m < 5; m++) {
        const float4 p = lds4(s, FLAG == 0 ? r + m : r + 1 + m, c);
        const float4 q = lds4(s, FLAG == 0 ? r - 1 - m : r - m, c);
        const float4 t = make_float4(fs(p.x, q.x), fs(p.y, q.y), fs(p.z, q.z), fs(p.w, q.w));
        if (m == 0) acc = make_float4(fm(a[0], t.x), fm(a[0], t.y), fm(a[0], t.z), fm(a[0], t.w));
        else acc = make_float4(fa(acc.x, fm(a[m], t.x)), fa(acc.y, fm(a[m], t.y)), fa(acc.z, fm(a[m], t.z)),
                               fa(acc.w, fm(a[m], t.w)));
    }
    return acc;
}

// z derivative (YPUB:1347-1407) of the same four cells: the window z-8 .. z+11 (c = column of z).
// d0: distance of the first cell below the free surface (large without one).  Cells d = 0..4
// rows below it take the lower orders of caluz (YPUB:1160-1343); the ones above it are not used.
template <int FLAG, bool FS>
__device__ __forceinline__ float4 dz4(const float* s, int r, int c, const IArgs& a, int d0) {
    float w[20];
#pragma unroll
    for (int j = 0; j < 5; j++) {
        const float4 v = lds4(s, r, c - 8 + 4 * j);
        w[4 * j] = v.x; w[4 * j + 1] = v.y; w[4 * j + 2] = v.z; w[4 * j + 3] = v.w;
    }
    float4 acc;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int d = d0 + q;
        const int M = !FS ? 5 : FLAG == 0 ? (d >= 5 ? 5 : (d < 1 ? 1 : d)) : (d >= 4 ? 5 : (d < 0 ? 1 : d + 1));
        float sum = 0.0f;
#pragma unroll
        for (int m = 0; m < 5; m++) {
            if (m >= M) break;
            const float cm = M == 5 ? a.a[m] : a.cr[M - 1 > 0 ? (M == 4 ? 3 : M == 3 ? 2 : 1) : 0][m & 3];
            const int z = 8 + q;  // index of cell q in w
            const float t = FLAG == 0 ? fs(w[z + m], w[z - 1 - m]) : fs(w[z + 1 + m], w[z - m]);
            sum = (m == 0) ? fm(cm, t) : fa(sum, fm(cm, t));
        }
        cmpr(acc, q) = sum;
    }
    return acc;
}

// z-part sponge: abc, the top table on rows t0 .. t0 + npz then the bottom table (YPUB:851-897);
// fsbc, the bottom table only (YPUB:901-934)
template <bool FS>
__device__ __forceinline__ float zsp(float u, int z, int t0, const IArgs& a, const float* tn, const float* tp) {
    if (!FS && z >= t0 && z <= t0 + a.npz) u = fm(u, tn[z - t0]);
    if (z >= a.nz - a.npz - 1) u = fm(u, tp[a.nz - 1 - z]);
    return u;
}

// four cells of a field: one 16-byte access when all four lie inside the grid, else per cell
__device__ __forceinline__ float4 ld4(const float* f, long long c, int nv) {
    if (nv == 4) return *reinterpret_cast<const float4*>(f + c);
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int q = 0; q < nv; q++) cmpr(v, q) = f[c + q];
    return v;
}
__device__ __forceinline__ void st4(float* f, long long c, int nv, const float4& v) {
    if (nv == 4) {
        *reinterpret_cast<float4*>(f + c) = v;
        return;
    }
    for (int q = 0; q < nv; q++) f[c + q] = cmp(v, q);
}

template <bool FS>
__global__ void __launch_bounds__(kThreads, 3) iso_velocity_kernel(const __grid_constant__ IArgs a) {
    extern __shared__ __align__(16) float smem[];
    float* sSxx = smem;
    float* sSxz = smem + SMEM;
    float* sSzz = smem + 2 * SMEM;
    TileRef t;
    if (!tile_of(a, t)) return;
    stage(sSxx, a, t, a.f[I_SXXX], a.f[I_SXXZ]);
    stage(sSxz, a, t, a.f[I_SXZX], a.f[I_SXZZ]);
    stage(sSzz, a, t, a.f[I_SZZX], a.f[I_SZZZ]);
    __syncthreads();
    const int nx = t.sd.nx, nz = a.nz;
    const float* tb = a.spg;
    const int st = a.spg_stride;
    const int zv = threadIdx.x & 15, z = 4 * zv, gz = t.z0 + z;
    const int nv = min(4, nz - gz);  // cells of the vector inside the grid
    if (nv <= 0) return;             // no barrier follows
#pragma unroll 1
    for (int j = 0; j < kItems; j++) {
        const int r = (threadIdx.x >> 4) + 16 * j, gx = t.x0 + r;
        if (gx >= nx) break;
        const long long c = cell(a, t.shot, gx, gz);
        const int mc = min(t.sd.x0 + gx, a.nx_model - 1);
        const long long mi = (long long)mc * a.mpitch + gz;
        // first updated row: zs = itopo - 1 (fsbc) or t0 = itopo - npz - 1 (abc)
        const int top = __ldg(a.itopo + mc) - (FS ? 1 : a.npz + 1);
        const int d0 = FS ? gz - top : (1 << 20);
        float4 vxx = ld4(a.f[I_VXX], c, nv), vxz = ld4(a.f[I_VXZ], c, nv);
        float4 vzx = ld4(a.f[I_VZX], c, nv), vzz = ld4(a.f[I_VZZ], c, nv);
        const float4 b2 = __ldg(reinterpret_cast<const float4*>(a.b2e + mi));
        const float4 b1 = __ldg(reinterpret_cast<const float4*>(a.b1e + mi));
        const float4 d_xx = dx4<0>(sSxx, r + H, z + HZ, a.a);      // Dx0 strxx
        const float4 d_xz = dz4<0, FS>(sSxz, r + H, z + HZ, a, d0);    // Dz0 strxz
        const float4 d_zx = dx4<1>(sSxz, r + H, z + HZ, a.a);      // Dx1 strxz
        const float4 d_zz = dz4<1, FS>(sSzz, r + H, z + HZ, a, d0);    // Dz1 strzz
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int zq = min(gz + q, nz - 1);  // cells past nz are computed, not stored
            const bool below = gz + q >= top;  // rows above the first updated row keep their values
            // YPRI:310-316: vx parts, sponge spgxn/spgxp (x part), spgzn/spgzp (z part)
            if (below) {
                const float n_xx = fa(cmp(vxx, q), fm(fm(a.dtdx, cmp(b2, q)), cmp(d_xx, q)));
                cmpr(vxx, q) = xs(n_xx, gx, nx, a.npx, tb + 0 * st, tb + 1 * st);
                cmpr(vxz, q) = fa(cmp(vxz, q), fm(fm(a.dtdz, cmp(b2, q)), cmp(d_xz, q)));
            }
            cmpr(vxz, q) = zsp<FS>(cmp(vxz, q), zq, top, a, tb + 2 * st, tb + 3 * st);
            // YPRI:320-326: vz parts, sponge spg1xn/spg2xp, spg1zn/spg2zp
            if (below) {
                const float n_zx = fa(cmp(vzx, q), fm(fm(a.dtdx, cmp(b1, q)), cmp(d_zx, q)));
                cmpr(vzx, q) = xs(n_zx, gx, nx, a.npx, tb + 4 * st, tb + 5 * st);
                cmpr(vzz, q) = fa(cmp(vzz, q), fm(fm(a.dtdz, cmp(b1, q)), cmp(d_zz, q)));
            }
            cmpr(vzz, q) = zsp<FS>(cmp(vzz, q), zq, top, a, tb + 6 * st, tb + 7 * st);
        }
        st4(a.f[I_VXX], c, nv, vxx); st4(a.f[I_VXZ], c, nv, vxz);
        st4(a.f[I_VZX], c, nv, vzx); st4(a.f[I_VZZ], c, nv, vzz);
    }
}

template <bool FS>
__global__ void __launch_bounds__(kThreads, 3) iso_stress_kernel(const __grid_constant__ IArgs a) {
    __shared__ __align__(16) float sVx[SMEM];
    __shared__ __align__(16) float sVz[SMEM];
    TileRef t;
    if (!tile_of(a, t)) return;
    stage(sVx, a, t, a.f[I_VXX], a.f[I_VXZ]);  // vx = vxx + vxz (YPRI:316)
    stage(sVz, a, t, a.f[I_VZX], a.f[I_VZZ]);  // vz = vzx + vzz (YPRI:326)
    __syncthreads();
    const int nx = t.sd.nx, nz = a.nz;
    const float* tb = a.spg;
    const int st = a.spg_stride;
    const ShotDev& sd = t.sd;
    const float wav = __ldg(a.wavelets + sd.wav_off + a.step);
    const int zv = threadIdx.x & 15, z = 4 * zv, gz = t.z0 + z;
    const int nv = min(4, nz - gz);
    // YPRI:163-168: in fsbc mode strxx takes the source only below the surface at the source column
    const bool src_xx = !FS || sd.sz + 1 > __ldg(a.itopo + min(sd.x0 + sd.sx, a.nx_model - 1));
#pragma unroll 1
    for (int j = 0; j < kItems && nv > 0; j++) {
        const int r = (threadIdx.x >> 4) + 16 * j, gx = t.x0 + r;
        if (gx >= nx) break;
        const long long c = cell(a, t.shot, gx, gz);
        const int mc = min(sd.x0 + gx, a.nx_model - 1);
        const long long mi = (long long)mc * a.mpitch + gz;
        const int top = __ldg(a.itopo + mc) - (FS ? 1 : a.npz + 1);  // zs (fsbc) or t0 (abc)
        const int d0 = FS ? gz - top : (1 << 20);
        float4 v[6];  // strxxx strxxz strzzx strzzz strxzx strxzz
#pragma unroll
        for (int k = 0; k < 6; k++) v[k] = ld4(a.f[I_SXXX + k], c, nv);
        const float4 lm2 = __ldg(reinterpret_cast<const float4*>(a.lm2 + mi));
        const float4 lam = __ldg(reinterpret_cast<const float4*>(a.lam + mi));
        const float4 mue = __ldg(reinterpret_cast<const float4*>(a.mue + mi));
        const float4 d1 = dx4<1>(sVx, r + H, z + HZ, a.a);       // Dx1 vx
        const float4 d2 = dz4<0, FS>(sVz, r + H, z + HZ, a, d0);     // Dz0 vz
        const float4 d3 = dx4<0>(sVz, r + H, z + HZ, a.a);       // Dx0 vz
        const float4 d4 = dz4<1, FS>(sVx, r + H, z + HZ, a, d0);     // Dz1 vx
        const int bx = gx - sd.stamp_x0;
        const bool xin = bx >= 0 && bx < sd.stamp_w;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int zq = min(gz + q, nz - 1);  // cells past nz are computed, not stored
            const int bz = zq - sd.stamp_z0;
            const bool in_stamp = xin && bz >= 0 && bz < sd.stamp_h;
            float src = 0.0f;
            if (in_stamp)  // YPUB:1458 wavelet*gc2d*dt/(dz**2)
                src = __fdiv_rn(fm(fm(wav, __ldg(a.stamps + sd.stamp_off + bx * sd.stamp_h + bz)), a.dt), a.dz2);
            // rows above the first updated row keep their values (the loops start at itopo or
            // itopo - npzn)
            const bool below = gz + q >= top;
            const bool zero_zz = FS && gz + q <= top;  // YPUB:978-1007, rows <= itopo
            // YPRI:331-338: strxx parts, sponge spg1xn/spg2xp, spgzn/spgzp, then the source
            float s0 = cmp(v[0], q), s1 = cmp(v[1], q), s2 = cmp(v[2], q), s3 = cmp(v[3], q);
            float s4 = cmp(v[4], q), s5 = cmp(v[5], q);
            if (below) {
                s0 = xs(fa(s0, fm(fm(a.dtdx, cmp(lm2, q)), cmp(d1, q))), gx, nx, a.npx, tb + 4 * st, tb + 5 * st);
                s1 = fa(s1, fm(fm(a.dtdz, cmp(lam, q)), cmp(d2, q)));
            }
            s1 = zsp<FS>(s1, zq, top, a, tb + 2 * st, tb + 3 * st);
            if (in_stamp && src_xx) s0 = fa(src, s0);
            // YPRI:342-349: strzz parts; fsbc: zero on rows <= the surface before the source
            if (below) {
                s2 = xs(fa(s2, fm(fm(a.dtdx, cmp(lam, q)), cmp(d1, q))), gx, nx, a.npx, tb + 4 * st, tb + 5 * st);
                s3 = fa(s3, fm(fm(a.dtdz, cmp(lm2, q)), cmp(d2, q)));
            }
            s3 = zsp<FS>(s3, zq, top, a, tb + 2 * st, tb + 3 * st);
            if (zero_zz) s2 = s3 = 0.0f;
            if (in_stamp) s2 = fa(src, s2);
            // YPRI:353-359: strxz parts, sponge spgxn/spgxp, spg1zn/spg2zp
            if (below) {
                s4 = xs(fa(s4, fm(fm(a.dtdx, cmp(mue, q)), cmp(d3, q))), gx, nx, a.npx, tb + 0 * st, tb + 1 * st);
                s5 = fa(s5, fm(fm(a.dtdz, cmp(mue, q)), cmp(d4, q)));
            }
            s5 = zsp<FS>(s5, zq, top, a, tb + 6 * st, tb + 7 * st);
            cmpr(v[0], q) = s0; cmpr(v[1], q) = s1; cmpr(v[2], q) = s2;
            cmpr(v[3], q) = s3; cmpr(v[4], q) = s4; cmpr(v[5], q) = s5;
        }
#pragma unroll
        for (int k = 0; k < 6; k++) st4(a.f[I_SXXX + k], c, nv, v[k]);
    }
    // receivers: record1 = vx, record2 = vz after the step (YPRI:361-367, YPUB:2-16); the
    // velocities are final after the velocity kernel and staged here
    const int* trp = a.tile_rec_ptr + sd.tile_rec_base + t.tile;
    const int rb = trp[0], re = trp[1];
    for (int j = rb + threadIdx.x; j < re; j += kThreads) {
        const int ridx = a.tile_rec_idx[j];
        const int rr = a.rec_x[sd.rec_list + ridx] - t.x0 + H, rz = a.rec_z[sd.rec_list + ridx] - t.z0 + HZ;
        const long long o = sd.rec_base + (long long)a.step * sd.nrec + ridx;
        a.records[o] = sVx[rr * SW + rz];
        a.records2[o] = sVz[rr * SW + rz];
    }
}

// Free surface, after the stress kernel (one thread per column, zs = itopo(x) - 1): the image strxz(zs - 1) =
// -strxz(zs) of both split parts (YPUB:1009-1024), and vz(zs - 1) = vz(zs) + lambsg/lambmusg
// (vx(zs, x + 1) - vx(zs, x)) for both pairs of split parts (YPUB:938-976, columns but the last).
__global__ void iso_surface_kernel(const __grid_constant__ IArgs a) {
    const int shot = a.slot_to_shot[blockIdx.y];
    const ShotDev sd = a.shots[shot];
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= sd.nx) return;
    const int mc = min(sd.x0 + x, a.nx_model - 1);
    const int zs = __ldg(a.itopo + mc) - 1;
    if (zs < 1) return;  // the row above the surface is the split fields' unused row 0
    const long long c = cell(a, shot, x, zs), cu = c - 1;
    a.f[I_SXZX][cu] = -a.f[I_SXZX][c];
    a.f[I_SXZZ][cu] = -a.f[I_SXZZ][c];
    if (x + 1 < sd.nx) {
        const long long cn = cell(a, shot, x + 1, zs);
        const long long mi = (long long)mc * a.mpitch + zs;
        const float ratio = __fdiv_rn(__ldg(a.lam + mi), __ldg(a.lm2 + mi));
        a.f[I_VZX][cu] = fa(a.f[I_VZX][c], fm(ratio, fs(a.f[I_VXX][cn], a.f[I_VXX][c])));
        a.f[I_VZZ][cu] = fa(a.f[I_VZZ][c], fm(ratio, fs(a.f[I_VXZ][cn], a.f[I_VXZ][c])));
    }
}

// YPUB:592-634, one sequential chain per (window, array), one warp each: cells (z < itopo) in
// the serial loop order, each replaced by the weighted sum of its window as it stands at that
// moment.  The warp's lanes form the cell's products u(m, n) gc(idx1, idx2) in parallel (each
// is one rounded multiply, whoever computes it) into shared memory in the loop's (n, m) order;
// lane 0 then adds them in that order, so the sum is rounded exactly as the serial loop rounds
// it.  Terms with an exact zero weight (table columns outside [lo, hi], rows outside the
// column's non-zero range) are left out: adding them would leave the sum unchanged (it starts
// at +0 and never becomes -0).  __syncwarp orders lane 0's store of a cell before the loads of
// the next cells.
struct SmoothArgs {
    float* arr[5];
    const int* win;   // nwin (start column, width) pairs
    const int* rng;   // per table column idx2: first and last row idx1 with a non-zero weight
    const int* itopo; // per prepared column: rows z < itopo are smoothed
    int nwin, mpitch, ghost, nz, rgau, lo, hi;
    const float* gc;
};

__global__ void __launch_bounds__(32) iso_smooth_kernel(const __grid_constant__ SmoothArgs s) {
    extern __shared__ __align__(16) float prod[];
    const int t = blockIdx.x, lane = threadIdx.x;
    const int b = t / 5;
    float* u = s.arr[t - 5 * b] + (long long)s.win[2 * b] * s.mpitch;
    const int* itopo = s.itopo + s.win[2 * b];
    const int nxw = s.win[2 * b + 1];
    const int w = 2 * s.rgau - 1, r1 = s.rgau - 1;
    for (int i = 0; i < nxw; i++)
        for (int k = 0, kn = min(itopo[i], s.nz); k < kn; k++) {
            const int nlo = max(i - r1 + s.lo, 0), nhi = min(i - r1 + s.hi, nxw - 1);
            // lane L forms the products of columns nlo + L and nlo + L + 32; their offsets in the
            // loop order come from a warp prefix sum of the column lengths
            int mlo[2], cnt[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int n = nlo + lane + 32 * h;
                mlo[h] = 0;
                cnt[h] = 0;
                if (n <= nhi) {
                    const int j2 = n - i + r1;  // idx2 - 1
                    mlo[h] = max(k - r1 + s.rng[2 * j2], 0);
                    cnt[h] = max(min(k - r1 + s.rng[2 * j2 + 1], s.nz - 1) - mlo[h] + 1, 0);
                }
            }
            int off[2], total = 0;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                int x = cnt[h];
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, x, d);
                    if (lane >= d) x += y;
                }
                off[h] = total + x - cnt[h];
                total += __shfl_sync(0xffffffffu, x, 31);
            }
#pragma unroll
            for (int h = 0; h < 2; h++) {
                if (cnt[h] == 0) continue;
                const int n = nlo + lane + 32 * h;
                const float* col = u + (long long)n * s.mpitch + mlo[h];
                const float* g = s.gc + (n - i + r1) * w + r1 - k + mlo[h];  // gc(m - k + r1 + 1, idx2)
                float* p = prod + off[h];
#pragma unroll 4
                for (int q = 0; q < cnt[h]; q++) p[q] = fm(col[q], g[q]);
            }
            __syncwarp();
            if (lane == 0) {
                float acc = 0.0f;
                int q = 0;
#pragma unroll 4
                for (; q + 4 <= total; q += 4) {
                    const float4 v = *reinterpret_cast<const float4*>(prod + q);
                    acc = fa(fa(fa(fa(acc, v.x), v.y), v.z), v.w);
                }
                for (; q < total; q++) acc = fa(acc, prod[q]);
                u[(long long)i * s.mpitch + k] = acc;
            }
            __syncwarp();
        }
    for (int c = lane; c < nxw; c += 32)  // the replicated rows above z = 0 follow the smoothed row
        for (int g = 1; g <= s.ghost; g++) u[(long long)c * s.mpitch - g] = u[(long long)c * s.mpitch];
}

}  // namespace

cudaError_t elastic2d_launch_step(const IArgs& a, int active, int nx_max, cudaStream_t st, int* launches) {
    dim3 grid(a.L.ntx * a.L.ntz, active);
    const size_t smem = sizeof(float) * 3 * SMEM;
    static bool attr0[kMaxDevices] = {}, attr1[kMaxDevices] = {};
    if (cudaError_t e = smem_attr_once((const void*)iso_velocity_kernel<false>, (int)smem, attr0)) return e;
    if (cudaError_t e = smem_attr_once((const void*)iso_velocity_kernel<true>, (int)smem, attr1)) return e;
    *launches = 2;
    if (a.fs) {
        iso_velocity_kernel<true><<<grid, kThreads, smem, st>>>(a);
        iso_stress_kernel<true><<<grid, kThreads, 0, st>>>(a);
        iso_surface_kernel<<<dim3((nx_max + 127) / 128, active), 128, 0, st>>>(a);
        *launches = 3;
    } else {
        iso_velocity_kernel<false><<<grid, kThreads, smem, st>>>(a);
        iso_stress_kernel<false><<<grid, kThreads, 0, st>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t elastic2d_smooth(float* const arrays[5], int mpitch, int ghost, int nz, const int* itopo_dev,
                             const int* win_host, int nwin, const std::vector<float>& gc, int rgau, int lo, int hi,
                             cudaStream_t st) {
    if (nwin <= 0) return cudaSuccess;
    SmoothArgs s{};
    for (int i = 0; i < 5; i++) s.arr[i] = arrays[i];
    const int w = 2 * rgau - 1;
    std::vector<int> rng(2 * (size_t)w), buf(2 * (size_t)nwin);  // per table column: non-zero rows
    for (int j = 0; j < w; j++) {
        int a = w, b = -1;
        for (int i = 0; i < w; i++)
            if (gc[(size_t)j * w + i] != 0.0f) {
                a = std::min(a, i);
                b = std::max(b, i);
            }
        rng[2 * j] = a;
        rng[2 * j + 1] = b;
    }
    for (int i = 0; i < 2 * nwin; i++) buf[i] = win_host[i];
    buf.insert(buf.end(), rng.begin(), rng.end());
    int* d_win = nullptr;
    float* d_gc = nullptr;
    cudaError_t e = cudaMalloc(&d_win, sizeof(int) * buf.size());
    if (e == cudaSuccess) e = cudaMalloc(&d_gc, sizeof(float) * gc.size());
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_win, buf.data(), sizeof(int) * buf.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_gc, gc.data(), sizeof(float) * gc.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        s.win = d_win;
        s.rng = d_win + 2 * nwin;
        s.gc = d_gc;
        s.nwin = nwin;
        s.mpitch = mpitch;
        s.ghost = ghost;
        s.nz = nz;
        s.itopo = itopo_dev;
        s.rgau = rgau;
        s.lo = lo;
        s.hi = hi;
        // shared memory: the products of one cell, at most (hi - lo + 1)^2; the kernel gives each
        // lane two table columns (the sigma = 2 table has at most 57 non-zero ones)
        const size_t smem = sizeof(float) * ((size_t)(hi - lo + 1) * (hi - lo + 1) + 4);
        if (smem > 200 * 1024 || hi - lo + 1 > 64) {
            e = cudaErrorInvalidValue;
        } else {
            if (smem > 48 * 1024)
                e = cudaFuncSetAttribute(iso_smooth_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e == cudaSuccess) {
                iso_smooth_kernel<<<5 * nwin, 32, smem, st>>>(s);
                e = cudaGetLastError();
            }
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_win);
    cudaFree(d_gc);
    return e;
}

bool elastic2d_prepare(int nx, int nz, const float* vp, const float* vs, const float* rho, const int* itopo,
                       float* b2e, float* b1e, float* lm2, float* lam, float* mue) {
    const size_t n = (size_t)nx * nz;
    auto at = [nz](int k, int i) { return (size_t)i * nz + k; };  // Fortran (k, i), 0-based
    std::vector<float> mu(n), lamb(n), busg1(n, 0.0f), busg2(n), musg(n);
    for (int i = 0; i < nx; i++)
        for (int k = 0; k < nz; k++) {
            const size_t c = at(k, i);
            mu[c] = rho[c] * vs[c] * vs[c];
            lamb[c] = rho[c] * vp[c] * vp[c] - 2.0f * mu[c];
        }
    for (int i = 0; i < nx - 1; i++)
        for (int k = 0; k < nz - 1; k++)
            busg1[at(k, i)] = 0.25f * (rho[at(k, i)] + rho[at(k + 1, i)] + rho[at(k + 1, i + 1)] + rho[at(k, i + 1)]);
    for (int i = 0; i < nx; i++) busg1[at(nz - 1, i)] = busg1[at(nz - 2, i)];
    for (int k = 0; k < nz; k++) busg1[at(k, nx - 1)] = busg1[at(k, nx - 2)];
    for (size_t c = 0; c < n; c++) {
        if (busg1[c] == 0.0f || rho[c] == 0.0f) return false;  // YPUB:370, 400
        busg1[c] = 1.0f / busg1[c];
        busg2[c] = 1.0f / rho[c];
    }
    for (int i = 0; i < nx; i++) {
        for (int k = 1; k < nz; k++) b1e[at(k, i)] = 0.5f * (busg1[at(k, i)] + busg1[at(k - 1, i)]);
        b1e[at(0, i)] = busg1[at(0, i)];
    }
    for (int k = 0; k < nz; k++) {
        for (int i = 0; i < nx - 1; i++) b2e[at(k, i)] = 0.5f * (busg2[at(k, i)] + busg2[at(k, i + 1)]);
        b2e[at(k, nx - 1)] = busg2[at(k, nx - 1)];
    }
    for (int i = 0; i < nx; i++) {
        for (int k = 0; k < nz - 1; k++) musg[at(k, i)] = 0.5f * (mu[at(k + 1, i)] + mu[at(k, i)]);
        musg[at(nz - 1, i)] = mu[at(nz - 1, i)];
    }
    for (int i = 0; i < nx - 1; i++)
        for (int k = 1; k < nz; k++) {
            const float q0 = musg[at(k, i)], q1 = musg[at(k, i + 1)], q2 = musg[at(k - 1, i + 1)], q3 = musg[at(k - 1, i)];
            mue[at(k, i)] = (q0 != 0.0f && q1 != 0.0f && q2 != 0.0f && q3 != 0.0f)
                                ? 4.0f / (1.0f / q0 + 1.0f / q1 + 1.0f / q2 + 1.0f / q3)
                                : 0.0f;
        }
    for (int i = 0; i < nx; i++) mue[at(0, i)] = musg[at(0, i)];
    for (int k = 0; k < nz; k++) mue[at(k, nx - 1)] = musg[at(k, nx - 1)];
    for (int k = 0; k < nz; k++) {
        for (int i = 0; i < nx - 1; i++) {
            lam[at(k, i)] = 0.5f * (lamb[at(k, i + 1)] + lamb[at(k, i)]);
            lm2[at(k, i)] = 0.5f * (lamb[at(k, i)] + 2.0f * mu[at(k, i)] + lamb[at(k, i + 1)] + 2.0f * mu[at(k, i + 1)]);
        }
        lam[at(k, nx - 1)] = lamb[at(k, nx - 1)];
        lm2[at(k, nx - 1)] = lamb[at(k, nx - 1)] + 2.0f * mu[at(k, nx - 1)];
    }
    // YPUB:484-501: rows above itopo (1-based) take row itopo's values
    for (float* f : {b2e, b1e, lm2, lam, mue})
        for (int i = 0; i < nx; i++)
            for (int k = std::min(itopo[i], nz) - 1; k >= 1; k--) f[at(k - 1, i)] = f[at(k, i)];
    return true;
}

void elastic2d_gauss_table(int rgau, std::vector<float>* out, int* lo, int* hi) {
    const int w = 2 * rgau - 1, cen = (w + 1) / 2;
    const float pi = 3.1415926f, sigma2 = 2.0f * 2.0f;
    out->assign((size_t)w * w, 0.0f);
    for (int j = 1; j <= w; j++)
        for (int i = 1; i <= w; i++) {
            const float dis = (float)((j - cen) * (j - cen) + (i - cen) * (i - cen));
            (*out)[(size_t)(j - 1) * w + (i - 1)] = 1.0f / (2.0f * pi * sigma2) * std::exp(-(dis / (2.0f * sigma2)));
        }
    float sum = 0.0f;
    for (int j = 0; j < w; j++)
        for (int i = 0; i < w; i++) sum = sum + (*out)[(size_t)j * w + i];
    int l = w, h = -1;
    for (int j = 0; j < w; j++)
        for (int i = 0; i < w; i++) {
            float& v = (*out)[(size_t)j * w + i];
            v = v / sum;
            if (v != 0.0f) {
                l = std::min(l, std::min(i, j));
                h = std::max(h, std::max(i, j));
            }
        }
    *lo = l;
    *hi = h;
}

void elastic2d_stamp(int nx, int nz, int sx, int sz, int rgau, const std::vector<float>& gc, int* box,
                     std::vector<float>* out) {
    const int w = 2 * rgau - 1, r1 = rgau - 1;
    int xlo = 1 << 30, xhi = -1, zlo = 1 << 30, zhi = -1;
    for (int x = std::max(sx - r1, 0); x <= std::min(sx + r1, nx - 1); x++)
        for (int z = std::max(sz - r1, 0); z <= std::min(sz + r1, nz - 1); z++)
            if (gc[(size_t)(x - sx + r1) * w + (z - sz + r1)] != 0.0f) {
                xlo = std::min(xlo, x); xhi = std::max(xhi, x);
                zlo = std::min(zlo, z); zhi = std::max(zhi, z);
            }
    if (xhi < 0) {
        box[0] = box[1] = box[2] = box[3] = 0;
        return;
    }
    box[0] = xlo; box[1] = zlo; box[2] = xhi - xlo + 1; box[3] = zhi - zlo + 1;
    for (int x = xlo; x <= xhi; x++)
        for (int z = zlo; z <= zhi; z++) out->push_back(gc[(size_t)(x - sx + r1) * w + (z - sz + r1)]);
}

}  // namespace sfd
