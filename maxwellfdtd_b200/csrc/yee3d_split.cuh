// yee3d_split.cuh -- 3-D updates (single and double precision) split by CPML region (sm_100a).
//
// A 3-D grid with CPML layers on the y and z faces is cut into
//   core  : rows outside the y and z layers (all x), marched along z by h3d_core_kernel /
//           e3d_core_kernel.  The only layers a core cell can be in are the x layers, and
//           for a given column that membership, the layer's coefficients and its psi stride
//           are fixed, so they are loaded once and the psi pair of the next plane is
//           prefetched with the fields: a layer cell costs its psi traffic and a few flops;
//   slab  : every cell of the y and z layers (h3d_slab_kernel / e3d_slab_kernel), one cell
//           per thread with all of its loads issued together, general CPML (any faces).
// The per-cell arithmetic is that of h3d_f32_kernel / e3d_f32_kernel (single precision) and
// h3d_kernel / e3d_kernel (double precision) in yee.cuh, operation for operation and with
// the faces in the same order, so results are bit-identical.  The
// split needs layers that do not overlap in any dimension (checked on the host, which
// otherwise launches the unsplit kernels).
#pragma once

#include "yee.cuh"

#define MFD_CORE_MINB 4   // single-precision core kernels: blocks of 256 threads' worth per SM (64 registers)
#define MFD_SLAB_MINB 16  // single-precision slab kernels: 16 blocks of 128 threads per SM (32 registers; measured faster than 40)

namespace mfd {

// Rows of the core box and the slab region.  Cells with iz < zl or iz >= zr are in a z layer,
// iy < yl or iy >= yr in a y layer (zl <= zr, yl <= yr).  Slab rows are numbered z-layer
// rows first (plane-major: nzr = (zl + nz - zr) * ny of them), then y-layer rows of the
// core planes (zr - zl planes of yl + ny - yr rows).
struct SplitBox {
    int yl, yr, zl, zr;
    int zc;     // planes per core block
    int nzr;    // slab rows in z layers
};

// Tiles of the core rows that the staged E kernel leaves to the register march with the
// material map: columns x0 .. x1-1, rows y0 .. y1-1, planes z0 .. z1-1 (aligned to the
// tiles; empty when y0 == y1).
struct TileSkip {
    int x0, x1, y0, y1, z0, z1;
};

__device__ __forceinline__ void slab_row(const SplitBox& s, int ny, int r, int& iy, int& iz) {
    if (r < s.nzr) {
        const int pz = r / ny;
        iy = r - pz * ny;
        iz = pz < s.zl ? pz : s.zr + (pz - s.zl);
    } else {
        const int nys = s.yl + (ny - s.yr);
        const int r2 = r - s.nzr;
        const int zz = r2 / nys, yy = r2 - zz * nys;
        iz = s.zl + zz;
        iy = yy < s.yl ? yy : s.yr + (yy - s.yl);
    }
}

// The six curl derivatives of a cell, q = num / (dy, dz, dx, dz, dx, dy): for single precision
// the verified branch-free division (div6), for double precision IEEE division.
template <typename T, int FAST>
__device__ __forceinline__ void curl_div(const Div3& D3, const DivC<T>& ddx, const DivC<T>& ddy, const DivC<T>& ddz,
                                         const T (&num)[6], T (&q)[6]) {
    if constexpr (sizeof(T) == 4) {
        div6<FAST>(D3, num, q);
    } else {
        q[0] = cdiv<FAST>(num[0], ddy); q[1] = cdiv<FAST>(num[1], ddz); q[2] = cdiv<FAST>(num[2], ddx);
        q[3] = cdiv<FAST>(num[3], ddz); q[4] = cdiv<FAST>(num[4], ddx); q[5] = cdiv<FAST>(num[5], ddy);
    }
}

template <typename T>
__device__ __forceinline__ bool maybe_nonfinite(T x) {
    if constexpr (sizeof(T) == 4) return !(fabsf(x) <= FLT_MAX);
    else return !(fabs(x) <= DBL_MAX);
}

// x-layer state of one column: which face (none / left / right), its coefficients and psi.
template <typename T>
struct XCol {
    bool in;
    int q, nb;
    T A, B;
    DivC<T> K;
    T* pa;
    T* pb;
};

template <typename T>
__device__ __forceinline__ XCol<T> xcol(const LayerDev<T>& lxl, const LayerDev<T>& lxr, int ix, int ia, int ib) {
    XCol<T> x;
    const bool l = lxl.nb && ix < lxl.ib;
    const bool r = lxr.nb && ix >= lxr.ib - 1;
    x.in = l || r;
    x.q = l ? ix : ix - (lxr.ib - 1);
    x.nb = l ? lxl.nb : lxr.nb;
    x.pa = l ? lxl.psi[ia] : lxr.psi[ia];
    x.pb = l ? lxl.psi[ib] : lxr.psi[ib];
    if (x.in) {
        const LayerDev<T>& lx = l ? lxl : lxr;
        x.A = lx.A[x.q];
        x.B = lx.B[x.q];
        x.K = lx.K[x.q];
    } else {
        x.A = x.B = T(0);
        x.K = DivC<T>{};
    }
    return x;
}

template <typename T>
struct HCoreLoad {
    T ez, eyx, ezx, exy, ezy, exz, eyz, hx, hy, hz, sa, e2, pa, pb;
    int g;
};

template <typename T, bool MATH, int FAST, bool ACC, bool E2S>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? MFD_CORE_MINB : 2) h3d_core_kernel(const __grid_constant__ HParams<T> p,
                                                                               const Div3 D3, const SplitBox s) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = s.yl + blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = p.L.nx, ny = p.L.ny, nz = p.L.nz;
    if (ix >= nx || iy >= s.yr) return;
    const int z0 = s.zl + blockIdx.z * s.zc;
    const int z1 = min(z0 + s.zc, s.zr);
    const int sy = p.L.px, sz = p.L.sz;
    const int bxr = p.bc[MFD_XR], byr = p.bc[MFD_YR], bzr = p.bc[MFD_ZR];
    const bool xr = ix == nx - 1, yr = iy == ny - 1;
    const int ox = !xr ? 1 : (bxr == MFD_BC_PERIODIC ? -(nx - 1) : 0);
    const int oy = !yr ? sy : (byr == MFD_BC_PERIODIC ? -(ny - 1) * sy : 0);
    const int ozw = bzr == MFD_BC_PERIODIC ? -(nz - 1) * sz : 0;
    const int zlast_zero = bzr == MFD_BC_DIRICHLET ? nz - 1 : -1;
    const bool zx = xr && bxr == MFD_BC_DIRICHLET, zy = yr && byr == MFD_BC_DIRICHLET;
    const XCol<T> X = xcol<T>(p.lay[MFD_XL], p.lay[MFD_XR], ix, 2, 3);   // H uses psi pair (2, 3)
    const int kstep = X.nb * ny;
    int k = X.q + X.nb * (iy + ny * z0);
    const T dt = p.dt, Mh0 = p.Mh0;
    const T* __restrict__ Ex = p.Ex;
    const T* __restrict__ Ey = p.Ey;
    const T* __restrict__ Ez = p.Ez;
    T* Hx = p.Hx;
    T* Hy = p.Hy;
    T* Hz = p.Hz;
    T* Sa = p.Sa;
    T* E2 = p.E2;
    int c = ix + sy * iy + sz * z0;
    T ex = Ex[c], ey = Ey[c];
    auto load = [&](int cc, int iz, int kk) {
        HCoreLoad<T> v;
        const int oz = iz < nz - 1 ? sz : ozw;
        v.ez = Ez[cc];
        v.eyx = Ey[cc + ox];
        v.ezx = Ez[cc + ox];
        v.exy = Ex[cc + oy];
        v.ezy = Ez[cc + oy];
        v.exz = Ex[cc + oz];
        v.eyz = Ey[cc + oz];
        v.hx = Hx[cc];
        v.hy = Hy[cc];
        v.hz = Hz[cc];
        v.sa = ACC ? Sa[cc] : T(0);
        v.e2 = (ACC && E2S) ? E2[cc] : T(0);
        v.g = MATH ? (int)p.geom[cc] : 0;
        v.pa = X.in ? X.pa[kk] : T(0);
        v.pb = X.in ? X.pb[kk] : T(0);
        return v;
    };
    HCoreLoad<T> cur = load(c, z0, k);
    for (int iz = z0; iz < z1; ++iz, c += sz, k += kstep) {
        HCoreLoad<T> nxt;
        if (iz + 1 < z1) nxt = load(c + sz, iz + 1, k + kstep);
        const T ez = cur.ez;
        const T ey_xp = zx ? T(0) : cur.eyx, ez_xp = zx ? T(0) : cur.ezx;
        const T ex_yp = zy ? T(0) : cur.exy, ez_yp = zy ? T(0) : cur.ezy;
        const bool zz = iz == zlast_zero;
        const T ex_zp = zz ? T(0) : cur.exz, ey_zp = zz ? T(0) : cur.eyz;
        T hx = cur.hx, hy = cur.hy, hz = cur.hz;
        if (ACC) {
            const T a = mad<FAST>(ey, hz, -(ez * hy)), b = mad<FAST>(ez, hx, -(ex * hz)), d = mad<FAST>(ex, hy, -(ey * hx));
            Sa[c] = mad<FAST>(sqrtm<FAST>(sum3sq<FAST>(a, b, d)), dt, cur.sa);
            if (E2S) E2[c] = mad<FAST>(sum3sq<FAST>(ex, ey, ez), dt, cur.e2);
            if (maybe_nonfinite(ex)) guard(p, ex);
        }
        T Mh = Mh0;
        if (MATH && cur.g) Mh = p.matMh[cur.g - 1];
        const T num[6] = {ex_yp - ex, ex_zp - ex, ey_xp - ey, ey_zp - ey, ez_xp - ez, ez_yp - ez};
        T q[6];
        curl_div<T, FAST>(D3, p.ddx, p.ddy, p.ddz, num, q);
        const T dExy = q[0], dExz = q[1], dEyz = q[3], dEzy = q[5];
        T dEyx = q[2], dEzx = q[4];
        if (X.in) {   // cpml_h<+1> of the column's x face
            const T pa = mad<FAST>(X.B, cur.pa, X.A * dEyx);
            const T pb = mad<FAST>(X.B, cur.pb, X.A * dEzx);
            X.pa[k] = pa;
            X.pb[k] = pb;
            hy = mad<FAST>(Mh, pb, hy);
            hz = mad<FAST>(-Mh, pa, hz);
            dEyx = cdiv<FAST>(dEyx, X.K);
            dEzx = cdiv<FAST>(dEzx, X.K);
        }
        hx = mad<FAST>(-Mh, dEzy - dEyz, hx);
        hy = mad<FAST>(-Mh, dExz - dEzx, hy);
        hz = mad<FAST>(-Mh, dEyx - dExy, hz);
        Hx[c] = hx;
        Hy[c] = hy;
        Hz[c] = hz;
        ex = cur.exz;
        ey = cur.eyz;
        cur = nxt;
    }
}

// One cell of the 3-D H update with every CPML face it lies in (one thread per cell; also the
// cell code of batched 3-D models).  prev_step indexes the NaN/Inf flags of the running sums.
template <typename T, bool MATH, int FAST, bool ACC, bool E2S>
__device__ __forceinline__ void h3d_cell(const HParams<T>& p, const Div3& D3, long long prev_step, int ix, int iy, int iz) {
    const int nx = p.L.nx, ny = p.L.ny, nz = p.L.nz;
    const int sy = p.L.px, sz = p.L.sz;
    const int bxr = p.bc[MFD_XR], byr = p.bc[MFD_YR], bzr = p.bc[MFD_ZR];
    const bool xr = ix == nx - 1, yr = iy == ny - 1, zr = iz == nz - 1;
    const int ox = !xr ? 1 : (bxr == MFD_BC_PERIODIC ? -(nx - 1) : 0);
    const int oy = !yr ? sy : (byr == MFD_BC_PERIODIC ? -(ny - 1) * sy : 0);
    const int oz = !zr ? sz : (bzr == MFD_BC_PERIODIC ? -(nz - 1) * sz : 0);
    const bool zx = xr && bxr == MFD_BC_DIRICHLET, zy = yr && byr == MFD_BC_DIRICHLET, zz = zr && bzr == MFD_BC_DIRICHLET;
    const int c = ix + sy * iy + sz * iz;
    const T ex = p.Ex[c], ey = p.Ey[c], ez = p.Ez[c];
    const T ey_xp = zx ? T(0) : p.Ey[c + ox], ez_xp = zx ? T(0) : p.Ez[c + ox];
    const T ex_yp = zy ? T(0) : p.Ex[c + oy], ez_yp = zy ? T(0) : p.Ez[c + oy];
    const T ex_zp = zz ? T(0) : p.Ex[c + oz], ey_zp = zz ? T(0) : p.Ey[c + oz];
    T hx = p.Hx[c], hy = p.Hy[c], hz = p.Hz[c];
    if (ACC) {
        const T a = mad<FAST>(ey, hz, -(ez * hy)), b = mad<FAST>(ez, hx, -(ex * hz)), d = mad<FAST>(ex, hy, -(ey * hx));
        p.Sa[c] = mad<FAST>(sqrtm<FAST>(sum3sq<FAST>(a, b, d)), p.dt, p.Sa[c]);
        if (E2S) p.E2[c] = mad<FAST>(sum3sq<FAST>(ex, ey, ez), p.dt, p.E2[c]);
        if (maybe_nonfinite(ex)) guard_at(p.flags, prev_step, ex);
    }
    T Mh = p.Mh0;
    if (MATH) {
        const int g = p.geom[c];
        if (g) Mh = p.matMh[g - 1];
    }
    const T num[6] = {ex_yp - ex, ex_zp - ex, ey_xp - ey, ey_zp - ey, ez_xp - ez, ez_yp - ez};
    T q[6];
    curl_div<T, FAST>(D3, p.ddx, p.ddy, p.ddz, num, q);
    T dExy = q[0], dExz = q[1], dEyx = q[2], dEyz = q[3], dEzx = q[4], dEzy = q[5];
    const LayerDev<T>&lxl = p.lay[MFD_XL], &lxr = p.lay[MFD_XR], &lyl = p.lay[MFD_YL], &lyr = p.lay[MFD_YR],
                          &lzl = p.lay[MFD_ZL], &lzr = p.lay[MFD_ZR];
    if (lxl.nb && ix < lxl.ib) cpml_h<+1, FAST>(lxl, ix, ix + lxl.nb * (iy + ny * iz), Mh, dEyx, dEzx, hy, hz);
    if (lxr.nb && ix >= lxr.ib - 1) {
        const int qq = ix - (lxr.ib - 1);
        cpml_h<+1, FAST>(lxr, qq, qq + lxr.nb * (iy + ny * iz), Mh, dEyx, dEzx, hy, hz);
    }
    if (lyl.nb && iy < lyl.ib) cpml_h<-1, FAST>(lyl, iy, ix + sy * (iy + lyl.nb * iz), Mh, dExy, dEzy, hx, hz);
    if (lyr.nb && iy >= lyr.ib - 1) {
        const int qq = iy - (lyr.ib - 1);
        cpml_h<-1, FAST>(lyr, qq, ix + sy * (qq + lyr.nb * iz), Mh, dExy, dEzy, hx, hz);
    }
    if (lzl.nb && iz < lzl.ib) cpml_h<+1, FAST>(lzl, iz, ix + sy * (iy + ny * iz), Mh, dExz, dEyz, hx, hy);
    if (lzr.nb && iz >= lzr.ib - 1) {
        const int qq = iz - (lzr.ib - 1);
        cpml_h<+1, FAST>(lzr, qq, ix + sy * (iy + ny * qq), Mh, dExz, dEyz, hx, hy);
    }
    hx = mad<FAST>(-Mh, dEzy - dEyz, hx);
    hy = mad<FAST>(-Mh, dExz - dEzx, hy);
    hz = mad<FAST>(-Mh, dEyx - dExy, hz);
    p.Hx[c] = hx;
    p.Hy[c] = hy;
    p.Hz[c] = hz;
}

template <typename T, bool MATH, int FAST, bool ACC, bool E2S>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? MFD_SLAB_MINB : 1) h3d_slab_kernel(const __grid_constant__ HParams<T> p, const Div3 D3,
                                                       const SplitBox s) {
    const int ix = blockIdx.y * blockDim.x + threadIdx.x;
    if (ix >= p.L.nx) return;
    int iy, iz;
    slab_row(s, p.L.ny, (int)blockIdx.x, iy, iz);
    h3d_cell<T, MATH, FAST, ACC, E2S>(p, D3, p.prev_step, ix, iy, iz);
}

template <typename T>
struct ECoreLoad {
    T hx, hy, hz, hyx, hzx, hxy, hzy, dx, dy, dz, pa, pb;
    int g;
};

// RESP: the cells of dispersive, Kerr or plasma materials also take their material response
// here (material_cell, models.jl:1042-1154), right after their D update, instead of in the
// material kernel that otherwise follows the E update; cur is the ADE ping-pong parity.
// The response reads only the cell's own E^n (not yet overwritten: such cells skip E = D Me),
// D, polarisation and plasma state, so doing it cell by cell inside the E update changes
// nothing.  The engine uses it when every such material lies in the core rows this kernel
// covers.
template <typename T, typename R, bool MAT, int FAST, bool RESP = false>
__global__ void __launch_bounds__(256, RESP ? 2 : (sizeof(T) == 4 ? MFD_CORE_MINB : 2))
    e3d_core_kernel(const __grid_constant__ EParams<T, R> p, const Div3 D3, const SplitBox s, const int cur = 0,
                    const int xoff = 0) {
    const int ix = xoff + blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = s.yl + blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = p.L.nx, ny = p.L.ny, nz = p.L.nz;
    if (ix >= nx || iy >= s.yr) return;
    const int z0 = s.zl + blockIdx.z * s.zc;
    const int z1 = min(z0 + s.zc, s.zr);
    const int sy = p.L.px, sz = p.L.sz;
    const int bxl = p.bc[MFD_XL], byl = p.bc[MFD_YL], bzl = p.bc[MFD_ZL];
    const bool xl = ix == 0, yl = iy == 0;
    const int ox = !xl ? -1 : (bxl == MFD_BC_PERIODIC ? nx - 1 : 0);
    const int oy = !yl ? -sy : (byl == MFD_BC_PERIODIC ? (ny - 1) * sy : 0);
    const bool zx = xl && bxl == MFD_BC_DIRICHLET, zy = yl && byl == MFD_BC_DIRICHLET;
    const XCol<T> X = xcol<T>(p.lay[MFD_XL], p.lay[MFD_XR], ix, 0, 1);   // E uses psi pair (0, 1)
    const int kstep = X.nb * ny;
    int k = X.q + X.nb * (iy + ny * z0);
    const T Md10 = p.Md10, Md20 = p.Md20, Me0 = p.Me0;
    const T* __restrict__ Hx = p.Hx;
    const T* __restrict__ Hy = p.Hy;
    const T* __restrict__ Hz = p.Hz;
    T* Dx = p.Dx;
    T* Dy = p.Dy;
    T* Dz = p.Dz;
    T* Ex = p.Ex;
    T* Ey = p.Ey;
    T* Ez = p.Ez;
    int c = ix + sy * iy + sz * z0;
    T hx_zm, hy_zm;
    if (z0 > 0) {
        hx_zm = Hx[c - sz];
        hy_zm = Hy[c - sz];
    } else {
        const int oz = bzl == MFD_BC_PERIODIC ? (nz - 1) * sz : 0;
        hx_zm = bzl == MFD_BC_DIRICHLET ? T(0) : Hx[c + oz];
        hy_zm = bzl == MFD_BC_DIRICHLET ? T(0) : Hy[c + oz];
    }
    auto load = [&](int cc, int kk) {
        ECoreLoad<T> v;
        v.hx = Hx[cc];
        v.hy = Hy[cc];
        v.hz = Hz[cc];
        v.hyx = Hy[cc + ox];
        v.hzx = Hz[cc + ox];
        v.hxy = Hx[cc + oy];
        v.hzy = Hz[cc + oy];
        v.dx = Dx[cc];
        v.dy = Dy[cc];
        v.dz = Dz[cc];
        v.g = MAT ? (int)p.geom[cc] : 0;
        v.pa = X.in ? X.pa[kk] : T(0);
        v.pb = X.in ? X.pb[kk] : T(0);
        return v;
    };
    ECoreLoad<T> ld = load(c, k);
    for (int iz = z0; iz < z1; ++iz, c += sz, k += kstep) {
        ECoreLoad<T> nxt;
        if (iz + 1 < z1) nxt = load(c + sz, k + kstep);
        const T hx = ld.hx, hy = ld.hy, hz = ld.hz;
        const T hy_xm = zx ? T(0) : ld.hyx, hz_xm = zx ? T(0) : ld.hzx;
        const T hx_ym = zy ? T(0) : ld.hxy, hz_ym = zy ? T(0) : ld.hzy;
        const T num[6] = {hx - hx_ym, hx - hx_zm, hy - hy_xm, hy - hy_zm, hz - hz_xm, hz - hz_ym};
        T q[6];
        curl_div<T, FAST>(D3, p.ddx, p.ddy, p.ddz, num, q);
        const T dHxy = q[0], dHxz = q[1], dHyz = q[3], dHzy = q[5];
        T dHyx = q[2], dHzx = q[4];
        T Md1 = Md10, Md2 = Md20, Me = Me0;
        bool simple = true;
        if (MAT && ld.g) {
            const MatDev<T, R>& m = p.mats[ld.g - 1];
            Md1 = m.Md1; Md2 = m.Md2; Me = m.Me; simple = m.simple != 0;
        }
        T D0 = ld.dx, D1 = ld.dy, D2 = ld.dz;
        if (X.in) {   // cpml_e<-1> of the column's x face
            const T pa = mad<FAST>(X.B, ld.pa, X.A * dHyx);
            const T pb = mad<FAST>(X.B, ld.pb, X.A * dHzx);
            X.pa[k] = pa;
            X.pb[k] = pb;
            D1 = mad<FAST>(-Md2, pb, D1);
            D2 = mad<FAST>(Md2, pa, D2);
            dHyx = cdiv<FAST>(dHyx, X.K);
            dHzx = cdiv<FAST>(dHzx, X.K);
        }
        D0 = mad<FAST>(Md1, D0, Md2 * (dHzy - dHyz));
        D1 = mad<FAST>(Md1, D1, Md2 * (dHxz - dHzx));
        D2 = mad<FAST>(Md1, D2, Md2 * (dHyx - dHxy));
        if (RESP && !simple) {
            // The response before this cell's D stores (it takes D from registers).  In
            // single precision the pole count is a template argument: every load it makes
            // (E^n, both buffers of every pole, the plasma state) is then issued at once
            // instead of one pole buffer per round trip.  Double precision keeps the pole
            // loop (the unrolled form spills there).
            const MatDev<T, R>* mm = p.mats + (ld.g - 1);
            T* Ep[3] = {Ex, Ey, Ez};
            const T Dv[3] = {D0, D1, D2};
            if constexpr (sizeof(T) == 4) {
                const long long bi = (long long)(ix - mm->bx0) +
                                     (long long)mm->bnx * ((long long)(iy - mm->by0) + (long long)mm->bny * (iz - mm->bz0));
                switch (mm->nq) {
                    case 0: material_cell_n<T, R, 3, 0>(mm, bi, Ep, c, Dv, cur, p.dt); break;
                    case 1: material_cell_n<T, R, 3, 1>(mm, bi, Ep, c, Dv, cur, p.dt); break;
                    case 2: material_cell_n<T, R, 3, 2>(mm, bi, Ep, c, Dv, cur, p.dt); break;
                    case 3: material_cell_n<T, R, 3, 3>(mm, bi, Ep, c, Dv, cur, p.dt); break;
                    default: material_cell<T, R, 3>(mm, ix, iy, iz, Ep, c, Dv, cur, p.dt); break;
                }
            } else {
                material_cell<T, R, 3>(mm, ix, iy, iz, Ep, c, Dv, cur, p.dt);
            }
        }
        Dx[c] = D0;
        Dy[c] = D1;
        Dz[c] = D2;
        if (simple) {
            Ex[c] = D0 * Me;
            Ey[c] = D1 * Me;
            Ez[c] = D2 * Me;
        }
        hx_zm = hx;
        hy_zm = hy;
        ld = nxt;
    }
}

// One cell of the 3-D E update with every CPML face it lies in (also the cell code of batched
// 3-D models).
template <typename T, typename R, bool MAT, int FAST>
__device__ __forceinline__ void e3d_cell(const EParams<T, R>& p, const Div3& D3, int ix, int iy, int iz) {
    const int nx = p.L.nx, ny = p.L.ny, nz = p.L.nz;
    const int sy = p.L.px, sz = p.L.sz;
    const int bxl = p.bc[MFD_XL], byl = p.bc[MFD_YL], bzl = p.bc[MFD_ZL];
    const bool xl = ix == 0, yl = iy == 0, zl = iz == 0;
    const int ox = !xl ? -1 : (bxl == MFD_BC_PERIODIC ? nx - 1 : 0);
    const int oy = !yl ? -sy : (byl == MFD_BC_PERIODIC ? (ny - 1) * sy : 0);
    const int oz = !zl ? -sz : (bzl == MFD_BC_PERIODIC ? (nz - 1) * sz : 0);
    const bool zx = xl && bxl == MFD_BC_DIRICHLET, zy = yl && byl == MFD_BC_DIRICHLET, zz = zl && bzl == MFD_BC_DIRICHLET;
    const int c = ix + sy * iy + sz * iz;
    const T hx = p.Hx[c], hy = p.Hy[c], hz = p.Hz[c];
    const T hy_xm = zx ? T(0) : p.Hy[c + ox], hz_xm = zx ? T(0) : p.Hz[c + ox];
    const T hx_ym = zy ? T(0) : p.Hx[c + oy], hz_ym = zy ? T(0) : p.Hz[c + oy];
    const T hx_zm = zz ? T(0) : p.Hx[c + oz], hy_zm = zz ? T(0) : p.Hy[c + oz];
    const T num[6] = {hx - hx_ym, hx - hx_zm, hy - hy_xm, hy - hy_zm, hz - hz_xm, hz - hz_ym};
    T q[6];
    curl_div<T, FAST>(D3, p.ddx, p.ddy, p.ddz, num, q);
    T dHxy = q[0], dHxz = q[1], dHyx = q[2], dHyz = q[3], dHzx = q[4], dHzy = q[5];
    T Md1 = p.Md10, Md2 = p.Md20, Me = p.Me0;
    bool simple = true;
    if (MAT) {
        const int g = p.geom[c];
        if (g) {
            const MatDev<T, R>& m = p.mats[g - 1];
            Md1 = m.Md1; Md2 = m.Md2; Me = m.Me; simple = m.simple != 0;
        }
    }
    T D0 = p.Dx[c], D1 = p.Dy[c], D2 = p.Dz[c];
    const LayerDev<T>&lxl = p.lay[MFD_XL], &lxr = p.lay[MFD_XR], &lyl = p.lay[MFD_YL], &lyr = p.lay[MFD_YR],
                          &lzl = p.lay[MFD_ZL], &lzr = p.lay[MFD_ZR];
    if (lxl.nb && ix < lxl.ib) cpml_e<-1, FAST>(lxl, ix, ix + lxl.nb * (iy + ny * iz), Md2, dHyx, dHzx, D1, D2);
    if (lxr.nb && ix >= lxr.ib - 1) {
        const int qq = ix - (lxr.ib - 1);
        cpml_e<-1, FAST>(lxr, qq, qq + lxr.nb * (iy + ny * iz), Md2, dHyx, dHzx, D1, D2);
    }
    if (lyl.nb && iy < lyl.ib) cpml_e<+1, FAST>(lyl, iy, ix + sy * (iy + lyl.nb * iz), Md2, dHxy, dHzy, D0, D2);
    if (lyr.nb && iy >= lyr.ib - 1) {
        const int qq = iy - (lyr.ib - 1);
        cpml_e<+1, FAST>(lyr, qq, ix + sy * (qq + lyr.nb * iz), Md2, dHxy, dHzy, D0, D2);
    }
    if (lzl.nb && iz < lzl.ib) cpml_e<-1, FAST>(lzl, iz, ix + sy * (iy + ny * iz), Md2, dHxz, dHyz, D0, D1);
    if (lzr.nb && iz >= lzr.ib - 1) {
        const int qq = iz - (lzr.ib - 1);
        cpml_e<-1, FAST>(lzr, qq, ix + sy * (iy + ny * qq), Md2, dHxz, dHyz, D0, D1);
    }
    D0 = mad<FAST>(Md1, D0, Md2 * (dHzy - dHyz));
    D1 = mad<FAST>(Md1, D1, Md2 * (dHxz - dHzx));
    D2 = mad<FAST>(Md1, D2, Md2 * (dHyx - dHxy));
    p.Dx[c] = D0;
    p.Dy[c] = D1;
    p.Dz[c] = D2;
    if (simple) {
        p.Ex[c] = D0 * Me;
        p.Ey[c] = D1 * Me;
        p.Ez[c] = D2 * Me;
    }
}

template <typename T, typename R, bool MAT, int FAST>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? MFD_SLAB_MINB : 1) e3d_slab_kernel(const __grid_constant__ EParams<T, R> p, const Div3 D3,
                                                       const SplitBox s) {
    const int ix = blockIdx.y * blockDim.x + threadIdx.x;
    if (ix >= p.L.nx) return;
    int iy, iz;
    slab_row(s, p.L.ny, (int)blockIdx.x, iy, iz);
    e3d_cell<T, R, MAT, FAST>(p, D3, ix, iy, iz);
}

}  // namespace mfd
