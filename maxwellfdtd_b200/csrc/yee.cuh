// yee.cuh -- Yee H and E update kernels (1-D, 2-D, 3-D) for sm_100a.
//
// 3-D kernels march along z: a thread owns one (ix, iy) column of a z-chunk and keeps the
// z-neighbour plane in registers (E at iz+1 for the H update, H at iz-1 for the E update),
// so each plane of the read-only field is fetched from memory once per chunk; x and y
// neighbours come from the same or adjacent warps through L1.  The CPML psi recursions are
// fused into the curls, the material response (ADE poles, plasma, Kerr) into the E update,
// and the running sums Sa/E2 of the previous step plus the NaN/Inf guard on Ex into the H
// update, which reads every E and H value of the cell anyway.
//
// Reference kernels: src/models.jl:248-437 (1-D), 450-719 (2-D), 735-1162 (3-D).
#pragma once

#include "mfd_device.cuh"

namespace mfd {

template <typename T>
struct HParams {
    Layout L;
    DivC<T> ddx, ddy, ddz;
    T dt;
    int bc[6];
    LayerDev<T> lay[6];
    T Mh0;
    const uint8_t* __restrict__ geom;
    const T* __restrict__ matMh;     // Mh of material g at matMh[g-1]
    T* Hx; T* Hy; T* Hz;
    const T* __restrict__ Ex; const T* __restrict__ Ey; const T* __restrict__ Ez;
    // running sums of the previous step (outputs.jl:475-485) and NaN/Inf guard (models.jl:202-209)
    int accum;
    int sum_e2;
    T* Sa; T* E2;
    int* flags;            // per-step NaN (bit 0) / Inf (bit 1) flags of Ex, index step-1
    long long prev_step;
};

template <typename T, typename R>
struct EParams {
    Layout L;
    DivC<T> ddx, ddy, ddz;
    T dt;
    int bc[6];
    LayerDev<T> lay[6];
    T Me0, Md10, Md20;
    const uint8_t* __restrict__ geom;
    const MatDev<T, R>* __restrict__ mats;
    const T* __restrict__ Hx; const T* __restrict__ Hy; const T* __restrict__ Hz;
    T* Dx; T* Dy; T* Dz;
    T* Ex; T* Ey; T* Ez;
    int cur;    // ping-pong buffer holding P^n
};

template <typename T>
__device__ __forceinline__ void guard(const HParams<T>& p, T ex) {
    const int bad = (isnan(ex) ? 1 : 0) | (isinf(ex) ? 2 : 0);
    if (bad) atomicOr(p.flags + (p.prev_step - 1), bad);
}

// ------------------------------------------------------------------------------------------
// 3-D
//
// Software-pipelined z march: all loads of plane iz+1 are issued before the arithmetic and
// stores of plane iz, so two planes of memory traffic are in flight per thread.  Boundary
// conditions are folded into per-thread neighbour offsets (periodic: the wrapped cell;
// Neumann: the cell itself; Dirichlet: the cell itself, zeroed after the load), so the
// prefetch never depends on values of the current plane.
// ------------------------------------------------------------------------------------------
template <typename T>
struct HLoad {
    T ez, eyx, ezx, exy, ezy, exz, eyz, hx, hy, hz, sa, e2;
    int g;
};

template <typename T, bool MATH>
__device__ __forceinline__ HLoad<T> h3d_load(const HParams<T>& p, int c, int iz, int ox, int oy, int ozw) {
    HLoad<T> v;
    const int oz = iz < p.L.nz - 1 ? p.L.sz : ozw;
    v.ez = p.Ez[c];
    v.eyx = p.Ey[c + ox];
    v.ezx = p.Ez[c + ox];
    v.exy = p.Ex[c + oy];
    v.ezy = p.Ez[c + oy];
    v.exz = p.Ex[c + oz];
    v.eyz = p.Ey[c + oz];
    v.hx = p.Hx[c];
    v.hy = p.Hy[c];
    v.hz = p.Hz[c];
    if (p.accum) {
        v.sa = p.Sa[c];
        v.e2 = p.sum_e2 ? p.E2[c] : T(0);
    } else {
        v.sa = v.e2 = T(0);
    }
    v.g = MATH ? (int)p.geom[c] : 0;
    return v;
}

template <typename T, bool MATH>
__global__ void __launch_bounds__(256, 4) h3d_kernel(const __grid_constant__ HParams<T> p, const int zc) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = p.L.nx, ny = p.L.ny, nz = p.L.nz;
    if (ix >= nx || iy >= ny) return;
    const int z0 = blockIdx.z * zc;
    const int z1 = min(z0 + zc, nz);
    const int sy = p.L.px, sz = p.L.sz;
    const int bxr = p.bc[MFD_XR], byr = p.bc[MFD_YR], bzr = p.bc[MFD_ZR];
    const bool xr = ix == nx - 1, yr = iy == ny - 1;
    const int ox = !xr ? 1 : (bxr == MFD_BC_PERIODIC ? -(nx - 1) : 0);
    const int oy = !yr ? sy : (byr == MFD_BC_PERIODIC ? -(ny - 1) * sy : 0);
    const int ozw = bzr == MFD_BC_PERIODIC ? -(nz - 1) * sz : 0;
    const bool zx = xr && bxr == MFD_BC_DIRICHLET, zy = yr && byr == MFD_BC_DIRICHLET;
    int c = ix + sy * iy + sz * z0;
    T ex = p.Ex[c], ey = p.Ey[c];
    HLoad<T> cur = h3d_load<T, MATH>(p, c, z0, ox, oy, ozw);
    for (int iz = z0; iz < z1; ++iz, c += sz) {
        HLoad<T> nxt;
        if (iz + 1 < z1) nxt = h3d_load<T, MATH>(p, c + sz, iz + 1, ox, oy, ozw);
        const T ez = cur.ez;
        const T ey_xp = zx ? T(0) : cur.eyx, ez_xp = zx ? T(0) : cur.ezx;
        const T ex_yp = zy ? T(0) : cur.exy, ez_yp = zy ? T(0) : cur.ezy;
        const bool zz = iz == nz - 1 && bzr == MFD_BC_DIRICHLET;
        const T ex_zp = zz ? T(0) : cur.exz, ey_zp = zz ? T(0) : cur.eyz;
        T hx = cur.hx, hy = cur.hy, hz = cur.hz;
        if (p.accum) {
            const T a = ey * hz - ez * hy, b = ez * hx - ex * hz, d = ex * hy - ey * hx;
            p.Sa[c] = cur.sa + sqrt0(a * a + b * b + d * d) * p.dt;
            if (p.sum_e2) p.E2[c] = cur.e2 + (ex * ex + ey * ey + ez * ez) * p.dt;
            guard(p, ex);
        }
        T Mh = p.Mh0;
        if (MATH && cur.g) Mh = p.matMh[cur.g - 1];
        T dExy = cdiv(ex_yp - ex, p.ddy);
        T dExz = cdiv(ex_zp - ex, p.ddz);
        T dEyx = cdiv(ey_xp - ey, p.ddx);
        T dEyz = cdiv(ey_zp - ey, p.ddz);
        T dEzx = cdiv(ez_xp - ez, p.ddx);
        T dEzy = cdiv(ez_yp - ez, p.ddy);
        // CPML (models.jl:811-871)
        {
            const LayerDev<T>& l = p.lay[MFD_XL];
            if (l.nb && ix < l.ib) {
                const int q = ix;
                const int k = q + l.nb * (iy + ny * iz);
                const T B = l.B[q], A = l.A[q];
                const T pEyx = B * l.psi[2][k] + A * dEyx;
                const T pEzx = B * l.psi[3][k] + A * dEzx;
                l.psi[2][k] = pEyx; l.psi[3][k] = pEzx;
                hy += Mh * pEzx;
                hz -= Mh * pEyx;
                dEyx = cdiv(dEyx, l.K[q]);
                dEzx = cdiv(dEzx, l.K[q]);
            }
        }
        {
            const LayerDev<T>& l = p.lay[MFD_XR];
            if (l.nb && ix >= l.ib - 1) {
                const int q = ix - (l.ib - 1);
                const int k = q + l.nb * (iy + ny * iz);
                const T B = l.B[q], A = l.A[q];
                const T pEyx = B * l.psi[2][k] + A * dEyx;
                const T pEzx = B * l.psi[3][k] + A * dEzx;
                l.psi[2][k] = pEyx; l.psi[3][k] = pEzx;
                hy += Mh * pEzx;
                hz -= Mh * pEyx;
                dEyx = cdiv(dEyx, l.K[q]);
                dEzx = cdiv(dEzx, l.K[q]);
            }
        }
        {
            const LayerDev<T>& l = p.lay[MFD_YL];
            if (l.nb && iy < l.ib) {
                const int q = iy;
                const int k = ix + sy * (q + l.nb * iz);
                const T B = l.B[q], A = l.A[q];
                const T pExy = B * l.psi[2][k] + A * dExy;
                const T pEzy = B * l.psi[3][k] + A * dEzy;
                l.psi[2][k] = pExy; l.psi[3][k] = pEzy;
                hx -= Mh * pEzy;
                hz += Mh * pExy;
                dExy = cdiv(dExy, l.K[q]);
                dEzy = cdiv(dEzy, l.K[q]);
            }
        }
        {
            const LayerDev<T>& l = p.lay[MFD_YR];
            if (l.nb && iy >= l.ib - 1) {
                const int q = iy - (l.ib - 1);
                const int k = ix + sy * (q + l.nb * iz);
                const T B = l.B[q], A = l.A[q];
                const T pExy = B * l.psi[2][k] + A * dExy;
                const T pEzy = B * l.psi[3][k] + A * dEzy;
                l.psi[2][k] = pExy; l.psi[3][k] = pEzy;
                hx -= Mh * pEzy;
                hz += Mh * pExy;
                dExy = cdiv(dExy, l.K[q]);
                dEzy = cdiv(dEzy, l.K[q]);
            }
        }
        {
            const LayerDev<T>& l = p.lay[MFD_ZL];
            if (l.nb && iz < l.ib) {
                const int q = iz;
                const int k = ix + sy * (iy + ny * q);
                const T B = l.B[q], A = l.A[q];
                const T pExz = B * l.psi[2][k] + A * dExz;
                const T pEyz = B * l.psi[3][k] + A * dEyz;
                l.psi[2][k] = pExz; l.psi[3][k] = pEyz;
                hx += Mh * pEyz;
                hy -= Mh * pExz;
                dExz = cdiv(dExz, l.K[q]);
                dEyz = cdiv(dEyz, l.K[q]);
            }
        }
        {
            const LayerDev<T>& l = p.lay[MFD_ZR];
            if (l.nb && iz >= l.ib - 1) {
                const int q = iz - (l.ib - 1);
                const int k = ix + sy * (iy + ny * q);
                const T B = l.B[q], A = l.A[q];
                const T pExz = B * l.psi[2][k] + A * dExz;
                const T pEyz = B * l.psi[3][k] + A * dEyz;
                l.psi[2][k] = pExz; l.psi[3][k] = pEyz;
                hx += Mh * pEyz;
                hy -= Mh * pExz;
                dExz = cdiv(dExz, l.K[q]);
                dEyz = cdiv(dEyz, l.K[q]);
            }
        }
        hx -= Mh * (dEzy - dEyz);
        hy -= Mh * (dExz - dEzx);
        hz -= Mh * (dEyx - dExy);
        p.Hx[c] = hx; p.Hy[c] = hy; p.Hz[c] = hz;
        ex = cur.exz;
        ey = cur.eyz;
        cur = nxt;
    }
}

template <typename T>
struct ELoad {
    T hx, hy, hz, hyx, hzx, hxy, hzy, dx, dy, dz;
    int g;
};

template <typename T, typename R, bool MAT>
__device__ __forceinline__ ELoad<T> e3d_load(const EParams<T, R>& p, int c, int ox, int oy) {
    ELoad<T> v;
    v.hx = p.Hx[c];
    v.hy = p.Hy[c];
    v.hz = p.Hz[c];
    v.hyx = p.Hy[c + ox];
    v.hzx = p.Hz[c + ox];
    v.hxy = p.Hx[c + oy];
    v.hzy = p.Hz[c + oy];
    v.dx = p.Dx[c];
    v.dy = p.Dy[c];
    v.dz = p.Dz[c];
    v.g = MAT ? (int)p.geom[c] : 0;
    return v;
}

template <typename T, typename R, bool MAT>
__global__ void __launch_bounds__(256, 4) e3d_kernel(const __grid_constant__ EParams<T, R> p, const int zc) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = p.L.nx, ny = p.L.ny, nz = p.L.nz;
    if (ix >= nx || iy >= ny) return;
    const int z0 = blockIdx.z * zc;
    const int z1 = min(z0 + zc, nz);
    const int sy = p.L.px, sz = p.L.sz;
    const int bxl = p.bc[MFD_XL], byl = p.bc[MFD_YL], bzl = p.bc[MFD_ZL];
    const bool xl = ix == 0, yl = iy == 0;
    const int ox = !xl ? -1 : (bxl == MFD_BC_PERIODIC ? nx - 1 : 0);
    const int oy = !yl ? -sy : (byl == MFD_BC_PERIODIC ? (ny - 1) * sy : 0);
    const bool zx = xl && bxl == MFD_BC_DIRICHLET, zy = yl && byl == MFD_BC_DIRICHLET;
    int c = ix + sy * iy + sz * z0;
    T hx_zm, hy_zm;
    if (z0 > 0) {
        hx_zm = p.Hx[c - sz];
        hy_zm = p.Hy[c - sz];
    } else {
        const int oz = bzl == MFD_BC_PERIODIC ? (nz - 1) * sz : 0;
        hx_zm = bzl == MFD_BC_DIRICHLET ? T(0) : p.Hx[c + oz];
        hy_zm = bzl == MFD_BC_DIRICHLET ? T(0) : p.Hy[c + oz];
    }
    T* const Ep[3] = {p.Ex, p.Ey, p.Ez};
    ELoad<T> cur = e3d_load<T, R, MAT>(p, c, ox, oy);
    for (int iz = z0; iz < z1; ++iz, c += sz) {
        ELoad<T> nxt;
        if (iz + 1 < z1) nxt = e3d_load<T, R, MAT>(p, c + sz, ox, oy);
        const T hx = cur.hx, hy = cur.hy, hz = cur.hz;
        const T hy_xm = zx ? T(0) : cur.hyx, hz_xm = zx ? T(0) : cur.hzx;
        const T hx_ym = zy ? T(0) : cur.hxy, hz_ym = zy ? T(0) : cur.hzy;
        T dHxy = cdiv(hx - hx_ym, p.ddy);
        T dHxz = cdiv(hx - hx_zm, p.ddz);
        T dHyx = cdiv(hy - hy_xm, p.ddx);
        T dHyz = cdiv(hy - hy_zm, p.ddz);
        T dHzx = cdiv(hz - hz_xm, p.ddx);
        T dHzy = cdiv(hz - hz_ym, p.ddy);
        const int g = cur.g;
        T Md1 = p.Md10, Md2 = p.Md20;
        if (MAT && g) { Md1 = p.mats[g - 1].Md1; Md2 = p.mats[g - 1].Md2; }
        T Dv[3] = {cur.dx, cur.dy, cur.dz};
        // CPML (models.jl:975-1035)
        {
            const LayerDev<T>& l = p.lay[MFD_XL];
            if (l.nb && ix < l.ib) {
                const int q = ix;
                const int k = q + l.nb * (iy + ny * iz);
                const T B = l.B[q], A = l.A[q];
                const T pHyx = B * l.psi[0][k] + A * dHyx;
                const T pHzx = B * l.psi[1][k] + A * dHzx;
                l.psi[0][k] = pHyx; l.psi[1][k] = pHzx;
                Dv[1] -= Md2 * pHzx;
                Dv[2] += Md2 * pHyx;
                dHyx = cdiv(dHyx, l.K[q]);
                dHzx = cdiv(dHzx, l.K[q]);
            }
        }
        {
            const LayerDev<T>& l = p.lay[MFD_XR];
            if (l.nb && ix >= l.ib - 1) {
                const int q = ix - (l.ib - 1);
                const int k = q + l.nb * (iy + ny * iz);
                const T B = l.B[q], A = l.A[q];
                const T pHyx = B * l.psi[0][k] + A * dHyx;
                const T pHzx = B * l.psi[1][k] + A * dHzx;
                l.psi[0][k] = pHyx; l.psi[1][k] = pHzx;
                Dv[1] -= Md2 * pHzx;
                Dv[2] += Md2 * pHyx;
                dHyx = cdiv(dHyx, l.K[q]);
                dHzx = cdiv(dHzx, l.K[q]);
            }
        }
        {
            const LayerDev<T>& l = p.lay[MFD_YL];
            if (l.nb && iy < l.ib) {
                const int q = iy;
                const int k = ix + sy * (q + l.nb * iz);
                const T B = l.B[q], A = l.A[q];
                const T pHxy = B * l.psi[0][k] + A * dHxy;
                const T pHzy = B * l.psi[1][k] + A * dHzy;
                l.psi[0][k] = pHxy; l.psi[1][k] = pHzy;
                Dv[0] += Md2 * pHzy;
                Dv[2] -= Md2 * pHxy;
                dHxy = cdiv(dHxy, l.K[q]);
                dHzy = cdiv(dHzy, l.K[q]);
            }
        }
        {
            const LayerDev<T>& l = p.lay[MFD_YR];
            if (l.nb && iy >= l.ib - 1) {
                const int q = iy - (l.ib - 1);
                const int k = ix + sy * (q + l.nb * iz);
                const T B = l.B[q], A = l.A[q];
                const T pHxy = B * l.psi[0][k] + A * dHxy;
                const T pHzy = B * l.psi[1][k] + A * dHzy;
                l.psi[0][k] = pHxy; l.psi[1][k] = pHzy;
                Dv[0] += Md2 * pHzy;
                Dv[2] -= Md2 * pHxy;
                dHxy = cdiv(dHxy, l.K[q]);
                dHzy = cdiv(dHzy, l.K[q]);
            }
        }
        {
            const LayerDev<T>& l = p.lay[MFD_ZL];
            if (l.nb && iz < l.ib) {
                const int q = iz;
                const int k = ix + sy * (iy + ny * q);
                const T B = l.B[q], A = l.A[q];
                const T pHxz = B * l.psi[0][k] + A * dHxz;
                const T pHyz = B * l.psi[1][k] + A * dHyz;
                l.psi[0][k] = pHxz; l.psi[1][k] = pHyz;
                Dv[0] -= Md2 * pHyz;
                Dv[1] += Md2 * pHxz;
                dHxz = cdiv(dHxz, l.K[q]);
                dHyz = cdiv(dHyz, l.K[q]);
            }
        }
        {
            const LayerDev<T>& l = p.lay[MFD_ZR];
            if (l.nb && iz >= l.ib - 1) {
                const int q = iz - (l.ib - 1);
                const int k = ix + sy * (iy + ny * q);
                const T B = l.B[q], A = l.A[q];
                const T pHxz = B * l.psi[0][k] + A * dHxz;
                const T pHyz = B * l.psi[1][k] + A * dHyz;
                l.psi[0][k] = pHxz; l.psi[1][k] = pHyz;
                Dv[0] -= Md2 * pHyz;
                Dv[1] += Md2 * pHxz;
                dHxz = cdiv(dHxz, l.K[q]);
                dHyz = cdiv(dHyz, l.K[q]);
            }
        }
        Dv[0] = Md1 * Dv[0] + Md2 * (dHzy - dHyz);
        Dv[1] = Md1 * Dv[1] + Md2 * (dHxz - dHzx);
        Dv[2] = Md1 * Dv[2] + Md2 * (dHyx - dHxy);
        p.Dx[c] = Dv[0]; p.Dy[c] = Dv[1]; p.Dz[c] = Dv[2];
        if (MAT && g) {
            material_cell<T, R, 3>(p.mats + (g - 1), ix, iy, iz, Ep, c, Dv, p.cur, p.dt);
        } else {
            p.Ex[c] = Dv[0] * p.Me0;
            p.Ey[c] = Dv[1] * p.Me0;
            p.Ez[c] = Dv[2] * p.Me0;
        }
        hx_zm = hx;
        hy_zm = hy;
        cur = nxt;
    }
}

// ------------------------------------------------------------------------------------------
// 2-D (x-z plane): one thread per cell
// ------------------------------------------------------------------------------------------
template <typename T, bool MATH>
__global__ void __launch_bounds__(256) h2d_kernel(const __grid_constant__ HParams<T> p) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iz = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = p.L.nx, nz = p.L.nz;
    if (ix >= nx || iz >= nz) return;
    const int sz = p.L.sz;
    const int c = ix + sz * iz;
    const T ex = p.Ex[c], ez = p.Ez[c];
    T ez_xp, ex_zp;
    if (ix < nx - 1) ez_xp = p.Ez[c + 1];
    else { const int b = p.bc[MFD_XR]; ez_xp = bc_value(b, b == MFD_BC_PERIODIC ? p.Ez[c - (nx - 1)] : T(0), ez); }
    if (iz < nz - 1) ex_zp = p.Ex[c + sz];
    else { const int b = p.bc[MFD_ZR]; ex_zp = bc_value(b, b == MFD_BC_PERIODIC ? p.Ex[c - (nz - 1) * sz] : T(0), ex); }
    T hy = p.Hy[c];
    if (p.accum) {
        const T a = -ez * hy, b = ex * hy;
        p.Sa[c] = p.Sa[c] + sqrt0(a * a + b * b) * p.dt;
        if (p.sum_e2) p.E2[c] = p.E2[c] + (ex * ex + ez * ez) * p.dt;
        guard(p, ex);
    }
    T Mh = p.Mh0;
    if (MATH) { const int g = p.geom[c]; if (g) Mh = p.matMh[g - 1]; }
    T dExz = cdiv(ex_zp - ex, p.ddz);
    T dEzx = cdiv(ez_xp - ez, p.ddx);
    {
        const LayerDev<T>& l = p.lay[MFD_XL];
        if (l.nb && ix < l.ib) {
            const int q = ix;
            const int k = q + l.nb * iz;
            const T ps = l.B[q] * l.psi[1][k] + l.A[q] * dEzx;
            l.psi[1][k] = ps;
            hy += Mh * ps;
            dEzx = cdiv(dEzx, l.K[q]);
        }
    }
    {
        const LayerDev<T>& l = p.lay[MFD_XR];
        if (l.nb && ix >= l.ib - 1) {
            const int q = ix - (l.ib - 1);
            const int k = q + l.nb * iz;
            const T ps = l.B[q] * l.psi[1][k] + l.A[q] * dEzx;
            l.psi[1][k] = ps;
            hy += Mh * ps;
            dEzx = cdiv(dEzx, l.K[q]);
        }
    }
    {
        const LayerDev<T>& l = p.lay[MFD_ZL];
        if (l.nb && iz < l.ib) {
            const int q = iz;
            const int k = ix + p.L.px * q;
            const T ps = l.B[q] * l.psi[1][k] + l.A[q] * dExz;
            l.psi[1][k] = ps;
            hy -= Mh * ps;
            dExz = cdiv(dExz, l.K[q]);
        }
    }
    {
        const LayerDev<T>& l = p.lay[MFD_ZR];
        if (l.nb && iz >= l.ib - 1) {
            const int q = iz - (l.ib - 1);
            const int k = ix + p.L.px * q;
            const T ps = l.B[q] * l.psi[1][k] + l.A[q] * dExz;
            l.psi[1][k] = ps;
            hy -= Mh * ps;
            dExz = cdiv(dExz, l.K[q]);
        }
    }
    hy -= Mh * (dExz - dEzx);
    p.Hy[c] = hy;
}

template <typename T, typename R, bool MAT>
__global__ void __launch_bounds__(256) e2d_kernel(const __grid_constant__ EParams<T, R> p) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iz = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = p.L.nx, nz = p.L.nz;
    if (ix >= nx || iz >= nz) return;
    const int sz = p.L.sz;
    const int c = ix + sz * iz;
    const T hy = p.Hy[c];
    T hy_xm, hy_zm;
    if (ix > 0) hy_xm = p.Hy[c - 1];
    else { const int b = p.bc[MFD_XL]; hy_xm = bc_value(b, b == MFD_BC_PERIODIC ? p.Hy[c + (nx - 1)] : T(0), hy); }
    if (iz > 0) hy_zm = p.Hy[c - sz];
    else { const int b = p.bc[MFD_ZL]; hy_zm = bc_value(b, b == MFD_BC_PERIODIC ? p.Hy[c + (nz - 1) * sz] : T(0), hy); }
    T dHyx = cdiv(hy - hy_xm, p.ddx);
    T dHyz = cdiv(hy - hy_zm, p.ddz);
    int g = 0;
    T Md1 = p.Md10, Md2 = p.Md20;
    if (MAT) {
        g = p.geom[c];
        if (g) { Md1 = p.mats[g - 1].Md1; Md2 = p.mats[g - 1].Md2; }
    }
    T Dv[2] = {p.Dx[c], p.Dz[c]};
    {
        const LayerDev<T>& l = p.lay[MFD_XL];
        if (l.nb && ix < l.ib) {
            const int q = ix;
            const int k = q + l.nb * iz;
            const T ps = l.B[q] * l.psi[0][k] + l.A[q] * dHyx;
            l.psi[0][k] = ps;
            Dv[1] += Md2 * ps;
            dHyx = cdiv(dHyx, l.K[q]);
        }
    }
    {
        const LayerDev<T>& l = p.lay[MFD_XR];
        if (l.nb && ix >= l.ib - 1) {
            const int q = ix - (l.ib - 1);
            const int k = q + l.nb * iz;
            const T ps = l.B[q] * l.psi[0][k] + l.A[q] * dHyx;
            l.psi[0][k] = ps;
            Dv[1] += Md2 * ps;
            dHyx = cdiv(dHyx, l.K[q]);
        }
    }
    {
        const LayerDev<T>& l = p.lay[MFD_ZL];
        if (l.nb && iz < l.ib) {
            const int q = iz;
            const int k = ix + p.L.px * q;
            const T ps = l.B[q] * l.psi[0][k] + l.A[q] * dHyz;
            l.psi[0][k] = ps;
            Dv[0] -= Md2 * ps;
            dHyz = cdiv(dHyz, l.K[q]);
        }
    }
    {
        const LayerDev<T>& l = p.lay[MFD_ZR];
        if (l.nb && iz >= l.ib - 1) {
            const int q = iz - (l.ib - 1);
            const int k = ix + p.L.px * q;
            const T ps = l.B[q] * l.psi[0][k] + l.A[q] * dHyz;
            l.psi[0][k] = ps;
            Dv[0] -= Md2 * ps;
            dHyz = cdiv(dHyz, l.K[q]);
        }
    }
    Dv[0] = Md1 * Dv[0] + Md2 * (T(0) - dHyz);
    Dv[1] = Md1 * Dv[1] + Md2 * (dHyx - T(0));
    p.Dx[c] = Dv[0]; p.Dz[c] = Dv[1];
    if (MAT && g) {
        T* const Ep[2] = {p.Ex, p.Ez};
        material_cell<T, R, 2>(p.mats + (g - 1), ix, 0, iz, Ep, c, Dv, p.cur, p.dt);
    } else {
        p.Ex[c] = Dv[0] * p.Me0;
        p.Ez[c] = Dv[1] * p.Me0;
    }
}

// ------------------------------------------------------------------------------------------
// 1-D (z)
// ------------------------------------------------------------------------------------------
template <typename T, bool MATH>
__global__ void __launch_bounds__(256) h1d_kernel(const __grid_constant__ HParams<T> p) {
    const int iz = blockIdx.x * blockDim.x + threadIdx.x;
    const int nz = p.L.nz;
    if (iz >= nz) return;
    const int c = iz;
    const T ex = p.Ex[c];
    T ex_zp;
    if (iz < nz - 1) ex_zp = p.Ex[c + 1];
    else { const int b = p.bc[MFD_ZR]; ex_zp = bc_value(b, b == MFD_BC_PERIODIC ? p.Ex[0] : T(0), ex); }
    T hy = p.Hy[c];
    if (p.accum) {
        const T a = ex * hy;
        p.Sa[c] = p.Sa[c] + sqrt0(a * a) * p.dt;
        if (p.sum_e2) p.E2[c] = p.E2[c] + ex * ex * p.dt;
        guard(p, ex);
    }
    T Mh = p.Mh0;
    if (MATH) { const int g = p.geom[c]; if (g) Mh = p.matMh[g - 1]; }
    T dExz = cdiv(ex_zp - ex, p.ddz);
    {
        const LayerDev<T>& l = p.lay[MFD_ZL];
        if (l.nb && iz < l.ib) {
            const int q = iz;
            const T ps = l.B[q] * l.psi[1][q] + l.A[q] * dExz;
            l.psi[1][q] = ps;
            hy -= Mh * ps;
            dExz = cdiv(dExz, l.K[q]);
        }
    }
    {
        const LayerDev<T>& l = p.lay[MFD_ZR];
        if (l.nb && iz >= l.ib - 1) {
            const int q = iz - (l.ib - 1);
            const T ps = l.B[q] * l.psi[1][q] + l.A[q] * dExz;
            l.psi[1][q] = ps;
            hy -= Mh * ps;
            dExz = cdiv(dExz, l.K[q]);
        }
    }
    hy -= Mh * (T(0) + dExz);
    p.Hy[c] = hy;
}

template <typename T, typename R, bool MAT>
__global__ void __launch_bounds__(256) e1d_kernel(const __grid_constant__ EParams<T, R> p) {
    const int iz = blockIdx.x * blockDim.x + threadIdx.x;
    const int nz = p.L.nz;
    if (iz >= nz) return;
    const int c = iz;
    const T hy = p.Hy[c];
    T hy_zm;
    if (iz > 0) hy_zm = p.Hy[c - 1];
    else { const int b = p.bc[MFD_ZL]; hy_zm = bc_value(b, b == MFD_BC_PERIODIC ? p.Hy[nz - 1] : T(0), hy); }
    T dHyz = cdiv(hy - hy_zm, p.ddz);
    int g = 0;
    T Md1 = p.Md10, Md2 = p.Md20;
    if (MAT) {
        g = p.geom[c];
        if (g) { Md1 = p.mats[g - 1].Md1; Md2 = p.mats[g - 1].Md2; }
    }
    T Dv[1] = {p.Dx[c]};
    {
        const LayerDev<T>& l = p.lay[MFD_ZL];
        if (l.nb && iz < l.ib) {
            const int q = iz;
            const T ps = l.B[q] * l.psi[0][q] + l.A[q] * dHyz;
            l.psi[0][q] = ps;
            Dv[0] -= Md2 * ps;
            dHyz = cdiv(dHyz, l.K[q]);
        }
    }
    {
        const LayerDev<T>& l = p.lay[MFD_ZR];
        if (l.nb && iz >= l.ib - 1) {
            const int q = iz - (l.ib - 1);
            const T ps = l.B[q] * l.psi[0][q] + l.A[q] * dHyz;
            l.psi[0][q] = ps;
            Dv[0] -= Md2 * ps;
            dHyz = cdiv(dHyz, l.K[q]);
        }
    }
    Dv[0] = Md1 * Dv[0] + Md2 * (T(0) - dHyz);
    p.Dx[c] = Dv[0];
    if (MAT && g) {
        T* const Ep[1] = {p.Ex};
        material_cell<T, R, 1>(p.mats + (g - 1), 0, 0, iz, Ep, c, Dv, p.cur, p.dt);
    } else {
        p.Ex[c] = Dv[0] * p.Me0;
    }
}

// Running sums and NaN/Inf guard for the last step of a run (the H kernel of the next step
// does this for every other step).
template <typename T>
__global__ void __launch_bounds__(256) sums_kernel(const __grid_constant__ HParams<T> p, const int ndim) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y;
    const int iz = blockIdx.z;
    if (ix >= p.L.nx) return;
    const int c = ix + p.L.px * iy + p.L.sz * iz;
    const T ex = p.Ex[c];
    if (ndim == 3) {
        const T ey = p.Ey[c], ez = p.Ez[c], hx = p.Hx[c], hy = p.Hy[c], hz = p.Hz[c];
        const T a = ey * hz - ez * hy, b = ez * hx - ex * hz, d = ex * hy - ey * hx;
        p.Sa[c] = p.Sa[c] + sqrt0(a * a + b * b + d * d) * p.dt;
        if (p.sum_e2) p.E2[c] = p.E2[c] + (ex * ex + ey * ey + ez * ez) * p.dt;
    } else if (ndim == 2) {
        const T ez = p.Ez[c], hy = p.Hy[c];
        const T a = -ez * hy, b = ex * hy;
        p.Sa[c] = p.Sa[c] + sqrt0(a * a + b * b) * p.dt;
        if (p.sum_e2) p.E2[c] = p.E2[c] + (ex * ex + ez * ez) * p.dt;
    } else {
        const T hy = p.Hy[c];
        const T a = ex * hy;
        p.Sa[c] = p.Sa[c] + sqrt0(a * a) * p.dt;
        if (p.sum_e2) p.E2[c] = p.E2[c] + ex * ex * p.dt;
    }
    guard(p, ex);
}

}  // namespace mfd
