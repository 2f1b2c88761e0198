// yee.cuh -- Yee H and E update kernels (1-D, 2-D, 3-D) and the material kernel, sm_100a.
//
// 3-D kernels march along z: a thread owns one (ix, iy) column of a z-chunk.  The march is
// software-pipelined: all loads of plane iz+1 are issued before the arithmetic and stores of
// plane iz, so two planes of traffic are in flight per thread, and the z-neighbour plane is
// carried in registers (E at iz+1 for the H update, H at iz-1 for the E update).  x and y
// neighbours come from the same or adjacent warps through L1.  Boundary conditions are
// folded into per-thread neighbour offsets (periodic: the wrapped cell; Neumann: the cell
// itself; Dirichlet: the cell itself, zeroed after the load).
//
// Fused into the H update: the CPML psi recursions of the E curl, and -- for the previous
// step -- the running sums Sa/E2 (outputs.jl:475-485) and the NaN/Inf guard on Ex
// (models.jl:202-209), since it reads every E and H value of the cell anyway.
// Fused into the E update: the CPML psi recursions of the H curl, the D update and E = D Me
// for vacuum and plain dielectrics.  Cells of dispersive, plasma or Kerr materials get E
// from material_kernel, which runs over each such material's bounding box right after.
//
// Every cell update follows the reference kernels (src/models.jl:248-437 1-D, 450-719 2-D,
// 735-1162 3-D) operation by operation with the same operand types.
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
    int accum;             // add the running sums of the previous step
    int sum_e2;            // E2 is kept (any material cell)
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
};

template <typename T>
__device__ __forceinline__ void guard(const HParams<T>& p, T ex) {
    const int bad = (isnan(ex) ? 1 : 0) | (isinf(ex) ? 2 : 0);
    if (bad) atomicOr(p.flags + (p.prev_step - 1), bad);
}

// The same for an explicit step (batched launches keep the step per member on the device).
template <typename T>
__device__ __forceinline__ void guard_at(int* flags, long long prev_step, T ex) {
    const int bad = (isnan(ex) ? 1 : 0) | (isinf(ex) ? 2 : 0);
    if (bad) atomicOr(flags + (prev_step - 1), bad);
}

template <typename T>
__device__ __forceinline__ bool in_layers(const LayerDev<T>& lo, const LayerDev<T>& hi, int i) {
    return (lo.nb && i < lo.ib) || (hi.nb && i >= hi.ib - 1);
}

// CPML of the E curl in the H update, one face (models.jl:811-871).  The face's psi pair
// (psi[2], psi[3]) follows derivatives (da, db); S = +1: h1 += Mh pb, h2 -= Mh pa;
// S = -1: h1 -= Mh pb, h2 += Mh pa.  Then da, db are divided by kappa.
template <int S, int FAST, typename T>
__device__ __forceinline__ void cpml_h(const LayerDev<T>& l, int q, int k, T Mh, T& da, T& db, T& h1, T& h2) {
    const T B = l.B[q], A = l.A[q];
    const T pa = mad<FAST>(B, l.psi[2][k], A * da);
    const T pb = mad<FAST>(B, l.psi[3][k], A * db);
    l.psi[2][k] = pa;
    l.psi[3][k] = pb;
    if (S > 0) { h1 = mad<FAST>(Mh, pb, h1); h2 = mad<FAST>(-Mh, pa, h2); }
    else { h1 = mad<FAST>(-Mh, pb, h1); h2 = mad<FAST>(Mh, pa, h2); }
    da = cdiv<FAST>(da, l.K[q]);
    db = cdiv<FAST>(db, l.K[q]);
}

// CPML of the H curl in the E update, one face (models.jl:975-1035), psi pair (psi[0],
// psi[1]); S = +1: D1 += Md2 pb, D2 -= Md2 pa; S = -1: D1 -= Md2 pb, D2 += Md2 pa.
template <int S, int FAST, typename T>
__device__ __forceinline__ void cpml_e(const LayerDev<T>& l, int q, int k, T Md2, T& da, T& db, T& d1, T& d2) {
    const T B = l.B[q], A = l.A[q];
    const T pa = mad<FAST>(B, l.psi[0][k], A * da);
    const T pb = mad<FAST>(B, l.psi[1][k], A * db);
    l.psi[0][k] = pa;
    l.psi[1][k] = pb;
    if (S > 0) { d1 = mad<FAST>(Md2, pb, d1); d2 = mad<FAST>(-Md2, pa, d2); }
    else { d1 = mad<FAST>(-Md2, pb, d1); d2 = mad<FAST>(Md2, pa, d2); }
    da = cdiv<FAST>(da, l.K[q]);
    db = cdiv<FAST>(db, l.K[q]);
}

// ------------------------------------------------------------------------------------------
// 3-D
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

template <typename T, bool MATH, int FAST>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 3) h3d_kernel(const __grid_constant__ HParams<T> p, const int zc) {
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
    const bool cxy = in_layers(p.lay[MFD_XL], p.lay[MFD_XR], ix) || in_layers(p.lay[MFD_YL], p.lay[MFD_YR], iy);
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
            const T a = mad<FAST>(ey, hz, -(ez * hy)), b = mad<FAST>(ez, hx, -(ex * hz)), d = mad<FAST>(ex, hy, -(ey * hx));
            p.Sa[c] = mad<FAST>(sqrtm<FAST>(sum3sq<FAST>(a, b, d)), p.dt, cur.sa);
            if (p.sum_e2) p.E2[c] = mad<FAST>(sum3sq<FAST>(ex, ey, ez), p.dt, cur.e2);
            guard(p, ex);
        }
        T Mh = p.Mh0;
        if (MATH && cur.g) Mh = p.matMh[cur.g - 1];
        T dExy = cdiv<FAST>(ex_yp - ex, p.ddy);
        T dExz = cdiv<FAST>(ex_zp - ex, p.ddz);
        T dEyx = cdiv<FAST>(ey_xp - ey, p.ddx);
        T dEyz = cdiv<FAST>(ey_zp - ey, p.ddz);
        T dEzx = cdiv<FAST>(ez_xp - ez, p.ddx);
        T dEzy = cdiv<FAST>(ez_yp - ez, p.ddy);
        if (cxy || in_layers(p.lay[MFD_ZL], p.lay[MFD_ZR], iz)) {
            const LayerDev<T>&lxl = p.lay[MFD_XL], &lxr = p.lay[MFD_XR], &lyl = p.lay[MFD_YL], &lyr = p.lay[MFD_YR],
                             &lzl = p.lay[MFD_ZL], &lzr = p.lay[MFD_ZR];
            if (lxl.nb && ix < lxl.ib) cpml_h<+1, FAST>(lxl, ix, ix + lxl.nb * (iy + ny * iz), Mh, dEyx, dEzx, hy, hz);
            if (lxr.nb && ix >= lxr.ib - 1) {
                const int q = ix - (lxr.ib - 1);
                cpml_h<+1, FAST>(lxr, q, q + lxr.nb * (iy + ny * iz), Mh, dEyx, dEzx, hy, hz);
            }
            if (lyl.nb && iy < lyl.ib) cpml_h<-1, FAST>(lyl, iy, ix + sy * (iy + lyl.nb * iz), Mh, dExy, dEzy, hx, hz);
            if (lyr.nb && iy >= lyr.ib - 1) {
                const int q = iy - (lyr.ib - 1);
                cpml_h<-1, FAST>(lyr, q, ix + sy * (q + lyr.nb * iz), Mh, dExy, dEzy, hx, hz);
            }
            if (lzl.nb && iz < lzl.ib) cpml_h<+1, FAST>(lzl, iz, ix + sy * (iy + ny * iz), Mh, dExz, dEyz, hx, hy);
            if (lzr.nb && iz >= lzr.ib - 1) {
                const int q = iz - (lzr.ib - 1);
                cpml_h<+1, FAST>(lzr, q, ix + sy * (iy + ny * q), Mh, dExz, dEyz, hx, hy);
            }
        }
        hx = mad<FAST>(-Mh, dEzy - dEyz, hx);
        hy = mad<FAST>(-Mh, dExz - dEzx, hy);
        hz = mad<FAST>(-Mh, dEyx - dExy, hz);
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

template <typename T, typename R, bool MAT, int FAST>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 3) e3d_kernel(const __grid_constant__ EParams<T, R> p, const int zc) {
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
    const bool cxy = in_layers(p.lay[MFD_XL], p.lay[MFD_XR], ix) || in_layers(p.lay[MFD_YL], p.lay[MFD_YR], iy);
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
    ELoad<T> cur = e3d_load<T, R, MAT>(p, c, ox, oy);
    for (int iz = z0; iz < z1; ++iz, c += sz) {
        ELoad<T> nxt;
        if (iz + 1 < z1) nxt = e3d_load<T, R, MAT>(p, c + sz, ox, oy);
        const T hx = cur.hx, hy = cur.hy, hz = cur.hz;
        const T hy_xm = zx ? T(0) : cur.hyx, hz_xm = zx ? T(0) : cur.hzx;
        const T hx_ym = zy ? T(0) : cur.hxy, hz_ym = zy ? T(0) : cur.hzy;
        T dHxy = cdiv<FAST>(hx - hx_ym, p.ddy);
        T dHxz = cdiv<FAST>(hx - hx_zm, p.ddz);
        T dHyx = cdiv<FAST>(hy - hy_xm, p.ddx);
        T dHyz = cdiv<FAST>(hy - hy_zm, p.ddz);
        T dHzx = cdiv<FAST>(hz - hz_xm, p.ddx);
        T dHzy = cdiv<FAST>(hz - hz_ym, p.ddy);
        const int g = cur.g;
        T Md1 = p.Md10, Md2 = p.Md20, Me = p.Me0;
        bool simple = true;
        if (MAT && g) {
            const MatDev<T, R>& m = p.mats[g - 1];
            Md1 = m.Md1; Md2 = m.Md2; Me = m.Me; simple = m.simple != 0;
        }
        T D0 = cur.dx, D1 = cur.dy, D2 = cur.dz;
        if (cxy || in_layers(p.lay[MFD_ZL], p.lay[MFD_ZR], iz)) {
            const LayerDev<T>&lxl = p.lay[MFD_XL], &lxr = p.lay[MFD_XR], &lyl = p.lay[MFD_YL], &lyr = p.lay[MFD_YR],
                             &lzl = p.lay[MFD_ZL], &lzr = p.lay[MFD_ZR];
            if (lxl.nb && ix < lxl.ib) cpml_e<-1, FAST>(lxl, ix, ix + lxl.nb * (iy + ny * iz), Md2, dHyx, dHzx, D1, D2);
            if (lxr.nb && ix >= lxr.ib - 1) {
                const int q = ix - (lxr.ib - 1);
                cpml_e<-1, FAST>(lxr, q, q + lxr.nb * (iy + ny * iz), Md2, dHyx, dHzx, D1, D2);
            }
            if (lyl.nb && iy < lyl.ib) cpml_e<+1, FAST>(lyl, iy, ix + sy * (iy + lyl.nb * iz), Md2, dHxy, dHzy, D0, D2);
            if (lyr.nb && iy >= lyr.ib - 1) {
                const int q = iy - (lyr.ib - 1);
                cpml_e<+1, FAST>(lyr, q, ix + sy * (q + lyr.nb * iz), Md2, dHxy, dHzy, D0, D2);
            }
            if (lzl.nb && iz < lzl.ib) cpml_e<-1, FAST>(lzl, iz, ix + sy * (iy + ny * iz), Md2, dHxz, dHyz, D0, D1);
            if (lzr.nb && iz >= lzr.ib - 1) {
                const int q = iz - (lzr.ib - 1);
                cpml_e<-1, FAST>(lzr, q, ix + sy * (iy + ny * q), Md2, dHxz, dHyz, D0, D1);
            }
        }
        D0 = mad<FAST>(Md1, D0, Md2 * (dHzy - dHyz));
        D1 = mad<FAST>(Md1, D1, Md2 * (dHxz - dHzx));
        D2 = mad<FAST>(Md1, D2, Md2 * (dHyx - dHxy));
        p.Dx[c] = D0; p.Dy[c] = D1; p.Dz[c] = D2;
        if (simple) {   // E = (D - 0) Me (models.jl:1136-1153 with no polarisation)
            p.Ex[c] = D0 * Me;
            p.Ey[c] = D1 * Me;
            p.Ez[c] = D2 * Me;
        }
        hx_zm = hx;
        hy_zm = hy;
        cur = nxt;
    }
}

// ------------------------------------------------------------------------------------------
// 3-D, single precision: the same updates as h3d_kernel / e3d_kernel with the instruction
// count cut down -- the six derivative divisions are branch-free (div6), the run-level
// flags (accumulate sums, E2 kept) are template parameters, loop invariants are hoisted
// into registers, and the z march is unrolled twice so the prefetched plane is renamed
// instead of copied.
// ------------------------------------------------------------------------------------------
template <bool MATH, int FAST, bool ACC, bool E2S>
__global__ void __launch_bounds__(256, 4) h3d_f32_kernel(const __grid_constant__ HParams<float> p, const Div3 D3,
                                                         const int zc) {
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
    const int zlast_zero = bzr == MFD_BC_DIRICHLET ? nz - 1 : -1;   // plane whose z+1 neighbour is zero
    const bool zx = xr && bxr == MFD_BC_DIRICHLET, zy = yr && byr == MFD_BC_DIRICHLET;
    const bool cxy = in_layers(p.lay[MFD_XL], p.lay[MFD_XR], ix) || in_layers(p.lay[MFD_YL], p.lay[MFD_YR], iy);
    const int zl = p.lay[MFD_ZL].nb ? p.lay[MFD_ZL].ib : 0;          // iz < zl: left z layer
    const int zr = p.lay[MFD_ZR].nb ? p.lay[MFD_ZR].ib - 1 : nz;     // iz >= zr: right z layer
    const float dt = p.dt, Mh0 = p.Mh0;
    const float* __restrict__ Ex = p.Ex;
    const float* __restrict__ Ey = p.Ey;
    const float* __restrict__ Ez = p.Ez;
    float* Hx = p.Hx;
    float* Hy = p.Hy;
    float* Hz = p.Hz;
    float* Sa = p.Sa;
    float* E2 = p.E2;
    int c = ix + sy * iy + sz * z0;
    float ex = Ex[c], ey = Ey[c];
    auto load = [&](int cc, int iz) {
        HLoad<float> v;
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
        v.sa = ACC ? Sa[cc] : 0.0f;
        v.e2 = (ACC && E2S) ? E2[cc] : 0.0f;
        v.g = MATH ? (int)p.geom[cc] : 0;
        return v;
    };
    HLoad<float> cur = load(c, z0);
#pragma unroll 2
    for (int iz = z0; iz < z1; ++iz, c += sz) {
        HLoad<float> nxt;
        if (iz + 1 < z1) nxt = load(c + sz, iz + 1);
        const float ez = cur.ez;
        const float ey_xp = zx ? 0.0f : cur.eyx, ez_xp = zx ? 0.0f : cur.ezx;
        const float ex_yp = zy ? 0.0f : cur.exy, ez_yp = zy ? 0.0f : cur.ezy;
        const bool zz = iz == zlast_zero;
        const float ex_zp = zz ? 0.0f : cur.exz, ey_zp = zz ? 0.0f : cur.eyz;
        float hx = cur.hx, hy = cur.hy, hz = cur.hz;
        if (ACC) {
            const float a = mad<FAST>(ey, hz, -(ez * hy)), b = mad<FAST>(ez, hx, -(ex * hz)), d = mad<FAST>(ex, hy, -(ey * hx));
            Sa[c] = mad<FAST>(sqrtm<FAST>(sum3sq<FAST>(a, b, d)), dt, cur.sa);
            if (E2S) E2[c] = mad<FAST>(sum3sq<FAST>(ex, ey, ez), dt, cur.e2);
            if (!(fabsf(ex) <= FLT_MAX)) guard(p, ex);
        }
        float Mh = Mh0;
        if (MATH && cur.g) Mh = p.matMh[cur.g - 1];
        const float num[6] = {ex_yp - ex, ex_zp - ex, ey_xp - ey, ey_zp - ey, ez_xp - ez, ez_yp - ez};
        float q[6];
        div6<FAST>(D3, num, q);
        float dExy = q[0], dExz = q[1], dEyx = q[2], dEyz = q[3], dEzx = q[4], dEzy = q[5];
        if (cxy || iz < zl || iz >= zr) {
            const LayerDev<float>&lxl = p.lay[MFD_XL], &lxr = p.lay[MFD_XR], &lyl = p.lay[MFD_YL],
                                  &lyr = p.lay[MFD_YR], &lzl = p.lay[MFD_ZL], &lzr = p.lay[MFD_ZR];
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

template <typename R, bool MAT, int FAST>
__global__ void __launch_bounds__(256, 4) e3d_f32_kernel(const __grid_constant__ EParams<float, R> p, const Div3 D3,
                                                         const int zc) {
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
    const bool cxy = in_layers(p.lay[MFD_XL], p.lay[MFD_XR], ix) || in_layers(p.lay[MFD_YL], p.lay[MFD_YR], iy);
    const int zl = p.lay[MFD_ZL].nb ? p.lay[MFD_ZL].ib : 0;
    const int zr = p.lay[MFD_ZR].nb ? p.lay[MFD_ZR].ib - 1 : nz;
    const float Md10 = p.Md10, Md20 = p.Md20, Me0 = p.Me0;
    const float* __restrict__ Hx = p.Hx;
    const float* __restrict__ Hy = p.Hy;
    const float* __restrict__ Hz = p.Hz;
    float* Dx = p.Dx;
    float* Dy = p.Dy;
    float* Dz = p.Dz;
    float* Ex = p.Ex;
    float* Ey = p.Ey;
    float* Ez = p.Ez;
    int c = ix + sy * iy + sz * z0;
    float hx_zm, hy_zm;
    if (z0 > 0) {
        hx_zm = Hx[c - sz];
        hy_zm = Hy[c - sz];
    } else {
        const int oz = bzl == MFD_BC_PERIODIC ? (nz - 1) * sz : 0;
        hx_zm = bzl == MFD_BC_DIRICHLET ? 0.0f : Hx[c + oz];
        hy_zm = bzl == MFD_BC_DIRICHLET ? 0.0f : Hy[c + oz];
    }
    auto load = [&](int cc) {
        ELoad<float> v;
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
        return v;
    };
    ELoad<float> cur = load(c);
#pragma unroll 2
    for (int iz = z0; iz < z1; ++iz, c += sz) {
        ELoad<float> nxt;
        if (iz + 1 < z1) nxt = load(c + sz);
        const float hx = cur.hx, hy = cur.hy, hz = cur.hz;
        const float hy_xm = zx ? 0.0f : cur.hyx, hz_xm = zx ? 0.0f : cur.hzx;
        const float hx_ym = zy ? 0.0f : cur.hxy, hz_ym = zy ? 0.0f : cur.hzy;
        const float num[6] = {hx - hx_ym, hx - hx_zm, hy - hy_xm, hy - hy_zm, hz - hz_xm, hz - hz_ym};
        float q[6];
        div6<FAST>(D3, num, q);
        float dHxy = q[0], dHxz = q[1], dHyx = q[2], dHyz = q[3], dHzx = q[4], dHzy = q[5];
        float Md1 = Md10, Md2 = Md20, Me = Me0;
        bool simple = true;
        if (MAT && cur.g) {
            const MatDev<float, R>& m = p.mats[cur.g - 1];
            Md1 = m.Md1; Md2 = m.Md2; Me = m.Me; simple = m.simple != 0;
        }
        float D0 = cur.dx, D1 = cur.dy, D2 = cur.dz;
        if (cxy || iz < zl || iz >= zr) {
            const LayerDev<float>&lxl = p.lay[MFD_XL], &lxr = p.lay[MFD_XR], &lyl = p.lay[MFD_YL],
                                  &lyr = p.lay[MFD_YR], &lzl = p.lay[MFD_ZL], &lzr = p.lay[MFD_ZR];
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
        }
        D0 = mad<FAST>(Md1, D0, Md2 * (dHzy - dHyz));
        D1 = mad<FAST>(Md1, D1, Md2 * (dHxz - dHzx));
        D2 = mad<FAST>(Md1, D2, Md2 * (dHyx - dHxy));
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
        cur = nxt;
    }
}

// ------------------------------------------------------------------------------------------
// 2-D (x-z plane): one thread per cell
// ------------------------------------------------------------------------------------------
// One cell of the 2-D H update; `accum` and `prev_step` are the step's running-sum flag and
// the previous step (p.accum / p.prev_step for a single model, per-member state in a batch).
template <typename T, bool MATH, int FAST>
__device__ __forceinline__ void h2d_cell(const HParams<T>& p, int accum, long long prev_step, int ix, int iz) {
    const int nx = p.L.nx, nz = p.L.nz;
    const int sz = p.L.sz;
    const int c = ix + sz * iz;
    const T ex = p.Ex[c], ez = p.Ez[c];
    T ez_xp, ex_zp;
    if (ix < nx - 1) ez_xp = p.Ez[c + 1];
    else { const int b = p.bc[MFD_XR]; ez_xp = bc_value(b, b == MFD_BC_PERIODIC ? p.Ez[c - (nx - 1)] : T(0), ez); }
    if (iz < nz - 1) ex_zp = p.Ex[c + sz];
    else { const int b = p.bc[MFD_ZR]; ex_zp = bc_value(b, b == MFD_BC_PERIODIC ? p.Ex[c - (nz - 1) * sz] : T(0), ex); }
    T hy = p.Hy[c];
    if (accum) {
        const T a = -ez * hy, b = ex * hy;
        p.Sa[c] = p.Sa[c] + sqrt0(a * a + b * b) * p.dt;
        if (p.sum_e2) p.E2[c] = p.E2[c] + (ex * ex + ez * ez) * p.dt;
        guard_at(p.flags, prev_step, ex);
    }
    T Mh = p.Mh0;
    if (MATH) { const int g = p.geom[c]; if (g) Mh = p.matMh[g - 1]; }
    T dExz = cdiv<FAST>(ex_zp - ex, p.ddz);
    T dEzx = cdiv<FAST>(ez_xp - ez, p.ddx);
    {
        const LayerDev<T>& l = p.lay[MFD_XL];
        if (l.nb && ix < l.ib) {
            const int q = ix, k = q + l.nb * iz;
            const T ps = l.B[q] * l.psi[1][k] + l.A[q] * dEzx;
            l.psi[1][k] = ps;
            hy = mad<FAST>(Mh, ps, hy);
            dEzx = cdiv<FAST>(dEzx, l.K[q]);
        }
    }
    {
        const LayerDev<T>& l = p.lay[MFD_XR];
        if (l.nb && ix >= l.ib - 1) {
            const int q = ix - (l.ib - 1), k = q + l.nb * iz;
            const T ps = l.B[q] * l.psi[1][k] + l.A[q] * dEzx;
            l.psi[1][k] = ps;
            hy = mad<FAST>(Mh, ps, hy);
            dEzx = cdiv<FAST>(dEzx, l.K[q]);
        }
    }
    {
        const LayerDev<T>& l = p.lay[MFD_ZL];
        if (l.nb && iz < l.ib) {
            const int q = iz, k = ix + p.L.px * q;
            const T ps = l.B[q] * l.psi[1][k] + l.A[q] * dExz;
            l.psi[1][k] = ps;
            hy = mad<FAST>(-Mh, ps, hy);
            dExz = cdiv<FAST>(dExz, l.K[q]);
        }
    }
    {
        const LayerDev<T>& l = p.lay[MFD_ZR];
        if (l.nb && iz >= l.ib - 1) {
            const int q = iz - (l.ib - 1), k = ix + p.L.px * q;
            const T ps = l.B[q] * l.psi[1][k] + l.A[q] * dExz;
            l.psi[1][k] = ps;
            hy = mad<FAST>(-Mh, ps, hy);
            dExz = cdiv<FAST>(dExz, l.K[q]);
        }
    }
    hy = mad<FAST>(-Mh, dExz - dEzx, hy);
    p.Hy[c] = hy;
}

template <typename T, bool MATH, int FAST>
__global__ void __launch_bounds__(256) h2d_kernel(const __grid_constant__ HParams<T> p) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iz = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= p.L.nx || iz >= p.L.nz) return;
    h2d_cell<T, MATH, FAST>(p, p.accum, p.prev_step, ix, iz);
}

// One cell of the 2-D E update (D with CPML; E of cells without a response material).
template <typename T, typename R, bool MAT, int FAST>
__device__ __forceinline__ void e2d_cell(const EParams<T, R>& p, int ix, int iz) {
    const int nx = p.L.nx, nz = p.L.nz;
    const int sz = p.L.sz;
    const int c = ix + sz * iz;
    const T hy = p.Hy[c];
    T hy_xm, hy_zm;
    if (ix > 0) hy_xm = p.Hy[c - 1];
    else { const int b = p.bc[MFD_XL]; hy_xm = bc_value(b, b == MFD_BC_PERIODIC ? p.Hy[c + (nx - 1)] : T(0), hy); }
    if (iz > 0) hy_zm = p.Hy[c - sz];
    else { const int b = p.bc[MFD_ZL]; hy_zm = bc_value(b, b == MFD_BC_PERIODIC ? p.Hy[c + (nz - 1) * sz] : T(0), hy); }
    T dHyx = cdiv<FAST>(hy - hy_xm, p.ddx);
    T dHyz = cdiv<FAST>(hy - hy_zm, p.ddz);
    T Md1 = p.Md10, Md2 = p.Md20, Me = p.Me0;
    bool simple = true;
    if (MAT) {
        const int g = p.geom[c];
        if (g) {
            const MatDev<T, R>& m = p.mats[g - 1];
            Md1 = m.Md1; Md2 = m.Md2; Me = m.Me; simple = m.simple != 0;
        }
    }
    T D0 = p.Dx[c], D2 = p.Dz[c];
    {
        const LayerDev<T>& l = p.lay[MFD_XL];
        if (l.nb && ix < l.ib) {
            const int q = ix, k = q + l.nb * iz;
            const T ps = l.B[q] * l.psi[0][k] + l.A[q] * dHyx;
            l.psi[0][k] = ps;
            D2 = mad<FAST>(Md2, ps, D2);
            dHyx = cdiv<FAST>(dHyx, l.K[q]);
        }
    }
    {
        const LayerDev<T>& l = p.lay[MFD_XR];
        if (l.nb && ix >= l.ib - 1) {
            const int q = ix - (l.ib - 1), k = q + l.nb * iz;
            const T ps = l.B[q] * l.psi[0][k] + l.A[q] * dHyx;
            l.psi[0][k] = ps;
            D2 = mad<FAST>(Md2, ps, D2);
            dHyx = cdiv<FAST>(dHyx, l.K[q]);
        }
    }
    {
        const LayerDev<T>& l = p.lay[MFD_ZL];
        if (l.nb && iz < l.ib) {
            const int q = iz, k = ix + p.L.px * q;
            const T ps = l.B[q] * l.psi[0][k] + l.A[q] * dHyz;
            l.psi[0][k] = ps;
            D0 = mad<FAST>(-Md2, ps, D0);
            dHyz = cdiv<FAST>(dHyz, l.K[q]);
        }
    }
    {
        const LayerDev<T>& l = p.lay[MFD_ZR];
        if (l.nb && iz >= l.ib - 1) {
            const int q = iz - (l.ib - 1), k = ix + p.L.px * q;
            const T ps = l.B[q] * l.psi[0][k] + l.A[q] * dHyz;
            l.psi[0][k] = ps;
            D0 = mad<FAST>(-Md2, ps, D0);
            dHyz = cdiv<FAST>(dHyz, l.K[q]);
        }
    }
    D0 = Md1 * D0 + Md2 * (T(0) - dHyz);
    D2 = Md1 * D2 + Md2 * (dHyx - T(0));
    p.Dx[c] = D0;
    p.Dz[c] = D2;
    if (simple) {
        p.Ex[c] = D0 * Me;
        p.Ez[c] = D2 * Me;
    }
}

template <typename T, typename R, bool MAT, int FAST>
__global__ void __launch_bounds__(256) e2d_kernel(const __grid_constant__ EParams<T, R> p) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iz = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= p.L.nx || iz >= p.L.nz) return;
    e2d_cell<T, R, MAT, FAST>(p, ix, iz);
}

// ------------------------------------------------------------------------------------------
// 2-D, second field set (Hx, Hz, Dy, Ey): the 3-D cell updates with every y derivative zero,
// in their operation order (src/models.jl:735-878, 895-1162).  psi[0] of a layer holds
// psiHzx / psiHxz (E update), psi[1] psiEyx / psiEyz (H update).
// ------------------------------------------------------------------------------------------
template <typename T, bool MATH, int FAST>
__device__ __forceinline__ void h2e_cell(const HParams<T>& p, int accum, long long prev_step, int ix, int iz) {
    const int nx = p.L.nx, nz = p.L.nz;
    const int sz = p.L.sz;
    const int c = ix + sz * iz;
    const T ey = p.Ey[c];
    T ey_xp, ey_zp;
    if (ix < nx - 1) ey_xp = p.Ey[c + 1];
    else { const int b = p.bc[MFD_XR]; ey_xp = bc_value(b, b == MFD_BC_PERIODIC ? p.Ey[c - (nx - 1)] : T(0), ey); }
    if (iz < nz - 1) ey_zp = p.Ey[c + sz];
    else { const int b = p.bc[MFD_ZR]; ey_zp = bc_value(b, b == MFD_BC_PERIODIC ? p.Ey[c - (nz - 1) * sz] : T(0), ey); }
    T hx = p.Hx[c], hz = p.Hz[c];
    if (accum) {
        const T a = ey * hz, d = T(0) - ey * hx;
        p.Sa[c] = p.Sa[c] + sqrt0(a * a + d * d) * p.dt;
        if (p.sum_e2) p.E2[c] = p.E2[c] + ey * ey * p.dt;
        guard_at(p.flags, prev_step, ey);
    }
    T Mh = p.Mh0;
    if (MATH) { const int g = p.geom[c]; if (g) Mh = p.matMh[g - 1]; }
    T dEyx = cdiv<FAST>(ey_xp - ey, p.ddx);
    T dEyz = cdiv<FAST>(ey_zp - ey, p.ddz);
#pragma unroll
    for (int f = MFD_XL; f <= MFD_XR; ++f) {
        const LayerDev<T>& l = p.lay[f];
        if (l.nb && (f == MFD_XL ? ix < l.ib : ix >= l.ib - 1)) {
            const int q = f == MFD_XL ? ix : ix - (l.ib - 1), k = q + l.nb * iz;
            const T ps = l.B[q] * l.psi[1][k] + l.A[q] * dEyx;
            l.psi[1][k] = ps;
            hz = mad<FAST>(-Mh, ps, hz);
            dEyx = cdiv<FAST>(dEyx, l.K[q]);
        }
    }
#pragma unroll
    for (int f = MFD_ZL; f <= MFD_ZR; ++f) {
        const LayerDev<T>& l = p.lay[f];
        if (l.nb && (f == MFD_ZL ? iz < l.ib : iz >= l.ib - 1)) {
            const int q = f == MFD_ZL ? iz : iz - (l.ib - 1), k = ix + p.L.px * q;
            const T ps = l.B[q] * l.psi[1][k] + l.A[q] * dEyz;
            l.psi[1][k] = ps;
            hx = mad<FAST>(Mh, ps, hx);
            dEyz = cdiv<FAST>(dEyz, l.K[q]);
        }
    }
    hx = mad<FAST>(-Mh, T(0) - dEyz, hx);
    hz = mad<FAST>(-Mh, dEyx - T(0), hz);
    p.Hx[c] = hx;
    p.Hz[c] = hz;
}

template <typename T, bool MATH, int FAST>
__global__ void __launch_bounds__(256) h2e_kernel(const __grid_constant__ HParams<T> p) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iz = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= p.L.nx || iz >= p.L.nz) return;
    h2e_cell<T, MATH, FAST>(p, p.accum, p.prev_step, ix, iz);
}

template <typename T, typename R, bool MAT, int FAST>
__device__ __forceinline__ void e2e_cell(const EParams<T, R>& p, int ix, int iz) {
    const int nx = p.L.nx, nz = p.L.nz;
    const int sz = p.L.sz;
    const int c = ix + sz * iz;
    const T hx = p.Hx[c], hz = p.Hz[c];
    T hz_xm, hx_zm;
    if (ix > 0) hz_xm = p.Hz[c - 1];
    else { const int b = p.bc[MFD_XL]; hz_xm = bc_value(b, b == MFD_BC_PERIODIC ? p.Hz[c + (nx - 1)] : T(0), hz); }
    if (iz > 0) hx_zm = p.Hx[c - sz];
    else { const int b = p.bc[MFD_ZL]; hx_zm = bc_value(b, b == MFD_BC_PERIODIC ? p.Hx[c + (nz - 1) * sz] : T(0), hx); }
    T dHxz = cdiv<FAST>(hx - hx_zm, p.ddz);
    T dHzx = cdiv<FAST>(hz - hz_xm, p.ddx);
    T Md1 = p.Md10, Md2 = p.Md20, Me = p.Me0;
    bool simple = true;
    if (MAT) {
        const int g = p.geom[c];
        if (g) {
            const MatDev<T, R>& m = p.mats[g - 1];
            Md1 = m.Md1; Md2 = m.Md2; Me = m.Me; simple = m.simple != 0;
        }
    }
    T D1 = p.Dy[c];
#pragma unroll
    for (int f = MFD_XL; f <= MFD_XR; ++f) {
        const LayerDev<T>& l = p.lay[f];
        if (l.nb && (f == MFD_XL ? ix < l.ib : ix >= l.ib - 1)) {
            const int q = f == MFD_XL ? ix : ix - (l.ib - 1), k = q + l.nb * iz;
            const T ps = l.B[q] * l.psi[0][k] + l.A[q] * dHzx;
            l.psi[0][k] = ps;
            D1 = mad<FAST>(-Md2, ps, D1);
            dHzx = cdiv<FAST>(dHzx, l.K[q]);
        }
    }
#pragma unroll
    for (int f = MFD_ZL; f <= MFD_ZR; ++f) {
        const LayerDev<T>& l = p.lay[f];
        if (l.nb && (f == MFD_ZL ? iz < l.ib : iz >= l.ib - 1)) {
            const int q = f == MFD_ZL ? iz : iz - (l.ib - 1), k = ix + p.L.px * q;
            const T ps = l.B[q] * l.psi[0][k] + l.A[q] * dHxz;
            l.psi[0][k] = ps;
            D1 = mad<FAST>(Md2, ps, D1);
            dHxz = cdiv<FAST>(dHxz, l.K[q]);
        }
    }
    D1 = Md1 * D1 + Md2 * (dHxz - dHzx);
    p.Dy[c] = D1;
    if (simple) p.Ey[c] = D1 * Me;
}

template <typename T, typename R, bool MAT, int FAST>
__global__ void __launch_bounds__(256) e2e_kernel(const __grid_constant__ EParams<T, R> p) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iz = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= p.L.nx || iz >= p.L.nz) return;
    e2e_cell<T, R, MAT, FAST>(p, ix, iz);
}

// ------------------------------------------------------------------------------------------
// 1-D (z)
// ------------------------------------------------------------------------------------------
template <typename T, bool MATH, int FAST>
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
    T dExz = cdiv<FAST>(ex_zp - ex, p.ddz);
    {
        const LayerDev<T>& l = p.lay[MFD_ZL];
        if (l.nb && iz < l.ib) {
            const int q = iz;
            const T ps = l.B[q] * l.psi[1][q] + l.A[q] * dExz;
            l.psi[1][q] = ps;
            hy = mad<FAST>(-Mh, ps, hy);
            dExz = cdiv<FAST>(dExz, l.K[q]);
        }
    }
    {
        const LayerDev<T>& l = p.lay[MFD_ZR];
        if (l.nb && iz >= l.ib - 1) {
            const int q = iz - (l.ib - 1);
            const T ps = l.B[q] * l.psi[1][q] + l.A[q] * dExz;
            l.psi[1][q] = ps;
            hy = mad<FAST>(-Mh, ps, hy);
            dExz = cdiv<FAST>(dExz, l.K[q]);
        }
    }
    hy -= Mh * (T(0) + dExz);
    p.Hy[c] = hy;
}

template <typename T, typename R, bool MAT, int FAST>
__global__ void __launch_bounds__(256) e1d_kernel(const __grid_constant__ EParams<T, R> p) {
    const int iz = blockIdx.x * blockDim.x + threadIdx.x;
    const int nz = p.L.nz;
    if (iz >= nz) return;
    const int c = iz;
    const T hy = p.Hy[c];
    T hy_zm;
    if (iz > 0) hy_zm = p.Hy[c - 1];
    else { const int b = p.bc[MFD_ZL]; hy_zm = bc_value(b, b == MFD_BC_PERIODIC ? p.Hy[nz - 1] : T(0), hy); }
    T dHyz = cdiv<FAST>(hy - hy_zm, p.ddz);
    T Md1 = p.Md10, Md2 = p.Md20, Me = p.Me0;
    bool simple = true;
    if (MAT) {
        const int g = p.geom[c];
        if (g) {
            const MatDev<T, R>& m = p.mats[g - 1];
            Md1 = m.Md1; Md2 = m.Md2; Me = m.Me; simple = m.simple != 0;
        }
    }
    T D0 = p.Dx[c];
    {
        const LayerDev<T>& l = p.lay[MFD_ZL];
        if (l.nb && iz < l.ib) {
            const int q = iz;
            const T ps = l.B[q] * l.psi[0][q] + l.A[q] * dHyz;
            l.psi[0][q] = ps;
            D0 = mad<FAST>(-Md2, ps, D0);
            dHyz = cdiv<FAST>(dHyz, l.K[q]);
        }
    }
    {
        const LayerDev<T>& l = p.lay[MFD_ZR];
        if (l.nb && iz >= l.ib - 1) {
            const int q = iz - (l.ib - 1);
            const T ps = l.B[q] * l.psi[0][q] + l.A[q] * dHyz;
            l.psi[0][q] = ps;
            D0 = mad<FAST>(-Md2, ps, D0);
            dHyz = cdiv<FAST>(dHyz, l.K[q]);
        }
    }
    D0 = Md1 * D0 + Md2 * (T(0) - dHyz);
    p.Dx[c] = D0;
    if (simple) p.Ex[c] = D0 * Me;
}

// ------------------------------------------------------------------------------------------
// Material response (ADE poles, plasma, Kerr; models.jl:1042-1154, 622-712, 365-431) for the
// cells of material g inside its bounding box: reads the new D and the old E of the cell.
// ------------------------------------------------------------------------------------------
template <typename T, typename R, int NC>
__global__ void __launch_bounds__(128) material_kernel(const MatDev<T, R>* __restrict__ mats, int g,
                                                      const uint8_t* __restrict__ geom, Layout L,
                                                      const T* D0, const T* D1, const T* D2, T* E0, T* E1, T* E2,
                                                      int cur, T dt) {
    const MatDev<T, R>* m = mats + (g - 1);
    const int bx = blockIdx.x * blockDim.x + threadIdx.x;
    if (bx >= m->bnx) return;
    const int ix = m->bx0 + bx, iy = m->by0 + (int)blockIdx.y, iz = m->bz0 + (int)blockIdx.z;
    const int c = ix + L.px * iy + L.sz * iz;
    if (geom[c] != g) return;
    T Dv[NC];
    T* Ep[NC];
    if (NC == 3) {
        Dv[0] = D0[c]; Dv[1 % NC] = D1[c]; Dv[2 % NC] = D2[c];
        Ep[0] = E0; Ep[1 % NC] = E1; Ep[2 % NC] = E2;
    } else if (NC == 2) {   // x and z
        Dv[0] = D0[c]; Dv[1 % NC] = D2[c];
        Ep[0] = E0; Ep[1 % NC] = E2;
    } else {
        Dv[0] = D0[c];
        Ep[0] = E0;
    }
    material_cell<T, R, NC>(m, ix, iy, iz, Ep, c, Dv, cur, dt);
}

// The same with the box flattened (one thread per box cell, full warps whatever the box's
// width) and the number of poles NQ known at compile time (material_cell_n).
template <typename T, typename R, int NC, int NQ>
__global__ void __launch_bounds__(256) material_flat_kernel(const MatDev<T, R>* __restrict__ mats, int g,
                                                           const uint8_t* __restrict__ geom, Layout L,
                                                           const T* D0, const T* D1, const T* D2, T* E0, T* E1, T* E2,
                                                           int cur, T dt) {
    const MatDev<T, R>* m = mats + (g - 1);
    const long long bi = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (bi >= m->bsize) return;
    const int bnx = m->bnx, bny = m->bny;
    const long long row = bi / bnx;
    const int bx = (int)(bi - row * bnx);
    const long long bz = row / bny;
    const int by = (int)(row - bz * bny);
    const int ix = m->bx0 + bx, iy = m->by0 + by, iz = m->bz0 + (int)bz;
    const int c = ix + L.px * iy + L.sz * iz;
    if (geom[c] != g) return;
    T Dv[NC];
    T* Ep[NC];
    if (NC == 3) {
        Dv[0] = D0[c]; Dv[1 % NC] = D1[c]; Dv[2 % NC] = D2[c];
        Ep[0] = E0; Ep[1 % NC] = E1; Ep[2 % NC] = E2;
    } else if (NC == 2) {
        Dv[0] = D0[c]; Dv[1 % NC] = D2[c];
        Ep[0] = E0; Ep[1 % NC] = E2;
    } else {
        Dv[0] = D0[c];
        Ep[0] = E0;
    }
    material_cell_n<T, R, NC, NQ>(m, bi, Ep, c, Dv, cur, dt);
}

// Running sums and NaN/Inf guard for the last step of a run (the H kernel of the next step
// does this for every other step).
// fset: the model's field set -- 3, 2 or 1 (its dimension) or FSET_EY2 (the second 2-D
// field set: Hx, Hz, Dy, Ey).
constexpr int FSET_EY2 = 4;

template <typename T>
__global__ void __launch_bounds__(256) sums_kernel(const __grid_constant__ HParams<T> p, const int fset) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y;
    const int iz = blockIdx.z;
    if (ix >= p.L.nx) return;
    const int c = ix + p.L.px * iy + p.L.sz * iz;
    if (fset == FSET_EY2) {   // the 3-D norm with Ex = Ez = Hy = 0
        const T ey = p.Ey[c], hx = p.Hx[c], hz = p.Hz[c];
        const T a = ey * hz, d = T(0) - ey * hx;
        p.Sa[c] = p.Sa[c] + sqrt0(a * a + d * d) * p.dt;
        if (p.sum_e2) p.E2[c] = p.E2[c] + ey * ey * p.dt;
        guard(p, ey);
        return;
    }
    const T ex = p.Ex[c];
    if (fset == 3) {
        const T ey = p.Ey[c], ez = p.Ez[c], hx = p.Hx[c], hy = p.Hy[c], hz = p.Hz[c];
        const T a = ey * hz - ez * hy, b = ez * hx - ex * hz, d = ex * hy - ey * hx;
        p.Sa[c] = p.Sa[c] + sqrt0(a * a + b * b + d * d) * p.dt;
        if (p.sum_e2) p.E2[c] = p.E2[c] + (ex * ex + ey * ey + ez * ez) * p.dt;
    } else if (fset == 2) {
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

// NaN/Inf guard of Ex (Ey in the second 2-D field set) for one step (models.jl:202-209), for a step whose running sums (and
// the guard done with them) are left to the next H update.
template <typename T>
__global__ void __launch_bounds__(256) guard_kernel(const T* __restrict__ Ex, const Layout L, int* flags, const long long step) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    if (ix >= L.nx) return;
    guard_at(flags, step, Ex[ix + L.px * (int)blockIdx.y + L.sz * (int)blockIdx.z]);
}

}  // namespace mfd
