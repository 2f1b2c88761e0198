// yee3d_tma.cuh -- TMA-fed 3-D Yee updates for single precision (sm_100a).
//
// A CTA of 32 x 8 threads owns a 32 x 8 (x, y) tile and marches a z-chunk.  One thread
// streams whole planes of the tile -- each field array as one cp.async.bulk.tensor box, with
// the halo the stencil needs -- into a ring of TMA_STAGES shared-memory stages, up to
// TMA_STAGES-1 planes ahead, each stage completing on its own mbarrier.  The other threads
// only read shared memory and store results, so memory latency is hidden by the ring instead
// of by per-thread loads, and no thread spends instructions on load addresses.
//
// Boxes (x extent x y extent, elements): x boxes start on multiples of 4 floats (16 bytes),
// as TMA requires; cells outside the grid are zero-filled by the TMA unit, which is the
// Dirichlet value.  Cells on the grid's upper (H update) or lower (E update) faces take
// periodic / Neumann neighbour values from global memory instead.
//   H update, plane iz and iz+1:  Ex 32x9 at (x0, y0), Ey 36x8 at (x0, y0), Ez 36x9 at (x0, y0),
//                                Hx Hy Hz Sa E2 32x8, material map 32x8 (bytes).
//   E update, plane iz-1 and iz: Hx 32x9 at (x0, y0-1), Hy 36x8 at (x0-4, y0), Hz 36x9 at
//                                (x0-4, y0-1), Dx Dy Dz 32x8, material map 32x8.
// The arithmetic per cell is that of h3d_kernel / e3d_kernel (yee.cuh), operation by
// operation.
#pragma once

#include "tma.cuh"
#include "yee.cuh"

namespace mfd {

#define TMA_BX 32
#define TMA_BY 8
#define TMA_STAGES 4

// Shared-memory stage layouts (byte offsets, each array 128-byte aligned).
struct HStage {
    static constexpr int EX = 0;                         // float [9][32]   1152
    static constexpr int EY = EX + 1152;                 // float [8][36]   1152
    static constexpr int EZ = EY + 1152;                 // float [9][36]   1296 -> 1408
    static constexpr int HX = EZ + 1408;                 // float [8][32]   1024
    static constexpr int HY = HX + 1024;
    static constexpr int HZ = HY + 1024;
    static constexpr int SA = HZ + 1024;
    static constexpr int E2 = SA + 1024;
    static constexpr int G = E2 + 1024;                  // uint8 [8][32]   256
    static constexpr int BYTES = G + 256;                // 9088
};

struct EStage {
    static constexpr int HX = 0;                         // float [9][32]   1152
    static constexpr int HY = HX + 1152;                 // float [8][36]   1152
    static constexpr int HZ = HY + 1152;                 // float [9][36]   1296 -> 1408
    static constexpr int DX = HZ + 1408;                 // float [8][32]   1024
    static constexpr int DY = DX + 1024;
    static constexpr int DZ = DY + 1024;
    static constexpr int G = DZ + 1024;                  // uint8 [8][32]   256
    static constexpr int BYTES = G + 256;                // 7040
};

struct HTmaParams {
    CUtensorMap mEx, mEy, mEz, mHx, mHy, mHz, mSa, mE2, mG;
    HParams<float> p;
    int* timeout;
};

template <typename R>
struct ETmaParams {
    CUtensorMap mHx, mHy, mHz, mDx, mDy, mDz, mG;
    EParams<float, R> p;
    int* timeout;
};

template <bool MATH>
__device__ __forceinline__ uint32_t h_stage_bytes(const HTmaParams& P) {
    uint32_t b = 1152 + 1152 + 1296 + 3 * 1024 + (P.p.accum ? 1024 : 0) + (P.p.accum && P.p.sum_e2 ? 1024 : 0);
    return b + (MATH ? 256 : 0);
}

template <bool MATH>
__device__ __forceinline__ void h_issue(const HTmaParams& P, unsigned char* st, uint64_t* bar, int x0, int y0, int z) {
    mbar_expect_tx(bar, h_stage_bytes<MATH>(P));
    tma_load_3d(st + HStage::EX, &P.mEx, x0, y0, z, bar);
    tma_load_3d(st + HStage::EY, &P.mEy, x0, y0, z, bar);
    tma_load_3d(st + HStage::EZ, &P.mEz, x0, y0, z, bar);
    tma_load_3d(st + HStage::HX, &P.mHx, x0, y0, z, bar);
    tma_load_3d(st + HStage::HY, &P.mHy, x0, y0, z, bar);
    tma_load_3d(st + HStage::HZ, &P.mHz, x0, y0, z, bar);
    if (P.p.accum) {
        tma_load_3d(st + HStage::SA, &P.mSa, x0, y0, z, bar);
        if (P.p.sum_e2) tma_load_3d(st + HStage::E2, &P.mE2, x0, y0, z, bar);
    }
    if (MATH) tma_load_3d(st + HStage::G, &P.mG, x0, y0, z, bar);
}

template <bool MATH, bool FAST>
__global__ void __launch_bounds__(256, 3) h3d_tma_kernel(const __grid_constant__ HTmaParams P, const int zc) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[TMA_STAGES];
    const HParams<float>& p = P.p;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TMA_BX + tx;
    const int x0 = blockIdx.x * TMA_BX, y0 = blockIdx.y * TMA_BY;
    const int ix = x0 + tx, iy = y0 + ty;
    const int nx = p.L.nx, ny = p.L.ny, nz = p.L.nz;
    const int z0 = blockIdx.z * zc;
    const int z1 = min(z0 + zc, nz);
    const int NP = z1 - z0 + 1;                     // planes z0 .. z1 (z1 for the z+1 neighbour)
    if (tid == 0) {
        for (int s = 0; s < TMA_STAGES; ++s) mbar_init(&bars[s], 1);
        fence_async_shared();
    }
    __syncthreads();
    int issued = 0;   // planes issued so far (thread 0 is the only issuer)
    if (tid == 0)
        for (; issued < TMA_STAGES && issued < NP; ++issued)
            h_issue<MATH>(P, smem + issued * HStage::BYTES, &bars[issued], x0, y0, z0 + issued);
    const bool active = ix < nx && iy < ny;
    const int sy = p.L.px, sz = p.L.sz;
    const int bxr = p.bc[MFD_XR], byr = p.bc[MFD_YR], bzr = p.bc[MFD_ZR];
    const bool cxy = in_layers(p.lay[MFD_XL], p.lay[MFD_XR], ix) || in_layers(p.lay[MFD_YL], p.lay[MFD_YR], iy);
    int lfail = -1;
    for (int l = 0; l + 1 < NP; ++l) {
        const int iz = z0 + l;
        const int s0 = l % TMA_STAGES, s1 = (l + 1) % TMA_STAGES;
        const bool w = mbar_wait(&bars[s0], (l / TMA_STAGES) & 1) && mbar_wait(&bars[s1], ((l + 1) / TMA_STAGES) & 1);
        if (!__syncthreads_and(w)) {   // block-uniform decision
            lfail = l;
            break;
        }
        const unsigned char* A = smem + s0 * HStage::BYTES;
        const unsigned char* Bn = smem + s1 * HStage::BYTES;
        if (active) {
            const float* sEx = (const float*)(A + HStage::EX);
            const float* sEy = (const float*)(A + HStage::EY);
            const float* sEz = (const float*)(A + HStage::EZ);
            const int c = ix + sy * iy + sz * iz;
            const float ex = sEx[ty * 32 + tx], ey = sEy[ty * 36 + tx], ez = sEz[ty * 36 + tx];
            float ey_xp = sEy[ty * 36 + tx + 1], ez_xp = sEz[ty * 36 + tx + 1];
            float ex_yp = sEx[(ty + 1) * 32 + tx], ez_yp = sEz[(ty + 1) * 36 + tx];
            float ex_zp = ((const float*)(Bn + HStage::EX))[ty * 32 + tx];
            float ey_zp = ((const float*)(Bn + HStage::EY))[ty * 36 + tx];
            if (ix == nx - 1 && bxr != MFD_BC_DIRICHLET) {
                ey_xp = bxr == MFD_BC_PERIODIC ? p.Ey[c - (nx - 1)] : ey;
                ez_xp = bxr == MFD_BC_PERIODIC ? p.Ez[c - (nx - 1)] : ez;
            }
            if (iy == ny - 1 && byr != MFD_BC_DIRICHLET) {
                ex_yp = byr == MFD_BC_PERIODIC ? p.Ex[c - (ny - 1) * sy] : ex;
                ez_yp = byr == MFD_BC_PERIODIC ? p.Ez[c - (ny - 1) * sy] : ez;
            }
            if (iz == nz - 1 && bzr != MFD_BC_DIRICHLET) {
                ex_zp = bzr == MFD_BC_PERIODIC ? p.Ex[c - (nz - 1) * sz] : ex;
                ey_zp = bzr == MFD_BC_PERIODIC ? p.Ey[c - (nz - 1) * sz] : ey;
            }
            float hx = ((const float*)(A + HStage::HX))[ty * 32 + tx];
            float hy = ((const float*)(A + HStage::HY))[ty * 32 + tx];
            float hz = ((const float*)(A + HStage::HZ))[ty * 32 + tx];
            if (p.accum) {
                const float a = ey * hz - ez * hy, b = ez * hx - ex * hz, d = ex * hy - ey * hx;
                p.Sa[c] = ((const float*)(A + HStage::SA))[ty * 32 + tx] + sqrt0(a * a + b * b + d * d) * p.dt;
                if (p.sum_e2)
                    p.E2[c] = ((const float*)(A + HStage::E2))[ty * 32 + tx] + (ex * ex + ey * ey + ez * ez) * p.dt;
                guard(p, ex);
            }
            float Mh = p.Mh0;
            if (MATH) {
                const int g = (A + HStage::G)[ty * 32 + tx];
                if (g) Mh = p.matMh[g - 1];
            }
            float dExy = cdiv<FAST>(ex_yp - ex, p.ddy);
            float dExz = cdiv<FAST>(ex_zp - ex, p.ddz);
            float dEyx = cdiv<FAST>(ey_xp - ey, p.ddx);
            float dEyz = cdiv<FAST>(ey_zp - ey, p.ddz);
            float dEzx = cdiv<FAST>(ez_xp - ez, p.ddx);
            float dEzy = cdiv<FAST>(ez_yp - ez, p.ddy);
            if (cxy || in_layers(p.lay[MFD_ZL], p.lay[MFD_ZR], iz)) {
                const LayerDev<float>&lxl = p.lay[MFD_XL], &lxr = p.lay[MFD_XR], &lyl = p.lay[MFD_YL],
                                      &lyr = p.lay[MFD_YR], &lzl = p.lay[MFD_ZL], &lzr = p.lay[MFD_ZR];
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
            hx -= Mh * (dEzy - dEyz);
            hy -= Mh * (dExz - dEzx);
            hz -= Mh * (dEyx - dExy);
            p.Hx[c] = hx;
            p.Hy[c] = hy;
            p.Hz[c] = hz;
        }
        __syncthreads();   // stage s0 fully read
        if (tid == 0 && l + TMA_STAGES < NP) {
            h_issue<MATH>(P, smem + s0 * HStage::BYTES, &bars[s0], x0, y0, z0 + l + TMA_STAGES);
            ++issued;
        }
    }
    if (lfail >= 0 && tid == 0) {
        atomicExch(P.timeout, 1);
        // let the copies still in flight land (bounded) before the CTA's shared memory is released
        for (int l = lfail; l < issued; ++l) mbar_wait(&bars[l % TMA_STAGES], (l / TMA_STAGES) & 1);
    }
}

template <bool MAT, typename R>
__device__ __forceinline__ void e_issue(const ETmaParams<R>& P, unsigned char* st, uint64_t* bar, int x0, int y0, int z) {
    mbar_expect_tx(bar, 1152 + 1152 + 1296 + 3 * 1024 + (MAT ? 256 : 0));
    tma_load_3d(st + EStage::HX, &P.mHx, x0, y0 - 1, z, bar);
    tma_load_3d(st + EStage::HY, &P.mHy, x0 - 4, y0, z, bar);
    tma_load_3d(st + EStage::HZ, &P.mHz, x0 - 4, y0 - 1, z, bar);
    tma_load_3d(st + EStage::DX, &P.mDx, x0, y0, z, bar);
    tma_load_3d(st + EStage::DY, &P.mDy, x0, y0, z, bar);
    tma_load_3d(st + EStage::DZ, &P.mDz, x0, y0, z, bar);
    if (MAT) tma_load_3d(st + EStage::G, &P.mG, x0, y0, z, bar);
}

template <typename R, bool MAT, bool FAST>
__global__ void __launch_bounds__(256, 3) e3d_tma_kernel(const __grid_constant__ ETmaParams<R> P, const int zc) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[TMA_STAGES];
    const EParams<float, R>& p = P.p;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TMA_BX + tx;
    const int x0 = blockIdx.x * TMA_BX, y0 = blockIdx.y * TMA_BY;
    const int ix = x0 + tx, iy = y0 + ty;
    const int nx = p.L.nx, ny = p.L.ny, nz = p.L.nz;
    const int z0 = blockIdx.z * zc;
    const int z1 = min(z0 + zc, nz);
    const int NP = z1 - z0 + 1;                     // planes z0-1 .. z1-1 (z0-1 for the z-1 neighbour)
    if (tid == 0) {
        for (int s = 0; s < TMA_STAGES; ++s) mbar_init(&bars[s], 1);
        fence_async_shared();
    }
    __syncthreads();
    int issued = 0;   // planes issued so far (thread 0 is the only issuer)
    if (tid == 0)
        for (; issued < TMA_STAGES && issued < NP; ++issued)
            e_issue<MAT>(P, smem + issued * EStage::BYTES, &bars[issued], x0, y0, z0 - 1 + issued);
    const bool active = ix < nx && iy < ny;
    const int sy = p.L.px, sz = p.L.sz;
    const int bxl = p.bc[MFD_XL], byl = p.bc[MFD_YL], bzl = p.bc[MFD_ZL];
    const bool cxy = in_layers(p.lay[MFD_XL], p.lay[MFD_XR], ix) || in_layers(p.lay[MFD_YL], p.lay[MFD_YR], iy);
    int lfail = __syncthreads_and(mbar_wait(&bars[0], 0)) ? -1 : 0;
    for (int l = 1; l < NP && lfail < 0; ++l) {
        const int iz = z0 + l - 1;
        const int sp = (l - 1) % TMA_STAGES, s0 = l % TMA_STAGES;
        if (!__syncthreads_and(mbar_wait(&bars[s0], (l / TMA_STAGES) & 1))) {   // block-uniform decision
            lfail = l;
            break;
        }
        const unsigned char* Pv = smem + sp * EStage::BYTES;
        const unsigned char* A = smem + s0 * EStage::BYTES;
        if (active) {
            const float* sHx = (const float*)(A + EStage::HX);
            const float* sHy = (const float*)(A + EStage::HY);
            const float* sHz = (const float*)(A + EStage::HZ);
            const int c = ix + sy * iy + sz * iz;
            const float hx = sHx[(ty + 1) * 32 + tx], hy = sHy[ty * 36 + tx + 4], hz = sHz[(ty + 1) * 36 + tx + 4];
            float hy_xm = sHy[ty * 36 + tx + 3], hz_xm = sHz[(ty + 1) * 36 + tx + 3];
            float hx_ym = sHx[ty * 32 + tx], hz_ym = sHz[ty * 36 + tx + 4];
            float hx_zm = ((const float*)(Pv + EStage::HX))[(ty + 1) * 32 + tx];
            float hy_zm = ((const float*)(Pv + EStage::HY))[ty * 36 + tx + 4];
            if (ix == 0 && bxl != MFD_BC_DIRICHLET) {
                hy_xm = bxl == MFD_BC_PERIODIC ? p.Hy[c + (nx - 1)] : hy;
                hz_xm = bxl == MFD_BC_PERIODIC ? p.Hz[c + (nx - 1)] : hz;
            }
            if (iy == 0 && byl != MFD_BC_DIRICHLET) {
                hx_ym = byl == MFD_BC_PERIODIC ? p.Hx[c + (ny - 1) * sy] : hx;
                hz_ym = byl == MFD_BC_PERIODIC ? p.Hz[c + (ny - 1) * sy] : hz;
            }
            if (iz == 0 && bzl != MFD_BC_DIRICHLET) {
                hx_zm = bzl == MFD_BC_PERIODIC ? p.Hx[c + (nz - 1) * sz] : hx;
                hy_zm = bzl == MFD_BC_PERIODIC ? p.Hy[c + (nz - 1) * sz] : hy;
            }
            float dHxy = cdiv<FAST>(hx - hx_ym, p.ddy);
            float dHxz = cdiv<FAST>(hx - hx_zm, p.ddz);
            float dHyx = cdiv<FAST>(hy - hy_xm, p.ddx);
            float dHyz = cdiv<FAST>(hy - hy_zm, p.ddz);
            float dHzx = cdiv<FAST>(hz - hz_xm, p.ddx);
            float dHzy = cdiv<FAST>(hz - hz_ym, p.ddy);
            float Md1 = p.Md10, Md2 = p.Md20, Me = p.Me0;
            bool simple = true;
            if (MAT) {
                const int g = (A + EStage::G)[ty * 32 + tx];
                if (g) {
                    const MatDev<float, R>& m = p.mats[g - 1];
                    Md1 = m.Md1; Md2 = m.Md2; Me = m.Me; simple = m.simple != 0;
                }
            }
            float D0 = ((const float*)(A + EStage::DX))[ty * 32 + tx];
            float D1 = ((const float*)(A + EStage::DY))[ty * 32 + tx];
            float D2 = ((const float*)(A + EStage::DZ))[ty * 32 + tx];
            if (cxy || in_layers(p.lay[MFD_ZL], p.lay[MFD_ZR], iz)) {
                const LayerDev<float>&lxl = p.lay[MFD_XL], &lxr = p.lay[MFD_XR], &lyl = p.lay[MFD_YL],
                                      &lyr = p.lay[MFD_YR], &lzl = p.lay[MFD_ZL], &lzr = p.lay[MFD_ZR];
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
            D0 = Md1 * D0 + Md2 * (dHzy - dHyz);
            D1 = Md1 * D1 + Md2 * (dHxz - dHzx);
            D2 = Md1 * D2 + Md2 * (dHyx - dHxy);
            p.Dx[c] = D0;
            p.Dy[c] = D1;
            p.Dz[c] = D2;
            if (simple) {
                p.Ex[c] = D0 * Me;
                p.Ey[c] = D1 * Me;
                p.Ez[c] = D2 * Me;
            }
        }
        __syncthreads();   // stage sp fully read
        if (tid == 0 && (l - 1) + TMA_STAGES < NP) {
            e_issue<MAT>(P, smem + sp * EStage::BYTES, &bars[sp], x0, y0, z0 - 1 + (l - 1) + TMA_STAGES);
            ++issued;
        }
    }
    if (lfail >= 0 && tid == 0) {
        atomicExch(P.timeout, 1);
        for (int l = lfail; l < issued; ++l) mbar_wait(&bars[l % TMA_STAGES], (l / TMA_STAGES) & 1);
    }
}

}  // namespace mfd
