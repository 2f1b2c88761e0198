// yee3d_async.cuh -- single-precision 3-D core-row updates with the z-planes staged in shared
// memory by asynchronous copies (sm_100a).
//
// h3d_core_kernel / e3d_core_kernel keep the next plane's values in registers, so the bytes a
// warp has in flight are bounded by its registers.  Here a block of 32 x 4 threads owns a
// 32 x 4 column tile of the core rows and marches it along z through a ring of shared-memory
// stages.  A stage holds one plane of the curl's operand field for the tile plus the halo
// the stencil needs (H update: the x+1 column and y+1 row of E; E update: the x-1 column and
// y-1 row of H) and the tile's own arrays (Hx Hy Hz Sa E2, or Dx Dy Dz).  Each thread issues
// its share of the 16-byte cp.async copies a few planes ahead from addresses computed once;
// the copies hold no registers.  The neighbours come from shared memory (z+1 from the next
// stage, z-1 from the previous one); a cell whose neighbour lies across a grid face takes the
// boundary condition's value (a plain load for a periodic face).  The x-layer psi pair and the
// material index are prefetched in registers as in the register march.  The per-cell
// arithmetic is h3d_core_kernel's / e3d_core_kernel's, operation for operation, so results
// are bit-identical.
//
// Ring safety: the copy issued while plane iz is computed goes to the stage last read at
// iteration iz - 2, and every thread has passed the barrier of iteration iz - 1, so one
// barrier per plane suffices.
#pragma once

#include <type_traits>

#include "yee3d_split.cuh"

namespace mfd {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

#define MFD_AS_TY 4   // rows of a staged tile (a block is 32 x MFD_AS_TY threads)
constexpr int AS_TX = 32, AS_TY = MFD_AS_TY, AS_NST = 5, AS_AHEAD = 3;
constexpr int AS_EW = AS_TX + 4;   // E rows: the tile's 32 columns and the 16-byte chunk holding x+1
static_assert(AS_NST - AS_AHEAD == 2, "one barrier per plane needs two stages of slack");

struct HAStage {
    float ex[AS_TY + 1][AS_EW];   // rows y0 .. y0+AS_TY (the last is the y+1 row)
    float ey[AS_TY + 1][AS_EW];
    float ez[AS_TY + 1][AS_EW];
    float hx[AS_TY][AS_TX], hy[AS_TY][AS_TX], hz[AS_TY][AS_TX], sa[AS_TY][AS_TX], e2[AS_TY][AS_TX];
};
constexpr int AS_NE = 3 * (AS_TY + 1) * (AS_EW / 4);   // 16-byte chunks of E per stage
constexpr int AS_NO = 5 * AS_TY * (AS_TX / 4);          // ... of the tile's own arrays
constexpr int AS_SLOTS = (AS_NE + AS_NO + AS_TX * AS_TY - 1) / (AS_TX * AS_TY);

__device__ __forceinline__ void cp_async16(uint32_t smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

#define MFD_HASYNC_MINB (1024 / (32 * MFD_AS_TY))   // 1024 resident threads per SM (64 registers)
// The tolerance mode's shorter cell code fits 10 blocks per SM (48 registers): 256^3 plasmonics
// 42.2 against 41.9 Gcell/s; the exact code there lost more (37.1 against 40.1), so it keeps 8.
#define MFD_ASYNC_MINB_RECIP 10
// The layer launches' exact-mode cell code (x, y and z faces) spills at 64 registers: 6 blocks.
#define MFD_ASYNC_MINB_LAY 6

// LAY: 0 the core rows; 1 the rows of the y layers over the core planes (s.yl .. s.yr is
// one y layer's rows); 2 the planes of one z layer (s.zl .. s.zr), every row.  A thread's row
// keeps its y face along the march and a plane's z face holds for the whole block, so a layer
// cell costs its psi pair (prefetched with the next plane like the x face's) and a few flops,
// in the CPML slab kernels' face order (x, y, z).
template <bool MATH, int FAST, bool ACC, bool E2S, int LAY = 0>
__global__ void __launch_bounds__(AS_TX * AS_TY, LAY ? (FAST == DIV_RECIP ? MFD_HASYNC_MINB : MFD_ASYNC_MINB_LAY)
                                                      : (FAST == DIV_RECIP ? MFD_ASYNC_MINB_RECIP : MFD_HASYNC_MINB))
    h3d_core_async_kernel(const __grid_constant__ HParams<float> p, const Div3 D3, const SplitBox s) {
    __shared__ __align__(16) HAStage S[AS_NST];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + AS_TX * ty;
    const int nx = p.L.nx, ny = p.L.ny, nz = p.L.nz;
    const int sy = p.L.px, sz = p.L.sz;
    const int x0 = blockIdx.x * AS_TX;
    const int y0 = s.yl + blockIdx.y * AS_TY;
    const int z0 = s.zl + blockIdx.z * s.zc;
    const int z1 = min(z0 + s.zc, s.zr);
    const int ix = x0 + tx, iy = y0 + ty;
    const bool act = ix < nx && iy < s.yr;

    // This thread's copy slots: source (plane 0), destination (stage 0) and the planes it
    // copies -- E chunks of rows y <= yr (the tile's rows and the y+1 row) for planes up to
    // z1, own-array chunks of rows y < yr for the computed planes.  The x+1 chunk only when
    // the tile's x+1 column is a grid cell.  Rows start on 16-byte boundaries (pitch and
    // x0 are multiples of 32 elements), and a row's 32-column chunks stay inside its pitch.
    const float* src[AS_SLOTS];
    uint32_t dst[AS_SLOTS];
    int last[AS_SLOTS];   // last plane the slot copies (exclusive bound), -1: unused
#pragma unroll
    for (int j = 0; j < AS_SLOTS; ++j) {
        const int q = tid + j * AS_TX * AS_TY;
        src[j] = p.Ex;
        dst[j] = 0;
        last[j] = -1;
        if (q < AS_NE) {
            const int a = q / ((AS_TY + 1) * (AS_EW / 4)), rem = q - a * ((AS_TY + 1) * (AS_EW / 4));
            const int r = rem / (AS_EW / 4), c = rem - r * (AS_EW / 4);
            const int y = y0 + r;
            if (y < ny && y <= s.yr && (c < AS_TX / 4 || x0 + AS_TX <= nx - 1)) {
                src[j] = (a == 0 ? p.Ex : a == 1 ? p.Ey : p.Ez) + (long long)sy * y + x0 + 4 * c;
                dst[j] = smem_u32(a == 0 ? &S[0].ex[r][4 * c] : a == 1 ? &S[0].ey[r][4 * c] : &S[0].ez[r][4 * c]);
                last[j] = min(z1 + 1, nz);
            }
        } else if (q < AS_NE + AS_NO) {
            const int q2 = q - AS_NE, a = q2 / (AS_TY * AS_TX / 4), rem = q2 - a * (AS_TY * AS_TX / 4);
            const int r = rem / (AS_TX / 4), c = rem - r * (AS_TX / 4);
            const int y = y0 + r;
            const bool want = a < 3 || (a == 3 && ACC) || (a == 4 && ACC && E2S);
            if (want && y < s.yr) {
                const float* base = a == 0 ? p.Hx : a == 1 ? p.Hy : a == 2 ? p.Hz : a == 3 ? p.Sa : p.E2;
                float* d = a == 0 ? &S[0].hx[r][4 * c]
                         : a == 1 ? &S[0].hy[r][4 * c]
                         : a == 2 ? &S[0].hz[r][4 * c]
                         : a == 3 ? &S[0].sa[r][4 * c] : &S[0].e2[r][4 * c];
                src[j] = base + (long long)sy * y + x0 + 4 * c;
                dst[j] = smem_u32(d);
                last[j] = z1;
            }
        }
    }
    auto issue = [&](int pz) {
        const uint32_t so = (uint32_t)((pz % AS_NST) * sizeof(HAStage));
#pragma unroll
        for (int j = 0; j < AS_SLOTS; ++j)
            if (pz < last[j]) cp_async16(dst[j] + so, src[j] + (long long)sz * pz);
        cp_async_commit();
    };

    const int bxr = p.bc[MFD_XR], byr = p.bc[MFD_YR], bzr = p.bc[MFD_ZR];
    const XCol<float> X = xcol<float>(p.lay[MFD_XL], p.lay[MFD_XR], act ? ix : 0, 2, 3);   // H uses psi pair (2, 3)
    const bool xin = act && X.in;
    const int kstep = X.nb * ny;
    int k = X.q + X.nb * (iy + ny * z0);
    const float dt = p.dt, Mh0 = p.Mh0;
    int c = ix + sy * iy + sz * z0;
    // the next plane's material index and x-layer psi pair, prefetched in registers
    int g_next = (MATH && act) ? (int)p.geom[c] : 0;
    float pa_next = xin ? X.pa[k] : 0.0f, pb_next = xin ? X.pb[k] : 0.0f;
    // the row's y face (LAY >= 1) and the planes' z face (LAY 2)
    const XCol<float> Y = LAY ? xcol<float>(p.lay[MFD_YL], p.lay[MFD_YR], act ? iy : 0, 2, 3) : XCol<float>{};
    const bool yin = LAY && act && Y.in;
    const int kystep = sy * Y.nb;
    int ky = ix + sy * (Y.q + Y.nb * z0);
    float ya_next = yin ? Y.pa[ky] : 0.0f, yb_next = yin ? Y.pb[ky] : 0.0f;
    const bool zlo = p.lay[MFD_ZL].nb && z0 < p.lay[MFD_ZL].ib;
    const LayerDev<float>& LZ = p.lay[zlo ? MFD_ZL : MFD_ZR];
    const int zq0 = zlo ? 0 : LZ.ib - 1;   // plane iz is the layer's point iz - zq0
    const bool zin = LAY == 2 && act;
    int kz = ix + sy * (iy + ny * (z0 - zq0));
    float za_next = zin ? LZ.psi[2][kz] : 0.0f, zb_next = zin ? LZ.psi[3][kz] : 0.0f;

    // Blocks away from the upper x and y faces, on planes below the last, need no boundary
    // condition and no activity test (a block-uniform choice of the code path).
    const bool inner_xy = x0 + AS_TX <= nx - 1 && y0 + AS_TY <= s.yr && y0 + AS_TY <= ny - 1;
    auto cell = [&](auto inner_tag, const HAStage& A, const HAStage& Bn, int iz, int g, float cpa, float cpb, float cya,
                    float cyb, float cza, float czb) {
        constexpr bool IN = decltype(inner_tag)::value;
        const float ex = A.ex[ty][tx], ey = A.ey[ty][tx], ez = A.ez[ty][tx];
        float ey_xp, ez_xp, ex_yp, ez_yp, ex_zp, ey_zp;
        if (IN || ix < nx - 1) {
            ey_xp = A.ey[ty][tx + 1];
            ez_xp = A.ez[ty][tx + 1];
        } else if (bxr == MFD_BC_PERIODIC) {
            ey_xp = p.Ey[c - (nx - 1)];
            ez_xp = p.Ez[c - (nx - 1)];
        } else if (bxr == MFD_BC_DIRICHLET) {
            ey_xp = 0.0f;
            ez_xp = 0.0f;
        } else {
            ey_xp = ey;
            ez_xp = ez;
        }
        if (IN || iy < ny - 1) {
            ex_yp = A.ex[ty + 1][tx];
            ez_yp = A.ez[ty + 1][tx];
        } else if (byr == MFD_BC_PERIODIC) {
            ex_yp = p.Ex[c - (ny - 1) * sy];
            ez_yp = p.Ez[c - (ny - 1) * sy];
        } else if (byr == MFD_BC_DIRICHLET) {
            ex_yp = 0.0f;
            ez_yp = 0.0f;
        } else {
            ex_yp = ex;
            ez_yp = ez;
        }
        if (IN || iz < nz - 1) {
            ex_zp = Bn.ex[ty][tx];
            ey_zp = Bn.ey[ty][tx];
        } else if (bzr == MFD_BC_PERIODIC) {
            ex_zp = p.Ex[c - (nz - 1) * sz];
            ey_zp = p.Ey[c - (nz - 1) * sz];
        } else if (bzr == MFD_BC_DIRICHLET) {
            ex_zp = 0.0f;
            ey_zp = 0.0f;
        } else {
            ex_zp = ex;
            ey_zp = ey;
        }
        float hx = A.hx[ty][tx], hy = A.hy[ty][tx], hz = A.hz[ty][tx];
        if (ACC) {
            const float a = mad<FAST>(ey, hz, -(ez * hy)), b = mad<FAST>(ez, hx, -(ex * hz)), d = mad<FAST>(ex, hy, -(ey * hx));
            p.Sa[c] = mad<FAST>(sqrtm<FAST>(sum3sq<FAST>(a, b, d)), dt, A.sa[ty][tx]);
            if (E2S) p.E2[c] = mad<FAST>(sum3sq<FAST>(ex, ey, ez), dt, A.e2[ty][tx]);
            if (maybe_nonfinite(ex)) guard(p, ex);
        }
        float Mh = Mh0;
        if (MATH && g) Mh = p.matMh[g - 1];
        const float num[6] = {ex_yp - ex, ex_zp - ex, ey_xp - ey, ey_zp - ey, ez_xp - ez, ez_yp - ez};
        float q[6];
        div6<FAST>(D3, num, q);
        float dExy = q[0], dExz = q[1], dEyz = q[3], dEzy = q[5];
        float dEyx = q[2], dEzx = q[4];
        if (xin) {   // cpml_h<+1> of the column's x face
            const float pa = mad<FAST>(X.B, cpa, X.A * dEyx);
            const float pb = mad<FAST>(X.B, cpb, X.A * dEzx);
            X.pa[k] = pa;
            X.pb[k] = pb;
            hy = mad<FAST>(Mh, pb, hy);
            hz = mad<FAST>(-Mh, pa, hz);
            dEyx = cdiv<FAST>(dEyx, X.K);
            dEzx = cdiv<FAST>(dEzx, X.K);
        }
        if (LAY && yin) {   // cpml_h<-1> of the row's y face
            const float pa = mad<FAST>(Y.B, cya, Y.A * dExy);
            const float pb = mad<FAST>(Y.B, cyb, Y.A * dEzy);
            Y.pa[ky] = pa;
            Y.pb[ky] = pb;
            hx = mad<FAST>(-Mh, pb, hx);
            hz = mad<FAST>(Mh, pa, hz);
            dExy = cdiv<FAST>(dExy, Y.K);
            dEzy = cdiv<FAST>(dEzy, Y.K);
        }
        if (LAY == 2) {   // cpml_h<+1> of the plane's z face
            const int qz = iz - zq0;
            const float B = LZ.B[qz], A = LZ.A[qz];
            const float pa = mad<FAST>(B, cza, A * dExz);
            const float pb = mad<FAST>(B, czb, A * dEyz);
            LZ.psi[2][kz] = pa;
            LZ.psi[3][kz] = pb;
            hx = mad<FAST>(Mh, pb, hx);
            hy = mad<FAST>(-Mh, pa, hy);
            dExz = cdiv<FAST>(dExz, LZ.K[qz]);
            dEyz = cdiv<FAST>(dEyz, LZ.K[qz]);
        }
        hx = mad<FAST>(-Mh, dEzy - dEyz, hx);
        hy = mad<FAST>(-Mh, dExz - dEzx, hy);
        hz = mad<FAST>(-Mh, dEyx - dExy, hz);
        p.Hx[c] = hx;
        p.Hy[c] = hy;
        p.Hz[c] = hz;
    };

#pragma unroll
    for (int j = 0; j < AS_AHEAD; ++j) issue(z0 + j);
    int sc = z0 % AS_NST;   // stage of plane iz
    for (int iz = z0; iz < z1; ++iz, c += sz, k += kstep, ky += kystep, kz += sy * ny) {
        issue(iz + AS_AHEAD);
        const int g = g_next;
        const float cpa = pa_next, cpb = pb_next, cya = ya_next, cyb = yb_next, cza = za_next, czb = zb_next;
        if (iz + 1 < z1) {
            g_next = (MATH && act) ? (int)p.geom[c + sz] : 0;
            pa_next = xin ? X.pa[k + kstep] : 0.0f;
            pb_next = xin ? X.pb[k + kstep] : 0.0f;
            if (LAY) {
                ya_next = yin ? Y.pa[ky + kystep] : 0.0f;
                yb_next = yin ? Y.pb[ky + kystep] : 0.0f;
            }
            if (LAY == 2) {
                za_next = zin ? LZ.psi[2][kz + sy * ny] : 0.0f;
                zb_next = zin ? LZ.psi[3][kz + sy * ny] : 0.0f;
            }
        }
        const int sn = sc == AS_NST - 1 ? 0 : sc + 1;
        cp_async_wait<AS_AHEAD - 1>();   // this thread's copies of planes iz and iz+1 have landed
        __syncthreads();                 // ... and every other thread's
        if (inner_xy && iz < nz - 1) cell(std::true_type{}, S[sc], S[sn], iz, g, cpa, cpb, cya, cyb, cza, czb);
        else if (act) cell(std::false_type{}, S[sc], S[sn], iz, g, cpa, cpb, cya, cyb, cza, czb);
        sc = sn;
    }
    cp_async_wait<0>();
}

// The E update of the core rows.  The z-1 neighbours are the previous plane's stage, so a
// block's ring starts one plane before its first.
struct EAStage {
    float hx[AS_TY + 1][AS_EW];   // rows y0-1 .. y0+3 (row 0 is the y-1 row), columns x0-4 .. x0+31
    float hy[AS_TY + 1][AS_EW];
    float hz[AS_TY + 1][AS_EW];
    float dx[AS_TY][AS_TX], dy[AS_TY][AS_TX], dz[AS_TY][AS_TX];
};
constexpr int EA_NO = 3 * AS_TY * (AS_TX / 4);
constexpr int EA_SLOTS = (AS_NE + EA_NO + AS_TX * AS_TY - 1) / (AS_TX * AS_TY);
constexpr int EA_NST = 5, EA_AHEAD = EA_NST - 3;   // the copy issued at plane iz lands in the stage last read at iz - 2

#define MFD_EASYNC_MINB (1024 / (32 * MFD_AS_TY))   // 1024 resident threads per SM (64 registers)
// The tolerance mode's E layer launches without a material map fit 9 blocks per SM (56
// registers, at most 4 bytes of spill): 256^3 plasmonics 45.19 against 44.97-44.99 Gcell/s
// at 8 (the H layer code spills 32-116 bytes there and measured slower: 44.78-44.79 with
// both at 9).  With the map (materials in a layer) the z-layer code would spill 84 bytes at
// 56 registers, so those keep 8 blocks.
#define MFD_EASYNC_MINB_LAY_RECIP 9

// skip: the tiles of the materials' columns, rows and planes, left to another kernel (the
// register march with the material map).
// LAY as for h3d_core_async_kernel: the rows of a y layer (1) or the planes of a z layer (2).
template <typename R, bool MAT, int FAST, int LAY = 0>
__global__ void __launch_bounds__(AS_TX * AS_TY, LAY ? (FAST == DIV_RECIP ? (MAT ? MFD_EASYNC_MINB : MFD_EASYNC_MINB_LAY_RECIP)
                                                                            : MFD_ASYNC_MINB_LAY)
                                                      : (FAST == DIV_RECIP ? MFD_ASYNC_MINB_RECIP : MFD_EASYNC_MINB))
    e3d_core_async_kernel(const __grid_constant__ EParams<float, R> p, const Div3 D3, const SplitBox s, const TileSkip skip) {
    __shared__ __align__(16) EAStage S[EA_NST];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + AS_TX * ty;
    const int nx = p.L.nx, ny = p.L.ny, nz = p.L.nz;
    const int sy = p.L.px, sz = p.L.sz;
    const int x0 = blockIdx.x * AS_TX;
    const int y0 = s.yl + blockIdx.y * AS_TY;
    const int z0 = s.zl + blockIdx.z * s.zc;
    if (x0 >= skip.x0 && x0 < skip.x1 && y0 >= skip.y0 && y0 < skip.y1 && z0 >= skip.z0 && z0 < skip.z1) return;   // block-uniform
    const int z1 = min(z0 + s.zc, s.zr);
    const int ix = x0 + tx, iy = y0 + ty;
    const bool act = ix < nx && iy < s.yr;

    // Copy slots: H rows y0-1 .. y0+3 inside the grid and below yr (the x-1 chunk when x0 > 0)
    // for planes z0-1 .. z1-1, the tile's Dx Dy Dz rows (y < yr) for the computed planes.
    const float* src[EA_SLOTS];
    uint32_t dst[EA_SLOTS];
    unsigned hmask = 0, dmask = 0;   // slot j copies H (planes z0-1 .. z1-1) / D (planes z0 .. z1-1)
#pragma unroll
    for (int j = 0; j < EA_SLOTS; ++j) {
        const int q = tid + j * AS_TX * AS_TY;
        src[j] = p.Hx;
        dst[j] = 0;
        if (q < AS_NE) {
            const int a = q / ((AS_TY + 1) * (AS_EW / 4)), rem = q - a * ((AS_TY + 1) * (AS_EW / 4));
            const int r = rem / (AS_EW / 4), c = rem - r * (AS_EW / 4);
            const int y = y0 - 1 + r;
            if (y >= 0 && y < s.yr && (c > 0 || x0 > 0)) {
                src[j] = (a == 0 ? p.Hx : a == 1 ? p.Hy : p.Hz) + (long long)sy * y + x0 - 4 + 4 * c;
                dst[j] = smem_u32(a == 0 ? &S[0].hx[r][4 * c] : a == 1 ? &S[0].hy[r][4 * c] : &S[0].hz[r][4 * c]);
                hmask |= 1u << j;
            }
        } else if (q < AS_NE + EA_NO) {
            const int q2 = q - AS_NE, a = q2 / (AS_TY * AS_TX / 4), rem = q2 - a * (AS_TY * AS_TX / 4);
            const int r = rem / (AS_TX / 4), c = rem - r * (AS_TX / 4);
            const int y = y0 + r;
            if (y < s.yr) {
                src[j] = (a == 0 ? p.Dx : a == 1 ? p.Dy : p.Dz) + (long long)sy * y + x0 + 4 * c;
                dst[j] = smem_u32(a == 0 ? &S[0].dx[r][4 * c] : a == 1 ? &S[0].dy[r][4 * c] : &S[0].dz[r][4 * c]);
                dmask |= 1u << j;
            }
        }
    }
    auto issue = [&](int pz) {
        if (pz >= 0 && pz < z1) {
            const uint32_t so = (uint32_t)((pz % EA_NST) * sizeof(EAStage));
            const unsigned m = hmask | (pz >= z0 ? dmask : 0u);
#pragma unroll
            for (int j = 0; j < EA_SLOTS; ++j)
                if (m & (1u << j)) cp_async16(dst[j] + so, src[j] + (long long)sz * pz);
        }
        cp_async_commit();
    };

    const int bxl = p.bc[MFD_XL], byl = p.bc[MFD_YL], bzl = p.bc[MFD_ZL];
    const XCol<float> X = xcol<float>(p.lay[MFD_XL], p.lay[MFD_XR], act ? ix : 0, 0, 1);   // E uses psi pair (0, 1)
    const bool xin = act && X.in;
    const int kstep = X.nb * ny;
    int k = X.q + X.nb * (iy + ny * z0);
    const float Md10 = p.Md10, Md20 = p.Md20, Me0 = p.Me0;
    int c = ix + sy * iy + sz * z0;
    // the next plane's material index and x-layer psi pair, prefetched in registers
    int g_next = (MAT && act) ? (int)p.geom[c] : 0;
    float pa_next = xin ? X.pa[k] : 0.0f, pb_next = xin ? X.pb[k] : 0.0f;
    // the row's y face (LAY >= 1) and the planes' z face (LAY 2)
    const XCol<float> Y = LAY ? xcol<float>(p.lay[MFD_YL], p.lay[MFD_YR], act ? iy : 0, 0, 1) : XCol<float>{};
    const bool yin = LAY && act && Y.in;
    const int kystep = sy * Y.nb;
    int ky = ix + sy * (Y.q + Y.nb * z0);
    float ya_next = yin ? Y.pa[ky] : 0.0f, yb_next = yin ? Y.pb[ky] : 0.0f;
    const bool zlo = p.lay[MFD_ZL].nb && z0 < p.lay[MFD_ZL].ib;
    const LayerDev<float>& LZ = p.lay[zlo ? MFD_ZL : MFD_ZR];
    const int zq0 = zlo ? 0 : LZ.ib - 1;   // plane iz is the layer's point iz - zq0
    const bool zin = LAY == 2 && act;
    int kz = ix + sy * (iy + ny * (z0 - zq0));
    float za_next = zin ? LZ.psi[0][kz] : 0.0f, zb_next = zin ? LZ.psi[1][kz] : 0.0f;

    // Blocks away from the lower x and y faces (and the grid's x end), on planes above the
    // first, need no boundary condition and no activity test.
    const bool inner_xy = x0 > 0 && x0 + AS_TX <= nx && y0 > 0 && y0 + AS_TY <= s.yr;
    auto cell = [&](auto inner_tag, const EAStage& A, const EAStage& P, int iz, int g, float cpa, float cpb, float cya,
                    float cyb, float cza, float czb) {
        constexpr bool IN = decltype(inner_tag)::value;
        const float hx = A.hx[ty + 1][tx + 4], hy = A.hy[ty + 1][tx + 4], hz = A.hz[ty + 1][tx + 4];
        float hy_xm, hz_xm, hx_ym, hz_ym, hx_zm, hy_zm;
        if (IN || ix > 0) {
            hy_xm = A.hy[ty + 1][tx + 3];
            hz_xm = A.hz[ty + 1][tx + 3];
        } else if (bxl == MFD_BC_PERIODIC) {
            hy_xm = p.Hy[c + (nx - 1)];
            hz_xm = p.Hz[c + (nx - 1)];
        } else if (bxl == MFD_BC_DIRICHLET) {
            hy_xm = 0.0f;
            hz_xm = 0.0f;
        } else {
            hy_xm = hy;
            hz_xm = hz;
        }
        if (IN || iy > 0) {
            hx_ym = A.hx[ty][tx + 4];
            hz_ym = A.hz[ty][tx + 4];
        } else if (byl == MFD_BC_PERIODIC) {
            hx_ym = p.Hx[c + (ny - 1) * sy];
            hz_ym = p.Hz[c + (ny - 1) * sy];
        } else if (byl == MFD_BC_DIRICHLET) {
            hx_ym = 0.0f;
            hz_ym = 0.0f;
        } else {
            hx_ym = hx;
            hz_ym = hz;
        }
        if (IN || iz > 0) {
            hx_zm = P.hx[ty + 1][tx + 4];
            hy_zm = P.hy[ty + 1][tx + 4];
        } else if (bzl == MFD_BC_PERIODIC) {
            hx_zm = p.Hx[c + (nz - 1) * sz];
            hy_zm = p.Hy[c + (nz - 1) * sz];
        } else if (bzl == MFD_BC_DIRICHLET) {
            hx_zm = 0.0f;
            hy_zm = 0.0f;
        } else {
            hx_zm = hx;
            hy_zm = hy;
        }
        const float num[6] = {hx - hx_ym, hx - hx_zm, hy - hy_xm, hy - hy_zm, hz - hz_xm, hz - hz_ym};
        float q[6];
        div6<FAST>(D3, num, q);
        float dHxy = q[0], dHxz = q[1], dHyz = q[3], dHzy = q[5];
        float dHyx = q[2], dHzx = q[4];
        float Md1 = Md10, Md2 = Md20, Me = Me0;
        bool simple = true;
        if (MAT && g) {
            const MatDev<float, R>& m = p.mats[g - 1];
            Md1 = m.Md1; Md2 = m.Md2; Me = m.Me; simple = m.simple != 0;
        }
        float D0 = A.dx[ty][tx], D1 = A.dy[ty][tx], D2 = A.dz[ty][tx];
        if (xin) {   // cpml_e<-1> of the column's x face
            const float pa = mad<FAST>(X.B, cpa, X.A * dHyx);
            const float pb = mad<FAST>(X.B, cpb, X.A * dHzx);
            X.pa[k] = pa;
            X.pb[k] = pb;
            D1 = mad<FAST>(-Md2, pb, D1);
            D2 = mad<FAST>(Md2, pa, D2);
            dHyx = cdiv<FAST>(dHyx, X.K);
            dHzx = cdiv<FAST>(dHzx, X.K);
        }
        if (LAY && yin) {   // cpml_e<+1> of the row's y face
            const float pa = mad<FAST>(Y.B, cya, Y.A * dHxy);
            const float pb = mad<FAST>(Y.B, cyb, Y.A * dHzy);
            Y.pa[ky] = pa;
            Y.pb[ky] = pb;
            D0 = mad<FAST>(Md2, pb, D0);
            D2 = mad<FAST>(-Md2, pa, D2);
            dHxy = cdiv<FAST>(dHxy, Y.K);
            dHzy = cdiv<FAST>(dHzy, Y.K);
        }
        if (LAY == 2) {   // cpml_e<-1> of the plane's z face
            const int qz = iz - zq0;
            const float B = LZ.B[qz], A = LZ.A[qz];
            const float pa = mad<FAST>(B, cza, A * dHxz);
            const float pb = mad<FAST>(B, czb, A * dHyz);
            LZ.psi[0][kz] = pa;
            LZ.psi[1][kz] = pb;
            D0 = mad<FAST>(-Md2, pb, D0);
            D1 = mad<FAST>(Md2, pa, D1);
            dHxz = cdiv<FAST>(dHxz, LZ.K[qz]);
            dHyz = cdiv<FAST>(dHyz, LZ.K[qz]);
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
    };

#pragma unroll
    for (int j = -1; j < EA_AHEAD; ++j) issue(z0 + j);
    int sc = z0 % EA_NST;                             // stage of plane iz
    int sp = sc == 0 ? EA_NST - 1 : sc - 1;           // ... of plane iz - 1
    for (int iz = z0; iz < z1; ++iz, c += sz, k += kstep, ky += kystep, kz += sy * ny) {
        issue(iz + EA_AHEAD);
        const int g = g_next;
        const float cpa = pa_next, cpb = pb_next, cya = ya_next, cyb = yb_next, cza = za_next, czb = zb_next;
        if (iz + 1 < z1) {
            g_next = (MAT && act) ? (int)p.geom[c + sz] : 0;
            pa_next = xin ? X.pa[k + kstep] : 0.0f;
            pb_next = xin ? X.pb[k + kstep] : 0.0f;
            if (LAY) {
                ya_next = yin ? Y.pa[ky + kystep] : 0.0f;
                yb_next = yin ? Y.pb[ky + kystep] : 0.0f;
            }
            if (LAY == 2) {
                za_next = zin ? LZ.psi[0][kz + sy * ny] : 0.0f;
                zb_next = zin ? LZ.psi[1][kz + sy * ny] : 0.0f;
            }
        }
        cp_async_wait<EA_AHEAD>();   // this thread's copies of planes up to iz have landed
        __syncthreads();             // ... and every other thread's
        if (inner_xy && iz > 0) cell(std::true_type{}, S[sc], S[sp], iz, g, cpa, cpb, cya, cyb, cza, czb);
        else if (act) cell(std::false_type{}, S[sc], S[sp], iz, g, cpa, cpb, cya, cyb, cza, czb);
        sp = sc;
        sc = sc == EA_NST - 1 ? 0 : sc + 1;
    }
    cp_async_wait<0>();
}

}  // namespace mfd
