// batch.cuh -- many independent 2-D and 3-D models stepped together (sm_100a).
//
// Each half-step of every member of a batch is one persistent launch: the grid is sized to
// the GPU (SMs x resident blocks) and each block walks a table of tiles (member, tile
// origin), so hundreds of small, unevenly sized models cost a handful of launches per step
// instead of a handful per model.  Every per-member quantity that changes from step to step
// (the step index, the running-sum flag, the polarisation ping-pong parity) lives in the
// member's device state and is advanced on the device, so a CUDA graph of several steps can
// be replayed unchanged.  The per-cell arithmetic is the single-model code (h2d_cell /
// e2d_cell, the 3-D h3d_cell / e3d_cell of the CPML slabs, material_cell, the point-source
// expression), so a member's results are bit-identical to running it alone.  2-D and 3-D
// members have their own tile tables and kernels (the 3-D cell code needs more registers);
// a 3-D tile covers x cells by (y, z) rows numbered y + ny z.  A block copies its tile's
// member parameter block into shared memory whenever the member changes, so the cells read
// the layout, pointers and coefficients from there rather than through dependent global loads.
#pragma once

#include "aux.cuh"
#include "yee.cuh"
#include "yee3d_split.cuh"

namespace mfd {

enum { BF_MATH = 1, BF_MAT = 2, BF_FAST = 4, BF_3D = 8, BF_RECIP = 16 };

// The half-step kernels come in two sets: DSET 0 runs the members of the exact arithmetic
// (IEEE or the verified constant division), DSET 1 those of the tolerance mode (reciprocal
// multiplies), each launched only when the batch holds such members.  One kernel for both
// measured slower: the extra cell code raised the 2-D E kernel from 32 to 40 registers.
template <int DSET>
__device__ __forceinline__ bool b_other_set(int flags) { return ((flags & BF_RECIP) != 0) != (DSET == 1); }

// Per-member state (device).  Steps are 1-based; the member runs steps first..last.
struct BMember {
    const HParams<float>* hp;              // the member's update parameters (static fields)
    const EParams<float, double>* ep;
    const MonParams<float>* mp;            // monitors (gathered every step)
    const RectParams<float>* rp;           // TFSF statements (null: none)
    long long it;                          // step being run; > last once the member is done
    long long first, last;
    long long ring_first;                  // 0-based step staged in ring slot 0
    int flags;                             // BF_*
    int pad;
    Div3 d3;                               // grid-spacing divisors of a 3-D member (div6)
};

struct BTile {      // cells x0 .. x0+blockDim.x-1 of rows z0 .. z0+blockDim.y-1 of member m
    int m, x0, z0, w;  // 3-D linear tiles: (x0, z0, w) = (x, y, z) of the tile's first cell
};

struct BMatTile {   // one row segment of material g's bounding box: x0 .. x0+blockDim.x-1 at (iy, iz)
    int m, g, x0, iy, iz;
};

struct BSrc {       // one point source of a member (sources.jl:122-131, 235-244)
    float* F;
    const long long* cells;
    const double* wave;
    const double* amp;
    const double* gt;
    long long npts;
    int kind;
    float coeff;
};

struct BPoint {     // point i of source s (entries of one source pass) or of monitor s
    int m, s;
    long long i;
};

struct BRow {       // TFSF statement s of member m (grid rows of one TFSF pass)
    int m, s;
};

__device__ __forceinline__ bool b_active(const BMember& M) { return M.it <= M.last; }

// Copies the member's parameter block (8-byte words) into shared memory; every thread of the
// block takes part (call it where the whole block is).
template <typename P>
__device__ __forceinline__ void b_stage(P* dst, const P* src) {
    static_assert(sizeof(P) % 8 == 0, "parameter blocks are whole 8-byte words");
    const int tid = threadIdx.x + blockDim.x * threadIdx.y, nth = blockDim.x * blockDim.y;
    const long long* s = reinterpret_cast<const long long*>(src);
    long long* d = reinterpret_cast<long long*>(dst);
    for (int i = tid; i < (int)(sizeof(P) / 8); i += nth) d[i] = s[i];
}


#define MFD_B2D_CHUNK 4  // a block takes runs of this many consecutive tiles (fewer member changes)
#define MFD_B2D_MINB 4   // batched 2-D updates: 4 blocks of 512 threads per SM (32 registers; the tolerance set's E
                         // kernel spills 36 bytes there, and still measured 43.9 against 41.4 Gcell/s at 3 blocks)


template <int DSET>
__global__ void __launch_bounds__(512, MFD_B2D_MINB) batch_h2d_kernel(const BMember* __restrict__ mem, const BTile* __restrict__ tiles,
                                                        const int* __restrict__ ntiles) {
    __shared__ __align__(16) HParams<float> sp;
    const int n = *ntiles;
    int cur = -1;
    // Tile t of the block's k-th turn: runs of MFD_B2D_CHUNK tiles, the runs dealt out to the
    // blocks in turn, so t grows with k.
    for (int k = 0;; ++k) {
        const int t = ((k / MFD_B2D_CHUNK) * (int)gridDim.x + (int)blockIdx.x) * MFD_B2D_CHUNK + k % MFD_B2D_CHUNK;
        if (t >= n) break;
        const BTile tl = tiles[t];
        const BMember& M = mem[tl.m];
        if (!b_active(M) || b_other_set<DSET>(M.flags)) continue;   // the same for the whole block
        const int acc = M.it > M.first ? 1 : 0;
        const long long prev = M.it - 1;
        const int flags = M.flags;
        if (tl.m != cur) {   // the block copies the member's parameters to shared memory (42.1 vs 40.8 Gcell/s)
            __syncthreads();          // the previous member's parameters are no longer read
            b_stage(&sp, M.hp);
            __syncthreads();
            cur = tl.m;
        }
        const HParams<float>& p = sp;
        const int ix = tl.x0 + threadIdx.x, iz = tl.z0 + threadIdx.y;
        if (ix >= p.L.nx || iz >= p.L.nz) continue;
        if constexpr (DSET == 1) {
            if (flags & BF_MATH) h2d_cell<float, true, DIV_RECIP>(p, acc, prev, ix, iz);
            else h2d_cell<float, false, DIV_RECIP>(p, acc, prev, ix, iz);
        } else {
            switch (flags & (BF_MATH | BF_FAST)) {
                case 0: h2d_cell<float, false, DIV_IEEE>(p, acc, prev, ix, iz); break;
                case BF_MATH: h2d_cell<float, true, DIV_IEEE>(p, acc, prev, ix, iz); break;
                case BF_FAST: h2d_cell<float, false, DIV_EXACT>(p, acc, prev, ix, iz); break;
                default: h2d_cell<float, true, DIV_EXACT>(p, acc, prev, ix, iz); break;
            }
        }
    }
}

template <int DSET>
__global__ void __launch_bounds__(512, MFD_B2D_MINB) batch_e2d_kernel(const BMember* __restrict__ mem, const BTile* __restrict__ tiles,
                                                        const int* __restrict__ ntiles) {
    __shared__ __align__(16) EParams<float, double> sp;
    const int n = *ntiles;
    int cur = -1;
    // Tile t of the block's k-th turn: runs of MFD_B2D_CHUNK tiles, the runs dealt out to the
    // blocks in turn, so t grows with k.
    for (int k = 0;; ++k) {
        const int t = ((k / MFD_B2D_CHUNK) * (int)gridDim.x + (int)blockIdx.x) * MFD_B2D_CHUNK + k % MFD_B2D_CHUNK;
        if (t >= n) break;
        const BTile tl = tiles[t];
        const BMember& M = mem[tl.m];
        if (!b_active(M) || b_other_set<DSET>(M.flags)) continue;   // the same for the whole block
        const int flags = M.flags;
        if (tl.m != cur) {   // the block copies the member's parameters to shared memory (42.1 vs 40.8 Gcell/s)
            __syncthreads();
            b_stage(&sp, M.ep);
            __syncthreads();
            cur = tl.m;
        }
        const EParams<float, double>& p = sp;
        const int ix = tl.x0 + threadIdx.x, iz = tl.z0 + threadIdx.y;
        if (ix >= p.L.nx || iz >= p.L.nz) continue;
        if constexpr (DSET == 1) {
            if (flags & BF_MAT) e2d_cell<float, double, true, DIV_RECIP>(p, ix, iz);
            else e2d_cell<float, double, false, DIV_RECIP>(p, ix, iz);
        } else {
            switch (flags & (BF_MAT | BF_FAST)) {
                case 0: e2d_cell<float, double, false, DIV_IEEE>(p, ix, iz); break;
                case BF_MAT: e2d_cell<float, double, true, DIV_IEEE>(p, ix, iz); break;
                case BF_FAST: e2d_cell<float, double, false, DIV_EXACT>(p, ix, iz); break;
                default: e2d_cell<float, double, true, DIV_EXACT>(p, ix, iz); break;
            }
        }
    }
}

// ADE / Kerr / plasma response of material g's cells (material_kernel for 2-D members).
__global__ void __launch_bounds__(128) batch_material2d_kernel(const BMember* __restrict__ mem,
                                                               const BMatTile* __restrict__ tiles,
                                                               const int* __restrict__ ntiles) {
    const int n = *ntiles;
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const BMatTile tl = tiles[t];
        const BMember& M = mem[tl.m];
        if (!b_active(M)) continue;
        const EParams<float, double>& p = *M.ep;
        const MatDev<float, double>* m = p.mats + (tl.g - 1);
        const int ix = tl.x0 + threadIdx.x;
        if (ix >= m->bx0 + m->bnx) continue;
        const int c = ix + p.L.sz * tl.iz;
        if (p.geom[c] != tl.g) continue;
        float Dv[2] = {p.Dx[c], p.Dz[c]};
        float* Ep[2] = {p.Ex, p.Ez};
        const int cur = (int)((M.it - 1) & 1);
        const long long bi = (long long)(ix - m->bx0) + (long long)m->bnx * (tl.iz - m->bz0);
        switch (m->nq) {
            case 0: material_cell_n<float, double, 2, 0>(m, bi, Ep, c, Dv, cur, p.dt); break;
            case 1: material_cell_n<float, double, 2, 1>(m, bi, Ep, c, Dv, cur, p.dt); break;
            case 2: material_cell_n<float, double, 2, 2>(m, bi, Ep, c, Dv, cur, p.dt); break;
            case 3: material_cell_n<float, double, 2, 3>(m, bi, Ep, c, Dv, cur, p.dt); break;
            default: material_cell<float, double, 2>(m, ix, 0, tl.iz, Ep, c, Dv, cur, p.dt); break;
        }
    }
}

#define MFD_B3D_MINB 3   // batched 3-D updates held to 40 registers (measured 16.0 against 15.0 Gcell/s at 58)


// The cell of a 3-D tile's thread.  A 3-D tile is a run of cells in x-fastest order (no
// idle lanes at rows shorter than the block): the block's threads take the
// blockDim.x * blockDim.y cells from the tile's first cell (x0, z0, w) = (x, y, z).
__device__ __forceinline__ bool b_cell3(const Layout& L, const BTile& tl, int& ix, int& iy, int& iz) {
    // offset / nx row steps, a few at the tile shapes used: cheaper than two divisions
    ix = tl.x0 + (int)(threadIdx.y * blockDim.x + threadIdx.x);
    iy = tl.z0;
    iz = tl.w;
    while (ix >= L.nx) {
        ix -= L.nx;
        if (++iy == L.ny) {
            iy = 0;
            ++iz;
        }
    }
    return iz < L.nz;
}

#define MFD_B3D_CHUNK 16 // a block takes runs of this many consecutive tiles (fewer member changes)


// The running sums of the previous step are added from a member's second step on.
template <bool MATH, int FAST>
__device__ __forceinline__ void b_h3d_p(const HParams<float>& p, const Div3& d3, long long it, long long first, int ix, int iy,
                                        int iz) {
    if (it == first) h3d_cell<float, MATH, FAST, false, false>(p, d3, it - 1, ix, iy, iz);
    else if (p.sum_e2) h3d_cell<float, MATH, FAST, true, true>(p, d3, it - 1, ix, iy, iz);
    else h3d_cell<float, MATH, FAST, true, false>(p, d3, it - 1, ix, iy, iz);
}

template <int DSET>
__global__ void __launch_bounds__(512, MFD_B3D_MINB) batch_h3d_kernel(const BMember* __restrict__ mem, const BTile* __restrict__ tiles,
                                                        const int* __restrict__ ntiles) {
    __shared__ __align__(16) HParams<float> sp;
    __shared__ Div3 sd3;
    const int n = *ntiles;
    int cur = -1;
    // Tile t of the block's k-th turn: runs of MFD_B3D_CHUNK tiles, the runs dealt out to the
    // blocks in turn, so t grows with k.
    for (int k = 0;; ++k) {
        const int t = ((k / MFD_B3D_CHUNK) * (int)gridDim.x + (int)blockIdx.x) * MFD_B3D_CHUNK + k % MFD_B3D_CHUNK;
        if (t >= n) break;
        const BTile tl = tiles[t];
        const BMember& M = mem[tl.m];
        if (!b_active(M) || b_other_set<DSET>(M.flags)) continue;   // the same for the whole block
        const long long it = M.it, first = M.first;
        const int flags = M.flags;
        if (tl.m != cur) {   // the block copies the member's parameters to shared memory
            __syncthreads();          // the previous member's parameters are no longer read
            b_stage(&sp, M.hp);
            if (threadIdx.x == 0 && threadIdx.y == 0) sd3 = M.d3;
            __syncthreads();
            cur = tl.m;
        }
        const HParams<float>& p = sp;
        const Div3& d3 = sd3;
        int ix, iy, iz;
        if (!b_cell3(p.L, tl, ix, iy, iz)) continue;
        if constexpr (DSET == 1) {
            if (flags & BF_MATH) b_h3d_p<true, DIV_RECIP>(p, d3, it, first, ix, iy, iz);
            else b_h3d_p<false, DIV_RECIP>(p, d3, it, first, ix, iy, iz);
        } else {
            switch (flags & (BF_MATH | BF_FAST)) {
                case 0: b_h3d_p<false, DIV_IEEE>(p, d3, it, first, ix, iy, iz); break;
                case BF_MATH: b_h3d_p<true, DIV_IEEE>(p, d3, it, first, ix, iy, iz); break;
                case BF_FAST: b_h3d_p<false, DIV_EXACT>(p, d3, it, first, ix, iy, iz); break;
                default: b_h3d_p<true, DIV_EXACT>(p, d3, it, first, ix, iy, iz); break;
            }
        }
    }
}

template <int DSET>
__global__ void __launch_bounds__(512, MFD_B3D_MINB) batch_e3d_kernel(const BMember* __restrict__ mem, const BTile* __restrict__ tiles,
                                                        const int* __restrict__ ntiles) {
    __shared__ __align__(16) EParams<float, double> sp;
    __shared__ Div3 sd3;
    const int n = *ntiles;
    int cur = -1;
    // Tile t of the block's k-th turn: runs of MFD_B3D_CHUNK tiles, the runs dealt out to the
    // blocks in turn, so t grows with k.
    for (int k = 0;; ++k) {
        const int t = ((k / MFD_B3D_CHUNK) * (int)gridDim.x + (int)blockIdx.x) * MFD_B3D_CHUNK + k % MFD_B3D_CHUNK;
        if (t >= n) break;
        const BTile tl = tiles[t];
        const BMember& M = mem[tl.m];
        if (!b_active(M) || b_other_set<DSET>(M.flags)) continue;   // the same for the whole block
        const int flags = M.flags;
        if (tl.m != cur) {   // the block copies the member's parameters to shared memory
            __syncthreads();
            b_stage(&sp, M.ep);
            if (threadIdx.x == 0 && threadIdx.y == 0) sd3 = M.d3;
            __syncthreads();
            cur = tl.m;
        }
        const EParams<float, double>& p = sp;
        const Div3& d3 = sd3;
        int ix, iy, iz;
        if (!b_cell3(p.L, tl, ix, iy, iz)) continue;
        if constexpr (DSET == 1) {
            if (flags & BF_MAT) e3d_cell<float, double, true, DIV_RECIP>(p, d3, ix, iy, iz);
            else e3d_cell<float, double, false, DIV_RECIP>(p, d3, ix, iy, iz);
        } else {
            switch (flags & (BF_MAT | BF_FAST)) {
                case 0: e3d_cell<float, double, false, DIV_IEEE>(p, d3, ix, iy, iz); break;
                case BF_MAT: e3d_cell<float, double, true, DIV_IEEE>(p, d3, ix, iy, iz); break;
                case BF_FAST: e3d_cell<float, double, false, DIV_EXACT>(p, d3, ix, iy, iz); break;
                default: e3d_cell<float, double, true, DIV_EXACT>(p, d3, ix, iy, iz); break;
            }
        }
    }
}

// ADE / Kerr / plasma response of material g's cells of 3-D members.
__global__ void __launch_bounds__(128) batch_material3d_kernel(const BMember* __restrict__ mem,
                                                               const BMatTile* __restrict__ tiles,
                                                               const int* __restrict__ ntiles) {
    const int n = *ntiles;
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const BMatTile tl = tiles[t];
        const BMember& M = mem[tl.m];
        if (!b_active(M)) continue;
        const EParams<float, double>& p = *M.ep;
        const MatDev<float, double>* m = p.mats + (tl.g - 1);
        const int ix = tl.x0 + threadIdx.x;
        if (ix >= m->bx0 + m->bnx) continue;
        const int c = ix + p.L.px * tl.iy + p.L.sz * tl.iz;
        if (p.geom[c] != tl.g) continue;
        float Dv[3] = {p.Dx[c], p.Dy[c], p.Dz[c]};
        float* Ep[3] = {p.Ex, p.Ey, p.Ez};
        const int cur = (int)((M.it - 1) & 1);
        const long long bi = (long long)(ix - m->bx0) + (long long)m->bnx * ((tl.iy - m->by0) + (long long)m->bny * (tl.iz - m->bz0));
        switch (m->nq) {
            case 0: material_cell_n<float, double, 3, 0>(m, bi, Ep, c, Dv, cur, p.dt); break;
            case 1: material_cell_n<float, double, 3, 1>(m, bi, Ep, c, Dv, cur, p.dt); break;
            case 2: material_cell_n<float, double, 3, 2>(m, bi, Ep, c, Dv, cur, p.dt); break;
            case 3: material_cell_n<float, double, 3, 3>(m, bi, Ep, c, Dv, cur, p.dt); break;
            default: material_cell<float, double, 3>(m, ix, tl.iy, tl.iz, Ep, c, Dv, cur, p.dt); break;
        }
    }
}

// One pass of point sources: entry i is a point of the k-th source of its member, so a
// member's sources act in tuple order across passes (models.jl:128-130).
__global__ void __launch_bounds__(256) batch_source_kernel(const BMember* __restrict__ mem, const BSrc* __restrict__ srcs,
                                                           const BPoint* __restrict__ pts, const int* __restrict__ npts) {
    const int n = *npts;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const BPoint e = pts[i];
        const BMember& M = mem[e.m];
        if (!b_active(M)) continue;
        const BSrc& S = srcs[e.s];
        const long long it0 = M.it - 1;
        const double w = S.wave ? S.wave[it0 * S.npts + e.i] : S.amp[e.i] * S.gt[it0];
        const long long c = S.cells[e.i];
        if (S.kind == MFD_SRC_SOFT) S.F[c] = (float)((double)S.F[c] + (double)S.coeff * w);
        else S.F[c] = (float)w;
    }
}

// TFSF injection of the members whose TFSF acts in this source pass: grid row = (member,
// statement), as tfsf_kernel.
__global__ void __launch_bounds__(256) batch_tfsf_kernel(const BMember* __restrict__ mem, const BRow* __restrict__ rows) {
    const BRow r = rows[blockIdx.y];
    const BMember& M = mem[r.m];
    if (!b_active(M)) return;
    tfsf_point(*M.rp, r.s, blockIdx.x * blockDim.x + threadIdx.x, M.it - 1);
}

// Monitor gather (monitor_gather_kernel): field monitors without sum to their history,
// the others to the member's staging ring, slot = steps since ring_first.
__global__ void __launch_bounds__(256) batch_gather_kernel(const BMember* __restrict__ mem, const BPoint* __restrict__ pts,
                                                           const int* __restrict__ npts) {
    const int n = *npts;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const BPoint e = pts[i];
        const BMember& M = mem[e.m];
        if (!b_active(M)) continue;
        const MonParams<float>& p = *M.mp;
        const MonDev<float>& D = p.mons[e.s];
        const long long it0 = M.it - 1;
        const int cell = D.cells[e.i];
        if (D.kind == MFD_MON_FIELD && !D.sum) {
            for (int k = 0; k < p.ncomp; ++k) D.hist[((long long)k * p.nt + it0) * D.npts + e.i] = p.comp[k][cell];
        } else {
            const long long slot = it0 - M.ring_first;
            for (int k = 0; k < p.ncomp; ++k) D.ring[(slot * p.ncomp + k) * D.npts + e.i] = p.comp[k][cell];
        }
    }
}

// End of a batch step: every active member moves to its next step.
__global__ void batch_advance_kernel(BMember* __restrict__ mem, int n) {
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x)
        if (mem[m].it <= mem[m].last) mem[m].it += 1;
}

}  // namespace mfd
