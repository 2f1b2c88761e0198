// aux.cuh -- per-step kernels around the Yee updates: point sources, TFSF injection, TFSF
// record, monitors and the DFT accumulation.
#pragma once

#include "mfd_device.cuh"

namespace mfd {

// ------------------------------------------------------------------------------------------
// Soft / hard point sources (sources.jl:77-131, 190-244).  The waveform is tabulated in
// double; the add is done in double and rounded to T as the reference's mixed-type
// expression FC + coeff*waveform(...) is.
// ------------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) point_source_kernel(T* F, const long long* __restrict__ cells, long long npts,
                                                           const double* __restrict__ wave, const double* __restrict__ amp,
                                                           const double* __restrict__ gt, long long it0, int kind, T coeff) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= npts) return;
    const double w = wave ? wave[it0 * npts + i] : amp[i] * gt[it0];
    const long long c = cells[i];
    if (kind == MFD_SRC_SOFT) F[c] = (T)((double)F[c] + (double)coeff * w);
    else F[c] = (T)w;
}

// ------------------------------------------------------------------------------------------
// Rectangle statements: F[comp][rect] op= coef * inc[k][it][local]  (TFSF add_source!,
// sources.jl:320-346, 469-497, 713-776) or rec[k][it][local] = F[comp][rect] (TFSF record,
// sources.jl:372-384, 534-550, 839-877).  Rectangles are 0-based inclusive.
// ------------------------------------------------------------------------------------------
#define MFD_MAX_STMT 36

struct RectStmt {
    int comp;
    int x0, x1, y0, y1, z0, z1;
    int k;            // incident / record array
    int sign;         // +1 add, -1 subtract
    int tprec;        // 1: coefficient and product in T; 0: in double
    double coef;
    double coefT;     // T-rounded coefficient for tprec
    long long len;    // rectangle size
    int shape;        // MFD_INC_* layout of the incident array (TFSF; record arrays are full)
    int na;           // extent of the face's first in-plane axis (a)
    long long clen;   // array values per step: len, len / na, na or 1 by shape
    unsigned long long prev;   // earlier statements of the same component whose rectangle meets this one
    unsigned long long next;   // later ones
};

template <typename T>
struct RectParams {
    int n;
    long long it0;    // 0-based step
    Layout L;
    T* F[9];
    T* arr[24];       // TFSF: incident arrays; record: destination arrays
    RectStmt s[MFD_MAX_STMT];
};

// Offset within a step's incident values of rectangle element `local` = ia + na * ib.
__device__ __forceinline__ long long inc_off(const RectStmt& s, long long local) {
    switch (s.shape) {
        case MFD_INC_ALONG_B: return local / s.na;
        case MFD_INC_ALONG_A: return local % s.na;
        case MFD_INC_UNIFORM: return 0;
        default: return local;
    }
}

__device__ __forceinline__ bool rect_has(const RectStmt& s, int ix, int iy, int iz) {
    return ix >= s.x0 && ix <= s.x1 && iy >= s.y0 && iy <= s.y1 && iz >= s.z0 && iz <= s.z1;
}

__device__ __forceinline__ long long rect_local(const RectStmt& s, int ix, int iy, int iz) {
    const long long nxr = s.x1 - s.x0 + 1, nyr = s.y1 - s.y0 + 1;
    return (ix - s.x0) + nxr * ((iy - s.y0) + nyr * (long long)(iz - s.z0));
}

template <typename T>
__device__ __forceinline__ T tfsf_apply(const RectStmt& t, T v, T inc) {
    if (t.tprec) {
        const T u = (T)t.coefT * inc;
        return t.sign > 0 ? v + u : v - u;
    }
    const double u = t.coef * (double)inc;
    return (T)(t.sign > 0 ? (double)v + u : (double)v - u);
}

// Grid row blockIdx.y = statement.  A cell reached by several statements of the same
// component (edges of the 3-D TFSF box) is updated by the thread of its first statement,
// which applies all of them in statement order -- the order of the reference's broadcasts.
// Point `local` of statement si at step it0 (0-based).
template <typename T>
__device__ __forceinline__ void tfsf_point(const RectParams<T>& p, int si, int local, long long it0) {
    const RectStmt& s = p.s[si];
    if (local >= s.len) return;
    const int nxr = s.x1 - s.x0 + 1, nyr = s.y1 - s.y0 + 1;
    const int rest = local / nxr;
    const int ix = s.x0 + (local - rest * nxr);
    const int iz0 = rest / nyr;
    const int iy = s.y0 + (rest - iz0 * nyr);
    const int iz = s.z0 + iz0;
    for (unsigned long long m = s.prev; m; m &= m - 1)
        if (rect_has(p.s[__ffsll((long long)m) - 1], ix, iy, iz)) return;
    T* F = p.F[s.comp];
    const int c = ix + p.L.px * iy + p.L.sz * iz;
    T v = tfsf_apply(s, F[c], p.arr[s.k][it0 * s.clen + inc_off(s, local)]);
    for (unsigned long long m = s.next; m; m &= m - 1) {
        const RectStmt& t = p.s[__ffsll((long long)m) - 1];
        if (rect_has(t, ix, iy, iz)) v = tfsf_apply(t, v, p.arr[t.k][it0 * t.clen + inc_off(t, rect_local(t, ix, iy, iz))]);
    }
    F[c] = v;
}

template <typename T>
__global__ void __launch_bounds__(256) tfsf_kernel(const __grid_constant__ RectParams<T> p) {
    tfsf_point(p, blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x, p.it0);
}

template <typename T>
__global__ void __launch_bounds__(256) record_kernel(const __grid_constant__ RectParams<T> p) {
    const RectStmt& s = p.s[blockIdx.y];
    const int local = blockIdx.x * blockDim.x + threadIdx.x;
    if (local >= s.len) return;
    const int nxr = s.x1 - s.x0 + 1, nyr = s.y1 - s.y0 + 1;
    const int rest = local / nxr;
    const int ix = s.x0 + (local - rest * nxr);
    const int iz0 = rest / nyr;
    const int iy = s.y0 + (rest - iz0 * nyr);
    const int iz = s.z0 + iz0;
    const int c = ix + p.L.px * iy + p.L.sz * iz;
    p.arr[s.k][p.it0 * s.len + local] = p.F[s.comp][c];
}

// ------------------------------------------------------------------------------------------
// Monitors (monitors.jl, dft.jl).  Every step the gather kernel copies each monitor's point
// values: field monitors without sum go straight to their full history [comp][nt][npts];
// summed field monitors and spectral monitors go to a staging ring [slot][comp][npts] that
// a flush kernel consumes every K steps.
// ------------------------------------------------------------------------------------------
template <typename T>
struct MonDev {
    int kind, sum, nw;
    long long npts;
    const int* cells;         // padded cell indices
    T* hist;                  // field, no sum: [ncomp][nt][npts]; field sum: [ncomp][nt]
    T* ring;                  // staging [K][ncomp][npts]
    double2* S;               // spectral: [ncomp][nw][npts] or [ncomp][nw]
    const double2* phasor;    // [nt][nw]: exp(-i w (t - tshift)) with sum, 2 exp(...) dt without
};

template <typename T>
struct MonParams {
    int nmon, ncomp;
    long long nt;
    const T* comp[6];         // field arrays of the monitored components
    const MonDev<T>* mons;
};

// Grid row blockIdx.y = monitor; a thread gathers every component of one point (one cell
// index load, the component loads independent of each other).
template <typename T>
__global__ void __launch_bounds__(256) monitor_gather_kernel(const __grid_constant__ MonParams<T> p, long long it0, int slot) {
    const MonDev<T>& M = p.mons[blockIdx.y];
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= M.npts) return;
    const int cell = M.cells[j];
    T v[6];
#pragma unroll
    for (int k = 0; k < 6; ++k)
        if (k < p.ncomp) v[k] = p.comp[k][cell];
    const bool hist = M.kind == MFD_MON_FIELD && !M.sum;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        if (k >= p.ncomp) break;
        if (hist) M.hist[((long long)k * p.nt + it0) * M.npts + j] = v[k];
        else M.ring[((long long)slot * p.ncomp + k) * M.npts + j] = v[k];
    }
}

// Summed field monitor: hist[k][it] = sum over points (block reduction in T).
template <typename T>
__global__ void __launch_bounds__(256) monitor_fieldsum_kernel(const MonDev<T>* __restrict__ mon, int ncomp, long long nt,
                                                               long long it0_first) {
    __shared__ T red[256];
    const MonDev<T>& M = *mon;
    const int k = blockIdx.x, slot = blockIdx.y;
    const T* src = M.ring + ((long long)slot * ncomp + k) * M.npts;
    T acc = T(0);
    for (long long j = threadIdx.x; j < M.npts; j += blockDim.x) acc += src[j];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) M.hist[(long long)k * nt + it0_first + slot] = red[0];
}

// Spectral monitor, per point: S[k][w][j] += F * (2 e_w(t) dt) for each staged step in
// order (dft.jl:43-48), every product and sum rounded in double as the reference does.
// The fold is a [points x steps] . [steps x frequencies] product in FP64, bound by the FP64
// pipe once its operands come from shared memory.  A block owns DFT_PT points of one
// component and a tile of up to DFT_WT frequencies: it stages the points' staged values
// for every slot (the ring tile) and the tile's factors for every slot in shared memory
// once, then each thread accumulates DFT_PS points x DFT_W frequencies in registers over
// the slots -- per slot DFT_PS ring loads (consecutive threads, consecutive points) and
// DFT_W factor loads (one address per warp: a broadcast) feed 4 * DFT_PS * DFT_W FP64
// operations.  threadIdx.x picks the points (j, j + 32, ...), threadIdx.y the frequency
// group of DFT_W.
constexpr int MFD_DFT_MAXSLOTS = 64;
constexpr int DFT_W = 4, DFT_PS = 2, DFT_PT = 32 * DFT_PS, DFT_WT = 32;

template <typename T>
__global__ void __launch_bounds__(32 * DFT_WT / DFT_W, 2) monitor_dft_kernel(const MonDev<T>* __restrict__ mon, int ncomp,
                                                                              int nslots, long long it0_first) {
    extern __shared__ __align__(16) unsigned char dft_smem[];
    double2* tw = reinterpret_cast<double2*>(dft_smem);                                  // [slot][w of the tile]
    T* rt = reinterpret_cast<T*>(dft_smem + sizeof(double2) * MFD_DFT_MAXSLOTS * DFT_WT);   // [slot][point of the tile]
    const MonDev<T>& M = *mon;
    const int k = blockIdx.y;
    const int nw = M.nw;
    const int wt0 = blockIdx.z * DFT_WT;
    const int wtn = min(DFT_WT, nw - wt0);
    const long long npts = M.npts;
    const long long p0 = (long long)blockIdx.x * DFT_PT;
    const int tid = threadIdx.x + 32 * threadIdx.y, nth = 32 * blockDim.y;
    for (int i = tid; i < nslots * DFT_WT; i += nth) {
        const int sl = i / DFT_WT, w = i - sl * DFT_WT;
        tw[i] = w < wtn ? M.phasor[(it0_first + sl) * nw + wt0 + w] : make_double2(0.0, 0.0);
    }
    const long long rstride = (long long)ncomp * npts;
    const T* ring = M.ring + (long long)k * npts;
    for (int i = tid; i < nslots * DFT_PT; i += nth) {
        const int sl = i / DFT_PT, q = i - sl * DFT_PT;
        rt[i] = p0 + q < npts ? ring[sl * rstride + p0 + q] : T(0);
    }
    __syncthreads();
    const int w0 = DFT_W * threadIdx.y;          // within the tile
    if (w0 >= wtn) return;
    const int wn = min(DFT_W, wtn - w0);
    double ar[DFT_PS][DFT_W], ai[DFT_PS][DFT_W];
    double2* S = M.S + ((long long)k * nw + wt0 + w0) * npts;
#pragma unroll
    for (int a = 0; a < DFT_PS; ++a) {
        const long long j = p0 + threadIdx.x + 32 * a;
#pragma unroll
        for (int w = 0; w < DFT_W; ++w) {
            ar[a][w] = ai[a][w] = 0.0;
            if (w < wn && j < npts) {
                const double2 v = S[(long long)w * npts + j];
                ar[a][w] = v.x;
                ai[a][w] = v.y;
            }
        }
    }
    for (int sl = 0; sl < nslots; ++sl) {
        double f[DFT_PS];
#pragma unroll
        for (int a = 0; a < DFT_PS; ++a) f[a] = (double)rt[sl * DFT_PT + threadIdx.x + 32 * a];
        const double2* e = tw + sl * DFT_WT + w0;
#pragma unroll
        for (int w = 0; w < DFT_W; ++w) {
            const double2 t = e[w];
#pragma unroll
            for (int a = 0; a < DFT_PS; ++a) {
                ar[a][w] = ar[a][w] + f[a] * t.x;
                ai[a][w] = ai[a][w] + f[a] * t.y;
            }
        }
    }
#pragma unroll
    for (int a = 0; a < DFT_PS; ++a) {
        const long long j = p0 + threadIdx.x + 32 * a;
        if (j >= npts) continue;
#pragma unroll
        for (int w = 0; w < DFT_W; ++w)
            if (w < wn) S[(long long)w * npts + j] = make_double2(ar[a][w], ai[a][w]);
    }
}

// Shared memory of monitor_dft_kernel: the factor tile and the ring tile.
template <typename T>
constexpr size_t dft_smem_bytes() {
    return sizeof(double2) * MFD_DFT_MAXSLOTS * DFT_WT + sizeof(T) * MFD_DFT_MAXSLOTS * DFT_PT;
}

// Spectral monitor with sum: S[k][w] += 2 * sum_j(F_j e_w(t)) * dt (dft.jl:38-41).
template <typename T>
__global__ void __launch_bounds__(256) monitor_dftsum_kernel(const MonDev<T>* __restrict__ mon, int ncomp, int nslots,
                                                             long long it0_first, double dt) {
    __shared__ double rr[256], ri[256];
    const MonDev<T>& M = *mon;
    const int k = blockIdx.x, w = blockIdx.y;
    double2 S = M.S[(long long)k * M.nw + w];
    for (int slot = 0; slot < nslots; ++slot) {
        const double2 e = M.phasor[(it0_first + slot) * M.nw + w];
        const T* src = M.ring + ((long long)slot * ncomp + k) * M.npts;
        double ar = 0, ai = 0;
        for (long long j = threadIdx.x; j < M.npts; j += blockDim.x) {
            const double f = (double)src[j];
            ar += f * e.x;
            ai += f * e.y;
        }
        rr[threadIdx.x] = ar;
        ri[threadIdx.x] = ai;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) { rr[threadIdx.x] += rr[threadIdx.x + s]; ri[threadIdx.x] += ri[threadIdx.x + s]; }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            S.x = S.x + (2 * rr[0]) * dt;
            S.y = S.y + (2 * ri[0]) * dt;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) M.S[(long long)k * M.nw + w] = S;
}

// The per-step DFT factor 2 exp(-i w (t - tshift)) dt of dft.jl:44, from the phasor table.
__global__ void dft_factor_kernel(double2* ph, long long n, double dt) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double2 e = ph[i];
    ph[i] = make_double2((2 * e.x) * dt, (2 * e.y) * dt);
}

// ------------------------------------------------------------------------------------------
// Material state -> dense outputs: JE (T) and rho_end = rho*rho0 (double) (outputs.jl:46-65)
// ------------------------------------------------------------------------------------------
template <typename T, typename R>
__global__ void __launch_bounds__(256) scatter_state_kernel(const MatDev<T, R>* __restrict__ mats, const uint8_t* __restrict__ geom,
                                                            Layout L, void* out, int which) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y, iz = blockIdx.z;
    if (ix >= L.nx) return;
    const long long c = ix + (long long)L.px * iy + L.sz * iz;
    const int g = geom[c];
    const MatDev<T, R>* m = g ? mats + (g - 1) : nullptr;
    const bool pl = m && m->plasma;
    long long bi = 0;
    if (pl) bi = (long long)(ix - m->bx0) + (long long)m->bnx * ((long long)(iy - m->by0) + (long long)m->bny * (iz - m->bz0));
    if (which == MFD_INT_JE) ((T*)out)[c] = pl ? m->JE[bi] : T(0);
    else ((double*)out)[c] = pl ? 0.0 + (double)(m->rho[bi] * m->rho0) : 0.0;
}

// The same values for the z-planes z0 .. z0 + gridDim.z - 1 only, written densely (x fastest,
// then y, then z) from `out`, for the allocation-free read that stages a few planes at a time
// through a fixed device buffer.
template <typename T, typename R>
__global__ void __launch_bounds__(256) scatter_state_planes_kernel(const MatDev<T, R>* __restrict__ mats,
                                                                   const uint8_t* __restrict__ geom, Layout L,
                                                                   void* out, int which, int z0) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y, iz = z0 + (int)blockIdx.z;
    if (ix >= L.nx) return;
    const long long c = ix + (long long)L.px * iy + L.sz * iz;
    const long long o = ix + (long long)L.nx * (iy + (long long)L.ny * blockIdx.z);
    const int g = geom[c];
    const MatDev<T, R>* m = g ? mats + (g - 1) : nullptr;
    const bool pl = m && m->plasma;
    long long bi = 0;
    if (pl) bi = (long long)(ix - m->bx0) + (long long)m->bnx * ((long long)(iy - m->by0) + (long long)m->bny * (iz - m->bz0));
    if (which == MFD_INT_JE) ((T*)out)[o] = pl ? m->JE[bi] : T(0);
    else ((double*)out)[o] = pl ? 0.0 + (double)(m->rho[bi] * m->rho0) : 0.0;
}

}  // namespace mfd
