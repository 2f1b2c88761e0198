// dft_tc.cuh -- the spectral monitors' ring fold on the tensor cores (tcgen05), for Float32
// models in the tolerance mode.
//
// The fold of dft.jl:39-51 over the staged steps of a ring is a complex matrix product per
// monitor component k:
//
//     S[k][w][p] += sum_s ring[s][k][p] * phasor[s][w]          (phasor = 2 e^{-i w t_s} dt)
//
// i.e. D[p][n] = sum_s A[p][s] B[n][s] with A the ring tile (points x slots) and B the
// factor tile (n = 32 frequencies x (re, im), slots).  The exact mode folds it with FP64
// multiplies and adds, unfused (monitor_dft_kernel), one point at a time in the reference's
// order.  Here one CTA takes tiles of 128 points x 32 frequencies:
//
//   * A (Float32 samples) and B (FP64 factors, scaled by a power of two) are split into a
//     TF32 high part and a TF32 low part (x = hi + lo to about 2^-22 relative), staged by
//     the threads in shared memory in the K-major no-swizzle layout of the UMMA descriptor
//     (16-byte rows of 4 slots; 8-row core matrices 128 B apart; slot chunks of all rows
//     next to each other);
//   * one thread issues tcgen05.mma kind::tf32, M = 128, N = 64, K = 8 per instruction:
//     hi*hi + hi*lo + lo*hi for each 8 slots, accumulating in TMEM (64 columns, FP32);
//   * tcgen05.commit arrives on an mbarrier; every warp waits on it (bounded; the first
//     spectra it adds to are loaded meanwhile), reads its 32 TMEM lanes x 32 columns with
//     tcgen05.ld and adds the products, unscaled, to S in FP64.
//
// The fold is bound by S's read-modify-write (16 B per point, component and frequency); the
// products take about a microsecond per tile.  Per fold, the partial sums carry the TF32x3
// product error (about 2^-21 relative) and FP32 accumulation over at most 64 slots, which
// the tolerance mode's bound (relative L2 1e-5 against the FP64 oracle) covers many times.
#pragma once

#include "aux.cuh"

namespace mfd {

constexpr int TC_M = 128;                 // points per tile = TMEM lanes
constexpr int TC_W = 32;                  // frequencies per tile
constexpr int TC_N = 2 * TC_W;            // columns: re of the tile's frequencies, then im
constexpr int TC_K = MFD_DFT_MAXSLOTS;    // slots per fold (64)
constexpr int TC_THREADS = 256;           // 8 warps: two per TMEM lane quarter
constexpr int TC_A_CHUNK = TC_M * 16;     // 4 slots of the 128 point rows
constexpr int TC_B_CHUNK = TC_N * 16;     // 4 slots of the 64 factor rows
constexpr int TC_A_BYTES = TC_K / 4 * TC_A_CHUNK;   // 32 KB
constexpr int TC_B_BYTES = TC_K / 4 * TC_B_CHUNK;   // 16 KB
constexpr size_t dft_tc_smem_bytes = 2 * (size_t)TC_A_BYTES + 2 * (size_t)TC_B_BYTES + 128;   // two blocks per SM
constexpr unsigned TC_WAIT_LIMIT = 1u << 24;    // mbarrier polls before the fold gives up

// Round to TF32 (10 explicit mantissa bits), nearest with ties away from zero.
__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// x = hi + lo, both TF32 values.
__device__ __forceinline__ void tf32_split(float x, float& hi, float& lo) {
    hi = tf32_rna(x);
    lo = tf32_rna(x - hi);   // exact difference: x and hi share the binade
}
__device__ __forceinline__ void tf32_split(double x, float& hi, float& lo) {
    hi = tf32_rna((float)x);
    lo = tf32_rna((float)(x - (double)hi));
}

__device__ __forceinline__ uint32_t tc_saddr(const void* p) {   // shared-window address
    return (uint32_t)__cvta_generic_to_shared(p);
}

// UMMA shared-memory descriptor, K-major, no swizzle: start address, leading byte offset
// (next 16-byte slot chunk along K), stride byte offset (next 8-row core matrix), version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::tf32: D FP32, A and B TF32, both K-major, N = 64, M = 128.
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ void umma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile("{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                 "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n"
                 :: "r"(tmem), "l"(a), "l"(b), "r"(TC_IDESC), "r"(acc));
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.b32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}

// 32 lanes x 16 columns of FP32 from TMEM into 16 registers per thread.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Persistent fold of one spectral monitor (no sum) of a Float32 model.  Block b keeps the
// frequency tile b % nwt (its factor tile staged once) and takes the (component, point tile)
// items b / nwt, b / nwt + G, ... (G = gridDim.x / nwt), so the blocks of one point tile run
// side by side and the second read of its ring values comes from L2.  Two blocks per SM: one
// stages and multiplies while the other adds its products to S.  bscale (a power of two)
// brings the factors near 1 for TF32; S receives D / bscale.  On an mbarrier wait that does
// not end, the block sets *fault, frees its TMEM and returns.
__global__ void __launch_bounds__(TC_THREADS, 2) monitor_dft_tc_kernel(const MonDev<float>* __restrict__ mon, int ncomp,
                                                                       int nslots, long long it0_first, double bscale,
                                                                       int* __restrict__ fault) {
    extern __shared__ __align__(128) unsigned char tc_smem[];
    unsigned char* Ah = tc_smem;
    unsigned char* Al = Ah + TC_A_BYTES;
    unsigned char* Bh = Al + TC_A_BYTES;
    unsigned char* Bl = Bh + TC_B_BYTES;
    uint64_t* bar = reinterpret_cast<uint64_t*>(Bl + TC_B_BYTES);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);

    const MonDev<float>& M = *mon;
    const int nw = M.nw;
    const long long npts = M.npts;
    const int ntile = (int)((npts + TC_M - 1) / TC_M);
    const int nwt = (nw + TC_W - 1) / TC_W;
    const int G = gridDim.x / nwt;                  // blocks per frequency tile
    const int wt = blockIdx.x % nwt, b0 = blockIdx.x / nwt;
    if (b0 >= G) return;                            // a remainder block (none when the grid is a multiple of nwt)
    const long long nitems = (long long)ncomp * ntile;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int kchunks = 2 * ((nslots + 7) / 8);      // 4-slot chunks staged (whole 8-slot MMA steps)
    const long long rstride = (long long)ncomp * npts;
    const double unscale = 1.0 / bscale;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                     :: "r"(tc_saddr(tmem_slot)), "r"(TC_N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" :: "r"(tc_saddr(bar)));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    // Factor tile B[n][slot]: row n = frequency wt*32 + (n & 31), re (n < 32) or im.
    {
        const int n = tid & (TC_N - 1);
        const int w = wt * TC_W + (n & (TC_W - 1));
        const bool im = n >= TC_W;
        for (int c = tid / TC_N; c < TC_K / 4; c += TC_THREADS / TC_N) {
            float hv[4], lv[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int s = 4 * c + j;
                double v = 0.0;
                if (s < nslots && w < nw) {
                    const double2 e = M.phasor[(it0_first + s) * nw + w];
                    v = (im ? e.y : e.x) * bscale;
                }
                tf32_split(v, hv[j], lv[j]);
            }
            *reinterpret_cast<float4*>(Bh + c * TC_B_CHUNK + n * 16) = make_float4(hv[0], hv[1], hv[2], hv[3]);
            *reinterpret_cast<float4*>(Bl + c * TC_B_CHUNK + n * 16) = make_float4(lv[0], lv[1], lv[2], lv[3]);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    const int r = tid & (TC_M - 1);   // staging: row of the tile
    const int c0 = tid / TC_M;        // staging: first chunk (0 or 1), then every second
    uint32_t phase = 0;
    bool failed = false;

    for (long long item = b0; item < nitems && !failed; item += G) {
        const int k = (int)(item / ntile);
        const long long p0 = (item - (long long)k * ntile) * TC_M;

        // Ring tile A[p][slot] of component k: every load of the thread issued, then split.
        {
            const long long p = p0 + r;
            const float* src = M.ring + (long long)k * npts + p;
            float v[TC_K / 8][4];
#pragma unroll
            for (int i = 0; i < TC_K / 8; ++i) {
                const int c = c0 + 2 * i;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int s = 4 * c + j;
                    v[i][j] = (c < kchunks && s < nslots && p < npts) ? src[s * rstride] : 0.f;
                }
            }
#pragma unroll
            for (int i = 0; i < TC_K / 8; ++i) {
                const int c = c0 + 2 * i;
                if (c >= kchunks) break;
                float hv[4], lv[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) tf32_split(v[i][j], hv[j], lv[j]);
                *reinterpret_cast<float4*>(Ah + c * TC_A_CHUNK + r * 16) = make_float4(hv[0], hv[1], hv[2], hv[3]);
                *reinterpret_cast<float4*>(Al + c * TC_A_CHUNK + r * 16) = make_float4(lv[0], lv[1], lv[2], lv[3]);
            }
        }
        // generic-proxy stores -> visible to the tensor core's async proxy
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();

        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t ah = tc_saddr(Ah), al = tc_saddr(Al), bh = tc_saddr(Bh), bl = tc_saddr(Bl);
            for (int ks = 0; ks < kchunks / 2; ++ks) {
                const uint32_t oa = (uint32_t)(2 * ks * TC_A_CHUNK), ob = (uint32_t)(2 * ks * TC_B_CHUNK);
                const uint64_t dah = umma_desc(ah + oa, TC_A_CHUNK, 128), dal = umma_desc(al + oa, TC_A_CHUNK, 128);
                const uint64_t dbh = umma_desc(bh + ob, TC_B_CHUNK, 128), dbl = umma_desc(bl + ob, TC_B_CHUNK, 128);
                umma_tf32(tmem, dah, dbh, ks > 0);
                umma_tf32(tmem, dah, dbl, 1);
                umma_tf32(tmem, dal, dbh, 1);
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                         :: "r"(tc_saddr(bar)) : "memory");
        }
        // The spectra this thread adds to do not depend on the products: its first 8 are
        // loaded while the tensor core works.
        const int q = warp & 3, h = warp >> 2;     // TMEM lane quarter, frequency half
        const long long p = p0 + 32 * q + lane;
        const int wb = wt * TC_W + 16 * h;
        const bool mine = p < npts && wb < nw;
        const int wn = mine ? min(16, nw - wb) : 0;
        double2* S = M.S + ((long long)k * nw + wb) * npts + p;
        double2 v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if (j < wn) v[j] = S[(long long)j * npts];
        // every thread waits for the products (bounded)
        {
            unsigned polls = 0;
            while (!mbar_try(tc_saddr(bar), phase)) {
                if (++polls >= TC_WAIT_LIMIT) { failed = true; break; }
            }
            phase ^= 1u;
        }
        failed = __syncthreads_or(failed);   // one decision for the whole block
        if (failed) {
            if (tid == 0) atomicOr(fault, 1);
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");

        // Epilogue: warp (quarter q, half h) holds lanes 32q.. and frequencies 16h.. of the tile.
        const uint32_t lane_base = (uint32_t)(32 * q) << 16;
        float re[16], imv[16];
        tmem_ld16(tmem + lane_base + (uint32_t)(16 * h), re);
        tmem_ld16(tmem + lane_base + (uint32_t)(TC_W + 16 * h), imv);
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");

        if (mine) {
#pragma unroll
            for (int j0 = 0; j0 < 16; j0 += 8) {
                if (j0) {
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                        if (j0 + j < wn) v[j] = S[(long long)(j0 + j) * npts];
                }
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    if (j0 + j < wn) {
                        v[j].x += (double)re[j0 + j] * unscale;
                        v[j].y += (double)imv[j0 + j] * unscale;
                        S[(long long)(j0 + j) * npts] = v[j];
                    }
            }
        }
        __syncthreads();   // TMEM read by every warp before the next tile's products
    }

    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" :: "r"(tmem), "r"(TC_N));
    }
}

}  // namespace mfd
