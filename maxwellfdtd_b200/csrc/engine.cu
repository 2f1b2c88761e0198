// engine.cu -- the handle behind the C ABI (include/maxwellfdtd.h): device memory, the
// per-step launch sequence and host<->device transfers.
//
// Per step it (reference order, models.jl:125-132 and 199-234):
//   H update  [+ Sa/E2 and NaN/Inf guard of step it-1]        h?d_kernel
//   E update  (CPML, ADE, plasma, Kerr fused)                 e?d_kernel
//   sources in tuple order (point sources, TFSF)             point_source_kernel, tfsf_kernel
//   monitors                                                  monitor_gather_kernel (+ flush)
//   TFSF record                                               record_kernel
// and after the last step of a run: Sa/E2 + guard of that step (sums_kernel).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "aux.cuh"
#include "dft_tc.cuh"
#include "yee.cuh"
#include "yee3d_async.cuh"
#include "yee3d_split.cuh"
#include "batch.cuh"
#include "geometry.cuh"

namespace mfd {

constexpr double EPS0 = 8.8541878128e-12;
constexpr double MU0 = 1.25663706212e-6;

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define MFD_CK(call)                                                                              \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            throw ::mfd::Error(e_ == cudaErrorMemoryAllocation ? MFD_ERR_OOM : MFD_ERR_CUDA,      \
                               std::string(#call) + ": " + cudaGetErrorString(e_));               \
    } while (0)

enum { KC_H = 0, KC_E, KC_SRC, KC_TFSF, KC_MON, KC_DFT, KC_SUMS, KC_MAT, KC_N };

struct HandleBase {
    std::string err;
    virtual ~HandleBase() = default;
    virtual int run(int64_t a, int64_t b) = 0;
    virtual int read_field(int comp, void* dst) = 0;
    virtual int read_geometry(uint8_t* dst) = 0;
    virtual int write_field(int comp, const void* src) = 0;
    virtual int read_integral(int which, void* dst) = 0;
    virtual int read_integral_noalloc(int which, void* dst) = 0;
    virtual int set_snapshots(int ncomp, const int32_t* comps, int64_t nsteps, const int64_t* steps, void* dst) = 0;
    virtual int read_monitor(int m, int comp, void* dst) = 0;
    virtual int read_record(int k, void* dst) = 0;
    virtual int64_t record_size(int k) const = 0;
    virtual void status(int64_t* d, int64_t* b, int32_t* k) const = 0;
    virtual void set_profiling(bool on) = 0;
    virtual int kernel_times(double* ms, int64_t* launches, int n) const = 0;
    virtual double last_run_ms() const = 0;
    virtual int64_t device_bytes() const = 0;
    virtual int64_t state_size() const = 0;
    virtual int read_state(void* dst, int64_t n) = 0;
    virtual int write_state(const void* src, int64_t n) = 0;
};

// Header of a state image (mfd_read_state): the buffers follow in allocation order.
struct StateHeader {
    char magic[8];          // "MFDSTATE"
    uint32_t version, nbuf;
    uint64_t layout;        // hash of the model's dimensions, element sizes and buffer sizes
    int64_t done, bad_step;
    int32_t bad_kind, pad;
};

static double wait_timeout_s() {
    const char* s = std::getenv("MFD_WAIT_TIMEOUT_S");
    double v = s ? std::atof(s) : 0.0;
    return v > 0 ? v : 3600.0;
}

// Bounded wait on a stream: polls instead of blocking so a run that does not finish turns
// into MFD_ERR_TIMEOUT rather than a hung host thread.
static void bounded_sync(cudaStream_t st) {
    auto t0 = std::chrono::steady_clock::now();
    const double limit = wait_timeout_s();
    int spins = 0;
    while (true) {
        cudaError_t e = cudaStreamQuery(st);
        if (e == cudaSuccess) return;
        if (e != cudaErrorNotReady) throw Error(MFD_ERR_CUDA, std::string("stream: ") + cudaGetErrorString(e));
        double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > limit) throw Error(MFD_ERR_TIMEOUT, "device work did not finish within the wait limit");
        if (++spins > 64) std::this_thread::sleep_for(std::chrono::microseconds(spins > 1000 ? 200 : 20));
    }
}

static long long round_up(long long a, long long b) { return (a + b - 1) / b * b; }

// Runs fn(lo, hi) over [0, n) split into contiguous ranges on up to 16 host threads (one
// range, on the calling thread, below min_per_thread items per thread).
template <typename Fn>
static void parallel_ranges(long long n, long long min_per_thread, Fn&& fn) {
    const long long hw = std::max(1u, std::thread::hardware_concurrency());
    const long long nth = std::max(1LL, std::min({16LL, hw, n / std::max(1LL, min_per_thread)}));
    if (nth == 1) {
        fn(0LL, n);
        return;
    }
    std::vector<std::thread> th;
    const long long chunk = (n + nth - 1) / nth;
    for (long long t = 0; t < nth; ++t) {
        const long long lo = t * chunk, hi = std::min(n, lo + chunk);
        if (lo < hi) th.emplace_back([&fn, lo, hi] { fn(lo, hi); });
    }
    for (auto& t : th) t.join();
}

// True when any byte of [p, p + bytes) is not zero.  A float array that holds only +0.0 is
// all zero; one holding -0.0 counts as not zero, which only keeps work that changes nothing.
static bool any_nonzero_bytes(const void* p, size_t bytes) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    std::atomic<bool> found{false};
    parallel_ranges((long long)bytes, 4LL << 20, [&](long long lo, long long hi) {
        constexpr long long BLK = 1 << 16;
        for (long long a = lo; a < hi && !found.load(std::memory_order_relaxed); a += BLK) {
            const long long e = std::min(hi, a + BLK);
            uint64_t acc = 0;
            long long i = a;
            for (; i < e && (i & 7); ++i) acc |= b[i];
            for (; i + 8 <= e; i += 8) {
                uint64_t w;
                std::memcpy(&w, b + i, 8);
                acc |= w;
            }
            for (; i < e; ++i) acc |= b[i];
            if (acc) found.store(true, std::memory_order_relaxed);
        }
    });
    return found.load();
}

// Device memory comes from the device's stream-ordered pool (cudaMallocAsync / cudaFreeAsync
// on the owning stream): creating or destroying a model then never synchronises the whole
// device, so models created and destroyed while others run (a serving loop) do not stall
// them.  The pool keeps freed memory for reuse instead of returning it at each sync.
static void retain_pool(int dev) {
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lock(mu);
    if (std::find(done.begin(), done.end(), dev) != done.end()) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    done.push_back(dev);
}

// Staging buffer of mfd_read_integral_noalloc: a file-scope device array, so reading JE and
// rho_end needs no device allocation at read time.  Shared by every handle on a device.
static __device__ __align__(256) unsigned char g_read_scratch[MFD_NOALLOC_SCRATCH_BYTES];

// Kernels that stage planes in static shared memory ask for the largest shared-memory
// carveout, so that as many blocks as their registers allow are resident per SM.
static void prefer_shared(const void* f) {
    cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
}

// Device address of g_read_scratch on the current device.  Looked up on every call (cheap
// once the module is loaded; the first lookup makes the driver load the module's device
// globals), so an address never outlives the context it belongs to: after the host program
// resets the device, the next call finds the reloaded array.
static void* read_scratch() {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_read_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        throw Error(MFD_ERR_CUDA, std::string("cudaGetSymbolAddress of the read scratch buffer failed: ") + cudaGetErrorString(e));
    }
    return p;
}

// Exhaustive check of the constant-divisor fast path (see DivC in mfd_device.cuh): for every
// significand x of the binade [1, 2) and of the band's lowest and highest binades (the
// values of those binades inside [lo, hi]), the correction step must reproduce IEEE x/d bit
// for bit.  blockIdx.z selects the binade.
__global__ void verify_div_kernel(const float* __restrict__ ds, const float* __restrict__ rs, const float* __restrict__ los,
                                  const float* __restrict__ his, int* fails) {
    const int j = blockIdx.y;
    const float d = ds[j], r = rs[j], lo = los[j], hi = his[j];
    const unsigned eb = blockIdx.z == 0 ? 0x3f800000u
                      : blockIdx.z == 1 ? (__float_as_uint(lo) & 0x7f800000u) : (__float_as_uint(hi) & 0x7f800000u);
    int bad = 0;
    for (unsigned m = blockIdx.x * blockDim.x + threadIdx.x; m < (1u << 23); m += gridDim.x * blockDim.x) {
        const float x = __uint_as_float(eb | m);
        if (x < lo || x > hi) continue;
        const float q0 = __fmul_rn(x, r);
        const float e = __fmaf_rn(-q0, d, x);
        const float q = __fmaf_rn(e, r, q0);
        bad += __float_as_int(q) != __float_as_int(__fdiv_rn(x, d));
    }
    if (bad) atomicAdd(&fails[j], bad);
}

// Divisor descriptors, verified once per process and divisor value.
class DivisorCache {
   public:
    static DivisorCache& get() {
        static DivisorCache c;
        return c;
    }
    // Fills ok for each float divisor; runs the device check for values not seen yet.
    void verify(std::vector<DivC<float>>& dv, cudaStream_t st) {
        std::lock_guard<std::mutex> lk(mu_);
        std::vector<float> todo_d, todo_r, todo_lo, todo_hi;
        for (auto& D : dv) {
            uint32_t key;
            std::memcpy(&key, &D.d, 4);
            if (!known_.count(key) && std::find(todo_d.begin(), todo_d.end(), D.d) == todo_d.end()) {
                todo_d.push_back(D.d);
                todo_r.push_back(D.r);
                todo_lo.push_back(D.lo);
                todo_hi.push_back(D.hi);
            }
        }
        if (!todo_d.empty()) {
            const int n = (int)todo_d.size();
            float *dd = nullptr, *dr = nullptr, *dlo = nullptr, *dhi = nullptr;
            int* df = nullptr;
            MFD_CK(cudaMallocAsync(&dd, n * sizeof(float), st));
            MFD_CK(cudaMallocAsync(&dr, n * sizeof(float), st));
            MFD_CK(cudaMallocAsync(&dlo, n * sizeof(float), st));
            MFD_CK(cudaMallocAsync(&dhi, n * sizeof(float), st));
            MFD_CK(cudaMallocAsync(&df, n * sizeof(int), st));
            MFD_CK(cudaMemcpyAsync(dd, todo_d.data(), n * sizeof(float), cudaMemcpyHostToDevice, st));
            MFD_CK(cudaMemcpyAsync(dr, todo_r.data(), n * sizeof(float), cudaMemcpyHostToDevice, st));
            MFD_CK(cudaMemcpyAsync(dlo, todo_lo.data(), n * sizeof(float), cudaMemcpyHostToDevice, st));
            MFD_CK(cudaMemcpyAsync(dhi, todo_hi.data(), n * sizeof(float), cudaMemcpyHostToDevice, st));
            MFD_CK(cudaMemsetAsync(df, 0, n * sizeof(int), st));
            verify_div_kernel<<<dim3(128, n, 3), 256, 0, st>>>(dd, dr, dlo, dhi, df);
            MFD_CK(cudaGetLastError());
            std::vector<int> fails(n);
            MFD_CK(cudaMemcpyAsync(fails.data(), df, n * sizeof(int), cudaMemcpyDeviceToHost, st));
            cudaFreeAsync(dd, st);
            cudaFreeAsync(dr, st);
            cudaFreeAsync(dlo, st);
            cudaFreeAsync(dhi, st);
            cudaFreeAsync(df, st);
            MFD_CK(cudaStreamSynchronize(st));
            for (int j = 0; j < n; ++j) {
                uint32_t key;
                std::memcpy(&key, &todo_d[j], 4);
                known_[key] = fails[j] == 0;
            }
        }
        for (auto& D : dv) {
            uint32_t key;
            std::memcpy(&key, &D.d, 4);
            D.ok = D.ok && known_[key] ? 1 : 0;
        }
    }

   private:
    std::mutex mu_;
    std::map<uint32_t, bool> known_;
};

// Lowest |x| of the fast path: 2^-100 keeps x - q0 d an exact float (its quantum stays at or
// above the subnormal one) with two binades of margin; the device check covers the band's
// lowest binade as well.
#define MFD_DIV_LO_EXP -100

template <typename T>
static DivC<T> make_div(T d) {
    DivC<T> D{};
    D.d = d;
    D.r = T(1) / d;
    D.ok = 0;
    if (sizeof(T) == 4 && d > T(0) && std::isnormal((double)d)) {
        const double r = (double)D.r;
        D.lo = (T)std::max(std::ldexp(1.0, MFD_DIV_LO_EXP), std::ldexp(1.0, -100) / r);
        D.hi = (T)std::min(std::ldexp(1.0, 100), std::ldexp(1.0, 100) / r);
        D.ok = (D.lo <= T(1) && D.hi >= T(2)) ? 1 : 0;   // the checked binade lies in the band
        const float lo = (float)D.lo, hi = (float)D.hi;
        uint32_t a, b;
        std::memcpy(&a, &lo, 4);
        std::memcpy(&b, &hi, 4);
        D.lob = a;
        D.span = b - a;
    }
    return D;
}

template <typename T, typename R>
class Engine : public HandleBase {
   public:
    int ndim = 0, nx = 0, ny = 0, nz = 0, px = 0, dev = 0;
    bool ey2 = false;           // the second 2-D field set (Hx, Hz, Dy, Ey: MFD_POL_EY)
    long long sz = 0, Np = 0, N = 0;
    int64_t nt = 0;
    T dx{}, dy{}, dz{}, dt{};
    DivC<T> ddx{}, ddy{}, ddz{};
    bool fastdiv = false;        // every divisor passed the device check
    bool recip = false;          // tolerance mode: derivatives by reciprocal multiply, fused multiply-adds
    Div3 d3{};                   // grid constants for the branch-free 3-D division (single precision)
    int bc[6] = {1, 1, 1, 1, 1, 1};
    cudaStream_t st = nullptr;
    std::vector<void*> allocs;
    int64_t bytes = 0;

    T* F[9] = {};
    T* Sa = nullptr;
    T* E2 = nullptr;
    uint8_t* geom = nullptr;
    bool any_geom = false, math_needed = false;
    LayerDev<T> lay[6] = {};
    T Mh0{}, Me0{}, Md10{}, Md20{};
    int nmat = 0;
    T* matMh = nullptr;
    MatDev<T, R>* mats_dev = nullptr;
    std::vector<MatDev<T, R>> mats_host;
    std::vector<int> response_mats;   // present materials whose E comes from material_kernel
    bool any_plasma = false;

    struct Src {
        int kind, comp;
        T coeff;
        long long npts;
        long long* cells;
        double* wave;
        double* amp;
        double* gt;
    };
    std::vector<Src> srcs;
    bool tfsf = false;
    int tfsf_order = 0;
    RectParams<T> tfsf_p{};
    long long tfsf_maxlen = 0, rec_maxlen = 0;
    bool record = false;

    // Field snapshots (mfd_set_snapshots): after each listed step the listed components are
    // copied on the device into one of two staging slots (the compute stream), and from the
    // slot to the caller's host buffer on a copy stream while the steps go on.
    std::vector<int> snap_comps;
    std::vector<int64_t> snap_steps;
    size_t snap_next = 0;
    char* snap_dst = nullptr;
    T* snap_stage = nullptr;            // [2][ncomp][Np]
    int snap_cap = 0;                   // components the staging slots hold
    bool snap_busy[2] = {false, false};
    cudaStream_t st3 = nullptr;
    // The split 3-D updates run their slab and material-row launches on a side stream,
    // concurrently with the core-row launch: within one half-step the launches write
    // disjoint cells and only read the other field (fork / join below).
    bool overlap = true;
    cudaStream_t st_side = nullptr, st_side2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_join2 = nullptr;
    cudaEvent_t ev_snap_ready[2] = {nullptr, nullptr}, ev_snap_free[2] = {nullptr, nullptr};
    RectParams<T> rec_p{};
    int rec_narr = 0;

    // monitors
    int ncomp_mon = 0;
    int mon_comps[6] = {};
    std::vector<MonDev<T>> mons_host;
    MonDev<T>* mons_dev = nullptr;
    MonParams<T> mon_p{};
    int ring_k = 0, ring_used = 0;
    long long mon_maxpts = 0;
    long long ring_first = 0;
    bool need_ring = false;
    bool mon_apart = false;     // no monitor cell is written by a source: gather beside them
    // Tolerance mode, Float32: spectral monitors folded on the tensor cores (dft_tc.cuh)
    bool tc_fold = false;
    int tc_sms = 1;
    double tc_bscale = 1.0;     // power of two bringing the factors 2 e^{-iwt} dt near 1
    int* d_tcfault = nullptr;   // set by a fold whose tensor-core wait ran out
    int h_tcfault = 0;

    int* d_flags = nullptr;     // [nt] per-step NaN/Inf flags of Ex
    int* h_flags = nullptr;     // host copy
    std::vector<int> h_flags_v;

    int64_t done = 0, bad_step = 0;
    int32_t bad_kind = 0;

    // launch shapes
    bool core_async = true;    // single-precision core rows staged by cp.async (MFD_CORE_ASYNC=0: register z-march)
    int async_zc = 8;          // planes per block of the staged core kernels (MFD_ASYNC_ZC)
    int bx3 = 32, by3 = 4, zc3 = 4;   // 3-D z-march tiles: 32x4 columns, 4 planes (best at 100^3, neutral at 256^3)
    // planes per block of the material-row E launch: one (more, shorter-lived blocks beside
    // the staged kernel's; 256^3 plasmonics: E 0.193 ms per update against 0.198 at 4)
    int zc_mat = 1;
    // The y- and z-layer cells of the single-precision split updates go through the staged
    // kernels (LAY 1 / 2) instead of the one-cell-per-thread slab kernels: in the tolerance
    // mode, for the H update (256^3 plasmonics: 43.5 against 42.5 Gcell/s with both updates
    // layered; the exact mode's layer code needs 80 registers and measured slower, 38.0
    // against 40.2).
    bool lay_H = true, lay_E = true;
    // Planes per block of a z-layer launch of n planes: the whole layer in one march up to 16
    // planes, else even chunks of at most 12.  At 256^3 plasmonics (13-plane layers, side
    // streams at the highest priority): 13 gave 44.64-44.65 against 44.31-44.32 for chunks of
    // 12 + 1 (same box); 6 + 6 + 1 gave 44.08-44.10 and 4 43.86 Gcell/s; before the priority
    // streams 6 gave 43.9 and 12 gave 42.2.
    static int zc_layer(int n) {
        if (n <= 16) return std::max(1, n);
        const int chunks = (n + 11) / 12;
        return (n + chunks - 1) / chunks;
    }
    bool mat_in_layers = false;       // some material cell lies in a y or z layer
    // single-precision 3-D updates split into core rows and CPML slabs (yee3d_split.cuh)
    bool use_split = false;
    SplitBox sbox{};
    SplitBox mat_rows{};   // core rows/planes holding material cells, aligned to the staged E tiles
    int mat_x0 = 0, mat_x1 = 0;   // ... and their columns, aligned to the tiles of both E kernels
    int mbox[6] = {0, -1, 0, -1, 0, -1};   // bounding box of the material cells (x0, x1, y0, y1, z0, z1; empty: none)
    long long slab_rows = 0;
    bool resp_fused = false;   // material response inside the E kernel of the core rows (RESP)
    int kcount = 1;             // kernels issued by the current launch() call

    // timing
    bool profiling = false;
    double k_ms[KC_N] = {};
    int64_t k_n[KC_N] = {};
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pend;
    std::vector<cudaEvent_t> ev_pool;
    cudaEvent_t run_ev[2] = {nullptr, nullptr};
    double run_ms = 0;

    ~Engine() override {
        cudaSetDevice(dev);
        if (st3) cudaStreamSynchronize(st3);
        if (st_side) cudaStreamSynchronize(st_side);
        if (st) {
            for (void* p : allocs) cudaFreeAsync(p, st);
            cudaStreamSynchronize(st);
        }
        for (auto e : ev_pool) cudaEventDestroy(e);
        for (auto& pe : pend) { cudaEventDestroy(pe.second.first); cudaEventDestroy(pe.second.second); }
        if (run_ev[0]) cudaEventDestroy(run_ev[0]);
        if (run_ev[1]) cudaEventDestroy(run_ev[1]);
        for (auto e : ev_snap_ready) if (e) cudaEventDestroy(e);
        for (auto e : ev_snap_free) if (e) cudaEventDestroy(e);
        if (st3) cudaStreamDestroy(st3);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (ev_join2) cudaEventDestroy(ev_join2);
        if (st_side2) { cudaStreamSynchronize(st_side2); cudaStreamDestroy(st_side2); }
        if (st_side) cudaStreamDestroy(st_side);
        if (st) cudaStreamDestroy(st);
    }

    // Buffers that the steps change (fields, running sums, psi, material and plasma state,
    // monitor records and accumulators, the record arrays, the per-step flags), in allocation
    // order: the model state that mfd_read_state / mfd_write_state carry.
    std::vector<std::pair<void*, size_t>> state_bufs;

    template <typename U>
    U* dalloc(size_t n, bool state = true) {
        if (n == 0) n = 1;
        void* p = nullptr;
        cudaError_t e = cudaMallocAsync(&p, n * sizeof(U), st);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Error(MFD_ERR_OOM, "device allocation of " + std::to_string(n * sizeof(U)) + " bytes failed: " + cudaGetErrorString(e));
        }
        allocs.push_back(p);
        bytes += (int64_t)(n * sizeof(U));
        MFD_CK(cudaMemsetAsync(p, 0, n * sizeof(U), st));
        if (state) state_bufs.push_back({p, n * sizeof(U)});
        return (U*)p;
    }

    template <typename U>
    U* upload(const U* h, size_t n) {
        U* d = dalloc<U>(n, false);
        if (n) MFD_CK(cudaMemcpyAsync(d, h, n * sizeof(U), cudaMemcpyHostToDevice, st));
        MFD_CK(cudaStreamSynchronize(st));   // the host buffer may be a temporary
        return d;
    }

    template <typename U>
    U* upload_cast(const double* h, size_t n) {
        std::vector<U> tmp(h, h + n);
        return upload(tmp.data(), n);
    }

    long long pad_index(long long c) const {   // dense x-fastest -> padded
        return (c % nx) + (long long)px * (c / nx);
    }

    Layout layout() const { return Layout{nx, ny, nz, px, (int)sz}; }

    void verify_divs(std::vector<DivC<T>>& dv) {
        if (sizeof(T) != 4) return;
        DivisorCache::get().verify(reinterpret_cast<std::vector<DivC<float>>&>(dv), st);
    }

    bool has_comp(int c) const {
        if (ndim == 3) return true;
        if (ey2) return c == MFD_HX || c == MFD_HZ || c == MFD_DY || c == MFD_EY;
        if (ndim == 2) return c == MFD_HY || c == MFD_DX || c == MFD_DZ || c == MFD_EX || c == MFD_EZ;
        return c == MFD_HY || c == MFD_DX || c == MFD_EX;
    }
    // The component the NaN/Inf guard reads: Ex (models.jl:202-209), Ey in the second 2-D
    // field set, which has no Ex.
    int guard_comp() const { return ey2 ? MFD_EY : MFD_EX; }

    // The material map built on the device from the descriptor's shapes (geometry.cuh), and
    // each material's bounding box read back for the compact state.  geom stays allocated
    // only when some cell holds a material.
    void device_geometry(const mfd_desc* d, std::vector<int>& bx0, std::vector<int>& bx1, std::vector<int>& by0,
                         std::vector<int>& by1, std::vector<int>& bz0, std::vector<int>& bz1) {
        if (d->geometry) throw Error(MFD_ERR_INVALID, "give either a geometry array or shapes, not both");
        if (!d->shapes || !d->coords[2] || (ndim >= 2 && !d->coords[0]) || (ndim == 3 && !d->coords[1]))
            throw Error(MFD_ERR_INVALID, "shapes need the shape list and the grid coordinates");
        for (int i = 0; i < d->nshape; ++i) {
            const mfd_shape& sh = d->shapes[i];
            if (sh.kind < MFD_SHAPE_BALL || sh.kind > MFD_SHAPE_ALL) throw Error(MFD_ERR_INVALID, "unknown shape kind");
            if (sh.material < 1 || sh.material > nmat) throw Error(MFD_ERR_INVALID, "shape material beyond nmat");
        }
        mfd_shape* ds = upload(d->shapes, (size_t)d->nshape);
        const double* xs = ndim >= 2 ? upload(d->coords[0], (size_t)nx) : nullptr;
        const double* ys = ndim == 3 ? upload(d->coords[1], (size_t)ny) : nullptr;
        const double* zs = upload(d->coords[2], (size_t)nz);
        geom = dalloc<uint8_t>((size_t)Np, false);
        std::vector<int> box(6 * (size_t)nmat);
        for (int g = 0; g < nmat; ++g)
            for (int k = 0; k < 6; ++k) box[6 * g + k] = (k % 2) ? -1 : INT32_MAX;
        int* dbox = upload(box.data(), box.size());
        const dim3 grd((nx + 255) / 256, ny, nz);
        geometry_kernel<<<grd, 256, 0, st>>>(geom, layout(), ds, d->nshape, xs, ys, zs);
        MFD_CK(cudaGetLastError());
        geometry_box_kernel<<<grd, 256, 0, st>>>(geom, layout(), dbox);
        MFD_CK(cudaGetLastError());
        MFD_CK(cudaMemcpyAsync(box.data(), dbox, box.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
        MFD_CK(cudaStreamSynchronize(st));
        for (int g = 1; g <= nmat; ++g) {
            const int* b = box.data() + 6 * (g - 1);
            bx0[g] = b[0]; bx1[g] = b[1]; by0[g] = b[2]; by1[g] = b[3]; bz0[g] = b[4]; bz1[g] = b[5];
            if (b[1] >= 0) any_geom = true;
        }
    }

    // ---------------------------------------------------------------------------------
    void init(const mfd_desc* d) {
        dev = d->device;
        MFD_CK(cudaSetDevice(dev));
        retain_pool(dev);
        MFD_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        MFD_CK(cudaEventCreate(&run_ev[0]));
        MFD_CK(cudaEventCreate(&run_ev[1]));
        ndim = d->ndim; nx = d->nx; ny = d->ny; nz = d->nz;
        ey2 = ndim == 2 && d->polarization == MFD_POL_EY;
        px = ndim == 1 ? 1 : (int)round_up(nx, 32);
        sz = (long long)px * ny;
        Np = sz * nz;
        N = (long long)nx * ny * nz;
        nt = d->nt;
        dx = (T)d->dx; dy = (T)d->dy; dz = (T)d->dz; dt = (T)d->dt;
        recip = d->mode == MFD_MODE_FAST;
        if (Np >= (1ll << 31)) throw Error(MFD_ERR_INVALID, "grid too large: padded cell count must stay below 2^31");
        {
            std::vector<DivC<T>> dv = {make_div<T>(dx), make_div<T>(dy), make_div<T>(dz)};
            verify_divs(dv);
            ddx = dv[0]; ddy = dv[1]; ddz = dv[2];
            fastdiv = sizeof(T) == 4 && ddx.ok && ddy.ok && ddz.ok;
            if constexpr (sizeof(T) == 4) {   // band common to the three divisors (div6)
                d3.dx = ddx.d; d3.dy = ddy.d; d3.dz = ddz.d;
                d3.rx = ddx.r; d3.ry = ddy.r; d3.rz = ddz.r;
                const unsigned lob = std::max(ddx.lob, std::max(ddy.lob, ddz.lob));
                const unsigned hib = std::min(ddx.lob + ddx.span, std::min(ddy.lob + ddy.span, ddz.lob + ddz.span));
                d3.lob1 = lob - 1u;
                d3.hib = hib;
            }
        }
        for (int f = 0; f < 6; ++f) bc[f] = d->bc[f];
        Mh0 = (T)d->Mh0; Me0 = (T)d->Me0; Md10 = (T)d->Md10; Md20 = (T)d->Md20;
        for (int c = 0; c < 9; ++c)
            if (has_comp(c)) F[c] = dalloc<T>(Np);
        Sa = dalloc<T>(Np);
        // materials
        nmat = d->nmat;
        std::vector<int> bx0(nmat + 1, INT32_MAX), bx1(nmat + 1, -1), by0(nmat + 1, INT32_MAX), by1(nmat + 1, -1),
            bz0(nmat + 1, INT32_MAX), bz1(nmat + 1, -1);
        if (d->geometry) {
            // each material's bounding box, z-planes split over host threads (per-thread
            // boxes merged after); the map goes to its padded device layout in one 2-D copy
            // below, with no host copy
            std::mutex mu;
            bool bad = false;
            parallel_ranges(nz, 4, [&](long long z0, long long z1) {
                std::vector<int> a0(nmat + 1, INT32_MAX), a1(nmat + 1, -1), b0(nmat + 1, INT32_MAX), b1(nmat + 1, -1),
                    c0(nmat + 1, INT32_MAX), c1(nmat + 1, -1);
                bool any = false, over = false;
                for (int iz = (int)z0; iz < (int)z1; ++iz)
                    for (int iy = 0; iy < ny; ++iy) {
                        const uint8_t* row = d->geometry + (size_t)nx * (iy + (size_t)ny * iz);
                        uint8_t orv = 0;
                        for (int ix = 0; ix < nx; ++ix) orv |= row[ix];
                        if (!orv) continue;
                        for (int ix = 0; ix < nx; ++ix) {
                            const int g = row[ix];
                            if (!g) continue;
                            if (g > nmat) { over = true; continue; }
                            any = true;
                            a0[g] = std::min(a0[g], ix); a1[g] = std::max(a1[g], ix);
                            b0[g] = std::min(b0[g], iy); b1[g] = std::max(b1[g], iy);
                            c0[g] = std::min(c0[g], iz); c1[g] = std::max(c1[g], iz);
                        }
                    }
                std::lock_guard<std::mutex> lk(mu);
                bad = bad || over;
                any_geom = any_geom || any;
                for (int g = 1; g <= nmat; ++g) {
                    bx0[g] = std::min(bx0[g], a0[g]); bx1[g] = std::max(bx1[g], a1[g]);
                    by0[g] = std::min(by0[g], b0[g]); by1[g] = std::max(by1[g], b1[g]);
                    bz0[g] = std::min(bz0[g], c0[g]); bz1[g] = std::max(bz1[g], c1[g]);
                }
            });
            if (bad) throw Error(MFD_ERR_INVALID, "geometry index beyond nmat");
        } else if (d->nshape > 0) {
            device_geometry(d, bx0, bx1, by0, by1, bz0, bz1);
        }
        if (d->geometry || d->nshape > 0) {
            for (int g = 1; g <= nmat; ++g) {
                if (bx1[g] < 0) continue;
                const bool first = mbox[1] < mbox[0];
                mbox[0] = first ? bx0[g] : std::min(mbox[0], bx0[g]); mbox[1] = std::max(mbox[1], bx1[g]);
                mbox[2] = first ? by0[g] : std::min(mbox[2], by0[g]); mbox[3] = std::max(mbox[3], by1[g]);
                mbox[4] = first ? bz0[g] : std::min(mbox[4], bz0[g]); mbox[5] = std::max(mbox[5], bz1[g]);
            }
        }
        if (any_geom) {
            if (!geom) {   // the caller's map, rows of nx bytes, into rows of px (the padding stays 0)
                geom = dalloc<uint8_t>((size_t)Np, false);
                MFD_CK(cudaMemcpy2DAsync(geom, (size_t)px, d->geometry, (size_t)nx, (size_t)nx, (size_t)ny * nz,
                                         cudaMemcpyHostToDevice, st));
            }
            E2 = dalloc<T>(Np);
        }
        const int nc = ndim;   // field components per vector quantity
        std::vector<T> mh(std::max(nmat, 1));
        mats_host.resize(nmat);
        for (int m = 0; m < nmat; ++m) {
            const mfd_material& s = d->mats[m];
            MatDev<T, R>& M = mats_host[m];
            std::memset(&M, 0, sizeof(M));
            M.Mh = (T)s.Mh; M.Me = (T)s.Me; M.Md1 = (T)s.Md1; M.Md2 = (T)s.Md2;
            mh[m] = M.Mh;
            if (M.Mh != Mh0) math_needed = true;
            if (s.nq < 0 || s.nq > MFD_MAXQ) throw Error(MFD_ERR_INVALID, "a material has more than 16 ADE poles");
            M.nq = s.nq;
            for (int q = 0; q < s.nq; ++q) { M.Aq[q] = (T)s.Aq[q]; M.Bq[q] = (T)s.Bq[q]; M.Cq[q] = (T)s.Cq[q]; }
            M.kerr = s.kerr ? 1 : 0; M.Mk2 = (T)s.Mk2; M.Mk3 = (T)s.Mk3;
            M.plasma = s.plasma ? 1 : 0;
            M.simple = (M.nq == 0 && !M.plasma && !M.kerr) ? 1 : 0;
            const int g = m + 1;
            const bool present = bx1[g] >= 0;
            if (present && !M.simple) response_mats.push_back(g);
            if (present) {
                M.bx0 = bx0[g]; M.by0 = by0[g]; M.bz0 = bz0[g];
                M.bnx = bx1[g] - bx0[g] + 1; M.bny = by1[g] - by0[g] + 1; M.bnz = bz1[g] - bz0[g] + 1;
                M.bsize = (long long)M.bnx * M.bny * M.bnz;
            }
            if (present && M.nq > 0) M.P = dalloc<T>((size_t)2 * M.nq * nc * M.bsize);
            if (M.plasma) {
                any_plasma = true;
                M.Rava = (T)s.Rava; M.ksi = (T)s.ksi; M.rho0 = (T)s.rho0;
                M.Ap = (T)s.Ap; M.Bp = (T)s.Bp; M.Cp = (T)s.Cp; M.Ma = (T)s.Ma;
                M.rate_kind = s.rate_kind;
                M.rate_order = (T)s.rate_order; M.rate_log10c = s.rate_log10c;
                if (s.rate_kind == MFD_RATE_TABLE) {
                    if (s.rate_n < 2) throw Error(MFD_ERR_INVALID, "rate table needs >= 2 knots");
                    M.rate_n = s.rate_n;
                    M.rate_x = upload_cast<T>(s.rate_x, s.rate_n);
                    M.rate_y = upload_cast<T>(s.rate_y, s.rate_n);
                }
                if (present) {
                    M.Pp = dalloc<T>((size_t)2 * nc * M.bsize);
                    M.Pa = dalloc<T>((size_t)nc * M.bsize);
                    M.rho = dalloc<R>(M.bsize);
                    M.drho = dalloc<R>(M.bsize);
                    M.JE = dalloc<T>(M.bsize);
                }
            }
        }
        if (nmat) {
            matMh = upload(mh.data(), nmat);
            mats_dev = upload(mats_host.data(), nmat);
        }
        // CPML
        for (int f = 0; f < 6; ++f) {
            const mfd_pml_layer& L = d->pml[f];
            lay[f].ib = L.ib; lay[f].nb = L.nb;
            if (L.nb <= 0) { lay[f].nb = 0; continue; }
            const int axis = f / 2;
            const int n = axis == 0 ? nx : axis == 1 ? ny : nz;
            const bool used = ndim == 3 || (ndim == 2 && axis != 1) || (ndim == 1 && axis == 2);
            if (!used) { lay[f].nb = 0; continue; }
            if (L.ib < 1 || L.ib > n) throw Error(MFD_ERR_INVALID, "CPML boundary index out of range");
            const bool left = (f % 2) == 0;
            if (left ? (L.nb != L.ib) : (L.nb != n - L.ib + 1)) throw Error(MFD_ERR_INVALID, "CPML layer size does not match its boundary index");
            {
                std::vector<DivC<T>> kv;
                for (int i = 0; i < L.nb; ++i) kv.push_back(make_div<T>((T)L.K[i]));
                verify_divs(kv);
                for (auto& D : kv) fastdiv = fastdiv && D.ok;
                lay[f].K = upload(kv.data(), kv.size());
            }
            lay[f].A = upload_cast<T>(L.A, L.nb);
            lay[f].B = upload_cast<T>(L.B, L.nb);
            long long cnt;
            if (ndim == 3) cnt = axis == 0 ? (long long)L.nb * ny * nz : axis == 1 ? (long long)px * L.nb * nz : (long long)px * ny * L.nb;
            else if (ndim == 2) cnt = axis == 0 ? (long long)L.nb * nz : (long long)px * L.nb;
            else cnt = L.nb;
            const int npsi = ndim == 3 ? 4 : 2;
            for (int k = 0; k < npsi; ++k) lay[f].psi[k] = dalloc<T>(cnt);
        }
        // sources
        for (int i = 0; i < d->nsrc; ++i) {
            const mfd_source& s = d->srcs[i];
            if (s.comp < 0 || s.comp > 8 || !has_comp(s.comp)) throw Error(MFD_ERR_INVALID, "source component not in this field");
            if (s.npts < 1) throw Error(MFD_ERR_INVALID, "source without points");
            Src S{};
            S.kind = s.kind; S.comp = s.comp; S.coeff = (T)s.coeff; S.npts = s.npts;
            std::vector<long long> cells(s.npts);
            for (long long j = 0; j < s.npts; ++j) {
                if (s.cells[j] < 0 || s.cells[j] >= N) throw Error(MFD_ERR_INVALID, "source cell out of range");
                cells[j] = pad_index(s.cells[j]);
            }
            S.cells = upload(cells.data(), cells.size());
            if (s.wave) S.wave = upload(s.wave, (size_t)nt * s.npts);
            else {
                if (!s.amp || !s.gt) throw Error(MFD_ERR_INVALID, "source needs wave or amp+gt");
                S.amp = upload(s.amp, s.npts);
                S.gt = upload(s.gt, nt);
            }
            srcs.push_back(S);
        }
        if (d->tfsf.enabled) init_tfsf(d);
        if (d->tfsf_record) init_record(d);
        init_monitors(d);
        d_flags = dalloc<int>((size_t)nt);
        h_flags_v.assign((size_t)nt, 0);
        h_flags = h_flags_v.data();
        MFD_CK(cudaStreamSynchronize(st));
        init_split();
        mon_apart = overlap && monitors_apart_from_sources(d);
        if (mon_apart) make_side_stream();
    }

    void make_side_stream() {
        if (st_side) return;
        // The side streams take the device's highest priority: the block scheduler then
        // places the slab, layer and material-row blocks ahead of the core-row launch's,
        // whose many short blocks fill the SMs behind them (256^3 plasmonics: 44.4-44.5
        // against 43.8 Gcell/s at the default priority, 43.4 with the core rows' stream
        // first).
        int pr_least = 0, pr_greatest = 0;
        MFD_CK(cudaDeviceGetStreamPriorityRange(&pr_least, &pr_greatest));
        MFD_CK(cudaStreamCreateWithPriority(&st_side, cudaStreamNonBlocking, pr_greatest));
        MFD_CK(cudaStreamCreateWithPriority(&st_side2, cudaStreamNonBlocking, pr_greatest));
        MFD_CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        MFD_CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        MFD_CK(cudaEventCreateWithFlags(&ev_join2, cudaEventDisableTiming));
    }

    // The split needs layers that do not overlap in any dimension; MFD_KERNEL3D=unsplit
    // keeps the single-kernel updates (for comparison).
    void init_split() {
        if (ndim != 3) return;
        if (const char* k = std::getenv("MFD_KERNEL3D"))
            if (!std::strcmp(k, "unsplit")) return;
        const int xl = lay[MFD_XL].nb ? lay[MFD_XL].ib : 0, xr = lay[MFD_XR].nb ? lay[MFD_XR].ib - 1 : nx;
        int yl = lay[MFD_YL].nb ? lay[MFD_YL].ib : 0, yr = lay[MFD_YR].nb ? lay[MFD_YR].ib - 1 : ny;
        const int zl = lay[MFD_ZL].nb ? lay[MFD_ZL].ib : 0, zr = lay[MFD_ZR].nb ? lay[MFD_ZR].ib - 1 : nz;
        if (xl > xr || yl > yr || zl > zr) return;
        if (const char* a = std::getenv("MFD_CORE_ASYNC")) core_async = std::atoi(a) != 0;
        if (const char* z = std::getenv("MFD_ASYNC_ZC")) async_zc = std::max(1, std::atoi(z));
        // In the tolerance mode the y layers' rows go through the staged kernel in tiles of
        // AS_TY rows.  Each y-layer launch is widened to whole tiles: the rows it gains are
        // core rows, which that kernel updates as the core launch would (no y face there), so
        // no layer tile runs with idle rows and the core box starts on a tile (256^3
        // plasmonics: 13-row layers become 16-row launches, the core 224 rows; 44.77-44.82
        // against 44.59-44.63 Gcell/s on one box).  The exact mode keeps the layer bounds:
        // its slab kernels update the rows outside the core box one cell per thread.
        if (sizeof(T) == 4 && recip && core_async) {
            const int yl_a = (yl + AS_TY - 1) / AS_TY * AS_TY;
            const int yr_a = ny - (ny - yr + AS_TY - 1) / AS_TY * AS_TY;
            if (yl_a < yr_a) { yl = yl_a; yr = yr_a; }
        }
        sbox = SplitBox{yl, yr, zl, zr, zc3, (zl + nz - zr) * ny};
        slab_rows = (long long)sbox.nzr + (long long)(zr - zl) * (yl + ny - yr);
        use_split = true;
        if (overlap) make_side_stream();
        // rows and planes of the core box that hold material cells, widened to the staged
        // E kernel's tiles (AS_TY rows, async_zc planes from the core box's corner)
        // The material response runs inside the core-row E kernel that covers the materials'
        // rows when every dispersive, Kerr or plasma material lies in the core rows (none in
        // a y or z layer, where the slab kernel updates the cells).
        resp_fused = !response_mats.empty();
        for (int g : response_mats) {
            const MatDev<T, R>& m = mats_host[g - 1];
            if (m.by0 < yl || m.by0 + m.bny > yr || m.bz0 < zl || m.bz0 + m.bnz > zr) resp_fused = false;
        }
        mat_rows = SplitBox{0, 0, 0, 0, async_zc, 0};
        mat_in_layers = mbox[1] >= mbox[0] && (mbox[2] < yl || mbox[3] >= yr || mbox[4] < zl || mbox[5] >= zr);
        if (mbox[1] >= mbox[0]) {
            const int y0 = std::max(mbox[2], yl), y1 = std::min(mbox[3] + 1, yr);
            const int z0 = std::max(mbox[4], zl), z1 = std::min(mbox[5] + 1, zr);
            if (y0 < y1 && z0 < z1) {
                mat_rows.yl = yl + (y0 - yl) / AS_TY * AS_TY;
                mat_rows.yr = std::min(yr, yl + (y1 - yl + AS_TY - 1) / AS_TY * AS_TY);
                mat_rows.zl = zl + (z0 - zl) / async_zc * async_zc;
                mat_rows.zr = std::min(zr, zl + (z1 - zl + async_zc - 1) / async_zc * async_zc);
                mat_x0 = mbox[0] / bx3 * bx3;
                mat_x1 = std::min(nx, (mbox[1] + bx3) / bx3 * bx3);
            }
        }

    }

    // Statement lists: sources.jl:727-773 (3-D), 477-495 (2-D), 326-334 (1-D).
    struct S6 { int comp, x0, x1, y0, y1, z0, z1, k, sign, kind; };   // kind 0: dt/MU0-type, 1: dt/EPS0-type, 2: D
    void init_tfsf(const mfd_desc* d) {
        tfsf = true;
        tfsf_order = d->tfsf.order;
        const int* i1 = d->tfsf.i1;
        const int* i2 = d->tfsf.i2;
        for (int a = 0; a < 3; ++a) {
            const bool used = ndim == 3 || (ndim == 2 && a != 1) || (ndim == 1 && a == 2);
            const int n = a == 0 ? nx : a == 1 ? ny : nz;
            if (used && (i1[a] < 2 || i2[a] > n || i1[a] >= i2[a]))
                throw Error(MFD_ERR_INVALID, "TFSF box must satisfy 2 <= i1 < i2 <= n on every axis");
        }
        // 0-based box
        const int X1 = i1[0] - 1, X2 = i2[0] - 1, Y1 = i1[1] - 1, Y2 = i2[1] - 1, Z1 = i1[2] - 1, Z2 = i2[2] - 1;
        std::vector<S6> v;
        const double Cm = (double)dt / MU0, Ce = (double)dt / EPS0;
        std::vector<double> coef;
        std::vector<int> tp;
        std::vector<T> coefT;
        auto add = [&](int comp, int x0, int x1, int y0, int y1, int z0, int z1, int k, int sign, double c, int tprec, T cT) {
            v.push_back(S6{comp, x0, x1, y0, y1, z0, z1, k, sign, 0});
            coef.push_back(c); tp.push_back(tprec); coefT.push_back(cT);
        };
        if (ndim == 3) {
            const double cmx = Cm / (double)dx, cmy = Cm / (double)dy, cmz = Cm / (double)dz;
            const double cex = Ce / (double)dx, cey = Ce / (double)dy, cez = Ce / (double)dz;
            const double cdx = EPS0 * Ce / (double)dx, cdy = EPS0 * Ce / (double)dy, cdz = EPS0 * Ce / (double)dz;
            // 1yz
            add(MFD_HY, X1 - 1, X1 - 1, Y1, Y2, Z1, Z2 - 1, 3, -1, cmx, 0, 0);
            add(MFD_HZ, X1 - 1, X1 - 1, Y1, Y2 - 1, Z1, Z2, 2, +1, cmx, 0, 0);
            add(MFD_EY, X1, X1, Y1, Y2 - 1, Z1, Z2, 1, +1, cex, 0, 0);
            add(MFD_EZ, X1, X1, Y1, Y2, Z1, Z2 - 1, 0, -1, cex, 0, 0);
            add(MFD_DY, X1, X1, Y1, Y2 - 1, Z1, Z2, 1, +1, cdx, 0, 0);
            add(MFD_DZ, X1, X1, Y1, Y2, Z1, Z2 - 1, 0, -1, cdx, 0, 0);
            // 2yz
            add(MFD_HY, X2, X2, Y1, Y2, Z1, Z2 - 1, 7, +1, cmx, 0, 0);
            add(MFD_HZ, X2, X2, Y1, Y2 - 1, Z1, Z2, 6, -1, cmx, 0, 0);
            add(MFD_EY, X2, X2, Y1, Y2 - 1, Z1, Z2, 5, -1, cex, 0, 0);
            add(MFD_EZ, X2, X2, Y1, Y2, Z1, Z2 - 1, 4, +1, cex, 0, 0);
            add(MFD_DY, X2, X2, Y1, Y2 - 1, Z1, Z2, 5, -1, cdx, 0, 0);
            add(MFD_DZ, X2, X2, Y1, Y2, Z1, Z2 - 1, 4, +1, cdx, 0, 0);
            // x1z
            add(MFD_HX, X1, X2, Y1 - 1, Y1 - 1, Z1, Z2 - 1, 11, +1, cmy, 0, 0);
            add(MFD_HZ, X1, X2 - 1, Y1 - 1, Y1 - 1, Z1, Z2, 10, -1, cmy, 0, 0);
            add(MFD_EX, X1, X2 - 1, Y1, Y1, Z1, Z2, 9, -1, cey, 0, 0);
            add(MFD_EZ, X1, X2, Y1, Y1, Z1, Z2 - 1, 8, +1, cey, 0, 0);
            add(MFD_DX, X1, X2 - 1, Y1, Y1, Z1, Z2, 9, -1, cdy, 0, 0);
            add(MFD_DZ, X1, X2, Y1, Y1, Z1, Z2 - 1, 8, +1, cdy, 0, 0);
            // x2z
            add(MFD_HX, X1, X2, Y2, Y2, Z1, Z2 - 1, 15, -1, cmy, 0, 0);
            add(MFD_HZ, X1, X2 - 1, Y2, Y2, Z1, Z2, 14, +1, cmy, 0, 0);
            add(MFD_EX, X1, X2 - 1, Y2, Y2, Z1, Z2, 13, +1, cey, 0, 0);
            add(MFD_EZ, X1, X2, Y2, Y2, Z1, Z2 - 1, 12, -1, cey, 0, 0);
            add(MFD_DX, X1, X2 - 1, Y2, Y2, Z1, Z2, 13, +1, cdy, 0, 0);
            add(MFD_DZ, X1, X2, Y2, Y2, Z1, Z2 - 1, 12, -1, cdy, 0, 0);
            // xy1
            add(MFD_HX, X1, X2, Y1, Y2 - 1, Z1 - 1, Z1 - 1, 19, -1, cmz, 0, 0);
            add(MFD_HY, X1, X2 - 1, Y1, Y2, Z1 - 1, Z1 - 1, 18, +1, cmz, 0, 0);
            add(MFD_EX, X1, X2 - 1, Y1, Y2, Z1, Z1, 17, +1, cez, 0, 0);
            add(MFD_EY, X1, X2, Y1, Y2 - 1, Z1, Z1, 16, -1, cez, 0, 0);
            add(MFD_DX, X1, X2 - 1, Y1, Y2, Z1, Z1, 17, +1, cdz, 0, 0);
            add(MFD_DY, X1, X2, Y1, Y2 - 1, Z1, Z1, 16, -1, cdz, 0, 0);
            // xy2
            add(MFD_HX, X1, X2, Y1, Y2 - 1, Z2, Z2, 23, +1, cmz, 0, 0);
            add(MFD_HY, X1, X2 - 1, Y1, Y2, Z2, Z2, 22, -1, cmz, 0, 0);
            add(MFD_EX, X1, X2 - 1, Y1, Y2, Z2, Z2, 21, -1, cez, 0, 0);
            add(MFD_EY, X1, X2, Y1, Y2 - 1, Z2, Z2, 20, +1, cez, 0, 0);
            add(MFD_DX, X1, X2 - 1, Y1, Y2, Z2, Z2, 21, -1, cdz, 0, 0);
            add(MFD_DY, X1, X2, Y1, Y2 - 1, Z2, Z2, 20, +1, cdz, 0, 0);
        } else if (ey2) {
            // the 3-D faces 1yz, 2yz, xy1, xy2 restricted to Hz, Ey / Hx, Ey (sources.jl:728-776),
            // with the 2-D coefficients (sources.jl:478-495)
            const double cmx = (double)dt / (MU0 * (double)dx), cex = (double)dt / (EPS0 * (double)dx);
            const double cmz = (double)dt / (MU0 * (double)dz), cez = (double)dt / (EPS0 * (double)dz);
            const T cdx = dt / dx, cdz = dt / dz;
            add(MFD_HZ, X1 - 1, X1 - 1, 0, 0, Z1, Z2, 1, +1, cmx, 0, 0);
            add(MFD_EY, X1, X1, 0, 0, Z1, Z2, 0, +1, cex, 0, 0);
            add(MFD_DY, X1, X1, 0, 0, Z1, Z2, 0, +1, 0, 1, cdx);
            add(MFD_HZ, X2, X2, 0, 0, Z1, Z2, 3, -1, cmx, 0, 0);
            add(MFD_EY, X2, X2, 0, 0, Z1, Z2, 2, -1, cex, 0, 0);
            add(MFD_DY, X2, X2, 0, 0, Z1, Z2, 2, -1, 0, 1, cdx);
            add(MFD_HX, X1, X2, 0, 0, Z1 - 1, Z1 - 1, 5, -1, cmz, 0, 0);
            add(MFD_EY, X1, X2, 0, 0, Z1, Z1, 4, -1, cez, 0, 0);
            add(MFD_DY, X1, X2, 0, 0, Z1, Z1, 4, -1, 0, 1, cdz);
            add(MFD_HX, X1, X2, 0, 0, Z2, Z2, 7, +1, cmz, 0, 0);
            add(MFD_EY, X1, X2, 0, 0, Z2, Z2, 6, +1, cez, 0, 0);
            add(MFD_DY, X1, X2, 0, 0, Z2, Z2, 6, +1, 0, 1, cdz);
        } else if (ndim == 2) {
            const double cmx = (double)dt / (MU0 * (double)dx), cex = (double)dt / (EPS0 * (double)dx);
            const double cmz = (double)dt / (MU0 * (double)dz), cez = (double)dt / (EPS0 * (double)dz);
            const T cdx = dt / dx, cdz = dt / dz;
            add(MFD_HY, X1 - 1, X1 - 1, 0, 0, Z1, Z2 - 1, 1, -1, cmx, 0, 0);
            add(MFD_EZ, X1, X1, 0, 0, Z1, Z2 - 1, 0, -1, cex, 0, 0);
            add(MFD_DZ, X1, X1, 0, 0, Z1, Z2 - 1, 0, -1, 0, 1, cdx);
            add(MFD_HY, X2, X2, 0, 0, Z1, Z2 - 1, 3, +1, cmx, 0, 0);
            add(MFD_EZ, X2, X2, 0, 0, Z1, Z2 - 1, 2, +1, cex, 0, 0);
            add(MFD_DZ, X2, X2, 0, 0, Z1, Z2 - 1, 2, +1, 0, 1, cdx);
            add(MFD_HY, X1, X2 - 1, 0, 0, Z1 - 1, Z1 - 1, 5, +1, cmz, 0, 0);
            add(MFD_EX, X1, X2 - 1, 0, 0, Z1, Z1, 4, +1, cez, 0, 0);
            add(MFD_DX, X1, X2 - 1, 0, 0, Z1, Z1, 4, +1, 0, 1, cdz);
            add(MFD_HY, X1, X2 - 1, 0, 0, Z2, Z2, 7, -1, cmz, 0, 0);
            add(MFD_EX, X1, X2 - 1, 0, 0, Z2, Z2, 6, -1, cez, 0, 0);
            add(MFD_DX, X1, X2 - 1, 0, 0, Z2, Z2, 6, -1, 0, 1, cdz);
        } else {
            const double cm = (double)dt / (MU0 * (double)dz), ce = (double)dt / (EPS0 * (double)dz);
            const T cd = dt / dz;
            add(MFD_HY, 0, 0, 0, 0, Z1 - 1, Z1 - 1, 1, +1, cm, 0, 0);
            add(MFD_EX, 0, 0, 0, 0, Z1, Z1, 0, +1, ce, 0, 0);
            add(MFD_DX, 0, 0, 0, 0, Z1, Z1, 0, +1, 0, 1, cd);
            add(MFD_HY, 0, 0, 0, 0, Z2, Z2, 3, -1, cm, 0, 0);
            add(MFD_EX, 0, 0, 0, 0, Z2, Z2, 2, -1, ce, 0, 0);
            add(MFD_DX, 0, 0, 0, 0, Z2, Z2, 2, -1, 0, 1, cd);
        }
        // An incident array that is zero at every step changes nothing (F +- c*0 == F up to
        // the sign of a zero): its statements are dropped and the array is not uploaded.
        const int narr = ndim == 3 ? 24 : ndim == 2 ? 8 : 4;
        // per array: face size, extent of the face's first in-plane axis, values per step
        std::vector<long long> alen(24, -1), clen(24, -1);
        std::vector<int> ana(24, 1);
        for (size_t i = 0; i < v.size(); ++i) {
            const S6& q = v[i];
            const int ex = q.x1 - q.x0 + 1, ey = q.y1 - q.y0 + 1, ez = q.z1 - q.z0 + 1;
            alen[q.k] = (long long)ex * ey * ez;
            // a: y on the x faces (arrays 0-7), x on the y and z faces; a 2-D face is a line
            // (its only axis is a), a 1-D face a point
            ana[q.k] = ndim == 3 ? (q.k < 8 ? ey : ex) : ndim == 2 ? ex * ez : 1;
        }
        std::vector<bool> nonzero(24, false);
        for (int k = 0; k < narr; ++k) {
            if (!d->tfsf.inc[k]) throw Error(MFD_ERR_INVALID, "missing TFSF incident array");
            const int sh = d->tfsf.shape[k];
            if (sh < MFD_INC_FULL || sh > MFD_INC_UNIFORM) throw Error(MFD_ERR_INVALID, "bad TFSF incident-array shape");
            clen[k] = sh == MFD_INC_FULL ? alen[k] : sh == MFD_INC_ALONG_B ? alen[k] / ana[k] : sh == MFD_INC_ALONG_A ? ana[k] : 1;
            nonzero[k] = any_nonzero_bytes(d->tfsf.inc[k], (size_t)clen[k] * nt * sizeof(T));
        }
        RectParams<T>& p = tfsf_p;
        std::memset(&p, 0, sizeof(p));
        p.L = layout();
        for (int c = 0; c < 9; ++c) p.F[c] = F[c];
        int n = 0;
        for (size_t i = 0; i < v.size(); ++i) {
            if (!nonzero[v[i].k]) continue;
            RectStmt& s = p.s[n++];
            s.comp = v[i].comp; s.x0 = v[i].x0; s.x1 = v[i].x1; s.y0 = v[i].y0; s.y1 = v[i].y1; s.z0 = v[i].z0; s.z1 = v[i].z1;
            s.k = v[i].k; s.sign = v[i].sign; s.tprec = tp[i]; s.coef = coef[i]; s.coefT = (double)coefT[i];
            s.len = alen[s.k];
            s.shape = d->tfsf.shape[s.k];
            s.na = ana[s.k];
            s.clen = clen[s.k];
        }
        p.n = n;
        auto meets = [](const RectStmt& a, const RectStmt& b) {
            return a.comp == b.comp && a.x0 <= b.x1 && b.x0 <= a.x1 && a.y0 <= b.y1 && b.y0 <= a.y1 && a.z0 <= b.z1 && b.z0 <= a.z1;
        };
        tfsf_maxlen = 0;
        for (int i = 0; i < n; ++i) {
            p.s[i].prev = p.s[i].next = 0;
            for (int j = 0; j < n; ++j) {
                if (j == i || !meets(p.s[i], p.s[j])) continue;
                if (j < i) p.s[i].prev |= 1ull << j; else p.s[i].next |= 1ull << j;
            }
            tfsf_maxlen = std::max(tfsf_maxlen, p.s[i].len);
            if (p.s[i].len >= (1ll << 31)) throw Error(MFD_ERR_INVALID, "TFSF face larger than 2^31 cells");
        }
        for (int k = 0; k < narr; ++k)
            if (nonzero[k]) p.arr[k] = upload((const T*)d->tfsf.inc[k], (size_t)clen[k] * nt);
        tfsf = n > 0;
        MFD_CK(cudaStreamSynchronize(st));
    }

    // Record statements: sources.jl:372-384, 534-550, 839-877.
    void init_record(const mfd_desc* d) {
        record = true;
        const int* i1 = d->rec_i1;
        const int* i2 = d->rec_i2;
        for (int a = 0; a < 3; ++a) {
            const bool used = ndim == 3 || (ndim == 2 && a != 1) || (ndim == 1 && a == 2);
            const int n = a == 0 ? nx : a == 1 ? ny : nz;
            if (used && (i1[a] < 2 || i2[a] > n || i1[a] >= i2[a]))
                throw Error(MFD_ERR_INVALID, "record box must satisfy 2 <= i1 < i2 <= n on every axis");
        }
        const int X1 = i1[0] - 1, X2 = i2[0] - 1, Y1 = i1[1] - 1, Y2 = i2[1] - 1, Z1 = i1[2] - 1, Z2 = i2[2] - 1;
        std::vector<S6> v;
        auto add = [&](int comp, int x0, int x1, int y0, int y1, int z0, int z1) {
            v.push_back(S6{comp, x0, x1, y0, y1, z0, z1, (int)v.size(), 0, 0});
        };
        if (ndim == 3) {
            add(MFD_HY, X1 - 1, X1 - 1, Y1, Y2, Z1, Z2 - 1); add(MFD_HZ, X1 - 1, X1 - 1, Y1, Y2 - 1, Z1, Z2);
            add(MFD_EY, X1, X1, Y1, Y2 - 1, Z1, Z2); add(MFD_EZ, X1, X1, Y1, Y2, Z1, Z2 - 1);
            add(MFD_HY, X2, X2, Y1, Y2, Z1, Z2 - 1); add(MFD_HZ, X2, X2, Y1, Y2 - 1, Z1, Z2);
            add(MFD_EY, X2, X2, Y1, Y2 - 1, Z1, Z2); add(MFD_EZ, X2, X2, Y1, Y2, Z1, Z2 - 1);
            add(MFD_HX, X1, X2, Y1 - 1, Y1 - 1, Z1, Z2 - 1); add(MFD_HZ, X1, X2 - 1, Y1 - 1, Y1 - 1, Z1, Z2);
            add(MFD_EX, X1, X2 - 1, Y1, Y1, Z1, Z2); add(MFD_EZ, X1, X2, Y1, Y1, Z1, Z2 - 1);
            add(MFD_HX, X1, X2, Y2, Y2, Z1, Z2 - 1); add(MFD_HZ, X1, X2 - 1, Y2, Y2, Z1, Z2);
            add(MFD_EX, X1, X2 - 1, Y2, Y2, Z1, Z2); add(MFD_EZ, X1, X2, Y2, Y2, Z1, Z2 - 1);
            add(MFD_HX, X1, X2, Y1, Y2 - 1, Z1 - 1, Z1 - 1); add(MFD_HY, X1, X2 - 1, Y1, Y2, Z1 - 1, Z1 - 1);
            add(MFD_EX, X1, X2 - 1, Y1, Y2, Z1, Z1); add(MFD_EY, X1, X2, Y1, Y2 - 1, Z1, Z1);
            add(MFD_HX, X1, X2, Y1, Y2 - 1, Z2, Z2); add(MFD_HY, X1, X2 - 1, Y1, Y2, Z2, Z2);
            add(MFD_EX, X1, X2 - 1, Y1, Y2, Z2, Z2); add(MFD_EY, X1, X2, Y1, Y2 - 1, Z2, Z2);
        } else if (ey2) {
            add(MFD_HZ, X1 - 1, X1 - 1, 0, 0, Z1, Z2); add(MFD_EY, X1, X1, 0, 0, Z1, Z2);
            add(MFD_HZ, X2, X2, 0, 0, Z1, Z2); add(MFD_EY, X2, X2, 0, 0, Z1, Z2);
            add(MFD_HX, X1, X2, 0, 0, Z1 - 1, Z1 - 1); add(MFD_EY, X1, X2, 0, 0, Z1, Z1);
            add(MFD_HX, X1, X2, 0, 0, Z2, Z2); add(MFD_EY, X1, X2, 0, 0, Z2, Z2);
        } else if (ndim == 2) {
            add(MFD_HY, X1 - 1, X1 - 1, 0, 0, Z1, Z2 - 1); add(MFD_EZ, X1, X1, 0, 0, Z1, Z2 - 1);
            add(MFD_HY, X2, X2, 0, 0, Z1, Z2 - 1); add(MFD_EZ, X2, X2, 0, 0, Z1, Z2 - 1);
            add(MFD_HY, X1, X2 - 1, 0, 0, Z1 - 1, Z1 - 1); add(MFD_EX, X1, X2 - 1, 0, 0, Z1, Z1);
            add(MFD_HY, X1, X2 - 1, 0, 0, Z2, Z2); add(MFD_EX, X1, X2 - 1, 0, 0, Z2, Z2);
        } else {
            add(MFD_HY, 0, 0, 0, 0, Z1 - 1, Z1 - 1); add(MFD_EX, 0, 0, 0, 0, Z1, Z1);
            add(MFD_HY, 0, 0, 0, 0, Z2, Z2); add(MFD_EX, 0, 0, 0, 0, Z2, Z2);
        }
        RectParams<T>& p = rec_p;
        std::memset(&p, 0, sizeof(p));
        p.n = (int)v.size();
        rec_narr = p.n;
        p.L = layout();
        for (int c = 0; c < 9; ++c) p.F[c] = F[c];
        for (int i = 0; i < p.n; ++i) {
            RectStmt& s = p.s[i];
            s.comp = v[i].comp; s.x0 = v[i].x0; s.x1 = v[i].x1; s.y0 = v[i].y0; s.y1 = v[i].y1; s.z0 = v[i].z0; s.z1 = v[i].z1;
            s.k = i;
            s.len = (long long)(s.x1 - s.x0 + 1) * (s.y1 - s.y0 + 1) * (s.z1 - s.z0 + 1);
            s.shape = MFD_INC_FULL;
            s.clen = s.len;
            rec_maxlen = std::max(rec_maxlen, s.len);
            if (s.len >= (1ll << 31)) throw Error(MFD_ERR_INVALID, "TFSF record face larger than 2^31 cells");
            p.arr[i] = dalloc<T>((size_t)s.len * nt);
        }
    }

    // True when no source (point source or TFSF statement) writes a cell that a monitor
    // reads.  The monitor gather of a step then runs on the side stream while the sources
    // run: it reads only its points' own cells, and the sources write only theirs.
    bool monitors_apart_from_sources(const mfd_desc* d) const {
        if (d->nmon <= 0) return false;
        long long lo = N, hi = -1;   // the monitored cells' index range: the marks cover only it
        for (int m = 0; m < d->nmon; ++m)
            for (long long j = 0; j < d->mons[m].npts; ++j) {
                lo = std::min(lo, (long long)d->mons[m].cells[j]);
                hi = std::max(hi, (long long)d->mons[m].cells[j]);
            }
        if (hi < lo) return true;
        std::vector<bool> mark((size_t)(hi - lo + 1), false);
        for (int m = 0; m < d->nmon; ++m)
            for (long long j = 0; j < d->mons[m].npts; ++j) mark[(size_t)(d->mons[m].cells[j] - lo)] = true;
        auto marked = [&](long long c) { return c >= lo && c <= hi && mark[(size_t)(c - lo)]; };
        for (int i = 0; i < d->nsrc; ++i)
            for (long long j = 0; j < d->srcs[i].npts; ++j)
                if (marked(d->srcs[i].cells[j])) return false;
        if (tfsf)
            for (int i = 0; i < tfsf_p.n; ++i) {
                const RectStmt& q = tfsf_p.s[i];
                for (int z = q.z0; z <= q.z1; ++z)
                    for (int y = q.y0; y <= q.y1; ++y)
                        for (int x = q.x0; x <= q.x1; ++x)
                            if (marked((long long)x + (long long)nx * ((long long)y + (long long)ny * z))) return false;
            }
        return true;
    }

    void init_monitors(const mfd_desc* d) {
        if (d->nmon <= 0) return;
        static const int c3[6] = {MFD_HX, MFD_HY, MFD_HZ, MFD_EX, MFD_EY, MFD_EZ};
        static const int c2[3] = {MFD_HY, MFD_EX, MFD_EZ};
        static const int c2e[3] = {MFD_HX, MFD_HZ, MFD_EY};
        static const int c1[2] = {MFD_HY, MFD_EX};
        ncomp_mon = ndim == 3 ? 6 : ndim == 2 ? 3 : 2;
        for (int k = 0; k < ncomp_mon; ++k) mon_comps[k] = ndim == 3 ? c3[k] : ey2 ? c2e[k] : ndim == 2 ? c2[k] : c1[k];
        long long ring_vals = 0;
        for (int m = 0; m < d->nmon; ++m) {
            const mfd_monitor& a = d->mons[m];
            if (a.npts < 1) throw Error(MFD_ERR_INVALID, "monitor without points");
            if (a.kind == MFD_MON_SPECTRAL && (a.nw + DFT_WT - 1) / DFT_WT > 65535)
                throw Error(MFD_ERR_INVALID, "a spectral monitor has more than 4194240 frequencies");
            if (a.kind == MFD_MON_SPECTRAL || a.sum) ring_vals += (long long)ncomp_mon * a.npts;
        }
        need_ring = ring_vals > 0;
        MFD_CK(cudaFuncSetAttribute(monitor_dft_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dft_smem_bytes<T>()));
        if (need_ring) {
            // staging depth: up to 64 steps, at most ~512 MB of staged values
            long long cap = (512ll << 20) / ((long long)sizeof(T) * ring_vals);
            ring_k = (int)std::max(1ll, std::min((long long)MFD_DFT_MAXSLOTS, cap));
        }
        for (int m = 0; m < d->nmon; ++m) {
            const mfd_monitor& a = d->mons[m];
            MonDev<T> M{};
            M.kind = a.kind; M.sum = a.sum ? 1 : 0; M.npts = a.npts; M.nw = a.nw;
            mon_maxpts = std::max(mon_maxpts, (long long)a.npts);
            std::vector<int> cells(a.npts);
            for (long long j = 0; j < a.npts; ++j) {
                if (a.cells[j] < 0 || a.cells[j] >= N) throw Error(MFD_ERR_INVALID, "monitor cell out of range");
                cells[j] = (int)pad_index(a.cells[j]);
            }
            M.cells = upload(cells.data(), cells.size());
            if (a.kind == MFD_MON_FIELD) {
                if (M.sum) M.hist = dalloc<T>((size_t)ncomp_mon * nt);
                else M.hist = dalloc<T>((size_t)ncomp_mon * nt * a.npts);
            } else {
                if (a.nw < 1 || !a.phasor) throw Error(MFD_ERR_INVALID, "spectral monitor needs frequencies");
                M.S = dalloc<double2>((size_t)ncomp_mon * a.nw * (M.sum ? 1 : a.npts));
                double2* ph = (double2*)upload(a.phasor, (size_t)nt * a.nw * 2);
                if (!M.sum) {   // tabulate 2 exp(...) dt once (dft.jl:44)
                    const long long n = (long long)nt * a.nw;
                    dft_factor_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(ph, n, (double)dt);
                    MFD_CK(cudaGetLastError());
                }
                M.phasor = ph;
            }
            if (a.kind == MFD_MON_SPECTRAL || M.sum) M.ring = dalloc<T>((size_t)ring_k * ncomp_mon * a.npts);
            mons_host.push_back(M);
        }
        if constexpr (sizeof(T) == 4) {
            bool spectral = false;
            for (const MonDev<T>& M : mons_host) spectral |= M.kind == MFD_MON_SPECTRAL && !M.sum;
            if (recip && spectral) {
                tc_fold = true;
                MFD_CK(cudaFuncSetAttribute(monitor_dft_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)dft_tc_smem_bytes));
                MFD_CK(cudaDeviceGetAttribute(&tc_sms, cudaDevAttrMultiProcessorCount, dev));
                tc_bscale = std::ldexp(1.0, -std::ilogb(2.0 * (double)dt));
                d_tcfault = dalloc<int>(1, false);
            }
        }
        mons_dev = upload(mons_host.data(), mons_host.size());
        mon_p.nmon = (int)mons_host.size();
        mon_p.ncomp = ncomp_mon;
        mon_p.nt = nt;
        for (int k = 0; k < ncomp_mon; ++k) mon_p.comp[k] = F[mon_comps[k]];
        mon_p.mons = mons_dev;
        MFD_CK(cudaStreamSynchronize(st));
    }

    // ---------------------------------------------------------------------------------
    cudaEvent_t get_event() {
        if (!ev_pool.empty()) { cudaEvent_t e = ev_pool.back(); ev_pool.pop_back(); return e; }
        cudaEvent_t e;
        MFD_CK(cudaEventCreate(&e));
        return e;
    }

    template <typename F_>
    void launch(int cls, F_&& f) {
        kcount = 1;
        if (profiling) {
            cudaEvent_t a = get_event(), b = get_event();
            MFD_CK(cudaEventRecord(a, st));
            f();
            MFD_CK(cudaEventRecord(b, st));
            pend.push_back({cls, {a, b}});
        } else {
            f();
        }
        MFD_CK(cudaGetLastError());
        k_n[cls] += kcount;
    }

    // Side-stream launches of a split update: fork() before the core launch, the side
    // launches on st_side, join() after them (the next work on st waits for both).
    void fork(bool two = false) {
        MFD_CK(cudaEventRecord(ev_fork, st));
        MFD_CK(cudaStreamWaitEvent(st_side, ev_fork, 0));
        if (two) MFD_CK(cudaStreamWaitEvent(st_side2, ev_fork, 0));
    }
    void join(bool two = false) {
        MFD_CK(cudaEventRecord(ev_join, st_side));
        MFD_CK(cudaStreamWaitEvent(st, ev_join, 0));
        if (two) {
            MFD_CK(cudaEventRecord(ev_join2, st_side2));
            MFD_CK(cudaStreamWaitEvent(st, ev_join2, 0));
        }
    }


    void collect_times() {
        for (auto& pe : pend) {
            float ms = 0;
            MFD_CK(cudaEventElapsedTime(&ms, pe.second.first, pe.second.second));
            k_ms[pe.first] += ms;
            ev_pool.push_back(pe.second.first);
            ev_pool.push_back(pe.second.second);
        }
        pend.clear();
    }

    HParams<T> hparams(int accum, long long prev_step) {
        HParams<T> p{};
        p.L = layout();
        p.ddx = ddx; p.ddy = ddy; p.ddz = ddz; p.dt = dt;
        for (int f = 0; f < 6; ++f) { p.bc[f] = bc[f]; p.lay[f] = lay[f]; }
        p.Mh0 = Mh0;
        p.geom = geom;
        p.matMh = matMh;
        p.Hx = F[MFD_HX]; p.Hy = F[MFD_HY]; p.Hz = F[MFD_HZ];
        p.Ex = F[MFD_EX]; p.Ey = F[MFD_EY]; p.Ez = F[MFD_EZ];
        p.accum = accum;
        p.sum_e2 = any_geom ? 1 : 0;
        p.Sa = Sa; p.E2 = E2;
        p.flags = d_flags;
        p.prev_step = prev_step;
        return p;
    }

    EParams<T, R> eparams() {
        EParams<T, R> p{};
        p.L = layout();
        p.ddx = ddx; p.ddy = ddy; p.ddz = ddz; p.dt = dt;
        for (int f = 0; f < 6; ++f) { p.bc[f] = bc[f]; p.lay[f] = lay[f]; }
        p.Me0 = Me0; p.Md10 = Md10; p.Md20 = Md20;
        p.geom = geom;
        p.mats = mats_dev;
        p.Hx = F[MFD_HX]; p.Hy = F[MFD_HY]; p.Hz = F[MFD_HZ];
        p.Dx = F[MFD_DX]; p.Dy = F[MFD_DY]; p.Dz = F[MFD_DZ];
        p.Ex = F[MFD_EX]; p.Ey = F[MFD_EY]; p.Ez = F[MFD_EZ];
        return p;
    }

    template <bool MATH, int FAST>
    void launch_H_t(const HParams<T>& p) {
        if (ndim == 3) {
            dim3 blk(bx3, by3), grd((nx + bx3 - 1) / bx3, (ny + by3 - 1) / by3, (nz + zc3 - 1) / zc3);
            h3d_kernel<T, MATH, FAST><<<grd, blk, 0, st>>>(p, zc3);
        } else if (ndim == 2) {
            dim3 blk(32, 8), grd((nx + 31) / 32, (nz + 7) / 8);
            if (ey2) h2e_kernel<T, MATH, FAST><<<grd, blk, 0, st>>>(p);
            else h2d_kernel<T, MATH, FAST><<<grd, blk, 0, st>>>(p);
        } else {
            dim3 blk(256), grd((nz + 255) / 256);
            h1d_kernel<T, MATH, FAST><<<grd, blk, 0, st>>>(p);
        }
    }

    // 3-D updates split into core rows and CPML slabs (yee3d_split.cuh), either element type
    template <bool MATH, int FAST, bool ACC, bool E2S>
    void launch_H_split(const HParams<T>& p) {
        kcount = 0;
        const int zn = sbox.zr - sbox.zl;
        const bool core = sbox.yr > sbox.yl && zn > 0;
        const bool lay = sizeof(T) == 4 && core_async && lay_H && recip && core && slab_rows;
        const bool ov = st_side && slab_rows && core;
        if (ov) fork(lay);
        if constexpr (sizeof(T) == 4)
            if (lay) launch_H_layers<MATH, FAST, ACC, E2S>(p, ov ? st_side : st, ov ? st_side2 : st);
        if (core) {
            if constexpr (sizeof(T) == 4) {
                if (core_async) {
                    prefer_shared((const void*)h3d_core_async_kernel<MATH, FAST, ACC, E2S>);
                    SplitBox sa = sbox;
                    sa.zc = async_zc;
                    dim3 blk(AS_TX, AS_TY), grd((nx + AS_TX - 1) / AS_TX, (sbox.yr - sbox.yl + AS_TY - 1) / AS_TY, (zn + async_zc - 1) / async_zc);
                    h3d_core_async_kernel<MATH, FAST, ACC, E2S><<<grd, blk, 0, st>>>(p, d3, sa);
                    kcount++;
                }
            }
            if (!(sizeof(T) == 4 && core_async)) {
                dim3 blk(bx3, by3), grd((nx + bx3 - 1) / bx3, (sbox.yr - sbox.yl + by3 - 1) / by3, (zn + zc3 - 1) / zc3);
                h3d_core_kernel<T, MATH, FAST, ACC, E2S><<<grd, blk, 0, st>>>(p, d3, sbox);
                kcount++;
            }
        }
        if (slab_rows && !lay) {
            dim3 grd((unsigned)slab_rows, (nx + 127) / 128);
            h3d_slab_kernel<T, MATH, FAST, ACC, E2S><<<grd, 128, 0, ov ? st_side : st>>>(p, d3, sbox);
            kcount++;
        }
        if (ov) join(lay);
    }

    // The y-layer rows over the core planes (LAY 1, on sy_) and the z-layer planes (LAY 2,
    // every row, on sz_) of a single-precision H update, by the staged kernel.
    template <bool MATH, int FAST, bool ACC, bool E2S>
    void launch_H_layers(const HParams<float>& p, cudaStream_t sy_, cudaStream_t sz_) {
        const dim3 blk(AS_TX, AS_TY);
        const int zn = sbox.zr - sbox.zl;
        for (int side = 0; side < 2; ++side) {
            const int ya = side ? sbox.yr : 0, yb = side ? ny : sbox.yl;
            if (yb <= ya || zn <= 0) continue;
            prefer_shared((const void*)h3d_core_async_kernel<MATH, FAST, ACC, E2S, 1>);
            const SplitBox sl{ya, yb, sbox.zl, sbox.zr, async_zc, 0};
            const dim3 grd((nx + AS_TX - 1) / AS_TX, (yb - ya + AS_TY - 1) / AS_TY, (zn + async_zc - 1) / async_zc);
            h3d_core_async_kernel<MATH, FAST, ACC, E2S, 1><<<grd, blk, 0, sy_>>>(p, d3, sl);
            kcount++;
        }
        for (int side = 0; side < 2; ++side) {
            const int za = side ? sbox.zr : 0, zb = side ? nz : sbox.zl;
            if (zb <= za) continue;
            prefer_shared((const void*)h3d_core_async_kernel<MATH, FAST, ACC, E2S, 2>);
            const int zc = zc_layer(zb - za);
            const SplitBox sl{0, ny, za, zb, zc, 0};
            const dim3 grd((nx + AS_TX - 1) / AS_TX, (ny + AS_TY - 1) / AS_TY, (zb - za + zc - 1) / zc);
            h3d_core_async_kernel<MATH, FAST, ACC, E2S, 2><<<grd, blk, 0, sz_>>>(p, d3, sl);
            kcount++;
        }
    }

    template <bool MATH, int FAST>
    void launch_H_split_acc(const HParams<T>& p) {
        if (!p.accum) launch_H_split<MATH, FAST, false, false>(p);
        else if (p.sum_e2) launch_H_split<MATH, FAST, true, true>(p);
        else launch_H_split<MATH, FAST, true, false>(p);
    }

    template <bool MAT, int FAST>
    void launch_E_split(const EParams<T, R>& p, int cur) {
        kcount = 0;
        const int zn = sbox.zr - sbox.zl;
        const bool core = sbox.yr > sbox.yl && zn > 0;
        const bool ov = st_side && core;
        if (ov) fork(true);
        if (core) {
            // The staged E kernel has no material-map variant (compiled with the map it
            // measured slower than e3d_core_kernel: 0.239 vs 0.218 ms per E update at 256^3
            // with a dispersive sphere).  With a map, the staged kernel without it updates
            // every tile outside the rows and planes of the materials' bounding box, and the
            // register march with the map updates those (mat_rows, aligned to the tiles).
            if constexpr (sizeof(T) == 4) {
                if (core_async) {
                    prefer_shared((const void*)e3d_core_async_kernel<R, false, FAST>);
                    SplitBox sa = sbox;
                    sa.zc = async_zc;
                    const TileSkip skip = MAT ? TileSkip{mat_x0, mat_x1, mat_rows.yl, mat_rows.yr, mat_rows.zl, mat_rows.zr}
                                              : TileSkip{0, 0, 0, 0, 0, 0};
                    const bool all_mat = MAT && mat_x0 == 0 && mat_x1 >= nx && mat_rows.yl == sbox.yl && mat_rows.yr == sbox.yr &&
                                         mat_rows.zl == sbox.zl && mat_rows.zr == sbox.zr;   // nothing left for the staged kernel
                    dim3 blk(AS_TX, AS_TY), grd((nx + AS_TX - 1) / AS_TX, (sbox.yr - sbox.yl + AS_TY - 1) / AS_TY, (zn + async_zc - 1) / async_zc);
                    // the material rows first, on their own side stream: their few
                    // long-running blocks then share the SMs with the staged kernel's
                    if (MAT && mat_rows.yr > mat_rows.yl && mat_rows.zr > mat_rows.zl) {
                        SplitBox sm = mat_rows;
                        sm.zc = zc_mat;
                        dim3 blk2(bx3, by3), grd2((mat_x1 - mat_x0 + bx3 - 1) / bx3, (sm.yr - sm.yl + by3 - 1) / by3,
                                                  (sm.zr - sm.zl + zc_mat - 1) / zc_mat);
                        const cudaStream_t s2 = ov ? st_side2 : st;
                        if (resp_fused) e3d_core_kernel<T, R, MAT, FAST, true><<<grd2, blk2, 0, s2>>>(p, d3, sm, cur, mat_x0);
                        else e3d_core_kernel<T, R, MAT, FAST><<<grd2, blk2, 0, s2>>>(p, d3, sm, 0, mat_x0);
                        kcount++;
                    }
                    if (!all_mat) {
                        e3d_core_async_kernel<R, false, FAST><<<grd, blk, 0, st>>>(p, d3, sa, skip);
                        kcount++;
                    }
                }
            }
            if (!(sizeof(T) == 4 && core_async)) {
                dim3 blk(bx3, by3), grd((nx + bx3 - 1) / bx3, (sbox.yr - sbox.yl + by3 - 1) / by3, (zn + zc3 - 1) / zc3);
                if (MAT && resp_fused) e3d_core_kernel<T, R, MAT, FAST, true><<<grd, blk, 0, st>>>(p, d3, sbox, cur);
                else e3d_core_kernel<T, R, MAT, FAST><<<grd, blk, 0, st>>>(p, d3, sbox);
                kcount++;
            }
        }
        const bool lay = sizeof(T) == 4 && core_async && lay_E && recip && core && slab_rows;
        if constexpr (sizeof(T) == 4) {
            if (lay) {
                if (MAT && mat_in_layers) launch_E_layers<true, FAST>(p, ov ? st_side : st, ov ? st_side2 : st);
                else launch_E_layers<false, FAST>(p, ov ? st_side : st, ov ? st_side2 : st);
            }
        }
        if (slab_rows && !lay) {
            dim3 grd((unsigned)slab_rows, (nx + 127) / 128);
            e3d_slab_kernel<T, R, MAT, FAST><<<grd, 128, 0, ov ? st_side : st>>>(p, d3, sbox);
            kcount++;
        }
        if (ov) join(true);
    }

    // The y-layer rows over the core planes (LAY 1, on sy_) and the z-layer planes (LAY 2, on
    // sz_) of a single-precision E update, by the staged kernel; MAT when a material cell lies
    // in a layer.
    template <bool MAT, int FAST>
    void launch_E_layers(const EParams<float, R>& p, cudaStream_t sy_, cudaStream_t sz_) {
        const dim3 blk(AS_TX, AS_TY);
        const TileSkip none{0, 0, 0, 0, 0, 0};
        const int zn = sbox.zr - sbox.zl;
        for (int side = 0; side < 2; ++side) {
            const int ya = side ? sbox.yr : 0, yb = side ? ny : sbox.yl;
            if (yb <= ya || zn <= 0) continue;
            prefer_shared((const void*)e3d_core_async_kernel<R, MAT, FAST, 1>);
            const SplitBox sl{ya, yb, sbox.zl, sbox.zr, async_zc, 0};
            const dim3 grd((nx + AS_TX - 1) / AS_TX, (yb - ya + AS_TY - 1) / AS_TY, (zn + async_zc - 1) / async_zc);
            e3d_core_async_kernel<R, MAT, FAST, 1><<<grd, blk, 0, sy_>>>(p, d3, sl, none);
            kcount++;
        }
        for (int side = 0; side < 2; ++side) {
            const int za = side ? sbox.zr : 0, zb = side ? nz : sbox.zl;
            if (zb <= za) continue;
            prefer_shared((const void*)e3d_core_async_kernel<R, MAT, FAST, 2>);
            const int zc = zc_layer(zb - za);
            const SplitBox sl{0, ny, za, zb, zc, 0};
            const dim3 grd((nx + AS_TX - 1) / AS_TX, (ny + AS_TY - 1) / AS_TY, (zb - za + zc - 1) / zc);
            e3d_core_async_kernel<R, MAT, FAST, 2><<<grd, blk, 0, sz_>>>(p, d3, sl, none);
            kcount++;
        }
    }

    // single-kernel single-precision 3-D updates (CPML layers that overlap in a dimension)
    template <bool MATH, int FAST, bool ACC, bool E2S>
    void launch_H_f32(const HParams<float>& p) {
        dim3 blk(bx3, by3), grd((nx + bx3 - 1) / bx3, (ny + by3 - 1) / by3, (nz + zc3 - 1) / zc3);
        h3d_f32_kernel<MATH, FAST, ACC, E2S><<<grd, blk, 0, st>>>(p, d3, zc3);
    }

    template <bool MATH, int FAST>
    void launch_H_f32_acc(const HParams<float>& p) {
        if (!p.accum) launch_H_f32<MATH, FAST, false, false>(p);
        else if (p.sum_e2) launch_H_f32<MATH, FAST, true, true>(p);
        else launch_H_f32<MATH, FAST, true, false>(p);
    }

    template <bool MAT, int FAST>
    void launch_E_f32(const EParams<float, R>& p) {
        dim3 blk(bx3, by3), grd((nx + bx3 - 1) / bx3, (ny + by3 - 1) / by3, (nz + zc3 - 1) / zc3);
        e3d_f32_kernel<R, MAT, FAST><<<grd, blk, 0, st>>>(p, d3, zc3);
    }

    // Calls f with the division mode of the model's kernels as a compile-time constant:
    // DIV_RECIP in the tolerance mode, else DIV_EXACT when every divisor passed the device
    // check, else DIV_IEEE.
    template <typename F_>
    void with_div(F_&& f) {
        if (recip) f(std::integral_constant<int, DIV_RECIP>{});
        else if (fastdiv) f(std::integral_constant<int, DIV_EXACT>{});
        else f(std::integral_constant<int, DIV_IEEE>{});
    }

    void launch_H(int accum, long long prev_step) {
        HParams<T> p = hparams(accum, prev_step);
        if (ndim == 3 && use_split) {
            launch(KC_H, [&] {
                with_div([&](auto dm) {
                    constexpr int D = decltype(dm)::value;
                    if (math_needed) launch_H_split_acc<true, D>(p);
                    else launch_H_split_acc<false, D>(p);
                });
            });
            return;
        }
        if constexpr (sizeof(T) == 4) {
            if (ndim == 3) {
                const HParams<float>& pf = reinterpret_cast<const HParams<float>&>(p);
                launch(KC_H, [&] {
                    with_div([&](auto dm) {
                        constexpr int D = decltype(dm)::value;
                        if (math_needed) launch_H_f32_acc<true, D>(pf);
                        else launch_H_f32_acc<false, D>(pf);
                    });
                });
                return;
            }
        }
        launch(KC_H, [&] {
            with_div([&](auto dm) {
                constexpr int D = decltype(dm)::value;
                if (math_needed) launch_H_t<true, D>(p);
                else launch_H_t<false, D>(p);
            });
        });
    }

    template <bool MAT, int FAST>
    void launch_E_t(const EParams<T, R>& p) {
        if (ndim == 3) {
            dim3 blk(bx3, by3), grd((nx + bx3 - 1) / bx3, (ny + by3 - 1) / by3, (nz + zc3 - 1) / zc3);
            e3d_kernel<T, R, MAT, FAST><<<grd, blk, 0, st>>>(p, zc3);
        } else if (ndim == 2) {
            dim3 blk(32, 8), grd((nx + 31) / 32, (nz + 7) / 8);
            if (ey2) e2e_kernel<T, R, MAT, FAST><<<grd, blk, 0, st>>>(p);
            else e2d_kernel<T, R, MAT, FAST><<<grd, blk, 0, st>>>(p);
        } else {
            dim3 blk(256), grd((nz + 255) / 256);
            e1d_kernel<T, R, MAT, FAST><<<grd, blk, 0, st>>>(p);
        }
    }

    void launch_E(int cur) {
        EParams<T, R> p = eparams();
        bool done = false;
        if (ndim == 3 && use_split) {
            launch(KC_E, [&] {
                with_div([&](auto dm) {
                    constexpr int D = decltype(dm)::value;
                    if (any_geom) launch_E_split<true, D>(p, cur);
                    else launch_E_split<false, D>(p, cur);
                });
            });
            done = true;
        }
        if constexpr (sizeof(T) == 4) {
            if (ndim == 3 && !done) {
                const EParams<float, R>& pf = reinterpret_cast<const EParams<float, R>&>(p);
                launch(KC_E, [&] {
                    with_div([&](auto dm) {
                        constexpr int D = decltype(dm)::value;
                        if (any_geom) launch_E_f32<true, D>(pf);
                        else launch_E_f32<false, D>(pf);
                    });
                });
                done = true;
            }
        }
        if (!done)
            launch(KC_E, [&] {
                with_div([&](auto dm) {
                    constexpr int D = decltype(dm)::value;
                    if (any_geom) launch_E_t<true, D>(p);
                    else launch_E_t<false, D>(p);
                });
            });
        // E of dispersive / plasma / Kerr cells: material_flat_kernel for up to 3 poles,
        // material_kernel (poles in a runtime loop) beyond -- unless the E update did it
        if (ndim == 3 && use_split && resp_fused) return;
        for (int g : response_mats) {
            const MatDev<T, R>& m = mats_host[g - 1];
            launch(KC_MAT, [&] {
                if (m.nq <= 3 && ndim >= 2) {
                    if (ndim == 3) launch_mat_flat<3>(g, m, cur);
                    else if (ey2) launch_mat_flat<1>(g, m, cur);
                    else launch_mat_flat<2>(g, m, cur);
                    return;
                }
                dim3 grd((m.bnx + 127) / 128, m.bny, m.bnz);
                if (ey2)   // one component: Dy, Ey
                    material_kernel<T, R, 1><<<grd, 128, 0, st>>>(mats_dev, g, geom, layout(), F[MFD_DY], nullptr, nullptr,
                                                                  F[MFD_EY], nullptr, nullptr, cur, dt);
                else if (ndim == 3)
                    material_kernel<T, R, 3><<<grd, 128, 0, st>>>(mats_dev, g, geom, layout(), F[MFD_DX], F[MFD_DY], F[MFD_DZ],
                                                                  F[MFD_EX], F[MFD_EY], F[MFD_EZ], cur, dt);
                else if (ndim == 2)
                    material_kernel<T, R, 2><<<grd, 128, 0, st>>>(mats_dev, g, geom, layout(), F[MFD_DX], nullptr, F[MFD_DZ],
                                                                  F[MFD_EX], nullptr, F[MFD_EZ], cur, dt);
                else
                    material_kernel<T, R, 1><<<grd, 128, 0, st>>>(mats_dev, g, geom, layout(), F[MFD_DX], nullptr, nullptr,
                                                                  F[MFD_EX], nullptr, nullptr, cur, dt);
            });
        }
    }

    template <int NC>
    void launch_mat_flat(int g, const MatDev<T, R>& m, int cur) {
        const unsigned blocks = (unsigned)((m.bsize + 255) / 256);
        // NC = 3: x, y, z; 2: x, z; 1: the one component (Dy, Ey of the second 2-D field set)
        T* D0 = NC == 1 ? F[MFD_DY] : F[MFD_DX];
        T* E0 = NC == 1 ? F[MFD_EY] : F[MFD_EX];
        T* Dy = NC == 3 ? F[MFD_DY] : nullptr;
        T* Ey = NC == 3 ? F[MFD_EY] : nullptr;
        T* Dz = NC == 1 ? nullptr : F[MFD_DZ];
        T* Ez = NC == 1 ? nullptr : F[MFD_EZ];
        switch (m.nq) {
            case 0: material_flat_kernel<T, R, NC, 0><<<blocks, 256, 0, st>>>(mats_dev, g, geom, layout(), D0, Dy, Dz, E0, Ey, Ez, cur, dt); break;
            case 1: material_flat_kernel<T, R, NC, 1><<<blocks, 256, 0, st>>>(mats_dev, g, geom, layout(), D0, Dy, Dz, E0, Ey, Ez, cur, dt); break;
            case 2: material_flat_kernel<T, R, NC, 2><<<blocks, 256, 0, st>>>(mats_dev, g, geom, layout(), D0, Dy, Dz, E0, Ey, Ez, cur, dt); break;
            default: material_flat_kernel<T, R, NC, 3><<<blocks, 256, 0, st>>>(mats_dev, g, geom, layout(), D0, Dy, Dz, E0, Ey, Ez, cur, dt); break;
        }
    }

    void launch_sources(int64_t it) {
        const long long it0 = it - 1;
        for (size_t s = 0; s <= srcs.size(); ++s) {
            if (tfsf && (int)s == tfsf_order) {
                tfsf_p.it0 = it0;
                launch(KC_TFSF, [&] {
                    const long long nb = (tfsf_maxlen + 255) / 256;
                    tfsf_kernel<T><<<dim3((unsigned)nb, tfsf_p.n), 256, 0, st>>>(tfsf_p);
                });
            }
            if (s < srcs.size()) {
                const Src& S = srcs[s];
                launch(KC_SRC, [&] {
                    const long long nb = (S.npts + 255) / 256;
                    point_source_kernel<T><<<(unsigned)nb, 256, 0, st>>>(F[S.comp], S.cells, S.npts, S.wave, S.amp, S.gt, it0, S.kind, S.coeff);
                });
            }
        }
    }

    // A tensor-core fold whose completion wait ran out leaves its spectra incomplete.
    void check_fold() const {
        if (tc_fold && h_tcfault)
            throw Error(MFD_ERR_TIMEOUT, "a spectral monitor's tensor-core fold did not complete within its wait limit");
    }

    void flush_monitors() {
        if (!need_ring || ring_used == 0) return;
        const double dtd = (double)dt;
        for (size_t m = 0; m < mons_host.size(); ++m) {
            const MonDev<T>& M = mons_host[m];
            const MonDev<T>* md = mons_dev + m;
            if (M.kind == MFD_MON_FIELD && M.sum) {
                launch(KC_DFT, [&] {
                    monitor_fieldsum_kernel<T><<<dim3(ncomp_mon, ring_used), 256, 0, st>>>(md, ncomp_mon, nt, ring_first);
                });
            } else if (M.kind == MFD_MON_SPECTRAL && !M.sum && tc_fold) {
                if constexpr (sizeof(T) == 4) {
                    launch(KC_DFT, [&] {
                        // persistent: two blocks per SM, G blocks per frequency tile over the
                        // (component, point tile) items
                        const long long nwt = (M.nw + TC_W - 1) / TC_W;
                        const long long items = (long long)ncomp_mon * ((M.npts + TC_M - 1) / TC_M);
                        const long long G = std::max(1ll, std::min(items, 2ll * tc_sms / nwt));
                        const int grid = (int)(nwt * G);
                        monitor_dft_tc_kernel<<<grid, TC_THREADS, dft_tc_smem_bytes, st>>>(md, ncomp_mon, ring_used, ring_first,
                                                                                          tc_bscale, d_tcfault);
                    });
                }
            } else if (M.kind == MFD_MON_SPECTRAL && !M.sum) {
                launch(KC_DFT, [&] {
                    // blocks of 32 x (frequency groups of the tile), tiles of DFT_PT points
                    const int wtile = std::min(DFT_WT, (M.nw + DFT_W - 1) / DFT_W * DFT_W);
                    dim3 blk(32, wtile / DFT_W);
                    dim3 grd((unsigned)((M.npts + DFT_PT - 1) / DFT_PT), ncomp_mon, (M.nw + DFT_WT - 1) / DFT_WT);
                    monitor_dft_kernel<T><<<grd, blk, dft_smem_bytes<T>(), st>>>(md, ncomp_mon, ring_used, ring_first);
                });
            } else if (M.kind == MFD_MON_SPECTRAL) {
                launch(KC_DFT, [&] {
                    monitor_dftsum_kernel<T><<<dim3(ncomp_mon, M.nw), 256, 0, st>>>(md, ncomp_mon, ring_used, ring_first, dtd);
                });
            }
        }
        ring_used = 0;
    }

    void launch_monitors(int64_t it, cudaStream_t s = nullptr) {
        if (mons_host.empty()) return;
        if (need_ring && ring_used == 0) ring_first = it - 1;
        const int slot = ring_used;
        launch(KC_MON, [&] {
            const long long nb = (mon_maxpts + 255) / 256;
            monitor_gather_kernel<T><<<dim3((unsigned)nb, mon_p.nmon), 256, 0, s ? s : st>>>(mon_p, it - 1, slot);
        });
        if (need_ring) ring_used++;
    }
    // The ring fold when the ring is full (on st, after the gather has joined).
    void fold_if_full() {
        if (need_ring && ring_used == ring_k) flush_monitors();
    }

    void launch_record(int64_t it) {
        rec_p.it0 = it - 1;
        launch(KC_MON, [&] {
            const long long nb = (rec_maxlen + 255) / 256;
            record_kernel<T><<<dim3((unsigned)nb, rec_p.n), 256, 0, st>>>(rec_p);
        });
    }

    void launch_sums(int64_t step) {
        HParams<T> p = hparams(1, step);
        launch(KC_SUMS, [&] {
            dim3 grd((nx + 255) / 256, ny, nz);
            sums_kernel<T><<<grd, 256, 0, st>>>(p, ey2 ? FSET_EY2 : ndim);
        });
    }

    bool in_batch = false;     // stepped by a batch until it retires

    // A run that ends before the last step leaves two things for later, so that the cost of
    // a step does not depend on where the caller splits a run into calls: the values staged
    // for summed and spectral monitors stay in the ring until it is full (the fold every
    // ring_k steps), and the running sums of the run's last step are added by the next run's
    // first H update (as within a run).  settle() completes both; every read that sees them,
    // a field write, a state image and joining a batch settle first.
    bool sums_pending = false;   // the running sums of step `done` are not yet added

    void launch_guard(int64_t step) {
        launch(KC_SUMS, [&] {
            dim3 grd((nx + 255) / 256, ny, nz);
            guard_kernel<T><<<grd, 256, 0, st>>>(F[guard_comp()], layout(), d_flags, step);
        });
    }

    void settle() {
        MFD_CK(cudaSetDevice(dev));
        flush_monitors();
        if (sums_pending) {
            launch_sums(done);
            sums_pending = false;
        }
    }

    int run(int64_t a, int64_t b) override {
        if (in_batch) { err = "the model is being stepped by a batch"; return MFD_ERR_INVALID; }
        if (bad_step) { err = "the model holds non-finite fields from step " + std::to_string(bad_step); return MFD_ERR_NONFINITE; }
        if (a != done + 1 || b < a - 1 || b > nt) { err = "steps must be consecutive and within 1..Nt"; return MFD_ERR_INVALID; }
        if (b < a) return MFD_OK;
        MFD_CK(cudaSetDevice(dev));
        MFD_CK(cudaEventRecord(run_ev[0], st));
        for (int64_t it = a; it <= b; ++it) {
            launch_H((it > a || sums_pending) ? 1 : 0, it - 1);
            sums_pending = false;
            launch_E((int)((it - 1) & 1));
            if (mon_apart && !profiling) {   // gather beside the sources (disjoint cells)
                fork();
                launch_monitors(it, st_side);
                launch_sources(it);
                join();
            } else {
                launch_sources(it);
                launch_monitors(it);
            }
            fold_if_full();
            if (record) launch_record(it);
            if (snap_next < snap_steps.size() && snap_steps[snap_next] == it) snapshot();
        }
        return finish(a, b, true);
    }

    // Frame snap_next: device copies into a free staging slot, then the host copies on st3.
    void snapshot() {
        const int slot = (int)(snap_next & 1);
        if (snap_busy[slot]) MFD_CK(cudaStreamWaitEvent(st, ev_snap_free[slot], 0));
        const int nc = (int)snap_comps.size();
        for (int k = 0; k < nc; ++k)
            MFD_CK(cudaMemcpyAsync(snap_stage + ((size_t)slot * nc + k) * Np, F[snap_comps[k]], (size_t)Np * sizeof(T),
                                   cudaMemcpyDeviceToDevice, st));
        MFD_CK(cudaEventRecord(ev_snap_ready[slot], st));
        MFD_CK(cudaStreamWaitEvent(st3, ev_snap_ready[slot], 0));
        for (int k = 0; k < nc; ++k) {
            char* h = snap_dst + ((size_t)snap_next * nc + k) * (size_t)N * sizeof(T);
            MFD_CK(cudaMemcpy2DAsync(h, (size_t)nx * sizeof(T), snap_stage + ((size_t)slot * nc + k) * Np, (size_t)px * sizeof(T),
                                     (size_t)nx * sizeof(T), (size_t)ny * nz, cudaMemcpyDeviceToHost, st3));
        }
        MFD_CK(cudaEventRecord(ev_snap_free[slot], st3));
        snap_busy[slot] = true;
        snap_next++;
    }

    int set_snapshots(int ncomp, const int32_t* comps, int64_t nsteps, const int64_t* steps, void* dst) override {
        if (in_batch) { err = "the model is being stepped by a batch"; return MFD_ERR_INVALID; }
        if (ncomp < 1 || ncomp > 9 || nsteps < 0 || (nsteps > 0 && (!comps || !steps || !dst))) {
            err = "snapshots need 1..9 components, the steps and a destination";
            return MFD_ERR_INVALID;
        }
        for (int k = 0; k < ncomp; ++k)
            if (comps[k] < 0 || comps[k] > 8 || !F[comps[k]]) { err = "snapshot component not in this field"; return MFD_ERR_INVALID; }
        for (int64_t i = 0; i < nsteps; ++i)
            if (steps[i] <= done || steps[i] > nt || (i && steps[i] <= steps[i - 1])) {
                err = "snapshot steps must increase and lie after the model's current step, within 1..Nt";
                return MFD_ERR_INVALID;
            }
        MFD_CK(cudaSetDevice(dev));
        if (st3) MFD_CK(cudaStreamSynchronize(st3));
        if (!st3) {
            MFD_CK(cudaStreamCreateWithFlags(&st3, cudaStreamNonBlocking));
            for (int i = 0; i < 2; ++i) {
                MFD_CK(cudaEventCreateWithFlags(&ev_snap_ready[i], cudaEventDisableTiming));
                MFD_CK(cudaEventCreateWithFlags(&ev_snap_free[i], cudaEventDisableTiming));
            }
        }
        if (nsteps > 0 && ncomp > snap_cap) {
            snap_stage = dalloc<T>((size_t)2 * ncomp * Np, false);   // kept until the handle is destroyed
            snap_cap = ncomp;
            MFD_CK(cudaStreamSynchronize(st));
        }
        snap_comps.assign(comps, comps + ncomp);
        snap_steps.assign(steps, steps + nsteps);
        snap_next = 0;
        snap_dst = (char*)dst;
        snap_busy[0] = snap_busy[1] = false;
        return MFD_OK;
    }

    // End of a run of steps a..b (also of a batch member's window): staged monitors, the
    // running sums of step b, and the per-step NaN/Inf flags.  With defer (mfd_run) and b
    // before the last step, the monitors' ring and the sums of step b are left for later
    // (settle) and only the NaN/Inf guard of step b runs now.
    int finish(int64_t a, int64_t b, bool defer = false) {
        if (defer && b < nt) {
            launch_guard(b);
            sums_pending = true;
        } else {
            flush_monitors();
            launch_sums(b);
        }
        if (st3 && (snap_busy[0] || snap_busy[1])) bounded_sync(st3);   // frames of steps <= b are on the host
        MFD_CK(cudaEventRecord(run_ev[1], st));
        MFD_CK(cudaMemcpyAsync(h_flags + (a - 1), d_flags + (a - 1), (size_t)(b - a + 1) * sizeof(int),
                               cudaMemcpyDeviceToHost, st));
        if (tc_fold) MFD_CK(cudaMemcpyAsync(&h_tcfault, d_tcfault, sizeof(int), cudaMemcpyDeviceToHost, st));
        bounded_sync(st);
        check_fold();
        float ms = 0;
        MFD_CK(cudaEventElapsedTime(&ms, run_ev[0], run_ev[1]));
        run_ms = ms;
        if (profiling) collect_times();
        done = b;
        int64_t first = 0;
        for (int64_t it = a; it <= b && !first; ++it)
            if (h_flags[it - 1]) first = it;
        if (first) {
            bad_kind = h_flags[first - 1];
            bad_step = first;
            err = (bad_kind & 1) ? "Something went wrong. I found NaN field values."
                                 : "Something went wrong. I found Inf field values.";
            err += " (step " + std::to_string(bad_step) + ")";
            return MFD_ERR_NONFINITE;
        }
        return MFD_OK;
    }

    void copy_out(const void* dsrc, void* hdst, size_t esize) {
        MFD_CK(cudaSetDevice(dev));
        MFD_CK(cudaMemcpy2DAsync(hdst, (size_t)nx * esize, dsrc, (size_t)px * esize, (size_t)nx * esize, (size_t)ny * nz,
                                 cudaMemcpyDeviceToHost, st));
        bounded_sync(st);
    }

    int read_geometry(uint8_t* dst) override {
        if (geom) copy_out(geom, dst, 1);
        else std::memset(dst, 0, (size_t)N);
        return MFD_OK;
    }

    int read_field(int comp, void* dst) override {
        if (comp < 0 || comp > 8 || !F[comp]) { err = "bad component"; return MFD_ERR_INVALID; }
        copy_out(F[comp], dst, sizeof(T));
        return MFD_OK;
    }

    int write_field(int comp, const void* src) override {
        if (comp < 0 || comp > 8 || !F[comp]) { err = "bad component"; return MFD_ERR_INVALID; }
        settle();   // the pending running sums belong to the fields before the write
        MFD_CK(cudaMemcpy2DAsync(F[comp], (size_t)px * sizeof(T), src, (size_t)nx * sizeof(T), (size_t)nx * sizeof(T),
                                 (size_t)ny * nz, cudaMemcpyHostToDevice, st));
        bounded_sync(st);
        return MFD_OK;
    }

    int read_integral(int which, void* dst) override {
        settle();
        if (which == MFD_INT_SA) { copy_out(Sa, dst, sizeof(T)); return MFD_OK; }
        if (which == MFD_INT_E2) {
            if (E2) copy_out(E2, dst, sizeof(T));
            else std::memset(dst, 0, (size_t)N * sizeof(T));
            return MFD_OK;
        }
        if (which == MFD_INT_JE || which == MFD_INT_RHO) {
            const size_t es = which == MFD_INT_JE ? sizeof(T) : sizeof(double);
            if (!any_plasma || !any_geom) { std::memset(dst, 0, (size_t)N * es); return MFD_OK; }
            void* tmp = nullptr;
            MFD_CK(cudaMallocAsync(&tmp, (size_t)Np * es, st));
            dim3 grd((nx + 255) / 256, ny, nz);
            scatter_state_kernel<T, R><<<grd, 256, 0, st>>>(mats_dev, geom, layout(), tmp, which);
            MFD_CK(cudaGetLastError());
            try {
                copy_out(tmp, dst, es);
            } catch (...) {
                cudaFreeAsync(tmp, st);
                throw;
            }
            MFD_CK(cudaFreeAsync(tmp, st));
            bounded_sync(st);
            return MFD_OK;
        }
        err = "bad integral";
        return MFD_ERR_INVALID;
    }

    // JE / rho_end staged through g_read_scratch a few z-planes at a time (no device
    // allocation); Sa and E2 are plain copies from their arrays.
    bool noalloc_ready = false;
    int read_integral_noalloc(int which, void* dst) override {
        MFD_CK(cudaSetDevice(dev));
        if (which == MFD_INT_SA || which == MFD_INT_E2) return read_integral(which, dst);
        if (which != MFD_INT_JE && which != MFD_INT_RHO) { err = "bad integral"; return MFD_ERR_INVALID; }
        const size_t es = which == MFD_INT_JE ? sizeof(T) : sizeof(double);
        // no plasma: zeros without touching the device, as mfd_read_integral returns them
        if (!any_plasma || !any_geom) { std::memset(dst, 0, (size_t)N * es); return MFD_OK; }
        const size_t plane = (size_t)nx * ny * es;
        if (plane > (size_t)MFD_NOALLOC_SCRATCH_BYTES) {
            err = "mfd_read_integral_noalloc: one z-plane of this grid is " + std::to_string(plane) +
                  " bytes, more than its " + std::to_string((size_t)MFD_NOALLOC_SCRATCH_BYTES) +
                  "-byte scratch buffer; use mfd_read_integral";
            return MFD_ERR_INVALID;
        }
        unsigned char* scratch = (unsigned char*)read_scratch();
        if (!noalloc_ready) {   // load the kernel now rather than at its first launch
            cudaFuncAttributes fa;
            MFD_CK(cudaFuncGetAttributes(&fa, scatter_state_planes_kernel<T, R>));
            noalloc_ready = true;
        }
        const int per = (int)std::min<size_t>({(size_t)nz, (size_t)MFD_NOALLOC_SCRATCH_BYTES / plane, (size_t)65535});
        for (int z0 = 0; z0 < nz; z0 += per) {
            const int n = std::min(per, nz - z0);
            dim3 grd((nx + 255) / 256, ny, n);
            scatter_state_planes_kernel<T, R><<<grd, 256, 0, st>>>(mats_dev, geom, layout(), scratch, which, z0);
            MFD_CK(cudaGetLastError());
            MFD_CK(cudaMemcpyAsync((char*)dst + (size_t)z0 * plane, scratch, (size_t)n * plane, cudaMemcpyDeviceToHost, st));
        }
        bounded_sync(st);
        return MFD_OK;
    }

    int read_monitor(int m, int comp, void* dst) override {
        if (m < 0 || m >= (int)mons_host.size()) { err = "bad monitor"; return MFD_ERR_INVALID; }
        int k = -1;
        for (int j = 0; j < ncomp_mon; ++j) if (mon_comps[j] == comp) k = j;
        if (k < 0) { err = "bad monitor component"; return MFD_ERR_INVALID; }
        const MonDev<T>& M = mons_host[m];
        MFD_CK(cudaSetDevice(dev));
        flush_monitors();   // the values still staged in the ring
        if (M.kind == MFD_MON_FIELD) {
            const size_t n = M.sum ? (size_t)nt : (size_t)nt * M.npts;
            MFD_CK(cudaMemcpyAsync(dst, M.hist + (size_t)k * n, n * sizeof(T), cudaMemcpyDeviceToHost, st));
        } else {
            const size_t n = (size_t)M.nw * (M.sum ? 1 : M.npts);
            MFD_CK(cudaMemcpyAsync(dst, M.S + (size_t)k * n, n * sizeof(double2), cudaMemcpyDeviceToHost, st));
        }
        if (tc_fold) MFD_CK(cudaMemcpyAsync(&h_tcfault, d_tcfault, sizeof(int), cudaMemcpyDeviceToHost, st));
        bounded_sync(st);
        check_fold();
        return MFD_OK;
    }

    int read_record(int k, void* dst) override {
        if (!record || k < 0 || k >= rec_narr) { err = "no such record array"; return MFD_ERR_INVALID; }
        MFD_CK(cudaSetDevice(dev));
        MFD_CK(cudaMemcpyAsync(dst, rec_p.arr[k], (size_t)rec_p.s[k].len * nt * sizeof(T), cudaMemcpyDeviceToHost, st));
        bounded_sync(st);
        return MFD_OK;
    }

    int64_t record_size(int k) const override {
        if (!record || k < 0 || k >= rec_narr) return 0;
        return (int64_t)rec_p.s[k].len * nt;
    }

    void status(int64_t* d, int64_t* b, int32_t* k) const override {
        if (d) *d = done;
        if (b) *b = bad_step;
        if (k) *k = bad_kind;
    }

    void set_profiling(bool on) override { profiling = on; }

    int kernel_times(double* ms, int64_t* launches, int n) const override {
        for (int k = 0; k < n && k < KC_N; ++k) {
            if (ms) ms[k] = k_ms[k];
            if (launches) launches[k] = k_n[k];
        }
        return KC_N;
    }

    double last_run_ms() const override { return run_ms; }
    int64_t device_bytes() const override { return bytes; }

    // ---- state images -----------------------------------------------------------------
    uint64_t layout_hash() const {
        uint64_t hsh = 1469598103934665603ull;   // FNV-1a over the dimensions and buffer sizes
        auto mix = [&](uint64_t v) {
            for (int i = 0; i < 8; ++i) { hsh ^= (v >> (8 * i)) & 0xff; hsh *= 1099511628211ull; }
        };
        mix((uint64_t)ndim); mix((uint64_t)ey2); mix(sizeof(T)); mix(sizeof(R)); mix((uint64_t)nx); mix((uint64_t)ny); mix((uint64_t)nz);
        mix((uint64_t)nt); mix(state_bufs.size());
        for (auto& b : state_bufs) mix(b.second);
        return hsh;
    }

    int64_t state_size() const override {
        int64_t n = (int64_t)sizeof(StateHeader);
        for (auto& b : state_bufs) n += (int64_t)b.second;
        return n;
    }

    int read_state(void* dst, int64_t n) override {
        if (in_batch) { err = "the model is being stepped by a batch"; return MFD_ERR_INVALID; }
        if (n < state_size()) { err = "state buffer smaller than mfd_state_size()"; return MFD_ERR_INVALID; }
        settle();   // the image holds no staged values and no pending sums
        if (st3) bounded_sync(st3);
        StateHeader hd{};
        std::memcpy(hd.magic, "MFDSTATE", 8);
        hd.version = 1;
        hd.nbuf = (uint32_t)state_bufs.size();
        hd.layout = layout_hash();
        hd.done = done; hd.bad_step = bad_step; hd.bad_kind = bad_kind;
        char* out = (char*)dst;
        std::memcpy(out, &hd, sizeof(hd));
        size_t off = sizeof(hd);
        for (auto& b : state_bufs) {
            MFD_CK(cudaMemcpyAsync(out + off, b.first, b.second, cudaMemcpyDeviceToHost, st));
            off += b.second;
        }
        bounded_sync(st);
        return MFD_OK;
    }

    int write_state(const void* src, int64_t n) override {
        if (in_batch) { err = "the model is being stepped by a batch"; return MFD_ERR_INVALID; }
        if (n < (int64_t)sizeof(StateHeader)) { err = "state image too short"; return MFD_ERR_INVALID; }
        StateHeader hd;
        std::memcpy(&hd, src, sizeof(hd));
        if (std::memcmp(hd.magic, "MFDSTATE", 8) != 0 || hd.version != 1) { err = "not a state image of this library"; return MFD_ERR_INVALID; }
        if (hd.nbuf != state_bufs.size() || hd.layout != layout_hash() || n < state_size()) {
            err = "the state image belongs to a model of another layout (create the handle from the same descriptor)";
            return MFD_ERR_INVALID;
        }
        if (hd.done < 0 || hd.done > nt) { err = "state image with a step beyond Nt"; return MFD_ERR_INVALID; }
        MFD_CK(cudaSetDevice(dev));
        if (st3) bounded_sync(st3);
        const char* in = (const char*)src;
        size_t off = sizeof(hd);
        for (auto& b : state_bufs) {
            MFD_CK(cudaMemcpyAsync(b.first, in + off, b.second, cudaMemcpyHostToDevice, st));
            off += b.second;
        }
        bounded_sync(st);
        done = hd.done;
        bad_step = hd.bad_step;
        bad_kind = hd.bad_kind;
        ring_used = 0;
        sums_pending = false;
        snap_steps.clear();
        snap_next = 0;
        snap_busy[0] = snap_busy[1] = false;
        return MFD_OK;
    }
};

thread_local std::string g_create_error;

}  // namespace mfd

using namespace mfd;

struct mfd_handle {
    std::unique_ptr<HandleBase> impl;
};

// ------------------------------------------------------------------------------------------
// Batch of 2-D and 3-D single-precision models (batch.cuh): members are ordinary handles; the batch
// runs each one's steps first..last with persistent batched launches replayed from a CUDA
// graph of `gsteps` steps, then retires it with the same end-of-run work as mfd_run.
// ------------------------------------------------------------------------------------------
template <typename U>
struct DevBuf {   // a device table that grows; stream-ordered pool memory of the batch's stream
    U* p = nullptr;
    size_t cap = 0;
    cudaStream_t st = nullptr;
    void reserve(size_t n, cudaStream_t s) {
        st = s;
        if (n <= cap) return;
        if (p) cudaFreeAsync(p, st);
        p = nullptr;
        cap = 0;
        const size_t c = std::max<size_t>(n, 64);
        if (cudaMallocAsync(&p, c * sizeof(U), st) != cudaSuccess) {
            cudaGetLastError();
            throw Error(MFD_ERR_OOM, "batch table allocation failed");
        }
        cap = c;
    }
    void upload(const std::vector<U>& v, cudaStream_t s) {
        reserve(v.size(), s);
        if (!v.empty()) MFD_CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(U), cudaMemcpyHostToDevice, st));
    }
    void release() {
        if (p && st) cudaFreeAsync(p, st);
        p = nullptr;
        cap = 0;
    }
    ~DevBuf() { release(); }
};

struct mfd_batch {
    using E = Engine<float, double>;
    struct Member {
        mfd_handle* h;
        E* e;
        long long first, last, it;
        int flags;
        HParams<float>* hp = nullptr;
        EParams<float, double>* ep = nullptr;
        MonParams<float>* mp = nullptr;
        RectParams<float>* rp = nullptr;
        long long cells;
    };
    int dev = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    std::string err;
    std::vector<Member> mem;
    // tables
    DevBuf<BMember> d_mem;
    DevBuf<BTile> d_tiles, d_tiles3;       // tiles of 2-D / 3-D members
    DevBuf<BMatTile> d_mtiles, d_mtiles3;
    DevBuf<BSrc> d_srcs;
    DevBuf<BPoint> d_mpts;
    std::vector<std::unique_ptr<DevBuf<BPoint>>> d_spass;
    std::vector<std::unique_ptr<DevBuf<BRow>>> d_tpass;   // TFSF rows of source pass k
    std::vector<int> tpass_n, tpass_len;
    // [0] 2-D tiles, [1] 2-D material tiles, [2] monitor points, [3] 3-D tiles, [4] 3-D material
    // tiles, [5 + k] points of source pass k
    DevBuf<int> d_counts;
    int ntiles = 0, nmtiles = 0, nmpts = 0, ntiles3 = 0, nmtiles3 = 0;
    bool has_set[2] = {false, false};   // members of the exact arithmetic / the tolerance mode
    std::vector<int> spass_n;
    // graph
    cudaGraphExec_t gexec = nullptr;
    int gsteps = 16, built_steps = 0;
    bool dirty = true;
    // tiles and autotuning
    int tx = 0, tz = 0;           // fixed shape, or 0 = autotune
    int cur_tx = 32, cur_tz = 8;
    std::vector<std::pair<int, int>> cands{{32, 4}, {32, 8}, {64, 4}, {128, 2}, {32, 16}, {64, 8}, {32, 2}};
    size_t tune_next = 0;
    std::vector<double> tune_cost;
    bool tuned = false;
    // statistics
    double dev_ms = 0;
    long long cell_updates = 0, launches = 0;

    ~mfd_batch() {
        cudaSetDevice(dev);
        if (st) cudaStreamSynchronize(st);
        if (gexec) cudaGraphExecDestroy(gexec);
        for (auto& m : mem) release(m);
        d_mem.release(); d_tiles.release(); d_mtiles.release(); d_tiles3.release(); d_mtiles3.release();
        d_srcs.release(); d_mpts.release(); d_counts.release();
        d_spass.clear();
        d_tpass.clear();
        if (st) cudaStreamSynchronize(st);
        for (auto e : ev) if (e) cudaEventDestroy(e);
        if (st) cudaStreamDestroy(st);
    }

    void release(Member& m) {
        if (m.hp) cudaFreeAsync(m.hp, st);
        if (m.ep) cudaFreeAsync(m.ep, st);
        if (m.mp) cudaFreeAsync(m.mp, st);
        if (m.rp) cudaFreeAsync(m.rp, st);
        m.hp = nullptr; m.ep = nullptr; m.mp = nullptr; m.rp = nullptr;
        if (m.e) m.e->in_batch = false;
    }

    template <typename U>
    U* copy_struct(const U& v) {
        U* d = nullptr;
        if (cudaMallocAsync(&d, sizeof(U), st) != cudaSuccess) { cudaGetLastError(); throw Error(MFD_ERR_OOM, "batch member allocation failed"); }
        MFD_CK(cudaMemcpyAsync(d, &v, sizeof(U), cudaMemcpyHostToDevice, st));
        MFD_CK(cudaStreamSynchronize(st));   // the host copy is a temporary
        return d;
    }

    void init(int device) {
        dev = device;
        MFD_CK(cudaSetDevice(dev));
        MFD_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        MFD_CK(cudaEventCreate(&ev[0]));
        MFD_CK(cudaEventCreate(&ev[1]));
        retain_pool(dev);
        d_counts.reserve(64, st);
    }

    int add(mfd_handle* h, long long last) {
        if (!h || !h->impl) { err = "null handle"; return MFD_ERR_INVALID; }
        E* e = dynamic_cast<E*>(h->impl.get());
        if (!e) { err = "batch members must be single precision with double-precision plasma density (the default)"; return MFD_ERR_INVALID; }
        if (e->ndim < 2) { err = "batch members must be 2-D or 3-D models"; return MFD_ERR_INVALID; }
        if (e->ey2) { err = "batch members use the first 2-D field set (MFD_POL_HY)"; return MFD_ERR_INVALID; }
        if (e->dev != dev) { err = "batch member on another device"; return MFD_ERR_INVALID; }
        if (e->in_batch) { err = "model already in a batch"; return MFD_ERR_INVALID; }
        if (e->record) { err = "batch members cannot record TFSF data"; return MFD_ERR_INVALID; }
        if (e->snap_next < e->snap_steps.size()) { err = "batch members cannot take field snapshots"; return MFD_ERR_INVALID; }
        if (e->bad_step) { err = "the model holds non-finite fields"; return MFD_ERR_NONFINITE; }
        if (last <= e->done || last > e->nt) { err = "the last step must be after the model's current step and within 1..Nt"; return MFD_ERR_INVALID; }
        e->settle();   // a member starts with an empty ring and its sums added
        bounded_sync(e->st);
        MFD_CK(cudaSetDevice(dev));
        Member m{};
        m.h = h; m.e = e; m.first = e->done + 1; m.last = last; m.it = m.first;
        m.flags = (e->math_needed ? BF_MATH : 0) | (e->any_geom ? BF_MAT : 0) | (e->fastdiv ? BF_FAST : 0) | (e->ndim == 3 ? BF_3D : 0) |
                  (e->recip ? BF_RECIP : 0);
        m.cells = (long long)e->nx * e->ny * e->nz;
        try {
            m.hp = copy_struct(e->hparams(0, 0));
            m.ep = copy_struct(e->eparams());
            m.mp = copy_struct(e->mon_p);
            if (e->tfsf) m.rp = copy_struct(e->tfsf_p);
        } catch (...) {
            release(m);
            throw;
        }
        MFD_CK(cudaStreamSynchronize(e->st));          // the member's own work is complete
        MFD_CK(cudaEventRecord(e->run_ev[0], e->st));
        e->in_batch = true;
        mem.push_back(m);
        dirty = true;
        return MFD_OK;
    }

    // Tables of the current members and tile shape, then the graph of gsteps steps.
    void rebuild() {
        std::vector<BMember> hm;
        std::vector<BTile> tiles, tiles3;
        std::vector<BMatTile> mt, mt3;
        std::vector<BSrc> srcs;
        std::vector<std::vector<BPoint>> passes;
        std::vector<std::vector<BRow>> tpasses;
        std::vector<int> tlen;
        std::vector<BPoint> mpts;
        has_set[0] = has_set[1] = false;
        for (size_t i = 0; i < mem.size(); ++i) {
            const Member& m = mem[i];
            E* e = m.e;
            has_set[(m.flags & BF_RECIP) ? 1 : 0] = true;
            hm.push_back(BMember{m.hp, m.ep, m.mp, m.rp, m.it, m.first, m.last, e->ring_first, m.flags, 0, e->d3});
            const int mi = (int)i;
            const bool d3 = e->ndim == 3;
            const int rows = d3 ? e->ny * e->nz : e->nz;   // 3-D: rows y + ny z
            if (d3) {
                const int ncell = e->nx * rows;
                for (int l = 0; l < ncell; l += cur_tx * cur_tz) {   // (x, y, z) of the tile's first cell
                    const int r = l / e->nx;
                    tiles3.push_back(BTile{mi, l - r * e->nx, r % e->ny, r / e->ny});
                }
            } else {
                for (int z = 0; z < rows; z += cur_tz)
                    for (int x = 0; x < e->nx; x += cur_tx) (d3 ? tiles3 : tiles).push_back(BTile{mi, x, z, 0});
            }
            for (int g : e->response_mats) {
                const MatDev<float, double>& md = e->mats_host[g - 1];
                const int y0 = d3 ? md.by0 : 0, y1 = d3 ? md.by0 + md.bny : 1;
                for (int z = md.bz0; z < md.bz0 + md.bnz; ++z)
                    for (int y = y0; y < y1; ++y)
                        for (int x = md.bx0; x < md.bx0 + md.bnx; x += 128) (d3 ? mt3 : mt).push_back(BMatTile{mi, g, x, y, z});
            }
            if (e->tfsf) {   // TFSF acts in source pass tfsf_order, before point source tfsf_order
                const size_t k = (size_t)e->tfsf_order;
                if (tpasses.size() <= k) { tpasses.resize(k + 1); tlen.resize(k + 1, 0); }
                for (int q = 0; q < e->tfsf_p.n; ++q) tpasses[k].push_back(BRow{mi, q});
                tlen[k] = std::max(tlen[k], (int)e->tfsf_maxlen);
            }
            for (size_t k = 0; k < e->srcs.size(); ++k) {
                const auto& S = e->srcs[k];
                if (passes.size() <= k) passes.emplace_back();
                const int si = (int)srcs.size();
                srcs.push_back(BSrc{e->F[S.comp], S.cells, S.wave, S.amp, S.gt, S.npts, S.kind, S.coeff});
                for (long long j = 0; j < S.npts; ++j) passes[k].push_back(BPoint{mi, si, j});
            }
            for (size_t k = 0; k < e->mons_host.size(); ++k)
                for (long long j = 0; j < e->mons_host[k].npts; ++j) mpts.push_back(BPoint{mi, (int)k, j});
        }
        d_mem.upload(hm, st);
        d_tiles.upload(tiles, st);
        d_mtiles.upload(mt, st);
        d_tiles3.upload(tiles3, st);
        d_mtiles3.upload(mt3, st);
        d_srcs.upload(srcs, st);
        d_mpts.upload(mpts, st);
        if (tpasses.size() > passes.size()) passes.resize(tpasses.size());
        tpasses.resize(passes.size());
        tlen.resize(passes.size(), 0);
        while (d_spass.size() < passes.size()) d_spass.emplace_back(new DevBuf<BPoint>());
        while (d_tpass.size() < passes.size()) d_tpass.emplace_back(new DevBuf<BRow>());
        spass_n.assign(passes.size(), 0);
        tpass_n.assign(passes.size(), 0);
        tpass_len = tlen;
        for (size_t k = 0; k < passes.size(); ++k) {
            d_spass[k]->upload(passes[k], st);
            spass_n[k] = (int)passes[k].size();
            d_tpass[k]->upload(tpasses[k], st);
            tpass_n[k] = (int)tpasses[k].size();
            if (tpass_n[k] > 65535) throw Error(MFD_ERR_INVALID, "too many TFSF statements in one batch pass");
        }
        // graph length: at most the smallest staging ring of any member (rings are flushed between replays)
        ring_cap = gsteps;
        for (auto& m : mem)
            if (m.e->need_ring) ring_cap = std::min(ring_cap, m.e->ring_k);
        if (passes.size() + 5 > 64) throw Error(MFD_ERR_INVALID, "batch members have at most 59 sources");
        std::vector<int> counts(5 + passes.size());
        ntiles = counts[0] = (int)tiles.size();
        nmtiles = counts[1] = (int)mt.size();
        nmpts = counts[2] = (int)mpts.size();
        ntiles3 = counts[3] = (int)tiles3.size();
        nmtiles3 = counts[4] = (int)mt3.size();
        for (size_t k = 0; k < passes.size(); ++k) counts[5 + k] = spass_n[k];
        d_counts.upload(counts, st);
        MFD_CK(cudaStreamSynchronize(st));
        build_graph();
        dirty = false;
    }

    int grid_for(const void* fn, int threads, int work) {
        int per_sm = 0, sms = 0;
        MFD_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, 0));
        MFD_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        return std::max(1, std::min(std::max(1, per_sm) * sms, work));
    }

    int ring_cap = 16;          // steps per graph replay (gsteps, or less when a member's ring is shorter)

    int kernels_per_step() const {
        int k = 1 + (ntiles ? 2 : 0) + (ntiles3 ? 2 : 0) + (nmtiles ? 1 : 0) + (nmtiles3 ? 1 : 0) + (nmpts ? 1 : 0);
        for (int n : spass_n) k += n ? 1 : 0;
        for (int n : tpass_n) k += n ? 1 : 0;
        return k;
    }

    void launch_step() {
        const dim3 blk(cur_tx, cur_tz);
        // the half-step kernels of each arithmetic set the batch holds (batch.cuh)
        for (int set = 0; set < 2; ++set) {
            if (!has_set[set]) continue;
            if (ntiles) {
                const void* k = set ? (const void*)batch_h2d_kernel<1> : (const void*)batch_h2d_kernel<0>;
                const int gt = grid_for(k, cur_tx * cur_tz, ntiles);
                if (set) batch_h2d_kernel<1><<<gt, blk, 0, st>>>(d_mem.p, d_tiles.p, d_counts.p + 0);
                else batch_h2d_kernel<0><<<gt, blk, 0, st>>>(d_mem.p, d_tiles.p, d_counts.p + 0);
            }
            if (ntiles3) {
                const void* k = set ? (const void*)batch_h3d_kernel<1> : (const void*)batch_h3d_kernel<0>;
                const int gt = grid_for(k, cur_tx * cur_tz, ntiles3);
                if (set) batch_h3d_kernel<1><<<gt, blk, 0, st>>>(d_mem.p, d_tiles3.p, d_counts.p + 3);
                else batch_h3d_kernel<0><<<gt, blk, 0, st>>>(d_mem.p, d_tiles3.p, d_counts.p + 3);
            }
        }
        for (int set = 0; set < 2; ++set) {
            if (!has_set[set]) continue;
            if (ntiles) {
                const void* k = set ? (const void*)batch_e2d_kernel<1> : (const void*)batch_e2d_kernel<0>;
                const int gt = grid_for(k, cur_tx * cur_tz, ntiles);
                if (set) batch_e2d_kernel<1><<<gt, blk, 0, st>>>(d_mem.p, d_tiles.p, d_counts.p + 0);
                else batch_e2d_kernel<0><<<gt, blk, 0, st>>>(d_mem.p, d_tiles.p, d_counts.p + 0);
            }
            if (ntiles3) {
                const void* k = set ? (const void*)batch_e3d_kernel<1> : (const void*)batch_e3d_kernel<0>;
                const int gt = grid_for(k, cur_tx * cur_tz, ntiles3);
                if (set) batch_e3d_kernel<1><<<gt, blk, 0, st>>>(d_mem.p, d_tiles3.p, d_counts.p + 3);
                else batch_e3d_kernel<0><<<gt, blk, 0, st>>>(d_mem.p, d_tiles3.p, d_counts.p + 3);
            }
        }
        if (nmtiles) {
            const int g = grid_for((const void*)batch_material2d_kernel, 128, nmtiles);
            batch_material2d_kernel<<<g, 128, 0, st>>>(d_mem.p, d_mtiles.p, d_counts.p + 1);
        }
        if (nmtiles3) {
            const int g = grid_for((const void*)batch_material3d_kernel, 128, nmtiles3);
            batch_material3d_kernel<<<g, 128, 0, st>>>(d_mem.p, d_mtiles3.p, d_counts.p + 4);
        }
        for (size_t k = 0; k < spass_n.size(); ++k) {
            if (tpass_n[k])
                batch_tfsf_kernel<<<dim3((unsigned)((tpass_len[k] + 255) / 256), tpass_n[k]), 256, 0, st>>>(d_mem.p, d_tpass[k]->p);
            if (spass_n[k])
                batch_source_kernel<<<(spass_n[k] + 255) / 256, 256, 0, st>>>(d_mem.p, d_srcs.p, d_spass[k]->p, d_counts.p + 5 + k);
        }
        if (nmpts) batch_gather_kernel<<<(nmpts + 255) / 256, 256, 0, st>>>(d_mem.p, d_mpts.p, d_counts.p + 2);
        batch_advance_kernel<<<((int)mem.size() + 255) / 256, 256, 0, st>>>(d_mem.p, (int)mem.size());
    }

    void build_graph() {
        if (gexec) { MFD_CK(cudaGraphExecDestroy(gexec)); gexec = nullptr; }
        cudaGraph_t g = nullptr;
        MFD_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < ring_cap; ++i) launch_step();
        const cudaError_t ce = cudaStreamEndCapture(st, &g);
        if (ce != cudaSuccess) { cudaGetLastError(); throw Error(MFD_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce)); }
        const cudaError_t ie = cudaGraphInstantiate(&gexec, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) { cudaGetLastError(); throw Error(MFD_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie)); }
        built_steps = ring_cap;
    }

    // Before a replay of n steps: flush members whose staging ring cannot take n more steps,
    // and start a new ring window where one is empty (its first slot is this step).
    void prepare_rings(int n) {
        for (size_t i = 0; i < mem.size(); ++i) {
            Member& m = mem[i];
            E* e = m.e;
            if (!e->need_ring || m.it > m.last) continue;
            if (e->ring_used > 0 && e->ring_used + n > e->ring_k) {
                e->flush_monitors();
                bounded_sync(e->st);
            }
            if (e->ring_used == 0 && e->ring_first != m.it - 1) {
                e->ring_first = m.it - 1;
                MFD_CK(cudaMemcpyAsync(&d_mem.p[i].ring_first, &e->ring_first, sizeof(long long), cudaMemcpyHostToDevice, st));
            }
        }
    }

    // Retire members whose window is done: the end-of-run work of mfd_run on their streams.
    void retire() {
        std::vector<Member> keep;
        for (auto& m : mem) {
            if (m.it <= m.last) { keep.push_back(m); continue; }
            m.e->in_batch = false;
            m.e->finish(m.first, m.last);   // its status (NaN/Inf step) is kept by the handle
            release(m);
            dirty = true;
        }
        mem.swap(keep);
    }

    int run(long long max_steps, int* n_active) {
        MFD_CK(cudaSetDevice(dev));
        long long done_steps = 0;
        while (done_steps < max_steps && !mem.empty()) {
            // autotune: one graph chunk per candidate tile shape, then the cheapest per cell-update
            if (!tuned) {
                if (tx > 0) { cur_tx = tx; cur_tz = tz; tuned = true; dirty = true; }
                else if (tune_next < cands.size()) {
                    if (cur_tx != cands[tune_next].first || cur_tz != cands[tune_next].second || !gexec) {
                        cur_tx = cands[tune_next].first; cur_tz = cands[tune_next].second; dirty = true;
                    }
                }
            }
            if (dirty) rebuild();
            const int gs = built_steps;
            long long active_cells = 0;
            for (auto& m : mem) active_cells += m.cells * std::min<long long>(gs, m.last - m.it + 1);
            const bool chunk = max_steps - done_steps >= gs;
            const int n = chunk ? gs : (int)(max_steps - done_steps);
            prepare_rings(n);
            MFD_CK(cudaEventRecord(ev[0], st));
            if (chunk) MFD_CK(cudaGraphLaunch(gexec, st));
            else for (int i = 0; i < n; ++i) launch_step();
            MFD_CK(cudaEventRecord(ev[1], st));
            MFD_CK(cudaGetLastError());
            bounded_sync(st);
            float ms = 0;
            MFD_CK(cudaEventElapsedTime(&ms, ev[0], ev[1]));
            long long cu = 0;
            for (auto& m : mem) {
                const long long adv = std::max<long long>(0, std::min<long long>(n, m.last - m.it + 1));
                cu += m.cells * adv;
                m.it += adv;
                if (m.e->need_ring) m.e->ring_used += (int)adv;
            }
            dev_ms += ms;
            cell_updates += cu;
            launches += (long long)n * kernels_per_step();
            if (!tuned && tx == 0 && chunk) {
                tune_cost.push_back(active_cells > 0 ? ms / (double)active_cells : 1e30);
                if (++tune_next >= cands.size()) {
                    size_t best = 0;
                    for (size_t i = 1; i < tune_cost.size(); ++i) if (tune_cost[i] < tune_cost[best]) best = i;
                    cur_tx = cands[best].first; cur_tz = cands[best].second;
                    tuned = true;
                    dirty = true;
                }
            }
            // the device advanced every member; members that finished leave the tables
            bool any_done = false;
            for (auto& m : mem) any_done = any_done || m.it > m.last;
            if (any_done) retire();
            done_steps += n;
        }
        if (n_active) *n_active = (int)mem.size();
        return MFD_OK;
    }
};

static int validate_desc(const mfd_desc* d) {
    if (!d) { g_create_error = "null descriptor"; return MFD_ERR_INVALID; }
    if (d->abi_version != MFD_ABI_VERSION) { g_create_error = "ABI version mismatch"; return MFD_ERR_INVALID; }
    if (d->ndim < 1 || d->ndim > 3 || d->nx < 1 || d->ny < 1 || d->nz < 1 || d->nt < 1) { g_create_error = "bad dims"; return MFD_ERR_INVALID; }
    if (d->ndim == 1 && (d->nx != 1 || d->ny != 1)) { g_create_error = "1-D model needs nx = ny = 1"; return MFD_ERR_INVALID; }
    if (d->ndim == 2 && d->ny != 1) { g_create_error = "2-D model needs ny = 1"; return MFD_ERR_INVALID; }
    if (d->dtype != MFD_F32 && d->dtype != MFD_F64) { g_create_error = "bad dtype"; return MFD_ERR_INVALID; }
    if (d->mode != MFD_MODE_EXACT && d->mode != MFD_MODE_FAST) { g_create_error = "bad mode"; return MFD_ERR_INVALID; }
    if (d->polarization != MFD_POL_HY && (d->ndim != 2 || d->polarization != MFD_POL_EY)) {
        g_create_error = "polarization must be MFD_POL_HY, or MFD_POL_EY for a 2-D model"; return MFD_ERR_INVALID;
    }
    if (d->nmat < 0 || d->nmat > 255) { g_create_error = "at most 255 materials"; return MFD_ERR_INVALID; }
    if ((long long)d->nx * d->ny * d->nz > (1ll << 34)) { g_create_error = "grid too large"; return MFD_ERR_INVALID; }
    return MFD_OK;
}

extern "C" {

int mfd_abi_version(void) { return MFD_ABI_VERSION; }

}  // extern "C"

// mfd_create with the split updates' side streams on or off (the server's lanes run several
// models at once and leave them off: their streams would share the device's few hardware
// queues with every other lane's).
static int create_handle(const mfd_desc* desc, mfd_handle** out, bool overlap) {
    if (!out) return MFD_ERR_INVALID;
    *out = nullptr;
    int st = validate_desc(desc);
    if (st) return st;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        g_create_error = "no CUDA device";
        return MFD_ERR_NODEVICE;
    }
    if (desc->device < 0 || desc->device >= ndev) { g_create_error = "bad device ordinal"; return MFD_ERR_INVALID; }
    std::unique_ptr<mfd_handle> h(new mfd_handle);
    try {
        if (desc->dtype == MFD_F64) {
            auto e = std::make_unique<Engine<double, double>>();
            e->overlap = overlap;
            e->init(desc);
            h->impl = std::move(e);
        } else if (desc->rho_fp64) {
            auto e = std::make_unique<Engine<float, double>>();
            e->overlap = overlap;
            e->init(desc);
            h->impl = std::move(e);
        } else {
            auto e = std::make_unique<Engine<float, float>>();
            e->overlap = overlap;
            e->init(desc);
            h->impl = std::move(e);
        }
    } catch (const Error& e) {
        g_create_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_create_error = "out of host memory";
        return MFD_ERR_OOM;
    }
    *out = h.release();
    return MFD_OK;
}

extern "C" {

int mfd_create(const mfd_desc* desc, mfd_handle** out) { return create_handle(desc, out, true); }

void mfd_destroy(mfd_handle* h) { delete h; }

#define MFD_GUARD(h, expr)                                   \
    do {                                                     \
        if (!(h) || !(h)->impl) return MFD_ERR_INVALID;      \
        try {                                                \
            return (expr);                                   \
        } catch (const Error& e) {                           \
            (h)->impl->err = e.what();                       \
            return e.code;                                   \
        } catch (const std::bad_alloc&) {                    \
            (h)->impl->err = "out of host memory";           \
            return MFD_ERR_OOM;                              \
        }                                                    \
    } while (0)

int mfd_run(mfd_handle* h, int64_t a, int64_t b) { MFD_GUARD(h, h->impl->run(a, b)); }

#define MFD_BGUARD(b, expr)                                  \
    do {                                                     \
        if (!(b)) return MFD_ERR_INVALID;                    \
        try {                                                \
            return (expr);                                   \
        } catch (const Error& e) {                           \
            (b)->err = e.what();                             \
            return e.code;                                   \
        } catch (const std::bad_alloc&) {                    \
            (b)->err = "out of host memory";                 \
            return MFD_ERR_OOM;                              \
        }                                                    \
    } while (0)

int mfd_batch_create(int32_t device, mfd_batch** out) {
    if (!out) return MFD_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); g_create_error = "no CUDA device"; return MFD_ERR_NODEVICE; }
    if (device < 0 || device >= ndev) { g_create_error = "bad device ordinal"; return MFD_ERR_INVALID; }
    std::unique_ptr<mfd_batch> b(new mfd_batch);
    try {
        b->init(device);
    } catch (const Error& e) {
        g_create_error = e.what();
        return e.code;
    }
    *out = b.release();
    return MFD_OK;
}

void mfd_batch_destroy(mfd_batch* b) { delete b; }

int mfd_batch_add(mfd_batch* b, mfd_handle* h, int64_t it_last) { MFD_BGUARD(b, b->add(h, it_last)); }

int mfd_batch_run(mfd_batch* b, int64_t max_steps, int32_t* n_active) { MFD_BGUARD(b, b->run(max_steps, n_active)); }

int mfd_batch_config(mfd_batch* b, int32_t tile_x, int32_t tile_z, int32_t graph_steps) {
    if (!b) return MFD_ERR_INVALID;
    if (tile_x < 0 || tile_z < 0 || (tile_x > 0) != (tile_z > 0) || tile_x * tile_z > 512 || (tile_x && tile_x % 32) ||
        graph_steps < 0 || graph_steps > 4096) {
        b->err = "tile_x must be a multiple of 32 with tile_x * tile_z <= 512 (0, 0 = autotune); graph_steps in 1..4096 (0 = keep)";
        return MFD_ERR_INVALID;
    }
    b->tx = tile_x; b->tz = tile_z;
    b->tuned = false; b->tune_next = 0; b->tune_cost.clear();
    if (graph_steps) b->gsteps = graph_steps;
    b->dirty = true;
    return MFD_OK;
}

int mfd_batch_info(const mfd_batch* b, int32_t* tile_x, int32_t* tile_z, double* device_ms, int64_t* cell_updates,
                   int64_t* launches) {
    if (!b) return MFD_ERR_INVALID;
    if (tile_x) *tile_x = b->cur_tx;
    if (tile_z) *tile_z = b->cur_tz;
    if (device_ms) *device_ms = b->dev_ms;
    if (cell_updates) *cell_updates = b->cell_updates;
    if (launches) *launches = b->launches;
    return MFD_OK;
}

const char* mfd_batch_last_error(const mfd_batch* b) { return b ? b->err.c_str() : "null batch"; }
// A NULL host buffer is an argument error (MFD_ERR_INVALID), never a copy to address 0.
#define MFD_NEED_BUF(h, buf)                                           \
    do {                                                               \
        if (!(h) || !(h)->impl) return MFD_ERR_INVALID;                \
        if (!(buf)) {                                                  \
            (h)->impl->err = "null host buffer";                       \
            return MFD_ERR_INVALID;                                    \
        }                                                              \
    } while (0)

int mfd_read_field(mfd_handle* h, int32_t comp, void* dst) {
    MFD_NEED_BUF(h, dst);
    MFD_GUARD(h, h->impl->read_field(comp, dst));
}
int mfd_read_geometry(mfd_handle* h, uint8_t* dst) {
    MFD_NEED_BUF(h, dst);
    MFD_GUARD(h, h->impl->read_geometry(dst));
}
int mfd_write_field(mfd_handle* h, int32_t comp, const void* src) {
    MFD_NEED_BUF(h, src);
    MFD_GUARD(h, h->impl->write_field(comp, src));
}
int mfd_read_integral(mfd_handle* h, int32_t which, void* dst) {
    MFD_NEED_BUF(h, dst);
    MFD_GUARD(h, h->impl->read_integral(which, dst));
}
int mfd_read_integral_noalloc(mfd_handle* h, int32_t which, void* dst) {
    MFD_NEED_BUF(h, dst);
    MFD_GUARD(h, h->impl->read_integral_noalloc(which, dst));
}
int mfd_set_snapshots(mfd_handle* h, int32_t ncomp, const int32_t* comps, int64_t nsteps, const int64_t* steps, void* dst) {
    MFD_GUARD(h, h->impl->set_snapshots(ncomp, comps, nsteps, steps, dst));
}
int mfd_read_monitor(mfd_handle* h, int32_t m, int32_t comp, void* dst) {
    MFD_NEED_BUF(h, dst);
    MFD_GUARD(h, h->impl->read_monitor(m, comp, dst));
}
int mfd_read_tfsf_record(mfd_handle* h, int32_t k, void* dst) {
    MFD_NEED_BUF(h, dst);
    MFD_GUARD(h, h->impl->read_record(k, dst));
}

int64_t mfd_tfsf_record_size(const mfd_handle* h, int32_t k) {
    if (!h || !h->impl) return 0;
    return h->impl->record_size(k);
}

int mfd_status(const mfd_handle* h, int64_t* d, int64_t* b, int32_t* k) {
    if (!h || !h->impl) return MFD_ERR_INVALID;
    h->impl->status(d, b, k);
    return MFD_OK;
}

int mfd_set_profiling(mfd_handle* h, int32_t on) {
    if (!h || !h->impl) return MFD_ERR_INVALID;
    h->impl->set_profiling(on != 0);
    return MFD_OK;
}

int mfd_kernel_times(const mfd_handle* h, double* ms, int64_t* launches, int32_t n) {
    if (!h || !h->impl) return MFD_ERR_INVALID;
    return h->impl->kernel_times(ms, launches, n);
}

int mfd_last_run_ms(const mfd_handle* h, double* ms) {
    if (!h || !h->impl || !ms) return MFD_ERR_INVALID;
    *ms = h->impl->last_run_ms();
    return MFD_OK;
}

int64_t mfd_state_size(const mfd_handle* h) {
    if (!h || !h->impl) return 0;
    return h->impl->state_size();
}

int mfd_read_state(mfd_handle* h, void* dst, int64_t bytes) {
    MFD_NEED_BUF(h, dst);
    MFD_GUARD(h, h->impl->read_state(dst, bytes));
}

int mfd_write_state(mfd_handle* h, const void* src, int64_t bytes) {
    MFD_NEED_BUF(h, src);
    MFD_GUARD(h, h->impl->write_state(src, bytes));
}

int64_t mfd_device_bytes(const mfd_handle* h) {
    if (!h || !h->impl) return 0;
    return h->impl->device_bytes();
}

const char* mfd_last_error(const mfd_handle* h) {
    if (!h || !h->impl) return "invalid handle";
    return h->impl->err.c_str();
}

const char* mfd_create_error(void) { return g_create_error.c_str(); }

}  // extern "C"

#include "serve.cuh"
