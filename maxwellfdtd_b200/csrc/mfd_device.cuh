// mfd_device.cuh -- device-side data layout and per-cell physics of the B200 FDTD stepper.
//
// HBM layout (one handle):
//  * every grid array (9 field components, Sa, E2, the uint8 material map) is x-fastest with
//    the x row padded to a pitch px (a multiple of 32 elements) so rows start on 128-byte
//    (float) / 256-byte (double) boundaries: cell (ix,iy,iz) -> ix + px*(iy + ny*iz);
//  * CPML psi arrays exist only inside their slabs: x faces [iz][iy][p] (p < nb), y faces
//    [iz][p][ix], z faces [p][iy][ix] (pitch px);
//  * polarisation / plasma state exists only inside the bounding box of each material's
//    cells, x-fastest, with two ping-pong buffers per recursion instead of the reference's
//    three dense arrays P, oldP1, oldP2 (materials.jl:424-426):
//      P^{n+1} = Aq P^n + Bq P^{n-1} + Cq E^n  is written over P^{n-1}.
//
// The arithmetic of every cell update follows the reference kernels operation by operation
// (src/models.jl) with the same operand types; kernels are compiled with --fmad=false so no
// a*b+c is fused, as Julia does not fuse either.
#pragma once

#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

#include "../../include/maxwellfdtd.h"

#define MFD_MAXQ 16

namespace mfd {

template <typename T> struct Eps;
template <> struct Eps<float> { static __device__ __forceinline__ float v() { return FLT_EPSILON; } };
template <> struct Eps<double> { static __device__ __forceinline__ double v() { return DBL_EPSILON; } };

struct Layout {
    int nx, ny, nz;
    int px;            // x pitch (elements)
    int sz;            // px*ny (z-plane stride); padded grids stay below 2^31 cells
};

// Division by a positive grid constant (dx, dy, dz, CPML kappa).
//
// The reference divides by these constants in every cell (models.jl:803-808, 968-973,
// 819-820 ...).  An IEEE division costs a long instruction sequence, and a much longer one
// for the zero or tiny numerators that fill most of a grid early in a run.  For a constant
// divisor d the library uses Markstein's correction step (P. W. Markstein, "Computation of
// elementary functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990):
//     r = RN(1/d),  q0 = RN(x r),  e = RN(x - q0 d) (fma),  q = RN(q0 + e r) (fma).
// Scaling x by 2^k scales q0, e and q by 2^k exactly while all of them stay normal, so the
// result equals RN(x/d) for every x in the band [lo, hi] (where they do) as soon as it does
// for every significand of one binade.  The engine checks exactly that on the device, for
// each divisor, against IEEE division over all 2^23 significands in [1, 2), and over the
// band's lowest and highest binades, before the first step; a divisor that fails (or any
// double-precision divisor) keeps IEEE division (ok = 0), as do numerators outside the band.
// Kernels take FAST = true only when every divisor of the model passed the check; the
// band test is one unsigned compare on the bit pattern (lob = bits(lo), span = bits(hi) -
// bits(lo)).  A zero numerator returns x (0/d keeps the sign of x since d > 0).
template <typename T>
struct DivC {
    T d, r;          // divisor and its correctly rounded reciprocal
    T lo, hi;        // |x| band in which the correction step is exact
    unsigned lob, span;
    int ok;          // verified for every significand
};

// Division mode of a kernel (its FAST template parameter):
//   DIV_IEEE  -- IEEE division (double precision, or a divisor that failed the check);
//   DIV_EXACT -- the verified correction step above, bit-identical to IEEE division;
//   DIV_RECIP -- the tolerance mode: x * RN(1/d) (within an ulp of x/d), and the update
//                expressions fused into multiply-adds (mad below) and the Poynting norm
//                by the hardware reciprocal square root.  Results are no longer
//                bit-identical to the reference's operation order; they stay within the
//                relative L2 tolerance stated for the model's precision.
enum { DIV_IEEE = 0, DIV_EXACT = 1, DIV_RECIP = 2 };

template <int FAST, typename T>
__device__ __forceinline__ T cdiv(T x, const DivC<T>& D) {
    if constexpr (FAST == DIV_RECIP) return x * D.r;
    else return x / D.d;
}

// a * b + c: one fused multiply-add in the tolerance mode, else the product rounded and then
// the sum rounded, as the reference computes it (the library is built without contraction).
template <int FAST, typename T>
__device__ __forceinline__ T mad(T a, T b, T c) {
    if constexpr (FAST == DIV_RECIP) return fma(a, b, c);
    else return a * b + c;
}

__device__ __forceinline__ float qscaled(float x, float d, float r, unsigned lob1, unsigned hib);

template <>
__device__ __forceinline__ float cdiv<DIV_EXACT, float>(float x, const DivC<float>& D) {
    const unsigned ax = __float_as_uint(x) & 0x7fffffffu;
    if (ax - D.lob <= D.span) {
        const float q0 = __fmul_rn(x, D.r);
        const float e = __fmaf_rn(-q0, D.d, x);
        return __fmaf_rn(e, D.r, q0);
    }
    if (ax == 0u) return x;
    return qscaled(x, D.d, D.r, D.lob - 1u, D.lob + D.span);
}

// The six curl derivatives of a cell divide by the three grid constants.  Div3 holds the
// three divisors and reciprocals and the band common to the three (lob1 = bits(lo) - 1,
// hib = bits(hi)), so one integer min/max reduction checks all six numerators: a nonzero
// |x| outside the band, or an unverified divisor, takes the IEEE division in one rarely
// taken branch.  copysign(q, x) makes zero numerators exact too (q = RN(x/d) has the sign
// of x since d > 0).
struct Div3 {
    float dx, dy, dz, rx, ry, rz;
    unsigned lob1, hib;
};

__device__ __forceinline__ float qcorr(float x, float d, float r) {
    const float q0 = __fmul_rn(x, r);
    const float e = __fmaf_rn(-q0, d, x);
    return copysignf(__fmaf_rn(e, r, q0), x);
}

// q[i] = RN(x[i] / d[i]) for the six derivatives, d = (dy, dz, dx, dz, dx, dy) in the order
// (x-y, x-z, y-x, y-z, z-x, z-y) of the curl.
// RN(x/d) for a numerator outside the band.  A normal x below the band is scaled by 2^32
// into it (exact), divided by the correction step, and scaled back (exact while the
// quotient stays normal, |q| >= 2^-126); anything else takes the IEEE division.  lob1 and
// hib bound the band's bit patterns as in Div3.
__device__ __forceinline__ float qscaled(float x, float d, float r, unsigned lob1, unsigned hib) {
    const unsigned ax = __float_as_uint(x) & 0x7fffffffu;
    if (ax >= 0x00800000u && ax - 1u < lob1) {
        const float xs = x * 0x1p32f;
        const unsigned axs = __float_as_uint(xs) & 0x7fffffffu;
        if (axs - 1u >= lob1 && axs <= hib) {
            const float qs = qcorr(xs, d, r);
            if (fabsf(qs) >= 0x1p-94f) return qs * 0x1p-32f;
        }
    }
    return __fdiv_rn(x, d);
}

template <int FAST>
__device__ __forceinline__ void div6(const Div3& D, const float (&x)[6], float (&q)[6]) {
    const float d[6] = {D.dy, D.dz, D.dx, D.dz, D.dx, D.dy};
    if constexpr (FAST == DIV_RECIP) {
        const float r[6] = {D.ry, D.rz, D.rx, D.rz, D.rx, D.ry};
#pragma unroll
        for (int i = 0; i < 6; ++i) q[i] = x[i] * r[i];
    } else if constexpr (FAST == DIV_EXACT) {
        const float r[6] = {D.ry, D.rz, D.rx, D.rz, D.rx, D.ry};
        unsigned mn = 0xffffffffu, mx = 0u;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            q[i] = qcorr(x[i], d[i], r[i]);
            const unsigned ax = __float_as_uint(x[i]) & 0x7fffffffu;
            mn = min(mn, ax - 1u);   // zero wraps to the maximum: excluded from the lower bound
            mx = max(mx, ax);
        }
        if (mn >= D.lob1 && mx <= D.hib) return;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            const unsigned ax = __float_as_uint(x[i]) & 0x7fffffffu;
            if (ax != 0u && (ax - 1u < D.lob1 || ax > D.hib)) q[i] = qscaled(x[i], d[i], r[i], D.lob1, D.hib);
        }
    } else {
#pragma unroll
        for (int i = 0; i < 6; ++i) q[i] = __fdiv_rn(x[i], d[i]);
    }
}

// sqrt of a sum of squares; zero (most cells early in a run) skips the special-case path.
template <typename T>
__device__ __forceinline__ T sqrt0(T v) {
    return v == T(0) ? T(0) : sqrt(v);
}

// The same in a kernel's division mode: the tolerance mode takes v * rsqrt(v) in single
// precision (the hardware reciprocal square root, a few ulp) instead of the correctly
// rounded square root's longer sequence.
template <int FAST, typename T>
__device__ __forceinline__ T sqrtm(T v) {
    if constexpr (FAST == DIV_RECIP && sizeof(T) == 4) return v > T(0) ? v * rsqrtf(v) : T(0);
    else return sqrt0(v);
}

// |a|^2 + |b|^2 + |c|^2 of the Poynting vector in the reference's order (a^2 + b^2) + c^2,
// fused in the tolerance mode.
template <int FAST, typename T>
__device__ __forceinline__ T sum3sq(T a, T b, T c) {
    return mad<FAST>(c, c, mad<FAST>(a, a, b * b));
}

template <typename T>
struct LayerDev {
    int ib, nb;        // 1-based boundary index, points in layer (0 = none)
    const DivC<T>* K;  // kappa as a divisor
    const T* A;
    const T* B;
    T* psi[4];         // 3-D: x faces Hyx,Hzx,Eyx,Ezx; y: Hxy,Hzy,Exy,Ezy; z: Hxz,Hyz,Exz,Eyz
                       // 2-D: x faces Hyx,Ezx; z faces Hyz,Exz.  1-D: z faces Hyz,Exz.
};

// Material coefficients + pointers to its compact state (materials.jl:335-483).
template <typename T, typename R>
struct MatDev {
    T Mh, Me, Md1, Md2;
    int nq, kerr, plasma, rate_kind;
    T Aq[MFD_MAXQ], Bq[MFD_MAXQ], Cq[MFD_MAXQ];
    T Mk2, Mk3;
    T Rava, ksi, rho0, Ap, Bp, Cp, Ma;
    T rate_order;
    double rate_log10c;
    int rate_n;
    const T* rate_x;
    const T* rate_y;
    int simple;                         // no poles, plasma or Kerr: E = D Me in the stencil
    int bx0, by0, bz0, bnx, bny, bnz;   // bounding box of the material's cells
    long long bsize;
    T* P;       // [2][nq][nc][bsize]
    T* Pp;      // [2][nc][bsize]
    T* Pa;      // [nc][bsize]
    R* rho;     // [bsize]
    R* drho;    // [bsize]
    T* JE;      // [bsize]
};

// Neighbour value across a grid face (models.jl:755-808, 920-973): periodic wraps,
// Dirichlet is zero, Neumann repeats the cell's own value.
template <typename T>
__device__ __forceinline__ T bc_value(int bc, T wrapped, T self) {
    return bc == MFD_BC_PERIODIC ? wrapped : (bc == MFD_BC_DIRICHLET ? T(0) : self);
}

// IonizationRate functor in T precision (IonizationRate.jl:42-52).
template <typename T>
__device__ __forceinline__ T rate_table(const T* __restrict__ X, const T* __restrict__ Y, int n, T x) {
    if (x <= T(0)) return T(0);
    T xi = log10(x);
    int i;
    if (xi <= X[0]) i = 0;
    else if (xi >= X[n - 1]) i = n - 2;
    else {
        int lo = 0, hi = n - 1;     // first j with X[j] >= xi, then i = j - 1
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (X[mid] < xi) lo = mid + 1; else hi = mid;
        }
        i = lo - 1;
    }
    T dydx = (Y[i + 1] - Y[i]) / (X[i + 1] - X[i]);
    T yl = Y[i] + dydx * (xi - X[i]);
    return pow(T(10), yl);
}

template <typename T, typename R, typename Q>
__device__ __forceinline__ void plasma_density(R& rho, R& drho, Q R1, T R2, T dt) {
    // models.jl:1116-1125: exact integration of drho/dt = R1 (1 - rho) - R2 rho over dt
    R r = rho;
    if (R2 == T(0)) {
        r = 1 - (1 - r) * exp(-R1 * dt);
    } else {
        auto R12 = R1 - R2;
        r = R1 / R12 * 1 - (R1 / R12 * 1 - r) * exp(-R12 * dt);
    }
    rho = r;
    drho = R1 * (1 - r);
}

// Material response of one cell after its D update: ADE poles, plasma, Kerr, E from D
// (models.jl:1042-1154; 2-D 622-712; 1-D 365-431).  NC field components; E[k] points to
// the k-th E component (x, [y,] z order), Dv[k] the updated D values.
template <typename T, typename R, int NC>
__device__ __forceinline__ void material_cell(const MatDev<T, R>* __restrict__ m, int ix, int iy, int iz,
                                              T* const* E, long long c, const T* Dv, int cur, T dt) {
    const T Me = m->Me;
    T sumP[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) sumP[k] = T(0);
    const int nq = m->nq;
    const bool plasma = m->plasma != 0;
    T En[NC];
    long long bi = 0;
    if (nq > 0 || plasma) {
#pragma unroll
        for (int k = 0; k < NC; ++k) En[k] = E[k][c];
        bi = (long long)(ix - m->bx0) + (long long)m->bnx * ((long long)(iy - m->by0) + (long long)m->bny * (iz - m->bz0));
    }
    const long long bs = m->bsize;
    for (int q = 0; q < nq; ++q) {
        const T Aq = m->Aq[q], Bq = m->Bq[q], Cq = m->Cq[q];
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            T* Pc = m->P + ((long long)(cur * nq + q) * NC + k) * bs;
            T* Po = m->P + ((long long)((1 - cur) * nq + q) * NC + k) * bs;
            T pn = Pc[bi], pm = Po[bi];
            T pnew = Aq * pn + Bq * pm + Cq * En[k];
            Po[bi] = pnew;
            sumP[k] += pnew;
        }
    }
    if (plasma) {
        T E2 = En[0] * En[0];
#pragma unroll
        for (int k = 1; k < NC; ++k) E2 = E2 + En[k] * En[k];
        T II = m->ksi * E2;
        R rho = m->rho[bi];
        R drho = m->drho[bi];
        T Ppn[NC], Ppm[NC], Ppnew[NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            T* Pc = m->Pp + ((long long)cur * NC + k) * bs;
            T* Po = m->Pp + ((long long)(1 - cur) * NC + k) * bs;
            Ppn[k] = Pc[bi];
            Ppm[k] = Po[bi];
            Ppnew[k] = m->Ap * Ppn[k] + m->Bp * Ppm[k] + m->Cp * rho * m->rho0 * En[k];
            Po[bi] = Ppnew[k];
        }
#pragma unroll
        for (int k = 0; k < NC; ++k) sumP[k] += Ppnew[k];
        T invE2 = (E2 >= Eps<T>::v()) ? T(1) / E2 : T(0);
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            T* pa = m->Pa + (long long)k * bs;
            T v = pa[bi] + m->Ma * drho * m->rho0 * En[k] * invE2;
            pa[bi] = v;
            sumP[k] += v;
        }
        if (m->rate_kind == MFD_RATE_TABLE) {
            T R1 = rate_table<T>(m->rate_x, m->rate_y, m->rate_n, II);
            plasma_density<T, R, T>(rho, drho, R1, m->Rava * E2, dt);
        } else if (m->rate_kind == MFD_RATE_POWER) {
            T lg = log10(II);
            T a = m->rate_order * lg;
            double R1 = pow(10.0, (double)a + m->rate_log10c);
            plasma_density<T, R, double>(rho, drho, R1, m->Rava * E2, dt);
        } else {
            plasma_density<T, R, T>(rho, drho, T(0), m->Rava * E2, dt);
        }
        m->rho[bi] = rho;
        m->drho[bi] = drho;
        T acc = (Ppnew[0] - Ppm[0]) / (2 * dt) * En[0];
#pragma unroll
        for (int k = 1; k < NC; ++k) acc = acc + (Ppnew[k] - Ppm[k]) / (2 * dt) * En[k];
        m->JE[bi] = m->JE[bi] + acc * dt;
    }
    if (m->kerr) {
        const T Mk2 = m->Mk2, Mk3 = m->Mk3;
        const T Me2 = Me * Me, Me3 = Me * Me * Me;
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            T X = Dv[k] - sumP[k];
            T X2 = X * X;
            // Kerr by Meep (models.jl:1143-1149)
            E[k][c] = (1 + 1 * Mk2 * Me2 * X + 2 * Mk3 * Me3 * X2) /
                      (1 + 2 * Mk2 * Me2 * X + 3 * Mk3 * Me3 * X2) * X * Me;
        }
    } else {
#pragma unroll
        for (int k = 0; k < NC; ++k) E[k][c] = (Dv[k] - sumP[k]) * Me;
    }
}

// material_cell with the number of poles NQ known at compile time: every load of the cell
// (E^n, both polarisation buffers of every pole, the plasma state) is issued before any
// store, so the poles do not become dependent round trips to memory.  The arithmetic is
// material_cell's, expression for expression.  bi is the cell's index in the material's box.
template <typename T, typename R, int NC, int NQ>
__device__ __forceinline__ void material_cell_n(const MatDev<T, R>* __restrict__ m, long long bi,
                                                T* const* E, long long c, const T* Dv, int cur, T dt) {
    const T Me = m->Me;
    const bool plasma = m->plasma != 0;
    const long long bs = m->bsize;
    T sumP[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) sumP[k] = T(0);
    T En[NC];
    if (NQ > 0 || plasma) {
#pragma unroll
        for (int k = 0; k < NC; ++k) En[k] = E[k][c];
    }
    constexpr int NQ1 = NQ > 0 ? NQ : 1;
    T pn[NQ1][NC], pm[NQ1][NC];
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            pn[q][k] = m->P[((long long)(cur * NQ + q) * NC + k) * bs + bi];
            pm[q][k] = m->P[((long long)((1 - cur) * NQ + q) * NC + k) * bs + bi];
        }
    R rho = R(0), drho = R(0);
    T Ppn[NC], Ppm[NC], Pav[NC], JEv = T(0);
    if (plasma) {
        rho = m->rho[bi];
        drho = m->drho[bi];
        JEv = m->JE[bi];
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            Ppn[k] = m->Pp[((long long)cur * NC + k) * bs + bi];
            Ppm[k] = m->Pp[((long long)(1 - cur) * NC + k) * bs + bi];
            Pav[k] = m->Pa[(long long)k * bs + bi];
        }
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        const T Aq = m->Aq[q], Bq = m->Bq[q], Cq = m->Cq[q];
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            const T pnew = Aq * pn[q][k] + Bq * pm[q][k] + Cq * En[k];
            m->P[((long long)((1 - cur) * NQ + q) * NC + k) * bs + bi] = pnew;
            sumP[k] += pnew;
        }
    }
    if (plasma) {
        T E2 = En[0] * En[0];
#pragma unroll
        for (int k = 1; k < NC; ++k) E2 = E2 + En[k] * En[k];
        T II = m->ksi * E2;
        T Ppnew[NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            Ppnew[k] = m->Ap * Ppn[k] + m->Bp * Ppm[k] + m->Cp * rho * m->rho0 * En[k];
            m->Pp[((long long)(1 - cur) * NC + k) * bs + bi] = Ppnew[k];
        }
#pragma unroll
        for (int k = 0; k < NC; ++k) sumP[k] += Ppnew[k];
        T invE2 = (E2 >= Eps<T>::v()) ? T(1) / E2 : T(0);
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            T v = Pav[k] + m->Ma * drho * m->rho0 * En[k] * invE2;
            m->Pa[(long long)k * bs + bi] = v;
            sumP[k] += v;
        }
        if (m->rate_kind == MFD_RATE_TABLE) {
            T R1 = rate_table<T>(m->rate_x, m->rate_y, m->rate_n, II);
            plasma_density<T, R, T>(rho, drho, R1, m->Rava * E2, dt);
        } else if (m->rate_kind == MFD_RATE_POWER) {
            T lg = log10(II);
            T a = m->rate_order * lg;
            double R1 = pow(10.0, (double)a + m->rate_log10c);
            plasma_density<T, R, double>(rho, drho, R1, m->Rava * E2, dt);
        } else {
            plasma_density<T, R, T>(rho, drho, T(0), m->Rava * E2, dt);
        }
        m->rho[bi] = rho;
        m->drho[bi] = drho;
        T acc = (Ppnew[0] - Ppm[0]) / (2 * dt) * En[0];
#pragma unroll
        for (int k = 1; k < NC; ++k) acc = acc + (Ppnew[k] - Ppm[k]) / (2 * dt) * En[k];
        m->JE[bi] = JEv + acc * dt;
    }
    if (m->kerr) {
        const T Mk2 = m->Mk2, Mk3 = m->Mk3;
        const T Me2 = Me * Me, Me3 = Me * Me * Me;
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            T X = Dv[k] - sumP[k];
            T X2 = X * X;
            E[k][c] = (1 + 1 * Mk2 * Me2 * X + 2 * Mk3 * Me3 * X2) /
                      (1 + 2 * Mk2 * Me2 * X + 3 * Mk3 * Me3 * X2) * X * Me;
        }
    } else {
#pragma unroll
        for (int k = 0; k < NC; ++k) E[k][c] = (Dv[k] - sumP[k]) * Me;
    }
}

}  // namespace mfd
