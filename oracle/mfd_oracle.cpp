// mfd_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the MaxwellFDTD time-step path (Julia package iamfedoroff/MaxwellFDTD),
// used as the parity oracle for the CUDA library and as the timed CPU baseline.  It is
// never linked into or called by the product library.  Only tests/, __graft_entry__.smoke()
// and the cpu_baseline / reference leg of bench.py load it.
//
// It follows the reference's CPU backend (KernelAbstractions kernels run on Julia threads)
// statement by statement: dense full-grid arrays, Int64 material map, psi arrays in the
// reference's shapes, dense P/oldP1/oldP2 polarisation arrays, the same per-step order and
// the same operation order inside every cell update.  C++ float/double arithmetic follows
// the same promotion rules as Julia for Float32/Float64 operands, so each expression is
// written with the operand types the reference has after adapt() (src/backends.jl:27-41).
// Build with -ffp-contract=off: Julia does not fuse a*b+c into an FMA.
//
// Pinned against the reference's own known-answer tests (test/*.jl), restated in
// tests/test_oracle_reference.py.  Paths no reference test covers (TFSF, Debye, Drude,
// Kerr, plasma, kmax != 1, Dirichlet/Neumann BCs, monitors) match the restatement only.
//
// Citations are file:line in the reference project.
#include "../include/maxwellfdtd.h"

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double EPS0 = 8.8541878128e-12;   // CODATA 2018, src/MaxwellFDTD.jl:19
constexpr double MU0 = 1.25663706212e-6;    // CODATA 2018, src/MaxwellFDTD.jl:20

thread_local std::string g_create_error;

struct OracleBase {
    std::string err;
    virtual ~OracleBase() = default;
    virtual int run(int64_t a, int64_t b) = 0;
    virtual int read_field(int comp, void* dst) = 0;
    virtual int read_geometry(uint8_t* dst) = 0;
    virtual int write_field(int comp, const void* src) = 0;
    virtual int read_integral(int which, void* dst) = 0;
    virtual int read_monitor(int m, int comp, void* dst) = 0;
    virtual int read_record(int k, void* dst) = 0;
    virtual int64_t record_size(int k) const = 0;
    virtual void status(int64_t* done, int64_t* bad, int32_t* kind) const = 0;
};

// IonizationRate functor in T precision (examples/5_nonlinear_propagation/IonizationRate.jl:
// 30-52): 0 for x <= 0, else 10^linterp(log10(x)) on the table's log10 knots X (even
// spacing, increasing) and log10 rates Y; linterp takes the first segment below X[0], the
// last above X[n-1], and otherwise segment searchsortedfirst(X, xi) - 1.
template <typename T>
T ionization_rate(const T* X, const T* Y, size_t n, T x) {
    if (x <= 0) return 0;
    T xi = std::log10(x);
    size_t i;
    if (xi <= X[0]) i = 0;
    else if (xi >= X[n - 1]) i = n - 2;
    else {
        size_t j = 0;   // searchsortedfirst(x, xi) - 1 (0-based: first j with X[j] >= xi, minus 1)
        while (X[j] < xi) ++j;
        i = j - 1;
    }
    T dydx = (Y[i + 1] - Y[i]) / (X[i + 1] - X[i]);
    T yl = Y[i] + dydx * (xi - X[i]);
    return std::pow((T)10, yl);
}

// An analytic shape covers (x, y, z): the header's double-precision test for its kind,
// left to right (the host restatement of the geometry closures of util.jl:1-31 for the
// shapes include/maxwellfdtd.h defines).
bool shape_covers(const mfd_shape& s, double x, double y, double z) {
    const double* p = s.p;
    switch (s.kind) {
        case MFD_SHAPE_BALL: {
            const double a = x - p[0], b = y - p[1], c = z - p[2];
            return (a * a + b * b) + c * c <= p[3] * p[3];
        }
        case MFD_SHAPE_BOX: return p[0] <= x && x <= p[1] && p[2] <= y && y <= p[3] && p[4] <= z && z <= p[5];
        case MFD_SHAPE_ELLIPSOID: {
            const double a = (x - p[0]) / p[3], b = (y - p[1]) / p[4], c = (z - p[2]) / p[5];
            return (a * a + b * b) + c * c <= 1.0;
        }
        case MFD_SHAPE_CYLINDER: {
            const double a = x - p[0], b = y - p[1];
            return a * a + b * b <= p[2] * p[2] && p[3] <= z && z <= p[4];
        }
        case MFD_SHAPE_HALFSPACE: return (p[0] * x + p[1] * y) + p[2] * z >= p[3];
        case MFD_SHAPE_ALL: return true;
        default: return false;
    }
}

// Layer profile (src/pml.jl:46-52).  0-based: a left layer covers cells [0, ib-1] with pml
// index ix; a right layer covers [ib-1, n-1] with pml index ix-(ib-1).
template <typename T>
struct Layer {
    int ib = 0, nb = 0;
    std::vector<T> K, A, B;
};

// MaterialStruct3D (src/materials.jl:335-483) with dense state arrays.
template <typename T, typename R>
struct Mat {
    T Mh, Me, Md1, Md2;
    bool disp = false;
    int nq = 0;
    std::vector<T> Aq, Bq, Cq;
    std::vector<T> P[3], oldP1[3], oldP2[3];   // (Nq, N) per component x,y,z
    bool kerr = false;
    T Mk2 = 0, Mk3 = 0;
    bool plasma = false;
    T Rava = 0, ksi = 0, rho0 = 0, Ap = 0, Bp = 0, Cp = 0, Ma = 0;
    int rate_kind = 0;
    T rate_order = 0;
    double rate_log10c = 0;
    std::vector<T> rate_x, rate_y;
    std::vector<R> rho, drho;
    std::vector<T> Pp[3], oldPp1[3], oldPp2[3], Pa[3];
};

template <typename T>
struct Source {
    int kind, comp;
    T coeff;
    std::vector<int64_t> cells;
    std::vector<double> wave, amp, gt;
};

template <typename T>
struct Monitor {
    int kind, sum;
    std::vector<int64_t> cells;
    int nw = 0;
    std::vector<double> phasor;                  // [nt][nw][2]
    std::vector<T> rec[9];                       // field monitor [nt][npts] or [nt]
    std::vector<std::complex<double>> S[9];      // spectral [nw][npts] or [nw]
};

template <typename T, typename R>
struct Oracle : OracleBase {
    int ndim, nx, ny, nz;
    int pol = MFD_POL_HY;   // the 2-D field set (include/maxwellfdtd.h)
    size_t N;
    T dx, dy, dz, dt;
    int64_t nt;
    int bc[6];
    Layer<T> L[6];
    T Mh0, Me0, Md10, Md20;
    std::vector<int64_t> geometry;
    bool isgeometry = false, isplasma = false;
    std::vector<Mat<T, R>> mats;
    std::vector<T> F[9];
    // psi arrays in the reference's shapes (src/pml.jl:133-304).
    // 3-D: x faces (Nb,Ny,Nz): Hyx,Hzx,Eyx,Ezx; y faces (Nx,Nb,Nz): Hxy,Hzy,Exy,Ezy;
    //      z faces (Nx,Ny,Nb): Hxz,Hyz,Exz,Eyz.  2-D: x faces (Nb,Nz): Hyx,Ezx;
    //      z faces (Nx,Nb): Hyz,Exz (second 2-D field set: Hzx,Eyx and Hxz,Eyz).
    //      1-D: z faces (Nb): Hyz,Exz.
    std::vector<T> psi[6][4];
    std::vector<T> JE, Sa, E2;
    std::vector<Source<T>> srcs;
    bool tfsf = false;
    int tfsf_order = 0;
    int ti1[3], ti2[3];
    std::vector<T> inc[24];
    size_t inc_len[24];
    std::vector<Monitor<T>> mons;
    bool record = false;
    int ri1[3], ri2[3];
    std::vector<T> rec[24];
    size_t rec_len[24];
    int64_t done = 0, bad_step = 0;
    int32_t bad_kind = 0;

    size_t id(int ix, int iy, int iz) const { return (size_t)ix + (size_t)nx * ((size_t)iy + (size_t)ny * (size_t)iz); }

    int init(const mfd_desc* d) {
        ndim = d->ndim; nx = d->nx; ny = d->ny; nz = d->nz;
        pol = ndim == 2 ? d->polarization : MFD_POL_HY;
        N = (size_t)nx * ny * nz;
        dx = (T)d->dx; dy = (T)d->dy; dz = (T)d->dz; dt = (T)d->dt;
        nt = d->nt;
        for (int f = 0; f < 6; ++f) {
            bc[f] = d->bc[f];
            L[f].ib = d->pml[f].ib; L[f].nb = d->pml[f].nb;
            for (int i = 0; i < L[f].nb; ++i) {
                L[f].K.push_back((T)d->pml[f].K[i]);
                L[f].A.push_back((T)d->pml[f].A[i]);
                L[f].B.push_back((T)d->pml[f].B[i]);
            }
        }
        Mh0 = (T)d->Mh0; Me0 = (T)d->Me0; Md10 = (T)d->Md10; Md20 = (T)d->Md20;
        geometry.assign(N, 0);
        if (d->geometry)
            for (size_t i = 0; i < N; ++i) {
                geometry[i] = d->geometry[i];
                if (geometry[i] > d->nmat) { err = "geometry index beyond nmat"; return MFD_ERR_INVALID; }
                if (geometry[i] > 0) isgeometry = true;
            }
        else if (d->nshape > 0) {   // the material map from analytic shapes (the reference's geometry2bool, util.jl:1-31)
            for (int iz = 0; iz < nz; ++iz)
                for (int iy = 0; iy < ny; ++iy)
                    for (int ix = 0; ix < nx; ++ix) {
                        const double x = ndim >= 2 ? d->coords[0][ix] : 0.0, y = ndim == 3 ? d->coords[1][iy] : 0.0;
                        const double z = d->coords[2][iz];
                        int g = 0;
                        for (int k = 0; k < d->nshape; ++k)
                            if (shape_covers(d->shapes[k], x, y, z)) g = d->shapes[k].material;
                        geometry[id(ix, iy, iz)] = g;
                        if (g > 0) isgeometry = true;
                    }
        }
        for (int m = 0; m < d->nmat; ++m) {
            const mfd_material& s = d->mats[m];
            Mat<T, R> M;
            M.Mh = (T)s.Mh; M.Me = (T)s.Me; M.Md1 = (T)s.Md1; M.Md2 = (T)s.Md2;
            M.nq = s.nq; M.disp = s.nq > 0;
            for (int q = 0; q < s.nq; ++q) {
                M.Aq.push_back((T)s.Aq[q]); M.Bq.push_back((T)s.Bq[q]); M.Cq.push_back((T)s.Cq[q]);
            }
            if (M.disp)
                for (int c = 0; c < 3; ++c) {
                    M.P[c].assign((size_t)M.nq * N, 0);
                    M.oldP1[c].assign((size_t)M.nq * N, 0);
                    M.oldP2[c].assign((size_t)M.nq * N, 0);
                }
            M.kerr = s.kerr != 0; M.Mk2 = (T)s.Mk2; M.Mk3 = (T)s.Mk3;
            M.plasma = s.plasma != 0;
            if (M.plasma) {
                isplasma = true;
                M.Rava = (T)s.Rava; M.ksi = (T)s.ksi; M.rho0 = (T)s.rho0;
                M.Ap = (T)s.Ap; M.Bp = (T)s.Bp; M.Cp = (T)s.Cp; M.Ma = (T)s.Ma;
                M.rate_kind = s.rate_kind;
                M.rate_order = (T)s.rate_order; M.rate_log10c = s.rate_log10c;
                if (s.rate_kind == MFD_RATE_TABLE) {
                    if (s.rate_n < 2) { err = "rate table needs >= 2 knots"; return MFD_ERR_INVALID; }
                    for (int i = 0; i < s.rate_n; ++i) {
                        M.rate_x.push_back((T)s.rate_x[i]); M.rate_y.push_back((T)s.rate_y[i]);
                    }
                }
                M.rho.assign(N, 0); M.drho.assign(N, 0);
                for (int c = 0; c < 3; ++c) {
                    M.Pp[c].assign(N, 0); M.oldPp1[c].assign(N, 0); M.oldPp2[c].assign(N, 0);
                    M.Pa[c].assign(N, 0);
                }
            }
            mats.push_back(std::move(M));
        }
        for (int c = 0; c < 9; ++c) F[c].assign(N, 0);
        // psi arrays
        for (int f = 0; f < 6; ++f) {
            size_t nb = L[f].nb, n = 0;
            int axis = f / 2;
            if (ndim == 3) n = axis == 0 ? nb * ny * nz : axis == 1 ? nx * nb * nz : nx * ny * nb;
            else if (ndim == 2) n = axis == 0 ? nb * nz : axis == 2 ? nx * nb : 0;
            else n = axis == 2 ? nb : 0;
            for (int k = 0; k < 4; ++k) psi[f][k].assign(n, 0);
        }
        if (isplasma) JE.assign(N, 0);
        Sa.assign(N, 0);
        if (isgeometry) E2.assign(N, 0);
        for (int s = 0; s < d->nsrc; ++s) {
            const mfd_source& a = d->srcs[s];
            Source<T> S;
            S.kind = a.kind; S.comp = a.comp; S.coeff = (T)a.coeff;
            S.cells.assign(a.cells, a.cells + a.npts);
            for (auto c : S.cells) if (c < 0 || (size_t)c >= N) { err = "source cell out of range"; return MFD_ERR_INVALID; }
            if (a.wave) S.wave.assign(a.wave, a.wave + (size_t)nt * a.npts);
            else { S.amp.assign(a.amp, a.amp + a.npts); S.gt.assign(a.gt, a.gt + nt); }
            srcs.push_back(std::move(S));
        }
        tfsf = d->tfsf.enabled != 0;
        if (tfsf) {
            tfsf_order = d->tfsf.order;
            for (int a = 0; a < 3; ++a) { ti1[a] = d->tfsf.i1[a]; ti2[a] = d->tfsf.i2[a]; }
            int narr = ndim == 3 ? 24 : ndim == 2 ? 8 : 4;
            for (int k = 0; k < narr; ++k) {
                inc_len[k] = face_len(k, ti1, ti2);
                const T* p = (const T*)d->tfsf.inc[k];
                const int sh = d->tfsf.shape[k];
                if (sh == MFD_INC_FULL) {
                    inc[k].assign(p, p + inc_len[k] * nt);
                    continue;
                }
                // compact layouts (maxwellfdtd.h): expand to the reference's [nt][b][a]
                const size_t na = face_a(k, ti1, ti2), nb = inc_len[k] / na;
                const size_t per = sh == MFD_INC_ALONG_B ? nb : sh == MFD_INC_ALONG_A ? na : 1;
                inc[k].assign(inc_len[k] * nt, 0);
                for (int64_t it = 0; it < nt; ++it)
                    for (size_t ib = 0; ib < nb; ++ib)
                        for (size_t ia = 0; ia < na; ++ia)
                            inc[k][it * inc_len[k] + ia + na * ib] =
                                p[it * per + (sh == MFD_INC_ALONG_B ? ib : sh == MFD_INC_ALONG_A ? ia : 0)];
            }
        }
        for (int m = 0; m < d->nmon; ++m) {
            const mfd_monitor& a = d->mons[m];
            Monitor<T> M;
            M.kind = a.kind; M.sum = a.sum;
            M.cells.assign(a.cells, a.cells + a.npts);
            for (auto c : M.cells) if (c < 0 || (size_t)c >= N) { err = "monitor cell out of range"; return MFD_ERR_INVALID; }
            M.nw = a.nw;
            int ncomp = 9;
            if (a.kind == MFD_MON_FIELD) {
                for (int c = 0; c < ncomp; ++c) if (has_comp(c) && !is_D(c)) M.rec[c].assign(a.sum ? nt : nt * a.npts, 0);
            } else {
                M.phasor.assign(a.phasor, a.phasor + (size_t)nt * a.nw * 2);
                for (int c = 0; c < ncomp; ++c) if (has_comp(c) && !is_D(c)) M.S[c].assign(a.sum ? a.nw : (size_t)a.nw * a.npts, 0);
            }
            mons.push_back(std::move(M));
        }
        record = d->tfsf_record != 0;
        if (record) {
            for (int a = 0; a < 3; ++a) { ri1[a] = d->rec_i1[a]; ri2[a] = d->rec_i2[a]; }
            int narr = ndim == 3 ? 24 : ndim == 2 ? 8 : 4;
            for (int k = 0; k < narr; ++k) { rec_len[k] = face_len(k, ri1, ri2); rec[k].assign(rec_len[k] * nt, 0); }
        }
        return MFD_OK;
    }

    bool has_comp(int c) const {
        if (ndim == 3) return true;
        if (ndim == 2 && pol == MFD_POL_EY) return c == MFD_HX || c == MFD_HZ || c == MFD_DY || c == MFD_EY;
        if (ndim == 2) return c == MFD_HY || c == MFD_DX || c == MFD_DZ || c == MFD_EX || c == MFD_EZ;
        return c == MFD_HY || c == MFD_DX || c == MFD_EX;
    }
    static bool is_D(int c) { return c >= MFD_DX && c <= MFD_DZ; }

    // Extent of a TFSF array's first face axis a (y on the x faces, x on the y and z faces;
    // the whole line of a 2-D face; 1 in 1-D).
    size_t face_a(int k, const int* i1, const int* i2) const {
        size_t Nxi = i2[0] - i1[0], Nyi = i2[1] - i1[1];
        if (ndim == 1) return 1;
        if (ndim == 2) return face_len(k, i1, i2);
        int face = k / 4, j = k % 4;
        if (face < 2) return (j == 0 || j == 3) ? Nyi + 1 : Nyi;
        return (j == 0 || j == 3) ? Nxi + 1 : Nxi;
    }

    // Face extents of the TFSF arrays (sources.jl:441-459, 646-699, 804-832).
    size_t face_len(int k, const int* i1, const int* i2) const {
        size_t Nxi = i2[0] - i1[0], Nyi = i2[1] - i1[1], Nzi = i2[2] - i1[2];
        if (ndim == 1) return 1;
        if (ndim == 2 && pol == MFD_POL_EY) return k < 4 ? Nzi + 1 : Nxi + 1;   // Hz, Ey / Hx, Ey on the nodes
        if (ndim == 2) return k < 4 ? Nzi : Nxi;
        int face = k / 4, j = k % 4;
        if (face < 2) return (j == 0 || j == 3) ? (Nyi + 1) * Nzi : Nyi * (Nzi + 1);
        if (face < 4) return (j == 0 || j == 3) ? (Nxi + 1) * Nzi : Nxi * (Nzi + 1);
        return (j == 0 || j == 3) ? (Nxi + 1) * Nyi : Nxi * (Nyi + 1);
    }

    // ----------------------------------------------------------------------------------
    // 3-D update_H_kernel! (src/models.jl:735-878)
    void update_H3() {
        std::vector<T>&Hx = F[MFD_HX], &Hy = F[MFD_HY], &Hz = F[MFD_HZ];
        const std::vector<T>&Ex = F[MFD_EX], &Ey = F[MFD_EY], &Ez = F[MFD_EZ];
#pragma omp parallel for schedule(static)
        for (int iz = 0; iz < nz; ++iz)
            for (int iy = 0; iy < ny; ++iy)
                for (int ix = 0; ix < nx; ++ix) {
                    size_t c = id(ix, iy, iz);
                    int64_t g = geometry[c];
                    T Mh = g > 0 ? mats[g - 1].Mh : Mh0;
                    T Ey_ixp1, Ez_ixp1, Ex_iyp1, Ez_iyp1, Ex_izp1, Ey_izp1;
                    if (ix == nx - 1) {
                        int b = bc[MFD_XR];
                        if (b == MFD_BC_PERIODIC) { Ey_ixp1 = Ey[id(0, iy, iz)]; Ez_ixp1 = Ez[id(0, iy, iz)]; }
                        else if (b == MFD_BC_DIRICHLET) { Ey_ixp1 = 0; Ez_ixp1 = 0; }
                        else { Ey_ixp1 = Ey[c]; Ez_ixp1 = Ez[c]; }
                    } else { Ey_ixp1 = Ey[id(ix + 1, iy, iz)]; Ez_ixp1 = Ez[id(ix + 1, iy, iz)]; }
                    if (iy == ny - 1) {
                        int b = bc[MFD_YR];
                        if (b == MFD_BC_PERIODIC) { Ex_iyp1 = Ex[id(ix, 0, iz)]; Ez_iyp1 = Ez[id(ix, 0, iz)]; }
                        else if (b == MFD_BC_DIRICHLET) { Ex_iyp1 = 0; Ez_iyp1 = 0; }
                        else { Ex_iyp1 = Ex[c]; Ez_iyp1 = Ez[c]; }
                    } else { Ex_iyp1 = Ex[id(ix, iy + 1, iz)]; Ez_iyp1 = Ez[id(ix, iy + 1, iz)]; }
                    if (iz == nz - 1) {
                        int b = bc[MFD_ZR];
                        if (b == MFD_BC_PERIODIC) { Ex_izp1 = Ex[id(ix, iy, 0)]; Ey_izp1 = Ey[id(ix, iy, 0)]; }
                        else if (b == MFD_BC_DIRICHLET) { Ex_izp1 = 0; Ey_izp1 = 0; }
                        else { Ex_izp1 = Ex[c]; Ey_izp1 = Ey[c]; }
                    } else { Ex_izp1 = Ex[id(ix, iy, iz + 1)]; Ey_izp1 = Ey[id(ix, iy, iz + 1)]; }
                    T dExy = (Ex_iyp1 - Ex[c]) / dy;
                    T dExz = (Ex_izp1 - Ex[c]) / dz;
                    T dEyx = (Ey_ixp1 - Ey[c]) / dx;
                    T dEyz = (Ey_izp1 - Ey[c]) / dz;
                    T dEzx = (Ez_ixp1 - Ez[c]) / dx;
                    T dEzy = (Ez_iyp1 - Ez[c]) / dy;
                    // CPML (models.jl:811-871); psi[f][2]=psiE?x.., [3]=psiE?x.. per face
                    if (L[MFD_XL].nb && ix < L[MFD_XL].ib) {
                        const Layer<T>& l = L[MFD_XL];
                        int p = ix;
                        size_t q = (size_t)p + (size_t)l.nb * ((size_t)iy + (size_t)ny * iz);
                        T& pEyx = psi[MFD_XL][2][q]; T& pEzx = psi[MFD_XL][3][q];
                        pEyx = l.B[p] * pEyx + l.A[p] * dEyx;
                        pEzx = l.B[p] * pEzx + l.A[p] * dEzx;
                        Hy[c] += Mh * pEzx;
                        Hz[c] -= Mh * pEyx;
                        dEyx = dEyx / l.K[p];
                        dEzx = dEzx / l.K[p];
                    }
                    if (L[MFD_XR].nb && ix >= L[MFD_XR].ib - 1) {
                        const Layer<T>& l = L[MFD_XR];
                        int p = ix - (l.ib - 1);
                        size_t q = (size_t)p + (size_t)l.nb * ((size_t)iy + (size_t)ny * iz);
                        T& pEyx = psi[MFD_XR][2][q]; T& pEzx = psi[MFD_XR][3][q];
                        pEyx = l.B[p] * pEyx + l.A[p] * dEyx;
                        pEzx = l.B[p] * pEzx + l.A[p] * dEzx;
                        Hy[c] += Mh * pEzx;
                        Hz[c] -= Mh * pEyx;
                        dEyx = dEyx / l.K[p];
                        dEzx = dEzx / l.K[p];
                    }
                    if (L[MFD_YL].nb && iy < L[MFD_YL].ib) {
                        const Layer<T>& l = L[MFD_YL];
                        int p = iy;
                        size_t q = (size_t)ix + (size_t)nx * ((size_t)p + (size_t)l.nb * iz);
                        T& pExy = psi[MFD_YL][2][q]; T& pEzy = psi[MFD_YL][3][q];
                        pExy = l.B[p] * pExy + l.A[p] * dExy;
                        pEzy = l.B[p] * pEzy + l.A[p] * dEzy;
                        Hx[c] -= Mh * pEzy;
                        Hz[c] += Mh * pExy;
                        dExy = dExy / l.K[p];
                        dEzy = dEzy / l.K[p];
                    }
                    if (L[MFD_YR].nb && iy >= L[MFD_YR].ib - 1) {
                        const Layer<T>& l = L[MFD_YR];
                        int p = iy - (l.ib - 1);
                        size_t q = (size_t)ix + (size_t)nx * ((size_t)p + (size_t)l.nb * iz);
                        T& pExy = psi[MFD_YR][2][q]; T& pEzy = psi[MFD_YR][3][q];
                        pExy = l.B[p] * pExy + l.A[p] * dExy;
                        pEzy = l.B[p] * pEzy + l.A[p] * dEzy;
                        Hx[c] -= Mh * pEzy;
                        Hz[c] += Mh * pExy;
                        dExy = dExy / l.K[p];
                        dEzy = dEzy / l.K[p];
                    }
                    if (L[MFD_ZL].nb && iz < L[MFD_ZL].ib) {
                        const Layer<T>& l = L[MFD_ZL];
                        int p = iz;
                        size_t q = (size_t)ix + (size_t)nx * ((size_t)iy + (size_t)ny * p);
                        T& pExz = psi[MFD_ZL][2][q]; T& pEyz = psi[MFD_ZL][3][q];
                        pExz = l.B[p] * pExz + l.A[p] * dExz;
                        pEyz = l.B[p] * pEyz + l.A[p] * dEyz;
                        Hx[c] += Mh * pEyz;
                        Hy[c] -= Mh * pExz;
                        dExz = dExz / l.K[p];
                        dEyz = dEyz / l.K[p];
                    }
                    if (L[MFD_ZR].nb && iz >= L[MFD_ZR].ib - 1) {
                        const Layer<T>& l = L[MFD_ZR];
                        int p = iz - (l.ib - 1);
                        size_t q = (size_t)ix + (size_t)nx * ((size_t)iy + (size_t)ny * p);
                        T& pExz = psi[MFD_ZR][2][q]; T& pEyz = psi[MFD_ZR][3][q];
                        pExz = l.B[p] * pExz + l.A[p] * dExz;
                        pEyz = l.B[p] * pEyz + l.A[p] * dEyz;
                        Hx[c] += Mh * pEyz;
                        Hy[c] -= Mh * pExz;
                        dExz = dExz / l.K[p];
                        dEyz = dEyz / l.K[p];
                    }
                    Hx[c] -= Mh * (dEzy - dEyz);
                    Hy[c] -= Mh * (dExz - dEzx);
                    Hz[c] -= Mh * (dEyx - dExy);
                }
    }

    // Material response at one cell after the D update (models.jl:1042-1154, 2-D 622-712,
    // 1-D 365-431).  ncomp components; comp[k] is the field component of the k-th (x,y,z).
    void materials_and_E(size_t c, int64_t g, int ncomp, const int* Dc, const int* Ec, const int* Pslot) {
        T Me;
        bool isdisp = false, iskerr = false, isplas = false;
        Mat<T, R>* M = nullptr;
        if (g > 0) {
            M = &mats[g - 1];
            isdisp = M->disp; iskerr = M->kerr; isplas = M->plasma; Me = M->Me;
        } else Me = Me0;
        T sumP[3] = {0, 0, 0};
        if (isdisp) {
            int Nq = M->nq;
            for (int iq = 0; iq < Nq; ++iq) {
                for (int k = 0; k < ncomp; ++k) {
                    int s = Pslot[k];
                    size_t q = (size_t)iq + (size_t)Nq * c;
                    M->oldP2[s][q] = M->oldP1[s][q];
                    M->oldP1[s][q] = M->P[s][q];
                    M->P[s][q] = M->Aq[iq] * M->P[s][q] + M->Bq[iq] * M->oldP2[s][q] + M->Cq[iq] * F[Ec[k]][c];
                }
                for (int k = 0; k < ncomp; ++k) sumP[k] += M->P[Pslot[k]][(size_t)iq + (size_t)Nq * c];
            }
        }
        if (isplas) {
            T E2 = 0;
            for (int k = 0; k < ncomp; ++k) {
                T e = F[Ec[k]][c];
                E2 = k == 0 ? e * e : E2 + e * e;   // abs2(Ex) + abs2(Ey) + abs2(Ez)
            }
            T II = M->ksi * E2;
            R rho = M->rho[c];
            for (int k = 0; k < ncomp; ++k) {
                int s = Pslot[k];
                M->oldPp2[s][c] = M->oldPp1[s][c];
                M->oldPp1[s][c] = M->Pp[s][c];
                M->Pp[s][c] = M->Ap * M->Pp[s][c] + M->Bp * M->oldPp2[s][c] + M->Cp * rho * M->rho0 * F[Ec[k]][c];
            }
            for (int k = 0; k < ncomp; ++k) sumP[k] += M->Pp[Pslot[k]][c];
            T invE2;
            if (E2 >= std::numeric_limits<T>::epsilon()) invE2 = 1 / E2;
            else invE2 = 0;
            R drho = M->drho[c];
            for (int k = 0; k < ncomp; ++k) {
                int s = Pslot[k];
                M->Pa[s][c] += M->Ma * drho * M->rho0 * F[Ec[k]][c] * invE2;
            }
            for (int k = 0; k < ncomp; ++k) sumP[k] += M->Pa[Pslot[k]][c];
            // electron density (models.jl:1116-1125)
            if (M->rate_kind == MFD_RATE_TABLE) {
                T R1 = rate_table(*M, II);
                plasma_rho(*M, c, R1, E2);
            } else if (M->rate_kind == MFD_RATE_POWER) {
                T lg = std::log10(II);
                T a = M->rate_order * lg;
                double R1 = std::pow(10.0, (double)a + M->rate_log10c);
                plasma_rho(*M, c, R1, E2);
            } else {
                plasma_rho(*M, c, (T)0, E2);
            }
            // delivered energy (models.jl:1127-1132)
            T J[3];
            for (int k = 0; k < ncomp; ++k) {
                int s = Pslot[k];
                J[k] = (M->Pp[s][c] - M->oldPp2[s][c]) / (2 * dt);
            }
            T acc = J[0] * F[Ec[0]][c];
            for (int k = 1; k < ncomp; ++k) acc = acc + J[k] * F[Ec[k]][c];
            JE[c] += acc * dt;
        }
        for (int k = 0; k < ncomp; ++k) {
            T DmP = F[Dc[k]][c] - sumP[k];
            if (iskerr) {
                T Mk2 = M->Mk2, Mk3 = M->Mk3;
                // Kerr by Meep (models.jl:1143-1149)
                F[Ec[k]][c] = (1 + 1 * Mk2 * (Me * Me) * DmP + 2 * Mk3 * (Me * Me * Me) * (DmP * DmP)) /
                              (1 + 2 * Mk2 * (Me * Me) * DmP + 3 * Mk3 * (Me * Me * Me) * (DmP * DmP)) * DmP * Me;
            } else {
                F[Ec[k]][c] = DmP * Me;
            }
        }
    }

    T rate_table(const Mat<T, R>& M, T x) const { return ionization_rate<T>(M.rate_x.data(), M.rate_y.data(), M.rate_x.size(), x); }

    template <typename Q>
    void plasma_rho(Mat<T, R>& M, size_t c, Q R1, T E2) {
        T R2 = M.Rava * E2;
        R rho = M.rho[c];
        if (R2 == 0) {
            M.rho[c] = 1 - (1 - rho) * std::exp(-R1 * dt);
        } else {
            auto R12 = R1 - R2;
            M.rho[c] = R1 / R12 * 1 - (R1 / R12 * 1 - rho) * std::exp(-R12 * dt);
        }
        M.drho[c] = R1 * (1 - M.rho[c]);
    }

    // 3-D update_E_kernel! (src/models.jl:895-1162)
    void update_E3() {
        std::vector<T>&Dx = F[MFD_DX], &Dy = F[MFD_DY], &Dz = F[MFD_DZ];
        const std::vector<T>&Hx = F[MFD_HX], &Hy = F[MFD_HY], &Hz = F[MFD_HZ];
        static const int Dc[3] = {MFD_DX, MFD_DY, MFD_DZ}, Ec[3] = {MFD_EX, MFD_EY, MFD_EZ}, Ps[3] = {0, 1, 2};
#pragma omp parallel for schedule(static)
        for (int iz = 0; iz < nz; ++iz)
            for (int iy = 0; iy < ny; ++iy)
                for (int ix = 0; ix < nx; ++ix) {
                    size_t c = id(ix, iy, iz);
                    int64_t g = geometry[c];
                    T Md1, Md2;
                    if (g > 0) { Md1 = mats[g - 1].Md1; Md2 = mats[g - 1].Md2; }
                    else { Md1 = Md10; Md2 = Md20; }
                    T Hy_ixm1, Hz_ixm1, Hx_iym1, Hz_iym1, Hx_izm1, Hy_izm1;
                    if (ix == 0) {
                        int b = bc[MFD_XL];
                        if (b == MFD_BC_PERIODIC) { Hy_ixm1 = Hy[id(nx - 1, iy, iz)]; Hz_ixm1 = Hz[id(nx - 1, iy, iz)]; }
                        else if (b == MFD_BC_DIRICHLET) { Hy_ixm1 = 0; Hz_ixm1 = 0; }
                        else { Hy_ixm1 = Hy[c]; Hz_ixm1 = Hz[c]; }
                    } else { Hy_ixm1 = Hy[id(ix - 1, iy, iz)]; Hz_ixm1 = Hz[id(ix - 1, iy, iz)]; }
                    if (iy == 0) {
                        int b = bc[MFD_YL];
                        if (b == MFD_BC_PERIODIC) { Hx_iym1 = Hx[id(ix, ny - 1, iz)]; Hz_iym1 = Hz[id(ix, ny - 1, iz)]; }
                        else if (b == MFD_BC_DIRICHLET) { Hx_iym1 = 0; Hz_iym1 = 0; }
                        else { Hx_iym1 = Hx[c]; Hz_iym1 = Hz[c]; }
                    } else { Hx_iym1 = Hx[id(ix, iy - 1, iz)]; Hz_iym1 = Hz[id(ix, iy - 1, iz)]; }
                    if (iz == 0) {
                        int b = bc[MFD_ZL];
                        if (b == MFD_BC_PERIODIC) { Hx_izm1 = Hx[id(ix, iy, nz - 1)]; Hy_izm1 = Hy[id(ix, iy, nz - 1)]; }
                        else if (b == MFD_BC_DIRICHLET) { Hx_izm1 = 0; Hy_izm1 = 0; }
                        else { Hx_izm1 = Hx[c]; Hy_izm1 = Hy[c]; }
                    } else { Hx_izm1 = Hx[id(ix, iy, iz - 1)]; Hy_izm1 = Hy[id(ix, iy, iz - 1)]; }
                    T dHxy = (Hx[c] - Hx_iym1) / dy;
                    T dHxz = (Hx[c] - Hx_izm1) / dz;
                    T dHyx = (Hy[c] - Hy_ixm1) / dx;
                    T dHyz = (Hy[c] - Hy_izm1) / dz;
                    T dHzx = (Hz[c] - Hz_ixm1) / dx;
                    T dHzy = (Hz[c] - Hz_iym1) / dy;
                    // CPML (models.jl:975-1035); psi[f][0],[1] are the H psi arrays of face f
                    if (L[MFD_XL].nb && ix < L[MFD_XL].ib) {
                        const Layer<T>& l = L[MFD_XL];
                        int p = ix;
                        size_t q = (size_t)p + (size_t)l.nb * ((size_t)iy + (size_t)ny * iz);
                        T& pHyx = psi[MFD_XL][0][q]; T& pHzx = psi[MFD_XL][1][q];
                        pHyx = l.B[p] * pHyx + l.A[p] * dHyx;
                        pHzx = l.B[p] * pHzx + l.A[p] * dHzx;
                        Dy[c] -= Md2 * pHzx;
                        Dz[c] += Md2 * pHyx;
                        dHyx = dHyx / l.K[p];
                        dHzx = dHzx / l.K[p];
                    }
                    if (L[MFD_XR].nb && ix >= L[MFD_XR].ib - 1) {
                        const Layer<T>& l = L[MFD_XR];
                        int p = ix - (l.ib - 1);
                        size_t q = (size_t)p + (size_t)l.nb * ((size_t)iy + (size_t)ny * iz);
                        T& pHyx = psi[MFD_XR][0][q]; T& pHzx = psi[MFD_XR][1][q];
                        pHyx = l.B[p] * pHyx + l.A[p] * dHyx;
                        pHzx = l.B[p] * pHzx + l.A[p] * dHzx;
                        Dy[c] -= Md2 * pHzx;
                        Dz[c] += Md2 * pHyx;
                        dHyx = dHyx / l.K[p];
                        dHzx = dHzx / l.K[p];
                    }
                    if (L[MFD_YL].nb && iy < L[MFD_YL].ib) {
                        const Layer<T>& l = L[MFD_YL];
                        int p = iy;
                        size_t q = (size_t)ix + (size_t)nx * ((size_t)p + (size_t)l.nb * iz);
                        T& pHxy = psi[MFD_YL][0][q]; T& pHzy = psi[MFD_YL][1][q];
                        pHxy = l.B[p] * pHxy + l.A[p] * dHxy;
                        pHzy = l.B[p] * pHzy + l.A[p] * dHzy;
                        Dx[c] += Md2 * pHzy;
                        Dz[c] -= Md2 * pHxy;
                        dHxy = dHxy / l.K[p];
                        dHzy = dHzy / l.K[p];
                    }
                    if (L[MFD_YR].nb && iy >= L[MFD_YR].ib - 1) {
                        const Layer<T>& l = L[MFD_YR];
                        int p = iy - (l.ib - 1);
                        size_t q = (size_t)ix + (size_t)nx * ((size_t)p + (size_t)l.nb * iz);
                        T& pHxy = psi[MFD_YR][0][q]; T& pHzy = psi[MFD_YR][1][q];
                        pHxy = l.B[p] * pHxy + l.A[p] * dHxy;
                        pHzy = l.B[p] * pHzy + l.A[p] * dHzy;
                        Dx[c] += Md2 * pHzy;
                        Dz[c] -= Md2 * pHxy;
                        dHxy = dHxy / l.K[p];
                        dHzy = dHzy / l.K[p];
                    }
                    if (L[MFD_ZL].nb && iz < L[MFD_ZL].ib) {
                        const Layer<T>& l = L[MFD_ZL];
                        int p = iz;
                        size_t q = (size_t)ix + (size_t)nx * ((size_t)iy + (size_t)ny * p);
                        T& pHxz = psi[MFD_ZL][0][q]; T& pHyz = psi[MFD_ZL][1][q];
                        pHxz = l.B[p] * pHxz + l.A[p] * dHxz;
                        pHyz = l.B[p] * pHyz + l.A[p] * dHyz;
                        Dx[c] -= Md2 * pHyz;
                        Dy[c] += Md2 * pHxz;
                        dHxz = dHxz / l.K[p];
                        dHyz = dHyz / l.K[p];
                    }
                    if (L[MFD_ZR].nb && iz >= L[MFD_ZR].ib - 1) {
                        const Layer<T>& l = L[MFD_ZR];
                        int p = iz - (l.ib - 1);
                        size_t q = (size_t)ix + (size_t)nx * ((size_t)iy + (size_t)ny * p);
                        T& pHxz = psi[MFD_ZR][0][q]; T& pHyz = psi[MFD_ZR][1][q];
                        pHxz = l.B[p] * pHxz + l.A[p] * dHxz;
                        pHyz = l.B[p] * pHyz + l.A[p] * dHyz;
                        Dx[c] -= Md2 * pHyz;
                        Dy[c] += Md2 * pHxz;
                        dHxz = dHxz / l.K[p];
                        dHyz = dHyz / l.K[p];
                    }
                    Dx[c] = Md1 * Dx[c] + Md2 * (dHzy - dHyz);
                    Dy[c] = Md1 * Dy[c] + Md2 * (dHxz - dHzx);
                    Dz[c] = Md1 * Dz[c] + Md2 * (dHyx - dHxy);
                    materials_and_E(c, g, 3, Dc, Ec, Ps);
                }
    }

    // 2-D update_H_kernel! (src/models.jl:450-529).  psi[xface][0]=psiHyx, [1]=psiEzx;
    // psi[zface][0]=psiHyz, [1]=psiExz.
    void update_H2() {
        std::vector<T>& Hy = F[MFD_HY];
        const std::vector<T>&Ex = F[MFD_EX], &Ez = F[MFD_EZ];
#pragma omp parallel for schedule(static)
        for (int iz = 0; iz < nz; ++iz)
            for (int ix = 0; ix < nx; ++ix) {
                size_t c = id(ix, 0, iz);
                int64_t g = geometry[c];
                T Mh = g > 0 ? mats[g - 1].Mh : Mh0;
                T Ez_ixp1, Ex_izp1;
                if (ix == nx - 1) {
                    int b = bc[MFD_XR];
                    if (b == MFD_BC_PERIODIC) Ez_ixp1 = Ez[id(0, 0, iz)];
                    else if (b == MFD_BC_DIRICHLET) Ez_ixp1 = 0;
                    else Ez_ixp1 = Ez[c];
                } else Ez_ixp1 = Ez[id(ix + 1, 0, iz)];
                if (iz == nz - 1) {
                    int b = bc[MFD_ZR];
                    if (b == MFD_BC_PERIODIC) Ex_izp1 = Ex[id(ix, 0, 0)];
                    else if (b == MFD_BC_DIRICHLET) Ex_izp1 = 0;
                    else Ex_izp1 = Ex[c];
                } else Ex_izp1 = Ex[id(ix, 0, iz + 1)];
                T dExz = (Ex_izp1 - Ex[c]) / dz;
                T dEzx = (Ez_ixp1 - Ez[c]) / dx;
                if (L[MFD_XL].nb && ix < L[MFD_XL].ib) {
                    const Layer<T>& l = L[MFD_XL];
                    int p = ix;
                    T& ps = psi[MFD_XL][1][(size_t)p + (size_t)l.nb * iz];
                    ps = l.B[p] * ps + l.A[p] * dEzx;
                    Hy[c] += Mh * ps;
                    dEzx = dEzx / l.K[p];
                }
                if (L[MFD_XR].nb && ix >= L[MFD_XR].ib - 1) {
                    const Layer<T>& l = L[MFD_XR];
                    int p = ix - (l.ib - 1);
                    T& ps = psi[MFD_XR][1][(size_t)p + (size_t)l.nb * iz];
                    ps = l.B[p] * ps + l.A[p] * dEzx;
                    Hy[c] += Mh * ps;
                    dEzx = dEzx / l.K[p];
                }
                if (L[MFD_ZL].nb && iz < L[MFD_ZL].ib) {
                    const Layer<T>& l = L[MFD_ZL];
                    int p = iz;
                    T& ps = psi[MFD_ZL][1][(size_t)ix + (size_t)nx * p];
                    ps = l.B[p] * ps + l.A[p] * dExz;
                    Hy[c] -= Mh * ps;
                    dExz = dExz / l.K[p];
                }
                if (L[MFD_ZR].nb && iz >= L[MFD_ZR].ib - 1) {
                    const Layer<T>& l = L[MFD_ZR];
                    int p = iz - (l.ib - 1);
                    T& ps = psi[MFD_ZR][1][(size_t)ix + (size_t)nx * p];
                    ps = l.B[p] * ps + l.A[p] * dExz;
                    Hy[c] -= Mh * ps;
                    dExz = dExz / l.K[p];
                }
                Hy[c] -= Mh * (dExz - dEzx);
            }
    }

    // 2-D update_E_kernel! (src/models.jl:539-719)
    void update_E2() {
        std::vector<T>&Dx = F[MFD_DX], &Dz = F[MFD_DZ];
        const std::vector<T>& Hy = F[MFD_HY];
        static const int Dc[2] = {MFD_DX, MFD_DZ}, Ec[2] = {MFD_EX, MFD_EZ}, Ps[2] = {0, 2};
#pragma omp parallel for schedule(static)
        for (int iz = 0; iz < nz; ++iz)
            for (int ix = 0; ix < nx; ++ix) {
                size_t c = id(ix, 0, iz);
                int64_t g = geometry[c];
                T Md1, Md2;
                if (g > 0) { Md1 = mats[g - 1].Md1; Md2 = mats[g - 1].Md2; }
                else { Md1 = Md10; Md2 = Md20; }
                T Hy_ixm1, Hy_izm1;
                if (ix == 0) {
                    int b = bc[MFD_XL];
                    if (b == MFD_BC_PERIODIC) Hy_ixm1 = Hy[id(nx - 1, 0, iz)];
                    else if (b == MFD_BC_DIRICHLET) Hy_ixm1 = 0;
                    else Hy_ixm1 = Hy[c];
                } else Hy_ixm1 = Hy[id(ix - 1, 0, iz)];
                if (iz == 0) {
                    int b = bc[MFD_ZL];
                    if (b == MFD_BC_PERIODIC) Hy_izm1 = Hy[id(ix, 0, nz - 1)];
                    else if (b == MFD_BC_DIRICHLET) Hy_izm1 = 0;
                    else Hy_izm1 = Hy[c];
                } else Hy_izm1 = Hy[id(ix, 0, iz - 1)];
                T dHyx = (Hy[c] - Hy_ixm1) / dx;
                T dHyz = (Hy[c] - Hy_izm1) / dz;
                if (L[MFD_XL].nb && ix < L[MFD_XL].ib) {
                    const Layer<T>& l = L[MFD_XL];
                    int p = ix;
                    T& ps = psi[MFD_XL][0][(size_t)p + (size_t)l.nb * iz];
                    ps = l.B[p] * ps + l.A[p] * dHyx;
                    Dz[c] += Md2 * ps;
                    dHyx = dHyx / l.K[p];
                }
                if (L[MFD_XR].nb && ix >= L[MFD_XR].ib - 1) {
                    const Layer<T>& l = L[MFD_XR];
                    int p = ix - (l.ib - 1);
                    T& ps = psi[MFD_XR][0][(size_t)p + (size_t)l.nb * iz];
                    ps = l.B[p] * ps + l.A[p] * dHyx;
                    Dz[c] += Md2 * ps;
                    dHyx = dHyx / l.K[p];
                }
                if (L[MFD_ZL].nb && iz < L[MFD_ZL].ib) {
                    const Layer<T>& l = L[MFD_ZL];
                    int p = iz;
                    T& ps = psi[MFD_ZL][0][(size_t)ix + (size_t)nx * p];
                    ps = l.B[p] * ps + l.A[p] * dHyz;
                    Dx[c] -= Md2 * ps;
                    dHyz = dHyz / l.K[p];
                }
                if (L[MFD_ZR].nb && iz >= L[MFD_ZR].ib - 1) {
                    const Layer<T>& l = L[MFD_ZR];
                    int p = iz - (l.ib - 1);
                    T& ps = psi[MFD_ZR][0][(size_t)ix + (size_t)nx * p];
                    ps = l.B[p] * ps + l.A[p] * dHyz;
                    Dx[c] -= Md2 * ps;
                    dHyz = dHyz / l.K[p];
                }
                Dx[c] = Md1 * Dx[c] + Md2 * (0 - dHyz);
                Dz[c] = Md1 * Dz[c] + Md2 * (dHyx - 0);
                materials_and_E(c, g, 2, Dc, Ec, Ps);
            }
    }

    // 2-D updates of the second field set (Hx, Hz, Dy, Ey): the 3-D update_H_kernel! /
    // update_E_kernel! (src/models.jl:735-878, 895-1162) with every y derivative zero, in
    // the 3-D operation order.  psi[xface][0]=psiHzx, [1]=psiEyx; psi[zface][0]=psiHxz,
    // [1]=psiEyz.
    void update_H2ey() {
        std::vector<T>&Hx = F[MFD_HX], &Hz = F[MFD_HZ];
        const std::vector<T>& Ey = F[MFD_EY];
#pragma omp parallel for schedule(static)
        for (int iz = 0; iz < nz; ++iz)
            for (int ix = 0; ix < nx; ++ix) {
                size_t c = id(ix, 0, iz);
                int64_t g = geometry[c];
                T Mh = g > 0 ? mats[g - 1].Mh : Mh0;
                T Ey_ixp1, Ey_izp1;
                if (ix == nx - 1) {
                    int b = bc[MFD_XR];
                    if (b == MFD_BC_PERIODIC) Ey_ixp1 = Ey[id(0, 0, iz)];
                    else if (b == MFD_BC_DIRICHLET) Ey_ixp1 = 0;
                    else Ey_ixp1 = Ey[c];
                } else Ey_ixp1 = Ey[id(ix + 1, 0, iz)];
                if (iz == nz - 1) {
                    int b = bc[MFD_ZR];
                    if (b == MFD_BC_PERIODIC) Ey_izp1 = Ey[id(ix, 0, 0)];
                    else if (b == MFD_BC_DIRICHLET) Ey_izp1 = 0;
                    else Ey_izp1 = Ey[c];
                } else Ey_izp1 = Ey[id(ix, 0, iz + 1)];
                T dEyx = (Ey_ixp1 - Ey[c]) / dx;
                T dEyz = (Ey_izp1 - Ey[c]) / dz;
                for (int f : {MFD_XL, MFD_XR}) {
                    const Layer<T>& l = L[f];
                    if (!l.nb || (f == MFD_XL ? ix >= l.ib : ix < l.ib - 1)) continue;
                    int p = f == MFD_XL ? ix : ix - (l.ib - 1);
                    T& ps = psi[f][1][(size_t)p + (size_t)l.nb * iz];
                    ps = l.B[p] * ps + l.A[p] * dEyx;
                    Hz[c] -= Mh * ps;
                    dEyx = dEyx / l.K[p];
                }
                for (int f : {MFD_ZL, MFD_ZR}) {
                    const Layer<T>& l = L[f];
                    if (!l.nb || (f == MFD_ZL ? iz >= l.ib : iz < l.ib - 1)) continue;
                    int p = f == MFD_ZL ? iz : iz - (l.ib - 1);
                    T& ps = psi[f][1][(size_t)ix + (size_t)nx * p];
                    ps = l.B[p] * ps + l.A[p] * dEyz;
                    Hx[c] += Mh * ps;
                    dEyz = dEyz / l.K[p];
                }
                Hx[c] -= Mh * (0 - dEyz);
                Hz[c] -= Mh * (dEyx - 0);
            }
    }

    void update_E2ey() {
        std::vector<T>& Dy = F[MFD_DY];
        const std::vector<T>&Hx = F[MFD_HX], &Hz = F[MFD_HZ];
        static const int Dc[1] = {MFD_DY}, Ec[1] = {MFD_EY}, Ps[1] = {1};
#pragma omp parallel for schedule(static)
        for (int iz = 0; iz < nz; ++iz)
            for (int ix = 0; ix < nx; ++ix) {
                size_t c = id(ix, 0, iz);
                int64_t g = geometry[c];
                T Md1, Md2;
                if (g > 0) { Md1 = mats[g - 1].Md1; Md2 = mats[g - 1].Md2; }
                else { Md1 = Md10; Md2 = Md20; }
                T Hz_ixm1, Hx_izm1;
                if (ix == 0) {
                    int b = bc[MFD_XL];
                    if (b == MFD_BC_PERIODIC) Hz_ixm1 = Hz[id(nx - 1, 0, iz)];
                    else if (b == MFD_BC_DIRICHLET) Hz_ixm1 = 0;
                    else Hz_ixm1 = Hz[c];
                } else Hz_ixm1 = Hz[id(ix - 1, 0, iz)];
                if (iz == 0) {
                    int b = bc[MFD_ZL];
                    if (b == MFD_BC_PERIODIC) Hx_izm1 = Hx[id(ix, 0, nz - 1)];
                    else if (b == MFD_BC_DIRICHLET) Hx_izm1 = 0;
                    else Hx_izm1 = Hx[c];
                } else Hx_izm1 = Hx[id(ix, 0, iz - 1)];
                T dHxz = (Hx[c] - Hx_izm1) / dz;
                T dHzx = (Hz[c] - Hz_ixm1) / dx;
                for (int f : {MFD_XL, MFD_XR}) {
                    const Layer<T>& l = L[f];
                    if (!l.nb || (f == MFD_XL ? ix >= l.ib : ix < l.ib - 1)) continue;
                    int p = f == MFD_XL ? ix : ix - (l.ib - 1);
                    T& ps = psi[f][0][(size_t)p + (size_t)l.nb * iz];
                    ps = l.B[p] * ps + l.A[p] * dHzx;
                    Dy[c] -= Md2 * ps;
                    dHzx = dHzx / l.K[p];
                }
                for (int f : {MFD_ZL, MFD_ZR}) {
                    const Layer<T>& l = L[f];
                    if (!l.nb || (f == MFD_ZL ? iz >= l.ib : iz < l.ib - 1)) continue;
                    int p = f == MFD_ZL ? iz : iz - (l.ib - 1);
                    T& ps = psi[f][0][(size_t)ix + (size_t)nx * p];
                    ps = l.B[p] * ps + l.A[p] * dHxz;
                    Dy[c] += Md2 * ps;
                    dHxz = dHxz / l.K[p];
                }
                Dy[c] = Md1 * Dy[c] + Md2 * (dHxz - dHzx);
                materials_and_E(c, g, 1, Dc, Ec, Ps);
            }
    }

    // 1-D kernels (src/models.jl:248-437).  psi[zface][0]=psiHyz, [1]=psiExz.
    void update_H1() {
        std::vector<T>& Hy = F[MFD_HY];
        const std::vector<T>& Ex = F[MFD_EX];
#pragma omp parallel for schedule(static)
        for (int iz = 0; iz < nz; ++iz) {
            size_t c = iz;
            int64_t g = geometry[c];
            T Mh = g > 0 ? mats[g - 1].Mh : Mh0;
            T Ex_izp1;
            if (iz == nz - 1) {
                int b = bc[MFD_ZR];
                if (b == MFD_BC_PERIODIC) Ex_izp1 = Ex[0];
                else if (b == MFD_BC_DIRICHLET) Ex_izp1 = 0;
                else Ex_izp1 = Ex[c];
            } else Ex_izp1 = Ex[c + 1];
            T dExz = (Ex_izp1 - Ex[c]) / dz;
            if (L[MFD_ZL].nb && iz < L[MFD_ZL].ib) {
                const Layer<T>& l = L[MFD_ZL];
                int p = iz;
                T& ps = psi[MFD_ZL][1][p];
                ps = l.B[p] * ps + l.A[p] * dExz;
                Hy[c] -= Mh * ps;
                dExz = dExz / l.K[p];
            }
            if (L[MFD_ZR].nb && iz >= L[MFD_ZR].ib - 1) {
                const Layer<T>& l = L[MFD_ZR];
                int p = iz - (l.ib - 1);
                T& ps = psi[MFD_ZR][1][p];
                ps = l.B[p] * ps + l.A[p] * dExz;
                Hy[c] -= Mh * ps;
                dExz = dExz / l.K[p];
            }
            Hy[c] -= Mh * (0 + dExz);
        }
    }

    void update_E1() {
        std::vector<T>& Dx = F[MFD_DX];
        const std::vector<T>& Hy = F[MFD_HY];
        static const int Dc[1] = {MFD_DX}, Ec[1] = {MFD_EX}, Ps[1] = {0};
#pragma omp parallel for schedule(static)
        for (int iz = 0; iz < nz; ++iz) {
            size_t c = iz;
            int64_t g = geometry[c];
            T Md1, Md2;
            if (g > 0) { Md1 = mats[g - 1].Md1; Md2 = mats[g - 1].Md2; }
            else { Md1 = Md10; Md2 = Md20; }
            T Hy_izm1;
            if (iz == 0) {
                int b = bc[MFD_ZL];
                if (b == MFD_BC_PERIODIC) Hy_izm1 = Hy[nz - 1];
                else if (b == MFD_BC_DIRICHLET) Hy_izm1 = 0;
                else Hy_izm1 = Hy[c];
            } else Hy_izm1 = Hy[c - 1];
            T dHyz = (Hy[c] - Hy_izm1) / dz;
            if (L[MFD_ZL].nb && iz < L[MFD_ZL].ib) {
                const Layer<T>& l = L[MFD_ZL];
                int p = iz;
                T& ps = psi[MFD_ZL][0][p];
                ps = l.B[p] * ps + l.A[p] * dHyz;
                Dx[c] -= Md2 * ps;
                dHyz = dHyz / l.K[p];
            }
            if (L[MFD_ZR].nb && iz >= L[MFD_ZR].ib - 1) {
                const Layer<T>& l = L[MFD_ZR];
                int p = iz - (l.ib - 1);
                T& ps = psi[MFD_ZR][0][p];
                ps = l.B[p] * ps + l.A[p] * dHyz;
                Dx[c] -= Md2 * ps;
                dHyz = dHyz / l.K[p];
            }
            Dx[c] = Md1 * Dx[c] + Md2 * (0 - dHyz);
            materials_and_E(c, g, 1, Dc, Ec, Ps);
        }
    }

    // ----------------------------------------------------------------------------------
    // Soft / hard sources (sources.jl:77-131, 190-244): waveform tabulated in double.
    void add_point_source(const Source<T>& s, int64_t it) {
        std::vector<T>& FC = F[s.comp];
        size_t np = s.cells.size();
        for (size_t p = 0; p < np; ++p) {
            double w = s.wave.empty() ? s.amp[p] * s.gt[it - 1] : s.wave[(size_t)(it - 1) * np + p];
            int64_t c = s.cells[p];
            if (s.kind == MFD_SRC_SOFT) FC[c] = (T)((double)FC[c] + (double)s.coeff * w);
            else FC[c] = (T)w;
        }
    }

    // TFSF add_source! (sources.jl:320-346, 469-497, 713-776).
    // One broadcast: F[range] op= coef * inc[:, :, it], evaluated in the promoted type U.
    template <typename U>
    void tfsf_apply(int comp, int xa, int xb, int ya, int yb, int za, int zb, int k, int64_t it, U coef, int sign) {
        std::vector<T>& FC = F[comp];
        const T* src = inc[k].data() + (size_t)(it - 1) * inc_len[k];
        size_t n = 0;
        for (int iz = za; iz <= zb; ++iz)
            for (int iy = ya; iy <= yb; ++iy)
                for (int ix = xa; ix <= xb; ++ix) {
                    size_t c = id(ix - 1, iy - 1, iz - 1);
                    U v = coef * (U)src[n++];
                    FC[c] = (T)(sign > 0 ? (U)FC[c] + v : (U)FC[c] - v);
                }
    }

    void add_tfsf(int64_t it) {
        int ix1 = ti1[0], iy1 = ti1[1], iz1 = ti1[2], ix2 = ti2[0], iy2 = ti2[1], iz2 = ti2[2];
        if (ndim == 3) {
            double Cm = (double)dt / MU0, Ce = (double)dt / EPS0;   // sources.jl:725
            double cmx = Cm / (double)dx, cmy = Cm / (double)dy, cmz = Cm / (double)dz;
            double cex = Ce / (double)dx, cey = Ce / (double)dy, cez = Ce / (double)dz;
            double cdx = EPS0 * Ce / (double)dx, cdy = EPS0 * Ce / (double)dy, cdz = EPS0 * Ce / (double)dz;
            // 1yz
            tfsf_apply<double>(MFD_HY, ix1 - 1, ix1 - 1, iy1, iy2, iz1, iz2 - 1, 3, it, cmx, -1);
            tfsf_apply<double>(MFD_HZ, ix1 - 1, ix1 - 1, iy1, iy2 - 1, iz1, iz2, 2, it, cmx, +1);
            tfsf_apply<double>(MFD_EY, ix1, ix1, iy1, iy2 - 1, iz1, iz2, 1, it, cex, +1);
            tfsf_apply<double>(MFD_EZ, ix1, ix1, iy1, iy2, iz1, iz2 - 1, 0, it, cex, -1);
            tfsf_apply<double>(MFD_DY, ix1, ix1, iy1, iy2 - 1, iz1, iz2, 1, it, cdx, +1);
            tfsf_apply<double>(MFD_DZ, ix1, ix1, iy1, iy2, iz1, iz2 - 1, 0, it, cdx, -1);
            // 2yz
            tfsf_apply<double>(MFD_HY, ix2, ix2, iy1, iy2, iz1, iz2 - 1, 7, it, cmx, +1);
            tfsf_apply<double>(MFD_HZ, ix2, ix2, iy1, iy2 - 1, iz1, iz2, 6, it, cmx, -1);
            tfsf_apply<double>(MFD_EY, ix2, ix2, iy1, iy2 - 1, iz1, iz2, 5, it, cex, -1);
            tfsf_apply<double>(MFD_EZ, ix2, ix2, iy1, iy2, iz1, iz2 - 1, 4, it, cex, +1);
            tfsf_apply<double>(MFD_DY, ix2, ix2, iy1, iy2 - 1, iz1, iz2, 5, it, cdx, -1);
            tfsf_apply<double>(MFD_DZ, ix2, ix2, iy1, iy2, iz1, iz2 - 1, 4, it, cdx, +1);
            // x1z
            tfsf_apply<double>(MFD_HX, ix1, ix2, iy1 - 1, iy1 - 1, iz1, iz2 - 1, 11, it, cmy, +1);
            tfsf_apply<double>(MFD_HZ, ix1, ix2 - 1, iy1 - 1, iy1 - 1, iz1, iz2, 10, it, cmy, -1);
            tfsf_apply<double>(MFD_EX, ix1, ix2 - 1, iy1, iy1, iz1, iz2, 9, it, cey, -1);
            tfsf_apply<double>(MFD_EZ, ix1, ix2, iy1, iy1, iz1, iz2 - 1, 8, it, cey, +1);
            tfsf_apply<double>(MFD_DX, ix1, ix2 - 1, iy1, iy1, iz1, iz2, 9, it, cdy, -1);
            tfsf_apply<double>(MFD_DZ, ix1, ix2, iy1, iy1, iz1, iz2 - 1, 8, it, cdy, +1);
            // x2z
            tfsf_apply<double>(MFD_HX, ix1, ix2, iy2, iy2, iz1, iz2 - 1, 15, it, cmy, -1);
            tfsf_apply<double>(MFD_HZ, ix1, ix2 - 1, iy2, iy2, iz1, iz2, 14, it, cmy, +1);
            tfsf_apply<double>(MFD_EX, ix1, ix2 - 1, iy2, iy2, iz1, iz2, 13, it, cey, +1);
            tfsf_apply<double>(MFD_EZ, ix1, ix2, iy2, iy2, iz1, iz2 - 1, 12, it, cey, -1);
            tfsf_apply<double>(MFD_DX, ix1, ix2 - 1, iy2, iy2, iz1, iz2, 13, it, cdy, +1);
            tfsf_apply<double>(MFD_DZ, ix1, ix2, iy2, iy2, iz1, iz2 - 1, 12, it, cdy, -1);
            // xy1
            tfsf_apply<double>(MFD_HX, ix1, ix2, iy1, iy2 - 1, iz1 - 1, iz1 - 1, 19, it, cmz, -1);
            tfsf_apply<double>(MFD_HY, ix1, ix2 - 1, iy1, iy2, iz1 - 1, iz1 - 1, 18, it, cmz, +1);
            tfsf_apply<double>(MFD_EX, ix1, ix2 - 1, iy1, iy2, iz1, iz1, 17, it, cez, +1);
            tfsf_apply<double>(MFD_EY, ix1, ix2, iy1, iy2 - 1, iz1, iz1, 16, it, cez, -1);
            tfsf_apply<double>(MFD_DX, ix1, ix2 - 1, iy1, iy2, iz1, iz1, 17, it, cdz, +1);
            tfsf_apply<double>(MFD_DY, ix1, ix2, iy1, iy2 - 1, iz1, iz1, 16, it, cdz, -1);
            // xy2
            tfsf_apply<double>(MFD_HX, ix1, ix2, iy1, iy2 - 1, iz2, iz2, 23, it, cmz, +1);
            tfsf_apply<double>(MFD_HY, ix1, ix2 - 1, iy1, iy2, iz2, iz2, 22, it, cmz, -1);
            tfsf_apply<double>(MFD_EX, ix1, ix2 - 1, iy1, iy2, iz2, iz2, 21, it, cez, -1);
            tfsf_apply<double>(MFD_EY, ix1, ix2, iy1, iy2 - 1, iz2, iz2, 20, it, cez, +1);
            tfsf_apply<double>(MFD_DX, ix1, ix2 - 1, iy1, iy2, iz2, iz2, 21, it, cdz, -1);
            tfsf_apply<double>(MFD_DY, ix1, ix2, iy1, iy2 - 1, iz2, iz2, 20, it, cdz, +1);
        } else if (ndim == 2 && pol == MFD_POL_EY) {
            // The 3-D faces 1yz, 2yz, xy1, xy2 restricted to Hz, Ey / Hx, Ey (their signs and
            // node ranges, sources.jl:728-776) with the 2-D coefficients (sources.jl:478-495).
            double cmx = (double)dt / (MU0 * (double)dx), cex = (double)dt / (EPS0 * (double)dx);
            double cmz = (double)dt / (MU0 * (double)dz), cez = (double)dt / (EPS0 * (double)dz);
            T cdx = dt / dx, cdz = dt / dz;
            // 1z
            tfsf_apply<double>(MFD_HZ, ix1 - 1, ix1 - 1, 1, 1, iz1, iz2, 1, it, cmx, +1);
            tfsf_apply<double>(MFD_EY, ix1, ix1, 1, 1, iz1, iz2, 0, it, cex, +1);
            tfsf_apply<T>(MFD_DY, ix1, ix1, 1, 1, iz1, iz2, 0, it, cdx, +1);
            // 2z
            tfsf_apply<double>(MFD_HZ, ix2, ix2, 1, 1, iz1, iz2, 3, it, cmx, -1);
            tfsf_apply<double>(MFD_EY, ix2, ix2, 1, 1, iz1, iz2, 2, it, cex, -1);
            tfsf_apply<T>(MFD_DY, ix2, ix2, 1, 1, iz1, iz2, 2, it, cdx, -1);
            // x1
            tfsf_apply<double>(MFD_HX, ix1, ix2, 1, 1, iz1 - 1, iz1 - 1, 5, it, cmz, -1);
            tfsf_apply<double>(MFD_EY, ix1, ix2, 1, 1, iz1, iz1, 4, it, cez, -1);
            tfsf_apply<T>(MFD_DY, ix1, ix2, 1, 1, iz1, iz1, 4, it, cdz, -1);
            // x2
            tfsf_apply<double>(MFD_HX, ix1, ix2, 1, 1, iz2, iz2, 7, it, cmz, +1);
            tfsf_apply<double>(MFD_EY, ix1, ix2, 1, 1, iz2, iz2, 6, it, cez, +1);
            tfsf_apply<T>(MFD_DY, ix1, ix2, 1, 1, iz2, iz2, 6, it, cdz, +1);
        } else if (ndim == 2) {
            // dt/(MU0*dx) and dt/(EPS0*dx) promote to double; dt/dx stays T (sources.jl:478-495)
            double cmx = (double)dt / (MU0 * (double)dx), cex = (double)dt / (EPS0 * (double)dx);
            double cmz = (double)dt / (MU0 * (double)dz), cez = (double)dt / (EPS0 * (double)dz);
            T cdx = dt / dx, cdz = dt / dz;
            // 1z
            tfsf_apply<double>(MFD_HY, ix1 - 1, ix1 - 1, 1, 1, iz1, iz2 - 1, 1, it, cmx, -1);
            tfsf_apply<double>(MFD_EZ, ix1, ix1, 1, 1, iz1, iz2 - 1, 0, it, cex, -1);
            tfsf_apply<T>(MFD_DZ, ix1, ix1, 1, 1, iz1, iz2 - 1, 0, it, cdx, -1);
            // 2z
            tfsf_apply<double>(MFD_HY, ix2, ix2, 1, 1, iz1, iz2 - 1, 3, it, cmx, +1);
            tfsf_apply<double>(MFD_EZ, ix2, ix2, 1, 1, iz1, iz2 - 1, 2, it, cex, +1);
            tfsf_apply<T>(MFD_DZ, ix2, ix2, 1, 1, iz1, iz2 - 1, 2, it, cdx, +1);
            // x1
            tfsf_apply<double>(MFD_HY, ix1, ix2 - 1, 1, 1, iz1 - 1, iz1 - 1, 5, it, cmz, +1);
            tfsf_apply<double>(MFD_EX, ix1, ix2 - 1, 1, 1, iz1, iz1, 4, it, cez, +1);
            tfsf_apply<T>(MFD_DX, ix1, ix2 - 1, 1, 1, iz1, iz1, 4, it, cdz, +1);
            // x2
            tfsf_apply<double>(MFD_HY, ix1, ix2 - 1, 1, 1, iz2, iz2, 7, it, cmz, -1);
            tfsf_apply<double>(MFD_EX, ix1, ix2 - 1, 1, 1, iz2, iz2, 6, it, cez, -1);
            tfsf_apply<T>(MFD_DX, ix1, ix2 - 1, 1, 1, iz2, iz2, 6, it, cdz, -1);
        } else {
            double cm = (double)dt / (MU0 * (double)dz), ce = (double)dt / (EPS0 * (double)dz);
            T cd = dt / dz;
            tfsf_apply<double>(MFD_HY, 1, 1, 1, 1, iz1 - 1, iz1 - 1, 1, it, cm, +1);
            tfsf_apply<double>(MFD_EX, 1, 1, 1, 1, iz1, iz1, 0, it, ce, +1);
            tfsf_apply<T>(MFD_DX, 1, 1, 1, 1, iz1, iz1, 0, it, cd, +1);
            tfsf_apply<double>(MFD_HY, 1, 1, 1, 1, iz2, iz2, 3, it, cm, -1);
            tfsf_apply<double>(MFD_EX, 1, 1, 1, 1, iz2, iz2, 2, it, ce, -1);
            tfsf_apply<T>(MFD_DX, 1, 1, 1, 1, iz2, iz2, 2, it, cd, -1);
        }
    }

    // write_tfsf_record (sources.jl:372-384, 534-550, 839-877)
    void rec_copy(int comp, int xa, int xb, int ya, int yb, int za, int zb, int k, int64_t it) {
        T* dst = rec[k].data() + (size_t)(it - 1) * rec_len[k];
        size_t n = 0;
        for (int iz = za; iz <= zb; ++iz)
            for (int iy = ya; iy <= yb; ++iy)
                for (int ix = xa; ix <= xb; ++ix) dst[n++] = F[comp][id(ix - 1, iy - 1, iz - 1)];
    }

    void write_record(int64_t it) {
        int ix1 = ri1[0], iy1 = ri1[1], iz1 = ri1[2], ix2 = ri2[0], iy2 = ri2[1], iz2 = ri2[2];
        if (ndim == 3) {
            rec_copy(MFD_HY, ix1 - 1, ix1 - 1, iy1, iy2, iz1, iz2 - 1, 0, it);
            rec_copy(MFD_HZ, ix1 - 1, ix1 - 1, iy1, iy2 - 1, iz1, iz2, 1, it);
            rec_copy(MFD_EY, ix1, ix1, iy1, iy2 - 1, iz1, iz2, 2, it);
            rec_copy(MFD_EZ, ix1, ix1, iy1, iy2, iz1, iz2 - 1, 3, it);
            rec_copy(MFD_HY, ix2, ix2, iy1, iy2, iz1, iz2 - 1, 4, it);
            rec_copy(MFD_HZ, ix2, ix2, iy1, iy2 - 1, iz1, iz2, 5, it);
            rec_copy(MFD_EY, ix2, ix2, iy1, iy2 - 1, iz1, iz2, 6, it);
            rec_copy(MFD_EZ, ix2, ix2, iy1, iy2, iz1, iz2 - 1, 7, it);
            rec_copy(MFD_HX, ix1, ix2, iy1 - 1, iy1 - 1, iz1, iz2 - 1, 8, it);
            rec_copy(MFD_HZ, ix1, ix2 - 1, iy1 - 1, iy1 - 1, iz1, iz2, 9, it);
            rec_copy(MFD_EX, ix1, ix2 - 1, iy1, iy1, iz1, iz2, 10, it);
            rec_copy(MFD_EZ, ix1, ix2, iy1, iy1, iz1, iz2 - 1, 11, it);
            rec_copy(MFD_HX, ix1, ix2, iy2, iy2, iz1, iz2 - 1, 12, it);
            rec_copy(MFD_HZ, ix1, ix2 - 1, iy2, iy2, iz1, iz2, 13, it);
            rec_copy(MFD_EX, ix1, ix2 - 1, iy2, iy2, iz1, iz2, 14, it);
            rec_copy(MFD_EZ, ix1, ix2, iy2, iy2, iz1, iz2 - 1, 15, it);
            rec_copy(MFD_HX, ix1, ix2, iy1, iy2 - 1, iz1 - 1, iz1 - 1, 16, it);
            rec_copy(MFD_HY, ix1, ix2 - 1, iy1, iy2, iz1 - 1, iz1 - 1, 17, it);
            rec_copy(MFD_EX, ix1, ix2 - 1, iy1, iy2, iz1, iz1, 18, it);
            rec_copy(MFD_EY, ix1, ix2, iy1, iy2 - 1, iz1, iz1, 19, it);
            rec_copy(MFD_HX, ix1, ix2, iy1, iy2 - 1, iz2, iz2, 20, it);
            rec_copy(MFD_HY, ix1, ix2 - 1, iy1, iy2, iz2, iz2, 21, it);
            rec_copy(MFD_EX, ix1, ix2 - 1, iy1, iy2, iz2, iz2, 22, it);
            rec_copy(MFD_EY, ix1, ix2, iy1, iy2 - 1, iz2, iz2, 23, it);
        } else if (ndim == 2 && pol == MFD_POL_EY) {
            rec_copy(MFD_HZ, ix1 - 1, ix1 - 1, 1, 1, iz1, iz2, 0, it);
            rec_copy(MFD_EY, ix1, ix1, 1, 1, iz1, iz2, 1, it);
            rec_copy(MFD_HZ, ix2, ix2, 1, 1, iz1, iz2, 2, it);
            rec_copy(MFD_EY, ix2, ix2, 1, 1, iz1, iz2, 3, it);
            rec_copy(MFD_HX, ix1, ix2, 1, 1, iz1 - 1, iz1 - 1, 4, it);
            rec_copy(MFD_EY, ix1, ix2, 1, 1, iz1, iz1, 5, it);
            rec_copy(MFD_HX, ix1, ix2, 1, 1, iz2, iz2, 6, it);
            rec_copy(MFD_EY, ix1, ix2, 1, 1, iz2, iz2, 7, it);
        } else if (ndim == 2) {
            rec_copy(MFD_HY, ix1 - 1, ix1 - 1, 1, 1, iz1, iz2 - 1, 0, it);
            rec_copy(MFD_EZ, ix1, ix1, 1, 1, iz1, iz2 - 1, 1, it);
            rec_copy(MFD_HY, ix2, ix2, 1, 1, iz1, iz2 - 1, 2, it);
            rec_copy(MFD_EZ, ix2, ix2, 1, 1, iz1, iz2 - 1, 3, it);
            rec_copy(MFD_HY, ix1, ix2 - 1, 1, 1, iz1 - 1, iz1 - 1, 4, it);
            rec_copy(MFD_EX, ix1, ix2 - 1, 1, 1, iz1, iz1, 5, it);
            rec_copy(MFD_HY, ix1, ix2 - 1, 1, 1, iz2, iz2, 6, it);
            rec_copy(MFD_EX, ix1, ix2 - 1, 1, 1, iz2, iz2, 7, it);
        } else {
            rec_copy(MFD_HY, 1, 1, 1, 1, iz1 - 1, iz1 - 1, 0, it);
            rec_copy(MFD_EX, 1, 1, 1, 1, iz1, iz1, 1, it);
            rec_copy(MFD_HY, 1, 1, 1, 1, iz2, iz2, 2, it);
            rec_copy(MFD_EX, 1, 1, 1, 1, iz2, iz2, 3, it);
        }
    }

    // Julia's sum over an array (Base.mapreduce_impl, pairwise_blocksize 1024): fewer than 16
    // terms, or a block of at most 1024, are added left to right; longer ranges split at
    // their midpoint and add the two halves' sums.  The leaf loop of Base carries @simd, which
    // lets LLVM reassociate inside a block for the host's vector width, so a Julia run can
    // differ from this tree in the last bits of a summed monitor; the tree above the blocks
    // is the same.  val(p) gives the p-th term.
    template <typename U, typename V>
    static U julia_sum(size_t lo, size_t hi, const V& val) {   // terms [lo, hi)
        const size_t n = hi - lo;
        if (n == 0) return U(0);
        if (n <= 1024) {
            U v = val(lo);
            for (size_t p = lo + 1; p < hi; ++p) v = v + val(p);
            return v;
        }
        const size_t mid = lo + (n - 1) / 2 + 1;   // ifirst + (ilast - ifirst) >> 1, inclusive
        return julia_sum<U>(lo, mid, val) + julia_sum<U>(mid, hi, val);
    }

    // update_monitor! (monitors.jl:59-69, 107-119, 161-179, 253-258, 299-305, 350-359) and
    // the DFT accumulation (dft.jl:36-51).
    void update_monitors(int64_t it) {
        for (auto& M : mons) {
            size_t np = M.cells.size();
            for (int comp = 0; comp < 9; ++comp) {
                if (!has_comp(comp) || is_D(comp)) continue;
                const std::vector<T>& FC = F[comp];
                if (M.kind == MFD_MON_FIELD) {
                    if (M.sum) {   // sum(field.X[inds]) (monitors.jl:62-63, 110-112, 164-169)
                        M.rec[comp][it - 1] = julia_sum<T>(0, np, [&](size_t p) { return FC[M.cells[p]]; });
                    } else {
                        T* dst = M.rec[comp].data() + (size_t)(it - 1) * np;
                        for (size_t p = 0; p < np; ++p) dst[p] = FC[M.cells[p]];
                    }
                } else {
                    const double* ph = M.phasor.data() + (size_t)(it - 1) * M.nw * 2;
                    double dtd = (double)dt;
                    for (int iw = 0; iw < M.nw; ++iw) {
                        double er = ph[2 * iw], ei = ph[2 * iw + 1];
                        if (M.sum) {   // 2 * sum(F * exp(...)) * dt (dft.jl:40)
                            const double sr = julia_sum<double>(0, np, [&](size_t p) { return (double)FC[M.cells[p]] * er; });
                            const double si = julia_sum<double>(0, np, [&](size_t p) { return (double)FC[M.cells[p]] * ei; });
                            std::complex<double>& S = M.S[comp][iw];
                            S = std::complex<double>(S.real() + (2 * sr) * dtd, S.imag() + (2 * si) * dtd);
                        } else {
                            double tr = (2 * er) * dtd, ti = (2 * ei) * dtd;
                            std::complex<double>* S = M.S[comp].data() + (size_t)iw * np;
                            for (size_t p = 0; p < np; ++p) {
                                double f = (double)FC[M.cells[p]];
                                S[p] = std::complex<double>(S[p].real() + f * tr, S[p].imag() + f * ti);
                            }
                        }
                    }
                }
            }
        }
    }

    // update_integral_variables! (outputs.jl:182-191, 318-327, 475-485)
    void update_integrals() {
#pragma omp parallel for schedule(static)
        for (long long c = 0; c < (long long)N; ++c) {
            if (ndim == 3) {
                T Hx = F[MFD_HX][c], Hy = F[MFD_HY][c], Hz = F[MFD_HZ][c];
                T Ex = F[MFD_EX][c], Ey = F[MFD_EY][c], Ez = F[MFD_EZ][c];
                T a = Ey * Hz - Ez * Hy, b = Ez * Hx - Ex * Hz, d = Ex * Hy - Ey * Hx;
                Sa[c] += std::sqrt(a * a + b * b + d * d) * dt;
                if (isgeometry) E2[c] += (Ex * Ex + Ey * Ey + Ez * Ez) * dt;
            } else if (ndim == 2 && pol == MFD_POL_EY) {
                // the 3-D norm with Ex = Ez = Hy = 0: a = Ey Hz, b = 0, d = -Ey Hx
                T Hx = F[MFD_HX][c], Hz = F[MFD_HZ][c], Ey = F[MFD_EY][c];
                T a = Ey * Hz, d = 0 - Ey * Hx;
                Sa[c] += std::sqrt(a * a + d * d) * dt;
                if (isgeometry) E2[c] += Ey * Ey * dt;
            } else if (ndim == 2) {
                T Hy = F[MFD_HY][c], Ex = F[MFD_EX][c], Ez = F[MFD_EZ][c];
                T a = -Ez * Hy, b = Ex * Hy;
                Sa[c] += std::sqrt(a * a + b * b) * dt;
                if (isgeometry) E2[c] += (Ex * Ex + Ez * Ez) * dt;
            } else {
                T Hy = F[MFD_HY][c], Ex = F[MFD_EX][c];
                T a = Ex * Hy;
                Sa[c] += std::sqrt(a * a) * dt;
                if (isgeometry) E2[c] += Ex * Ex * dt;
            }
        }
    }

    int check_finite(int64_t it) {
        const std::vector<T>& Ex = F[pol == MFD_POL_EY ? MFD_EY : MFD_EX];   // Ey when the model has no Ex
        bool nan = false, inf = false;
        for (size_t c = 0; c < N; ++c) {
            if (std::isnan(Ex[c])) nan = true;
            else if (std::isinf(Ex[c])) inf = true;
        }
        if (nan || inf) {
            bad_step = it;
            bad_kind = (nan ? 1 : 0) | (inf ? 2 : 0);
            err = nan ? "Something went wrong. I found NaN field values."
                      : "Something went wrong. I found Inf field values.";
            return MFD_ERR_NONFINITE;
        }
        return MFD_OK;
    }

    // One iteration of the solve! loop (models.jl:199-234) minus file output.
    int run(int64_t a, int64_t b) override {
        if (bad_step) { err = "model holds non-finite fields"; return MFD_ERR_NONFINITE; }
        if (a != done + 1 || b < a - 1 || b > nt) { err = "steps must be consecutive and within 1..Nt"; return MFD_ERR_INVALID; }
        for (int64_t it = a; it <= b; ++it) {
            // step! (models.jl:125-132)
            if (ndim == 3) { update_H3(); update_E3(); }
            else if (ndim == 2 && pol == MFD_POL_EY) { update_H2ey(); update_E2ey(); }
            else if (ndim == 2) { update_H2(); update_E2(); }
            else { update_H1(); update_E1(); }
            for (size_t s = 0; s <= srcs.size(); ++s) {
                if (tfsf && (int)s == tfsf_order) add_tfsf(it);
                if (s < srcs.size()) add_point_source(srcs[s], it);
            }
            done = it;
            int st = check_finite(it);
            if (st) return st;
            update_monitors(it);
            update_integrals();
            if (record) write_record(it);
        }
        return MFD_OK;
    }

    int read_geometry(uint8_t* dst) override {
        for (size_t i = 0; i < N; ++i) dst[i] = (uint8_t)geometry[i];
        return MFD_OK;
    }

    int read_field(int comp, void* dst) override {
        if (comp < 0 || comp > 8 || !has_comp(comp)) { err = "bad component"; return MFD_ERR_INVALID; }
        std::memcpy(dst, F[comp].data(), N * sizeof(T));
        return MFD_OK;
    }
    int write_field(int comp, const void* src) override {
        if (comp < 0 || comp > 8 || !has_comp(comp)) { err = "bad component"; return MFD_ERR_INVALID; }
        std::memcpy(F[comp].data(), src, N * sizeof(T));
        return MFD_OK;
    }
    int read_integral(int which, void* dst) override {
        if (which == MFD_INT_SA) std::memcpy(dst, Sa.data(), N * sizeof(T));
        else if (which == MFD_INT_E2) {
            if (isgeometry) std::memcpy(dst, E2.data(), N * sizeof(T));
            else std::memset(dst, 0, N * sizeof(T));
        } else if (which == MFD_INT_JE) {
            if (isplasma) std::memcpy(dst, JE.data(), N * sizeof(T));
            else std::memset(dst, 0, N * sizeof(T));
        } else if (which == MFD_INT_RHO) {
            // rho_end (outputs.jl:54-59): sum over materials of rho .* rho0
            double* r = (double*)dst;
            for (size_t c = 0; c < N; ++c) r[c] = 0;
            for (auto& M : mats) {
                if (!M.plasma) continue;
                for (size_t c = 0; c < N; ++c) r[c] = r[c] + (double)(M.rho[c] * M.rho0);
            }
        } else { err = "bad integral"; return MFD_ERR_INVALID; }
        return MFD_OK;
    }
    int read_monitor(int m, int comp, void* dst) override {
        if (m < 0 || m >= (int)mons.size() || comp < 0 || comp > 8 || !has_comp(comp) || is_D(comp)) {
            err = "bad monitor or component"; return MFD_ERR_INVALID;
        }
        const Monitor<T>& M = mons[m];
        if (M.kind == MFD_MON_FIELD) std::memcpy(dst, M.rec[comp].data(), M.rec[comp].size() * sizeof(T));
        else std::memcpy(dst, M.S[comp].data(), M.S[comp].size() * sizeof(std::complex<double>));
        return MFD_OK;
    }
    int read_record(int k, void* dst) override {
        if (!record || k < 0 || k >= 24 || rec[k].empty()) { err = "no such record array"; return MFD_ERR_INVALID; }
        std::memcpy(dst, rec[k].data(), rec[k].size() * sizeof(T));
        return MFD_OK;
    }
    int64_t record_size(int k) const override {
        if (!record || k < 0 || k >= 24) return 0;
        return (int64_t)rec[k].size();
    }
    void status(int64_t* d, int64_t* b, int32_t* k) const override {
        if (d) *d = done;
        if (b) *b = bad_step;
        if (k) *k = bad_kind;
    }
};

int validate(const mfd_desc* d) {
    if (!d) { g_create_error = "null descriptor"; return MFD_ERR_INVALID; }
    if (d->abi_version != MFD_ABI_VERSION) { g_create_error = "ABI version mismatch"; return MFD_ERR_INVALID; }
    if (d->ndim < 1 || d->ndim > 3 || d->nx < 1 || d->ny < 1 || d->nz < 1 || d->nt < 1) { g_create_error = "bad dims"; return MFD_ERR_INVALID; }
    if (d->ndim == 1 && (d->nx != 1 || d->ny != 1)) { g_create_error = "1-D model needs nx = ny = 1"; return MFD_ERR_INVALID; }
    if (d->ndim == 2 && d->ny != 1) { g_create_error = "2-D model needs ny = 1"; return MFD_ERR_INVALID; }
    if (d->dtype != MFD_F32 && d->dtype != MFD_F64) { g_create_error = "bad dtype"; return MFD_ERR_INVALID; }
    if (d->polarization != MFD_POL_HY && (d->ndim != 2 || d->polarization != MFD_POL_EY)) {
        g_create_error = "polarization must be MFD_POL_HY, or MFD_POL_EY for a 2-D model"; return MFD_ERR_INVALID;
    }
    if (d->tfsf.enabled) {
        for (int a = 0; a < 3; ++a) {
            if (d->ndim == 3 || (d->ndim == 2 && a != 1) || (d->ndim == 1 && a == 2)) {
                int n = a == 0 ? d->nx : a == 1 ? d->ny : d->nz;
                if (d->tfsf.i1[a] < 2 || d->tfsf.i2[a] > n || d->tfsf.i1[a] >= d->tfsf.i2[a]) {
                    g_create_error = "TFSF box must satisfy 2 <= i1 < i2 <= n on every axis"; return MFD_ERR_INVALID;
                }
            }
        }
    }
    if (d->tfsf_record) {
        for (int a = 0; a < 3; ++a) {
            if (d->ndim == 3 || (d->ndim == 2 && a != 1) || (d->ndim == 1 && a == 2)) {
                int n = a == 0 ? d->nx : a == 1 ? d->ny : d->nz;
                if (d->rec_i1[a] < 2 || d->rec_i2[a] > n || d->rec_i1[a] >= d->rec_i2[a]) {
                    g_create_error = "record box must satisfy 2 <= i1 < i2 <= n on every axis"; return MFD_ERR_INVALID;
                }
            }
        }
    }
    return MFD_OK;
}

}  // namespace

extern "C" {

int oracle_create(const mfd_desc* d, void** out) {
    *out = nullptr;
    int st = validate(d);
    if (st) return st;
    std::unique_ptr<OracleBase> o;
    int r = MFD_OK;
    try {
        if (d->dtype == MFD_F64) {
            auto p = std::make_unique<Oracle<double, double>>();
            r = p->init(d); if (r) g_create_error = p->err;
            o = std::move(p);
        } else if (d->rho_fp64) {
            auto p = std::make_unique<Oracle<float, double>>();
            r = p->init(d); if (r) g_create_error = p->err;
            o = std::move(p);
        } else {
            auto p = std::make_unique<Oracle<float, float>>();
            r = p->init(d); if (r) g_create_error = p->err;
            o = std::move(p);
        }
    } catch (const std::bad_alloc&) {
        g_create_error = "out of host memory";
        return MFD_ERR_OOM;
    }
    if (r) return r;
    *out = o.release();
    return MFD_OK;
}

void oracle_destroy(void* h) { delete (OracleBase*)h; }
int oracle_run(void* h, int64_t a, int64_t b) { return ((OracleBase*)h)->run(a, b); }
int oracle_read_field(void* h, int32_t comp, void* dst) { return ((OracleBase*)h)->read_field(comp, dst); }
int oracle_read_geometry(void* h, uint8_t* dst) { return ((OracleBase*)h)->read_geometry(dst); }
int oracle_write_field(void* h, int32_t comp, const void* src) { return ((OracleBase*)h)->write_field(comp, src); }
int oracle_read_integral(void* h, int32_t which, void* dst) { return ((OracleBase*)h)->read_integral(which, dst); }
int oracle_read_monitor(void* h, int32_t m, int32_t comp, void* dst) { return ((OracleBase*)h)->read_monitor(m, comp, dst); }
int oracle_read_tfsf_record(void* h, int32_t k, void* dst) { return ((OracleBase*)h)->read_record(k, dst); }
int64_t oracle_tfsf_record_size(void* h, int32_t k) { return ((OracleBase*)h)->record_size(k); }
int oracle_status(void* h, int64_t* d, int64_t* b, int32_t* k) { ((OracleBase*)h)->status(d, b, k); return MFD_OK; }
const char* oracle_last_error(void* h) { return ((OracleBase*)h)->err.c_str(); }
const char* oracle_create_error(void) { return g_create_error.c_str(); }

// The ionisation-rate table functor on its own (for the tests that pin it to the
// reference's IonizationRate semantics): x, y are the table's log10 knots as passed in
// mfd_material.rate_x / rate_y, cast to float when f32 != 0 as the library does.
int oracle_eval_rate_table(const double* x, const double* y, int32_t n, int32_t f32, const double* I, double* out,
                           int64_t count) {
    if (!x || !y || n < 2 || !I || !out || count < 0) return MFD_ERR_INVALID;
    if (f32) {
        std::vector<float> X(x, x + n), Y(y, y + n);
        for (int64_t k = 0; k < count; ++k) out[k] = (double)ionization_rate<float>(X.data(), Y.data(), (size_t)n, (float)I[k]);
    } else {
        for (int64_t k = 0; k < count; ++k) out[k] = ionization_rate<double>(x, y, (size_t)n, I[k]);
    }
    return MFD_OK;
}
int oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

}  // extern "C"
