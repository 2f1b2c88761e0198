/*
 * maxwellfdtd.h -- C ABI of the B200 FDTD time-stepper (libmaxwellfdtd_b200.so).
 *
 * This library replaces the time-step path of the Julia package MaxwellFDTD:
 *
 *   solve!(model; backend)         src/models.jl:166-242
 *     adapt(backend, model)        src/models.jl:183        -> mfd_create
 *     for it=1:Nt                  src/models.jl:199
 *       step!(model, it)           src/models.jl:125-132    -> mfd_run (chunks of steps)
 *         update_H!                src/models.jl:248-307, 450-536, 735-889
 *         update_E!                src/models.jl:310-444, 539-726, 895-1175
 *         add_source!              src/sources.jl:122-131, 235-244, 320-346, 469-497, 713-776
 *       NaN/Inf guard              src/models.jl:202-209    -> MFD_ERR_NONFINITE
 *       update_monitors!           src/outputs.jl:21-30     -> on-device monitors
 *       update_integral_variables! src/outputs.jl:182-191, 318-327, 475-485 (fused)
 *       write_tfsf_record          src/sources.jl:372-384, 534-550, 839-877 (on-device record)
 *     write_fields / write_monitors / write_integral_variables read back through
 *     mfd_read_field / mfd_read_monitor / mfd_read_integral.
 *
 * Conventions
 *  - Grid arrays are dense, x fastest: cell (ix,iy,iz) (0-based) is at ix + nx*(iy + ny*iz).
 *    This is the column-major layout of the reference's Julia arrays, so a Julia Array
 *    passes with no transpose.  A 1-D model has nx = ny = 1 and uses z; a 2-D model
 *    has ny = 1 and uses the x-z plane (reference Grid1D / Grid2D, src/grids.jl:182-258).
 *  - Bulk arrays (fields, TFSF incident data, monitor outputs) are in the handle's
 *    element type T (float for MFD_F32, double for MFD_F64).  Scalar coefficients and
 *    the coefficient tables are passed as double and cast to T inside the library, as
 *    the reference's adapt_storage does after computing them in Float64
 *    (src/backends.jl:27-41).
 *  - Step indices are 1-based, as in the reference loop `for it=1:Nt`.
 *  - Every call returns an int status (MFD_OK = 0).  Nothing aborts or exits.  Details of
 *    the last failure on a handle are in mfd_last_error().
 *  - A handle is used by one host thread at a time.  Distinct handles may be driven from
 *    different threads concurrently; each owns its CUDA stream and device memory.
 */
#ifndef MAXWELLFDTD_H
#define MAXWELLFDTD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define MFD_API __attribute__((visibility("default")))
#else
#define MFD_API
#endif

#define MFD_ABI_VERSION 2

/* ---- status codes ------------------------------------------------------------------ */
enum {
    MFD_OK = 0,
    MFD_ERR_INVALID = 1,    /* bad descriptor or argument                              */
    MFD_ERR_OOM = 2,        /* device or host allocation failed                        */
    MFD_ERR_CUDA = 3,       /* a CUDA runtime call failed                              */
    MFD_ERR_NONFINITE = 4,  /* NaN or Inf found in Ex (reference models.jl:202-209)    */
    MFD_ERR_TIMEOUT = 5,    /* a bounded host wait ran out                             */
    MFD_ERR_ADMISSION = 6,  /* job does not fit the device-memory budget               */
    MFD_ERR_NODEVICE = 7    /* no CUDA device available                                */
};

/* ---- element types ---------------------------------------------------------------- */
enum { MFD_F32 = 0, MFD_F64 = 1 };

/* ---- arithmetic of the field updates (mfd_desc.mode) ---------------------------------
 * MFD_MODE_EXACT: every cell update in the reference's operation order with no fused
 *   multiply-add, IEEE square roots and divisions (a division by a grid constant or a CPML
 *   kappa takes a correction step that the library verifies, per divisor, to give the IEEE
 *   quotient for every single-precision significand): fields are bit-identical to a CPU
 *   run of the same order in the same precision.
 * MFD_MODE_FAST: the tolerance mode.  Derivatives multiply by the reciprocal of the grid
 *   constant or kappa, the H/D/CPML/running-sum updates are fused multiply-adds and the
 *   Poynting norm uses the hardware reciprocal square root (single precision).  Results
 *   stay within relative L2 1e-5 (FP32) / 1e-12 (FP64) of the exact order; the material
 *   response (ADE, Kerr, plasma), sources and monitors keep the exact arithmetic.  A batch
 *   takes members of either mode, each with its own arithmetic. */
enum { MFD_MODE_EXACT = 0, MFD_MODE_FAST = 1 };

/* ---- boundary conditions: the reference's bc2int codes (src/models.jl:1199-1217) ---- */
enum { MFD_BC_PERIODIC = 1, MFD_BC_DIRICHLET = 2, MFD_BC_NEUMANN = 3 };

/* ---- faces: index into bc[] and pml[] ----------------------------------------------- */
enum { MFD_XL = 0, MFD_XR = 1, MFD_YL = 2, MFD_YR = 3, MFD_ZL = 4, MFD_ZR = 5 };

/* ---- field components (the reference Field3D field order, src/fields.jl:67-90) ------ */
enum {
    MFD_HX = 0, MFD_HY = 1, MFD_HZ = 2,
    MFD_DX = 3, MFD_DY = 4, MFD_DZ = 5,
    MFD_EX = 6, MFD_EY = 7, MFD_EZ = 8
};

/* ---- the 2-D field set (mfd_desc.polarization; ignored by 1-D and 3-D models) --------
 * MFD_POL_HY: Hy, Dx, Dz, Ex, Ez -- the reference's Field2D (src/fields.jl:36-55).
 * MFD_POL_EY: Hx, Hz, Dy, Ey -- the other polarisation of an x-z model, which the
 *   reference does not have.  Its updates are the reference's 3-D updates
 *   (src/models.jl:735-1162) with every y derivative zero, in the same operation order, so
 *   a run equals the Hx, Hz, Dy, Ey of a 3-D run with ny = 1 and periodic y bit for bit;
 *   Sa is that run's Poynting norm and the NaN/Inf guard reads Ey (there is no Ex). */
enum { MFD_POL_HY = 0, MFD_POL_EY = 1 };

/* ---- integral outputs (reference Output.Sa/E2, model.JE, rho_end: outputs.jl:46-65) -- */
enum { MFD_INT_SA = 0, MFD_INT_E2 = 1, MFD_INT_JE = 2, MFD_INT_RHO = 3 };

/* ---- sources ------------------------------------------------------------------------ */
enum { MFD_SRC_SOFT = 0, MFD_SRC_HARD = 1 };

/* ---- monitors ----------------------------------------------------------------------- */
enum { MFD_MON_FIELD = 0, MFD_MON_SPECTRAL = 1 };

/* ---- plasma ionisation-rate closures (reference Plasma.ionrate, models.jl:1117) ------ */
enum {
    MFD_RATE_NONE = 0,
    /* R(I) = 10^(order*log10(I) + log10c): the MPI form of
       examples/5_nonlinear_propagation/3D_plasma.jl:67.  order*log10(I) is evaluated in T,
       the sum and the power in double, as Julia's promotion does for that closure. */
    MFD_RATE_POWER = 1,
    /* log-log table, equally spaced log10(I) knots (IonizationRate.jl:13-52), in T. */
    MFD_RATE_TABLE = 2
};

/* ---- TFSF incident-data arrays ----------------------------------------------------------
 * 3-D: the 24 arrays of TFSFSource3D in its field order (src/sources.jl:556-587):
 *   face 1yz: incHy, incHz, incEy, incEz;  face 2yz: same;  face x1z: incHx, incHz, incEx,
 *   incEz;  face x2z: same;  face xy1: incHx, incHy, incEx, incEy;  face xy2: same.
 * 2-D: the 8 arrays of TFSFSource2D (sources.jl:390-403):
 *   1z: incHy, incEz; 2z: incHy, incEz; x1: incHy, incEx; x2: incHy, incEx.
 * 2-D, MFD_POL_EY: 1z: incHz, incEy; 2z: incHz, incEy; x1: incHx, incEy; x2: incHx, incEy,
 *   each over the face's Nzi + 1 (x faces) or Nxi + 1 (z faces) nodes, as the 3-D faces
 *   1yz / 2yz / xy1 / xy2 hold Hz, Ey and Hx, Ey.
 * 1-D: the 4 arrays of TFSFSource1D (sources.jl:272-279): incHy_1, incEx_1, incHy_2, incEx_2.
 * Each array is [nt][face extent] in T, the face extent laid out as in the reference
 * (column-major (a, b, Nt) => C order [nt][b][a]).
 *
 * An array may be passed in a compact form (mfd_tfsf.shape[k]), which the library expands
 * on the fly: the incident data of a plane wave along a grid axis vary along one face axis
 * or none, so [nt][b] or [nt] values describe the whole face for every step.  A face's
 * axes (a, b) are its two in-plane grid axes in x, y, z order (face 1yz: a = y, b = z;
 * x1z: a = x, b = z; xy1: a = x, b = y; a 2-D face has b of extent 1).
 *   MFD_INC_FULL    [nt][b][a]  every value (the reference's layout; the default)
 *   MFD_INC_ALONG_B [nt][b]     the same for every a (value (ia, ib) = v[ib])
 *   MFD_INC_ALONG_A [nt][a]     the same for every b (value (ia, ib) = v[ia])
 *   MFD_INC_UNIFORM [nt]        one value per step for the whole face
 * Device memory and upload then grow with nt times the compact extent only. */
#define MFD_TFSF_MAX_ARRAYS 24
enum { MFD_INC_FULL = 0, MFD_INC_ALONG_B = 1, MFD_INC_ALONG_A = 2, MFD_INC_UNIFORM = 3 };

/* One CPML layer profile (reference PMLLayer, src/pml.jl:46-121).  nb = 0: no layer. */
typedef struct mfd_pml_layer {
    int32_t ib;        /* 1-based boundary index (PMLLayer.ib)                       */
    int32_t nb;        /* number of grid points in the layer (PMLLayer.Nb)           */
    const double* K;   /* [nb] kappa                                                 */
    const double* A;   /* [nb]                                                       */
    const double* B;   /* [nb]                                                       */
} mfd_pml_layer;

/* Per-material update coefficients (reference MaterialStruct3D, src/materials.jl:335-483). */
typedef struct mfd_material {
    double Mh, Me, Md1, Md2;
    int32_t nq;                          /* ADE poles; 0 = no dispersion               */
    const double* Aq;                    /* [nq]                                       */
    const double* Bq;
    const double* Cq;
    int32_t kerr;                        /* iskerr                                     */
    double Mk2, Mk3;
    int32_t plasma;                      /* isplasma                                   */
    double Rava, ksi, rho0, Ap, Bp, Cp, Ma;
    int32_t rate_kind;                   /* MFD_RATE_*                                 */
    double rate_order, rate_log10c;      /* MFD_RATE_POWER                             */
    int32_t rate_n;                      /* MFD_RATE_TABLE: knots                      */
    const double* rate_x;                /* [rate_n] log10(I), equally spaced          */
    const double* rate_y;                /* [rate_n] log10(R)                          */
} mfd_material;

/* A soft or hard source (reference SoftSourceStruct / HardSourceStruct, sources.jl:41-244).
 * The host has already redirected E components to D with coeff = EPS0 (sources.jl:61-69).
 * The waveform is tabulated on the host in double: either wave[it][p] (general) or
 * amp[p] * gt[it] (separable). */
typedef struct mfd_source {
    int32_t kind;            /* MFD_SRC_SOFT / MFD_SRC_HARD                          */
    int32_t comp;            /* MFD_HX .. MFD_EZ                                     */
    double coeff;            /* soft sources: FC += coeff * w                        */
    int64_t npts;
    const int64_t* cells;    /* [npts] 0-based linear cell indices                   */
    const double* wave;      /* [nt][npts] or NULL                                   */
    const double* amp;       /* [npts] when wave == NULL                             */
    const double* gt;        /* [nt]   when wave == NULL                             */
} mfd_source;

/* TFSF replay source (reference TFSFSource{1,2,3}D + add_source!, sources.jl:272-776). */
typedef struct mfd_tfsf {
    int32_t enabled;
    int32_t order;           /* point sources applied before it (sources act in tuple
                                order, models.jl:128-130)                              */
    int32_t i1[3];           /* 1-based (ix1, iy1, iz1)                               */
    int32_t i2[3];           /* 1-based (ix2, iy2, iz2)                               */
    const void* inc[MFD_TFSF_MAX_ARRAYS];
    int32_t shape[MFD_TFSF_MAX_ARRAYS];   /* MFD_INC_* layout of inc[k] (0: full)   */
} mfd_tfsf;

/* Field or spectral monitor (reference monitors.jl:7-373, dft.jl:1-51). */
typedef struct mfd_monitor {
    int32_t kind;            /* MFD_MON_FIELD / MFD_MON_SPECTRAL                      */
    int32_t sum;             /* issum                                                 */
    int64_t npts;
    const int64_t* cells;    /* [npts] 0-based linear cell indices                    */
    int32_t nw;              /* spectral: number of frequencies                       */
    const double* phasor;    /* spectral: [nt][nw][2] = exp(-i w (t_it - tshift))     */
} mfd_monitor;

/* ---- analytic geometry evaluated on the device ------------------------------------------
 * The reference evaluates each material's geometry(x, y, z) at every grid point on the host
 * and writes the material index, later materials winning (src/util.jl:1-31,
 * src/models.jl:85-98).  For the shapes below the library builds the uint8 material map on
 * the device instead: shapes are applied in order (a later shape overwrites the cells it
 * covers), each writing its material index, and every test is the double-precision
 * expression written here, evaluated left to right with no fused multiply-add, at the grid
 * coordinates mfd_desc.coords -- so a host evaluating the same expression (numpy, Julia)
 * gets the same map bit for bit.  2-D grids use (x, z) and 1-D grids z only: the missing
 * coordinates are taken as 0.
 *   MFD_SHAPE_BALL       p = cx, cy, cz, r:
 *                        ((x-cx)*(x-cx) + (y-cy)*(y-cy)) + (z-cz)*(z-cz) <= r*r
 *   MFD_SHAPE_BOX        p = x0, x1, y0, y1, z0, z1:  x0 <= x <= x1 && y0 <= y <= y1 && z0 <= z <= z1
 *   MFD_SHAPE_ELLIPSOID  p = cx, cy, cz, ax, ay, az:
 *                        (((x-cx)/ax)*((x-cx)/ax) + ((y-cy)/ay)*((y-cy)/ay)) + ((z-cz)/az)*((z-cz)/az) <= 1
 *   MFD_SHAPE_CYLINDER   p = cx, cy, r, z0, z1 (axis along z):
 *                        (x-cx)*(x-cx) + (y-cy)*(y-cy) <= r*r && z0 <= z <= z1
 *   MFD_SHAPE_HALFSPACE  p = nx, ny, nz, d:  (nx*x + ny*y) + nz*z >= d
 *   MFD_SHAPE_ALL        every cell */
enum { MFD_SHAPE_BALL = 1, MFD_SHAPE_BOX = 2, MFD_SHAPE_ELLIPSOID = 3, MFD_SHAPE_CYLINDER = 4, MFD_SHAPE_HALFSPACE = 5,
       MFD_SHAPE_ALL = 6 };
typedef struct mfd_shape {
    int32_t kind;            /* MFD_SHAPE_*                                            */
    int32_t material;        /* 1..nmat, written into the cells the shape covers      */
    double p[8];             /* parameters by kind                                    */
} mfd_shape;

/* Complete description of one model (reference Model, src/models.jl:1-122). */
typedef struct mfd_desc {
    int32_t abi_version;     /* MFD_ABI_VERSION                                       */
    int32_t ndim;            /* 1, 2 or 3                                             */
    int32_t dtype;           /* MFD_F32 / MFD_F64                                     */
    int32_t nx, ny, nz;
    double dx, dy, dz;
    double dt;               /* time step (Float64 value; cast to T inside)           */
    int64_t nt;              /* number of steps Nt                                    */
    int32_t bc[6];           /* MFD_BC_* per face                                     */
    mfd_pml_layer pml[6];    /* per face                                              */
    double Mh0, Me0, Md10, Md20;   /* vacuum coefficients (models.jl:111-114)         */
    const uint8_t* geometry; /* [nx*ny*nz] material index, 0 = vacuum; NULL = vacuum  */
    int32_t nmat;            /* materials 1..nmat                                     */
    const mfd_material* mats;
    int32_t rho_fp64;        /* plasma density rho/drho kept in double for MFD_F32     */
    int32_t nsrc;
    const mfd_source* srcs;
    mfd_tfsf tfsf;
    int32_t nmon;
    const mfd_monitor* mons;
    int32_t tfsf_record;     /* record incident faces (prepare/write_tfsf_record)     */
    int32_t rec_i1[3];       /* 1-based record box                                   */
    int32_t rec_i2[3];
    int32_t device;          /* CUDA device ordinal                                   */
    int32_t mode;            /* MFD_MODE_EXACT / MFD_MODE_FAST                         */
    int32_t nshape;          /* shapes evaluated on the device (geometry must be NULL) */
    const mfd_shape* shapes;
    const double* coords[3]; /* grid coordinates x[nx], y[ny], z[nz] (for the shapes)  */
    int32_t polarization;    /* 2-D field set: MFD_POL_HY (0) or MFD_POL_EY            */
} mfd_desc;

typedef struct mfd_handle mfd_handle;

/* Model setup and device upload (replaces adapt(backend, model), models.jl:183). */
MFD_API int mfd_create(const mfd_desc* desc, mfd_handle** out);
MFD_API void mfd_destroy(mfd_handle* h);

/* Run steps it_first..it_last (1-based, inclusive, consecutive with the previous call).
 * Per step: update_H!, update_E!, add_source! for each source, then monitors, the
 * integral sums and the TFSF record -- the reference's per-step order
 * (models.jl:125-132, 199-234).  The NaN/Inf guard of models.jl:202-209 is evaluated on
 * the device; MFD_ERR_NONFINITE is returned at the end of the call with the first bad
 * step in mfd_status(). */
MFD_API int mfd_run(mfd_handle* h, int64_t it_first, int64_t it_last);

/* Number of steps completed and the first step whose Ex held NaN (bit 0) or Inf (bit 1). */
MFD_API int mfd_status(const mfd_handle* h, int64_t* steps_done, int64_t* bad_step, int32_t* bad_kind);

/* The material index map as the library holds it (nx*ny*nz bytes, x fastest): the
 * descriptor's geometry, or the map built on the device from its shapes. */
MFD_API int mfd_read_geometry(mfd_handle* h, uint8_t* dst);

/* Dense field component (MFD_HX..MFD_EZ) to/from host memory, nx*ny*nz elements of T. */
MFD_API int mfd_read_field(mfd_handle* h, int32_t comp, void* dst);
MFD_API int mfd_write_field(mfd_handle* h, int32_t comp, const void* src);

/* Integral outputs: Sa, E2, JE as nx*ny*nz of T; rho_end (sum over plasma materials of
 * rho*rho0) as nx*ny*nz double. */
MFD_API int mfd_read_integral(mfd_handle* h, int32_t which, void* dst);

/* mfd_read_integral without any device memory allocation.  No counterpart in the
 * reference (its integral outputs are plain arrays of the model).
 *
 * For callers that cannot allocate device memory when they read results: a host program
 * whose GPU memory is held by another allocator's pool (a framework's caching allocator
 * that reserved most of HBM, so cudaMalloc fails), or a serving loop that must not call
 * cudaMalloc/cudaFree between steps (they can synchronise the device and stall work on
 * other streams).  mfd_read_integral allocates a grid-sized temporary for JE and rho_end;
 * this entry point stages them through a fixed buffer inside the library instead -- a
 * device array of MFD_NOALLOC_SCRATCH_BYTES (16 MiB) -- a few z-planes at a time.  Sa and
 * E2 are copied straight from their arrays, as by mfd_read_integral.
 *
 * Limit: one z-plane (nx*ny elements; T for JE, double for rho_end) must fit in the
 * buffer, else MFD_ERR_INVALID with both sizes in mfd_last_error().
 * Nothing in the buffer has to start at zero: each call writes every element it copies out.
 * The buffer is shared by all handles on a device: calls that overlap in time on the same
 * device race on it, so serialise them.  Each call looks up the buffer's device address on
 * the current device; the first lookup on a device is the set-up (it makes the driver load
 * the library's device globals): make that first call before any stream capture on that
 * device.  A model without plasma returns zeros for JE and rho_end without touching the
 * device, whatever its plane size, as mfd_read_integral does. */
#define MFD_NOALLOC_SCRATCH_BYTES (16u << 20)
MFD_API int mfd_read_integral_noalloc(mfd_handle* h, int32_t which, void* dst);

/* Field snapshots taken during mfd_run (the frames write_fields saves at the output steps,
 * src/outputs.jl:156-179).  After each of the nsteps listed steps (1-based, increasing, after
 * the model's current step) the ncomp listed components (MFD_HX..MFD_EZ) are copied on the
 * device into a staging slot and from there to dst on a copy stream, while the following
 * steps run.  dst holds nsteps x ncomp x (nx*ny*nz) elements of T, frame f component k at
 * element (f*ncomp + k)*nx*ny*nz, each dense with x fastest; page-locked memory reaches full
 * DMA speed.  A frame is complete when the mfd_run call that ran its step returns.  Two
 * staging slots of ncomp fields are allocated on the device at the first call.  nsteps = 0
 * clears the list. */
MFD_API int mfd_set_snapshots(mfd_handle* h, int32_t ncomp, const int32_t* comps, int64_t nsteps,
                              const int64_t* steps, void* dst);

/* Monitor m, component comp.  Field monitor: T [nt][npts] ([nt] when sum).  Spectral
 * monitor: double complex [nw][npts] ([nw] when sum) as interleaved (re, im). */
MFD_API int mfd_read_monitor(mfd_handle* h, int32_t m, int32_t comp, void* dst);

/* TFSF record array k (same order and layout as mfd_tfsf.inc), T [nt][face extent]. */
MFD_API int mfd_read_tfsf_record(mfd_handle* h, int32_t k, void* dst);
/* Element count of TFSF array k for the record box (0 if k is unused). */
MFD_API int64_t mfd_tfsf_record_size(const mfd_handle* h, int32_t k);

/* ---- batches of 2-D and 3-D models -----------------------------------------------------
 * No counterpart in the reference, which runs one model per solve! call.  A batch steps
 * many independent 2-D and 3-D single-precision models together: each half-step of all
 * members is a persistent launch over a table of (member, tile) pairs (one for the 2-D and
 * one for the 3-D members), and a CUDA graph of several steps is replayed, so hundreds of
 * small models of different sizes do not each pay a handful of launches per step.  A member
 * is an ordinary handle (mfd_create, 2-D or 3-D, MFD_F32, rho_fp64 = 1) with any sources
 * (point, TFSF replay) and monitors, but no TFSF recording and no field snapshots; the batch
 * runs its steps
 * done+1 .. it_last exactly as mfd_run(h, done+1, it_last) would, with bit-identical results,
 * and then retires it: mfd_status / mfd_read_* work on it again.  Until it retires, the
 * caller must not run, read, write or destroy the handle (mfd_run returns MFD_ERR_INVALID).
 * Members join at any time (mfd_batch_add between mfd_batch_run calls), each with its own
 * step count; the persistent launches skip members whose window has ended. */
typedef struct mfd_batch mfd_batch;
MFD_API int mfd_batch_create(int32_t device, mfd_batch** out);
MFD_API void mfd_batch_destroy(mfd_batch* b);
MFD_API int mfd_batch_add(mfd_batch* b, mfd_handle* h, int64_t it_last);
/* Advance every member by up to max_steps steps; members that reach their last step are
 * retired.  n_active receives the number of members still running. */
MFD_API int mfd_batch_run(mfd_batch* b, int64_t max_steps, int32_t* n_active);
/* Tile shape of the persistent launches (tile_x a multiple of 32, tile_x*tile_z <= 512;
 * 0, 0 = autotune: the first graph replays try candidate shapes and keep the cheapest per
 * cell-update -- results do not depend on the shape) and steps per graph (0 = keep). */
MFD_API int mfd_batch_config(mfd_batch* b, int32_t tile_x, int32_t tile_z, int32_t graph_steps);
/* Current tile shape, device time of all mfd_batch_run calls (CUDA events), cell-updates and
 * kernel launches (graph nodes included) so far. */
MFD_API int mfd_batch_info(const mfd_batch* b, int32_t* tile_x, int32_t* tile_z, double* device_ms,
                           int64_t* cell_updates, int64_t* launches);
MFD_API const char* mfd_batch_last_error(const mfd_batch* b);

/* ---- model state ------------------------------------------------------------------------
 * The state a run carries from one step to the next, beyond the nine field components: the
 * running sums Sa and E2, the CPML psi arrays of every face (the reference's PML struct,
 * src/pml.jl:227-304), the polarisation of every dispersive material (P, oldP1 of
 * src/materials.jl:424-426; oldP2 is not needed), the plasma state (rho, drho, the plasma
 * currents, Pa, JE), the monitors' records and DFT accumulators, the TFSF record arrays,
 * the NaN/Inf flags and the number of steps done.  mfd_read_state copies it into one host
 * image of mfd_state_size() bytes; mfd_write_state loads such an image into a handle created
 * from the same descriptor (same grid, precision, materials, CPML, sources and monitors --
 * checked against a layout hash in the image), after which mfd_run continues from the
 * image's step exactly as the run it was taken from would have continued.  The image's
 * layout is the library's own (not a file format).  Writing clears any pending field
 * snapshots.  Both calls synchronise the handle's stream; neither may be used on a handle
 * that a batch is stepping.  Uses: checkpoint and resume, moving a model between devices,
 * and letting a serving loop evict a model from device memory and restore it later. */
MFD_API int64_t mfd_state_size(const mfd_handle* h);
MFD_API int mfd_read_state(mfd_handle* h, void* dst, int64_t bytes);
MFD_API int mfd_write_state(mfd_handle* h, const void* src, int64_t bytes);

/* ---- serving ----------------------------------------------------------------------------
 * No counterpart in the reference, which runs one solve! at a time.  A server solves a stream
 * of requests on one device.  mfd_server_submit queues a model descriptor; the server admits
 * queued requests in arrival order when the request's device-memory footprint (computed from
 * the descriptor before anything is allocated, mfd_server_footprint) fits the budget next to
 * the admitted requests and fewer than max_active requests are computing, and uploads it.
 * 2-D (first field set, MFD_POL_HY) and small 3-D (at most 2^20 cells) single-precision
 * requests (either mode) with rho_fp64 and no TFSF recording join one running batch (mfd_batch_*), which takes new
 * members between its runs of steps (continuous batching); every other request runs as a
 * solo lane on its own host thread and stream, at most max_solo at a time.  A request that
 * waits only for a solo lane does not hold back batch requests behind it; one that waits for
 * memory does.  Every request computes exactly what mfd_create + mfd_run(1, nt) compute.
 *
 * The descriptor and every array it points to must stay valid until mfd_server_poll reports
 * the request MFD_REQ_RUNNING (uploaded) or later.  A finished request (MFD_REQ_DONE) keeps
 * its handle and its share of the budget until mfd_server_release: read its results through
 * mfd_server_handle and the mfd_read_* calls first (do not run, write or destroy that
 * handle).  A failed request (MFD_REQ_FAILED; its status code is returned by poll and wait)
 * gives its memory back at once.  Times are seconds since the server's creation: submitted,
 * admitted, running (uploaded), finished.  The calls are safe from any host thread.
 * mfd_server_destroy waits for admitted requests to finish, drops queued ones and frees
 * every handle. */
enum { MFD_REQ_QUEUED = 0, MFD_REQ_ADMITTED = 1, MFD_REQ_RUNNING = 2, MFD_REQ_DONE = 3, MFD_REQ_FAILED = 4 };
typedef struct mfd_server mfd_server;
MFD_API int mfd_server_create(int32_t device, double budget_bytes, int32_t max_active, int32_t max_solo, mfd_server** out);
MFD_API void mfd_server_destroy(mfd_server* s);
/* MFD_ERR_ADMISSION when the request could never fit the budget. */
MFD_API int mfd_server_submit(mfd_server* s, const mfd_desc* desc, int64_t* id);
/* state, times[4] (may be NULL) and the footprint in bytes (may be NULL). */
MFD_API int mfd_server_poll(mfd_server* s, int64_t id, int32_t* state, double* times, int64_t* bytes);
/* Waits up to timeout_s seconds for the request to finish (MFD_ERR_TIMEOUT if it has not). */
MFD_API int mfd_server_wait(mfd_server* s, int64_t id, double timeout_s, int32_t* state);
MFD_API int mfd_server_handle(mfd_server* s, int64_t id, mfd_handle** h);
MFD_API int mfd_server_release(mfd_server* s, int64_t id);
MFD_API int mfd_server_info(mfd_server* s, int64_t* queued, int64_t* running, int64_t* done, int64_t* failed,
                            double* used_bytes, double* peak_used_bytes, int32_t* peak_active);
/* Device bytes mfd_create would allocate for the descriptor (-1: invalid descriptor). */
MFD_API int64_t mfd_server_footprint(const mfd_desc* desc);
MFD_API const char* mfd_server_last_error(mfd_server* s);

/* Device-time measurement: when on, every kernel launch of mfd_run is bracketed by CUDA
 * events on the handle's stream and its duration is summed per kernel class. */
MFD_API int mfd_set_profiling(mfd_handle* h, int32_t on);
/* Kernel classes: 0 H update, 1 E update, 2 sources, 3 TFSF, 4 monitors, 5 DFT,
 * 6 sums flush, 7 material response.  Fills ms[k], launches[k] for k < n; returns the number of classes. */
MFD_API int mfd_kernel_times(const mfd_handle* h, double* ms, int64_t* launches, int32_t n);
/* Device time of the last mfd_run call (CUDA events around the whole call), in ms. */
MFD_API int mfd_last_run_ms(const mfd_handle* h, double* ms);
/* Device bytes held by the handle. */
MFD_API int64_t mfd_device_bytes(const mfd_handle* h);

MFD_API const char* mfd_last_error(const mfd_handle* h);
/* Error text of the last failed mfd_create (no handle exists then). */
MFD_API const char* mfd_create_error(void);
MFD_API int mfd_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* MAXWELLFDTD_H */
