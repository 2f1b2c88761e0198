# MaxwellFDTDB200.jl -- the B200 backend of MaxwellFDTD: the time-step path of solve! handed
# to libmaxwellfdtd_b200.so through ccall.
#
# A maintainer adds this file to the reference package (src/, `include("MaxwellFDTDB200.jl")`
# after backends.jl, models.jl, materials.jl, sources.jl, monitors.jl and outputs.jl) and
# exports B200.  Everything above solve! -- Grid, Material, sources, CPML, monitors, Model --
# is unchanged; B200{T}() stands beside CPU{T}() and GPU{T}() (src/backends.jl:10-23).
# The C declarations are in include/maxwellfdtd.h of the B200 project; the structs below
# mirror them field for field (isbits, C layout).  This environment has no Julia, so the
# file is not run here; the same ABI is driven from Python (maxwellfdtd_b200/_abi.py,
# maxwellfdtd_b200/model.py build_desc) by every test of the project.

struct B200{T} end
B200() = B200{Float32}()

const libmfd = get(ENV, "MFD_LIBRARY", "libmaxwellfdtd_b200.so")

const MFD_ABI_VERSION = 2
const MFD_OK, MFD_ERR_INVALID, MFD_ERR_OOM, MFD_ERR_CUDA, MFD_ERR_NONFINITE = 0, 1, 2, 3, 4
const MFD_F32, MFD_F64 = 0, 1
const MFD_MODE_EXACT, MFD_MODE_FAST = 0, 1
const MFD_POL_HY, MFD_POL_EY = 0, 1
const MFD_SRC_SOFT, MFD_SRC_HARD = 0, 1
const MFD_MON_FIELD, MFD_MON_SPECTRAL = 0, 1
const MFD_RATE_NONE, MFD_RATE_POWER, MFD_RATE_TABLE = 0, 1, 2
const MFD_INT_SA, MFD_INT_E2, MFD_INT_JE, MFD_INT_RHO = 0, 1, 2, 3
const MFD_REQ_QUEUED, MFD_REQ_ADMITTED, MFD_REQ_RUNNING, MFD_REQ_DONE, MFD_REQ_FAILED = 0, 1, 2, 3, 4

# ---- descriptor mirror (include/maxwellfdtd.h) ---------------------------------------------
struct MfdPmlLayer
    ib::Int32; nb::Int32; K::Ptr{Cdouble}; A::Ptr{Cdouble}; B::Ptr{Cdouble}
end

struct MfdMaterial
    Mh::Cdouble; Me::Cdouble; Md1::Cdouble; Md2::Cdouble
    nq::Int32; Aq::Ptr{Cdouble}; Bq::Ptr{Cdouble}; Cq::Ptr{Cdouble}
    kerr::Int32; Mk2::Cdouble; Mk3::Cdouble
    plasma::Int32; Rava::Cdouble; ksi::Cdouble; rho0::Cdouble; Ap::Cdouble; Bp::Cdouble; Cp::Cdouble; Ma::Cdouble
    rate_kind::Int32; rate_order::Cdouble; rate_log10c::Cdouble
    rate_n::Int32; rate_x::Ptr{Cdouble}; rate_y::Ptr{Cdouble}
end

struct MfdSource
    kind::Int32; comp::Int32; coeff::Cdouble; npts::Int64; cells::Ptr{Int64}
    wave::Ptr{Cdouble}; amp::Ptr{Cdouble}; gt::Ptr{Cdouble}
end

struct MfdTFSF
    enabled::Int32; order::Int32; i1::NTuple{3,Int32}; i2::NTuple{3,Int32}
    inc::NTuple{24,Ptr{Cvoid}}; shape::NTuple{24,Int32}
end

struct MfdMonitor
    kind::Int32; sum::Int32; npts::Int64; cells::Ptr{Int64}; nw::Int32; phasor::Ptr{Cdouble}
end

struct MfdShape
    kind::Int32; material::Int32; p::NTuple{8,Cdouble}
end

struct MfdDesc
    abi_version::Int32; ndim::Int32; dtype::Int32; nx::Int32; ny::Int32; nz::Int32
    dx::Cdouble; dy::Cdouble; dz::Cdouble; dt::Cdouble; nt::Int64
    bc::NTuple{6,Int32}; pml::NTuple{6,MfdPmlLayer}
    Mh0::Cdouble; Me0::Cdouble; Md10::Cdouble; Md20::Cdouble
    geometry::Ptr{UInt8}; nmat::Int32; mats::Ptr{MfdMaterial}; rho_fp64::Int32
    nsrc::Int32; srcs::Ptr{MfdSource}; tfsf::MfdTFSF; nmon::Int32; mons::Ptr{MfdMonitor}
    tfsf_record::Int32; rec_i1::NTuple{3,Int32}; rec_i2::NTuple{3,Int32}; device::Int32; mode::Int32
    nshape::Int32; shapes::Ptr{MfdShape}; coords::NTuple{3,Ptr{Cdouble}}; polarization::Int32
end

# ---- descriptor from a reference Model ------------------------------------------------------
# `keep` holds every array a pointer in the descriptor refers to; wrap ccalls that read the
# descriptor in GC.@preserve keep.
_ptr(keep, v::AbstractArray{S}) where S = (a = collect(v); push!(keep, a); pointer(a))
_ptr(keep, ::Nothing) = C_NULL

function _pml_layer(keep, L)
    L.Nb <= 1 && all(iszero, L.A) && return MfdPmlLayer(L.ib, 0, C_NULL, C_NULL, C_NULL)   # Lx == 0: no layer
    MfdPmlLayer(L.ib, L.Nb, _ptr(keep, Float64.(L.K)), _ptr(keep, Float64.(L.A)), _ptr(keep, Float64.(L.B)))
end

# ionrate: an IonizationRate table is passed as its knots; any other closure is sampled on an
# even log10(I) grid (the library interpolates log-log), or give (order, log10c) of the MPI
# power law R = 10^(order log10 I + log10c) as `ionrate_params`.
function _rate(keep, m, ionrate_params)
    if !isnothing(ionrate_params)
        return MFD_RATE_POWER, Float64(ionrate_params[1]), Float64(ionrate_params[2]), 0, C_NULL, C_NULL
    end
    f = m.ionrate
    if hasproperty(f, :x) && hasproperty(f, :y)
        return MFD_RATE_TABLE, 0.0, 0.0, length(f.x), _ptr(keep, Float64.(f.x)), _ptr(keep, Float64.(f.y))
    end
    x = collect(range(8.0, 22.0; length=2001))
    y = [log10(max(f(10.0^v), floatmin(Float64))) for v in x]
    return MFD_RATE_TABLE, 0.0, 0.0, length(x), _ptr(keep, x), _ptr(keep, y)
end

function _material(keep, m, ionrate_params)
    nq = m.isdispersion ? length(m.Aq) : 0
    Aq, Bq, Cq = nq > 0 ? (_ptr(keep, Float64.(m.Aq)), _ptr(keep, Float64.(m.Bq)), _ptr(keep, Float64.(m.Cq))) :
                          (C_NULL, C_NULL, C_NULL)
    kind, order, l10c, rn, rx, ry = m.isplasma ? _rate(keep, m, ionrate_params) : (MFD_RATE_NONE, 0.0, 0.0, 0, C_NULL, C_NULL)
    pl(x) = m.isplasma ? Float64(x) : 0.0
    MfdMaterial(m.Mh, m.Me, m.Md1, m.Md2, nq, Aq, Bq, Cq, m.iskerr, m.Mk2, m.Mk3,
                m.isplasma, pl(m.Rava), pl(m.ksi), pl(m.rho0), pl(m.Ap), pl(m.Bp), pl(m.Cp), pl(m.Ma),
                kind, order, l10c, rn, rx, ry)
end

_linear(inds, dims) = Int64[LinearIndices(dims)[i] - 1 for i in inds]

# a waveform tabulated in Float64 for every point and step: wave[it][p] (sources.jl:52-131)
const MFD_COMP = Dict(:Hx => 0, :Hy => 1, :Hz => 2, :Dx => 3, :Dy => 4, :Dz => 5, :Ex => 6, :Ey => 7, :Ez => 8)

function _source(keep, s, field, grid, t, dims)
    kind = s isa HardSourceStruct ? MFD_SRC_HARD : MFD_SRC_SOFT
    coeff = s isa HardSourceStruct ? 1.0 : Float64(s.coeff)
    cells = _linear(s.isrc, dims)
    coords = [ntuple(d -> getproperty(grid, (:x, :y, :z)[end - length(dims) + d])[Tuple(i)[d]], length(dims))
              for i in s.isrc]
    args = isnothing(s.p) ? () : (s.p,)
    wave = Float64[s.waveform(c..., ti, args...) for c in coords, ti in t]   # (npts, nt): C order [nt][npts]
    comp = MFD_COMP[fieldnames(typeof(field))[s.icomp]]
    MfdSource(kind, comp, coeff, length(cells), _ptr(keep, cells), _ptr(keep, wave), C_NULL, C_NULL)
end

# spectral monitor phasors exp(-1im w (t - tshift)) as [nt][nw][2] (dft.jl:27-51)
function _monitor(keep, mon, t, dims)
    cells = _linear(mon.inds, dims)
    if hasproperty(mon, :dft)
        (; w, tshift) = mon.dft
        ph = Array{Float64}(undef, 2, length(w), length(t))
        for (it, ti) in enumerate(t), (iw, wv) in enumerate(w)
            e = exp(-1im * wv * (ti - tshift))
            ph[1, iw, it], ph[2, iw, it] = real(e), imag(e)
        end
        return MfdMonitor(MFD_MON_SPECTRAL, mon.issum, length(cells), _ptr(keep, cells), length(w), _ptr(keep, ph))
    end
    MfdMonitor(MFD_MON_FIELD, mon.issum, length(cells), _ptr(keep, cells), 0, C_NULL)
end

_layers(pml, nd) = nd == 3 ? (pml.xlayer1, pml.xlayer2, pml.ylayer1, pml.ylayer2, pml.zlayer1, pml.zlayer2) :
                   nd == 2 ? (pml.xlayer1, pml.xlayer2, nothing, nothing, pml.zlayer1, pml.zlayer2) :
                             (nothing, nothing, nothing, nothing, pml.zlayer1, pml.zlayer2)

const _NOLAYER = MfdPmlLayer(0, 0, C_NULL, C_NULL, C_NULL)

"""
    build_desc(model, T, monitors; mode=MFD_MODE_EXACT, device=0, ionrate_params=nothing)

The C descriptor of a reference Model (models.jl:1-122) in element type T, and the arrays
it points to.  TFSF incident data (TFSFSourceStruct, sources.jl:592-710) go in the full
[nt][b][a] layout; a caller that knows its source is a plane wave along a grid axis may
pass the compact layouts of include/maxwellfdtd.h instead.
"""
function build_desc(model, ::Type{T}, monitors; mode=MFD_MODE_EXACT, device=0, ionrate_params=nothing) where T
    keep = Any[]
    (; field, sources, bcs, pml, geometry, materials, Nt, dt, t, Mh, Me, Md1, Md2) = model
    grid = field.grid
    dims = size(field.Ex)
    nd = length(dims)
    nx, ny, nz = nd == 3 ? dims : nd == 2 ? (dims[1], 1, dims[2]) : (1, 1, dims[1])
    dx = nd >= 2 ? grid.dx : 1.0
    dy = nd == 3 ? grid.dy : 1.0
    bc6 = nd == 3 ? bcs : nd == 2 ? (bcs[1], bcs[2], 1, 1, bcs[3], bcs[4]) : (1, 1, 1, 1, bcs[1], bcs[2])
    lay = Tuple(L === nothing ? _NOLAYER : _pml_layer(keep, L) for L in _layers(pml, nd))
    mats = [_material(keep, m, ionrate_params) for m in materials]
    point = [s for s in sources if !(s isa TFSFSourceStruct)]
    srcs = [_source(keep, s, field, grid, t, dims) for s in point]
    tfsf = MfdTFSF(0, 0, (0, 0, 0), (0, 0, 0), ntuple(_ -> C_NULL, 24), ntuple(_ -> Int32(0), 24))
    for (k, s) in enumerate(sources)
        s isa TFSFSourceStruct || continue
        incs = [getfield(s, n) for n in fieldnames(typeof(s)) if startswith(String(n), "inc")]
        ptrs = ntuple(i -> i <= length(incs) ? Ptr{Cvoid}(_ptr(keep, T.(incs[i]))) : C_NULL, 24)
        tfsf = MfdTFSF(1, count(x -> !(x isa TFSFSourceStruct), sources[1:k-1]), s.i1, s.i2, ptrs, ntuple(_ -> Int32(0), 24))
    end
    mons = [_monitor(keep, m, t, dims) for m in monitors]
    d = MfdDesc(MFD_ABI_VERSION, nd, T == Float64 ? MFD_F64 : MFD_F32, nx, ny, nz, dx, dy, grid.dz, dt, Nt,
                Tuple(Int32.(bc6)), lay, Mh, Me, Md1, Md2, _ptr(keep, UInt8.(geometry)), length(mats),
                isempty(mats) ? C_NULL : _ptr(keep, mats), 1, length(srcs), isempty(srcs) ? C_NULL : _ptr(keep, srcs),
                tfsf, length(mons), isempty(mons) ? C_NULL : _ptr(keep, mons), 0, (0, 0, 0), (0, 0, 0), device, mode,
                0, C_NULL, (C_NULL, C_NULL, C_NULL),   # closures: the host map above, no device shapes
                MFD_POL_HY)                          # the reference's Field2D (fields.jl:36-55)
    return d, keep
end

_check(h, st) = st == MFD_OK ||
    error(unsafe_string(ccall((:mfd_last_error, libmfd), Cstring, (Ptr{Cvoid},), h)))

# readers: Julia Arrays are column-major with x fastest, the library's layout -> no transpose
read_field!(h, comp, A::Array) = _check(h, ccall((:mfd_read_field, libmfd), Cint, (Ptr{Cvoid}, Int32, Ptr{Cvoid}), h, comp, A))
read_geometry!(h, A::Array{UInt8}) = _check(h, ccall((:mfd_read_geometry, libmfd), Cint, (Ptr{Cvoid}, Ptr{UInt8}), h, A))
read_integral!(h, which, A::Array) = _check(h, ccall((:mfd_read_integral, libmfd), Cint, (Ptr{Cvoid}, Int32, Ptr{Cvoid}), h, which, A))
read_integral_noalloc!(h, which, A::Array) =
    _check(h, ccall((:mfd_read_integral_noalloc, libmfd), Cint, (Ptr{Cvoid}, Int32, Ptr{Cvoid}), h, which, A))
read_monitor!(h, m, comp, A::Array) =
    _check(h, ccall((:mfd_read_monitor, libmfd), Cint, (Ptr{Cvoid}, Int32, Int32, Ptr{Cvoid}), h, m, comp, A))

# model state images: checkpoint / resume, eviction (mfd_read_state / mfd_write_state)
function read_state(h)
    n = ccall((:mfd_state_size, libmfd), Int64, (Ptr{Cvoid},), h)
    img = Vector{UInt8}(undef, n)
    _check(h, ccall((:mfd_read_state, libmfd), Cint, (Ptr{Cvoid}, Ptr{UInt8}, Int64), h, img, n))
    return img
end
write_state!(h, img::Vector{UInt8}) =
    _check(h, ccall((:mfd_write_state, libmfd), Cint, (Ptr{Cvoid}, Ptr{UInt8}, Int64), h, img, length(img)))

# ---- solve! for the B200 backend (models.jl:166-242) -------------------------------------------
"""
    solve!(model, backend::B200{T}; fname="out.hdf", nframes, nstride, dtout, components,
           monitors, mode=MFD_MODE_EXACT, ionrate_params=nothing, max_chunk=4096)

The reference's solve! with the time steps run by the library: the output file is created by
the reference's Output (outputs.jl), the library runs the steps in chunks that end at the
output steps, and the fields, monitors and running sums are read back into the file.  The
NaN/Inf guard of every step runs on the device; its error carries the reference's message.
"""
function solve!(model, backend::B200{T}; fname="out.hdf", nframes=nothing, nstride=nothing, dtout=nothing,
                components=nothing, monitors=nothing, mode=MFD_MODE_EXACT, ionrate_params=nothing,
                max_chunk=4096) where T
    model = adapt(CPU{T}(), model)          # host arrays in element type T (backends.jl:27-41)
    (; Nt, dt, t, field) = model
    out = Output(model; fname, nstride, nframes, dtout, components, monitors)
    mons = out.ismonitors ? out.monitors : ()
    d, keep = build_desc(model, T, mons; mode, ionrate_params)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve keep begin
        st = ccall((:mfd_create, libmfd), Cint, (Ref{MfdDesc}, Ref{Ptr{Cvoid}}), d, h)
        st == MFD_OK || error(unsafe_string(ccall((:mfd_create_error, libmfd), Cstring, ())))
    end
    try
        it_out = [findfirst(ti -> abs(ti - tt) <= dt / 2, t) for tt in (out.isfields ? out.tout : ())]
        a = 1
        for stop in sort(unique([it_out; Nt]))
            while a <= stop
                b = min(stop, a + max_chunk - 1)
                st = ccall((:mfd_run, libmfd), Cint, (Ptr{Cvoid}, Int64, Int64), h[], a, b)
                st == MFD_OK || error(unsafe_string(ccall((:mfd_last_error, libmfd), Cstring, (Ptr{Cvoid},), h[])))
                a = b + 1
            end
            if stop in it_out                   # write_fields (outputs.jl:156-179, 437-472)
                HDF5.h5open(out.fname, "r+") do fp
                    group = fp["fields"]
                    for c in out.components
                        A = similar(getfield(field, c))
                        read_field!(h[], MFD_COMP[c], A)
                        group[String(c)][ntuple(_ -> Colon(), ndims(A))..., out.itout] = A
                    end
                    if out.isplasma
                        rho = zeros(Float64, size(field.Ex))
                        read_integral!(h[], MFD_INT_RHO, rho)
                        group["rho"][ntuple(_ -> Colon(), ndims(rho))..., out.itout] = rho
                    end
                end
                out.itout += 1
            end
        end
        # monitors (monitors.jl) and running sums (outputs.jl:46-65)
        for (n, mon) in enumerate(mons)
            for c in (:Hx, :Hy, :Hz, :Ex, :Ey, :Ez)
                hasproperty(mon, c) || continue
                # the library's [nt][npts] ([nw][npts] complex) is the column-major (npts, nt)
                # array of the reference; field records come in T, spectra in ComplexF64
                A = getfield(mon, c)
                tmp = Array{hasproperty(mon, :dft) ? ComplexF64 : T}(undef, size(A))
                read_monitor!(h[], n - 1, MFD_COMP[c], tmp)
                A .= tmp
            end
        end
        out.ismonitors && write_monitors(out)
        read_integral!(h[], MFD_INT_SA, out.Sa)
        HDF5.h5open(out.fname, "r+") do fp
            fp["Sa"] = out.Sa
            if out.isgeometry
                read_integral!(h[], MFD_INT_E2, out.E2)
                fp["E2"] = out.E2
                if out.isplasma
                    rho = zeros(Float64, size(field.Ex)); read_integral!(h[], MFD_INT_RHO, rho)
                    JE = similar(field.Ex); read_integral!(h[], MFD_INT_JE, JE)
                    fp["rho_end"] = rho
                    fp["JE"] = JE
                end
            end
        end
        for c in fieldnames(typeof(field))[2:end]     # the final fields back into the model
            read_field!(h[], MFD_COMP[c], getfield(field, c))
        end
    finally
        ccall((:mfd_destroy, libmfd), Cvoid, (Ptr{Cvoid},), h[])
    end
    return model
end

# ---- serving (mfd_server_*; no counterpart in the reference) ---------------------------------
# Requests are descriptors; each descriptor's arrays (`keep`) must stay alive until the request
# is running.  A finished request's handle is read with the readers above, then released.
function server_create(; device=0, budget_bytes=160e9, max_active=64, max_solo=16)
    s = Ref{Ptr{Cvoid}}(C_NULL)
    st = ccall((:mfd_server_create, libmfd), Cint, (Int32, Cdouble, Int32, Int32, Ref{Ptr{Cvoid}}),
               device, budget_bytes, max_active, max_solo, s)
    st == MFD_OK || error(unsafe_string(ccall((:mfd_create_error, libmfd), Cstring, ())))
    return s[]
end

function server_submit(s, d::MfdDesc)
    id = Ref{Int64}(0)
    st = ccall((:mfd_server_submit, libmfd), Cint, (Ptr{Cvoid}, Ref{MfdDesc}, Ref{Int64}), s, d, id)
    st == MFD_OK || error(unsafe_string(ccall((:mfd_server_last_error, libmfd), Cstring, (Ptr{Cvoid},), s)))
    return id[]
end

function server_wait(s, id; timeout_s=3600.0)
    state = Ref{Int32}(0)
    st = ccall((:mfd_server_wait, libmfd), Cint, (Ptr{Cvoid}, Int64, Cdouble, Ref{Int32}), s, id, timeout_s, state)
    st == MFD_OK || error(unsafe_string(ccall((:mfd_server_last_error, libmfd), Cstring, (Ptr{Cvoid},), s)))
    return state[]
end

function server_handle(s, id)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    st = ccall((:mfd_server_handle, libmfd), Cint, (Ptr{Cvoid}, Int64, Ref{Ptr{Cvoid}}), s, id, h)
    st == MFD_OK || error(unsafe_string(ccall((:mfd_server_last_error, libmfd), Cstring, (Ptr{Cvoid},), s)))
    return h[]
end

server_release(s, id) = ccall((:mfd_server_release, libmfd), Cint, (Ptr{Cvoid}, Int64), s, id)
server_destroy(s) = ccall((:mfd_server_destroy, libmfd), Cvoid, (Ptr{Cvoid},), s)
