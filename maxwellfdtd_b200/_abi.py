"""ctypes mirror of include/maxwellfdtd.h and a thin wrapper over any library that exports
that API under a symbol prefix (``mfd_`` for the CUDA library)."""
import ctypes as C
import os

import numpy as np

ABI_VERSION = 2

MFD_OK, MFD_ERR_INVALID, MFD_ERR_OOM, MFD_ERR_CUDA, MFD_ERR_NONFINITE, MFD_ERR_TIMEOUT, \
    MFD_ERR_ADMISSION, MFD_ERR_NODEVICE = range(8)
MFD_F32, MFD_F64 = 0, 1
MFD_MODE_EXACT, MFD_MODE_FAST = 0, 1
MFD_POL_HY, MFD_POL_EY = 0, 1
MFD_INC_FULL, MFD_INC_ALONG_B, MFD_INC_ALONG_A, MFD_INC_UNIFORM = range(4)
MFD_REQ_QUEUED, MFD_REQ_ADMITTED, MFD_REQ_RUNNING, MFD_REQ_DONE, MFD_REQ_FAILED = range(5)
MFD_INT_SA, MFD_INT_E2, MFD_INT_JE, MFD_INT_RHO = range(4)
MFD_RATE_NONE, MFD_RATE_POWER, MFD_RATE_TABLE = range(3)
MFD_MON_FIELD, MFD_MON_SPECTRAL = range(2)

_dp = C.POINTER(C.c_double)


class PmlLayer(C.Structure):
    _fields_ = [("ib", C.c_int32), ("nb", C.c_int32), ("K", _dp), ("A", _dp), ("B", _dp)]


class Material(C.Structure):
    _fields_ = [("Mh", C.c_double), ("Me", C.c_double), ("Md1", C.c_double), ("Md2", C.c_double),
                ("nq", C.c_int32), ("Aq", _dp), ("Bq", _dp), ("Cq", _dp),
                ("kerr", C.c_int32), ("Mk2", C.c_double), ("Mk3", C.c_double),
                ("plasma", C.c_int32),
                ("Rava", C.c_double), ("ksi", C.c_double), ("rho0", C.c_double), ("Ap", C.c_double),
                ("Bp", C.c_double), ("Cp", C.c_double), ("Ma", C.c_double),
                ("rate_kind", C.c_int32), ("rate_order", C.c_double), ("rate_log10c", C.c_double),
                ("rate_n", C.c_int32), ("rate_x", _dp), ("rate_y", _dp)]


class Source(C.Structure):
    _fields_ = [("kind", C.c_int32), ("comp", C.c_int32), ("coeff", C.c_double),
                ("npts", C.c_int64), ("cells", C.POINTER(C.c_int64)),
                ("wave", _dp), ("amp", _dp), ("gt", _dp)]


class Tfsf(C.Structure):
    _fields_ = [("enabled", C.c_int32), ("order", C.c_int32), ("i1", C.c_int32 * 3), ("i2", C.c_int32 * 3),
                ("inc", C.c_void_p * 24), ("shape", C.c_int32 * 24)]


class Monitor(C.Structure):
    _fields_ = [("kind", C.c_int32), ("sum", C.c_int32), ("npts", C.c_int64),
                ("cells", C.POINTER(C.c_int64)), ("nw", C.c_int32), ("phasor", _dp)]


class Shape(C.Structure):
    _fields_ = [("kind", C.c_int32), ("material", C.c_int32), ("p", C.c_double * 8)]


class Desc(C.Structure):
    _fields_ = [("abi_version", C.c_int32), ("ndim", C.c_int32), ("dtype", C.c_int32),
                ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("dt", C.c_double), ("nt", C.c_int64),
                ("bc", C.c_int32 * 6), ("pml", PmlLayer * 6),
                ("Mh0", C.c_double), ("Me0", C.c_double), ("Md10", C.c_double), ("Md20", C.c_double),
                ("geometry", C.POINTER(C.c_uint8)),
                ("nmat", C.c_int32), ("mats", C.POINTER(Material)),
                ("rho_fp64", C.c_int32),
                ("nsrc", C.c_int32), ("srcs", C.POINTER(Source)),
                ("tfsf", Tfsf),
                ("nmon", C.c_int32), ("mons", C.POINTER(Monitor)),
                ("tfsf_record", C.c_int32), ("rec_i1", C.c_int32 * 3), ("rec_i2", C.c_int32 * 3),
                ("device", C.c_int32), ("mode", C.c_int32),
                ("nshape", C.c_int32), ("shapes", C.POINTER(Shape)), ("coords", _dp * 3),
                ("polarization", C.c_int32)]


def dptr(a):
    """double* of a contiguous float64 array (None -> NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


class DescBuilder:
    """Owns every array the descriptor points to (keep it alive while the library reads it).

    host_alloc(n, dtype) -> 1-D array, when given, provides the storage of arrays of at least
    1 MiB (e.g. page-locked memory, which mfd_create uploads at full DMA speed)."""

    def __init__(self, host_alloc=None):
        self.keep = []
        self.desc = Desc()
        self.host_alloc = host_alloc

    def arr(self, a, dtype):
        a = np.ascontiguousarray(a, dtype=dtype)
        if self.host_alloc is not None and a.nbytes >= (1 << 20):
            dst = self.host_alloc(a.size, np.dtype(dtype))
            dst[...] = a.reshape(-1)
            a = dst.reshape(a.shape)
        self.keep.append(a)
        return a


class StepperError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class Library:
    """A loaded library exporting the maxwellfdtd C API with symbol prefix ``prefix``."""

    def __init__(self, path, prefix="mfd_"):
        self.path = os.path.abspath(path)
        self.lib = C.CDLL(self.path, mode=C.RTLD_GLOBAL)
        self.prefix = prefix
        L, p = self.lib, prefix
        vp = C.c_void_p

        def fn(name, res, args):
            f = getattr(L, p + name)
            f.restype = res
            f.argtypes = args
            return f

        self.create = fn("create", C.c_int, [C.POINTER(Desc), C.POINTER(vp)])
        self.destroy = fn("destroy", None, [vp])
        self.run = fn("run", C.c_int, [vp, C.c_int64, C.c_int64])
        self.read_field = fn("read_field", C.c_int, [vp, C.c_int32, vp])
        self.read_geometry = fn("read_geometry", C.c_int, [vp, vp])
        self.write_field = fn("write_field", C.c_int, [vp, C.c_int32, vp])
        self.read_integral = fn("read_integral", C.c_int, [vp, C.c_int32, vp])
        self.read_monitor = fn("read_monitor", C.c_int, [vp, C.c_int32, C.c_int32, vp])
        self.read_tfsf_record = fn("read_tfsf_record", C.c_int, [vp, C.c_int32, vp])
        self.tfsf_record_size = fn("tfsf_record_size", C.c_int64, [vp, C.c_int32])
        self.status = fn("status", C.c_int, [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int32)])
        self.last_error = fn("last_error", C.c_char_p, [vp])
        self.create_error = fn("create_error", C.c_char_p, [])
        # device-side measurement entry points (CUDA library only)
        self.has_timing = hasattr(L, p + "set_profiling")
        if self.has_timing:
            self.set_profiling = fn("set_profiling", C.c_int, [vp, C.c_int32])
            self.kernel_times = fn("kernel_times", C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.c_int32])
            self.last_run_ms = fn("last_run_ms", C.c_int, [vp, C.POINTER(C.c_double)])
            self.device_bytes = fn("device_bytes", C.c_int64, [vp])
        # field snapshots during a run (CUDA library only)
        self.has_snapshots = hasattr(L, p + "set_snapshots")
        if self.has_snapshots:
            self.set_snapshots = fn("set_snapshots", C.c_int, [vp, C.c_int32, C.POINTER(C.c_int32), C.c_int64,
                                                              C.POINTER(C.c_int64), vp])
        # model state images (CUDA library only)
        self.has_state = hasattr(L, p + "read_state")
        if self.has_state:
            self.state_size = fn("state_size", C.c_int64, [vp])
            self.read_state = fn("read_state", C.c_int, [vp, vp, C.c_int64])
            self.write_state = fn("write_state", C.c_int, [vp, vp, C.c_int64])
        # the serving loop (CUDA library only)
        self.has_server = hasattr(L, p + "server_create")
        if self.has_server:
            self.server_create = fn("server_create", C.c_int, [C.c_int32, C.c_double, C.c_int32, C.c_int32, C.POINTER(vp)])
            self.server_destroy = fn("server_destroy", None, [vp])
            self.server_submit = fn("server_submit", C.c_int, [vp, C.POINTER(Desc), C.POINTER(C.c_int64)])
            self.server_poll = fn("server_poll", C.c_int, [vp, C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                                           C.POINTER(C.c_int64)])
            self.server_wait = fn("server_wait", C.c_int, [vp, C.c_int64, C.c_double, C.POINTER(C.c_int32)])
            self.server_handle = fn("server_handle", C.c_int, [vp, C.c_int64, C.POINTER(vp)])
            self.server_release = fn("server_release", C.c_int, [vp, C.c_int64])
            self.server_info = fn("server_info", C.c_int, [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                                           C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                                           C.POINTER(C.c_double), C.POINTER(C.c_double),
                                                           C.POINTER(C.c_int32)])
            self.server_footprint = fn("server_footprint", C.c_int64, [C.POINTER(Desc)])
            self.server_last_error = fn("server_last_error", C.c_char_p, [vp])
        # batches of 2-D models (CUDA library only)
        self.has_batch = hasattr(L, p + "batch_create")
        if self.has_batch:
            self.batch_create = fn("batch_create", C.c_int, [C.c_int32, C.POINTER(vp)])
            self.batch_destroy = fn("batch_destroy", None, [vp])
            self.batch_add = fn("batch_add", C.c_int, [vp, vp, C.c_int64])
            self.batch_run = fn("batch_run", C.c_int, [vp, C.c_int64, C.POINTER(C.c_int32)])
            self.batch_config = fn("batch_config", C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32])
            self.batch_info = fn("batch_info", C.c_int, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                                         C.POINTER(C.c_double), C.POINTER(C.c_int64),
                                                         C.POINTER(C.c_int64)])
            self.batch_last_error = fn("batch_last_error", C.c_char_p, [vp])


class Stepper:
    """One model instance in a library (the handle)."""

    def __init__(self, lib, builder, dtype):
        self.lib = lib
        self.builder = builder
        self.dtype = np.dtype(dtype)
        d = builder.desc
        self.shape3 = (d.nx, d.ny, d.nz)
        self.N = d.nx * d.ny * d.nz
        h = C.c_void_p()
        st = lib.create(C.byref(d), C.byref(h))
        if st != MFD_OK:
            raise StepperError(st, f"create failed ({st}): {lib.create_error().decode()}")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != MFD_OK:
            raise StepperError(st, self.lib.last_error(self.h).decode())

    def run(self, a, b):
        self._check(self.lib.run(self.h, int(a), int(b)))

    def status(self):
        d, b, k = C.c_int64(), C.c_int64(), C.c_int32()
        self.lib.status(self.h, C.byref(d), C.byref(b), C.byref(k))
        return d.value, b.value, k.value

    @staticmethod
    def _dest(out, n, dtype, shape=None):
        """The caller's buffer (e.g. page-locked memory, which the copy reaches at full DMA
        speed) when given and of the right size and type, else a new array."""
        if out is None:
            return np.empty(shape if shape is not None else n, dtype=dtype)
        if out.dtype != np.dtype(dtype) or out.size != (int(np.prod(shape)) if shape is not None else n) \
                or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("output buffer of the wrong size, type or layout")
        return out

    def read_field(self, comp, out=None):
        out = self._dest(out, self.N, self.dtype)
        self._check(self.lib.read_field(self.h, int(comp), out.ctypes.data_as(C.c_void_p)))
        return out

    def read_geometry(self):
        """The material index map the library holds (nx*ny*nz bytes, x fastest)."""
        out = np.empty(self.N, dtype=np.uint8)
        self._check(self.lib.read_geometry(self.h, out.ctypes.data_as(C.c_void_p)))
        return out

    def write_field(self, comp, values):
        v = np.ascontiguousarray(values, dtype=self.dtype).ravel()
        assert v.size == self.N
        self._check(self.lib.write_field(self.h, int(comp), v.ctypes.data_as(C.c_void_p)))

    def read_integral(self, which, out=None):
        dt = np.float64 if which == MFD_INT_RHO else self.dtype
        out = self._dest(out, self.N, dt)
        self._check(self.lib.read_integral(self.h, int(which), out.ctypes.data_as(C.c_void_p)))
        return out

    def read_monitor(self, m, comp, shape, spectral, out=None):
        out = self._dest(out, None, np.complex128 if spectral else self.dtype, shape)
        self._check(self.lib.read_monitor(self.h, int(m), int(comp), out.ctypes.data_as(C.c_void_p)))
        return out

    def set_snapshots(self, comps, steps, dst):
        """Frames of the listed components after each listed step, copied into dst
        (len(steps) x len(comps) x N elements of the model's type) while the run goes on."""
        comps = np.ascontiguousarray(comps, dtype=np.int32)
        steps = np.ascontiguousarray(steps, dtype=np.int64)
        if dst.dtype != self.dtype or dst.size != len(steps) * len(comps) * self.N or not dst.flags["C_CONTIGUOUS"]:
            raise ValueError("snapshot buffer of the wrong size, type or layout")
        self._snap = (comps, steps, dst)   # kept alive while the library writes into dst
        self._check(self.lib.set_snapshots(self.h, len(comps), comps.ctypes.data_as(C.POINTER(C.c_int32)), len(steps),
                                           steps.ctypes.data_as(C.POINTER(C.c_int64)), dst.ctypes.data_as(C.c_void_p)))

    KERNEL_CLASSES = ("H", "E", "sources", "tfsf", "monitors", "dft", "sums", "material")

    def set_profiling(self, on):
        self._check(self.lib.set_profiling(self.h, int(bool(on))))

    def kernel_times(self):
        n = len(self.KERNEL_CLASSES)
        ms = (C.c_double * n)()
        cnt = (C.c_int64 * n)()
        self.lib.kernel_times(self.h, ms, cnt, n)
        return {k: (ms[i], cnt[i]) for i, k in enumerate(self.KERNEL_CLASSES)}

    def last_run_ms(self):
        v = C.c_double()
        self._check(self.lib.last_run_ms(self.h, C.byref(v)))
        return v.value

    def device_bytes(self):
        return int(self.lib.device_bytes(self.h))

    def read_state(self):
        """The model's state image (mfd_read_state) as a uint8 array."""
        n = int(self.lib.state_size(self.h))
        out = np.empty(n, dtype=np.uint8)
        self._check(self.lib.read_state(self.h, out.ctypes.data_as(C.c_void_p), n))
        return out

    def write_state(self, image):
        image = np.ascontiguousarray(image, dtype=np.uint8)
        self._check(self.lib.write_state(self.h, image.ctypes.data_as(C.c_void_p), image.size))

    def read_tfsf_record(self, k):
        n = self.lib.tfsf_record_size(self.h, int(k))
        out = np.empty(n, dtype=self.dtype)
        self._check(self.lib.read_tfsf_record(self.h, int(k), out.ctypes.data_as(C.c_void_p)))
        return out


class Batch:
    """A batch of 2-D single-precision models stepped together (mfd_batch_*).  Members are
    Steppers; each runs its steps done+1 .. it_last as one mfd_run call would and is then
    retired (usable again)."""

    def __init__(self, lib, device=0):
        if not getattr(lib, "has_batch", False):
            raise RuntimeError("this library has no batch entry points")
        self.lib = lib
        b = C.c_void_p()
        st = lib.batch_create(int(device), C.byref(b))
        if st != MFD_OK:
            raise StepperError(st, f"batch create failed ({st}): {lib.create_error().decode()}")
        self.b = b
        self.members = []

    def _check(self, st):
        if st != MFD_OK:
            raise StepperError(st, self.lib.batch_last_error(self.b).decode())

    def add(self, stepper, it_last):
        self._check(self.lib.batch_add(self.b, stepper.h, int(it_last)))
        self.members.append(stepper)

    def run(self, max_steps):
        """Advance every member by up to max_steps steps; returns the number still running."""
        n = C.c_int32()
        self._check(self.lib.batch_run(self.b, int(max_steps), C.byref(n)))
        return n.value

    def run_all(self, chunk=1 << 20):
        while self.run(chunk):
            pass

    def config(self, tile_x=0, tile_z=0, graph_steps=0):
        self._check(self.lib.batch_config(self.b, int(tile_x), int(tile_z), int(graph_steps)))

    def info(self):
        tx, tz, ms, cu, nl = C.c_int32(), C.c_int32(), C.c_double(), C.c_int64(), C.c_int64()
        self._check(self.lib.batch_info(self.b, C.byref(tx), C.byref(tz), C.byref(ms), C.byref(cu), C.byref(nl)))
        return {"tile": (tx.value, tz.value), "device_ms": ms.value, "cell_updates": cu.value, "launches": nl.value}

    def close(self):
        if getattr(self, "b", None):
            self.lib.batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass



class Borrowed(Stepper):
    """A handle owned by someone else (a server's finished request): readable like a
    Stepper, never destroyed by this object."""

    def __init__(self, lib, h, builder, dtype):
        self.lib = lib
        self.builder = builder
        self.dtype = np.dtype(dtype)
        d = builder.desc
        self.shape3 = (d.nx, d.ny, d.nz)
        self.N = d.nx * d.ny * d.nz
        self.h = h

    def close(self):
        self.h = None


class Server:
    """The library's serving loop (mfd_server_*): submit descriptors, poll, read the finished
    requests' handles, release them."""

    def __init__(self, lib, device=0, budget_bytes=160e9, max_active=64, max_solo=16):
        if not getattr(lib, "has_server", False):
            raise RuntimeError("this library has no server entry points")
        self.lib = lib
        s = C.c_void_p()
        st = lib.server_create(int(device), float(budget_bytes), int(max_active), int(max_solo), C.byref(s))
        if st != MFD_OK:
            raise StepperError(st, f"server create failed ({st}): {lib.create_error().decode()}")
        self.s = s
        self._keep = {}

    def _check(self, st):
        if st != MFD_OK:
            raise StepperError(st, self.lib.server_last_error(self.s).decode())

    def submit(self, builder):
        """Queue a descriptor (its DescBuilder is kept alive until the request is released)."""
        rid = C.c_int64()
        self._check(self.lib.server_submit(self.s, C.byref(builder.desc), C.byref(rid)))
        self._keep[rid.value] = builder
        return rid.value

    def poll(self, rid):
        """(state, [submitted, admitted, running, finished] seconds, footprint bytes, status)."""
        state, t, nb = C.c_int32(), (C.c_double * 4)(), C.c_int64()
        st = self.lib.server_poll(self.s, int(rid), C.byref(state), t, C.byref(nb))
        if st != MFD_OK and state.value != MFD_REQ_FAILED:
            self._check(st)
        return state.value, list(t), nb.value, st

    def wait(self, rid, timeout_s=3600.0):
        state = C.c_int32()
        self._check(self.lib.server_wait(self.s, int(rid), float(timeout_s), C.byref(state)))
        return state.value

    def handle(self, rid, dtype):
        h = C.c_void_p()
        self._check(self.lib.server_handle(self.s, int(rid), C.byref(h)))
        return Borrowed(self.lib, h, self._keep[rid], dtype)

    def release(self, rid):
        self._check(self.lib.server_release(self.s, int(rid)))
        self._keep.pop(rid, None)

    def info(self):
        q, r, d, f = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        u, pu, pa = C.c_double(), C.c_double(), C.c_int32()
        self._check(self.lib.server_info(self.s, C.byref(q), C.byref(r), C.byref(d), C.byref(f), C.byref(u),
                                         C.byref(pu), C.byref(pa)))
        return {"queued": q.value, "running": r.value, "done": d.value, "failed": f.value, "used_bytes": u.value,
                "peak_used_bytes": pu.value, "peak_active": pa.value}

    def close(self):
        if getattr(self, "s", None):
            self.lib.server_destroy(self.s)
            self.s = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
