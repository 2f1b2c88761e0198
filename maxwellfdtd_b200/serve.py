"""Serving loop: a stream of solves of mixed size and kind on one GPU.

The loop itself is the library's native server (mfd_server_*, csrc/serve.cuh), reachable
from any host language through the C ABI; Server below drives it from Python.  For a
library without one (the CPU oracle, which the host-logic tests use) the same policy runs
in Python threads.

No counterpart in the reference, which runs one solve! at a time.  Requests arrive over
time; each is admitted when its device-memory footprint fits the budget and a slot is
free, in arrival order.  Its state then stays resident on the device until it completes.
Admitted work overlaps on the device while earlier requests are still running:

- 2-D and small 3-D (at most BATCH_3D_MAX_CELLS cells) single-precision requests join the
  running batch (mfd_batch_*: persistent launches over all members, CUDA-graph replay),
  which admits them between its graph replays: continuous batching;
- every other request (larger 3-D, double precision) runs as a solo lane: its own handle
  and CUDA stream, stepped from a worker thread (the ctypes calls release the GIL), so
  several lanes and the batch keep the GPU busy together.  A large 3-D grid runs faster on
  its own: its core rows use the staged z-march kernels, while a batch updates one cell per
  thread.

Every request computes exactly what it computes alone (a batch member is bit-identical to
its solo run; a solo lane is a solo run), which the tests check.  The loop records arrival,
admission and completion times: queue wait and end-to-end latency (p50/p99) and the
aggregate Gcell-updates/s.
"""
import threading
import time
from collections import deque

import numpy as np

from . import _abi

BATCH_3D_MAX_CELLS = 1 << 20   # 3-D requests up to this many cells join the batch

_NCOMP = {1: 3, 2: 5, 3: 9}
_NCOMP_E = {1: 1, 2: 2, 3: 3}
_NCOMP_MON = {1: 2, 2: 3, 3: 6}


def footprint(builder, model, dtype=np.float32):
    """Device bytes mfd_create allocates for this descriptor: the fields and running sums
    in the padded layout, the material map and compact material state, CPML psi slabs,
    source, TFSF and monitor tables, per-step flags.  Used for admission (before anything
    is allocated)."""
    d = builder.desc
    T = np.dtype(dtype).itemsize
    R = 8 if (T == 8 or d.rho_fp64) else 4
    nd = d.ndim
    px = d.nx if nd == 1 else -(-d.nx // 32) * 32
    Np = px * d.ny * d.nz
    b = (_NCOMP[nd] + 1) * Np * T + d.nt * 4 + 4
    geom = np.asarray(model.geometry)
    if np.any(geom):
        b += Np + Np * T
    nc = _NCOMP_E[nd]
    for g in range(1, d.nmat + 1):
        m = d.mats[g - 1]
        b += T + 512
        idx = np.nonzero(geom == g)
        if len(idx[0]) == 0:
            continue
        bsize = 1
        for ax in idx:
            bsize *= int(ax.max() - ax.min() + 1)
        if m.nq > 0:
            b += 2 * m.nq * nc * bsize * T
        if m.plasma:
            b += 2 * m.rate_n * T + 3 * nc * bsize * T + 2 * bsize * R + bsize * T
    for f in range(6):
        L = d.pml[f]
        if L.nb <= 0:
            continue
        axis = f // 2
        used = nd == 3 or (nd == 2 and axis != 1) or (nd == 1 and axis == 2)
        if not used:
            continue
        b += L.nb * (8 * T) + 2 * L.nb * T
        if nd == 3:
            cnt = (L.nb * d.ny * d.nz, px * L.nb * d.nz, px * d.ny * L.nb)[axis]
            b += 4 * cnt * T
        elif nd == 2:
            cnt = L.nb * d.nz if axis == 0 else px * L.nb
            b += 2 * cnt * T
        else:
            b += 2 * L.nb * T
    for i in range(d.nsrc):
        s = d.srcs[i]
        b += s.npts * 8 + (d.nt * s.npts * 8 if s.wave else s.npts * 8 + d.nt * 8)
    if d.tfsf.enabled:
        b += sum(a.nbytes for a in builder.keep if isinstance(a, np.ndarray) and a.ndim == 2 and a.shape[0] == d.nt
                 and a.dtype == np.dtype(dtype))
    ring_vals = 0
    ncm = _NCOMP_MON[nd]
    for i in range(d.nmon):
        mo = d.mons[i]
        b += mo.npts * 4 + 64
        if mo.kind == _abi.MFD_MON_FIELD:
            b += ncm * d.nt * (1 if mo.sum else mo.npts) * T
        else:
            b += ncm * mo.nw * (1 if mo.sum else mo.npts) * 16 + d.nt * mo.nw * 16
        if mo.kind != _abi.MFD_MON_FIELD or mo.sum:
            ring_vals += ncm * mo.npts
    if ring_vals:
        ring_k = max(1, min(64, (512 << 20) // (T * ring_vals)))
        b += ring_k * ring_vals * T
    return int(b) + (64 << 10)   # small tables (descriptors, divisor checks) and rounding


class Request:
    """One solve: model + monitors, its descriptor (built by the client), times and results."""

    def __init__(self, rid, model, monitors, arrival, dtype=np.float32, mode="exact"):
        self.id = rid
        self.model = model
        self.monitors = monitors
        self.arrival = float(arrival)
        self.dtype = np.dtype(dtype)
        self.builder, self.meta = model.build_desc(dtype, monitors, mode=mode)
        self.bytes = footprint(self.builder, model, dtype)
        g = model.grid
        self.cells = g.Nx * g.Ny * g.Nz
        self.cell_updates = self.cells * model.Nt
        d = self.builder.desc
        small = (g.ndim == 2 and getattr(model, "polarization", "Hy") == "Hy") or \
            (g.ndim == 3 and self.cells <= BATCH_3D_MAX_CELLS)
        self.batchable = small and self.dtype == np.float32 and bool(d.rho_fp64) and not d.tfsf_record
        self.t_submit = self.t_admit = self.t_done = None
        self.t_created = self.t_ran = None       # upload finished, last step finished
        self.stepper = None
        self.out = None
        self.error = None


def read_results(st, req, fields=True):
    """The request's outputs: every monitor's record and, with fields, the final fields and Sa."""
    from .sources import comp_index, field_components
    nd = req.model.grid.ndim
    pol = getattr(req.model, "polarization", "Hy")
    out = {}
    if fields:
        out = {f"field/{c}": st.read_field(comp_index(c)) for c in field_components(nd, pol)}
        out["Sa"] = st.read_integral(_abi.MFD_INT_SA)
    comps = [c for c in field_components(nd, pol) if not c.startswith("D")]
    for k, mm in enumerate(req.meta["monitors"]):
        npts = len(mm["cells"])
        spectral = mm["kind"] == 1
        for c in comps:
            if spectral:
                nw = mm["dft"].Nw
                shape = (nw,) if mm["sum"] else (nw, npts)
            else:
                shape = (req.model.Nt,) if mm["sum"] else (req.model.Nt, npts)
            out[f"mon/{k}/{c}"] = st.read_monitor(k, comp_index(c), shape, spectral)
    return out


class Server:
    """Admission by device-memory footprint, continuous batching of 2-D and small 3-D
    requests, solo lanes for the rest; see the module docstring."""

    def __init__(self, lib, device=0, budget_bytes=160e9, max_active=64, max_solo=16, chunk=64,
                 use_batch=True, keep_results=True, read_fields=False):
        self.lib = lib
        self.device = device
        self.budget = float(budget_bytes)
        self.max_active = max_active
        self.max_solo = max_solo
        self.chunk = chunk
        self.use_batch = use_batch and getattr(lib, "has_batch", False)
        self.keep_results = keep_results
        self.read_fields = read_fields          # results: monitors, plus final fields and Sa when set
        self.lock = threading.Lock()            # server state
        self.wake = threading.Condition(self.lock)
        self.used = 0.0
        self.active = 0
        self.solo = 0
        self.batch = None                       # owned by the batch thread
        self.batch_members = []
        self.batch_pending = []                 # created, waiting to join the batch
        self.done = []
        self.errors = []
        self.admitted = []          # admission order
        self.peak_used = 0.0
        self.peak_active = 0

    # -- lanes ---------------------------------------------------------------------------
    def _finish(self, req, st, solo=False):
        """Reads a finished request and gives its memory, slot and (solo=True) its lane back,
        all in one critical section, so admission never sees a lane free while its request
        still counts as active."""
        req.t_ran = time.time()
        try:
            if self.keep_results:
                req.out = read_results(st, req, self.read_fields)
            req.status = st.status()
        except Exception as e:     # recorded per request, the loop goes on
            req.error = e
        finally:
            st.close()
        with self.lock:
            req.t_done = time.time()
            self.used -= req.bytes
            self.active -= 1
            if solo:
                self.solo -= 1
            self.done.append(req)
            if req.error is not None:
                self.errors.append(req)
            self.wake.notify_all()

    def _solo(self, req):
        st = None
        try:
            st = _abi.Stepper(self.lib, req.builder, req.dtype)
            req.t_created = time.time()
            st.run(1, req.model.Nt)
        except Exception as e:
            req.error = e
        if st is None:
            with self.lock:
                req.t_done = time.time()
                self.used -= req.bytes
                self.active -= 1
                self.solo -= 1
                self.done.append(req)
                self.errors.append(req)
                self.wake.notify_all()
            return
        self._finish(req, st, solo=True)

    def _batch_loop(self):
        """The batch's own thread: adds newly admitted members between graph replays
        (continuous batching), runs `chunk` steps, retires the members that finished."""
        while True:
            with self.lock:
                while not self.batch_members and not self.batch_pending and not self.stopping:
                    self.wake.wait(0.05)
                if self.stopping and not self.batch_members and not self.batch_pending:
                    return
                new, self.batch_pending = self.batch_pending, []
            for req in new:
                self.batch.add(req.stepper, req.model.Nt)
            with self.lock:
                self.batch_members.extend(new)
            self.batch.run(self.chunk)
            retired = []
            with self.lock:
                keep = []
                for req in self.batch_members:
                    (retired if req.stepper.status()[0] >= req.model.Nt else keep).append(req)
                self.batch_members = keep
            for req in retired:
                self._finish(req, req.stepper)

    # -- admission -----------------------------------------------------------------------
    def _admit(self, req):
        req.t_admit = time.time()
        self.used += req.bytes
        self.active += 1
        self.admitted.append(req.id)
        self.peak_used = max(self.peak_used, self.used)
        self.peak_active = max(self.peak_active, self.active)
        if req.batchable and self.use_batch:
            self.lock.release()
            try:
                req.stepper = _abi.Stepper(self.lib, req.builder, req.dtype)   # upload
                req.t_created = time.time()
            finally:
                self.lock.acquire()
            self.batch_pending.append(req)
            self.wake.notify_all()
        else:
            self.solo += 1
            threading.Thread(target=self._solo, args=(req,), daemon=True).start()

    def run(self, requests, realtime=True):
        """Serve `requests` (released at their arrival times, in seconds from now, when
        realtime; all at once otherwise).  Returns the statistics."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        for r in reqs:
            if r.bytes > self.budget:
                raise ValueError(f"request {r.id} needs {r.bytes} bytes, more than the budget")
        if getattr(self.lib, "has_server", False) and self.use_batch:
            return self._run_native(reqs, realtime)
        return self._run_python(reqs, realtime)

    def _run_native(self, reqs, realtime):
        """The library's server: requests are submitted at their arrival times; finished ones
        are read (their results kept when keep_results) and released."""
        srv = _abi.Server(self.lib, self.device, self.budget, self.max_active, self.max_solo)
        t0 = time.time()
        waiting = deque(reqs)
        live = {}
        try:
            while waiting or live:
                now = time.time() - t0
                while waiting and (not realtime or waiting[0].arrival <= now):
                    r = waiting.popleft()
                    r.t_submit = t0 + (r.arrival if realtime else 0.0)
                    live[srv.submit(r.builder)] = r
                for rid in list(live):
                    state, times, _, code = srv.poll(rid)
                    if state not in (_abi.MFD_REQ_DONE, _abi.MFD_REQ_FAILED):
                        continue
                    r = live.pop(rid)
                    r.t_admit, r.t_created, r.t_ran = t0 + times[1], t0 + times[2], t0 + times[3]
                    if state == _abi.MFD_REQ_DONE:
                        st = srv.handle(rid, r.dtype)
                        try:
                            if self.keep_results:
                                r.out = read_results(st, r, self.read_fields)
                            r.status = st.status()
                        except Exception as e:
                            r.error = e
                    else:
                        r.error = _abi.StepperError(code, self.lib.server_last_error(srv.s).decode())
                    srv.release(rid)
                    r.t_done = time.time()
                    self.done.append(r)
                    if r.error is not None:
                        self.errors.append(r)
                time.sleep(0.002)
            info = srv.info()
        finally:
            srv.close()
        self.admitted = [r.id for r in sorted(reqs, key=lambda r: (r.t_admit, r.arrival))]
        self.peak_used = info["peak_used_bytes"]
        self.peak_active = info["peak_active"]
        return self.stats(reqs, t0)

    def _run_python(self, reqs, realtime):
        self.stopping = False
        if self.use_batch:
            self.batch = _abi.Batch(self.lib, self.device)
            bt = threading.Thread(target=self._batch_loop, daemon=True)
            bt.start()
        t0 = time.time()
        waiting = deque(reqs)
        pending = deque()
        with self.lock:
            while len(self.done) < len(reqs):
                now = time.time() - t0
                while waiting and (not realtime or waiting[0].arrival <= now):
                    r = waiting.popleft()
                    r.t_submit = t0 + (r.arrival if realtime else 0.0)
                    pending.append(r)
                # admission in arrival order; a request that waits only for a solo lane does
                # not hold back batch requests behind it, one that waits for memory does
                blocked_solo = False
                for r in list(pending):
                    batch_lane = r.batchable and self.use_batch
                    if not batch_lane and (blocked_solo or self.solo >= self.max_solo):
                        blocked_solo = True
                        continue
                    if self.used + r.bytes > self.budget or self.active >= self.max_active:
                        break
                    pending.remove(r)
                    self._admit(r)
                timeout = 0.02
                if waiting and realtime:
                    timeout = max(0.0, min(timeout, waiting[0].arrival - (time.time() - t0)))
                self.wake.wait(timeout)
            self.stopping = True
            self.wake.notify_all()
        if self.use_batch:
            bt.join()
            self.batch.close()
            self.batch = None
        return self.stats(reqs, t0)

    @staticmethod
    def stats(reqs, t0):
        lat = np.array([r.t_done - r.t_submit for r in reqs])
        wait = np.array([r.t_admit - r.t_submit for r in reqs if r.t_admit is not None])
        t_first = min(r.t_submit for r in reqs)
        t_last = max(r.t_done for r in reqs)
        cu = sum(r.cell_updates for r in reqs)
        ph = lambda a, b: float(sum(getattr(r, b) - getattr(r, a) for r in reqs if getattr(r, a) and getattr(r, b)))
        return {"requests": len(reqs), "errors": sum(1 for r in reqs if r.error is not None),
                "phase_sum_s": {"queue": ph("t_submit", "t_admit"), "upload": ph("t_admit", "t_created"),
                                "steps": ph("t_created", "t_ran"), "read_back": ph("t_ran", "t_done")},
                "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
                "queue_wait_p50_s": float(np.percentile(wait, 50)) if len(wait) else None,
                "queue_wait_p99_s": float(np.percentile(wait, 99)) if len(wait) else None,
                "makespan_s": t_last - t_first, "cell_updates": int(cu),
                "gcell_updates_per_s": cu / (t_last - t_first) / 1e9,
                "batched": sum(1 for r in reqs if r.batchable), "solo": sum(1 for r in reqs if not r.batchable)}


def solve_alone(lib, req, fields=True):
    """The request solved by itself (mfd_create, one mfd_run, read-back); returns outputs and
    the wall time."""
    t = time.time()
    st = _abi.Stepper(lib, req.builder, req.dtype)
    st.run(1, req.model.Nt)
    out = read_results(st, req, fields)
    out_status = st.status()
    st.close()
    return out, out_status, time.time() - t
