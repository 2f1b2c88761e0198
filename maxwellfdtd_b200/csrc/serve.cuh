// serve.cuh -- the serving loop behind mfd_server_* (include/maxwellfdtd.h).
//
// No counterpart in the reference, which runs one solve! at a time.  Requests (model
// descriptors) arrive over time; each is admitted, in arrival order, when its device-memory
// footprint fits the budget and fewer than max_active requests are computing.  Admitted
// work overlaps on the device while earlier requests are still running:
//  - 2-D and small 3-D (at most MFD_SERVER_BATCH_3D_CELLS cells) single-precision requests
//    in the exact arithmetic join one running batch (mfd_batch_*: persistent launches over
//    all members, CUDA-graph replay), which takes new members between its runs of steps:
//    continuous batching;
//  - every other request runs as a solo lane: its own handle and stream, stepped by its own
//    host thread, at most max_solo at a time.
// A request that waits only for a solo lane does not hold back batch requests behind it;
// one that waits for memory does (arrival order).  Every request computes exactly what it
// computes alone: a batch member is bit-identical to its solo run, a solo lane is a solo run.
//
// A finished request keeps its handle (and its share of the budget) until the caller has
// read what it needs through mfd_read_* and calls mfd_server_release.
#pragma once

#include <condition_variable>
#include <deque>

#define MFD_SERVER_BATCH_3D_CELLS (1 << 20)

namespace mfd {

// Device bytes mfd_create allocates for a descriptor, before anything is allocated: fields
// and running sums in the padded layout, the material map and each material's compact state
// (from the bounding box of its cells), CPML psi slabs and profiles, source tables, TFSF
// incident arrays (compact layouts counted compact), monitor records, accumulators and the
// staging ring, the per-step flags, and 64 KiB for small tables.
static int64_t desc_footprint(const mfd_desc* d) {
    const int64_t T = d->dtype == MFD_F64 ? 8 : 4;
    const int64_t R = (T == 8 || d->rho_fp64) ? 8 : 4;
    const int nd = d->ndim;
    const int64_t px = nd == 1 ? d->nx : (d->nx + 31) / 32 * 32;
    const int64_t Np = px * d->ny * d->nz;
    static const int ncomp[4] = {0, 3, 5, 9};
    const bool ey2 = nd == 2 && d->polarization == MFD_POL_EY;   // Hx, Hz, Dy, Ey
    int64_t b = ((ey2 ? 4 : ncomp[nd]) + 1) * Np * T + d->nt * 4 + 4;
    const int nmat = d->nmat;
    std::vector<int> x0(nmat + 1, INT32_MAX), x1(nmat + 1, -1), y0(nmat + 1, INT32_MAX), y1(nmat + 1, -1),
        z0(nmat + 1, INT32_MAX), z1(nmat + 1, -1);
    bool any = false;
    if (d->geometry || (d->nshape > 0 && d->shapes && d->coords[2])) {
        for (int iz = 0; iz < d->nz; ++iz)
            for (int iy = 0; iy < d->ny; ++iy) {
                const uint8_t* row = d->geometry ? d->geometry + (size_t)d->nx * (iy + (size_t)d->ny * iz) : nullptr;
                for (int ix = 0; ix < d->nx; ++ix) {
                    int g = 0;
                    if (row) g = row[ix];
                    else {   // the shapes, as the device evaluates them (geometry.cuh)
                        const double x = nd >= 2 && d->coords[0] ? d->coords[0][ix] : 0.0;
                        const double y = nd == 3 && d->coords[1] ? d->coords[1][iy] : 0.0;
                        for (int k = 0; k < d->nshape; ++k)
                            if (shape_covers(d->shapes[k], x, y, d->coords[2][iz])) g = d->shapes[k].material;
                    }
                    if (!g || g > nmat) continue;
                    any = true;
                    x0[g] = std::min(x0[g], ix); x1[g] = std::max(x1[g], ix);
                    y0[g] = std::min(y0[g], iy); y1[g] = std::max(y1[g], iy);
                    z0[g] = std::min(z0[g], iz); z1[g] = std::max(z1[g], iz);
                }
            }
    }
    if (any) b += Np + Np * T;
    const int nc = ey2 ? 1 : nd;
    for (int g = 1; g <= nmat; ++g) {
        const mfd_material& m = d->mats[g - 1];
        b += T + 512;
        if (x1[g] < 0) continue;
        const int64_t bs = (int64_t)(x1[g] - x0[g] + 1) * (y1[g] - y0[g] + 1) * (z1[g] - z0[g] + 1);
        if (m.nq > 0) b += 2 * m.nq * nc * bs * T;
        if (m.plasma) b += 2 * (int64_t)m.rate_n * T + 3 * nc * bs * T + 2 * bs * R + bs * T;
    }
    for (int f = 0; f < 6; ++f) {
        const mfd_pml_layer& L = d->pml[f];
        if (L.nb <= 0) continue;
        const int axis = f / 2;
        const bool used = nd == 3 || (nd == 2 && axis != 1) || (nd == 1 && axis == 2);
        if (!used) continue;
        b += (int64_t)L.nb * (8 * T) + 2 * (int64_t)L.nb * T;
        if (nd == 3) {
            const int64_t cnt = axis == 0 ? (int64_t)L.nb * d->ny * d->nz : axis == 1 ? px * L.nb * d->nz : px * d->ny * L.nb;
            b += 4 * cnt * T;
        } else if (nd == 2) {
            const int64_t cnt = axis == 0 ? (int64_t)L.nb * d->nz : px * L.nb;
            b += 2 * cnt * T;
        } else {
            b += 2 * (int64_t)L.nb * T;
        }
    }
    for (int i = 0; i < d->nsrc; ++i) {
        const mfd_source& s = d->srcs[i];
        b += s.npts * 8 + (s.wave ? d->nt * s.npts * 8 : s.npts * 8 + d->nt * 8);
    }
    // TFSF face arrays: the extents (a, b) of array k of a box, bytes by its layout
    auto face_bytes = [&](const int* i1, const int* i2, const int32_t* shape) {
        const int64_t Nx = i2[0] - i1[0], Ny = i2[1] - i1[1], Nz = i2[2] - i1[2];
        const int narr = nd == 3 ? 24 : nd == 2 ? 8 : 4;
        int64_t sum = 0;
        for (int k = 0; k < narr; ++k) {
            int64_t a = 1, bb = 1;
            if (nd == 2) a = (k < 4 ? Nz : Nx) + (ey2 ? 1 : 0);   // the second field set spans the nodes
            if (nd == 3) {
                const int face = k / 4, j = k % 4;
                const bool p = j == 0 || j == 3;
                if (face < 2) { a = p ? Ny + 1 : Ny; bb = p ? Nz : Nz + 1; }
                else if (face < 4) { a = p ? Nx + 1 : Nx; bb = p ? Nz : Nz + 1; }
                else { a = p ? Nx + 1 : Nx; bb = p ? Ny : Ny + 1; }
            }
            const int sh = shape ? shape[k] : MFD_INC_FULL;
            sum += (sh == MFD_INC_ALONG_B ? bb : sh == MFD_INC_ALONG_A ? a : sh == MFD_INC_UNIFORM ? 1 : a * bb) * d->nt * T;
        }
        return sum;
    };
    if (d->tfsf.enabled) b += face_bytes(d->tfsf.i1, d->tfsf.i2, d->tfsf.shape);
    if (d->tfsf_record) b += face_bytes(d->rec_i1, d->rec_i2, nullptr);
    static const int ncm[4] = {0, 2, 3, 6};
    int64_t ring_vals = 0;
    for (int i = 0; i < d->nmon; ++i) {
        const mfd_monitor& m = d->mons[i];
        b += m.npts * 4 + 64;
        if (m.kind == MFD_MON_FIELD) b += ncm[nd] * d->nt * (m.sum ? 1 : m.npts) * T;
        else b += ncm[nd] * (int64_t)m.nw * (m.sum ? 1 : m.npts) * 16 + d->nt * (int64_t)m.nw * 16;
        if (m.kind != MFD_MON_FIELD || m.sum) ring_vals += ncm[nd] * m.npts;
    }
    if (ring_vals) {
        const int64_t k = std::max<int64_t>(1, std::min<int64_t>(64, (512ll << 20) / (T * ring_vals)));
        b += k * ring_vals * T;
    }
    return b + (64 << 10);
}

}  // namespace mfd

struct mfd_server {
    struct Req {
        int64_t id = 0;
        mfd_desc desc{};          // the caller's arrays: valid until the request is running
        int64_t bytes = 0;
        bool batchable = false;
        int state = MFD_REQ_QUEUED;
        double t[4] = {0, 0, 0, 0};   // submitted, admitted, running (uploaded), finished
        mfd_handle* h = nullptr;
        int code = MFD_OK;
        std::string err;
    };
    int dev = 0;
    double budget = 0;
    int max_active = 64, max_solo = 16, chunk = 64;
    bool use_batch = true;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    std::mutex mu;
    std::condition_variable cv;
    std::map<int64_t, std::unique_ptr<Req>> reqs;
    std::deque<Req*> queue;                // submitted, not admitted
    std::deque<Req*> batch_pending;        // uploaded, waiting to join the batch
    std::vector<Req*> batch_members;
    double used = 0, peak_used = 0;
    int active = 0, solo = 0, peak_active = 0;
    int64_t next_id = 1, n_done = 0, n_failed = 0;
    bool stopping = false;
    mfd_batch* batch = nullptr;
    std::thread sched, bthread;   // solo lanes run on detached threads, counted by `solo`
    std::string err;

    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }

    // with mu held
    void finish(Req* r, int code, const std::string& msg) {
        r->t[3] = now();
        r->code = code;
        r->err = msg;
        r->state = code == MFD_OK ? MFD_REQ_DONE : MFD_REQ_FAILED;
        active--;
        if (code == MFD_OK) n_done++;
        else n_failed++;
        if (code != MFD_OK && r->h) {   // a failed request gives its memory back at once
            mfd_destroy(r->h);
            r->h = nullptr;
            used -= (double)r->bytes;
            r->bytes = 0;
        }
        cv.notify_all();
    }

    void solo_lane(Req* r) {
        mfd_handle* h = nullptr;
        int rc = create_handle(&r->desc, &h, false);
        std::string msg;
        if (rc != MFD_OK) msg = mfd_create_error();
        {
            std::lock_guard<std::mutex> lk(mu);
            r->h = h;
            r->t[2] = now();
            if (rc == MFD_OK) r->state = MFD_REQ_RUNNING;
            cv.notify_all();
        }
        if (rc == MFD_OK) {
            rc = mfd_run(h, 1, r->desc.nt);
            if (rc != MFD_OK) msg = mfd_last_error(h);
        }
        std::lock_guard<std::mutex> lk(mu);
        finish(r, rc, msg);
        solo--;   // last: the destructor waits for this count to reach zero
        cv.notify_all();
    }

    void batch_loop() {
        while (true) {
            std::vector<Req*> add;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait_for(lk, std::chrono::milliseconds(50),
                            [&] { return stopping || !batch_members.empty() || !batch_pending.empty(); });
                if (stopping && batch_members.empty() && batch_pending.empty()) return;
                add.assign(batch_pending.begin(), batch_pending.end());
                batch_pending.clear();
            }
            for (Req* r : add) {
                const int rc = mfd_batch_add(batch, r->h, r->desc.nt);
                std::lock_guard<std::mutex> lk(mu);
                if (rc == MFD_OK) batch_members.push_back(r);
                else finish(r, rc, mfd_batch_last_error(batch));
            }
            bool any;
            {
                std::lock_guard<std::mutex> lk(mu);
                any = !batch_members.empty();
            }
            if (!any) continue;
            int32_t n_active = 0;
            const int rc = mfd_batch_run(batch, chunk, &n_active);
            std::lock_guard<std::mutex> lk(mu);
            std::vector<Req*> keep;
            for (Req* r : batch_members) {
                int64_t done_steps = 0, bad = 0;
                int32_t kind = 0;
                mfd_status(r->h, &done_steps, &bad, &kind);
                if (rc != MFD_OK) finish(r, rc, mfd_batch_last_error(batch));
                else if (bad) finish(r, MFD_ERR_NONFINITE, mfd_last_error(r->h));
                else if (done_steps >= r->desc.nt) finish(r, MFD_OK, "");
                else keep.push_back(r);
            }
            batch_members.swap(keep);
        }
    }

    // with the lock held (released while a batch member uploads)
    void admit(std::unique_lock<std::mutex>& lk, Req* r) {
        r->t[1] = now();
        r->state = MFD_REQ_ADMITTED;
        used += (double)r->bytes;
        active++;
        peak_used = std::max(peak_used, used);
        peak_active = std::max(peak_active, active);
        if (r->batchable && use_batch) {
            lk.unlock();
            mfd_handle* h = nullptr;
            const int rc = create_handle(&r->desc, &h, false);
            const std::string msg = rc == MFD_OK ? "" : mfd_create_error();
            lk.lock();
            r->h = h;
            r->t[2] = now();
            if (rc != MFD_OK) {
                finish(r, rc, msg);
                return;
            }
            r->state = MFD_REQ_RUNNING;
            batch_pending.push_back(r);
            cv.notify_all();
        } else {
            solo++;
            std::thread([this, r] { solo_lane(r); }).detach();
        }
    }

    void schedule() {
        std::unique_lock<std::mutex> lk(mu);
        while (!stopping) {
            bool blocked_solo = false;
            for (auto it = queue.begin(); it != queue.end();) {
                Req* r = *it;
                const bool batch_lane = r->batchable && use_batch;
                if (!batch_lane && (blocked_solo || solo >= max_solo)) {
                    blocked_solo = true;
                    ++it;
                    continue;
                }
                if (used + (double)r->bytes > budget || active >= max_active) break;
                it = queue.erase(it);
                admit(lk, r);
                if (stopping) break;
            }
            cv.wait_for(lk, std::chrono::milliseconds(20));
        }
    }

    ~mfd_server() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stopping = true;
            cv.notify_all();
        }
        if (sched.joinable()) sched.join();
        {
            std::unique_lock<std::mutex> lk(mu);   // admitted solo lanes run to their end
            cv.wait(lk, [&] { return solo == 0; });
        }
        if (bthread.joinable()) bthread.join();
        for (auto& kv : reqs)
            if (kv.second->h) mfd_destroy(kv.second->h);
        if (batch) mfd_batch_destroy(batch);
    }
};

extern "C" {

int mfd_server_create(int32_t device, double budget_bytes, int32_t max_active, int32_t max_solo, mfd_server** out) {
    if (!out) return MFD_ERR_INVALID;
    *out = nullptr;
    if (!(budget_bytes > 0) || max_active < 1 || max_solo < 0) {
        g_create_error = "server: budget_bytes > 0, max_active >= 1 and max_solo >= 0 are required";
        return MFD_ERR_INVALID;
    }
    std::unique_ptr<mfd_server> s(new mfd_server);
    s->dev = device;
    s->budget = budget_bytes;
    s->max_active = max_active;
    s->max_solo = max_solo;
    const int rc = mfd_batch_create(device, &s->batch);
    if (rc != MFD_OK) return rc;
    s->bthread = std::thread([p = s.get()] { p->batch_loop(); });
    s->sched = std::thread([p = s.get()] { p->schedule(); });
    *out = s.release();
    return MFD_OK;
}

void mfd_server_destroy(mfd_server* s) { delete s; }

int mfd_server_submit(mfd_server* s, const mfd_desc* desc, int64_t* id) {
    if (!s || !desc || !id) return MFD_ERR_INVALID;
    const int rc = validate_desc(desc);
    if (rc != MFD_OK) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->err = "submit: " + g_create_error;
        return rc;
    }
    std::unique_ptr<mfd_server::Req> r(new mfd_server::Req);
    r->desc = *desc;
    r->bytes = desc_footprint(desc);
    const long long cells = (long long)desc->nx * desc->ny * desc->nz;
    r->batchable = ((desc->ndim == 2 && desc->polarization == MFD_POL_HY) ||
                    (desc->ndim == 3 && cells <= MFD_SERVER_BATCH_3D_CELLS)) && desc->dtype == MFD_F32 &&
                   desc->rho_fp64 && !desc->tfsf_record;
    std::lock_guard<std::mutex> lk(s->mu);
    if ((double)r->bytes > s->budget) {
        s->err = "submit: the request needs " + std::to_string(r->bytes) + " device bytes, more than the server's budget";
        return MFD_ERR_ADMISSION;
    }
    r->id = s->next_id++;
    r->t[0] = s->now();
    *id = r->id;
    s->queue.push_back(r.get());
    s->reqs[r->id] = std::move(r);
    s->cv.notify_all();
    return MFD_OK;
}

int mfd_server_poll(mfd_server* s, int64_t id, int32_t* state, double* times, int64_t* bytes) {
    if (!s) return MFD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) { s->err = "no such request"; return MFD_ERR_INVALID; }
    const mfd_server::Req& r = *it->second;
    if (state) *state = r.state;
    if (times) for (int k = 0; k < 4; ++k) times[k] = r.t[k];
    if (bytes) *bytes = r.bytes;
    if (r.state == MFD_REQ_FAILED) {
        s->err = r.err;
        return r.code;
    }
    return MFD_OK;
}

int mfd_server_wait(mfd_server* s, int64_t id, double timeout_s, int32_t* state) {
    if (!s) return MFD_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) { s->err = "no such request"; return MFD_ERR_INVALID; }
    mfd_server::Req* r = it->second.get();
    const bool ok = s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 0.0),
                                   [&] { return r->state == MFD_REQ_DONE || r->state == MFD_REQ_FAILED; });
    if (state) *state = r->state;
    if (!ok) { s->err = "the request did not finish within the wait"; return MFD_ERR_TIMEOUT; }
    if (r->state == MFD_REQ_FAILED) { s->err = r->err; return r->code; }
    return MFD_OK;
}

int mfd_server_handle(mfd_server* s, int64_t id, mfd_handle** h) {
    if (!s || !h) return MFD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) { s->err = "no such request"; return MFD_ERR_INVALID; }
    if (it->second->state != MFD_REQ_DONE) { s->err = "the request has not finished"; return MFD_ERR_INVALID; }
    *h = it->second->h;
    return MFD_OK;
}

int mfd_server_release(mfd_server* s, int64_t id) {
    if (!s) return MFD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) { s->err = "no such request"; return MFD_ERR_INVALID; }
    mfd_server::Req* r = it->second.get();
    if (r->state != MFD_REQ_DONE && r->state != MFD_REQ_FAILED) { s->err = "the request has not finished"; return MFD_ERR_INVALID; }
    if (r->h) mfd_destroy(r->h);
    s->used -= (double)r->bytes;
    s->reqs.erase(it);
    s->cv.notify_all();
    return MFD_OK;
}

int mfd_server_info(mfd_server* s, int64_t* queued, int64_t* running, int64_t* done, int64_t* failed, double* used_bytes,
                    double* peak_used_bytes, int32_t* peak_active) {
    if (!s) return MFD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    if (queued) *queued = (int64_t)s->queue.size();
    if (running) *running = s->active;
    if (done) *done = s->n_done;
    if (failed) *failed = s->n_failed;
    if (used_bytes) *used_bytes = s->used;
    if (peak_used_bytes) *peak_used_bytes = s->peak_used;
    if (peak_active) *peak_active = s->peak_active;
    return MFD_OK;
}

int64_t mfd_server_footprint(const mfd_desc* desc) {
    if (!desc || validate_desc(desc) != MFD_OK) return -1;
    return desc_footprint(desc);
}

const char* mfd_server_last_error(mfd_server* s) {
    if (!s) return "null server";
    std::lock_guard<std::mutex> lk(s->mu);
    thread_local std::string copy;
    copy = s->err;
    return copy.c_str();
}

}  // extern "C"
