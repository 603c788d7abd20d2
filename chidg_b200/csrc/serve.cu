// serve.cu -- a continuous-batching solve server behind the C ABI.
//
// Requests (one assembled system each: pattern, packed block values, right-
// hand side) are submitted at any time and wait in arrival order.  A
// dispatcher thread forms a batch whenever a worker slot is free: the oldest
// request and, in arrival order, the later ones that share its number of time
// levels and fit the part of the device-memory budget that running batches do
// not hold, up to max_batch systems (a batch of one may exceed the budget).  Admission waits while the batches on the device already hold the
// budget.  Each slot is a worker thread with a context (and stream) of its
// own, so batches run concurrently; a batch is solved by
// chidg_gpu_fgmres_solve_batched, whose
// per-system arithmetic does not depend on the other systems of the batch.
// A request either hands over host arrays (uploaded into the batch in place)
// or a fill function that writes its system on the device when the batch is
// formed.  Every batch leaves a record of its phases (host clock) and of its
// solve's device time (CUDA events on the worker's stream).
// Host code only: no kernel of its own.
#include "chidg_gpu_internal.cuh"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

struct Request {
    int64_t ticket = 0;
    chidg_gpu_pattern pat{};
    std::vector<int32_t> nvars, nterms, proc, re, rt, ce, ct, kind;
    const double* values = nullptr;      // caller-owned until the request's wait returns
    const double* rhs = nullptr;
    chidg_gpu_fill_fn fill = nullptr;    // or: the system is written on the device by fill(user, ...)
    void* user = nullptr;
    int64_t nval = 0, n = 0, bytes = 0;
    double arrival = 0, start = 0, finish = 0;
    int32_t batch_size = 0;
    std::vector<double> x;
    chidg_gpu_fgmres_result result{};
    int status = CHIDG_GPU_OK;
    std::string error;
    bool done = false;
};

struct Job {
    std::vector<std::shared_ptr<Request>> batch;
    int64_t bytes = 0;
    int64_t index = 0;                   // the batch's number, in the order batches are formed
};

// formed, taken, on the device, set up, solved, on the host; device ms; systems; slot
struct BatchRecord {
    double t[6] = {0, 0, 0, 0, 0, 0};
    double device_ms = 0;
    int32_t nsys = 0, slot = -1;
    bool finished = false;
};

}  // namespace

struct chidg_gpu_server {
    int device = 0;
    int32_t max_batch = 16, precon_kind = CHIDG_PRECON_ILU0;
    int64_t budget = 0;
    chidg_gpu_fgmres_opts opts{};
    std::chrono::steady_clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv;              // queue, slots, memory and completion changes
    std::deque<std::shared_ptr<Request>> pending;
    std::map<int64_t, std::shared_ptr<Request>> live;   // submitted, not yet waited for
    std::deque<Job> jobs;                    // formed batches not yet taken by a worker
    int64_t next_ticket = 0;
    bool stopping = false;                   // no more submissions; the dispatcher drains the queue
    bool workers_stop = false;               // the workers exit once the job queue is empty
    int idle = 0;                            // workers without a batch
    int nslots = 0;
    int exclusive = 0;                       // a batch runs alone after running out of memory
    int waiting = 0;                         // batches waiting to run alone (form and admit nothing meanwhile)
    int64_t mem_used = 0, peak_mem = 0, batches = 0;
    std::vector<chidg_gpu_ctx*> all_ctx;
    std::vector<BatchRecord> log;            // one per formed batch
    std::thread dispatcher;
    std::vector<std::thread> workers;

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

// Device bytes one request needs: its blocks (nval values), the ILU factors
// (the values of its diagonal and lower blocks, nlow), their FP32 copies in a
// mixed mode, the Krylov basis and a few vectors.  An estimate for admission:
// a batch that does not fit after all is solved in halves.
int64_t request_bytes(int64_t nval, int64_t nlow, int64_t n, int32_t nkrylov, int32_t precision) {
    const int64_t blocks = 8 * (nval + nlow) + (precision != CHIDG_GPU_FP64 ? 4 * (nval + nlow) : 0);
    return blocks + 8 * n * (2 * ((int64_t)nkrylov + 1) + 6);
}

// Solve requests [first, last) of a batch as one packed system on ctx; on
// success each request's result and solution are filled in.  ph[2..5]
// accumulate the durations of the phases (on the device, set up, solved,
// solution on the host) and *dev_ms the solves' device time, over the parts
// solved; freeing the batch's objects afterwards is not counted.
int solve_group(chidg_gpu_server* S, chidg_gpu_ctx* ctx, std::vector<std::shared_ptr<Request>>& batch, int first,
                int last, double* ph, float* dev_ms, std::string& err, bool alone = false) {
    const int nsys = last - first;
    // the packed pattern: system s owns elements sys_elem[s] .. sys_elem[s+1]-1
    std::vector<int32_t> nv, nt, pr, re, rt, ce, ct, kd, sys_elem(nsys + 1, 0);
    int64_t n = 0;
    for (int s = 0; s < nsys; ++s) {
        const Request& q = *batch[first + s];
        const int32_t e0 = sys_elem[s];
        nv.insert(nv.end(), q.nvars.begin(), q.nvars.end());
        nt.insert(nt.end(), q.nterms.begin(), q.nterms.end());
        pr.insert(pr.end(), q.proc.begin(), q.proc.end());
        for (size_t k = 0; k < q.re.size(); ++k) {
            re.push_back(q.re[k] + e0); ce.push_back(q.ce[k] + e0);
            rt.push_back(q.rt[k]); ct.push_back(q.ct[k]); kd.push_back(q.kind[k]);
        }
        sys_elem[s + 1] = e0 + q.pat.nelem;
        n += q.n;
    }
    chidg_gpu_pattern pat{};
    pat.nelem = sys_elem[nsys]; pat.ntime = batch[first]->pat.ntime; pat.nblocks = (int64_t)re.size();
    pat.elem_nvars = nv.data(); pat.elem_nterms = nt.data(); pat.elem_proc = pr.data();
    pat.blk_row_elem = re.data(); pat.blk_row_time = rt.data(); pat.blk_col_elem = ce.data();
    pat.blk_col_time = ct.data(); pat.blk_kind = kd.data();

    chidg_gpu_matrix* A = nullptr;
    chidg_gpu_vector *b = nullptr, *x = nullptr;
    chidg_gpu_precon* M = nullptr;
    std::vector<chidg_gpu_fgmres_result> res(nsys);
    std::vector<double> xh;
    double t0 = S->now();
    int st = chidg_gpu_matrix_create(ctx, &pat, &A);
    if (!st) st = chidg_gpu_vector_create(A, &b);
    if (!st) st = chidg_gpu_vector_create(A, &x);
    {
        int64_t v0 = 0, o = 0;
        for (int s = 0; s < nsys && !st; ++s) {
            const Request& q = *batch[first + s];
            if (q.fill) {
                st = q.fill(q.user, ctx, A, b, x, sys_elem[s]);
            } else {
                st = chidg_gpu_matrix_upload_range(A, q.values, v0, q.nval);
                if (!st) st = chidg_gpu_vector_upload_range(b, q.rhs, o, q.n);
            }
            v0 += q.nval;
            o += q.n;
        }
    }
    if (!st) st = chidg_gpu_vector_clear(x);        // the initial guess (fill functions may use x as scratch)
    if (!st) st = chidg_gpu_ctx_sync(ctx);
    double t1 = S->now();
    ph[2] += t1 - t0;
    if (!st) st = chidg_gpu_precon_create(A, S->precon_kind, &M);
    double t2 = S->now();
    ph[3] += t2 - t1;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    const bool timed = cudaEventCreate(&ev[0]) == cudaSuccess && cudaEventCreate(&ev[1]) == cudaSuccess;
    if (timed) cudaEventRecord(ev[0], ctx->stream);
    if (!st) st = chidg_gpu_fgmres_solve_batched(A, M, nsys, sys_elem.data(), b, x, &S->opts, res.data(), nullptr, 0);
    if (timed) cudaEventRecord(ev[1], ctx->stream);
    ph[4] += S->now() - t2;
    const double t3 = S->now();
    if (!st) { xh.resize((size_t)n); st = chidg_gpu_vector_download(x, xh.data()); }
    ph[5] += S->now() - t3;
    float ms = 0.0f;
    if (timed && cudaEventSynchronize(ev[1]) == cudaSuccess && cudaEventElapsedTime(&ms, ev[0], ev[1]) == cudaSuccess)
        *dev_ms += ms;
    for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    if (st) {
        char buf[512] = {0};
        chidg_gpu_last_error(ctx, buf, (int32_t)sizeof(buf));
        err = buf;
    }
    if (M) chidg_gpu_precon_destroy(M);
    if (x) chidg_gpu_vector_destroy(x);
    if (b) chidg_gpu_vector_destroy(b);
    if (A) chidg_gpu_matrix_destroy(A);
    if (st == CHIDG_GPU_ENOMEM && nsys > 1) {
        // the estimate let in more than the device holds: solve the halves in turn
        chidg_gpu_ctx_sync(ctx);
        const int mid = first + nsys / 2;
        std::string e2;
        st = solve_group(S, ctx, batch, first, mid, ph, dev_ms, e2);
        if (!st) st = solve_group(S, ctx, batch, mid, last, ph, dev_ms, e2);
        err = e2;
        return st;
    }
    if (st == CHIDG_GPU_ENOMEM && !alone) {
        // one system that does not fit beside the other batches on the device:
        // admit nothing new, wait (bounded) until it is the only batch left, and
        // try once more
        chidg_gpu_ctx_sync(ctx);
        {
            // every other worker idle or waiting too (a waiting worker holds no
            // device memory), and no other batch running alone
            std::unique_lock<std::mutex> lk(S->mu);
            ++S->waiting;
            S->cv.notify_all();
            S->cv.wait_for(lk, std::chrono::seconds(600),
                           [S] { return S->exclusive == 0 && S->idle + S->waiting >= S->nslots; });
            --S->waiting;
            ++S->exclusive;
        }
        std::string e2;
        st = solve_group(S, ctx, batch, first, last, ph, dev_ms, e2, true);
        err = e2;
        std::lock_guard<std::mutex> lk(S->mu);
        --S->exclusive;
        S->cv.notify_all();
        return st;
    }
    if (!st) {
        int64_t o = 0;
        for (int s = 0; s < nsys; ++s) {
            Request& q = *batch[first + s];
            q.result = res[s];
            q.x.assign(xh.begin() + o, xh.begin() + o + q.n);
            o += q.n;
        }
    }
    return st;
}

void run_batch(chidg_gpu_server* S, chidg_gpu_ctx* ctx, int slot, Job job) {
    std::vector<std::shared_ptr<Request>>& batch = job.batch;
    double ph[6] = {0, 0, 0, 0, 0, 0};
    ph[1] = S->now();
    cudaSetDevice(ctx->device);
    const int nsys = (int)batch.size();
    float dev_ms = 0.0f;
    std::string err;
    const int st = solve_group(S, ctx, batch, 0, nsys, ph, &dev_ms, err);
    // phases as times from the durations (parts solved in turn add up)
    for (int i = 2; i < 6; ++i) ph[i] += ph[i - 1];

    std::lock_guard<std::mutex> lk(S->mu);
    for (int s = 0; s < nsys; ++s) {
        Request& q = *batch[s];
        q.status = st;
        q.error = err;
        q.start = ph[1];
        q.finish = ph[5];
        q.batch_size = nsys;
        if (st) q.x.clear();
        q.done = true;
    }
    BatchRecord& r = S->log[(size_t)job.index];
    for (int i = 1; i < 6; ++i) r.t[i] = ph[i];
    r.device_ms = dev_ms;
    r.nsys = nsys;
    r.slot = slot;
    r.finished = true;
    S->mem_used -= job.bytes;
    ++S->idle;
    S->cv.notify_all();
}

void work(chidg_gpu_server* S, chidg_gpu_ctx* ctx, int slot) {
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        S->cv.wait(lk, [S] { return !S->jobs.empty() || S->workers_stop; });
        if (S->jobs.empty()) return;         // workers_stop and nothing left
        Job job = std::move(S->jobs.front());
        S->jobs.pop_front();
        lk.unlock();
        run_batch(S, ctx, slot, std::move(job));
        lk.lock();
    }
}

void dispatch(chidg_gpu_server* S) {
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        S->cv.wait(lk, [S] {
            return (!S->pending.empty() && S->idle > 0 && S->exclusive == 0 && S->waiting == 0) ||
                   (S->stopping && S->pending.empty());
        });
        if (S->pending.empty()) break;       // stopping, queue drained
        // the oldest request, then the later ones of its number of time levels
        // that fit the memory not held by running batches, in arrival order;
        // requests passed over keep their place
        std::vector<std::shared_ptr<Request>> batch{S->pending.front()};
        S->pending.pop_front();
        int64_t bytes = batch[0]->bytes;
        const int64_t room = S->budget - S->mem_used;
        for (auto it = S->pending.begin(); it != S->pending.end() && (int32_t)batch.size() < S->max_batch;) {
            if ((*it)->pat.ntime == batch[0]->pat.ntime && bytes + (*it)->bytes <= room) {
                bytes += (*it)->bytes;
                batch.push_back(*it);
                it = S->pending.erase(it);
            } else {
                ++it;
            }
        }
        // admission by device memory: wait for running batches to finish
        S->cv.wait(lk, [S, bytes] {
            return (S->mem_used + bytes <= S->budget || S->mem_used == 0) && S->exclusive == 0 && S->waiting == 0;
        });
        S->mem_used += bytes;
        S->peak_mem = std::max(S->peak_mem, S->mem_used);
        const int64_t index = S->batches++;
        --S->idle;
        S->log.emplace_back();
        S->log.back().t[0] = S->now();
        S->jobs.push_back(Job{std::move(batch), bytes, index});
        S->cv.notify_all();
    }
}

}  // namespace

extern "C" int chidg_gpu_serve_create(int device, int32_t slots, int64_t mem_budget, int32_t max_batch,
                                      int32_t precon_kind, const chidg_gpu_fgmres_opts* opts, chidg_gpu_server** out) {
    if (!out || slots < 1 || mem_budget <= 0 || max_batch < 1 || precon_kind < CHIDG_PRECON_IDENTITY ||
        precon_kind > CHIDG_PRECON_HB)
        return CHIDG_GPU_EINVAL;
    *out = nullptr;
    auto* S = new chidg_gpu_server();
    S->device = device;
    S->budget = mem_budget;
    S->max_batch = max_batch;
    S->precon_kind = precon_kind;
    if (opts) S->opts = *opts;
    else chidg_gpu_fgmres_default_opts(&S->opts);
    S->t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < slots; ++i) {
        chidg_gpu_ctx* c = nullptr;
        const int st = chidg_gpu_ctx_create(device, nullptr, &c);
        if (st) {
            for (chidg_gpu_ctx* d : S->all_ctx) chidg_gpu_ctx_destroy(d);
            delete S;
            return st;
        }
        S->all_ctx.push_back(c);
    }
    S->idle = slots;
    S->nslots = slots;
    for (size_t i = 0; i < S->all_ctx.size(); ++i) S->workers.emplace_back(work, S, S->all_ctx[i], (int)i);
    S->dispatcher = std::thread(dispatch, S);
    *out = S;
    return CHIDG_GPU_OK;
}

namespace {
// a request's copy of the pattern and its sizes; nullptr for a pattern that is not valid
std::shared_ptr<Request> new_request(const chidg_gpu_server* S, const chidg_gpu_pattern* pat) {
    if (!pat || pat->nelem <= 0 || pat->ntime <= 0 || pat->nblocks <= 0 || !pat->elem_nvars || !pat->elem_nterms ||
        !pat->blk_row_elem || !pat->blk_row_time || !pat->blk_col_elem || !pat->blk_col_time || !pat->blk_kind)
        return nullptr;
    auto q = std::make_shared<Request>();
    const int32_t ne = pat->nelem;
    const int64_t nb = pat->nblocks;
    q->nvars.assign(pat->elem_nvars, pat->elem_nvars + ne);
    q->nterms.assign(pat->elem_nterms, pat->elem_nterms + ne);
    q->proc.assign(ne, 0);
    if (pat->elem_proc) q->proc.assign(pat->elem_proc, pat->elem_proc + ne);
    q->re.assign(pat->blk_row_elem, pat->blk_row_elem + nb);
    q->rt.assign(pat->blk_row_time, pat->blk_row_time + nb);
    q->ce.assign(pat->blk_col_elem, pat->blk_col_elem + nb);
    q->ct.assign(pat->blk_col_time, pat->blk_col_time + nb);
    q->kind.assign(pat->blk_kind, pat->blk_kind + nb);
    for (int32_t e = 0; e < ne; ++e) {
        if (q->nvars[e] <= 0 || q->nterms[e] <= 0) return nullptr;
        q->n += (int64_t)pat->ntime * q->nvars[e] * q->nterms[e];
    }
    int64_t nlow = 0;                        // values of the diagonal and lower blocks (natural order)
    for (int64_t k = 0; k < nb; ++k) {
        if (q->re[k] < 0 || q->re[k] >= ne || q->ce[k] < 0 || q->ce[k] >= ne) return nullptr;
        const int64_t v = (int64_t)q->nvars[q->re[k]] * q->nterms[q->re[k]] * q->nvars[q->ce[k]] * q->nterms[q->ce[k]];
        q->nval += v;
        if (q->ce[k] < q->re[k] || (q->ce[k] == q->re[k] && q->ct[k] <= q->rt[k])) nlow += v;
    }
    q->pat.nelem = pat->nelem;               // the arrays are copied above; keep only the sizes
    q->pat.ntime = pat->ntime;
    q->pat.nblocks = pat->nblocks;
    q->bytes = request_bytes(q->nval, nlow, q->n, S->opts.nkrylov, S->opts.precision);
    return q;
}

int enqueue(chidg_gpu_server* S, std::shared_ptr<Request> q, int64_t* ticket) {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stopping) return CHIDG_GPU_ESTATE;
    q->arrival = S->now();
    q->ticket = S->next_ticket++;
    *ticket = q->ticket;
    S->live[q->ticket] = q;
    S->pending.push_back(std::move(q));
    S->cv.notify_all();
    return CHIDG_GPU_OK;
}
}  // namespace

extern "C" int chidg_gpu_serve_submit(chidg_gpu_server* S, const chidg_gpu_pattern* pat, const double* values,
                                      const double* rhs, int64_t* ticket) {
    if (!S || !values || !rhs || !ticket) return CHIDG_GPU_EINVAL;
    std::shared_ptr<Request> q = new_request(S, pat);
    if (!q) return CHIDG_GPU_EINVAL;
    q->values = values;
    q->rhs = rhs;
    return enqueue(S, std::move(q), ticket);
}

extern "C" int chidg_gpu_serve_submit_fill(chidg_gpu_server* S, const chidg_gpu_pattern* pat, chidg_gpu_fill_fn fill,
                                           void* user, int64_t* ticket) {
    if (!S || !fill || !ticket) return CHIDG_GPU_EINVAL;
    std::shared_ptr<Request> q = new_request(S, pat);
    if (!q) return CHIDG_GPU_EINVAL;
    q->fill = fill;
    q->user = user;
    return enqueue(S, std::move(q), ticket);
}

extern "C" int chidg_gpu_serve_wait(chidg_gpu_server* S, int64_t ticket, double* x, chidg_gpu_fgmres_result* result,
                                    double* timing) {
    if (!S) return CHIDG_GPU_EINVAL;
    std::unique_lock<std::mutex> lk(S->mu);
    const auto it = S->live.find(ticket);
    if (it == S->live.end()) return CHIDG_GPU_EINVAL;
    const std::shared_ptr<Request> q = it->second;
    S->cv.wait(lk, [&q] { return q->done; });
    S->live.erase(ticket);
    if (x && !q->status) std::memcpy(x, q->x.data(), sizeof(double) * q->x.size());
    if (result) *result = q->result;
    if (timing) { timing[0] = q->arrival; timing[1] = q->start; timing[2] = q->finish; timing[3] = q->batch_size; }
    return q->status;
}

extern "C" int chidg_gpu_serve_stats(chidg_gpu_server* S, int64_t* batches, int64_t* peak_mem_bytes) {
    if (!S) return CHIDG_GPU_EINVAL;
    std::lock_guard<std::mutex> lk(S->mu);
    if (batches) *batches = S->batches;
    if (peak_mem_bytes) *peak_mem_bytes = S->peak_mem;
    return CHIDG_GPU_OK;
}

extern "C" int chidg_gpu_serve_batch_log(chidg_gpu_server* S, int64_t i, double* rec) {
    if (!S || !rec) return CHIDG_GPU_EINVAL;
    std::lock_guard<std::mutex> lk(S->mu);
    if (i < 0 || i >= (int64_t)S->log.size() || !S->log[(size_t)i].finished) return CHIDG_GPU_EINVAL;
    const BatchRecord& r = S->log[(size_t)i];
    for (int k = 0; k < 6; ++k) rec[k] = r.t[k];
    rec[6] = r.device_ms;
    rec[7] = r.nsys;
    rec[8] = r.slot;
    return CHIDG_GPU_OK;
}

extern "C" int chidg_gpu_serve_destroy(chidg_gpu_server* S) {
    if (!S) return CHIDG_GPU_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
        S->cv.notify_all();
    }
    S->dispatcher.join();                    // forms batches for every queued request, then stops
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->workers_stop = true;
        S->cv.notify_all();
    }
    for (std::thread& t : S->workers) t.join();   // each finishes the queued batches first
    for (chidg_gpu_ctx* c : S->all_ctx) chidg_gpu_ctx_destroy(c);
    delete S;
    return CHIDG_GPU_OK;
}
