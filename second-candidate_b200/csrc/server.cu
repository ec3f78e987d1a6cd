// Request loop with continuous batching.
//
// A server owns a few slots -- each a CUDA stream with its own search
// workspace and pinned staging -- and one device arena for the per-request
// buffers (queries, tables, outputs).  Callers submit requests (a batch of
// queries with its own parameters: k, T, arithmetic form, re-rank) from any
// thread and wait on a ticket.  One worker thread admits requests in arrival
// order whenever a slot is free and the arena has room for the request's
// buffers, enqueues copy-in, tables, search and copy-out on the slot's
// stream, and retires requests as their streams finish.  Requests that arrive
// while others run are admitted as soon as a slot and memory free up, and
// requests in different slots run concurrently on the device.  Codebooks and
// codes stay resident in the index; a request in the mix runs the same
// kernels on the same inputs as alone, so its results are identical.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <thread>
#include <unordered_map>
#include <vector>

#include "index.h"

namespace scg {

std::string last_error_string();

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t ticket = 0;
    scg_search_params p;
    const float *Q = nullptr;
    int nq = 0;
    int *ids = nullptr;
    float *dists = nullptr;
    int *sums = nullptr;
    size_t need = 0;  // arena bytes
    Clock::time_point t_submit, t_start, t_done;
    int state = 0;  // 0 queued, 1 running, 2 done
    int rc = SCG_OK;
    std::string err;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    Workspace ws;
    float *hq = nullptr;  // pinned staging: queries in, results out
    int *hids = nullptr;
    float *hd = nullptr;
    int *hs = nullptr;
    Request *req = nullptr;
    size_t off = 0, len = 0;  // arena range of the running request
};

size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace
}  // namespace scg

using namespace scg;

struct scg_server {
    scg_index *h = nullptr;
    int max_batch = 0, max_R = 0;
    std::vector<Slot> slots;
    DevBuf arena;
    size_t arena_bytes = 0;
    std::map<size_t, size_t> freelist;  // offset -> length
    std::deque<Request *> pending;
    std::unordered_map<uint64_t, Request *> reqs;
    uint64_t next_ticket = 1;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread worker;
    bool stop = false;
    int inflight = 0, max_inflight = 0;
    long long completed = 0;
};

namespace {

bool arena_alloc(scg_server *s, size_t len, size_t *off) {
    for (auto it = s->freelist.begin(); it != s->freelist.end(); ++it) {
        if (it->second >= len) {
            *off = it->first;
            const size_t rem = it->second - len, noff = it->first + len;
            s->freelist.erase(it);
            if (rem) s->freelist[noff] = rem;
            return true;
        }
    }
    return false;
}

void arena_free(scg_server *s, size_t off, size_t len) {
    auto it = s->freelist.emplace(off, len).first;
    auto nx = std::next(it);
    if (nx != s->freelist.end() && it->first + it->second == nx->first) {
        it->second += nx->second;
        s->freelist.erase(nx);
    }
    if (it != s->freelist.begin()) {
        auto pv = std::prev(it);
        if (pv->first + pv->second == it->first) {
            pv->second += it->second;
            s->freelist.erase(it);
        }
    }
}

size_t request_bytes(const scg_index *h, const scg_search_params *p, int nq) {
    return up256(4ull * nq * h->dim) + 2 * up256(4ull * nq * p->R) + up256(4ull * nq) +
           req_bytes(nq, h->dim, h->mc, h->kc, h->mp, h->kp, p->R, p->rerank);
}

// Re-searches a request whose visited lists outgrew the split kernels' pool
// with the fused kernel, on its slot, synchronously; results land in the
// slot's pinned staging like a normal completion.
int rerun_fused(scg_server *s, Slot &sl, Request *r) {
    scg_index *h = s->h;
    const int nq = r->nq, R = r->p.R;
    unsigned char *cur = s->arena.as<unsigned char>() + sl.off;
    auto take = [&](size_t bytes) {
        unsigned char *p = cur;
        cur += up256(bytes);
        return p;
    };
    float *dQ = (float *)take(4ull * nq * h->dim);
    int *d_ids = (int *)take(4ull * nq * R);
    float *d_d = (float *)take(4ull * nq * R);
    int *d_s = (int *)take(4ull * nq);
    ReqBufs rb = carve_req(cur, nq, h->mc, h->kc, h->mp, h->kp, r->p.rerank);
    int rc = run_search(h, &sl.ws, &rb, &r->p, dQ, nq, d_ids, d_d, d_s, sl.stream, true, nullptr, false);
    if (rc) return rc;
    cudaError_t e = cudaMemcpy(sl.hids, d_ids, 4ull * nq * R, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(sl.hd, d_d, 4ull * nq * R, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(sl.hs, d_s, 4ull * nq, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "result copy");
    return SCG_OK;
}

void finish(scg_server *s, Slot &sl, cudaError_t q) {
    Request *r = sl.req;
    int st = q == cudaSuccess ? *sl.ws.h_status : 0;
    int rc = SCG_OK;
    if (q != cudaSuccess) {
        rc = cuda_fail(q, "request stream");
    } else if (st == ST_POOL) {
        rc = rerun_fused(s, sl, r);
    } else if (st) {
        rc = status_result(st);
    }
    if (rc) {
        r->rc = rc;
        r->err = last_error_string();
    } else {
        const size_t n = (size_t)r->nq * r->p.R;
        memcpy(r->ids, sl.hids, 4 * n);
        memcpy(r->dists, sl.hd, 4 * n);
        if (r->sums) memcpy(r->sums, sl.hs, 4ull * r->nq);
    }
    r->t_done = Clock::now();
    r->state = 2;
    arena_free(s, sl.off, sl.len);
    sl.req = nullptr;
    s->inflight--;
    s->completed++;
    s->cv_done.notify_all();
}

void start(scg_server *s, Slot &sl, Request *r, size_t off) {
    scg_index *h = s->h;
    r->t_start = Clock::now();
    r->state = 1;
    sl.req = r;
    sl.off = off;
    sl.len = r->need;
    s->inflight++;
    if (s->inflight > s->max_inflight) s->max_inflight = s->inflight;
    const int nq = r->nq, R = r->p.R;
    unsigned char *cur = s->arena.as<unsigned char>() + off;
    auto take = [&](size_t bytes) {
        unsigned char *p = cur;
        cur += up256(bytes);
        return p;
    };
    float *dQ = (float *)take(4ull * nq * h->dim);
    int *d_ids = (int *)take(4ull * nq * R);
    float *d_d = (float *)take(4ull * nq * R);
    int *d_s = (int *)take(4ull * nq);
    ReqBufs rb = carve_req(cur, nq, h->mc, h->kc, h->mp, h->kp, r->p.rerank);
    memcpy(sl.hq, r->Q, 4ull * nq * h->dim);
    cudaError_t e = cudaMemcpyAsync(dQ, sl.hq, 4ull * nq * h->dim, cudaMemcpyHostToDevice, sl.stream);
    int rc = e == cudaSuccess ? run_search(h, &sl.ws, &rb, &r->p, dQ, nq, d_ids, d_d, d_s, sl.stream, false)
                              : cuda_fail(e, "query copy");
    if (rc == SCG_OK) {
        e = cudaMemcpyAsync(sl.hids, d_ids, 4ull * nq * R, cudaMemcpyDeviceToHost, sl.stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(sl.hd, d_d, 4ull * nq * R, cudaMemcpyDeviceToHost, sl.stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(sl.hs, d_s, 4ull * nq, cudaMemcpyDeviceToHost, sl.stream);
        if (e == cudaSuccess) e = cudaEventRecord(sl.done, sl.stream);
        if (e != cudaSuccess) rc = cuda_fail(e, "result copy");
    }
    if (rc != SCG_OK) {
        // nothing of this request may still run when its arena range is reused
        cudaStreamSynchronize(sl.stream);
        r->rc = rc;
        r->err = last_error_string();
        r->t_done = Clock::now();
        r->state = 2;
        arena_free(s, sl.off, sl.len);
        sl.req = nullptr;
        s->inflight--;
        s->completed++;
        s->cv_done.notify_all();
    }
}

void worker_main(scg_server *s) {
    cudaSetDevice(s->h->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        bool running = false;
        for (Slot &sl : s->slots) {
            if (!sl.req) continue;
            cudaError_t q = cudaEventQuery(sl.done);
            if (q == cudaErrorNotReady) {
                running = true;
                continue;
            }
            finish(s, sl, q);
        }
        // admit in arrival order while a slot and arena room are free
        while (!s->pending.empty()) {
            Slot *free_slot = nullptr;
            for (Slot &sl : s->slots)
                if (!sl.req) {
                    free_slot = &sl;
                    break;
                }
            if (!free_slot) break;
            Request *r = s->pending.front();
            size_t off = 0;
            if (!arena_alloc(s, r->need, &off)) break;
            s->pending.pop_front();
            start(s, *free_slot, r, off);
            if (free_slot->req) running = true;
        }
        if (!running && s->pending.empty()) {
            if (s->stop) break;
            s->cv_work.wait(lk);
            continue;
        }
        lk.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(20));
        lk.lock();
    }
}

}  // namespace

extern "C" {

int scg_server_create(scg_index *h, int nslots, int max_batch, int max_R, size_t arena_bytes, scg_server **out) {
    if (!out) return fail(SCG_ERR_ARG, "null output pointer");
    *out = nullptr;
    int rc;
    if ((rc = check_ready(h))) return rc;
    if (nslots < 1 || nslots > 64) return fail(SCG_ERR_ARG, "slots must be in [1, 64]");
    if (max_batch < 1 || max_R < 1 || max_R > 1024) return fail(SCG_ERR_ARG, "bad max_batch or max_R");
    if (arena_bytes < 4096) return fail(SCG_ERR_ARG, "arena too small");
    std::lock_guard<std::mutex> g(h->mu);
    if ((rc = set_device(h))) return rc;
    if ((rc = ensure_vterm(h, h->stream))) return rc;
    scg_server *s = new scg_server();
    s->h = h;
    s->max_batch = max_batch;
    s->max_R = max_R;
    s->arena_bytes = arena_bytes & ~(size_t)255;
    s->slots.resize((size_t)nslots);
    rc = s->arena.ensure(s->arena_bytes);
    cudaError_t e = cudaSuccess;
    for (Slot &sl : s->slots) {
        if (rc || e != cudaSuccess) break;
        e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMallocHost((void **)&sl.hq, 4ull * max_batch * h->dim);
        if (e == cudaSuccess) e = cudaMallocHost((void **)&sl.hids, 4ull * max_batch * max_R);
        if (e == cudaSuccess) e = cudaMallocHost((void **)&sl.hd, 4ull * max_batch * max_R);
        if (e == cudaSuccess) e = cudaMallocHost((void **)&sl.hs, 4ull * max_batch);
        if (e == cudaSuccess) rc = reserve_search(h, &sl.ws, index_mode(h), 0);
        if (rc == SCG_OK) rc = reserve_pool(h, &sl.ws, max_batch);
    }
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "scg_server_create");
    if (rc) {
        scg_server_destroy(s);
        return rc;
    }
    s->freelist[0] = s->arena_bytes;
    s->worker = std::thread(worker_main, s);
    *out = s;
    return SCG_OK;
}

int scg_server_submit(scg_server *s, const scg_search_params *p, const float *Q, int nq, int *ids, float *dists,
                      int *sums, uint64_t *ticket) {
    if (!s || !ticket) return fail(SCG_ERR_ARG, "null argument");
    int rc;
    if ((rc = check_params(s->h, p, nq))) return rc;
    if (nq < 1 || nq > s->max_batch) return fail(SCG_ERR_ARG, "nq must be in [1, max_batch]");
    if (p->R > s->max_R) return fail(SCG_ERR_ARG, "R exceeds the server's max_R");
    if (!Q || !ids || !dists) return fail(SCG_ERR_ARG, "null buffer");
    const size_t need = request_bytes(s->h, p, nq);
    if (need > s->arena_bytes)
        return fail(SCG_ERR_CAP, "the request needs " + std::to_string(need) + " bytes of device memory; the arena has " +
                                     std::to_string(s->arena_bytes));
    Request *r = new Request();
    r->p = *p;
    r->Q = Q;
    r->nq = nq;
    r->ids = ids;
    r->dists = dists;
    r->sums = sums;
    r->need = need;
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->stop) {
            delete r;
            return fail(SCG_ERR_STATE, "server is stopping");
        }
        r->ticket = s->next_ticket++;
        s->pending.push_back(r);
        s->reqs[r->ticket] = r;
        *ticket = r->ticket;
    }
    s->cv_work.notify_one();
    return SCG_OK;
}

int scg_server_wait_times(scg_server *s, uint64_t ticket, double timeout_s, double *times_ms) {
    if (!s) return fail(SCG_ERR_ARG, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fail(SCG_ERR_ARG, "unknown ticket");
    Request *r = it->second;
    auto ready = [&] { return r->state == 2; };
    if (timeout_s < 0) {
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
        return SCG_PENDING;
    }
    if (times_ms) {
        using ms = std::chrono::duration<double, std::milli>;
        times_ms[0] = ms(r->t_done - r->t_submit).count();
        times_ms[1] = ms(r->t_start - r->t_submit).count();
        times_ms[2] = ms(r->t_done - r->t_start).count();
    }
    const int rc = r->rc;
    if (rc) set_error(r->err);
    s->reqs.erase(it);
    delete r;
    return rc;
}

int scg_server_wait(scg_server *s, uint64_t ticket, double timeout_s, double *latency_ms) {
    double t[3];
    const int rc = scg_server_wait_times(s, ticket, timeout_s, t);
    if (rc != SCG_PENDING && latency_ms) *latency_ms = t[0];
    return rc;
}

int scg_server_stats(scg_server *s, long long *completed, int *max_inflight, int *queued) {
    if (!s) return fail(SCG_ERR_ARG, "null server");
    std::lock_guard<std::mutex> g(s->mu);
    if (completed) *completed = s->completed;
    if (max_inflight) *max_inflight = s->max_inflight;
    if (queued) *queued = (int)s->pending.size();
    return SCG_OK;
}

int scg_device_allocations(long long *count) {
    if (!count) return fail(SCG_ERR_ARG, "null output pointer");
    *count = g_device_allocs.load(std::memory_order_relaxed);
    return SCG_OK;
}

int scg_server_destroy(scg_server *s) {
    if (!s) return SCG_OK;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->h->device);
    for (Slot &sl : s->slots) {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        sl.ws.release();
        if (sl.hq) cudaFreeHost(sl.hq);
        if (sl.hids) cudaFreeHost(sl.hids);
        if (sl.hd) cudaFreeHost(sl.hd);
        if (sl.hs) cudaFreeHost(sl.hs);
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.stream) cudaStreamDestroy(sl.stream);
    }
    s->arena.release();
    for (auto &kv : s->reqs) delete kv.second;
    delete s;
    return SCG_OK;
}

}  // extern "C"
