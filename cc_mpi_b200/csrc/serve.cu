/*
 * CC request server: continuous batching of connected-components solves.
 *
 * No counterpart in the reference, which solves one graph per call; every
 * request gets exactly the labels compute_connected_components_pthreads
 * (include/cc.h:27-28) gives for its graph alone.
 *
 * One worker thread per server runs the loop:
 *   admit    pending requests, oldest first, while a slot is free and the
 *            request's CSR and labels fit in the server's HBM pool (first-fit
 *            over 256-byte blocks); the CSR copy to the pool is issued at
 *            once on the copy stream, so it overlaps the batches running.  A
 *            request that can never fit is refused at submission
 *   launch   whenever one of the `streams` batch slots is idle, up to
 *            max_batch admitted requests whose CSR has landed in HBM become
 *            one batch on that slot's stream: the batch descriptors and tile
 *            lists are uploaded, the batched solver enqueued and the
 *            component counts copied back - so a batch that forms while
 *            others run overlaps them on the device, and the copies of later
 *            requests keep flowing underneath
 *   retire   when a slot's completion event has fired, its requests are
 *            marked solved and their waiters woken
 * The waiting caller copies its labels out of the pool and frees the
 * request's blocks: CSR and labels stay in HBM from admission until then.
 * Every buffer a batch needs is reserved when the server is created, so the
 * loop allocates nothing.
 */
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch_core.h"

namespace {

constexpr size_t kAlign = 256;

size_t up(size_t x, size_t a)
{
    return (x + a - 1) / a * a;
}

struct Req {
    uint64_t ticket = 0;
    const uint64_t *h_rp = nullptr;
    const uint32_t *h_col = nullptr;
    uint32_t *h_lab = nullptr;
    uint32_t n = 0;
    uint64_t m = 0;
    size_t bytes = 0, off = 0;
    size_t rp_off = 0, col_off = 0, lab_off = 0; /* byte offsets in the pool */
    uint64_t round = 0;                          /* admission round of its copy */
    double t_submit = 0, t_admit = 0, t_start = 0, t_done = 0;
    uint32_t comps = 0, batch_graphs = 0;
    int status = CCGPU_OK;
    bool done = false;
    bool waited = false; /* a wait() owns the request */
};

struct Slot {
    BatchCore core;
    cudaStream_t st = nullptr;
    cudaEvent_t done_ev = nullptr;
    std::vector<Req *> reqs;
    bool busy = false;
    uint32_t *h_comps = nullptr; /* pinned, max_batch entries */
};

/* Events recorded on the copy stream after each admission round; a batch
 * waits for the round of its newest request.  A ring slot reused by a later
 * round only makes a batch wait longer, never too little (the copy stream
 * runs in order). */
constexpr int kRounds = 64;

/* First-fit allocator over the pool (host bookkeeping only). */
struct Pool {
    std::map<size_t, size_t> free_; /* offset -> size */
    size_t cap = 0, used = 0, peak = 0;
    void init(size_t bytes)
    {
        cap = bytes;
        free_.clear();
        free_[0] = bytes;
    }
    bool take(size_t bytes, size_t *off)
    {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= bytes) {
                *off = it->first;
                const size_t rest = it->second - bytes;
                const size_t at = it->first + bytes;
                free_.erase(it);
                if (rest)
                    free_[at] = rest;
                used += bytes;
                peak = std::max(peak, used);
                return true;
            }
        }
        return false;
    }
    void give(size_t off, size_t bytes)
    {
        used -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

} // namespace

struct ccgpu_server {
    int device = 0;
    ccgpu_ctx *ctx = nullptr;
    ccgpu_server_opts o;
    ccgpu_batch_tuning tune;
    char *pool_base = nullptr;
    Pool pool;
    std::vector<Slot> slots;
    cudaStream_t copy_st = nullptr;
    cudaEvent_t round_ev[kRounds] = {};
    uint64_t rounds = 0;      /* admission rounds issued              */
    uint64_t copied = 0;      /* rounds whose copies are known done   */
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req *> pending, admitted;
    std::unordered_map<uint64_t, Req *> live;
    uint64_t next_ticket = 1;
    uint32_t resident = 0;
    bool stop = false;
    std::thread worker;
    std::chrono::steady_clock::time_point t0;
    ccgpu_server_stats stats;
    std::string fatal;
    double now() const
    {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

size_t req_bytes(uint32_t n, uint64_t m)
{
    return up(8 * ((size_t)n + 1), kAlign) + up(4 * (size_t)m, kAlign) +
           up(4 * (size_t)(n ? n : 1), kAlign);
}

/* Copies a newly admitted request's CSR into its pool blocks on the copy
 * stream (worker thread, no lock held). */
int copy_in(ccgpu_server *S, Req *r)
{
    CC_CUDA(cudaMemcpyAsync(S->pool_base + r->rp_off, r->h_rp, 8 * ((size_t)r->n + 1),
                            cudaMemcpyHostToDevice, S->copy_st));
    if (r->m)
        CC_CUDA(cudaMemcpyAsync(S->pool_base + r->col_off, r->h_col, 4 * (size_t)r->m,
                                cudaMemcpyHostToDevice, S->copy_st));
    return CCGPU_OK;
}

/* Enqueues one batch on slot s (worker thread, no lock held). */
int launch(ccgpu_server *S, Slot &s)
{
    const uint32_t G = (uint32_t)s.reqs.size();
    std::vector<BGraph> gr(G);
    for (uint32_t g = 0; g < G; ++g) {
        Req *r = s.reqs[g];
        gr[g].rp = r->rp_off / 8;
        gr[g].col = r->col_off / 4;
        gr[g].lab = r->lab_off / 4;
        gr[g].n = r->n;
        gr[g].m = r->m;
        gr[g].pad = 0;
    }
    uint64_t newest = 0;
    for (Req *r : s.reqs)
        newest = std::max(newest, r->round);
    CC_CUDA(cudaStreamWaitEvent(s.st, S->round_ev[newest % kRounds], 0));
    CC_TRY(batch_core_set(&s.core, (const uint64_t *)S->pool_base,
                          (const uint32_t *)S->pool_base, (uint32_t *)S->pool_base, gr.data(), G,
                          s.st, 0));
    CC_TRY(batch_core_enqueue(&s.core, s.st, nullptr));
    CC_CUDA(cudaMemcpyAsync(s.h_comps, s.core.d_comps, (size_t)G * 4, cudaMemcpyDeviceToHost,
                            s.st));
    CC_CUDA(cudaEventRecord(s.done_ev, s.st));
    return CCGPU_OK;
}

void release_locked(ccgpu_server *S, Req *r)
{
    if (r->bytes) {
        S->pool.give(r->off, r->bytes);
        S->resident--;
        r->bytes = 0;
    }
}

void finish_locked(ccgpu_server *S, Req *r, int status)
{
    r->status = status;
    r->t_done = S->now();
    r->done = true;
    if (status != CCGPU_OK)
        release_locked(S, r);
    S->stats.completed++;
}

void worker_main(ccgpu_server *S)
{
    cudaSetDevice(S->device);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        bool progress = false;
        /* retire */
        for (Slot &s : S->slots) {
            if (!s.busy)
                continue;
            lk.unlock();
            cudaError_t e = cudaEventQuery(s.done_ev);
            if (e == cudaErrorNotReady) {
                lk.lock();
                continue;
            }
            int st = CCGPU_OK;
            if (e != cudaSuccess) {
                st = ccgpu_cuda_fail(e, "server batch", __FILE__, __LINE__);
            } else {
                for (size_t i = 0; i < s.reqs.size(); ++i)
                    s.reqs[i]->comps = s.h_comps[i];
            }
            lk.lock();
            if (st != CCGPU_OK && S->fatal.empty())
                S->fatal = ccgpu_last_error();
            for (Req *r : s.reqs)
                finish_locked(S, r, st);
            s.reqs.clear();
            s.busy = false;
            S->stats.in_flight--;
            progress = true;
            S->cv_done.notify_all();
        }
        /* admit, oldest first; the CSR copies start at once */
        std::vector<Req *> fresh;
        while (!S->stop && !S->pending.empty() && S->resident < S->o.max_graphs) {
            Req *r = S->pending.front();
            size_t off = 0;
            if (!S->pool.take(r->bytes, &off))
                break;
            S->pending.pop_front();
            r->off = off;
            r->rp_off = off;
            r->col_off = off + up(8 * ((size_t)r->n + 1), kAlign);
            r->lab_off = r->col_off + up(4 * (size_t)r->m, kAlign);
            r->t_admit = S->now();
            S->resident++;
            fresh.push_back(r);
            progress = true;
        }
        if (!fresh.empty()) {
            const uint64_t round = S->rounds++;
            lk.unlock();
            int rc = CCGPU_OK;
            for (Req *r : fresh) {
                r->round = round;
                if (rc == CCGPU_OK)
                    rc = copy_in(S, r);
            }
            if (rc == CCGPU_OK) {
                cudaError_t e = cudaEventRecord(S->round_ev[round % kRounds], S->copy_st);
                if (e != cudaSuccess)
                    rc = ccgpu_cuda_fail(e, "server copy round", __FILE__, __LINE__);
            }
            lk.lock();
            for (Req *r : fresh) {
                if (rc == CCGPU_OK) {
                    S->admitted.push_back(r);
                } else {
                    if (S->fatal.empty())
                        S->fatal = ccgpu_last_error();
                    finish_locked(S, r, rc);
                }
            }
            if (rc != CCGPU_OK)
                S->cv_done.notify_all();
        }
        S->stats.pool_peak = S->pool.peak;
        /* which admission rounds have landed in HBM (the copy stream runs in
         * order, so a later round's event also covers the earlier ones) */
        while (S->copied < S->rounds) {
            lk.unlock();
            cudaError_t e = cudaEventQuery(S->round_ev[S->copied % kRounds]);
            lk.lock();
            if (e != cudaSuccess)
                break;
            S->copied++;
            progress = true;
        }
        /* launch on idle slots: a batch takes the admitted requests whose
         * data is already resident, so copies keep flowing underneath */
        for (Slot &s : S->slots) {
            if (S->stop || s.busy || S->admitted.empty())
                continue;
            size_t ready = 0;
            while (ready < S->admitted.size() && ready < S->o.max_batch &&
                   S->admitted[ready]->round < S->copied)
                ++ready;
            if (ready == 0)
                continue;
            const uint32_t take = (uint32_t)ready;
            for (uint32_t i = 0; i < take; ++i) {
                Req *r = S->admitted.front();
                S->admitted.pop_front();
                r->batch_graphs = take;
                s.reqs.push_back(r);
            }
            s.busy = true;
            S->stats.in_flight++;
            S->stats.batches++;
            S->stats.max_in_flight = std::max(S->stats.max_in_flight, S->stats.in_flight);
            S->stats.max_batch_seen = std::max(S->stats.max_batch_seen, take);
            const double t = S->now();
            for (Req *r : s.reqs)
                r->t_start = t;
            lk.unlock();
            int rc = launch(S, s);
            lk.lock();
            if (rc != CCGPU_OK) {
                if (S->fatal.empty())
                    S->fatal = ccgpu_last_error();
                lk.unlock();
                cudaStreamSynchronize(s.st);
                lk.lock();
                for (Req *r : s.reqs)
                    finish_locked(S, r, rc);
                s.reqs.clear();
                s.busy = false;
                S->stats.in_flight--;
                S->cv_done.notify_all();
            }
            progress = true;
        }
        bool busy = S->copied < S->rounds;
        for (Slot &s : S->slots)
            busy |= s.busy;
        if (S->stop && !busy) {
            /* requests not yet in a batch are dropped */
            for (Req *r : S->pending)
                finish_locked(S, r, CCGPU_ERR_INVALID);
            for (Req *r : S->admitted)
                finish_locked(S, r, CCGPU_ERR_INVALID);
            S->pending.clear();
            S->admitted.clear();
            S->cv_done.notify_all();
            break;
        }
        if (!progress) {
            /* poll the GPU every 20 us while batches run, else sleep until
             * a submission or shutdown wakes the loop */
            if (busy)
                S->cv_work.wait_for(lk, std::chrono::microseconds(20));
            else
                S->cv_work.wait_for(lk, std::chrono::milliseconds(50));
        }
    }
}

} // namespace

/* ------------------------------------------------------------------ API */

extern "C" void ccgpu_server_opts_default(ccgpu_server_opts *o)
{
    if (!o)
        return;
    memset(o, 0, sizeof(*o));
    o->hbm_bytes = 0;
    o->max_graphs = 8192;
    o->max_batch = 4096;
    o->streams = 2;
}

extern "C" int ccgpu_server_create(const ccgpu_server_opts *opts,
                                   const ccgpu_batch_tuning *tuning, ccgpu_server **out)
{
    if (!out)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_server_create: NULL argument");
    *out = nullptr;
    ccgpu_server_opts o;
    ccgpu_server_opts_default(&o);
    if (opts)
        o = *opts;
    if (o.max_graphs == 0)
        o.max_graphs = 8192;
    if (o.max_batch == 0)
        o.max_batch = 4096;
    if (o.streams <= 0)
        o.streams = 2;
    if (o.streams > 8)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_server_create: streams %d above 8",
                               o.streams);
    ccgpu_batch_tuning t;
    if (tuning)
        t = *tuning;
    else
        ccgpu_batch_tuning_default(&t);
    CC_TRY(batch_check_tuning(&t));
    ccgpu_ctx *ctx = nullptr;
    CC_TRY(ccgpu_ctx_create(&ctx));
    ccgpu_server *S = new ccgpu_server();
    S->ctx = ctx;
    S->o = o;
    S->tune = t;
    memset(&S->stats, 0, sizeof(S->stats));
    S->t0 = std::chrono::steady_clock::now();
    int rc = CCGPU_OK;
    cudaError_t e = cudaGetDevice(&S->device);
    size_t free_b = 0, total_b = 0;
    if (e == cudaSuccess)
        e = cudaMemGetInfo(&free_b, &total_b);
    if (e != cudaSuccess)
        rc = ccgpu_cuda_fail(e, "ccgpu_server_create", __FILE__, __LINE__);
    if (rc == CCGPU_OK) {
        size_t bytes = o.hbm_bytes ? o.hbm_bytes : free_b / 2;
        bytes = up(bytes, kAlign);
        if (bytes > free_b)
            rc = ccgpu_set_error(CCGPU_ERR_OOM,
                                 "ccgpu_server_create: pool of %zu bytes above the %zu free",
                                 bytes, free_b);
        else if ((e = cudaMalloc((void **)&S->pool_base, bytes)) != cudaSuccess)
            rc = ccgpu_cuda_fail(e, "server pool", __FILE__, __LINE__);
        else
            S->pool.init(bytes);
        S->o.hbm_bytes = bytes;
    }
    /* a batch never holds more than the pool: every vertex costs at least
     * 12 bytes of it (row pointer and label), every entry 4 */
    int min_tile = t.cls[0].tile;
    for (int k = 1; k < CCGPU_BATCH_CLASSES; ++k)
        min_tile = std::min(min_tile, t.cls[k].tile);
    const size_t max_vertices = S->o.hbm_bytes / 12, max_entries = S->o.hbm_bytes / 4;
    const size_t tiles = max_vertices / (size_t)min_tile + o.max_batch + 1;
    const size_t heavy = max_entries / (size_t)t.heavy_degree + o.max_batch + 1;
    if (rc == CCGPU_OK && (e = cudaStreamCreateWithFlags(&S->copy_st, cudaStreamNonBlocking)) !=
                              cudaSuccess)
        rc = ccgpu_cuda_fail(e, "server copy stream", __FILE__, __LINE__);
    for (int i = 0; rc == CCGPU_OK && i < kRounds; ++i)
        if ((e = cudaEventCreateWithFlags(&S->round_ev[i], cudaEventDisableTiming)) !=
            cudaSuccess)
            rc = ccgpu_cuda_fail(e, "server copy events", __FILE__, __LINE__);
    S->slots.resize(o.streams);
    for (int i = 0; rc == CCGPU_OK && i < o.streams; ++i) {
        Slot &s = S->slots[i];
        rc = batch_core_init(&s.core, ctx, &t);
        if (rc == CCGPU_OK)
            rc = batch_core_reserve(&s.core, o.max_batch, tiles, heavy);
        if (rc == CCGPU_OK &&
            (e = cudaMallocHost((void **)&s.h_comps, (size_t)o.max_batch * 4)) != cudaSuccess)
            rc = ccgpu_cuda_fail(e, "server pinned counts", __FILE__, __LINE__);
        if (rc == CCGPU_OK && (e = cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking)) !=
                                  cudaSuccess)
            rc = ccgpu_cuda_fail(e, "server stream", __FILE__, __LINE__);
        if (rc == CCGPU_OK &&
            (e = cudaEventCreateWithFlags(&s.done_ev, cudaEventDisableTiming)) != cudaSuccess)
            rc = ccgpu_cuda_fail(e, "server event", __FILE__, __LINE__);
    }
    if (rc != CCGPU_OK) {
        ccgpu_server_destroy(S);
        return rc;
    }
    S->worker = std::thread(worker_main, S);
    *out = S;
    return CCGPU_OK;
}

extern "C" int ccgpu_server_submit(ccgpu_server *S, const uint64_t *h_row_ptr,
                                   const uint32_t *h_col_idx, uint32_t n, uint64_t m,
                                   uint32_t *h_labels, uint64_t *ticket)
{
    if (!S || !ticket || (n && (!h_row_ptr || !h_labels)) || (m && !h_col_idx))
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_server_submit: NULL argument");
    if (n == 0xffffffffu)
        return ccgpu_set_error(CCGPU_ERR_LIMIT, "ccgpu_server_submit: n must be below 2^32-1");
    if (n && h_row_ptr[n] != m)
        return ccgpu_set_error(CCGPU_ERR_INVALID,
                               "ccgpu_server_submit: row_ptr[n] = %llu is not m = %llu",
                               (unsigned long long)h_row_ptr[n], (unsigned long long)m);
    const size_t bytes = n ? req_bytes(n, m) : 0;
    if (bytes > S->pool.cap)
        return ccgpu_set_error(CCGPU_ERR_LIMIT,
                               "ccgpu_server_submit: the graph needs %zu bytes of HBM, above the "
                               "server's pool of %zu",
                               bytes, S->pool.cap);
    Req *r = new Req();
    r->h_rp = h_row_ptr;
    r->h_col = h_col_idx;
    r->h_lab = h_labels;
    r->n = n;
    r->m = m;
    r->bytes = bytes;
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) {
        delete r;
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_server_submit: server is stopping");
    }
    r->ticket = S->next_ticket++;
    r->t_submit = S->now();
    S->live[r->ticket] = r;
    S->stats.submitted++;
    if (n == 0) { /* nothing to solve: done at once, no components */
        r->t_admit = r->t_start = r->t_submit;
        finish_locked(S, r, CCGPU_OK);
        S->cv_done.notify_all();
    } else {
        S->pending.push_back(r);
        S->cv_work.notify_one();
    }
    *ticket = r->ticket;
    return CCGPU_OK;
}

extern "C" int ccgpu_server_wait(ccgpu_server *S, uint64_t ticket, double timeout_s,
                                 ccgpu_request_info *info)
{
    if (!S)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_server_wait: NULL server");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->live.find(ticket);
    if (it == S->live.end())
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_server_wait: unknown ticket %llu",
                               (unsigned long long)ticket);
    Req *r = it->second;
    if (r->waited)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_server_wait: ticket %llu is already "
                               "being waited on", (unsigned long long)ticket);
    r->waited = true;
    const auto until = std::chrono::steady_clock::now() +
                       std::chrono::duration_cast<std::chrono::steady_clock::duration>(
                           std::chrono::duration<double>(timeout_s < 0 ? 1e9 : timeout_s));
    while (!r->done)
        if (S->cv_done.wait_until(lk, until) == std::cv_status::timeout && !r->done) {
            r->waited = false;
            return ccgpu_set_error(CCGPU_ERR_TIMEOUT, "ccgpu_server_wait: ticket %llu not done",
                                   (unsigned long long)ticket);
        }
    int st = r->status;
    if (st == CCGPU_OK && r->n) {
        /* labels leave the pool on this thread's own stream, then the
         * request's blocks go back to the pool */
        const char *src = S->pool_base + r->lab_off;
        const size_t bytes = 4 * (size_t)r->n;
        lk.unlock();
        int dev = 0;
        cudaGetDevice(&dev);
        cudaError_t e = cudaSetDevice(S->device);
        static thread_local cudaStream_t rb[64] = {};
        cudaStream_t &q = rb[S->device & 63];
        if (e == cudaSuccess && !q)
            e = cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(r->h_lab, src, bytes, cudaMemcpyDeviceToHost, q);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(q);
        cudaSetDevice(dev);
        if (e != cudaSuccess)
            st = ccgpu_cuda_fail(e, "server label read-back", __FILE__, __LINE__);
        lk.lock();
        r->t_done = S->now(); /* labels are in the caller's buffer */
    }
    release_locked(S, r);
    S->cv_work.notify_one();
    if (info) {
        info->t_submit = r->t_submit;
        info->t_admit = r->t_admit;
        info->t_start = r->t_start;
        info->t_done = r->t_done;
        info->components = r->comps;
        info->batch_graphs = r->batch_graphs;
        info->status = st;
    }
    S->live.erase(ticket);
    delete r;
    if (st != CCGPU_OK)
        return ccgpu_set_error(st, "ccgpu_server_wait: request failed: %s",
                               S->fatal.empty() ? "server stopped before solving it"
                                                : S->fatal.c_str());
    return CCGPU_OK;
}

extern "C" int ccgpu_server_stats_get(ccgpu_server *S, ccgpu_server_stats *out)
{
    if (!S || !out)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_server_stats_get: NULL argument");
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->stats;
    out->pool_bytes = S->pool.cap;
    out->pool_used = S->pool.used;
    out->pending = (uint32_t)S->pending.size();
    out->resident = S->resident;
    return CCGPU_OK;
}

extern "C" double ccgpu_server_now(ccgpu_server *S)
{
    return S ? S->now() : 0.0;
}

extern "C" void ccgpu_server_destroy(ccgpu_server *S)
{
    if (!S)
        return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        S->cv_work.notify_all();
    }
    if (S->worker.joinable())
        S->worker.join();
    for (Slot &s : S->slots) {
        if (s.st)
            cudaStreamSynchronize(s.st);
        batch_core_free(&s.core);
        if (s.st)
            cudaStreamDestroy(s.st);
        if (s.done_ev)
            cudaEventDestroy(s.done_ev);
        if (s.h_comps)
            cudaFreeHost(s.h_comps);
    }
    if (S->copy_st) {
        cudaStreamSynchronize(S->copy_st);
        cudaStreamDestroy(S->copy_st);
    }
    for (int i = 0; i < kRounds; ++i)
        if (S->round_ev[i])
            cudaEventDestroy(S->round_ev[i]);
    for (auto &kv : S->live)
        delete kv.second;
    cudaFree(S->pool_base);
    ccgpu_ctx_destroy(S->ctx);
    delete S;
}
