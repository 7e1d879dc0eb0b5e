// Request serving over the multiply path: one scheduler thread, one CUDA
// stream per ring, continuous batching at operation granularity, admission by
// a device-memory budget. Interface and semantics: include/kbfv_serve.h.
#include "../../include/kbfv_serve.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

// First-fit allocator over [0, cap) with address-ordered free ranges (coalescing).
class RangeAllocator {
   public:
    explicit RangeAllocator(size_t cap = 0) { reset(cap); }
    void reset(size_t cap) {
        free_.clear();
        cap_ = cap;
        used_ = peak_ = 0;
        if (cap) free_[0] = cap;
    }
    bool alloc(size_t size, size_t& off) {
        size = (size + 255) & ~(size_t)255;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < size) continue;
            off = it->first;
            const size_t rest = it->second - size;
            free_.erase(it);
            if (rest) free_[off + size] = rest;
            used_ += size;
            peak_ = std::max(peak_, used_);
            return true;
        }
        return false;
    }
    void release(size_t off, size_t size) {
        size = (size + 255) & ~(size_t)255;
        used_ -= size;
        auto next = free_.lower_bound(off);
        if (next != free_.end() && off + size == next->first) {
            size += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += size;
                return;
            }
        }
        free_[off] = size;
    }
    size_t used() const { return used_; }
    size_t peak() const { return peak_; }

   private:
    std::map<size_t, size_t> free_;
    size_t cap_ = 0, used_ = 0, peak_ = 0;
};

struct Request {
    uint64_t id = 0;
    uint32_t ring = 0, nops = 0, flags = 0;
    uint8_t ops[8] = {0};
    uint64_t enc_id = 0;
    std::vector<uint64_t> input;  // (nops+1) x N, until admitted
    size_t dev_off = 0, dev_size = 0, pin_off = 0, pin_size = 0;
    uint64_t *d_pt = nullptr, *d_ct = nullptr, *d_res = nullptr;
    uint64_t *h_in = nullptr, *h_out = nullptr;
    uint32_t step = 0;  // operations issued
    bool encrypted = false;
    Clock::time_point t_submit, t_done;
    bool done = false;
    int status = KBFV_OK;
    std::string error;
    std::vector<uint64_t> result, ct;
};

struct Iteration {
    cudaEvent_t ev = nullptr;
    std::vector<Request*> finishing;
};

struct Ring {
    kbfv_context* ctx = nullptr;
    uint8_t seed[32];
    const uint64_t *pk = nullptr, *rlk = nullptr, *sk = nullptr;
    uint64_t n = 0, t = 0;
    uint32_t nq = 0, pt_prime = 0;  // pt_prime: index of the plain modulus in the prime table
    cudaStream_t st = nullptr;
    std::deque<Request*> pending;
    std::vector<Request*> active;
    std::deque<Iteration> inflight;
    std::vector<cudaEvent_t> spare_events;
};

}  // namespace

struct kbfv_server {
    kbfv_server_config cfg{};
    int device = 0;
    void* slab = nullptr;
    uint8_t* pinned = nullptr;
    RangeAllocator dev_alloc, pin_alloc;
    std::vector<std::unique_ptr<Ring>> rings;

    std::mutex mu;  // guards incoming, reqs, stats, done flags
    std::condition_variable cv_done, cv_work;
    std::deque<Request*> incoming;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
    uint64_t next_id = 1;
    kbfv_server_stats stats{};
    std::atomic<bool> stop{false};
    bool started = false;
    std::thread worker;
    std::string fatal;

    void run();
    bool admit(Ring& r, Request* q);
    void issue(Ring& r);
    void retire(Ring& r, Iteration& it, cudaError_t err);
    void fail(Request* q, int status, const std::string& msg);
    void release(Request* q);
};

#define SRV_CALL(expr)                                             \
    do {                                                           \
        int rc_ = (expr);                                          \
        if (rc_ != KBFV_OK) throw ServeError(rc_, kbfv_last_error()); \
    } while (0)

namespace {
struct ServeError : std::runtime_error {
    int code;
    ServeError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
thread_local std::string g_serve_error;
}  // namespace

void kbfv_server::fail(Request* q, int status, const std::string& msg) {
    q->status = status;
    q->error = msg;
}

void kbfv_server::release(Request* q) {
    if (q->dev_size) dev_alloc.release(q->dev_off, q->dev_size);
    if (q->pin_size) pin_alloc.release(q->pin_off, q->pin_size);
    q->dev_size = q->pin_size = 0;
}

// Reserve device and pinned space, stage the inputs and enqueue encode + encrypt.
bool kbfv_server::admit(Ring& r, Request* q) {
    const size_t n = r.n, lq = (size_t)r.nq * n, k1 = q->nops + 1;
    const size_t dev_words = k1 * n + k1 * 2 * lq + n;
    const size_t pin_words = k1 * n + n + ((q->flags & KBFV_REQ_RETURN_CT) ? 2 * lq : 0);
    size_t doff, poff;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!dev_alloc.alloc(dev_words * 8, doff)) return false;
        if (!pin_alloc.alloc(pin_words * 8, poff)) {
            dev_alloc.release(doff, dev_words * 8);
            return false;
        }
        stats.bytes_in_use = dev_alloc.used();
        stats.bytes_peak = dev_alloc.peak();
    }
    q->dev_off = doff;
    q->dev_size = dev_words * 8;
    q->pin_off = poff;
    q->pin_size = pin_words * 8;
    uint64_t* d = (uint64_t*)((uint8_t*)slab + doff);
    q->d_pt = d;
    q->d_ct = d + k1 * n;
    q->d_res = q->d_ct + k1 * 2 * lq;
    q->h_in = (uint64_t*)(pinned + poff);
    q->h_out = q->h_in + k1 * n;
    std::memcpy(q->h_in, q->input.data(), k1 * n * 8);
    std::vector<uint64_t>().swap(q->input);
    if (cudaMemcpyAsync(q->d_pt, q->h_in, k1 * n * 8, cudaMemcpyHostToDevice, r.st) != cudaSuccess)
        throw ServeError(KBFV_ERR_CUDA, "input copy failed");
    return true;  // encoding and encryption are batched over the iteration's admissions
}

// One iteration of a ring: admit, advance every admitted request by one
// operation (multiplies batched), decrypt finished chains, record an event.
void kbfv_server::issue(Ring& r) {
    Iteration it;
    while (!r.pending.empty() && (cfg.max_active == 0 || r.active.size() < cfg.max_active)) {
        Request* q = r.pending.front();
        bool ok = false;
        try {
            ok = admit(r, q);
        } catch (const ServeError& e) {  // staging failed: this request alone fails
            r.pending.pop_front();
            std::lock_guard<std::mutex> lk(mu);
            fail(q, e.code, e.what());
            release(q);
            q->done = true;
            stats.failed++;
            cv_done.notify_all();
            continue;
        }
        if (!ok) break;  // budget full: wait for running requests to finish
        r.pending.pop_front();
        r.active.push_back(q);
    }
    if (r.active.empty()) return;
    const size_t lq = (size_t)r.nq * r.n;
    // encode + encrypt everything admitted in this iteration in batched calls
    {
        std::vector<uint64_t*> pts, cts;
        std::vector<uint64_t> ids;
        for (Request* q : r.active) {
            if (q->step != 0 || q->encrypted) continue;
            for (uint32_t j = 0; j <= q->nops; j++) {
                pts.push_back(q->d_pt + (size_t)j * r.n);
                cts.push_back(q->d_ct + (size_t)j * 2 * lq);
                ids.push_back(q->enc_id + j);
            }
            q->encrypted = true;
        }
        if (!pts.empty()) {
            SRV_CALL(kbfv_ntt_inv_batch(r.ctx, pts.data(), (uint32_t)pts.size(), 1, r.pt_prime, r.st));
            std::vector<const uint64_t*> cpts(pts.begin(), pts.end());
            SRV_CALL(kbfv_encrypt_batch(r.ctx, r.seed, ids.data(), r.pk, cpts.data(), cts.data(), (uint32_t)cts.size(),
                                        r.st));
        }
    }
    std::vector<const uint64_t*> A, B;
    std::vector<uint64_t*> O;
    std::vector<Request*> adds;
    for (Request* q : r.active) {
        const uint64_t* nxt = q->d_ct + (size_t)(q->step + 1) * 2 * lq;
        if (q->ops[q->step] == KBFV_OP_MUL) {
            A.push_back(q->d_ct);
            B.push_back(nxt);
            O.push_back(q->d_ct);
        } else {
            adds.push_back(q);
        }
    }
    uint64_t mul_launches = 0;
    for (size_t off = 0; off < A.size(); off += cfg.max_batch) {
        const uint32_t cnt = (uint32_t)std::min<size_t>(cfg.max_batch, A.size() - off);
        SRV_CALL(kbfv_mul_relin_batch(r.ctx, r.rlk, A.data() + off, B.data() + off, O.data() + off, cnt, r.st));
        mul_launches++;
    }
    if (!adds.empty()) {
        std::vector<const uint64_t*> X, Y;
        std::vector<uint64_t*> Z;
        for (Request* q : adds) {
            X.push_back(q->d_ct);
            Y.push_back(q->d_ct + (size_t)(q->step + 1) * 2 * lq);
            Z.push_back(q->d_ct);
        }
        SRV_CALL(kbfv_add_batch(r.ctx, X.data(), Y.data(), Z.data(), (uint32_t)adds.size(), r.st));
    }
    std::vector<Request*> still;
    std::vector<const uint64_t*> dct;
    std::vector<uint64_t*> dres;
    for (Request* q : r.active) {
        q->step++;
        if (q->step < q->nops) {
            still.push_back(q);
            continue;
        }
        dct.push_back(q->d_ct);
        dres.push_back(q->d_res);
        it.finishing.push_back(q);
    }
    if (!dct.empty()) {  // decrypt + decode the finished chains together, then read them back
        SRV_CALL(kbfv_decrypt_batch(r.ctx, r.sk, dct.data(), dres.data(), (uint32_t)dct.size(), r.st));
        SRV_CALL(kbfv_ntt_fwd_batch(r.ctx, dres.data(), (uint32_t)dres.size(), 1, r.pt_prime, r.st));
        for (Request* q : it.finishing) {
            if (cudaMemcpyAsync(q->h_out, q->d_res, r.n * 8, cudaMemcpyDeviceToHost, r.st) != cudaSuccess)
                throw ServeError(KBFV_ERR_CUDA, "result copy failed");
            if ((q->flags & KBFV_REQ_RETURN_CT) &&
                cudaMemcpyAsync(q->h_out + r.n, q->d_ct, 2 * lq * 8, cudaMemcpyDeviceToHost, r.st) != cudaSuccess)
                throw ServeError(KBFV_ERR_CUDA, "ciphertext copy failed");
        }
    }
    if (r.spare_events.empty()) {
        cudaEvent_t e;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            throw ServeError(KBFV_ERR_CUDA, "event creation failed");
        r.spare_events.push_back(e);
    }
    it.ev = r.spare_events.back();
    r.spare_events.pop_back();
    if (cudaEventRecord(it.ev, r.st) != cudaSuccess) throw ServeError(KBFV_ERR_CUDA, "event record failed");
    {
        std::lock_guard<std::mutex> lk(mu);
        stats.iterations++;
        stats.mul_launches += mul_launches;
        stats.mul_ops += A.size();
        stats.add_ops += adds.size();
    }
    r.active.swap(still);
    r.inflight.push_back(std::move(it));
}

void kbfv_server::retire(Ring& r, Iteration& it, cudaError_t err) {
    const auto now = Clock::now();
    const size_t lq = (size_t)r.nq * r.n;
    std::lock_guard<std::mutex> lk(mu);
    for (Request* q : it.finishing) {
        if (err != cudaSuccess) {
            fail(q, KBFV_ERR_CUDA, cudaGetErrorString(err));
        } else {
            q->result.assign(q->h_out, q->h_out + r.n);
            if (q->flags & KBFV_REQ_RETURN_CT) q->ct.assign(q->h_out + r.n, q->h_out + r.n + 2 * lq);
        }
        q->t_done = now;
        release(q);
        q->done = true;
        if (q->status == KBFV_OK) stats.completed++;
        else stats.failed++;
    }
    stats.bytes_in_use = dev_alloc.used();
    r.spare_events.push_back(it.ev);
    cv_done.notify_all();
}

void kbfv_server::run() {
    cudaSetDevice(device);
    const unsigned depth = cfg.inflight_iterations ? cfg.inflight_iterations : 2;
    for (;;) {
        bool idle = true;
        {
            std::unique_lock<std::mutex> lk(mu);
            bool busy = !incoming.empty();
            for (auto& rp : rings) busy |= !rp->pending.empty() || !rp->active.empty() || !rp->inflight.empty();
            if (!busy) {
                if (stop) break;
                cv_work.wait_for(lk, std::chrono::milliseconds(2));
            }
            while (!incoming.empty()) {
                Request* q = incoming.front();
                incoming.pop_front();
                rings[q->ring]->pending.push_back(q);
            }
            uint32_t pend = 0, act = 0;
            for (auto& rp : rings) {
                pend += (uint32_t)rp->pending.size();
                act += (uint32_t)rp->active.size();
            }
            stats.pending = pend;
            stats.active = act;
        }
        for (auto& rp : rings) {
            Ring& r = *rp;
            while (!r.inflight.empty()) {
                cudaError_t e = cudaEventQuery(r.inflight.front().ev);
                if (e == cudaErrorNotReady) break;
                retire(r, r.inflight.front(), e);
                r.inflight.pop_front();
                idle = false;
            }
            if (r.inflight.size() >= depth) continue;
            if (r.active.empty() && r.pending.empty()) continue;
            try {
                const size_t queued = r.inflight.size();
                issue(r);
                idle = r.inflight.size() == queued && idle;
            } catch (const std::exception& ex) {
                // the iteration could not be issued: fail the requests it touched
                const int code = dynamic_cast<const ServeError*>(&ex) ? static_cast<const ServeError&>(ex).code
                                                                        : KBFV_ERR_CUDA;
                cudaStreamSynchronize(r.st);
                std::lock_guard<std::mutex> lk(mu);
                for (Request* q : r.active) {
                    fail(q, code, ex.what());
                    release(q);
                    q->done = true;
                    stats.failed++;
                }
                r.active.clear();
                cv_done.notify_all();
            }
        }
        if (idle) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

extern "C" {

const char* kbfv_server_last_error(void) { return g_serve_error.c_str(); }

int kbfv_server_create(const kbfv_server_config* cfg, kbfv_server** out) {
    if (!cfg || !out) return KBFV_ERR_INVALID;
    if (cfg->max_batch < 1 || cfg->max_batch > 128 || cfg->inflight_iterations > 8 || cfg->hbm_budget_bytes < (1u << 20))
        return KBFV_ERR_INVALID;
    auto* s = new kbfv_server();
    s->cfg = *cfg;
    if (!s->cfg.pinned_bytes) s->cfg.pinned_bytes = (uint64_t)256 << 20;
    if (cudaGetDevice(&s->device) != cudaSuccess || cudaMalloc(&s->slab, s->cfg.hbm_budget_bytes) != cudaSuccess) {
        delete s;
        return KBFV_ERR_NOMEM;
    }
    if (cudaHostAlloc((void**)&s->pinned, s->cfg.pinned_bytes, cudaHostAllocDefault) != cudaSuccess) {
        cudaFree(s->slab);
        delete s;
        return KBFV_ERR_NOMEM;
    }
    s->dev_alloc.reset(s->cfg.hbm_budget_bytes);
    s->pin_alloc.reset(s->cfg.pinned_bytes);
    *out = s;
    return KBFV_OK;
}

int kbfv_server_add_ring(kbfv_server* s, kbfv_context* ctx, const uint8_t seed[32], const uint64_t* d_pk,
                         const uint64_t* d_rlk, const uint64_t* d_sk, uint32_t* ring_id) {
    if (!s || !ctx || !seed || !d_pk || !d_rlk || !d_sk) return KBFV_ERR_INVALID;
    if (s->started) return KBFV_ERR_INVALID;
    auto r = std::make_unique<Ring>();
    r->ctx = ctx;
    std::memcpy(r->seed, seed, 32);
    r->pk = d_pk;
    r->rlk = d_rlk;
    r->sk = d_sk;
    uint32_t nq, np_, nr, nt, dnum, alpha;
    int rc = kbfv_context_info(ctx, &r->n, &nq, &np_, &nr, &nt, &dnum, &alpha);
    if (rc != KBFV_OK) return rc;
    r->nq = nq;
    r->t = kbfv_context_plain_modulus(ctx);
    uint32_t nprimes = 0;
    rc = kbfv_context_primes(ctx, nullptr, &nprimes);
    if (rc != KBFV_OK) return rc;
    r->pt_prime = nprimes - 1;
    // scratch for a full multiply batch and for encrypting 128 plaintexts at once
    rc = kbfv_reserve(ctx, std::max<uint32_t>(s->cfg.max_batch, 40));
    if (rc != KBFV_OK) return rc;
    if (cudaStreamCreateWithFlags(&r->st, cudaStreamNonBlocking) != cudaSuccess) return KBFV_ERR_CUDA;
    if (ring_id) *ring_id = (uint32_t)s->rings.size();
    s->rings.push_back(std::move(r));
    return KBFV_OK;
}

int kbfv_server_start(kbfv_server* s) {
    if (!s || s->started || s->rings.empty()) return KBFV_ERR_INVALID;
    s->started = true;
    s->worker = std::thread([s] { s->run(); });
    return KBFV_OK;
}

int kbfv_server_submit(kbfv_server* s, uint32_t ring, const uint64_t* h_slots, uint32_t n_ops, const uint8_t* ops,
                       uint64_t enc_id, uint32_t flags, uint64_t* request_id) {
    if (!s || !s->started || s->stop || ring >= s->rings.size() || !h_slots || !ops || n_ops < 1 || n_ops > 8)
        return KBFV_ERR_INVALID;
    const Ring& r = *s->rings[ring];
    auto q = std::make_unique<Request>();
    q->ring = ring;
    q->nops = n_ops;
    q->flags = flags;
    q->enc_id = enc_id;
    for (uint32_t i = 0; i < n_ops; i++) {
        if (ops[i] != KBFV_OP_MUL && ops[i] != KBFV_OP_ADD) return KBFV_ERR_INVALID;
        q->ops[i] = ops[i];
    }
    const size_t words = (size_t)(n_ops + 1) * r.n;
    for (size_t i = 0; i < words; i++)
        if (h_slots[i] >= r.t) return KBFV_ERR_INVALID;
    // a request larger than the whole budget could never be admitted
    const size_t lq = (size_t)r.nq * r.n;
    if (((n_ops + 1) * (r.n + 2 * lq) + r.n) * 8 > s->cfg.hbm_budget_bytes ||
        ((n_ops + 1) * r.n + r.n + 2 * lq) * 8 > s->cfg.pinned_bytes)
        return KBFV_ERR_NOMEM;
    q->input.assign(h_slots, h_slots + words);
    q->t_submit = Clock::now();
    Request* raw = q.get();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        q->id = s->next_id++;
        if (request_id) *request_id = q->id;
        s->reqs.emplace(q->id, std::move(q));
        s->incoming.push_back(raw);
        s->stats.submitted++;
    }
    s->cv_work.notify_one();
    return KBFV_OK;
}

int kbfv_server_wait(kbfv_server* s, uint64_t request_id, int64_t timeout_ms, uint64_t* h_slots_out,
                     uint64_t* h_ct_out, double* latency_ms) {
    if (!s) return KBFV_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return KBFV_ERR_INVALID;
    Request* q = it->second.get();
    auto ready = [&] { return q->done; };
    if (timeout_ms < 0) s->cv_done.wait(lk, ready);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return KBFV_ERR_UNSUPPORTED;
    const int status = q->status;
    if (status == KBFV_OK) {
        if (h_slots_out) std::memcpy(h_slots_out, q->result.data(), q->result.size() * 8);
        if (h_ct_out && !q->ct.empty()) std::memcpy(h_ct_out, q->ct.data(), q->ct.size() * 8);
        if (latency_ms)
            *latency_ms = std::chrono::duration<double, std::milli>(q->t_done - q->t_submit).count();
    } else {
        g_serve_error = q->error;
    }
    s->reqs.erase(it);
    return status;
}

int kbfv_server_get_stats(kbfv_server* s, kbfv_server_stats* out) {
    if (!s || !out) return KBFV_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    return KBFV_OK;
}

int kbfv_server_destroy(kbfv_server* s) {
    if (!s) return KBFV_OK;
    if (s->started) {
        s->stop = true;
        s->cv_work.notify_all();
        s->worker.join();
    }
    for (auto& r : s->rings) {
        if (r->st) {
            cudaStreamSynchronize(r->st);
            cudaStreamDestroy(r->st);
        }
        for (cudaEvent_t e : r->spare_events) cudaEventDestroy(e);
    }
    if (s->slab) cudaFree(s->slab);
    if (s->pinned) cudaFreeHost(s->pinned);
    delete s;
    return KBFV_OK;
}

}  // extern "C"
