// Captured multiplies (kbfv_plan_*): a caller that multiplies the same device
// buffers again and again (a request loop with fixed staging buffers) replays
// the whole multiply as one CUDA graph launch instead of issuing its ~14
// kernel launches one by one; a batch of pairs at mixed levels
// (kbfv_mul_relin_levels) likewise becomes one graph launch. No counterpart in
// the reference.
#include <vector>

#include "pipeline.cuh"

struct kbfv_plan {
    kbfv_context* ctx = nullptr;
    const uint64_t* rlk = nullptr;
    const uint64_t* a = nullptr;
    const uint64_t* b = nullptr;
    uint64_t* out = nullptr;
    uint32_t count = 0;
    // mixed levels: pair i at live_q[i] live primes, its own pointers
    bool levels = false;
    std::vector<uint32_t> live_q;
    std::vector<const uint64_t*> va, vb;
    std::vector<uint64_t*> vo;
    cudaStream_t cs = nullptr;  // the stream the graph is captured on
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // what the captured kernels address and how they were shaped
    void* scratch = nullptr;
    LaunchShape shape{};
    int branches = 0, min_branch_pairs = 0;
    uint64_t launches = 0, captures = 0;
};

namespace {

void drop_graph(kbfv_plan& p) {
    if (p.exec) cudaGraphExecDestroy(p.exec);
    if (p.graph) cudaGraphDestroy(p.graph);
    p.exec = nullptr;
    p.graph = nullptr;
}

bool graph_current(const kbfv_plan& p) {
    const Context& c = p.ctx->c;
    return p.exec && c.scratch == p.scratch && c.branches == p.branches && c.min_branch_pairs == p.min_branch_pairs &&
           std::memcmp(&c.dc.shape, &p.shape, sizeof(LaunchShape)) == 0;
}

// Runs the multiply on `st` (eagerly: first-use set-up such as module loading,
// kernel attributes and scratch growth happens here, outside any capture),
// then records the same launch sequence on the plan's own stream into a graph.
// Capturing executes nothing.
int run_once(kbfv_plan& p, cudaStream_t st) {
    if (p.levels)
        return kbfv_mul_relin_levels(p.ctx, p.rlk, p.live_q.data(), p.va.data(), p.vb.data(), p.vo.data(), p.count,
                                     (kbfv_stream)st);
    return kbfv_mul_relin(p.ctx, p.rlk, p.a, p.b, p.out, p.count, (kbfv_stream)st);
}

void run_and_capture(kbfv_plan& p, cudaStream_t st) {
    int rc = run_once(p, st);
    if (rc != KBFV_OK) throw KbfvError(rc, g_last_error);
    drop_graph(p);
    if (!p.cs) KB_CHECK_CUDA(cudaStreamCreateWithFlags(&p.cs, cudaStreamNonBlocking));
    KB_CHECK_CUDA(cudaStreamBeginCapture(p.cs, cudaStreamCaptureModeThreadLocal));
    rc = run_once(p, p.cs);
    const std::string err = rc == KBFV_OK ? std::string() : g_last_error;
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(p.cs, &g);  // ends the capture on every path
    if (rc != KBFV_OK) {
        if (g) cudaGraphDestroy(g);
        throw KbfvError(rc, "capturing the multiply: " + err);
    }
    if (e != cudaSuccess) throw KbfvError(KBFV_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
    p.graph = g;
    KB_CHECK_CUDA(cudaGraphInstantiate(&p.exec, p.graph, 0));
    const Context& c = p.ctx->c;
    p.scratch = c.scratch;
    p.shape = c.dc.shape;
    p.branches = c.branches;
    p.min_branch_pairs = c.min_branch_pairs;
    p.captures++;
}

}  // namespace

extern "C" {

int kbfv_plan_mul_relin(kbfv_context* ctx, const uint64_t* d_rlk, const uint64_t* d_ct_a, const uint64_t* d_ct_b,
                        uint64_t* d_out, uint32_t count, kbfv_plan** out) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(out, KBFV_ERR_INVALID, "null argument");
        KB_REQUIRE(d_rlk, KBFV_ERR_NO_KEY, "relinearisation key missing");
        KB_REQUIRE(d_ct_a && d_ct_b && d_out, KBFV_ERR_INVALID, "null ciphertext pointer");
        KB_REQUIRE(count >= 1, KBFV_ERR_INVALID, "a plan multiplies at least one pair");
        // size the arena now, so the first launch does not move it
        const int chunk = (int)std::min<uint32_t>(count, kMaxBatch);
        ensure_scratch(c, mul_scratch_need(c, chunk));
        auto* p = new kbfv_plan();
        p->ctx = ctx;
        p->rlk = d_rlk;
        p->a = d_ct_a;
        p->b = d_ct_b;
        p->out = d_out;
        p->count = count;
        *out = p;
    });
}

int kbfv_plan_mul_relin_levels(kbfv_context* ctx, const uint64_t* d_rlk, const uint32_t* live_q,
                               const uint64_t* const* ct_a, const uint64_t* const* ct_b, uint64_t* const* out,
                               uint32_t count, kbfv_plan** plan) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(!c.parent, KBFV_ERR_INVALID, "call on the top-level context");
        KB_REQUIRE(plan, KBFV_ERR_INVALID, "null argument");
        KB_REQUIRE(d_rlk, KBFV_ERR_NO_KEY, "relinearisation key missing");
        KB_REQUIRE(live_q && ct_a && ct_b && out, KBFV_ERR_INVALID, "null pointer array");
        KB_REQUIRE(count >= 1, KBFV_ERR_INVALID, "a plan multiplies at least one pair");
        for (uint32_t i = 0; i < count; i++) {
            KB_REQUIRE(live_q[i] >= 1 && live_q[i] <= (uint32_t)c.nq, KBFV_ERR_LEVEL, "live prime count out of range");
            KB_REQUIRE(ct_a[i] && ct_b[i] && out[i], KBFV_ERR_INVALID, "null ciphertext pointer");
        }
        // the mixed batch uses the top level's per-pair scratch layout
        ensure_scratch(c, mul_scratch_need(c, (int)std::min<uint32_t>(count, kMaxBatch)));
        auto* p = new kbfv_plan();
        p->ctx = ctx;
        p->rlk = d_rlk;
        p->count = count;
        p->levels = true;
        p->live_q.assign(live_q, live_q + count);
        p->va.assign(ct_a, ct_a + count);
        p->vb.assign(ct_b, ct_b + count);
        p->vo.assign(out, out + count);
        *plan = p;
    });
}

int kbfv_plan_launch(kbfv_plan* plan, kbfv_stream stream) {
    return guarded([&] {
        KB_REQUIRE(plan && plan->ctx, KBFV_ERR_INVALID, "null plan");
        kbfv_plan& p = *plan;
        cudaStream_t st = S(stream);
        if (!graph_current(p)) {
            run_and_capture(p, st);  // this launch's product comes from the eager run
        } else {
            KB_CHECK_CUDA(cudaGraphLaunch(p.exec, st));
        }
        p.launches++;
    });
}

int kbfv_plan_info(const kbfv_plan* plan, uint64_t* launches, uint64_t* captures) {
    return guarded([&] {
        KB_REQUIRE(plan, KBFV_ERR_INVALID, "null plan");
        if (launches) *launches = plan->launches;
        if (captures) *captures = plan->captures;
    });
}

int kbfv_plan_destroy(kbfv_plan* plan) {
    return guarded([&] {
        if (!plan) return;
        drop_graph(*plan);
        if (plan->cs) cudaStreamDestroy(plan->cs);
        delete plan;
    });
}

}  // extern "C"
