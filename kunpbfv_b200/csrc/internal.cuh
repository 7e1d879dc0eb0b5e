// Host-side plumbing shared by the library's translation units: errors and
// status codes, launch helpers of the NTT kernels, the dispatch of
// per-coefficient kernels, and the batch / scratch descriptors of the batched
// multiply.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/kbfv.h"
#include "context.cuh"
#include "host_math.hpp"
#include "kernels.cuh"
#include "ntt.cuh"
#include "klss.cuh"

using namespace kbfv;
namespace H = kbfv::host;

// ===========================================================================
// errors
// ===========================================================================
// last error message of the calling thread (kbfv_last_error)
extern thread_local std::string g_last_error;

struct KbfvError : std::runtime_error {
    int code;
    KbfvError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define KB_CHECK_CUDA(call)                                                                        \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            throw KbfvError(e_ == cudaErrorMemoryAllocation ? KBFV_ERR_NOMEM : KBFV_ERR_CUDA,      \
                            std::string(#call) + ": " + cudaGetErrorString(e_));                   \
    } while (0)

#define KB_REQUIRE(cond, code, msg) \
    do {                            \
        if (!(cond)) throw KbfvError((code), (msg)); \
    } while (0)

template <class F>
static int guarded(F&& f) {
    try {
        f();
        return KBFV_OK;
    } catch (const KbfvError& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return KBFV_ERR_INVALID;
    }
}

static inline void check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw KbfvError(KBFV_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
// ===========================================================================
// launch helpers
// ===========================================================================
static inline cudaStream_t S(kbfv_stream s) { return (cudaStream_t)s; }
static inline unsigned blocks_for(size_t total, unsigned threads) { return (unsigned)((total + threads - 1) / threads); }
// grid of a grid-stride kernel: enough blocks to cover `total`, at most 2^20
static inline unsigned stride_blocks(size_t total, unsigned threads) {
    return (unsigned)std::min<size_t>((total + threads - 1) / threads, (size_t)1 << 20);
}

// CTAs of `kernel` that fit on the device at once (SMs x CTAs per SM)
static inline int resident_ctas(const void* kernel, int threads, int smem) {
    int dev = 0, sms = 0, per = 0;
    KB_CHECK_CUDA(cudaGetDevice(&dev));
    KB_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    KB_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem));
    return sms * std::max(per, 1);
}

// the same for launch shapes chosen at run time: cached per CTA size (64..512)
static inline int resident_ctas_at(const void* kernel, int threads, int smem, int (&cache)[4]) {
    const int i = std::min(3, std::max(0, __builtin_ctz((unsigned)threads) - 6));
    if (!cache[i]) cache[i] = resident_ctas(kernel, threads, smem);
    return cache[i];
}

template <int LOGB, class Src, class Dst, bool FULL = true>
static void launch_fwd_block(const DevConsts& dc, Src s, Dst d, int rows, int logn, cudaStream_t st) {
    constexpr int SMEM = BlockShape<LOGB>::SMEM_BYTES;
    static bool configured = false;
    static int resident = 0;  // CTAs of this kernel resident at once on the device
    if (!configured) {
        KB_CHECK_CUDA(cudaFuncSetAttribute(ntt_fwd_block_kernel<LOGB, Src, Dst, FULL>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
        resident = resident_ctas((const void*)ntt_fwd_block_kernel<LOGB, Src, Dst, FULL>,
                                 BlockShape<LOGB>::THREADS, SMEM);
        configured = true;
    }
    const int nblk = 1 << (logn - LOGB);
    ntt_fwd_block_kernel<LOGB, Src, Dst, FULL><<<rows * nblk, BlockShape<LOGB>::THREADS, SMEM, st>>>(
        s, d, dc.tw_fwd, dc.mods, logn, dc.shape.l2_prefetch ? resident : 0);
}

template <int LOGB, class Src, class Dst, bool WHOLE>
static void launch_inv_block(const DevConsts& dc, Src s, Dst d, int rows, int logn, cudaStream_t st) {
    constexpr int SMEM = BlockShape<LOGB>::SMEM_BYTES;
    static bool configured = false;
    static int resident = 0;  // CTAs of this kernel resident at once on the device
    if (!configured) {
        KB_CHECK_CUDA(cudaFuncSetAttribute(ntt_inv_block_kernel<LOGB, Src, Dst, WHOLE>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
        resident = resident_ctas((const void*)ntt_inv_block_kernel<LOGB, Src, Dst, WHOLE>,
                                 BlockShape<LOGB>::THREADS, SMEM);
        configured = true;
    }
    const int nblk = 1 << (logn - LOGB);
    ntt_inv_block_kernel<LOGB, Src, Dst, WHOLE><<<rows * nblk, BlockShape<LOGB>::THREADS, SMEM, st>>>(
        s, d, dc.tw_inv, dc.mods, logn, dc.shape.l2_prefetch ? resident : 0);
}

// The view of a store target that the column pass of a split transform writes
// and the block kernel reads back: the target itself, unless its store adds an
// epilogue (an overload for that target returns its plain rows).
template <class Dst>
static inline Dst plain_of(const Dst& d) { return d; }

// At N = 2^14, launches of at most this many rows (fewer 1024-thread CTAs
// than SMs, e.g. one ciphertext pair per call: 2-45 rows) run as a radix-4
// column pass and 2^12-point blocks: four times the CTAs cover the SMs, 15-23 us
// instead of 29-31 us per launch of 8-45 rows on the B200. At 64 rows the
// split alone is still faster, but beside a concurrent sub-batch it cost the
// batched multiply ~1%, so 64-row launches keep the whole-ring blocks. The
// default of LaunchShape::split_rows14 (KBFV_TUNE_SPLIT_ROWS).
constexpr int kSplitRows14Default = 48;
// The same threshold for a multiply that runs as one stream (batches below two
// sub-batches, the tensor-only multiply): launches of up to 148 rows would
// leave SMs idle with one 1024-thread CTA per row, and no sibling sub-batch
// fills them, so they split (2 pairs: 0.211 -> 0.192 ms on the B200). The
// default of LaunchShape::split_rows_alone (KBFV_TUNE_SPLIT_ROWS_ALONE).
constexpr int kSplitRowsAloneDefault = 148;

// Forward NTT of `rows` rows read through `s` and written through `d`.
// For logn <= 14 one block kernel (N = 2^14 with at most shape.split_rows14 rows:
// as for 15/16 with a radix-4 column pass); for 15/16 a radix-8/16 column pass
// (s -> plain_of(d)) then 2^12-point block kernels from plain_of(d) to d in
// place (d must also be readable): several 256-thread CTAs per SM run faster
// than one 1024-thread CTA per 2^14-point block. FULL = false leaves outputs in [0, 8q) for consumers that reduce
// anyway (pipeline stages only).
template <class Src, class Dst, bool FULL = true>
static void ntt_fwd(const DevConsts& dc, Src s, Dst d, int rows, cudaStream_t st) {
    if (rows <= 0) return;
    switch (dc.logn) {
        case 10: launch_fwd_block<10, Src, Dst, FULL>(dc, s, d, rows, 10, st); break;
        case 11: launch_fwd_block<11, Src, Dst, FULL>(dc, s, d, rows, 11, st); break;
        case 12: launch_fwd_block<12, Src, Dst, FULL>(dc, s, d, rows, 12, st); break;
        case 13: launch_fwd_block<13, Src, Dst, FULL>(dc, s, d, rows, 13, st); break;
        case 14: {
            if (rows > dc.shape.split_rows14) {
                launch_fwd_block<14, Src, Dst, FULL>(dc, s, d, rows, 14, st);
                break;
            }
            const size_t total = (size_t)rows << 12;
            using DP = decltype(plain_of(d));
            const DP dp = plain_of(d);
            ntt_fwd_col_kernel<2, Src, DP><<<stride_blocks(total, 256), 256, 0, st>>>(s, dp, dc.tw_fwd, dc.mods, 14, total);
            launch_fwd_block<12, DP, Dst, FULL>(dc, dp, d, rows, 14, st);
            break;
        }
        case 15: {
            const size_t total = (size_t)rows << 12;
            using DP = decltype(plain_of(d));
            const DP dp = plain_of(d);
            ntt_fwd_col_kernel<3, Src, DP><<<stride_blocks(total, 256), 256, 0, st>>>(s, dp, dc.tw_fwd, dc.mods, 15, total);
            launch_fwd_block<12, DP, Dst, FULL>(dc, dp, d, rows, 15, st);
            break;
        }
        case 16: {
            const size_t total = (size_t)rows << 12;
            using DP = decltype(plain_of(d));
            const DP dp = plain_of(d);
            ntt_fwd_col16_kernel<4, Src, DP><<<stride_blocks(total, 256), 256, 0, st>>>(s, dp, dc.tw_fwd, dc.mods, 16, total);
            launch_fwd_block<12, DP, Dst, FULL>(dc, dp, d, rows, 16, st);
            break;
        }
        default: throw KbfvError(KBFV_ERR_INVALID, "unsupported ring degree");
    }
    check_launch("ntt_fwd");
}

template <class Src, class Dst>
static void ntt_inv(const DevConsts& dc, Src s, Dst d, int rows, cudaStream_t st) {
    if (rows <= 0) return;
    switch (dc.logn) {
        case 10: launch_inv_block<10, Src, Dst, true>(dc, s, d, rows, 10, st); break;
        case 11: launch_inv_block<11, Src, Dst, true>(dc, s, d, rows, 11, st); break;
        case 12: launch_inv_block<12, Src, Dst, true>(dc, s, d, rows, 12, st); break;
        case 13: launch_inv_block<13, Src, Dst, true>(dc, s, d, rows, 13, st); break;
        case 14: {
            if (rows > dc.shape.split_rows14) {
                launch_inv_block<14, Src, Dst, true>(dc, s, d, rows, 14, st);
                break;
            }
            launch_inv_block<12, Src, Dst, false>(dc, s, d, rows, 14, st);
            const size_t total = (size_t)rows << 12;
            ntt_inv_col_kernel<2, Dst, Dst><<<stride_blocks(total, 256), 256, 0, st>>>(d, d, dc.tw_inv, dc.mods, 14, total);
            break;
        }
        case 15: {
            launch_inv_block<12, Src, Dst, false>(dc, s, d, rows, 15, st);
            const size_t total = (size_t)rows << 12;
            ntt_inv_col_kernel<3, Dst, Dst><<<stride_blocks(total, 256), 256, 0, st>>>(d, d, dc.tw_inv, dc.mods, 15, total);
            break;
        }
        case 16: {
            launch_inv_block<12, Src, Dst, false>(dc, s, d, rows, 16, st);
            const size_t total = (size_t)rows << 12;
            ntt_inv_col16_kernel<4, Dst, Dst><<<stride_blocks(total, 256), 256, 0, st>>>(d, d, dc.tw_inv, dc.mods, 16, total);
            break;
        }
        default: throw KbfvError(KBFV_ERR_INVALID, "unsupported ring degree");
    }
    check_launch("ntt_inv");
}

static inline RowsIO rows_io(const DevConsts& dc, uint64_t* base, int p0, int period) {
    return RowsIO{base, dc.logn, p0, period};
}
// bucketed MAX template dispatch for per-coefficient kernels
#define DISPATCH_MAXQ(nq, MACRO) \
    do {                         \
        if ((nq) <= 8) { MACRO(8); }       \
        else if ((nq) <= 16) { MACRO(16); } \
        else if ((nq) <= 24) { MACRO(24); } \
        else { MACRO(33); }                 \
    } while (0)

// HPS base extension of `polys` polynomials (bconv_kernel), in and out strided
void launch_bconv(const DevConsts& dc, const BconvTables& tb, const uint64_t* in, uint64_t* out, int polys,
                  size_t in_stride, size_t out_stride, cudaStream_t st);
// context construction from a parameter set (tables in one device pool)
void build_context(Context& c, const kbfv_params& prm);
// pieces of a 60-bit residue in base 2^w
static inline int gadget_pieces(int w) { return (60 + w - 1) / w; }

// The context's scratch arena: grown to at least `bytes` (at least 64 MiB;
// never shrinks while the context lives). Synchronises the device when it grows.
uint8_t* ensure_scratch(Context& c, size_t bytes);

// ===========================================================================
// batch and scratch descriptors of the batched multiply
// ===========================================================================
constexpr int kMaxBatch = 128;  // pointer tables ride in kernel parameters
struct PtrBatch {
    const uint64_t* a[kMaxBatch];
    const uint64_t* b[kMaxBatch];
    uint64_t* o[kMaxBatch];
};

struct MulScratch {
    uint64_t *sa, *sb, *sc, *sd, *sd2, *se;
    uint64_t *st1, *st2;  // T-base key switch: digits [item][nqj][nt], products [item][2][nri][nt]
    size_t bytes;
};

static inline MulScratch mul_scratch_layout(const Context& c, int count, uint8_t* base) {
    const size_t limb = c.n * 8;
    const int npq = c.nq + c.np, nqr = c.nq + c.nr;
    size_t off = 0;
    MulScratch m{};
    auto take = [&](size_t limbs) {
        uint64_t* p = (uint64_t*)(base ? base + off : nullptr);
        off += limbs * limb;
        return p;
    };
    m.sa = take((size_t)count * 4 * c.nq);
    m.sb = take((size_t)count * 4 * c.nr);
    m.sc = take((size_t)count * 3 * nqr);
    m.sd = take((size_t)count * 2 * c.nq);
    m.sd2 = take((size_t)count * c.dnum * npq);
    m.se = take((size_t)count * 2 * npq);
    if (c.klss_ok) {
        m.st1 = take((size_t)count * c.kc.nqj * c.nt);
        m.st2 = take((size_t)count * 2 * c.kc.nri * c.nt);
    }
    m.bytes = off;
    return m;
}
// Sub-batches of a batched multiply hold at least Context::min_branch_pairs
// pairs (default 1; KBFV_TUNE_MIN_BRANCH_PAIRS): from 2 pairs on, two
// sub-batches on two streams fill the SMs that one batch's launches of fewer
// rows than SMs leave idle (3 pairs 0.252 -> 0.243 ms against a minimum of 2;
// 4 pairs 0.314 -> 0.265 ms, 8 pairs 0.481 -> 0.408 ms, 12 pairs 0.679 ->
// 0.597 ms on the B200 against a minimum of 8).
static inline int branch_count(const Context& c, int cnt) {
    return std::max(1, std::min(c.branches, cnt / std::max(1, c.min_branch_pairs)));
}
static inline size_t branch_region_bytes(const Context& c, int per) {
    return (mul_scratch_layout(c, per, nullptr).bytes + 255) & ~(size_t)255;
}
static inline size_t mul_scratch_need(const Context& c, int cnt) {
    const int nb = branch_count(c, cnt);
    const size_t whole = mul_scratch_layout(c, cnt, nullptr).bytes;
    return nb == 1 ? whole : std::max(whole, branch_region_bytes(c, (cnt + nb - 1) / nb) * nb);
}
static inline PtrBatch make_batch(const uint64_t* const* a, const uint64_t* const* b, uint64_t* const* o, int cnt) {
    PtrBatch pb;
    std::memset(&pb, 0, sizeof pb);
    for (int i = 0; i < cnt; i++) {
        pb.a[i] = a[i];
        pb.b[i] = b[i];
        pb.o[i] = o ? o[i] : nullptr;
    }
    return pb;
}

// Fused stages run as one block kernel for N <= 2^14; for split transforms
// (N = 2^15, 2^16, and launches of few rows at 2^14) the fused loader feeds
// the column pass and the store target is read back by the block kernel, which
// every functor here supports.
static inline void require_batchable(const Context& c) {
    KB_REQUIRE(c.logn >= 10 && c.logn <= 16, KBFV_ERR_UNSUPPORTED, "ring degree outside 2^10..2^16");
}
static inline void require_top(const Context& c) {
    KB_REQUIRE(!c.parent, KBFV_ERR_LEVEL, "keys and encryptions are made on the top-level context");
}
static inline void require_klss(const Context& c) {
    KB_REQUIRE(c.klss_ok, KBFV_ERR_INVALID,
               "context has no T-base key switch (needs T primes, q_count divisible by p_count, dnum = q_count / p_count)");
}

// opaque handle of the C ABI
struct kbfv_context {
    Context c;
};

static inline Context& CX(kbfv_context* h) {
    if (!h) throw KbfvError(KBFV_ERR_INVALID, "null context");
    return h->c;
}
