// iac_internal.cuh -- shared internals of libiac_b200 (context, errors,
// scratch memory, exact-arithmetic helpers).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/iac_b200.h"
#include <nvtx3/nvToolsExt.h>

#define IAC_COPY_CHUNKS 8

namespace iac {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
void set_error(const char *fmt, ...);

#define IAC_CUDA(call)                                                              \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) {                                                    \
            ::iac::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                             __FILE__, __LINE__);                                   \
            return e_ == cudaErrorMemoryAllocation ? IAC_ERR_NO_MEMORY : IAC_ERR_CUDA; \
        }                                                                           \
    } while (0)

#define IAC_REQUIRE(cond, ...)               \
    do {                                     \
        if (!(cond)) {                       \
            ::iac::set_error(__VA_ARGS__);   \
            return IAC_ERR_INVALID_ARG;      \
        }                                    \
    } while (0)

// NVTX range over a C-ABI call, named after it: visible to Nsight Systems and
// to ncu --nvtx when a tool is attached, a no-op otherwise (header-only NVTX)
struct TraceRange {
    explicit TraceRange(const char *name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
};
#define IAC_TRACE() ::iac::TraceRange iac_trace_range_(__func__)

#define IAC_LAUNCHED(ctx) ((ctx)->launches.fetch_add(1, std::memory_order_relaxed))

// ---------------------------------------------------------------------------
// device-side error counters, one block per context
// ---------------------------------------------------------------------------
struct DeviceCounters {
    unsigned long long out_of_mesh;
    unsigned long long timeouts;
    unsigned long long photon_overflow;  // photons beyond a photon-list capacity (dropped)
    unsigned long long timeout_sites;    // bit k: a kernel of WAIT_SITE_NAMES[k] gave up a bounded wait
    unsigned long long pad[4];
};

// kernels with bounded waits, as bits of DeviceCounters::timeout_sites
enum WaitSite {
    SITE_AVERAGE = 0,
    SITE_WAIT_TEST,
    SITE_CONV_TAP,
    SITE_CONV_SLAB,
    SITE_CONV_TMA,
    SITE_CONV_ZCOL,
    SITE_CONV_ZCAT,
    SITE_WGRAD_TC,
    SITE_WGRAD_ZS,
    SITE_COUNT
};
constexpr const char *WAIT_SITE_NAMES[SITE_COUNT] = {"average",        "flag wait",      "conv (per tap)",
                                                     "conv (slabs)",   "conv (TMA)",     "conv (z-column)",
                                                     "conv (dz-concat)", "weight gradient", "weight gradient (dz-stacked)"};

__device__ __forceinline__ void note_timeout(DeviceCounters *c, int site)
{
    if (!c) return;
    atomicAdd(&c->timeouts, 1ull);
    atomicOr(&c->timeout_sites, 1ull << site);
}

// A growable device scratch buffer owned by the context.
struct Scratch {
    void *ptr = nullptr;
    size_t bytes = 0;
    iac_status ensure(size_t need);
    void release();
};

// Per-stream scratch slots, so that host threads working on their own streams
// never share a work queue or a staging buffer.
enum ScratchSlot {
    SLOT_TILES = 0,   // sparse: per-frame tile table + queue counter
    SLOT_PHOTONS,     // host-buffer entry points: staged inputs / outputs
    SLOT_OFFSETS,
    SLOT_ROT,
    SLOT_HALF,
    SLOT_FULL,
    SLOT_AUX0,
    SLOT_AUX1,
    SLOT_PHOTONS2,    // second staging set of the host-buffer entry points
    SLOT_OFFSETS2,
    SLOT_ROT2,
    SLOT_COUNT
};
struct StreamScratch {
    Scratch bufs[SLOT_COUNT];
};

}  // namespace iac

struct iac_ctx {
    int device = 0;
    int sm_count = 0;
    int cc_major = 0, cc_minor = 0;
    std::mutex mu;  // guards scratch growth and tuning
    iac::DeviceCounters *d_counters = nullptr;
    iac::Scratch sparse_scratch;
    std::unordered_map<void *, iac::StreamScratch> stream_scratch;  // keyed by stream
    iac_sparse_tuning tuning{};  // explicit override (zeros: use the table)
    struct TuningRow {
        uint32_t edge, tile_pairs, block_threads, ctas_per_sm, cache_hints;
    };
    std::vector<TuningRow> tuning_table;  // autotuner results, tuning/sparse_tuning.tsv
    uint64_t scratch_limit = 0;  // largest scratch buffer the context may grow (0: no limit)
    cudaStream_t host_stream = nullptr;  // stream of the host-buffer entry points
    cudaStream_t copy_stream = nullptr;  // their host-to-device copies
    cudaEvent_t copy_events[IAC_COPY_CHUNKS + 1] = {};
    cudaEvent_t staging_free[2] = {};    // recorded after the binning that read host-entry staging set 0 / 1
    int staging_set = 0;                 // the set the next host-entry call fills
    std::mutex host_mu;                  // one host-buffer entry point at a time (shared copy stream)
    void *static_scratch = nullptr;      // device address of iac_sparse_ac_batch_static's fixed array
    std::atomic<uint64_t> launches{0};
};

namespace iac {

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Looks up, with the context's device current, the device address of the
// fixed scratch array of iac_sparse_ac_batch_static (sparse_ac.cu) and keeps
// it in the context.
iac_status static_scratch_setup(iac_ctx *ctx);

// Scratch slot `slot` of `stream`, grown to at least `bytes`.
inline iac_status stream_scratch(iac_ctx *ctx, void *stream, int slot, size_t bytes, void **out)
{
    std::lock_guard<std::mutex> lk(ctx->mu);
    Scratch &s = ctx->stream_scratch[stream].bufs[slot];
    if (ctx->scratch_limit && bytes > ctx->scratch_limit && bytes > s.bytes) {
        set_error("scratch of %zu bytes exceeds the context's limit of %llu bytes", bytes,
                  (unsigned long long)ctx->scratch_limit);
        *out = nullptr;
        return IAC_ERR_NO_MEMORY;
    }
    iac_status st = s.ensure(bytes);
    *out = s.ptr;
    return st;
}

// RAII guard that makes the context's device current for the calling thread.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// ---------------------------------------------------------------------------
// exact arithmetic: every operation explicitly rounded, never contracted
// into a fused multiply-add, in the reference's operation order.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// |q| as sqrt(q0*q0 + q1*q1 + q2*q2), left to right, IEEE sqrt.
__device__ __forceinline__ float norm3(float q0, float q1, float q2)
{
    return __fsqrt_rn(fadd(fadd(fmul(q0, q0), fmul(q1, q1)), fmul(q2, q2)));
}

// Row-major M*v as q0*R0 + q1*R1 + q2*R2 (ArrayOperators::Rotate order).
__device__ __forceinline__ float rot_row(float a, float b, float c, float r0, float r1, float r2)
{
    return fadd(fadd(fmul(a, r0), fmul(b, r1)), fmul(c, r2));
}

// C cast (unsigned long)(double) for the non-negative values of the path.
__device__ __forceinline__ unsigned long long d2u64(double x) { return __double2ull_rz(x); }

// ---------------------------------------------------------------------------
// 64-bit counters in shared memory kept as two 32-bit words.  32-bit shared
// atomics are native; 64-bit ones run several times slower on B200 (measured:
// 1.5e12 against 7.4e12 conflict-free adds per second), and more so when lanes
// of a warp meet at one word.  The low words take the low 32 bits of each
// addend; a carry out of a low word is seen by the add that caused it (the
// returned old value) and goes to the high word with the addend's high bits.
// The pair of words equals the 64-bit sum modulo 2^64, like a 64-bit counter.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void shared_add_u64_split(uint32_t *lo, uint32_t *hi, uint32_t i, unsigned long long v)
{
    const uint32_t vl = (uint32_t)v;
    const uint32_t old = atomicAdd(&lo[i], vl);
    const uint32_t up = (uint32_t)(v >> 32) + (old + vl < old ? 1u : 0u);
    if (up) atomicAdd(&hi[i], up);
}

__device__ __forceinline__ unsigned long long split_word(const uint32_t *lo, const uint32_t *hi, uint32_t i)
{
    return ((unsigned long long)hi[i] << 32) | lo[i];
}

// ---------------------------------------------------------------------------
// round half away from zero (C round / OpenCL round) with FP32 adds only.
// (|x| + 1.5*2^23) - 1.5*2^23 rounds |x| to the nearest integer, ties to even;
// a tie that went down is moved up.  Exact for |x| < 2^22; larger magnitudes
// (which only non-orthonormal rotations produce) take roundf.
// ---------------------------------------------------------------------------
constexpr float ROUND_MAGIC = 12582912.0f;  // 1.5 * 2^23

__device__ __forceinline__ float round_away_f(float x)
{
    const float a = fabsf(x);
    if (!(a < 4194304.0f)) return roundf(x);
    float r = fsub(fadd(a, ROUND_MAGIC), ROUND_MAGIC);
    if (fsub(a, r) == 0.5f) r = fadd(r, 1.0f);
    return copysignf(r, x);
}

// ---------------------------------------------------------------------------
// round half away from zero with two FP32 adds and an integer subtract, for
// the photon-pair kernel.  y = fl(|x| + 0.49999997) reaches the next integer
// exactly when |x| is at or past the half (exhaustive check over all floats
// below 2^23: tests/test_rounding.py), and __fadd_rz(y, 2^23) = 2^23 + floor(y)
// for 0 <= y < 2^23, so its bits minus those of 2^23 are round(|x|).
// ---------------------------------------------------------------------------
constexpr int TWO23_BITS = 0x4B000000;  // bits of 2^23

// exact for |x| < 2^23; larger, infinite or NaN x give |result| >= 2^23,
// outside every mesh
__device__ __forceinline__ int round_away_rz_i(float x)
{
    const int r = __float_as_int(__fadd_rz(fadd(fabsf(x), 0.49999997f), 8388608.0f)) - TWO23_BITS;
    return x < 0.0f ? -r : r;
}

// floor of 0 <= q < 2^23 as a float and as an integer on the FMA and integer
// pipes (no conversion-unit instruction): q +rz 2^23 = 2^23 + floor(q) exactly,
// and its bits minus those of 2^23 are floor(q).  A NaN q (non-finite
// k-vectors only) gives a large index: the host-route histogram counts it as
// out of range, the histograms that wrap their bins (as the reference's
// sub-histogram fold does) take it modulo their size.
__device__ __forceinline__ float floor_small(float q, uint32_t &iq)
{
    const float t = __fadd_rz(q, 8388608.0f);
    iq = (uint32_t)(__float_as_int(t) - TWO23_BITS);
    return fsub(t, 8388608.0f);
}

// as a float; exact for |x| < 2^23 (callers bound x), NaN stays NaN
__device__ __forceinline__ float round_away_rz_f(float x)
{
    return copysignf(fsub(__fadd_rz(fadd(fabsf(x), 0.49999997f), 8388608.0f), 8388608.0f), x);
}

}  // namespace iac
