// sparse_ac.cu -- (a) sparse photon pairs -> uint64 3D q-mesh.
//
// Replaces the device route of Detector::AutoCorrelateSparseList
// (IAC/Detector.cpp:1053-1181) and its kernel Autocor_sparseHL with helpers
// AddRotatedQToMesh / AddQToPositiveSS (IAC/kernel.cl:349-652), batched over
// many frames.
//
// Work decomposition.  A frame of n photons has n(n-1)/2 distinct pairs plus
// n self pairs.  The planner (one CTA) gives every frame
// max(1, ceil(pairs / tile_pairs)) tiles and writes the exclusive prefix sum of
// those counts: the device work queue.  The pair kernel is persistent: each
// CTA pops the next tile index with one atomic, finds its frame by binary
// search over the prefix table and walks the tile's pairs, one pair per thread
// per step.  Frames of 5 or 2 500 photons therefore cost in proportion to their
// pair count, and no CTA waits on another.
//
// Pair enumeration.  Local pair l of a frame maps to
//   d = l / n + 1,  i = l % n,  j = (i + d) mod n
// which lists every unordered pair {i, j}, i != j, exactly once for l in
// [0, n(n-1)/2) (a circulant walk: offsets d = 1 .. floor((n-1)/2) for every
// i, plus d = n/2 for i < n/2 when n is even).  Consecutive threads take
// consecutive i at the same offset d, so their photon loads are contiguous.
// The pair is then evaluated exactly as the reference's work item does for
// ind = min(i, j) and i = max(i, j): q = k_lo - k_hi.
//
// Exactness.  All float operations are the reference's, in its order, as
// explicitly rounded intrinsics (no contraction into FMA); sqrt is IEEE; the
// value (double)v_lo * v_hi * Multiplicator is truncated to uint64 as the C
// cast does.  Self pairs add (uint64)(v*v*Mult) at q = 0, which the reference
// writes to half-mesh voxel (C, C, 0) without a mirror for every second-level
// interpolation mode; they are summed per tile and added with one atomic.
//
// The half mesh accumulates with 64-bit atomic adds in L2 (the 201^3 half mesh
// is 32.6 MB and stays L2-resident).  Writes whose voxel would fall outside the
// mesh (possible only for non-orthonormal rotations; the reference writes them
// out of bounds) are skipped and counted in the context's error block.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "iac_internal.cuh"

namespace iac {

struct SparseArgs {
    const float4 *__restrict__ photons;
    const uint64_t *__restrict__ offsets;
    const float *__restrict__ rot;
    const unsigned long long *__restrict__ tile_off;  // nframes + 1
    unsigned long long *__restrict__ half;
    unsigned long long *queue;
    DeviceCounters *counters;
    uint32_t nframes;
    uint32_t tile_pairs;
    int S, C, half_ss;
    uint32_t plane;  // S * S (the half mesh has fewer than 2^32 words for S <= 1621)
    float maxq;
    float maxq2;  // largest float s with sqrtf(s) <= maxq: |q| > maxq  <=>  |q|^2 > maxq2
    float vpdq;   // (float)Voxel_per_dq
    double mult;
    float mult_f;                           // Multiplicator as float when it is an integer <= 1024
    const unsigned char *__restrict__ small_counts;  // per frame: counts are integers in [0, 128]
    int cache_hints;  // 1: mesh atomics evict-last, photon loads evict-first in L2
    uint64_t mesh_policy;  // set inside the kernel when cache_hints is on
    int box_r;        // half-width of the shared-memory box around q = 0 (0: none)
    int box_w;        // 2 * box_r + 1
    uint32_t box_base;  // shared-memory address of the box's low words (set inside the kernel)
    uint32_t box_hi;    // shared-memory address of its high words (set inside the kernel)
};

// L2 cache policies (PTX createpolicy) for the pair kernel: the half mesh is
// kept resident while the photon stream passes through.
__device__ __forceinline__ uint64_t l2_policy_evict_last()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_first()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ void red_add_hint(unsigned long long *addr, unsigned long long v, uint64_t pol)
{
    asm volatile("red.global.add.L2::cache_hint.u64 [%0], %1, %2;" ::"l"(addr), "l"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ float4 ld_photon_hint(const float4 *p, uint64_t pol)
{
    float4 r;
    asm volatile("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
                 : "l"(p), "l"(pol));
    return r;
}

// ---------------------------------------------------------------------------
// planner: tiles per frame, exclusive scan, queue reset (one CTA)
// ---------------------------------------------------------------------------
constexpr int PLAN_THREADS = 1024;

__device__ __forceinline__ unsigned long long frame_tiles(const uint64_t *off, uint32_t f,
                                                          uint32_t tile_pairs)
{
    const unsigned long long n = off[f + 1] - off[f];
    if (n == 0) return 0;
    const unsigned long long pairs = n * (n - 1) / 2;
    const unsigned long long t = (pairs + tile_pairs - 1) / tile_pairs;
    return t > 0 ? t : 1;
}

__global__ void __launch_bounds__(PLAN_THREADS)
    sparse_plan_kernel(const uint64_t *__restrict__ off, uint32_t nframes, uint32_t tile_pairs,
                       unsigned long long *__restrict__ tile_off, unsigned long long *queue)
{
    __shared__ unsigned long long warp_sums[PLAN_THREADS / 32];
    const uint32_t tid = threadIdx.x;
    const uint32_t chunk = (nframes + PLAN_THREADS - 1) / PLAN_THREADS;
    const uint32_t f0 = min(nframes, tid * chunk), f1 = min(nframes, f0 + chunk);
    unsigned long long local = 0;
    for (uint32_t f = f0; f < f1; f++) local += frame_tiles(off, f, tile_pairs);
    // block-wide exclusive scan of the per-thread sums
    const int lane = tid & 31, w = tid >> 5;
    unsigned long long incl = local;
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) warp_sums[w] = incl;
    __syncthreads();
    if (w == 0) {
        unsigned long long v = warp_sums[lane];
        unsigned long long s = v;
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long u = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += u;
        }
        warp_sums[lane] = s - v;  // exclusive warp prefix
    }
    __syncthreads();
    unsigned long long run = warp_sums[w] + incl - local;
    for (uint32_t f = f0; f < f1; f++) {
        tile_off[f] = run;
        run += frame_tiles(off, f, tile_pairs);
    }
    if (tid == PLAN_THREADS - 1) {
        tile_off[nframes] = warp_sums[w] + incl;
        *queue = 0ull;
    }
}

// ---------------------------------------------------------------------------
// per-frame check: are all photon values integers in [0, 128]?  Then the pair
// value v_lo * v_hi * Mult (Mult an integer <= 1024) is at most 2^24 and the
// FP32 product is exact, equal to the reference's double product.
// One warp per frame.
// ---------------------------------------------------------------------------
__global__ void sparse_count_check_kernel(const float4 *__restrict__ ph, const uint64_t *__restrict__ off,
                                          uint32_t nframes, unsigned char *__restrict__ flags)
{
    const uint32_t f = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (f >= nframes) return;
    bool ok = true;
    for (uint64_t i = off[f] + lane; i < off[f + 1]; i += 32) {
        const float w = ph[i].w;
        ok &= (w >= 0.0f) && (w <= 128.0f) && (w == truncf(w));
    }
    ok = __all_sync(0xffffffffu, ok);
    if (lane == 0) flags[f] = ok ? 1 : 0;
}

// ---------------------------------------------------------------------------
// binning helpers (IAC/kernel.cl:349-448)
// ---------------------------------------------------------------------------
// v into word k of the shared-memory box, a split 64-bit counter (low words at
// box_base, high words at box_hi): 32-bit shared atomics are native, 64-bit
// ones are several times slower, above all where the lanes of a warp meet at
// one voxel near q = 0
__device__ __forceinline__ void box_add(const SparseArgs &a, uint32_t k, unsigned long long v)
{
    const uint32_t vl = (uint32_t)v;
    uint32_t old;
    asm volatile("atom.shared.add.u32 %0, [%1], %2;" : "=r"(old) : "r"(a.box_base + 4u * k), "r"(vl) : "memory");
    const uint32_t up = (uint32_t)(v >> 32) + (old + vl < old ? 1u : 0u);
    if (up) asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(a.box_hi + 4u * k), "r"(up) : "memory");
}

__device__ __forceinline__ void hm_put(const SparseArgs &a, int fs, int ms, int ss,
                                       unsigned long long v)
{
    if ((unsigned)fs >= (unsigned)a.S || (unsigned)ms >= (unsigned)a.S ||
        (unsigned)ss >= (unsigned)a.half_ss) {
        atomicAdd(&a.counters->out_of_mesh, 1ull);
        return;
    }
    if (v == 0) return;
    if (a.box_r) {  // the voxels around q = 0 collect in the CTA's shared-memory box
        const uint32_t dx = (uint32_t)(fs - a.C + a.box_r), dy = (uint32_t)(ms - a.C + a.box_r);
        if (dx < (uint32_t)a.box_w && dy < (uint32_t)a.box_w && (uint32_t)ss <= (uint32_t)a.box_r) {
            const uint32_t k = ((uint32_t)ss * a.box_w + dy) * a.box_w + dx;
            box_add(a, k, v);
            return;
        }
    }
    unsigned long long *addr = &a.half[(uint32_t)fs + (uint32_t)ms * (uint32_t)a.S + (uint32_t)ss * a.plane];
    if (a.cache_hints)
        red_add_hint(addr, v, a.mesh_policy);
    else
        atomicAdd(addr, v);
}

// AddQToPositiveSS, IAC/kernel.cl:349-372 (q != 0 here; q = 0 is the self pair)
__device__ __forceinline__ void add_positive_ss(const SparseArgs &a, int fs, int ms, int ss,
                                                unsigned long long v)
{
    if (ss > 0) {
        hm_put(a, fs, ms, ss, v);
    } else {
        if (ss == 0) hm_put(a, fs, ms, ss, v);
        hm_put(a, 2 * a.C - fs, 2 * a.C - ms, -ss, v);
    }
}

// Second-level nearest neighbour of AddRotatedQToMesh (IAC/kernel.cl:380-389)
// followed by AddQToPositiveSS: fs = C + round(q0), ms = C + round(q1),
// ss = round(q2); a negative ss goes to the point reflection, ss = 0 goes to
// both.  (The reference adds the float centre to the rounded float, which is
// exact for every in-mesh index.)
__device__ __forceinline__ void add_nearest(const SparseArgs &a, float q0, float q1, float q2,
                                            unsigned long long v)
{
    int fs = a.C + round_away_rz_i(q0);
    int ms = a.C + round_away_rz_i(q1);
    int ss = round_away_rz_i(q2);
    if (ss < 0) {
        fs = 2 * a.C - fs;
        ms = 2 * a.C - ms;
        ss = -ss;
    }
    hm_put(a, fs, ms, ss, v);
    if (ss == 0) hm_put(a, 2 * a.C - fs, 2 * a.C - ms, 0, v);
}

// AddRotatedQToMesh, IAC/kernel.cl:374-448
template <int I2>
__device__ __forceinline__ void add_rotated(const SparseArgs &a, double val, float q0, float q1,
                                            float q2)
{
    const float Cf = (float)a.C;
    if (I2 == 0) {
        const unsigned long long v = d2u64(dmul(val, a.mult));
        add_nearest(a, q0, q1, q2, v);
    } else {
        const float f0 = floorf(q0), f1 = floorf(q1), f2 = floorf(q2);
        const double sf = dsub(1.0, (double)fsub(q0, f0));
        const double sm = dsub(1.0, (double)fsub(q1, f1));
        const double sz = dsub(1.0, (double)fsub(q2, f2));
        const int fs = (int)fadd(Cf, f0), ms = (int)fadd(Cf, f1), ss = (int)f2;
        const double tm = dmul(val, a.mult);
        const double xf[2] = {sf, dsub(1.0, sf)}, yf[2] = {sm, dsub(1.0, sm)},
                     zf[2] = {sz, dsub(1.0, sz)};
#pragma unroll
        for (int cz = 0; cz < 2; cz++)
#pragma unroll
            for (int cy = 0; cy < 2; cy++)
#pragma unroll
                for (int cx = 0; cx < 2; cx++) {
                    const double w = dmul(dmul(xf[cx], yf[cy]), zf[cz]);
                    add_positive_ss(a, fs + cx, ms + cy, ss + cz, d2u64(dmul(tm, w)));
                }
    }
}

// One distinct pair, the body of the reference's loop for i > ind
// (IAC/kernel.cl:493-649).
template <int DMAP, int I1, int I2>
__device__ __forceinline__ void bin_pair(const SparseArgs &a, const float4 A, const float4 B,
                                         const float *R, const bool small_counts)
{
    float q0 = fsub(A.x, B.x), q1 = fsub(A.y, B.y), q2 = fsub(A.z, B.z);
    // sqrt(|q|^2) > MaxQ, decided on |q|^2 against the exact float threshold
    if (fadd(fadd(fmul(q0, q0), fmul(q1, q1)), fmul(q2, q2)) > a.maxq2) return;
    q0 = fmul(q0, a.vpdq);
    q1 = fmul(q1, a.vpdq);
    q2 = fmul(q2, a.vpdq);
    const int C = a.C;
    const float Cf = (float)C;
    if (I2 == 0 && (DMAP == 0 || I1 == 0)) {
        // nearest neighbour at the second level: value (ulong)(v_lo * v_hi * Mult)
        unsigned long long v;
        if (small_counts)  // integers <= 128 and Mult <= 1024: the float product is exact
            v = (unsigned long long)__float2uint_rz(fmul(fmul(A.w, B.w), a.mult_f));
        else
            v = d2u64(dmul(dmul((double)A.w, (double)B.w), a.mult));
        float t0 = q0, t1 = q1, t2 = q2;
        if (DMAP) {  // first-level nearest neighbour: back to the voxel centre
            // |q| <= MaxQ * Voxel_per_dq < 2^22 here (MaxQ test, host check)
            t0 = round_away_rz_f(q0);
            t1 = round_away_rz_f(q1);
            t2 = round_away_rz_f(q2);
        }
        add_nearest(a, rot_row(t0, t1, t2, R[0], R[1], R[2]), rot_row(t0, t1, t2, R[3], R[4], R[5]),
                    rot_row(t0, t1, t2, R[6], R[7], R[8]), v);
        return;
    }
    const double val = dmul((double)A.w, (double)B.w);
    if (DMAP) {
        if (I1 == 0) {
            const float r0 = round_away_rz_f(q0), r1 = round_away_rz_f(q1), r2 = round_away_rz_f(q2);
            add_rotated<I2>(a, val, rot_row(r0, r1, r2, R[0], R[1], R[2]),
                            rot_row(r0, r1, r2, R[3], R[4], R[5]),
                            rot_row(r0, r1, r2, R[6], R[7], R[8]));
        } else {
            const float f0 = floorf(q0), f1 = floorf(q1), f2 = floorf(q2);
            const double sf = dsub(1.0, (double)fsub(q0, f0));
            const double sm = dsub(1.0, (double)fsub(q1, f1));
            const double sz = dsub(1.0, (double)fsub(q2, f2));
            const int fs = (int)fadd(Cf, f0), ms = (int)fadd(Cf, f1), ss = (int)fadd(Cf, f2);
            const float base = (float)val;
            const double xf[2] = {sf, dsub(1.0, sf)}, yf[2] = {sm, dsub(1.0, sm)},
                         zf[2] = {sz, dsub(1.0, sz)};
#pragma unroll
            for (int cz = 0; cz < 2; cz++)
#pragma unroll
                for (int cy = 0; cy < 2; cy++)
#pragma unroll
                    for (int cx = 0; cx < 2; cx++) {
                        const float tv =
                            (float)dmul((double)base, dmul(dmul(xf[cx], yf[cy]), zf[cz]));
                        const float r0 = (float)((fs + cx) - C), r1 = (float)((ms + cy) - C),
                                    r2 = (float)((ss + cz) - C);
                        add_rotated<I2>(a, (double)tv, rot_row(r0, r1, r2, R[0], R[1], R[2]),
                                        rot_row(r0, r1, r2, R[3], R[4], R[5]),
                                        rot_row(r0, r1, r2, R[6], R[7], R[8]));
                    }
        }
    } else {
        add_rotated<I2>(a, val, rot_row(q0, q1, q2, R[0], R[1], R[2]),
                        rot_row(q0, q1, q2, R[3], R[4], R[5]),
                        rot_row(q0, q1, q2, R[6], R[7], R[8]));
    }
}

// ---------------------------------------------------------------------------
// persistent pair kernel
// ---------------------------------------------------------------------------
template <int DMAP, int I1, int I2>
__global__ void __launch_bounds__(256) sparse_pairs_kernel(SparseArgs a)
{
    uint64_t photon_policy = 0;
    if (a.cache_hints) {
        a.mesh_policy = l2_policy_evict_last();
        photon_policy = l2_policy_evict_first();
    }
    __shared__ unsigned long long s_tile;
    __shared__ uint32_t s_frame;
    __shared__ float s_rot[9];
    __shared__ int s_small;
    __shared__ unsigned long long s_self[8];
    // (box_r + 1) x box_w x box_w split 64-bit counters, [ss][ms][fs]: low words, then high words
    extern __shared__ uint32_t s_box[];

    const unsigned long long ntiles = a.tile_off[a.nframes];
    const uint32_t nthr = blockDim.x;
    const uint32_t box_n = a.box_r ? (uint32_t)(a.box_r + 1) * a.box_w * a.box_w : 0u;
    a.box_base = (uint32_t)__cvta_generic_to_shared(s_box);
    a.box_hi = a.box_base + 4u * box_n;
    for (uint32_t k = threadIdx.x; k < 2 * box_n; k += nthr) s_box[k] = 0u;  // visible after the
                                                                            // loop's first barrier
    for (;;) {
        if (threadIdx.x == 0) {
            const unsigned long long t = atomicAdd(a.queue, 1ull);
            s_tile = t;
            if (t < ntiles) {
                // last frame f with tile_off[f] <= t
                uint32_t lo = 0, hi = a.nframes;  // tile_off[lo] <= t < tile_off[hi]
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (a.tile_off[mid] <= t)
                        lo = mid;
                    else
                        hi = mid;
                }
                s_frame = lo;
                s_small = a.small_counts ? a.small_counts[lo] : 0;
#pragma unroll
                for (int k = 0; k < 9; k++) s_rot[k] = a.rot[9 * (size_t)lo + k];
            }
        }
        __syncthreads();
        const unsigned long long t = s_tile;
        if (t >= ntiles) break;
        const uint32_t f = s_frame;
        const bool small = s_small != 0;
        float R[9];
#pragma unroll
        for (int k = 0; k < 9; k++) R[k] = s_rot[k];
        const uint64_t base = a.offsets[f];
        const uint32_t n = (uint32_t)(a.offsets[f + 1] - base);
        const unsigned long long chunk = t - a.tile_off[f];
        const float4 *__restrict__ P = a.photons + base;

        // self pairs (q = 0): once per frame, on its first tile
        if (chunk == 0) {
            unsigned long long s = 0;
            for (uint32_t i = threadIdx.x; i < n; i += nthr) {
                const double v = (double)P[i].w;
                s += d2u64(dmul(dmul(v, v), a.mult));
            }
            for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if ((threadIdx.x & 31) == 0) s_self[threadIdx.x >> 5] = s;
        }

        // distinct pairs of this tile
        const unsigned long long npairs = (unsigned long long)n * (n - 1) / 2;
        const unsigned long long p0 = chunk * a.tile_pairs;
        const unsigned long long p1 = min(npairs, p0 + a.tile_pairs);
        if (p0 + threadIdx.x < p1) {
            unsigned long long l = p0 + threadIdx.x;
            uint32_t d = (uint32_t)(l / n) + 1;
            uint32_t i = (uint32_t)(l - (unsigned long long)(d - 1) * n);
            const uint32_t dq = nthr / n, dr = nthr % n;
            for (; l < p1; l += nthr) {
                uint32_t j = i + d;
                if (j >= n) j -= n;
                const uint32_t lo = min(i, j), hi = max(i, j);
                if (a.cache_hints)
                    bin_pair<DMAP, I1, I2>(a, ld_photon_hint(P + lo, photon_policy),
                                           ld_photon_hint(P + hi, photon_policy), R, small);
                else
                    bin_pair<DMAP, I1, I2>(a, P[lo], P[hi], R, small);
                i += dr;
                d += dq;
                if (i >= n) {
                    i -= n;
                    d += 1;
                }
            }
        }
        __syncthreads();
        if (chunk == 0 && threadIdx.x == 0) {
            unsigned long long s = 0;
            for (uint32_t w = 0; w < (nthr + 31) / 32; w++) s += s_self[w];
            if (s) {  // q = 0: the box's centre when there is a box
                if (a.box_r)
                    box_add(a, (uint32_t)(a.box_r * a.box_w + a.box_r), s);
                else
                    atomicAdd(&a.half[(size_t)a.C + (size_t)a.C * a.S], s);
            }
        }
    }
    // the loop ends after a barrier: every shared-memory add is done; flush the box
    for (uint32_t k = threadIdx.x; k < box_n; k += nthr) {
        const unsigned long long v = split_word(s_box, s_box + box_n, k);
        if (v == 0) continue;
        const uint32_t ss = k / (uint32_t)(a.box_w * a.box_w), r = k - ss * (uint32_t)(a.box_w * a.box_w);
        const uint32_t ms = (uint32_t)(a.C - a.box_r) + r / (uint32_t)a.box_w;
        const uint32_t fs = (uint32_t)(a.C - a.box_r) + r % (uint32_t)a.box_w;
        unsigned long long *addr = &a.half[fs + ms * (uint32_t)a.S + ss * a.plane];
        if (a.cache_hints)
            red_add_hint(addr, v, a.mesh_policy);
        else
            atomicAdd(addr, v);
    }
}

// ---------------------------------------------------------------------------
// fold: full[fs, ms, ss + C] += half; full[2C - fs, 2C - ms, C - ss] += half
// for ss > 0 (IAC/Detector.cpp:1147-1170).  Every full-mesh voxel receives
// exactly one half-mesh voxel, so plain read-modify-write suffices.
// ---------------------------------------------------------------------------
__global__ void sparse_fold_kernel(const unsigned long long *__restrict__ half, uint32_t S,
                                   unsigned long long *__restrict__ full)
{
    const uint32_t C = (S - 1) / 2;
    const uint64_t plane = (uint64_t)S * S;
    const uint64_t total = plane * ((S + 1) / 2);
    for (uint64_t h = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; h < total;
         h += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t ss = (uint32_t)(h / plane);
        const uint32_t rem = (uint32_t)(h - (uint64_t)ss * plane);
        const uint32_t ms = rem / S, fs = rem - ms * S;
        const unsigned long long v = half[h];
        if (v == 0) continue;
        full[fs + (uint64_t)ms * S + (uint64_t)(ss + C) * plane] += v;
        if (ss != 0) full[(2 * C - fs) + (uint64_t)(2 * C - ms) * S + (uint64_t)(C - ss) * plane] += v;
    }
}

// ---------------------------------------------------------------------------
// AC_UW of sparse photon lists: both routes of Calculate_AC_UW_Mapped
// (IAC/AC1D.cpp:248-379).  The reference picks a route per frame: with fewer
// than 0.75 % of the detector's pixels hit ((float)n / (float)pixels < 0.0075f,
// :251-253) it loops on the host over k >= j (:254-293); otherwise it launches
// AutoCorr_sparseHL_AAV (IAC/kernel.cl:863-950, host side :295-379).
//
// Device route: every ordered pair of a frame, self pairs included, adds
// (uint64)(v_a * v_b * Mult) at bin floor(|q|/dq + 0.5) (nearest) or splits
// it over floor(|q|/dq) and the next bin (linear).  The two orders of a
// distinct pair give the same |q| and value, so each distinct pair adds twice
// its value.  Bins are taken modulo VecSize, which is what the reference's
// sub-histogram layout and index-modulo fold (IAC/AC1D.cpp:366-375) do to bins
// at or beyond VecSize.
//
// Host route: every unordered pair k >= j adds the float 2*(v_j*v_k)
// (nearest), or 2*((v_j*v_k)*(1-Sep)) and 2*((v_j*v_k)*Sep) (linear), to a
// double histogram of Size bins; the factor 2 also doubles the self pair.
// These floats are whole numbers for photon counts (nearest): those are summed
// in uint64, exactly, so the double totals equal the reference's sequential
// double sums bit for bit.  Any other value is summed with double atomics,
// whose order differs from the reference's loop by rounding only.
//
// The histograms live in shared memory for the whole launch; the work queue
// and the pair enumeration are the pair kernel's.  A tile belongs to one
// frame, so the route branch is uniform across the CTA.
// ---------------------------------------------------------------------------
// b % n without the division when b < n (bins past the histogram are rare)
__device__ __forceinline__ uint32_t wrap_bin(uint32_t b, uint32_t n)
{
    if (b >= n) b %= n;
    return b;
}

struct AC1DArgs {
    float maxq, dqdx;
    uint32_t vecsize;   // device-route bins (VecSize)
    uint32_t size;      // host-route bins (Shape.Size; 0 when no frame takes the host route)
    float det_pixels;   // (float) detector pixel count, for the route choice
    int route;          // -1: the reference's choice per frame, 0: host route, 1: device route
    unsigned long long *dev_out;  // vecsize words
    unsigned long long *int_out;  // size words: host-route whole-number values
    double *frac_out;             // size doubles: host-route other values
};

// shared-memory histograms of one CTA: 64-bit counters as split 32-bit words
// (shared_add_u64_split), host-route fractions as doubles
struct AC1DHist {
    uint32_t *dev_lo, *dev_hi;  // vecsize words each
    uint32_t *int_lo, *int_hi;  // size words each
    double *frac;               // size doubles
};

// host-route value v (>= 0) into bin b
__device__ __forceinline__ void host_route_add(const SparseArgs &a, const AC1DArgs &b, const AC1DHist &h,
                                               uint32_t bin, float v)
{
    if (bin >= b.size) {  // only for inconsistent MaxQ / dq; the reference writes out of bounds
        atomicAdd(&a.counters->out_of_mesh, 1ull);
        return;
    }
    if (v == 0.0f) return;
    if (v > 0.0f && v < 8388608.0f) {  // the usual case, without conversion-unit instructions
        const float t = __fadd_rz(v, 8388608.0f);  // 2^23 + floor(v)
        if (fsub(t, 8388608.0f) == v)
            shared_add_u64_split(h.int_lo, h.int_hi, bin, (unsigned long long)(uint32_t)(__float_as_int(t) - TWO23_BITS));
        else
            atomicAdd(&h.frac[bin], (double)v);
        return;
    }
    if (v == truncf(v) && v < 1.8e19f)
        shared_add_u64_split(h.int_lo, h.int_hi, bin, (unsigned long long)__float2ull_rz(v));
    else
        atomicAdd(&h.frac[bin], (double)v);
}

template <int INTERP>
__global__ void __launch_bounds__(256) ac1d_sparse_kernel(const SparseArgs a, const AC1DArgs b)
{
    extern __shared__ unsigned long long hist[];
    AC1DHist h;
    h.dev_lo = reinterpret_cast<uint32_t *>(hist);
    h.dev_hi = h.dev_lo + b.vecsize;
    h.int_lo = h.dev_hi + b.vecsize;
    h.int_hi = h.int_lo + b.size;
    h.frac = reinterpret_cast<double *>(hist + b.vecsize + b.size);
    __shared__ unsigned long long s_tile;
    __shared__ uint32_t s_frame;
    const uint32_t words = b.vecsize + 2 * b.size;
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) hist[i] = 0;  // 0 bits = +0.0
    const unsigned long long ntiles = a.tile_off[a.nframes];
    const uint32_t nthr = blockDim.x;
    const float maxq = b.maxq, dqdx = b.dqdx;
    for (;;) {
        if (threadIdx.x == 0) {
            const unsigned long long t = atomicAdd(a.queue, 1ull);
            s_tile = t;
            if (t < ntiles) {
                uint32_t lo = 0, hi = a.nframes;
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (a.tile_off[mid] <= t) lo = mid; else hi = mid;
                }
                s_frame = lo;
            }
        }
        __syncthreads();
        const unsigned long long t = s_tile;
        if (t >= ntiles) break;
        const uint32_t f = s_frame;
        const uint64_t base = a.offsets[f];
        const uint32_t n = (uint32_t)(a.offsets[f + 1] - base);
        const unsigned long long chunk = t - a.tile_off[f];
        const float4 *__restrict__ P = a.photons + base;
        // SHLsizeQuot < 0.0075f (IAC/AC1D.cpp:251-253), in the reference's float arithmetic
        const bool host =
            b.route == 0 || (b.route < 0 && __fdiv_rn(__uint2float_rn(n), b.det_pixels) < 0.0075f);
        if (chunk == 0)  // self pairs: q = 0, bin 0 (linear: bin 0 gets all of it, bin 1 nothing)
            for (uint32_t i = threadIdx.x; i < n; i += nthr) {
                const float w = P[i].w;
                if (host) {
                    host_route_add(a, b, h, 0, fmul(2.0f, fmul(w, w)));
                } else {
                    const double v = (double)w;
                    const unsigned long long u = d2u64(dmul(dmul(v, v), a.mult));
                    if (u) shared_add_u64_split(h.dev_lo, h.dev_hi, 0, u);
                }
            }
        const unsigned long long npairs = (unsigned long long)n * (n - 1) / 2;
        const unsigned long long p0 = chunk * a.tile_pairs;
        const unsigned long long p1 = min(npairs, p0 + a.tile_pairs);
        if (p0 + threadIdx.x < p1) {
            unsigned long long l = p0 + threadIdx.x;
            uint32_t d = (uint32_t)(l / n) + 1;
            uint32_t i = (uint32_t)(l - (unsigned long long)(d - 1) * n);
            const uint32_t dq = nthr / n, dr = nthr % n;
            for (; l < p1; l += nthr) {
                uint32_t j = i + d;
                if (j >= n) j -= n;
                const float4 A = P[min(i, j)], B = P[max(i, j)];
                const float dx = fsub(A.x, B.x), dy = fsub(A.y, B.y), dz = fsub(A.z, B.z);
                float q = __fsqrt_rn(fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz)));
                if (!(q > maxq)) {
                    q = __fdiv_rn(q, dqdx);
                    if (host) {
                        const float pv = fmul(A.w, B.w);
                        if (INTERP == 0) {
                            // (uint)floor(q + 0.5) in double, as floor(fl(q + 0.49999997f)) for q < 2^23
                            uint32_t iq;
                            floor_small(fadd(q, 0.49999997f), iq);
                            host_route_add(a, b, h, iq, fmul(2.0f, pv));
                        } else {
                            uint32_t iq;  // q = |q| / dq <= MaxQ / dq < 2^23
                            const float fq = floor_small(q, iq);
                            const float sep = fsub(q, fq);
                            host_route_add(a, b, h, iq, fmul(2.0f, fmul(pv, fsub(1.0f, sep))));
                            host_route_add(a, b, h, iq + 1, fmul(2.0f, fmul(pv, sep)));
                        }
                    } else {
                        const double val = dmul((double)A.w, (double)B.w);
                        if (INTERP == 0) {
                            uint32_t iq;  // (uint)floor(q + 0.5), as above
                            floor_small(fadd(q, 0.49999997f), iq);
                            const uint32_t sc = wrap_bin(iq, b.vecsize);
                            const unsigned long long w = d2u64(dmul(val, a.mult));
                            if (w) shared_add_u64_split(h.dev_lo, h.dev_hi, sc, 2ull * w);
                        } else {
                            uint32_t iq;
                            const float fq = floor_small(q, iq);
                            const double sep = (double)fsub(q, fq);
                            const unsigned long long w1 = d2u64(dmul(dmul(val, dsub(1.0, sep)), a.mult));
                            const unsigned long long w2 = d2u64(dmul(dmul(val, sep), a.mult));
                            if (w1) shared_add_u64_split(h.dev_lo, h.dev_hi, wrap_bin(iq, b.vecsize), 2ull * w1);
                            if (w2) shared_add_u64_split(h.dev_lo, h.dev_hi, wrap_bin(iq + 1, b.vecsize), 2ull * w2);
                        }
                    }
                }
                i += dr;
                d += dq;
                if (i >= n) {
                    i -= n;
                    d += 1;
                }
            }
        }
        __syncthreads();
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < b.vecsize; i += blockDim.x) {
        const unsigned long long v = split_word(h.dev_lo, h.dev_hi, i);
        if (v) atomicAdd(&b.dev_out[i], v);
    }
    for (uint32_t i = threadIdx.x; i < b.size; i += blockDim.x) {
        const unsigned long long v = split_word(h.int_lo, h.int_hi, i);
        if (v) atomicAdd(&b.int_out[i], v);
        if (h.frac[i] != 0.0) atomicAdd(&b.frac_out[i], h.frac[i]);
    }
}

// AC_UW[j] = dev[j] / Mult (j < VecSize) + int[j] + frac[j]
__global__ void ac1d_uw_finish_kernel(const unsigned long long *__restrict__ dev,
                                      const unsigned long long *__restrict__ in, const double *__restrict__ fr,
                                      uint32_t vecsize, uint32_t size, double mult, double *__restrict__ ac)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= size) return;
    double v = j < vecsize ? __ddiv_rn((double)dev[j], mult) : 0.0;
    v = dadd(v, (double)in[j]);
    ac[j] = dadd(v, fr[j]);
}

typedef void (*PairKernel)(SparseArgs);

static PairKernel pick_kernel(int dmap, int i1, int i2)
{
    if (!dmap) return i2 ? sparse_pairs_kernel<0, 0, 1> : sparse_pairs_kernel<0, 0, 0>;
    if (i1 == 0) return i2 ? sparse_pairs_kernel<1, 0, 1> : sparse_pairs_kernel<1, 0, 0>;
    return i2 ? sparse_pairs_kernel<1, 1, 1> : sparse_pairs_kernel<1, 1, 0>;
}

// Explicit settings win; otherwise the autotuner row of the nearest mesh edge;
// otherwise built-in defaults.
static iac_sparse_tuning effective_tuning(iac_ctx *ctx, uint32_t size_ab)
{
    iac_sparse_tuning t;
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        t = ctx->tuning;
        if (!ctx->tuning_table.empty() && size_ab >= 2) {
            const uint32_t edge = size_ab - 2;
            const iac_ctx::TuningRow *best = nullptr;
            for (const auto &r : ctx->tuning_table)
                if (!best || (r.edge > edge ? r.edge - edge : edge - r.edge) <
                                 (best->edge > edge ? best->edge - edge : edge - best->edge))
                    best = &r;
            if (t.tile_pairs == 0) t.tile_pairs = best->tile_pairs;
            if (t.block_threads == 0) t.block_threads = best->block_threads;
            if (t.ctas_per_sm == 0) t.ctas_per_sm = best->ctas_per_sm;
            if (t.cache_hints == 0) t.cache_hints = best->cache_hints;
        }
    }
    if (t.tile_pairs == 0) t.tile_pairs = 4096;
    if (t.block_threads == 0) t.block_threads = 256;
    if (t.ctas_per_sm == 0) t.ctas_per_sm = 8;
    return t;
}

// Largest float s with sqrtf(s) <= m: since IEEE sqrt is monotonic,
// sqrtf(x) > m exactly when x > s (host sqrtf is correctly rounded like the
// device's __fsqrt_rn).
static float sqrt_threshold(float m)
{
    if (!(m >= 0.0f) || std::isinf(m)) return m;
    float s = m * m;
    while (std::sqrt(s) > m) s = std::nextafter(s, 0.0f);
    for (;;) {
        const float n = std::nextafter(s, INFINITY);
        if (std::isinf(n) || std::sqrt(n) > m) break;
        s = n;
    }
    return s;
}

static iac_status check_params(const iac_sparse_params *p)
{
    IAC_REQUIRE(p != nullptr, "sparse params are NULL");
    const iac_mesh_shape &s = p->shape;
    IAC_REQUIRE(s.size_ab >= 5 && (s.size_ab % 2) == 1 && s.size_c == s.size_ab,
                "sparse pair mesh must be cubic with an odd edge (got %u x %u)", s.size_ab, s.size_c);
    IAC_REQUIRE(s.size_ab <= 1621, "mesh edge %u too large (at most 1621)", s.size_ab);
    IAC_REQUIRE(s.voxel_per_dq > 0, "Voxel_per_dq is 0");
    IAC_REQUIRE((double)s.max_q * s.voxel_per_dq <= 4194304.0,
                "MaxQ * Voxel_per_dq must be at most 2^22 voxels (got %g)", (double)s.max_q * s.voxel_per_dq);
    IAC_REQUIRE(p->interp_first == 0 || p->interp_first == 1, "interp_first must be 0 or 1");
    IAC_REQUIRE(p->interp_second == 0 || p->interp_second == 1, "interp_second must be 0 or 1");
    IAC_REQUIRE(p->multiplicator > 0, "multiplicator must be positive");
    return IAC_OK;
}

// Half-width R of the shared-memory box of voxels around q = 0 (ss <= R,
// |fs - C| <= R, |ms - C| <= R) that each CTA of the pair kernel accumulates
// privately and adds to the half mesh once, when it runs out of tiles.  Pair
// density peaks at q = 0: in a 201^3 mesh of the rotated workload the
// R = 10 box (4 851 voxels) takes 9 % of all updates, and without it those
// few hundred 128-byte lines are the most contended L2 atomic targets (one
// line takes about 4.5e9 atomic adds per second, the whole L2 about 1.9e11).
// R = IAC_PAIR_BOX_R (10: 38 KB per CTA) while ctas_per_sm boxes fit in
// 200 KB of the SM's shared memory, smaller beyond; at most C.
#ifndef IAC_PAIR_BOX_R
#define IAC_PAIR_BOX_R 10
#endif
static int pair_box_radius(int C, uint32_t ctas_per_sm)
{
    const size_t budget = (200u << 10) / std::max<uint32_t>(1, ctas_per_sm);
    int r = std::min(IAC_PAIR_BOX_R, C);
    while (r > 0 && sizeof(unsigned long long) * (size_t)(r + 1) * (2 * r + 1) * (2 * r + 1) > budget) r--;
    return r;
}

// Work-queue memory of one batch: tile table (nframes + 1), queue counter,
// per-frame small-count flags (nframes bytes).
struct QueueMem {
    unsigned long long *tile_off;
    unsigned long long *queue;
    unsigned char *flags;
};

// Planner, count check and pair kernel of one batch into the half mesh d_half.
static iac_status launch_pair_batch(iac_ctx *ctx, const float *d_photons, const uint64_t *d_off,
                                    const float *d_rot9, uint32_t nframes, const iac_sparse_params *p,
                                    const QueueMem &q, uint64_t *d_half, cudaStream_t s)
{
    const iac_sparse_tuning tun = effective_tuning(ctx, p->shape.size_ab);
    sparse_plan_kernel<<<1, PLAN_THREADS, 0, s>>>(d_off, nframes, tun.tile_pairs, q.tile_off, q.queue);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    const bool mult_small_int = p->multiplicator >= 1.0 && p->multiplicator <= 1024.0 &&
                                p->multiplicator == std::floor(p->multiplicator);
    unsigned char *flags = nullptr;
    if (mult_small_int && p->interp_second == 0 && !(p->double_map && p->interp_first == 1)) {
        const uint32_t blocks = (uint32_t)(((uint64_t)nframes * 32 + 255) / 256);
        sparse_count_check_kernel<<<blocks, 256, 0, s>>>(reinterpret_cast<const float4 *>(d_photons),
                                                         d_off, nframes, q.flags);
        IAC_LAUNCHED(ctx);
        IAC_CUDA(cudaGetLastError());
        flags = q.flags;
    }
    SparseArgs a;
    a.photons = reinterpret_cast<const float4 *>(d_photons);
    a.offsets = d_off;
    a.rot = d_rot9;
    a.tile_off = q.tile_off;
    a.half = reinterpret_cast<unsigned long long *>(d_half);
    a.queue = q.queue;
    a.counters = ctx->d_counters;
    a.nframes = nframes;
    a.tile_pairs = tun.tile_pairs;
    a.S = (int)p->shape.size_ab;
    a.C = (a.S - 1) / 2;
    a.half_ss = (a.S + 1) / 2;
    a.plane = (uint32_t)a.S * (uint32_t)a.S;
    a.maxq = p->shape.max_q;
    a.maxq2 = sqrt_threshold(p->shape.max_q);
    a.vpdq = (float)p->shape.voxel_per_dq;
    a.mult = p->multiplicator;
    a.mult_f = (float)p->multiplicator;
    a.small_counts = flags;
    a.cache_hints = tun.cache_hints == 1 ? 1 : 0;
    a.mesh_policy = 0;
    a.box_r = pair_box_radius(a.C, tun.ctas_per_sm);
    a.box_w = 2 * a.box_r + 1;
    a.box_base = 0;
    a.box_hi = 0;
    const size_t box_bytes = a.box_r ? sizeof(unsigned long long) * (a.box_r + 1) * a.box_w * a.box_w : 0;
    const PairKernel k = pick_kernel(p->double_map, p->interp_first, p->interp_second);
    if (box_bytes > (48u << 10))
        IAC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)box_bytes));
    k<<<ctx->sm_count * (int)tun.ctas_per_sm, tun.block_threads, box_bytes, s>>>(a);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}

// Planner and AC1D kernel of one batch (shared memory: both routes' histograms).
static iac_status launch_ac1d_batch(iac_ctx *ctx, const float *d_photons, const uint64_t *d_off,
                                    uint32_t nframes, int interp, double mult, const AC1DArgs &b, void *stream)
{
    DeviceGuard g(ctx->device);
    const iac_sparse_tuning tun = effective_tuning(ctx, 0);
    void *scratch = nullptr;
    const size_t table_bytes = ((sizeof(unsigned long long) * ((size_t)nframes + 1) + 127) / 128) * 128;
    iac_status st = stream_scratch(ctx, stream, SLOT_TILES, table_bytes + 128 + nframes, &scratch);
    if (st != IAC_OK) return st;
    unsigned long long *tile_off = (unsigned long long *)scratch;
    unsigned long long *queue = (unsigned long long *)((char *)scratch + table_bytes);
    cudaStream_t s = as_stream(stream);
    sparse_plan_kernel<<<1, PLAN_THREADS, 0, s>>>(d_off, nframes, tun.tile_pairs, tile_off, queue);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    SparseArgs a{};
    a.photons = reinterpret_cast<const float4 *>(d_photons);
    a.offsets = d_off;
    a.tile_off = tile_off;
    a.queue = queue;
    a.counters = ctx->d_counters;
    a.nframes = nframes;
    a.tile_pairs = tun.tile_pairs;
    a.mult = mult;
    const size_t smem = sizeof(unsigned long long) * ((size_t)b.vecsize + 2 * (size_t)b.size);
    auto k = interp == 0 ? ac1d_sparse_kernel<0> : ac1d_sparse_kernel<1>;
    IAC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // as many persistent CTAs as fit: four per SM, fewer when the histograms are large
    const int per_sm = (int)std::max<size_t>(1, std::min<size_t>(4, (200u << 10) / std::max<size_t>(smem, 1)));
    k<<<ctx->sm_count * per_sm, 256, smem, s>>>(a, b);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}

}  // namespace iac

using namespace iac;

extern "C" {

iac_status iac_sparse_set_tuning(iac_ctx *ctx, const iac_sparse_tuning *t)
{
    IAC_REQUIRE(ctx && t, "iac_sparse_set_tuning: NULL argument");
    IAC_REQUIRE(t->block_threads == 0 || (t->block_threads % 32 == 0 && t->block_threads <= 256 &&
                                          t->block_threads >= 64),
                "block_threads must be a multiple of 32 in [64, 256]");
    IAC_REQUIRE(t->tile_pairs == 0 || t->tile_pairs >= 64, "tile_pairs must be >= 64");
    IAC_REQUIRE(t->ctas_per_sm <= 32, "ctas_per_sm must be <= 32");
    IAC_REQUIRE(t->cache_hints <= 2, "cache_hints must be 0 (table), 1 (on) or 2 (off)");
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->tuning = *t;
    return IAC_OK;
}

iac_status iac_sparse_get_tuning(iac_ctx *ctx, uint32_t size_ab, iac_sparse_tuning *t)
{
    IAC_REQUIRE(ctx && t, "iac_sparse_get_tuning: NULL argument");
    *t = effective_tuning(ctx, size_ab);
    return IAC_OK;
}

iac_status iac_sparse_ac_batch(iac_ctx *ctx, const float *d_photons, const uint64_t *d_off,
                               const float *d_rot9, uint32_t nframes, const iac_sparse_params *p,
                               uint64_t *d_half, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx != nullptr, "iac_sparse_ac_batch: ctx is NULL");
    iac_status st = check_params(p);
    if (st != IAC_OK) return st;
    if (nframes == 0) return IAC_OK;
    IAC_REQUIRE(d_photons && d_off && d_rot9 && d_half, "iac_sparse_ac_batch: NULL pointer");
    IAC_REQUIRE((reinterpret_cast<uintptr_t>(d_photons) & 15) == 0,
                "photon array must be 16-byte aligned (float4 per photon)");
    DeviceGuard g(ctx->device);
    void *scratch = nullptr;
    const size_t table_bytes = ((sizeof(unsigned long long) * ((size_t)nframes + 1) + 127) / 128) * 128;
    st = stream_scratch(ctx, stream, SLOT_TILES, table_bytes + 128 + nframes, &scratch);
    if (st != IAC_OK) return st;
    const QueueMem q{(unsigned long long *)scratch, (unsigned long long *)((char *)scratch + table_bytes),
                     (unsigned char *)scratch + table_bytes + 128};
    return launch_pair_batch(ctx, d_photons, d_off, d_rot9, nframes, p, q, d_half, as_stream(stream));
}

iac_status iac_ac1d_sparse_batch(iac_ctx *ctx, const float *d_photons, const uint64_t *d_off,
                                 uint32_t nframes, float max_q, float dqdx, int interp,
                                 double mult, uint64_t *d_hist, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx != nullptr, "iac_ac1d_sparse_batch: ctx is NULL");
    IAC_REQUIRE(interp == 0 || interp == 1, "interpolation must be 0 or 1");
    IAC_REQUIRE(dqdx > 0 && max_q > 0, "iac_ac1d_sparse_batch: MaxQ and dq must be positive");
    IAC_REQUIRE(mult > 0, "multiplicator must be positive");
    const uint32_t vecsize = iac_ac1d_vecsize(max_q, dqdx);
    IAC_REQUIRE(vecsize >= 1 && vecsize <= 24576, "VecSize %u out of range [1, 24576]", vecsize);
    if (nframes == 0) return IAC_OK;
    IAC_REQUIRE(d_photons && d_off && d_hist, "iac_ac1d_sparse_batch: NULL pointer");
    IAC_REQUIRE((reinterpret_cast<uintptr_t>(d_photons) & 15) == 0,
                "photon array must be 16-byte aligned (float4 per photon)");
    AC1DArgs b{};
    b.maxq = max_q;
    b.dqdx = dqdx;
    b.vecsize = vecsize;
    b.size = 0;
    b.det_pixels = 1.0f;
    b.route = 1;
    b.dev_out = (unsigned long long *)d_hist;
    return launch_ac1d_batch(ctx, d_photons, d_off, nframes, interp, mult, b, stream);
}

uint64_t iac_ac1d_uw_words(const iac_ac1d_shape *sh)
{
    if (!sh || !(sh->dq_per_step > 0) || !(sh->max_q > 0)) return 0;
    return (uint64_t)iac_ac1d_vecsize(sh->max_q, sh->dq_per_step) + 2ull * sh->size;
}

iac_status iac_ac1d_uw_batch(iac_ctx *ctx, const float *d_photons, const uint64_t *d_off, uint32_t nframes,
                             uint64_t detector_pixels, const iac_ac1d_shape *sh, int interp, int route,
                             uint64_t *d_acc, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx != nullptr && sh != nullptr, "iac_ac1d_uw_batch: NULL argument");
    IAC_REQUIRE(interp == 0 || interp == 1, "interpolation must be 0 or 1");
    IAC_REQUIRE(route >= -1 && route <= 1, "route must be -1 (per frame), 0 (host) or 1 (device)");
    IAC_REQUIRE(sh->dq_per_step > 0 && sh->max_q > 0, "iac_ac1d_uw_batch: MaxQ and dq must be positive");
    IAC_REQUIRE(detector_pixels > 0 && detector_pixels < (1ull << 32),
                "iac_ac1d_uw_batch: detector pixel count %llu out of range", (unsigned long long)detector_pixels);
    const uint32_t vecsize = iac_ac1d_vecsize(sh->max_q, sh->dq_per_step);
    IAC_REQUIRE(sh->size >= 3 && vecsize >= 1, "AC1D size %u too small", sh->size);
    IAC_REQUIRE((uint64_t)vecsize + 2ull * sh->size <= 24576,
                "AC1D size %u too large: VecSize + 2 Size must be at most 24576 (shared-memory histograms)",
                sh->size);
    if (nframes == 0) return IAC_OK;
    IAC_REQUIRE(d_photons && d_off && d_acc, "iac_ac1d_uw_batch: NULL pointer");
    IAC_REQUIRE((reinterpret_cast<uintptr_t>(d_photons) & 15) == 0,
                "photon array must be 16-byte aligned (float4 per photon)");
    IAC_REQUIRE((reinterpret_cast<uintptr_t>(d_acc) & 7) == 0, "accumulator must be 8-byte aligned");
    AC1DArgs b{};
    b.maxq = sh->max_q;
    b.dqdx = sh->dq_per_step;
    b.vecsize = vecsize;
    b.size = sh->size;
    b.det_pixels = (float)detector_pixels;
    b.route = route;
    b.dev_out = (unsigned long long *)d_acc;
    b.int_out = b.dev_out + vecsize;
    b.frac_out = reinterpret_cast<double *>(b.int_out + sh->size);
    return launch_ac1d_batch(ctx, d_photons, d_off, nframes, interp, 100.0, b, stream);
}

iac_status iac_ac1d_uw_finish(iac_ctx *ctx, const uint64_t *d_acc, const iac_ac1d_shape *sh, double *d_ac_uw,
                              void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx && sh && d_acc && d_ac_uw, "iac_ac1d_uw_finish: NULL argument");
    IAC_REQUIRE(sh->dq_per_step > 0 && sh->max_q > 0 && sh->size >= 3, "iac_ac1d_uw_finish: bad shape");
    const uint32_t vecsize = iac_ac1d_vecsize(sh->max_q, sh->dq_per_step);
    DeviceGuard g(ctx->device);
    const unsigned long long *dev = (const unsigned long long *)d_acc;
    ac1d_uw_finish_kernel<<<(sh->size + 255) / 256, 256, 0, as_stream(stream)>>>(
        dev, dev + vecsize, reinterpret_cast<const double *>(dev + vecsize + sh->size), vecsize, sh->size, 100.0,
        d_ac_uw);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}

uint32_t iac_ac1d_vecsize(float max_q, float dqdx)
{
    return (uint32_t)((int)std::ceil(max_q / dqdx) - 1);
}

iac_status iac_sparse_fold(iac_ctx *ctx, const uint64_t *d_half, uint32_t S, uint64_t *d_full,
                           void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx && d_half && d_full, "iac_sparse_fold: NULL argument");
    IAC_REQUIRE(S >= 3 && (S % 2) == 1 && S <= 2047, "iac_sparse_fold: bad mesh edge %u", S);
    DeviceGuard g(ctx->device);
    sparse_fold_kernel<<<ctx->sm_count * 4, 256, 0, as_stream(stream)>>>(
        reinterpret_cast<const unsigned long long *>(d_half), S,
        reinterpret_cast<unsigned long long *>(d_full));
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}

}  // extern "C"

namespace iac {

// Streams and events of the host-buffer entry points, created on first use.
static iac_status host_streams(iac_ctx *ctx)
{
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!ctx->host_stream) IAC_CUDA(cudaStreamCreateWithFlags(&ctx->host_stream, cudaStreamNonBlocking));
    if (!ctx->copy_stream) IAC_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    if (!ctx->copy_events[0])
        for (auto &e : ctx->copy_events) IAC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    if (!ctx->staging_free[0])
        for (auto &e : ctx->staging_free) IAC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return IAC_OK;
}

// Host photon lists -> device staging (scratch of `key`) -> pair kernel into
// d_half on stream s.  Two staging sets alternate between calls, so a call's
// copies overlap the previous call's binning; each set is reused only after
// the binning that read it (staging_free).  When the previous call's binning
// is still running (a run of consecutive calls) the whole batch is copied
// behind it and binned in one launch.  Otherwise the frames are cut into
// chunks by photon count, chunk k+1 copied on the copy stream while chunk k
// is binned; binning is slower than the copy, so only the first chunk's copy
// is exposed: it is made a quarter of the others (1/29 of the photons for 8
// chunks).  Every chunk has its own rebased offsets so it is an independent
// batch.
static iac_status stage_and_bin(iac_ctx *ctx, const float *h_photons, const uint64_t *h_off, const float *h_rot9,
                                uint32_t nframes, const iac_sparse_params *p, uint64_t *d_half, cudaStream_t s,
                                void *key)
{
    iac_status st;
    cudaStream_t cs = ctx->copy_stream;
    const int set = ctx->staging_set;
    ctx->staging_set ^= 1;
    const bool behind = cudaEventQuery(ctx->staging_free[set ^ 1]) == cudaErrorNotReady;
    const uint64_t o0 = h_off[0];
    const uint64_t nph = h_off[nframes] - o0;
    const uint32_t nchunks =
        behind ? 1u : std::max<uint32_t>(1, std::min<uint32_t>(IAC_COPY_CHUNKS, nframes / 64));
    std::vector<uint32_t> cut(nchunks + 1, 0);
    cut[nchunks] = nframes;
    const uint64_t parts = 4 * (uint64_t)nchunks - 3;  // chunk 0: 1 part, the others 4
    for (uint32_t k = 1; k < nchunks; k++) {
        const uint64_t target = o0 + nph * (4 * (uint64_t)k - 3) / parts;
        cut[k] = (uint32_t)(std::lower_bound(h_off, h_off + nframes + 1, target) - h_off);
        cut[k] = std::max(cut[k], cut[k - 1]);
    }
    void *d_ph, *d_off, *d_rot;
    const int sp = set ? SLOT_PHOTONS2 : SLOT_PHOTONS, so = set ? SLOT_OFFSETS2 : SLOT_OFFSETS,
              sr = set ? SLOT_ROT2 : SLOT_ROT;
    if ((st = stream_scratch(ctx, key, sp, 16 * nph + 16, &d_ph)) != IAC_OK) return st;
    if ((st = stream_scratch(ctx, key, so, 8 * ((size_t)nframes + IAC_COPY_CHUNKS + 1), &d_off)) != IAC_OK)
        return st;
    if ((st = stream_scratch(ctx, key, sr, 36 * (size_t)nframes, &d_rot)) != IAC_OK) return st;
    std::vector<uint64_t> off((size_t)nframes + nchunks);
    size_t w = 0;
    std::vector<size_t> off_pos(nchunks);
    for (uint32_t k = 0; k < nchunks; k++) {
        off_pos[k] = w;
        for (uint32_t f = cut[k]; f <= cut[k + 1]; f++) off[w++] = h_off[f] - h_off[cut[k]];
    }
    {   // size the work-queue scratch for the largest chunk now: growing it
        // between chunk launches would synchronise the device
        void *t = nullptr;
        const size_t tb = ((sizeof(unsigned long long) * ((size_t)nframes + 1) + 127) / 128) * 128;
        if ((st = stream_scratch(ctx, key, SLOT_TILES, tb + 128 + nframes, &t)) != IAC_OK) return st;
    }
    // the binning that last read this staging set is done before it is overwritten
    IAC_CUDA(cudaStreamWaitEvent(cs, ctx->staging_free[set], 0));
    IAC_CUDA(cudaMemcpyAsync(d_off, off.data(), 8 * w, cudaMemcpyHostToDevice, cs));
    for (uint32_t k = 0; k < nchunks; k++) {
        const uint32_t f0 = cut[k], f1 = cut[k + 1];
        const uint64_t p0 = h_off[f0] - o0, p1 = h_off[f1] - o0;
        if (p1 > p0)
            IAC_CUDA(cudaMemcpyAsync((char *)d_ph + 16 * p0, h_photons + 4 * (o0 + p0), 16 * (p1 - p0),
                                     cudaMemcpyHostToDevice, cs));
        if (f1 > f0)
            IAC_CUDA(cudaMemcpyAsync((char *)d_rot + 36 * (size_t)f0, h_rot9 + 9 * (size_t)f0,
                                     36 * (size_t)(f1 - f0), cudaMemcpyHostToDevice, cs));
        IAC_CUDA(cudaEventRecord(ctx->copy_events[k], cs));
        IAC_CUDA(cudaStreamWaitEvent(s, ctx->copy_events[k], 0));
        if (f1 > f0) {
            st = iac_sparse_ac_batch(ctx, (const float *)((char *)d_ph + 16 * p0),
                                     (const uint64_t *)d_off + off_pos[k], (const float *)d_rot + 9 * (size_t)f0,
                                     f1 - f0, p, d_half, (void *)s);
            if (st != IAC_OK) return st;
        }
    }
    IAC_CUDA(cudaEventRecord(ctx->staging_free[set], s));
    return IAC_OK;
}

}  // namespace iac

extern "C" {

iac_status iac_sparse_ac_frames_host(iac_ctx *ctx, const float *h_photons,
                                     const uint64_t *h_off, const float *h_rot9, uint32_t nframes,
                                     const iac_sparse_params *p, uint64_t *h_full)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx != nullptr, "iac_sparse_ac_frames_host: ctx is NULL");
    iac_status st = check_params(p);
    if (st != IAC_OK) return st;
    IAC_REQUIRE(h_off && h_full, "iac_sparse_ac_frames_host: NULL pointer");
    if (nframes == 0) return IAC_OK;
    IAC_REQUIRE(h_photons && h_rot9, "iac_sparse_ac_frames_host: NULL pointer");
    DeviceGuard g(ctx->device);
    std::lock_guard<std::mutex> hl(ctx->host_mu);
    if ((st = host_streams(ctx)) != IAC_OK) return st;
    cudaStream_t s = ctx->host_stream, cs = ctx->copy_stream;
    void *key = (void *)s;
    const uint32_t S = p->shape.size_ab;
    const size_t half_b = sizeof(uint64_t) * iac_half_mesh_words(S);
    const size_t full_b = sizeof(uint64_t) * iac_full_mesh_words(S);
    void *d_half, *d_full;
    if ((st = stream_scratch(ctx, key, SLOT_HALF, half_b, &d_half)) != IAC_OK) return st;
    if ((st = stream_scratch(ctx, key, SLOT_FULL, full_b, &d_full)) != IAC_OK) return st;
    IAC_CUDA(cudaMemsetAsync(d_half, 0, half_b, s));
    if ((st = stage_and_bin(ctx, h_photons, h_off, h_rot9, nframes, p, (uint64_t *)d_half, s, key)) != IAC_OK)
        return st;
    // the mesh the caller holds, uploaded behind the photon stream
    const uint32_t ev = IAC_COPY_CHUNKS;
    IAC_CUDA(cudaMemcpyAsync(d_full, h_full, full_b, cudaMemcpyHostToDevice, cs));
    IAC_CUDA(cudaEventRecord(ctx->copy_events[ev], cs));
    IAC_CUDA(cudaStreamWaitEvent(s, ctx->copy_events[ev], 0));
    st = iac_sparse_fold(ctx, (const uint64_t *)d_half, S, (uint64_t *)d_full, key);
    if (st != IAC_OK) return st;
    IAC_CUDA(cudaMemcpyAsync(h_full, d_full, full_b, cudaMemcpyDeviceToHost, s));
    IAC_CUDA(cudaStreamSynchronize(s));
    return IAC_OK;
}

iac_status iac_sparse_ac_frames_host_to_device(iac_ctx *ctx, const float *h_photons, const uint64_t *h_off,
                                               const float *h_rot9, uint32_t nframes, const iac_sparse_params *p,
                                               uint64_t *d_half, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx != nullptr, "iac_sparse_ac_frames_host_to_device: ctx is NULL");
    iac_status st = check_params(p);
    if (st != IAC_OK) return st;
    IAC_REQUIRE(h_off && d_half, "iac_sparse_ac_frames_host_to_device: NULL pointer");
    if (nframes == 0) return IAC_OK;
    IAC_REQUIRE(h_photons && h_rot9, "iac_sparse_ac_frames_host_to_device: NULL pointer");
    DeviceGuard g(ctx->device);
    std::lock_guard<std::mutex> hl(ctx->host_mu);
    if ((st = host_streams(ctx)) != IAC_OK) return st;
    cudaStream_t s = as_stream(stream);
    if ((st = stage_and_bin(ctx, h_photons, h_off, h_rot9, nframes, p, d_half, s, stream)) != IAC_OK) return st;
    // the host buffers have been read once the copies are done; binning goes on
    IAC_CUDA(cudaStreamSynchronize(ctx->copy_stream));
    return IAC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free variant of iac_sparse_ac_batch.
//
// Some callers may not allocate device memory once they are running: a
// detector acquisition loop that cannot absorb the device-wide
// synchronisation and unbounded latency a cudaMalloc/cudaFree can cause, or a
// host framework that hands out all device memory from its own pool and
// forbids allocations behind its back.  iac_sparse_ac_batch grows a per-stream
// scratch buffer on first use; this entry point instead keeps the same work
// queue (tile table, queue counter, per-frame flags) in a fixed array of
// device memory that is part of the loaded library, so it never allocates.
//
// The array's name in host code only stands in for the symbol; the kernels
// need its device address, which cudaGetSymbolAddress gives.  The context
// looks it up once, when it is created (iac_ctx_create, with its device
// current: the step that may load the library's device code and place the
// array on that device), and keeps it; the entry point itself only reads it.
// A context does not outlive a reset of its device (cudaDeviceReset ends every
// context's device state), so the kept address is never stale while the
// context is usable.  The array is shared by every call on the device and
// keeps the previous call's contents: the planner kernel rewrites the whole
// tile table and resets the queue counter before the pair kernel reads them,
// so nothing has to be cleared from the host, but two calls running on the
// GPU at the same time (e.g. on two streams) would overwrite each other's
// queue.
// ---------------------------------------------------------------------------
namespace iac {

constexpr uint32_t STATIC_MAX_FRAMES = 200000;
constexpr size_t STATIC_TABLE_BYTES =
    ((sizeof(unsigned long long) * ((size_t)STATIC_MAX_FRAMES + 1) + 255) / 256) * 256;
constexpr size_t STATIC_QUEUE_BYTES = 256;
constexpr size_t STATIC_SCRATCH_BYTES = STATIC_TABLE_BYTES + STATIC_QUEUE_BYTES + STATIC_MAX_FRAMES;

static __device__ __align__(256) unsigned char g_sparse_static_scratch[STATIC_SCRATCH_BYTES];

iac_status static_scratch_setup(iac_ctx *ctx)
{
    DeviceGuard g(ctx->device);
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sparse_static_scratch);
    if (e != cudaSuccess || !p) {
        set_error("cudaGetSymbolAddress of the fixed scratch failed on device %d: %s", ctx->device,
                  cudaGetErrorString(e));
        return IAC_ERR_CUDA;
    }
    ctx->static_scratch = p;
    return IAC_OK;
}

}  // namespace iac

extern "C" iac_status iac_sparse_ac_batch_static(iac_ctx *ctx, const float *d_photons,
                                                 const uint64_t *d_off, const float *d_rot9,
                                                 uint32_t nframes, const iac_sparse_params *p,
                                                 uint64_t *d_half, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx != nullptr, "iac_sparse_ac_batch_static: ctx is NULL");
    iac_status st = check_params(p);
    if (st != IAC_OK) return st;
    if (nframes == 0) return IAC_OK;
    IAC_REQUIRE(d_photons && d_off && d_rot9 && d_half, "iac_sparse_ac_batch_static: NULL pointer");
    IAC_REQUIRE((reinterpret_cast<uintptr_t>(d_photons) & 15) == 0,
                "photon array must be 16-byte aligned (float4 per photon)");
    IAC_REQUIRE(nframes <= STATIC_MAX_FRAMES,
                "iac_sparse_ac_batch_static: %u frames requested; its fixed scratch holds the work "
                "queue of at most %u frames per call (split the batch or use iac_sparse_ac_batch)",
                nframes, STATIC_MAX_FRAMES);
    IAC_REQUIRE(ctx->static_scratch != nullptr, "iac_sparse_ac_batch_static: the context has no fixed scratch");
    DeviceGuard g(ctx->device);
    char *base = (char *)ctx->static_scratch;
    const QueueMem q{(unsigned long long *)base, (unsigned long long *)(base + STATIC_TABLE_BYTES),
                     (unsigned char *)base + STATIC_TABLE_BYTES + STATIC_QUEUE_BYTES};
    return launch_pair_batch(ctx, d_photons, d_off, d_rot9, nframes, p, q, d_half, as_stream(stream));
}
