// dense_pairs.cu -- (b) dense mean-intensity C(q) on the small mesh and
// (c) the AC1D |q| histogram of the mean intensity.
//
// Replaces AutoCorr_CQ_small (IAC/kernel.cl:27-184, host
// Detector::AutoCorrelate_CofQ_SmallMesh, IAC/Detector.cpp:1184-1315) and
// AutoCorr_CQ_AV (IAC/kernel.cl:656-764, host AC1D::Calculate_CQ,
// IAC/AC1D.cpp:61-195).
//
// Both reference kernels visit every ordered pixel pair (ind, i), self pairs
// included.  The pair (i, ind) is the point reflection of (ind, i): q changes
// sign exactly, the value I_ind*I_i is the same float, and round()/floor()
// based binning is reflected exactly (nearest: round(-x) = -round(x); linear:
// the corner weights 1 - (x - floor x) of -x are the reflected weights of x,
// bit for bit).  So each unordered pair is evaluated once and its mesh
// contribution is added at the voxel and at its reflection through the mesh
// centre; for |q| the two orders are identical and the bin gets twice the
// value.  Self pairs (q = 0) are added once at the centre.
//
// Work decomposition.  Pixels are cut into tiles of 256: 16 x 16 patches of
// the detector when its row length is given, else 256 consecutive pixels.
// A persistent CTA pops tile pairs (P <= Q) from a queue: thread t owns pixel
// t of tile P and walks the TILE pixels of Q, staged in shared memory as float4
// (k, I).  Tile pairs whose k bounding boxes are farther apart than MaxQ are
// skipped whole.  Contributions are accumulated per thread while consecutive
// pixels of Q fall into the same voxel (row-adjacent pixels move q by a
// fraction of a voxel), then added to a shared-memory window covering the
// tile pair's q range, which is flushed to the global mesh (voxel and
// reflection) once per tile pair.  Tile pairs whose window would not fit fall
// back to global atomics.  The AC1D histogram lives in shared memory for the
// whole launch and is flushed once per CTA.
//
// All FP32 operations are the reference's, in its order, without FMA
// contraction; values are (uint64)(double(I_a*I_b) * Mult) per pair as the
// reference's casts do, so the integer meshes are bit-identical.
#include <algorithm>
#include <cmath>

#include "iac_internal.cuh"

namespace iac {

constexpr int DTILE = 256;        // pixels per tile == threads per CTA
constexpr int WINDOW_WORDS = 2048;  // shared-memory window: 2048 split 64-bit counters (16 KB)

struct DenseArgs {
    const float *__restrict__ I;
    const float *__restrict__ K;     // 3 floats per pixel
    const float4 *__restrict__ box;  // per tile: min (x,y,z), max (x,y,z) as 2 float4
    unsigned long long *__restrict__ out;
    unsigned long long *queue;
    DeviceCounters *counters;
    uint64_t npix;
    uint32_t ntiles;
    unsigned long long npairs;  // tile pairs
    uint32_t part, nparts;      // this launch takes the tile pairs p with p % nparts == part
    uint32_t nx, ny, ptx;       // 2D patch tiling: row length, rows, patches per row (nx = 0: linear)
    uint32_t mult_int;          // Multiplicator as an integer below 2^29, else 0
    int key_ok;                 // |round(q * Voxel_per_dq)| < 512 for every pair within MaxQ
    float maxq, maxq2;
    float vpdq;
    double mult;
    // C(q) small mesh
    int ab, sc, cab, cc;  // sizes and centres
    int ka, kb, kc;       // q axis on mesh fs / ms / ss
    // AC1D
    uint32_t hsize;
    float dq;
};

// tile-pair index -> (P, Q): first the ntiles diagonal pairs, then the
// circulant walk over distinct pairs (d = l / T + 1, P = l % T, Q = P + d mod T)
__device__ __forceinline__ void decode_tile_pair(unsigned long long p, uint32_t T, uint32_t &P,
                                                 uint32_t &Q)
{
    if (p < T) {
        P = Q = (uint32_t)p;
        return;
    }
    const unsigned long long l = p - T;
    const uint32_t d = (uint32_t)(l / T) + 1;
    P = (uint32_t)(l % T);
    Q = P + d;
    if (Q >= T) Q -= T;
}

// Pixel of slot j (0..255) of tile t.  With the row length known the tiles
// are 16 x 16 pixel patches, whose pair differences cover a few voxels, so the
// shared-memory window of a tile pair stays small; otherwise 256 consecutive
// pixels.  Returns npix for a slot outside the detector.
__device__ __forceinline__ uint64_t tile_pixel(const DenseArgs &a, uint32_t t, uint32_t j)
{
    if (a.nx) {
        const uint32_t py = t / a.ptx, px = t - py * a.ptx;
        const uint32_t y = py * 16 + (j >> 4), x = px * 16 + (j & 15);
        return (y < a.ny && x < a.nx) ? (uint64_t)y * a.nx + x : a.npix;
    }
    const uint64_t i = (uint64_t)t * DTILE + j;
    return i < a.npix ? i : a.npix;
}

// (uint64)((double)p * M) for finite p >= 0 and an integer M < 2^29: the double
// product of a 24-bit mantissa and M is exact, so the cast is the floor of the
// exact product, formed here in integers.
__device__ __forceinline__ unsigned long long scaled_floor(float p, uint32_t M)
{
    const uint32_t b = __float_as_uint(p);
    const int e = (int)((b >> 23) & 0xff);
    const uint64_t m = (b & 0x7fffffu) | (e ? 0x800000u : 0u);
    const int sh = (e ? e : 1) - 150;  // p = m * 2^sh
    const uint64_t prod = m * (uint64_t)M;
    if (sh >= 0) return prod << sh;
    return sh <= -64 ? 0ull : (prod >> (-sh));
}

__global__ void tile_box_kernel(const DenseArgs a, float4 *__restrict__ box)
{
    const uint32_t t = blockIdx.x;
    const uint64_t i = tile_pixel(a, t, threadIdx.x);
    const float *__restrict__ K = a.K;
    const float *__restrict__ I = a.I;
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    float imax = 0.0f;  // largest |I| of the tile (NaN propagates: the tile then takes no fast path)
    if (i < a.npix && I[i] != 0.0f) {  // zero-intensity pixels never contribute
#pragma unroll
        for (int d = 0; d < 3; d++) mn[d] = mx[d] = K[3 * i + d];
        imax = fabsf(I[i]);
        if (imax != imax) imax = INFINITY;
    }
#pragma unroll
    for (int d = 0; d < 3; d++)
        for (int o = 16; o; o >>= 1) {
            mn[d] = fminf(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
            mx[d] = fmaxf(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
        }
    for (int o = 16; o; o >>= 1) imax = fmaxf(imax, __shfl_xor_sync(0xffffffffu, imax, o));
    __shared__ float s[7][DTILE / 32];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        for (int d = 0; d < 3; d++) {
            s[d][w] = mn[d];
            s[3 + d][w] = mx[d];
        }
        s[6][w] = imax;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float r[7];
        for (int d = 0; d < 7; d++) {
            r[d] = s[d][0];
            for (int j = 1; j < DTILE / 32; j++) r[d] = d < 3 ? fminf(r[d], s[d][j]) : fmaxf(r[d], s[d][j]);
        }
        box[2 * t] = make_float4(r[0], r[1], r[2], r[6]);
        box[2 * t + 1] = make_float4(r[3], r[4], r[5], 0.f);
    }
}

// lower bound of |k_a - k_b| over two boxes, inflated by a relative margin
__device__ __forceinline__ bool boxes_beyond(const float4 a0, const float4 a1, const float4 b0,
                                             const float4 b1, float maxq)
{
    const float gx = fmaxf(0.f, fmaxf(a0.x - b1.x, b0.x - a1.x));
    const float gy = fmaxf(0.f, fmaxf(a0.y - b1.y, b0.y - a1.y));
    const float gz = fmaxf(0.f, fmaxf(a0.z - b1.z, b0.z - a1.z));
    if (!(a0.x <= a1.x) || !(b0.x <= b1.x)) return true;  // an empty tile
    return sqrtf(gx * gx + gy * gy + gz * gz) > maxq * 1.0001f + 1e-6f;
}

__device__ __forceinline__ float pick(float x, float y, float z, int axis)
{
    return axis == 0 ? x : (axis == 1 ? y : z);
}

// --------------------------------------------------------------------------
// C(q) small mesh
// --------------------------------------------------------------------------
struct Window {
    int lo[3];  // first voxel (fs, ms, ss) of the window
    int dim[3];
    bool on;
};

__device__ __forceinline__ void global_put_pair(const DenseArgs &a, int fs, int ms, int ss,
                                                unsigned long long v)
{
    if (v == 0) return;
    if ((unsigned)fs >= (unsigned)a.ab || (unsigned)ms >= (unsigned)a.ab ||
        (unsigned)ss >= (unsigned)a.sc) {
        atomicAdd(&a.counters->out_of_mesh, 1ull);
    } else {
        atomicAdd(&a.out[(uint64_t)fs + (uint64_t)ms * a.ab + (uint64_t)ss * a.ab * a.ab], v);
    }
    const int rf = 2 * a.cab - fs, rm = 2 * a.cab - ms, rs = 2 * a.cc - ss;
    if ((unsigned)rf >= (unsigned)a.ab || (unsigned)rm >= (unsigned)a.ab ||
        (unsigned)rs >= (unsigned)a.sc) {
        atomicAdd(&a.counters->out_of_mesh, 1ull);
    } else {
        atomicAdd(&a.out[(uint64_t)rf + (uint64_t)rm * a.ab + (uint64_t)rs * a.ab * a.ab], v);
    }
}

__device__ __forceinline__ void put(const DenseArgs &a, const Window &w, uint32_t *win,
                                    int fs, int ms, int ss, unsigned long long v)
{
    if (v == 0) return;
    const int x = fs - w.lo[0], y = ms - w.lo[1], z = ss - w.lo[2];
    if (w.on && (unsigned)x < (unsigned)w.dim[0] && (unsigned)y < (unsigned)w.dim[1] &&
        (unsigned)z < (unsigned)w.dim[2])
        shared_add_u64_split(win, win + WINDOW_WORDS, x + w.dim[0] * (y + w.dim[1] * z), v);
    else
        global_put_pair(a, fs, ms, ss, v);
}

// round half away from zero as an int: (int)trunc(x + copysign(0.5 - 2^-25, x)).
// The FP32 sum is correctly rounded and never reaches the next integer unless
// x is at or past the half, so this equals round(x) for every |x| < 2^23
// (checked exhaustively against roundf over all such floats).
__device__ __forceinline__ int round_half_away(float x)
{
    return __float2int_rz(fadd(x, copysignf(0.49999997f, x)));
}

// component of (x, y, z) on axis K (0..2), or the runtime axis k when K < 0
template <int K>
__device__ __forceinline__ float axis(float x, float y, float z, int k)
{
    if (K == 0) return x;
    if (K == 1) return y;
    if (K == 2) return z;
    return pick(x, y, z, k);
}

// the pairs (own pixel, staged pixels j0..TILE-1): the exact reference
// arithmetic, per-thread run-length accumulation of consecutive pairs that
// land in the same voxel.  KA/KB/KC: axis of q on mesh fs/ms/ss (-1: runtime).
// CHECK: apply the per-pair MaxQ test (skipped when the two tiles' bounding
// boxes are entirely within MaxQ, where every pair passes it).
template <int INTERP, int KA, int KB, int KC, bool CHECK>
__device__ __forceinline__ void cq_pairs(const DenseArgs &a, const Window &w, uint32_t *win,
                                         const float4 *sq, int j0, float k0, float k1, float k2, float Ia)
{
    int cur_f = 0, cur_m = 0, cur_s = 0;
    unsigned long long acc[INTERP ? 8 : 1];
#pragma unroll
    for (int c = 0; c < (INTERP ? 8 : 1); c++) acc[c] = 0;
    bool have = false;
    for (int j = j0; j < DTILE; j++) {
        const float4 b = sq[j];
        const float pv = fmul(Ia, b.w);  // (double)(I_a*I_b) < 1e-37f  <=>  pv < 1e-37f
        if (pv < 1e-37f) continue;
        float qx = fsub(k0, b.x), qy = fsub(k1, b.y), qz = fsub(k2, b.z);
        if (CHECK && fadd(fadd(fmul(qx, qx), fmul(qy, qy)), fmul(qz, qz)) > a.maxq2) continue;
        qx = fmul(qx, a.vpdq);
        qy = fmul(qy, a.vpdq);
        qz = fmul(qz, a.vpdq);
        const float qa = axis<KA>(qx, qy, qz, a.ka), qb = axis<KB>(qx, qy, qz, a.kb),
                    qc = axis<KC>(qx, qy, qz, a.kc);
        int f, m, s;
        if (INTERP == 0) {
            // (int)(round(q) + centre) of the reference, in integers
            f = round_half_away(qa) + a.cab;
            m = round_half_away(qb) + a.cab;
            s = round_half_away(qc) + a.cc;
        } else {
            f = __float2int_rd(qa) + a.cab;
            m = __float2int_rd(qb) + a.cab;
            s = __float2int_rd(qc) + a.cc;
        }
        if (!have || f != cur_f || m != cur_m || s != cur_s) {
            if (have) {
                if (INTERP == 0) {
                    put(a, w, win, cur_f, cur_m, cur_s, acc[0]);
                } else {
#pragma unroll
                    for (int c = 0; c < 8; c++)
                        put(a, w, win, cur_f + (c >> 2), cur_m + ((c >> 1) & 1), cur_s + (c & 1), acc[c]);
                }
            }
            have = true;
            cur_f = f;
            cur_m = m;
            cur_s = s;
#pragma unroll
            for (int c = 0; c < (INTERP ? 8 : 1); c++) acc[c] = 0;
        }
        if (INTERP == 0) {
            acc[0] += a.mult_int ? scaled_floor(pv, a.mult_int) : d2u64(dmul((double)pv, a.mult));
        } else {
            const double vm = dmul((double)pv, a.mult);
            // IAC/kernel.cl:139-179: Sep = 1 - (q - floor q) in float
            const double sf = (double)fsub(1.0f, fsub(qa, floorf(qa)));
            const double sm = (double)fsub(1.0f, fsub(qb, floorf(qb)));
            const double sz = (double)fsub(1.0f, fsub(qc, floorf(qc)));
            const double xf[2] = {sf, dsub(1.0, sf)}, yf[2] = {sm, dsub(1.0, sm)}, zf[2] = {sz, dsub(1.0, sz)};
#pragma unroll
            for (int c = 0; c < 8; c++)
                acc[c] += d2u64(dmul(vm, dmul(dmul(xf[c >> 2], yf[(c >> 1) & 1]), zf[c & 1])));
        }
    }
    if (have) {
        if (INTERP == 0) {
            put(a, w, win, cur_f, cur_m, cur_s, acc[0]);
        } else {
#pragma unroll
            for (int c = 0; c < 8; c++)
                put(a, w, win, cur_f + (c >> 2), cur_m + ((c >> 1) & 1), cur_s + (c & 1), acc[c]);
        }
    }
}

// scaled_floor for a normal p > 0 (every product that passes the 1e-37 test)
__device__ __forceinline__ unsigned long long scaled_floor_normal(float p, uint32_t M)
{
    const uint32_t b = __float_as_uint(p);
    const unsigned long long prod = (unsigned long long)((b & 0x7fffffu) | 0x800000u) * M;
    const int sh = (int)(b >> 23) - 150;  // p = mantissa * 2^sh
    return sh >= 0 ? (prod << min(sh, 63)) : (prod >> min(-sh, 63));
}

// nearest-voxel pairs with a compile-time axis mapping: the voxel is compared
// as one packed key f + 1024 m + 2^20 s (components within +-511, which
// key_ok guarantees for every pair inside MaxQ), the value path is chosen at
// compile time (MINT: integer Multiplicator)
template <int KA, int KB, int KC, bool CHECK, bool MINT>
__device__ __forceinline__ void cq_pairs_nn(const DenseArgs &a, const Window &w, uint32_t *win,
                                            const float4 *sq, int j0, float k0, float k1, float k2, float Ia)
{
    constexpr int NONE = -2147483647 - 1;
    int cur = NONE, cf = 0, cm = 0, cs = 0;
    unsigned long long acc = 0;
    const float vpdq = a.vpdq;
#pragma unroll 2
    for (int j = j0; j < DTILE; j++) {
        const float4 b = sq[j];
        const float pv = fmul(Ia, b.w);
        if (pv < 1e-37f) continue;
        float qx = fsub(k0, b.x), qy = fsub(k1, b.y), qz = fsub(k2, b.z);
        if (CHECK && fadd(fadd(fmul(qx, qx), fmul(qy, qy)), fmul(qz, qz)) > a.maxq2) continue;
        qx = fmul(qx, vpdq);
        qy = fmul(qy, vpdq);
        qz = fmul(qz, vpdq);
        const int f = round_half_away(axis<KA>(qx, qy, qz, 0));
        const int m = round_half_away(axis<KB>(qx, qy, qz, 0));
        const int s = round_half_away(axis<KC>(qx, qy, qz, 0));
        const int key = f + m * 1024 + s * 1048576;
        if (key != cur) {
            if (cur != NONE) put(a, w, win, cf + a.cab, cm + a.cab, cs + a.cc, acc);
            cur = key;
            cf = f;
            cm = m;
            cs = s;
            acc = 0;
        }
        acc += MINT ? scaled_floor_normal(pv, a.mult_int) : d2u64(dmul((double)pv, a.mult));
    }
    if (cur != NONE) put(a, w, win, cf + a.cab, cm + a.cab, cs + a.cc, acc);
}


// cq_pairs_nn when the window is on: every pair inside MaxQ lands in the
// window (it spans the two tiles' q range with a voxel of margin), so the run
// key is the voxel's window index itself and a finished run is one split 64-bit
// shared-memory add.  Pairs that fail the intensity or MaxQ test are masked
// rather than skipped, so a warp never diverges on them; the only branch is
// the guard for an index outside the window (non-finite k-vectors), which
// takes the global path of put().
template <int KA, int KB, int KC, bool CHECK, bool MINT>
__device__ __forceinline__ void cq_pairs_win(const DenseArgs &a, const Window &w, uint32_t *win,
                                             const float4 *sq, int j0, float k0, float k1, float k2, float Ia)
{
    const int D0 = w.dim[0], D01 = w.dim[0] * w.dim[1];
    const int words = D01 * w.dim[2];
    const int base = (a.cab - w.lo[0]) + D0 * (a.cab - w.lo[1]) + D01 * (a.cc - w.lo[2]);
    const float vpdq = a.vpdq;
    int cur = 0;
    bool on = false;  // a run is pending at window index cur
    unsigned long long acc = 0;
#pragma unroll 2
    for (int j = j0; j < DTILE; j++) {
        const float4 b = sq[j];
        const float pv = fmul(Ia, b.w);
        float qx = fsub(k0, b.x), qy = fsub(k1, b.y), qz = fsub(k2, b.z);
        bool ok = !(pv < 1e-37f);
        if (CHECK) ok = ok && !(fadd(fadd(fmul(qx, qx), fmul(qy, qy)), fmul(qz, qz)) > a.maxq2);
        qx = fmul(qx, vpdq);
        qy = fmul(qy, vpdq);
        qz = fmul(qz, vpdq);
        const int f = round_half_away(axis<KA>(qx, qy, qz, 0));
        const int m = round_half_away(axis<KB>(qx, qy, qz, 0));
        const int sz = round_half_away(axis<KC>(qx, qy, qz, 0));
        const int key = base + f + D0 * m + D01 * sz;
        const unsigned long long v = MINT ? scaled_floor_normal(pv, a.mult_int) : d2u64(dmul((double)pv, a.mult));
        const bool brk = ok && (!on || key != cur);  // a new run starts at this pair
        if (brk && on) shared_add_u64_split(win, win + WINDOW_WORDS, (uint32_t)cur, acc);
        const bool inwin = (unsigned)key < (unsigned)words;
        if (brk && !inwin) global_put_pair(a, f + a.cab, m + a.cab, sz + a.cc, v);
        acc = brk ? (inwin ? v : 0ull) : (ok ? acc + v : acc);
        cur = brk ? key : cur;
        on = brk ? inwin : on;
    }
    if (on) shared_add_u64_split(win, win + WINDOW_WORDS, (uint32_t)cur, acc);
}

// ---- two consecutive staged pixels per step, FP32 work as f32x2 pairs ----
// add/sub/mul.rn.f32x2 (sm_100) round each lane exactly as the scalar
// instruction does, so the pair of results is bit-identical to two scalar ops.
// Unlike scalar mul.rn/add.rn, a packed multiply whose product feeds a packed
// add can come out of ptxas as one fused FFMA2 (one rounding instead of two),
// so products are only packed where no add consumes them.
__device__ __forceinline__ float2 f2sub(float2 a, float2 b)
{
    float2 r;
    asm("{\n\t.reg .b64 x, y, z;\n\tmov.b64 x, {%2, %3};\n\tmov.b64 y, {%4, %5};\n\t"
        "sub.rn.f32x2 z, x, y;\n\tmov.b64 {%0, %1}, z;\n\t}"
        : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 f2add(float2 a, float2 b)
{
    float2 r;
    asm("{\n\t.reg .b64 x, y, z;\n\tmov.b64 x, {%2, %3};\n\tmov.b64 y, {%4, %5};\n\t"
        "add.rn.f32x2 z, x, y;\n\tmov.b64 {%0, %1}, z;\n\t}"
        : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 f2mul(float2 a, float2 b)
{
    float2 r;
    asm("{\n\t.reg .b64 x, y, z;\n\tmov.b64 x, {%2, %3};\n\tmov.b64 y, {%4, %5};\n\t"
        "mul.rn.f32x2 z, x, y;\n\tmov.b64 {%0, %1}, z;\n\t}"
        : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}

// round half away from zero of both lanes, as ints (see round_half_away)
__device__ __forceinline__ int2 f2round_half_away(float2 x)
{
    const float2 t = f2add(x, make_float2(copysignf(0.49999997f, x.x), copysignf(0.49999997f, x.y)));
    return make_int2(__float2int_rz(t.x), __float2int_rz(t.y));
}

// floor(p * M) for 0 <= p < 2^23 and an integer M < 2^29: p's 24-bit
// significand times M is below 2^53, so the double product is exact and its
// truncation is the floor.  One multiply on the (otherwise idle) FP64 pipe and
// two conversions take fewer issue slots than the integer form (significand
// product shifted by the exponent), which measured 1.025 s against 0.864 s at
// 1024^2 with the run flush below.
__device__ __forceinline__ unsigned long long scaled_floor_small(float p, uint32_t M)
{
    return __double2ull_rz(__dmul_rn((double)p, (double)M));
}

// one pair of the packed window path: a pair that fails the intensity or
// MaxQ test adds 0 at the pending voxel (it neither starts nor ends a run)
__device__ __forceinline__ void win_step(const DenseArgs &a, uint32_t *win, int words, bool ok, int key, float pv,
                                         int f, int m, int sz, int &cur, unsigned long long &acc)
{
    if (ok && (unsigned)key >= (unsigned)words) {  // non-finite k-vectors only
        global_put_pair(a, f + a.cab, m + a.cab, sz + a.cc, scaled_floor_small(pv, a.mult_int));
        ok = false;
    }
    const int k = ok ? key : cur;
    const unsigned long long v = scaled_floor_small(ok ? pv : 0.0f, a.mult_int);
    const bool brk = k != cur;
    if (brk) shared_add_u64_split(win, win + WINDOW_WORDS, (uint32_t)cur, acc);  // acc may be 0: adds nothing
    acc = (brk ? 0ull : acc) + v;
    cur = k;
}

// cq_pairs_win for an integer Multiplicator and tile pairs whose products stay
// below 2^23: the staged tile holds consecutive pixels j, j+1 as
// (x_j, x_j+1, y_j, y_j+1), (z_j, z_j+1, I_j, I_j+1), and each step evaluates
// both pairs with f32x2 arithmetic (the same roundings as the scalar path),
// then bins them in order.  j0 may be odd (diagonal tiles): the first step
// then masks its lower lane.
template <int KA, int KB, int KC, bool CHECK>
__device__ __forceinline__ void cq_pairs_win2(const DenseArgs &a, const Window &w, uint32_t *win,
                                              const float4 *sp, int j0, float k0, float k1, float k2, float Ia)
{
    const int D0 = w.dim[0], D01 = w.dim[0] * w.dim[1];
    const int words = D01 * w.dim[2];
    const int base = (a.cab - w.lo[0]) + D0 * (a.cab - w.lo[1]) + D01 * (a.cc - w.lo[2]);
    const float2 vp2 = make_float2(a.vpdq, a.vpdq), K0 = make_float2(k0, k0), K1 = make_float2(k1, k1),
                 K2 = make_float2(k2, k2), IA = make_float2(Ia, Ia);
    int cur = 0;  // pending run: window index cur, value acc (0 before the first pair)
    unsigned long long acc = 0;
    auto step = [&](int jp, bool lo_on) {
        const float4 A = sp[2 * jp], B = sp[2 * jp + 1];
        const float2 pv = f2mul(IA, make_float2(B.z, B.w));
        float2 qx = f2sub(K0, make_float2(A.x, A.y)), qy = f2sub(K1, make_float2(A.z, A.w)),
               qz = f2sub(K2, make_float2(B.x, B.y));
        bool ok0 = lo_on && !(pv.x < 1e-37f), ok1 = !(pv.y < 1e-37f);
        if (CHECK) {  // scalar: ptxas may fuse a packed multiply and add into one FFMA2
            ok0 = ok0 && !(fadd(fadd(fmul(qx.x, qx.x), fmul(qy.x, qy.x)), fmul(qz.x, qz.x)) > a.maxq2);
            ok1 = ok1 && !(fadd(fadd(fmul(qx.y, qx.y), fmul(qy.y, qy.y)), fmul(qz.y, qz.y)) > a.maxq2);
        }
        qx = f2mul(qx, vp2);
        qy = f2mul(qy, vp2);
        qz = f2mul(qz, vp2);
        const int2 f = f2round_half_away(KA == 0 ? qx : KA == 1 ? qy : qz);
        const int2 m = f2round_half_away(KB == 0 ? qx : KB == 1 ? qy : qz);
        const int2 sz = f2round_half_away(KC == 0 ? qx : KC == 1 ? qy : qz);
        win_step(a, win, words, ok0, base + f.x + D0 * m.x + D01 * sz.x, pv.x, f.x, m.x, sz.x, cur, acc);
        win_step(a, win, words, ok1, base + f.y + D0 * m.y + D01 * sz.y, pv.y, f.y, m.y, sz.y, cur, acc);
    };
    int jp = j0 >> 1;
    if (j0 & 1) step(jp++, false);
#pragma unroll 2
    for (; jp < DTILE / 2; jp++) step(jp, true);
    if (acc) shared_add_u64_split(win, win + WINDOW_WORDS, (uint32_t)cur, acc);
}

// upper bound of |k_a - k_b| over two boxes is below MaxQ with a margin that
// covers the FP32 rounding of the per-pair test (every pair passes it)
__device__ __forceinline__ bool boxes_within(const float4 a0, const float4 a1, const float4 b0, const float4 b1,
                                             float maxq)
{
    const float dx = fmaxf(a1.x - b0.x, b1.x - a0.x);
    const float dy = fmaxf(a1.y - b0.y, b1.y - a0.y);
    const float dz = fmaxf(a1.z - b0.z, b1.z - a0.z);
    return dx * dx + dy * dy + dz * dz < maxq * maxq * 0.9999f;
}

// index within the 16 x 16 patch of thread t's own pixel: lane l of warp w takes
// x = 4 (l % 4) + w % 4, y = 2 (l / 4) + w / 4 (a bijection of 0..255)
__device__ __forceinline__ int own_pixel(int t)
{
    const int w = t >> 5, l = t & 31;
    return (2 * (l >> 2) + (w >> 2)) * 16 + 4 * (l & 3) + (w & 3);
}

template <int INTERP, int KA, int KB, int KC>
__global__ void __launch_bounds__(DTILE, 5) cq_small_kernel(const DenseArgs a)
{
    __shared__ float4 sq[DTILE];
    __shared__ uint32_t win[2 * WINDOW_WORDS];  // split 64-bit counters: low words, then high words
    __shared__ unsigned long long s_pair;
    __shared__ unsigned long long s_self[DTILE / 32];
    const uint32_t T = a.ntiles;
    for (;;) {
        if (threadIdx.x == 0) s_pair = atomicAdd(a.queue, 1ull);
        __syncthreads();
        const unsigned long long p = s_pair * a.nparts + a.part;
        if (p >= a.npairs) break;
        uint32_t P, Q;
        decode_tile_pair(p, T, P, Q);
        const float4 p0 = a.box[2 * P], p1 = a.box[2 * P + 1], q0 = a.box[2 * Q], q1 = a.box[2 * Q + 1];
        if (boxes_beyond(p0, p1, q0, q1, a.maxq)) {
            __syncthreads();
            continue;
        }
        const bool check = !boxes_within(p0, p1, q0, q1, a.maxq);
        // window over the q range of the pair (P - Q), one voxel of margin
        Window w;
        {
            const float lo3[3] = {p0.x - q1.x, p0.y - q1.y, p0.z - q1.z};
            const float hi3[3] = {p1.x - q0.x, p1.y - q0.y, p1.z - q0.z};
            const int ax[3] = {a.ka, a.kb, a.kc};
            const int cen[3] = {a.cab, a.cab, a.cc};
            int words = 1;
            bool ok = true;
            for (int d = 0; d < 3; d++) {
                const float l = (ax[d] == 0 ? lo3[0] : ax[d] == 1 ? lo3[1] : lo3[2]) * a.vpdq;
                const float h = (ax[d] == 0 ? hi3[0] : ax[d] == 1 ? hi3[1] : hi3[2]) * a.vpdq;
                w.lo[d] = (int)floorf(l) - 1 + cen[d];
                w.dim[d] = (int)ceilf(h) + 2 + cen[d] - w.lo[d] + (INTERP ? 1 : 0);
                ok &= w.dim[d] >= 1 && w.dim[d] <= WINDOW_WORDS;
                words *= max(1, min(w.dim[d], WINDOW_WORDS + 1));
            }
            w.on = ok && words <= WINDOW_WORDS;
            if (w.on)
                for (int i = threadIdx.x; i < words; i += DTILE) win[i] = win[WINDOW_WORDS + i] = 0u;
        }
        // integer Multiplicator and every product of the two tiles below 2^23
        // (the tiles' largest |I|): the packed window path
        const bool packed = INTERP == 0 && KA >= 0 && w.on && a.mult_int != 0u && fmul(p0.w, q0.w) < 8388608.0f;
        // stage tile Q: (k, I) per pixel, or interleaved per pixel pair for the packed path
        {
            const uint64_t j = tile_pixel(a, Q, threadIdx.x);
            const float4 v = j < a.npix ? make_float4(a.K[3 * j], a.K[3 * j + 1], a.K[3 * j + 2], a.I[j])
                                        : make_float4(0.f, 0.f, 0.f, 0.f);
            if (packed) {
                float *spf = reinterpret_cast<float *>(sq) + (threadIdx.x >> 1) * 8 + (threadIdx.x & 1);
                spf[0] = v.x;
                spf[2] = v.y;
                spf[4] = v.z;
                spf[6] = v.w;
            } else {
                sq[threadIdx.x] = v;
            }
        }
        __syncthreads();
        // own pixel: spread over the patch (x 4 apart, y 2 apart within a warp) so
        // that a warp's lanes rarely share a voxel and their window adds for one
        // staged pixel rarely meet at one address; the staged tile keeps its
        // order (runs of consecutive pixels land in one voxel)
        const int own = own_pixel(threadIdx.x);
        const uint64_t ia = tile_pixel(a, P, own);
        unsigned long long self = 0;
        if (ia < a.npix) {
            const float k0 = a.K[3 * ia], k1 = a.K[3 * ia + 1], k2 = a.K[3 * ia + 2];
            const float Ia = a.I[ia];
            if (P == Q) {
                const float sv = fmul(Ia, Ia);
                if (!(sv < 1e-37f))
                    self = a.mult_int ? scaled_floor(sv, a.mult_int) : d2u64(dmul((double)sv, a.mult));
            }
            const int j0 = (P == Q) ? own + 1 : 0;
            if (packed) {
                if (check)
                    cq_pairs_win2<KA, KB, KC, true>(a, w, win, sq, j0, k0, k1, k2, Ia);
                else
                    cq_pairs_win2<KA, KB, KC, false>(a, w, win, sq, j0, k0, k1, k2, Ia);
            } else if (INTERP == 0 && KA >= 0 && w.on) {
                if (a.mult_int) {
                    if (check)
                        cq_pairs_win<KA, KB, KC, true, true>(a, w, win, sq, j0, k0, k1, k2, Ia);
                    else
                        cq_pairs_win<KA, KB, KC, false, true>(a, w, win, sq, j0, k0, k1, k2, Ia);
                } else {
                    if (check)
                        cq_pairs_win<KA, KB, KC, true, false>(a, w, win, sq, j0, k0, k1, k2, Ia);
                    else
                        cq_pairs_win<KA, KB, KC, false, false>(a, w, win, sq, j0, k0, k1, k2, Ia);
                }
            } else if (INTERP == 0 && KA >= 0 && a.key_ok) {
                if (a.mult_int) {
                    if (check)
                        cq_pairs_nn<KA, KB, KC, true, true>(a, w, win, sq, j0, k0, k1, k2, Ia);
                    else
                        cq_pairs_nn<KA, KB, KC, false, true>(a, w, win, sq, j0, k0, k1, k2, Ia);
                } else {
                    if (check)
                        cq_pairs_nn<KA, KB, KC, true, false>(a, w, win, sq, j0, k0, k1, k2, Ia);
                    else
                        cq_pairs_nn<KA, KB, KC, false, false>(a, w, win, sq, j0, k0, k1, k2, Ia);
                }
            } else if (check) {
                cq_pairs<INTERP, KA, KB, KC, true>(a, w, win, sq, j0, k0, k1, k2, Ia);
            } else {
                cq_pairs<INTERP, KA, KB, KC, false>(a, w, win, sq, j0, k0, k1, k2, Ia);
            }
        }
        // self pairs of a diagonal tile: once, at the centre
        for (int o = 16; o; o >>= 1) self += __shfl_xor_sync(0xffffffffu, self, o);
        if ((threadIdx.x & 31) == 0) s_self[threadIdx.x >> 5] = self;
        __syncthreads();
        if (threadIdx.x == 0 && P == Q) {
            unsigned long long t = 0;
            for (int i = 0; i < DTILE / 32; i++) t += s_self[i];
            if (t) atomicAdd(&a.out[(uint64_t)a.cab + (uint64_t)a.cab * a.ab + (uint64_t)a.cc * a.ab * a.ab], t);
        }
        if (w.on) {
            const int words = w.dim[0] * w.dim[1] * w.dim[2];
            for (int i = threadIdx.x; i < words; i += DTILE) {
                const unsigned long long v = split_word(win, win + WINDOW_WORDS, i);
                if (!v) continue;
                const int x = i % w.dim[0], y = (i / w.dim[0]) % w.dim[1], z = i / (w.dim[0] * w.dim[1]);
                global_put_pair(a, x + w.lo[0], y + w.lo[1], z + w.lo[2], v);
            }
        }
        __syncthreads();
    }
}

// --------------------------------------------------------------------------
// AC1D C(q): |q| histogram in shared memory for the whole launch
// --------------------------------------------------------------------------
// b % n without the division when b < n (bins past the histogram are rare)
__device__ __forceinline__ uint32_t wrap_bin(uint32_t b, uint32_t n)
{
    if (b >= n) b %= n;
    return b;
}

template <int INTERP>
__global__ void __launch_bounds__(DTILE) ac1d_cq_kernel(const DenseArgs a)
{
    // the launch's histogram as split 64-bit counters: low words, then high words
    extern __shared__ uint32_t hist32[];
    uint32_t *const hlo = hist32, *const hhi = hist32 + a.hsize;
    __shared__ float4 sq[DTILE];
    __shared__ unsigned long long s_pair;
    for (uint32_t i = threadIdx.x; i < 2 * a.hsize; i += DTILE) hist32[i] = 0;
    const uint32_t T = a.ntiles;
    for (;;) {
        if (threadIdx.x == 0) s_pair = atomicAdd(a.queue, 1ull);
        __syncthreads();
        const unsigned long long p = s_pair * a.nparts + a.part;
        if (p >= a.npairs) break;
        uint32_t P, Q;
        decode_tile_pair(p, T, P, Q);
        const float4 p0 = a.box[2 * P], p1 = a.box[2 * P + 1], q0 = a.box[2 * Q], q1 = a.box[2 * Q + 1];
        if (boxes_beyond(p0, p1, q0, q1, a.maxq)) {
            __syncthreads();
            continue;
        }
        {
            const uint64_t j = tile_pixel(a, Q, threadIdx.x);
            sq[threadIdx.x] = j < a.npix ? make_float4(a.K[3 * j], a.K[3 * j + 1], a.K[3 * j + 2], a.I[j])
                                         : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        __syncthreads();
        // own pixel 8 apart from the neighbouring lanes' (a bijection of the tile):
        // the lanes of a warp then add into different bins for one staged pixel
        const int own = (int)((threadIdx.x & 31) * 8 + (threadIdx.x >> 5));
        const uint64_t ia = tile_pixel(a, P, own);
        if (ia < a.npix) {
            const float k0 = a.K[3 * ia], k1 = a.K[3 * ia + 1], k2 = a.K[3 * ia + 2];
            const float Ia = a.I[ia];
            if (P == Q) {  // self pair: q = 0 -> bin 0, once
                const float sv = fmul(Ia, Ia);
                if (!(sv < 1e-37f))
                    shared_add_u64_split(hlo, hhi, 0,
                                         a.mult_int ? scaled_floor(sv, a.mult_int)
                                                    : (unsigned long long)(long long)dmul((double)sv, a.mult));
            }
            const int j0 = (P == Q) ? own + 1 : 0;
            for (int j = j0; j < DTILE; j++) {
                const float4 b = sq[j];
                const float pv = fmul(Ia, b.w);
                if (pv < 1e-37f) continue;
                const double val = (double)pv;
                const float dx = fsub(k0, b.x), dy = fsub(k1, b.y), dz = fsub(k2, b.z);
                float q = __fsqrt_rn(fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz)));
                if (q > a.maxq) continue;
                q = __fdiv_rn(q, a.dq);
                if (INTERP == 0) {
                    // sc = (uint)floor(q + 0.5) with q + 0.5 in double: floor(fl(q +
                    // 0.49999997f)) equals it for every float 0 <= q < 2^23 (the
                    // identity of round_half_away); fl(q + 0.5f) does not at
                    // q = 0.5 - 2^-25, whose sum rounds up to 1
                    const uint32_t sc = wrap_bin((uint32_t)floorf(fadd(q, 0.49999997f)), a.hsize);
                    const unsigned long long v =
                        a.mult_int ? scaled_floor(pv, a.mult_int) : (unsigned long long)(long long)dmul(val, a.mult);
                    shared_add_u64_split(hlo, hhi, sc, 2ull * v);
                } else {
                    uint32_t iq;  // q = |q| / dq <= MaxQ / dq < 2^23
                    const float fq = floor_small(q, iq);
                    const uint32_t sc1 = wrap_bin(iq, a.hsize), sc2 = wrap_bin(iq + 1, a.hsize);
                    const double sep = (double)fsub(q, fq);
                    const unsigned long long v1 =
                        (unsigned long long)(long long)dmul(dmul(val, dsub(1.0, sep)), a.mult);
                    const unsigned long long v2 = (unsigned long long)(long long)dmul(dmul(val, sep), a.mult);
                    shared_add_u64_split(hlo, hhi, sc1, 2ull * v1);
                    shared_add_u64_split(hlo, hhi, sc2, 2ull * v2);
                }
            }
        }
        __syncthreads();
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < a.hsize; i += DTILE) {
        const unsigned long long v = split_word(hlo, hhi, i);
        if (v) atomicAdd(&a.out[i], v);
    }
}

// --------------------------------------------------------------------------
// Row lists: the reference's own work decomposition.  Work item `ind` of
// AutoCorr_CQ_small / AutoCorr_CQ_AV visits every pixel i and bins the
// ordered pair (ind, i) (IAC/kernel.cl:78-182, :696-762); the mesh is the sum
// of these independent items.  The kernels below evaluate the items of a list
// of rows, each pair in the reference's arithmetic and order, so that a
// full-size detector can be checked against the oracle on a subset of rows and
// the unordered-pair kernels above against the sum over every row.  A CTA
// stages 256 consecutive pixels and each thread walks them for its row.
// --------------------------------------------------------------------------
__device__ __forceinline__ void global_put(const DenseArgs &a, int fs, int ms, int ss, unsigned long long v)
{
    if (v == 0) return;
    if ((unsigned)fs >= (unsigned)a.ab || (unsigned)ms >= (unsigned)a.ab || (unsigned)ss >= (unsigned)a.sc)
        atomicAdd(&a.counters->out_of_mesh, 1ull);
    else
        atomicAdd(&a.out[(uint64_t)fs + (uint64_t)ms * a.ab + (uint64_t)ss * a.ab * a.ab], v);
}

// the staged column tile of a row-list kernel: 256 consecutive pixels as (k, I)
__device__ __forceinline__ void stage_columns(const DenseArgs &a, uint64_t col_tile, float4 *sq)
{
    const uint64_t j = col_tile * DTILE + threadIdx.x;
    sq[threadIdx.x] = j < a.npix ? make_float4(a.K[3 * j], a.K[3 * j + 1], a.K[3 * j + 2], a.I[j])
                                 : make_float4(0.f, 0.f, 0.f, 0.f);
}

// C(q) small mesh, rows x all pixels: grid (column tiles, row tiles)
template <int INTERP>
__global__ void __launch_bounds__(DTILE) cq_rows_kernel(const DenseArgs a, const uint32_t *__restrict__ rows,
                                                        uint32_t nrows)
{
    __shared__ float4 sq[DTILE];
    stage_columns(a, blockIdx.x, sq);
    __syncthreads();
    const uint32_t r = blockIdx.y * DTILE + threadIdx.x;
    if (r >= nrows) return;
    const uint32_t ind = rows[r];
    if (ind >= a.npix) {
        if (blockIdx.x == 0) atomicAdd(&a.counters->out_of_mesh, 1ull);
        return;
    }
    const float k0 = a.K[3 * (uint64_t)ind], k1 = a.K[3 * (uint64_t)ind + 1], k2 = a.K[3 * (uint64_t)ind + 2];
    const float Ia = a.I[ind];
    int cf = 0, cm = 0, cs = 0;
    bool have = false;
    unsigned long long acc[INTERP ? 8 : 1];
#pragma unroll
    for (int c = 0; c < (INTERP ? 8 : 1); c++) acc[c] = 0;
    for (int j = 0; j < DTILE; j++) {
        const float4 b = sq[j];
        const float pv = fmul(Ia, b.w);  // Val = (double)(I_ind * I_i)
        if (pv < 1e-37f) continue;
        float qx = fsub(k0, b.x), qy = fsub(k1, b.y), qz = fsub(k2, b.z);
        if (fadd(fadd(fmul(qx, qx), fmul(qy, qy)), fmul(qz, qz)) > a.maxq2) continue;
        qx = fmul(qx, a.vpdq);
        qy = fmul(qy, a.vpdq);
        qz = fmul(qz, a.vpdq);
        const float qa = pick(qx, qy, qz, a.ka), qb = pick(qx, qy, qz, a.kb), qc = pick(qx, qy, qz, a.kc);
        int f, m, sv;
        if (INTERP == 0) {
            f = round_half_away(qa) + a.cab;
            m = round_half_away(qb) + a.cab;
            sv = round_half_away(qc) + a.cc;
        } else {
            f = __float2int_rd(qa) + a.cab;
            m = __float2int_rd(qb) + a.cab;
            sv = __float2int_rd(qc) + a.cc;
        }
        if (!have || f != cf || m != cm || sv != cs) {
            if (have) {
#pragma unroll
                for (int c = 0; c < (INTERP ? 8 : 1); c++)
                    global_put(a, cf + (c >> 2), cm + ((c >> 1) & 1), cs + (c & 1), acc[c]);
            }
            have = true;
            cf = f;
            cm = m;
            cs = sv;
#pragma unroll
            for (int c = 0; c < (INTERP ? 8 : 1); c++) acc[c] = 0;
        }
        if (INTERP == 0) {
            acc[0] += a.mult_int ? scaled_floor(pv, a.mult_int) : d2u64(dmul((double)pv, a.mult));
        } else {
            const double vm = dmul((double)pv, a.mult);
            const double sf = (double)fsub(1.0f, fsub(qa, floorf(qa)));
            const double sm = (double)fsub(1.0f, fsub(qb, floorf(qb)));
            const double sz = (double)fsub(1.0f, fsub(qc, floorf(qc)));
            const double xf[2] = {sf, dsub(1.0, sf)}, yf[2] = {sm, dsub(1.0, sm)}, zf[2] = {sz, dsub(1.0, sz)};
#pragma unroll
            for (int c = 0; c < 8; c++) acc[c] += d2u64(dmul(vm, dmul(dmul(xf[c >> 2], yf[(c >> 1) & 1]), zf[c & 1])));
        }
    }
    if (have) {
#pragma unroll
        for (int c = 0; c < (INTERP ? 8 : 1); c++)
            global_put(a, cf + (c >> 2), cm + ((c >> 1) & 1), cs + (c & 1), acc[c]);
    }
}

// AC1D |q| histogram, rows x all pixels: persistent CTAs over (row tile,
// column tile) items, the histogram in shared memory for the whole launch
template <int INTERP>
__global__ void __launch_bounds__(DTILE) ac1d_rows_kernel(const DenseArgs a, const uint32_t *__restrict__ rows,
                                                          uint32_t nrows)
{
    extern __shared__ unsigned long long hist[];
    __shared__ float4 sq[DTILE];
    __shared__ unsigned long long s_item;
    for (uint32_t i = threadIdx.x; i < a.hsize; i += DTILE) hist[i] = 0;
    const uint64_t ncol = (a.npix + DTILE - 1) / DTILE;
    const unsigned long long nitems = (unsigned long long)ncol * ((nrows + DTILE - 1) / DTILE);
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(a.queue, 1ull);
        __syncthreads();
        const unsigned long long it = s_item;
        if (it >= nitems) break;
        const uint64_t rt = it / ncol, ct = it - rt * ncol;
        stage_columns(a, ct, sq);
        __syncthreads();
        const uint64_t r = rt * DTILE + threadIdx.x;
        const uint32_t ind = r < nrows ? rows[r] : 0xffffffffu;
        if (r < nrows && ind >= a.npix && ct == 0) atomicAdd(&a.counters->out_of_mesh, 1ull);
        if (ind < a.npix) {
            const float k0 = a.K[3 * (uint64_t)ind], k1 = a.K[3 * (uint64_t)ind + 1], k2 = a.K[3 * (uint64_t)ind + 2];
            const float Ia = a.I[ind];
            for (int j = 0; j < DTILE; j++) {
                const float4 b = sq[j];
                const float pv = fmul(Ia, b.w);
                if (pv < 1e-37f) continue;
                const double val = (double)pv;
                const float dx = fsub(k0, b.x), dy = fsub(k1, b.y), dz = fsub(k2, b.z);
                float q = __fsqrt_rn(fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz)));
                if (q > a.maxq) continue;
                q = __fdiv_rn(q, a.dq);
                if (INTERP == 0) {
                    const uint32_t sc = wrap_bin((uint32_t)floor(dadd((double)q, 0.5)), a.hsize);
                    atomicAdd(&hist[sc], a.mult_int ? scaled_floor(pv, a.mult_int)
                                                    : (unsigned long long)(long long)dmul(val, a.mult));
                } else {
                    const float fq = floorf(q);
                    const double sep = (double)fsub(q, fq);
                    atomicAdd(&hist[wrap_bin((uint32_t)fq, a.hsize)],
                              (unsigned long long)(long long)dmul(dmul(val, dsub(1.0, sep)), a.mult));
                    atomicAdd(&hist[wrap_bin((uint32_t)fq + 1, a.hsize)],
                              (unsigned long long)(long long)dmul(dmul(val, sep), a.mult));
                }
            }
        }
        __syncthreads();
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < a.hsize; i += DTILE)
        if (hist[i]) atomicAdd(&a.out[i], hist[i]);
}

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

// tile boxes + queue counter in stream scratch; returns args with common fields
static iac_status prepare(iac_ctx *ctx, void *stream, const float *d_I, const float *d_K,
                          uint64_t npix, uint32_t fast_size, double mult, DenseArgs &a)
{
    a.I = d_I;
    a.K = d_K;
    a.npix = npix;
    a.mult = mult;
    a.mult_int = (mult >= 1.0 && mult < 536870912.0 && mult == std::floor(mult)) ? (uint32_t)mult : 0u;
    if (fast_size >= 16 && npix % fast_size == 0) {
        a.nx = fast_size;
        a.ny = (uint32_t)(npix / fast_size);
        a.ptx = (a.nx + 15) / 16;
        a.ntiles = a.ptx * ((a.ny + 15) / 16);
    } else {
        a.nx = a.ny = a.ptx = 0;
        a.ntiles = (uint32_t)((npix + DTILE - 1) / DTILE);
    }
    a.npairs = (unsigned long long)a.ntiles * (a.ntiles + 1) / 2;
    a.part = 0;
    a.nparts = 1;
    a.counters = ctx->d_counters;
    void *scr = nullptr;
    const size_t box_bytes = sizeof(float4) * 2 * (size_t)a.ntiles;
    iac_status st = stream_scratch(ctx, stream, SLOT_AUX0, box_bytes + 256, &scr);
    if (st != IAC_OK) return st;
    a.box = (const float4 *)scr;
    a.queue = (unsigned long long *)((char *)scr + ((box_bytes + 127) / 128) * 128);
    cudaStream_t s = as_stream(stream);
    IAC_CUDA(cudaMemsetAsync(a.queue, 0, sizeof(unsigned long long), s));
    tile_box_kernel<<<a.ntiles, DTILE, 0, s>>>(a, (float4 *)scr);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}

}  // namespace iac

using namespace iac;

extern "C" {

iac_status iac_cq_small(iac_ctx *ctx, const float *d_I, const float *d_kmap, uint64_t npix,
                        uint32_t fast_size, const iac_mesh_shape *sh, int interp, double mult,
                        uint64_t *d_mesh, void *stream)
{
    return iac_cq_small_part(ctx, d_I, d_kmap, npix, fast_size, sh, interp, mult, 0, 1, d_mesh, stream);
}

iac_status iac_cq_small_part(iac_ctx *ctx, const float *d_I, const float *d_kmap, uint64_t npix,
                             uint32_t fast_size, const iac_mesh_shape *sh, int interp, double mult,
                             uint32_t part, uint32_t nparts, uint64_t *d_mesh, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx && d_I && d_kmap && sh && d_mesh, "iac_cq_small: NULL argument");
    IAC_REQUIRE(nparts >= 1 && part < nparts, "iac_cq_small_part: part %u of %u", part, nparts);
    IAC_REQUIRE(interp == 0 || interp == 1, "interpolation must be 0 or 1");
    IAC_REQUIRE(npix > 0 && npix < (1ull << 32), "iac_cq_small: pixel count %llu out of range",
                (unsigned long long)npix);
    IAC_REQUIRE(sh->size_ab >= 5 && sh->size_ab % 2 == 1 && sh->size_c >= 1 && sh->size_c % 2 == 1,
                "small mesh sizes must be odd");
    IAC_REQUIRE(sh->k_a < 3 && sh->k_b < 3 && sh->k_c < 3, "bad axis alignment");
    IAC_REQUIRE(mult > 0, "multiplicator must be positive");
    DeviceGuard g(ctx->device);
    DenseArgs a{};
    iac_status st = prepare(ctx, stream, d_I, d_kmap, npix, fast_size, mult, a);
    if (st != IAC_OK) return st;
    a.part = part;
    a.nparts = nparts;
    a.out = (unsigned long long *)d_mesh;
    a.maxq = sh->max_q;
    a.maxq2 = sqrt_threshold(sh->max_q);
    a.vpdq = (float)sh->voxel_per_dq;
    a.ab = (int)sh->size_ab;
    a.sc = (int)sh->size_c;
    a.cab = (a.ab - 1) / 2;
    a.cc = (a.sc - 1) / 2;
    a.ka = (int)sh->k_a;
    a.kb = (int)sh->k_b;
    a.kc = (int)sh->k_c;
    // every pair within MaxQ has |q * Voxel_per_dq| <= MaxQ * Voxel_per_dq (up to
    // rounding): below 500 the packed voxel key cannot alias
    a.key_ok = (double)sh->max_q * (double)sh->voxel_per_dq < 500.0;
    const int grid = ctx->sm_count * 8;
    // the axis mapping is a permutation for every real detector: one
    // instantiation per permutation, a runtime-mapped one otherwise
    const int perm = (a.ka == 0 && a.kb == 1 && a.kc == 2)   ? 0
                     : (a.ka == 0 && a.kb == 2 && a.kc == 1) ? 1
                     : (a.ka == 1 && a.kb == 0 && a.kc == 2) ? 2
                     : (a.ka == 1 && a.kb == 2 && a.kc == 0) ? 3
                     : (a.ka == 2 && a.kb == 0 && a.kc == 1) ? 4
                     : (a.ka == 2 && a.kb == 1 && a.kc == 0) ? 5
                                                             : 6;
    cudaStream_t s = as_stream(stream);
#define IAC_CQ_LAUNCH(I)                                                          \
    switch (perm) {                                                               \
    case 0: cq_small_kernel<I, 0, 1, 2><<<grid, DTILE, 0, s>>>(a); break;         \
    case 1: cq_small_kernel<I, 0, 2, 1><<<grid, DTILE, 0, s>>>(a); break;         \
    case 2: cq_small_kernel<I, 1, 0, 2><<<grid, DTILE, 0, s>>>(a); break;         \
    case 3: cq_small_kernel<I, 1, 2, 0><<<grid, DTILE, 0, s>>>(a); break;         \
    case 4: cq_small_kernel<I, 2, 0, 1><<<grid, DTILE, 0, s>>>(a); break;         \
    case 5: cq_small_kernel<I, 2, 1, 0><<<grid, DTILE, 0, s>>>(a); break;         \
    default: cq_small_kernel<I, -1, -1, -1><<<grid, DTILE, 0, s>>>(a); break;     \
    }
    if (interp == 0) {
        IAC_CQ_LAUNCH(0)
    } else {
        IAC_CQ_LAUNCH(1)
    }
#undef IAC_CQ_LAUNCH
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}

iac_status iac_ac1d_cq(iac_ctx *ctx, const float *d_I, const float *d_kmap, uint64_t npix,
                       const iac_ac1d_shape *sh, int interp, double mult, uint64_t *d_hist,
                       void *stream)
{
    return iac_ac1d_cq_part(ctx, d_I, d_kmap, npix, sh, interp, mult, 0, 1, d_hist, stream);
}

iac_status iac_ac1d_cq_part(iac_ctx *ctx, const float *d_I, const float *d_kmap, uint64_t npix,
                            const iac_ac1d_shape *sh, int interp, double mult, uint32_t part, uint32_t nparts,
                            uint64_t *d_hist, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx && d_I && d_kmap && sh && d_hist, "iac_ac1d_cq: NULL argument");
    IAC_REQUIRE(nparts >= 1 && part < nparts, "iac_ac1d_cq_part: part %u of %u", part, nparts);
    IAC_REQUIRE(interp == 0 || interp == 1, "interpolation must be 0 or 1");
    IAC_REQUIRE(npix > 0 && npix < (1ull << 32), "iac_ac1d_cq: pixel count out of range");
    IAC_REQUIRE(sh->size >= 3 && sh->size <= 24576, "AC1D size %u out of range [3, 24576]", sh->size);
    IAC_REQUIRE(sh->dq_per_step > 0 && (double)sh->max_q / sh->dq_per_step < 4194304.0,
                "iac_ac1d_cq: MaxQ / dq must be below 2^22 (dq %g, MaxQ %g)", (double)sh->dq_per_step,
                (double)sh->max_q);
    IAC_REQUIRE(mult > 0, "multiplicator must be positive");
    DeviceGuard g(ctx->device);
    DenseArgs a{};
    // linear tiles: the pixels of a 16 x 16 patch pair share few |q| bins, and
    // a warp's shared-memory histogram atomics would collide on them
    iac_status st = prepare(ctx, stream, d_I, d_kmap, npix, 0, mult, a);
    if (st != IAC_OK) return st;
    a.part = part;
    a.nparts = nparts;
    a.out = (unsigned long long *)d_hist;
    a.maxq = sh->max_q;
    a.maxq2 = sqrt_threshold(sh->max_q);
    a.hsize = sh->size;
    a.dq = sh->dq_per_step;
    const size_t smem = sizeof(unsigned long long) * sh->size;
    auto k = interp == 0 ? ac1d_cq_kernel<0> : ac1d_cq_kernel<1>;
    IAC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<ctx->sm_count * 8, DTILE, smem, as_stream(stream)>>>(a);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}

}  // extern "C"

extern "C" {

iac_status iac_cq_small_rows(iac_ctx *ctx, const float *d_I, const float *d_kmap, uint64_t npix,
                             const uint32_t *d_rows, uint32_t nrows, const iac_mesh_shape *sh, int interp,
                             double mult, uint64_t *d_mesh, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx && d_I && d_kmap && sh && d_mesh && d_rows, "iac_cq_small_rows: NULL argument");
    IAC_REQUIRE(interp == 0 || interp == 1, "interpolation must be 0 or 1");
    IAC_REQUIRE(npix > 0 && npix < (1ull << 32), "iac_cq_small_rows: pixel count %llu out of range",
                (unsigned long long)npix);
    IAC_REQUIRE(nrows >= 1 && nrows <= 65535u * DTILE, "iac_cq_small_rows: %u rows out of range [1, %u]", nrows,
                65535u * DTILE);
    IAC_REQUIRE(sh->size_ab >= 5 && sh->size_ab % 2 == 1 && sh->size_c >= 1 && sh->size_c % 2 == 1,
                "small mesh sizes must be odd");
    IAC_REQUIRE(sh->k_a < 3 && sh->k_b < 3 && sh->k_c < 3, "bad axis alignment");
    IAC_REQUIRE(mult > 0, "multiplicator must be positive");
    DeviceGuard g(ctx->device);
    DenseArgs a{};
    a.I = d_I;
    a.K = d_kmap;
    a.npix = npix;
    a.mult = mult;
    a.mult_int = (mult >= 1.0 && mult < 536870912.0 && mult == std::floor(mult)) ? (uint32_t)mult : 0u;
    a.counters = ctx->d_counters;
    a.out = (unsigned long long *)d_mesh;
    a.maxq = sh->max_q;
    a.maxq2 = sqrt_threshold(sh->max_q);
    a.vpdq = (float)sh->voxel_per_dq;
    a.ab = (int)sh->size_ab;
    a.sc = (int)sh->size_c;
    a.cab = (a.ab - 1) / 2;
    a.cc = (a.sc - 1) / 2;
    a.ka = (int)sh->k_a;
    a.kb = (int)sh->k_b;
    a.kc = (int)sh->k_c;
    const dim3 grid((unsigned)((npix + DTILE - 1) / DTILE), (nrows + DTILE - 1) / DTILE);
    if (interp == 0)
        cq_rows_kernel<0><<<grid, DTILE, 0, as_stream(stream)>>>(a, d_rows, nrows);
    else
        cq_rows_kernel<1><<<grid, DTILE, 0, as_stream(stream)>>>(a, d_rows, nrows);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}

iac_status iac_ac1d_cq_rows(iac_ctx *ctx, const float *d_I, const float *d_kmap, uint64_t npix,
                            const uint32_t *d_rows, uint32_t nrows, const iac_ac1d_shape *sh, int interp,
                            double mult, uint64_t *d_hist, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx && d_I && d_kmap && sh && d_hist && d_rows, "iac_ac1d_cq_rows: NULL argument");
    IAC_REQUIRE(interp == 0 || interp == 1, "interpolation must be 0 or 1");
    IAC_REQUIRE(npix > 0 && npix < (1ull << 32), "iac_ac1d_cq_rows: pixel count out of range");
    IAC_REQUIRE(nrows >= 1, "iac_ac1d_cq_rows: no rows");
    IAC_REQUIRE(sh->size >= 3 && sh->size <= 24576, "AC1D size %u out of range [3, 24576]", sh->size);
    IAC_REQUIRE(mult > 0, "multiplicator must be positive");
    DeviceGuard g(ctx->device);
    DenseArgs a{};
    a.I = d_I;
    a.K = d_kmap;
    a.npix = npix;
    a.mult = mult;
    a.mult_int = (mult >= 1.0 && mult < 536870912.0 && mult == std::floor(mult)) ? (uint32_t)mult : 0u;
    a.counters = ctx->d_counters;
    a.out = (unsigned long long *)d_hist;
    a.maxq = sh->max_q;
    a.hsize = sh->size;
    a.dq = sh->dq_per_step;
    void *scr = nullptr;
    iac_status st = stream_scratch(ctx, stream, SLOT_AUX0, 256, &scr);
    if (st != IAC_OK) return st;
    a.queue = (unsigned long long *)scr;
    cudaStream_t s = as_stream(stream);
    IAC_CUDA(cudaMemsetAsync(a.queue, 0, sizeof(unsigned long long), s));
    const size_t smem = sizeof(unsigned long long) * sh->size;
    auto k = interp == 0 ? ac1d_rows_kernel<0> : ac1d_rows_kernel<1>;
    IAC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<ctx->sm_count * 4, DTILE, smem, s>>>(a, d_rows, nrows);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}

}  // extern "C"
