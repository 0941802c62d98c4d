// denoise_kernels.cu -- kernels of the mesh denoiser (no reference
// counterpart): 3x3x3 convolutions as implicit GEMM on the BF16 tensor cores
// with FP32 accumulation, their data and weight gradients, pooling, the
// residual 1x1 head fused with the MSE loss, AdamW, and patch extraction.
//
// Implicit GEMM.  A CTA owns TILE_M = 128 consecutive voxels (GEMM rows) and
// all output channels (GEMM N = cout).  The K loop runs over the 27 taps; one
// pipeline stage holds one tap: the 128 shifted input rows x cin channels (A)
// and the tap's cout x cin weights (B).  Rows are gathered with 16-byte
// cp.async, out-of-volume neighbours zero-filled by the copy itself; the
// channel concatenation and the nearest 2x upsampling of the decoder inputs
// are folded into the gather, so neither is materialised.
//
// Shared-memory layout of a stage operand: [k-chunk][row][8 channels], one
// 16-byte row segment per (row, k-chunk).  Eight consecutive rows of one
// chunk form a contiguous 128-byte "core matrix", which is the canonical
// K-major, non-swizzled operand layout of tcgen05.mma (stride between 8-row
// groups = 128 B, stride between the two k-chunks of a K=16 step = rows*16 B)
// and a bank-conflict-free ldmatrix source for mma.sync.
//
// Two backends compute the same GEMM:
//   backend 0, tcgen05: one thread issues tcgen05.mma (M=128, N=cout, K=16)
//     into a TMEM accumulator; each stage's MMAs commit to an mbarrier that
//     releases the stage for the next cp.async; the epilogue reads TMEM with
//     tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = its 32 voxels);
//   backend 1, mma.sync.m16n8k16: four warps of 32 voxels x cout each.
// Backend 0 (the default, conv_slab_kernel) stages each input row once per
// (tile, dz) instead of once per tap; backend 2 is the per-tap tcgen05 form.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <utility>

#include "denoise_internal.cuh"

namespace iac {
namespace dn {

// kernels launched by this host thread since the last take_launches()
static thread_local uint64_t launch_count = 0;
uint64_t take_launches()
{
    const uint64_t n = launch_count;
    launch_count = 0;
    return n;
}

// --------------------------------------------------------------------------
// PTX helpers
// --------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t addr, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(addr), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t addr, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait: false after ~2^20 polls (each try_wait itself suspends for a
// bounded time), so a lost arrival ends the kernel with an error instead of
// hanging the GPU
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity)
{
    for (uint32_t i = 0; i < (1u << 20); i++)
        if (mbar_try_wait(addr, parity)) return true;
    return false;
}

__device__ __forceinline__ void tc_fence_before()
{
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after()
{
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(dst_smem),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols)
                 : "memory");
}
// D[tmem] (+)= A[smem] * B[smem]^T, kind::f16 (bf16 inputs, fp32 accumulator)
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
        "[%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15])
        : "r"(taddr)
        : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

// shared-memory matrix descriptor: K-major, no swizzle; lbo = byte stride
// between the two 8-element k-chunks of a K=16 step, sbo = byte stride between
// 8-row groups; bits 46-47 = 1 (descriptor version of sm_100)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// K-major operand with the 32-byte swizzle: rows of 16 bf16 (32 bytes, the two
// 16-byte halves exchanged in rows 4-7 of every 8), 8-row groups 256 bytes
// apart (SBO), layout type 6 at bit 61, base offset 0.  The swizzle acts on
// absolute shared-memory address bits, as the TMA's SWIZZLE_32B writes them,
// so the start may sit at any row (checked for row offsets 0 .. 67).
__device__ __forceinline__ uint64_t smem_desc_sw32(uint32_t addr)
{
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | (1ull << 16) | ((uint64_t)(256u >> 4) << 32) | (1ull << 46) |
           (6ull << 61);
}
// MN-major operand with rows of 32 or 64 bytes (16 or 32 M elements of one K
// index, the 32- or 64-byte swizzle), M blocks `mblock` bytes apart (LBO),
// 8-row groups 8 rows apart (SBO), layout type 6 or 4; as with the K-major
// operands the start may sit at any row (checked for both swizzles)
__device__ __forceinline__ uint64_t smem_desc_swz_mn(uint32_t addr, uint32_t rowbytes, uint32_t mblock)
{
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)((mblock >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((8u * rowbytes) >> 4) << 32) | (1ull << 46) | ((rowbytes == 32 ? 6ull : 4ull) << 61);
}
// instruction descriptor, kind::f16: D fp32 (bits 4-5 = 1), A and B bf16
// (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&h);
}

// --------------------------------------------------------------------------
// voxel decomposition and the shared gather of shifted input rows
// --------------------------------------------------------------------------
struct Vox {
    int n, z, y, x;
    bool ok;
};
__device__ __forceinline__ Vox decode(long long v, int D, int H, int W, long long V)
{
    Vox q;
    q.ok = v < V;
    if (!q.ok) v = 0;
    if (V < (1ll << 31)) {  // 32-bit divisions where the index fits
        const uint32_t u = (uint32_t)v;
        const uint32_t r1 = u / (uint32_t)W, r2 = r1 / (uint32_t)H;
        q.x = (int)(u - r1 * (uint32_t)W);
        q.y = (int)(r1 - r2 * (uint32_t)H);
        q.z = (int)(r2 % (uint32_t)D);
        q.n = (int)(r2 / (uint32_t)D);
        return q;
    }
    q.x = (int)(v % W);
    long long r = v / W;
    q.y = (int)(r % H);
    r /= H;
    q.z = (int)(r % D);
    q.n = (int)(r / D);
    return q;
}

// rows of X (concat of upsampled src0 and src1) shifted by tap, into the
// stage operand at sA ([cin/8][TILE_M][16 B]); zero-filled outside the volume
template <int CIN>
__device__ __forceinline__ void gather_rows(uint32_t sA, const bf16 *src0, const bf16 *src1, int c0, int c1,
                                            int up0, int D, int H, int W, const Vox &q, int row, int tap)
{
    const int z = q.z + tap / 9 - 1, y = q.y + (tap / 3) % 3 - 1, x = q.x + tap % 3 - 1;
    const bool ok = q.ok && (unsigned)z < (unsigned)D && (unsigned)y < (unsigned)H && (unsigned)x < (unsigned)W;
    const int n0 = c0 >> 3;
    const bf16 *p0 = src0, *p1 = src1;
    if (ok) {
        if (c0) {
            if (up0)
                p0 = src0 + ((((long long)q.n * (D >> 1) + (z >> 1)) * (H >> 1) + (y >> 1)) * (W >> 1) + (x >> 1)) * c0;
            else
                p0 = src0 + ((((long long)q.n * D + z) * H + y) * W + x) * c0;
        }
        if (c1) p1 = src1 + ((((long long)q.n * D + z) * H + y) * W + x) * c1;
    }
    const uint32_t bytes = ok ? 16u : 0u;
#pragma unroll
    for (int c = 0; c < CIN / 8; c++) {
        const bf16 *src = c < n0 ? p0 + c * 8 : p1 + (c - n0) * 8;
        cp_async16(sA + (uint32_t)((c * TILE_M + row) * 16), src, bytes);
    }
}

template <int CIN, int COUT>
__device__ __forceinline__ void load_weights(uint32_t sB, const bf16 *w, int tap, int tid)
{
    const bf16 *src = w + (size_t)tap * CIN * COUT;
    for (int i = tid; i < COUT * CIN / 8; i += CONV_THREADS) cp_async16(sB + i * 16, src + i * 8, 16);
}

// o[j] = 0 where the forward activation y (8 bf16 at y8) is not positive: the
// ReLU derivative applied to a data gradient in the epilogue that produces it
__device__ __forceinline__ void mask8(const bf16 *y8, float *o)
{
    const uint4 raw = *reinterpret_cast<const uint4 *>(y8);
    const uint32_t w[4] = {raw.x, raw.y, raw.z, raw.w};
#pragma unroll
    for (int j = 0; j < 4; j++) {
        // a bf16 is positive when its sign bit is clear and it is not +0
        if ((w[j] & 0x8000u) || !(w[j] & 0x7FFFu)) o[2 * j] = 0.0f;
        if ((w[j] & 0x80000000u) || !(w[j] & 0x7FFF0000u)) o[2 * j + 1] = 0.0f;
    }
}

// where output channels c .. of voxel v go: y ([V][cout]), or with a split
// output y ([V][split]) below `split` and y2 ([V][cout - split]) from it
__device__ __forceinline__ bf16 *out_ptr(const ConvArgs &a, int cout, long long v, int c)
{
    if (!a.y2) return a.y + v * cout + c;
    return c < a.split ? a.y + v * a.split + c : a.y2 + v * (cout - a.split) + (c - a.split);
}

// epilogue for one output row segment of 8 channels with the bias already in
// registers (b: channels c .. c+7): ReLU, bf16 (+fp32)
__device__ __forceinline__ void store8_b(const ConvArgs &a, int cout, long long v, int c, const float *val,
                                         const float *b)
{
    float o[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const float t = val[j] + b[j];
        o[j] = a.relu ? fmaxf(t, 0.0f) : t;
    }
    if (a.mask_y) mask8(a.mask_y + v * cout + c, o);
    uint4 pk;
    pk.x = pack_bf16(o[0], o[1]);
    pk.y = pack_bf16(o[2], o[3]);
    pk.z = pack_bf16(o[4], o[5]);
    pk.w = pack_bf16(o[6], o[7]);
    *reinterpret_cast<uint4 *>(out_ptr(a, cout, v, c)) = pk;
    if (a.y32) {
        float4 *d = reinterpret_cast<float4 *>(a.y32 + v * cout + c);
        d[0] = make_float4(o[0], o[1], o[2], o[3]);
        d[1] = make_float4(o[4], o[5], o[6], o[7]);
    }
}

// store8_b with the ReLU mask of the 8 channels already loaded (mk, when a.mask_y is set)
__device__ __forceinline__ void store8_bm(const ConvArgs &a, int cout, long long v, int c, const float *val,
                                          const float *b, uint4 mk)
{
    float o[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const float t = val[j] + b[j];
        o[j] = a.relu ? fmaxf(t, 0.0f) : t;
    }
    if (a.mask_y) {
        const uint32_t w[4] = {mk.x, mk.y, mk.z, mk.w};
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if ((w[j] & 0x8000u) || !(w[j] & 0x7FFFu)) o[2 * j] = 0.0f;
            if ((w[j] & 0x80000000u) || !(w[j] & 0x7FFF0000u)) o[2 * j + 1] = 0.0f;
        }
    }
    uint4 pk;
    pk.x = pack_bf16(o[0], o[1]);
    pk.y = pack_bf16(o[2], o[3]);
    pk.z = pack_bf16(o[4], o[5]);
    pk.w = pack_bf16(o[6], o[7]);
    *reinterpret_cast<uint4 *>(out_ptr(a, cout, v, c)) = pk;
    if (a.y32) {
        float4 *d = reinterpret_cast<float4 *>(a.y32 + v * cout + c);
        d[0] = make_float4(o[0], o[1], o[2], o[3]);
        d[1] = make_float4(o[4], o[5], o[6], o[7]);
    }
}

// epilogue for one output row segment of 8 channels: bias, ReLU, bf16 (+fp32)
__device__ __forceinline__ void store8(const ConvArgs &a, int cout, long long v, int c, const float *val)
{
    float o[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        float t = val[j] + (a.bias ? a.bias[c + j] : 0.0f);
        o[j] = a.relu ? fmaxf(t, 0.0f) : t;
    }
    if (a.mask_y) mask8(a.mask_y + v * cout + c, o);
    uint4 pk;
    pk.x = pack_bf16(o[0], o[1]);
    pk.y = pack_bf16(o[2], o[3]);
    pk.z = pack_bf16(o[4], o[5]);
    pk.w = pack_bf16(o[6], o[7]);
    *reinterpret_cast<uint4 *>(out_ptr(a, cout, v, c)) = pk;
    if (a.y32) {
        float4 *d = reinterpret_cast<float4 *>(a.y32 + v * cout + c);
        d[0] = make_float4(o[0], o[1], o[2], o[3]);
        d[1] = make_float4(o[4], o[5], o[6], o[7]);
    }
}

// --------------------------------------------------------------------------
// backend 0: tcgen05.mma with a TMEM accumulator
// --------------------------------------------------------------------------
template <int CIN, int COUT>
struct TcCfg {
    static constexpr int S = 4;   // stages
    static constexpr int PF = 2;  // taps in flight ahead of the one being multiplied
    static constexpr uint32_t A_BYTES = TILE_M * CIN * 2;
    static constexpr uint32_t B_BYTES = COUT * CIN * 2;
    static constexpr uint32_t STAGE = A_BYTES + B_BYTES;
    static constexpr uint32_t SMEM = S * STAGE;
    static constexpr uint32_t TCOLS = COUT <= 32 ? 32 : (COUT <= 64 ? 64 : 128);
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(CONV_THREADS) conv_tc_kernel(const ConvArgs a)
{
    using Cfg = TcCfg<CIN, COUT>;
    static_assert(COUT % 16 == 0 && COUT <= 256 && CIN % 16 == 0, "tcgen05 M=128 needs N % 16 == 0");
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar[Cfg::S];
    __shared__ uint32_t s_tmem;
    __shared__ int s_err;
    const int tid = threadIdx.x, warp = tid >> 5;
    const long long v0 = (long long)blockIdx.x * TILE_M;
    const Vox q = decode(v0 + tid, a.D, a.H, a.W, a.V);
    const uint32_t sbase = smem_u32(smem);
    if (tid == 0) {
        for (int s = 0; s < Cfg::S; s++) mbar_init(smem_u32(&mbar[s]), 1);
        fence_mbar_init();
        s_err = 0;
    }
    if (warp == 0) {
        tmem_alloc(smem_u32(&s_tmem), Cfg::TCOLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    constexpr uint32_t IDESC = idesc_bf16(TILE_M, COUT);

    for (int t = 0; t < Cfg::PF; t++) {
        const uint32_t sA = sbase + t * Cfg::STAGE;
        gather_rows<CIN>(sA, a.src0, a.src1, a.c0, a.c1, a.up0, a.D, a.H, a.W, q, tid, t);
        load_weights<CIN, COUT>(sA + Cfg::A_BYTES, a.w, t, tid);
        cp_async_commit();
    }
    int issued = 0;  // taps whose MMAs were issued
    for (int t = 0; t < 27; t++) {
        const int tn = t + Cfg::PF;
        if (tn < 27) {
            const int st = tn % Cfg::S;
            // the stage was last read by the MMAs of tap tn - S
            if (tn >= Cfg::S && !mbar_wait(smem_u32(&mbar[st]), ((tn - Cfg::S) / Cfg::S) & 1)) s_err = 1;
            const uint32_t sA = sbase + st * Cfg::STAGE;
            gather_rows<CIN>(sA, a.src0, a.src1, a.c0, a.c1, a.up0, a.D, a.H, a.W, q, tid, tn);
            load_weights<CIN, COUT>(sA + Cfg::A_BYTES, a.w, tn, tid);
        }
        cp_async_commit();
        cp_async_wait<Cfg::PF>();
        fence_proxy_async();
        __syncthreads();
        if (s_err) break;
        if (tid == 0) {
            tc_fence_after();
            const uint32_t sA = sbase + (t % Cfg::S) * Cfg::STAGE, sB = sA + Cfg::A_BYTES;
#pragma unroll
            for (int k = 0; k < CIN / 16; k++) {
                const uint64_t da = smem_desc(sA + k * 2 * (TILE_M * 16), TILE_M * 16, 128);
                const uint64_t db = smem_desc(sB + k * 2 * (COUT * 16), COUT * 16, 128);
                umma_bf16(tmem, da, db, IDESC, (t > 0 || k > 0) ? 1u : 0u);
            }
            umma_commit(smem_u32(&mbar[t % Cfg::S]));
        }
        issued = t + 1;
    }
    cp_async_wait_all();
    // the last commit arrives once every MMA issued before it has completed
    const bool done =
        issued > 0 && mbar_wait(smem_u32(&mbar[(issued - 1) % Cfg::S]), ((issued - 1) / Cfg::S) & 1);
    if ((s_err || !done) && tid == 0) note_timeout(a.counters, SITE_CONV_TAP);
    tc_fence_after();
    __syncthreads();
    if (!s_err && done && issued == 27) {  // CTA-uniform: the TMEM loads are warp-collective
        const long long v = v0 + tid;
#pragma unroll
        for (int c = 0; c < COUT; c += 16) {
            uint32_t r[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c, r);
            tmem_wait_ld();
            if (q.ok) {
                float f[16];
#pragma unroll
                for (int j = 0; j < 16; j++) f[j] = __uint_as_float(r[j]);
                store8(a, COUT, v, c, f);
                store8(a, COUT, v, c + 8, f + 8);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, Cfg::TCOLS);
}

// --------------------------------------------------------------------------
// backend 1: mma.sync.m16n8k16 (warp w: rows 32w..32w+31, all cout)
// --------------------------------------------------------------------------
template <int CIN, int COUT>
struct MmaCfg {
    static constexpr int S = 3;
    static constexpr int PF = S - 1;
    static constexpr uint32_t A_BYTES = TILE_M * CIN * 2;
    static constexpr uint32_t B_BYTES = COUT * CIN * 2;
    static constexpr uint32_t STAGE = A_BYTES + B_BYTES;
    static constexpr uint32_t SMEM = S * STAGE;
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(CONV_THREADS) conv_mma_kernel(const ConvArgs a)
{
    using Cfg = MmaCfg<CIN, COUT>;
    constexpr int NT = COUT / 8;
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long v0 = (long long)blockIdx.x * TILE_M;
    const Vox q = decode(v0 + tid, a.D, a.H, a.W, a.V);
    const uint32_t sbase = smem_u32(smem);
    float acc[2][NT][4];
#pragma unroll
    for (int m = 0; m < 2; m++)
#pragma unroll
        for (int n = 0; n < NT; n++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[m][n][j] = 0.0f;

    for (int t = 0; t < Cfg::PF; t++) {
        const uint32_t sA = sbase + t * Cfg::STAGE;
        gather_rows<CIN>(sA, a.src0, a.src1, a.c0, a.c1, a.up0, a.D, a.H, a.W, q, tid, t);
        load_weights<CIN, COUT>(sA + Cfg::A_BYTES, a.w, t, tid);
        cp_async_commit();
    }
    for (int t = 0; t < 27; t++) {
        const int tn = t + Cfg::PF;
        if (tn < 27) {
            __syncthreads();  // every warp is done with tap t - 1, whose stage is reused
            const uint32_t sA = sbase + (tn % Cfg::S) * Cfg::STAGE;
            gather_rows<CIN>(sA, a.src0, a.src1, a.c0, a.c1, a.up0, a.D, a.H, a.W, q, tid, tn);
            load_weights<CIN, COUT>(sA + Cfg::A_BYTES, a.w, tn, tid);
        }
        cp_async_commit();
        cp_async_wait<Cfg::PF>();
        __syncthreads();
        const uint32_t sA = sbase + (t % Cfg::S) * Cfg::STAGE, sB = sA + Cfg::A_BYTES;
#pragma unroll
        for (int k = 0; k < CIN / 16; k++) {
            uint32_t af[2][4];
#pragma unroll
            for (int m = 0; m < 2; m++) {
                const int row = warp * 32 + m * 16 + (lane & 15);
                const int ch = 2 * k + (lane >> 4);
                ldsm_x4(sA + (uint32_t)((ch * TILE_M + row) * 16), af[m][0], af[m][1], af[m][2], af[m][3]);
            }
#pragma unroll
            for (int n2 = 0; n2 < NT / 2; n2++) {
                uint32_t b0, b1, b2, b3;
                const int nrow = n2 * 16 + (lane & 7) + ((lane >> 4) << 3);
                const int ch = 2 * k + ((lane >> 3) & 1);
                ldsm_x4(sB + (uint32_t)((ch * COUT + nrow) * 16), b0, b1, b2, b3);
#pragma unroll
                for (int m = 0; m < 2; m++) {
                    mma_bf16(acc[m][2 * n2], af[m][0], af[m][1], af[m][2], af[m][3], b0, b1);
                    mma_bf16(acc[m][2 * n2 + 1], af[m][0], af[m][1], af[m][2], af[m][3], b2, b3);
                }
            }
        }
    }
    cp_async_wait_all();
    // epilogue: thread holds rows g, g+8 of each m16 tile, columns 2t, 2t+1 of each n8 tile
    const int g = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int m = 0; m < 2; m++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const long long v = v0 + warp * 32 + m * 16 + g + 8 * h;
            if (v >= a.V) continue;
#pragma unroll
            for (int n = 0; n < NT; n++) {
                const int c = n * 8 + 2 * tq;
                float o0 = acc[m][n][2 * h] + (a.bias ? a.bias[c] : 0.0f);
                float o1 = acc[m][n][2 * h + 1] + (a.bias ? a.bias[c + 1] : 0.0f);
                if (a.relu) {
                    o0 = fmaxf(o0, 0.0f);
                    o1 = fmaxf(o1, 0.0f);
                }
                if (a.mask_y) {  // ReLU derivative: 0 where the forward activation is not positive
                    const uint32_t w = *reinterpret_cast<const uint32_t *>(a.mask_y + v * COUT + c);
                    if ((w & 0x8000u) || !(w & 0x7FFFu)) o0 = 0.0f;
                    if ((w & 0x80000000u) || !(w & 0x7FFF0000u)) o1 = 0.0f;
                }
                const uint32_t pk = pack_bf16(o0, o1);
                *reinterpret_cast<uint32_t *>(out_ptr(a, COUT, v, c)) = pk;
                if (a.y32) *reinterpret_cast<float2 *>(a.y32 + v * COUT + c) = make_float2(o0, o1);
            }
        }
}

// --------------------------------------------------------------------------
// backend 0: tcgen05 on padded-row slabs (default)
//
// The output positions of one z-plane are numbered q = y (W+2) + x', x' = x+1,
// so every row carries its two halo columns; a tile is 128 consecutive q.  For
// tap (dz, dy, dx) the A row of position q is q + dy (W+2) + dx in plane z+dz,
// so the nine (dy, dx) taps of one dz read one slab of R = 128 + 2 (W+2) + 2
// consecutive padded positions at nine row offsets: each tap's operand is the
// slab's descriptor advanced by 16 B per row of shift (core matrices are any
// eight consecutive 16-byte rows).  A tile takes three stages (dz = -1, 0, 1),
// each the slab plus that dz's nine weight tiles; halo-column outputs are
// computed and dropped (2/(W+2) of the MACs).  CTAs are persistent over tiles
// and the TMEM accumulator is double-buffered, so the epilogue of tile k runs
// while the MMAs of tile k+1 execute.
// --------------------------------------------------------------------------
struct SlabGeom {
    int Wp;            // W + 2
    int R;             // slab rows
    int T;             // tiles per plane
    long long ntiles;  // nb * D * T
    uint32_t slab_bytes, stage_bytes;
    int S;             // stages in the ring (2..4)
};

// R consecutive padded positions q0 - (W+2) - 1 ... of plane z (batch item n)
// of X = concat(upsampled src0, src1) into sS ([cin/8][R][16 B]); zero rows
// for halo columns, rows outside the plane and planes outside the volume
template <int CIN>
__device__ __forceinline__ void slab_rows(uint32_t sS, const SlabGeom &g, int q0, int n, int z, const bf16 *src0,
                                          const bf16 *src1, int c0, int c1, int up0, int D, int H, int W, int tid)
{
    const bool zok = (unsigned)z < (unsigned)D;
    const int HW = H * W;
    const int n0 = c0 >> 3;
    for (int r = tid; r < g.R; r += CONV_THREADS) {
        const int q = q0 - g.Wp - 1 + r;  // >= -Wp - 1
        const int y = q >= 0 ? q / g.Wp : -1;
        const int xp = q - y * g.Wp;
        const bool ok = zok && y >= 0 && y < H && xp >= 1 && xp <= W;
        const int x = xp - 1;
        const bf16 *p0 = src0, *p1 = src1;
        if (ok) {
            if (c0) {
                if (up0)
                    p0 = src0 + ((((long long)n * (D >> 1) + (z >> 1)) * (H >> 1) + (y >> 1)) * (W >> 1) + (x >> 1)) * c0;
                else
                    p0 = src0 + (((long long)n * D + z) * HW + (long long)y * W + x) * c0;
            }
            p1 = src1 + (((long long)n * D + z) * HW + (long long)y * W + x) * c1;
        }
#pragma unroll
        for (int c = 0; c < CIN / 8; c++) {
            const bf16 *src = c < n0 ? p0 + c * 8 : p1 + (c - n0) * 8;
            cp_async16(sS + (uint32_t)((c * g.R + r) * 16), src, ok ? 16u : 0u);
        }
    }
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(CONV_THREADS) conv_slab_kernel(const ConvArgs a, const SlabGeom g)
{
    constexpr uint32_t TCOLS = 2 * COUT <= 32 ? 32 : (2 * COUT <= 64 ? 64 : (2 * COUT <= 128 ? 128 : 256));
    constexpr uint32_t IDESC = idesc_bf16(TILE_M, COUT);
    constexpr uint32_t WT_BYTES = COUT * CIN * 2;  // one tap's weight tile
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar[4];
    __shared__ __align__(8) uint64_t accbar[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_err;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t sbase = smem_u32(smem);
    if (tid == 0) {
        for (int k = 0; k < 4; k++) mbar_init(smem_u32(&mbar[k]), 1);
        mbar_init(smem_u32(&accbar[0]), 1);
        mbar_init(smem_u32(&accbar[1]), 1);
        fence_mbar_init();
        s_err = 0;
    }
    if (warp == 0) {
        tmem_alloc(smem_u32(&s_tmem), TCOLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const long long my_tiles =
        blockIdx.x < g.ntiles ? (g.ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    const long long nst = 3 * my_tiles;
    const int S = g.S, PF = S >= 3 ? 2 : 1;
    const int HW = a.H * a.W;

    auto load_stage = [&](long long i) {
        const long long tile = blockIdx.x + (i / 3) * (long long)gridDim.x;
        const int dz = (int)(i % 3) - 1;
        const uint32_t sS = sbase + (uint32_t)(i % S) * g.stage_bytes;
        const uint32_t sW = sS + g.slab_bytes;
        const long long plane = tile / g.T;  // n * D + z
        slab_rows<CIN>(sS, g, (int)(tile % g.T) * TILE_M, (int)(plane / a.D), (int)(plane % a.D) + dz, a.src0,
                       a.src1, a.c0, a.c1, a.up0, a.D, a.H, a.W, tid);
        const bf16 *wsrc = a.w + (size_t)(9 * (dz + 1)) * CIN * COUT;
        for (int k = tid; k < (int)(9 * WT_BYTES / 16); k += CONV_THREADS) cp_async16(sW + k * 16, wsrc + k * 8, 16);
    };

    auto epilogue = [&](long long k) {
        const long long tile = blockIdx.x + k * (long long)gridDim.x;
        const bool ok = mbar_wait(smem_u32(&accbar[k & 1]), (uint32_t)((k >> 1) & 1));
        if (!ok) s_err = 1;
        __syncwarp();  // converged for the warp-collective TMEM loads
        tc_fence_after();
        const long long plane = tile / g.T;
        const int q = (int)(tile % g.T) * TILE_M + tid;
        const int y = q / g.Wp, xp = q - (q / g.Wp) * g.Wp;
        const bool valid = ok && y < a.H && xp >= 1 && xp <= a.W;
        const long long v = plane * HW + (long long)y * a.W + (xp - 1);
#pragma unroll
        for (int c = 0; c < COUT; c += 16) {
            uint32_t r[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((k & 1) * COUT + c), r);
            tmem_wait_ld();
            if (valid) {
                float f[16];
#pragma unroll
                for (int j = 0; j < 16; j++) f[j] = __uint_as_float(r[j]);
                store8(a, COUT, v, c, f);
                store8(a, COUT, v, c + 8, f + 8);
            }
        }
        tc_fence_before();
    };

    for (long long i = 0; i < PF && i < nst; i++) {
        load_stage(i);
        cp_async_commit();
    }
    for (long long i = 0; i < nst; i++) {
        const long long j = i + PF;
        if (j < nst) {
            // the slot was last read by the MMAs of stage j - S
            if (j >= S && !mbar_wait(smem_u32(&mbar[j % S]), (uint32_t)(((j - S) / S) & 1))) s_err = 1;
            load_stage(j);
        }
        cp_async_commit();
        if (PF == 2)
            cp_async_wait<2>();
        else
            cp_async_wait<1>();
        fence_proxy_async();
        __syncthreads();
        if (s_err) break;
        const long long k = i / 3;
        const int dzi = (int)(i % 3);
        if (tid == 0) {
            tc_fence_after();
            const uint32_t sS = sbase + (uint32_t)(i % S) * g.stage_bytes, sW = sS + g.slab_bytes;
            const uint32_t dcol = tmem + (uint32_t)((k & 1) * COUT);
#pragma unroll 1
            for (int t = 0; t < 9; t++) {
                const uint32_t r0 = (uint32_t)(g.Wp + 1 + (t / 3 - 1) * g.Wp + (t % 3 - 1));
#pragma unroll
                for (int kk = 0; kk < CIN / 16; kk++) {
                    const uint64_t da = smem_desc(sS + (uint32_t)(kk * 2 * g.R * 16) + r0 * 16, (uint32_t)g.R * 16, 128);
                    const uint64_t db = smem_desc(sW + t * WT_BYTES + kk * 2 * (COUT * 16), COUT * 16, 128);
                    umma_bf16(dcol, da, db, IDESC, (dzi > 0 || t > 0 || kk > 0) ? 1u : 0u);
                }
            }
            umma_commit(smem_u32(&mbar[i % S]));
            if (dzi == 2) umma_commit(smem_u32(&accbar[k & 1]));
        }
        if (dzi == 0 && k > 0) epilogue(k - 1);
    }
    cp_async_wait_all();
    __syncthreads();
    if (!s_err && nst > 0) epilogue(my_tiles - 1);
    if (s_err && tid == 0) note_timeout(a.counters, SITE_CONV_SLAB);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, TCOLS);
}

template <int CIN, int COUT>
static bool launch_slab(const ConvArgs &a, cudaStream_t s, cudaError_t &err)
{
    SlabGeom g{};
    g.Wp = a.W + 2;
    g.R = TILE_M + 2 * g.Wp + 2;
    g.T = (a.H * g.Wp + TILE_M - 1) / TILE_M;
    const long long nb = a.V / ((long long)a.D * a.H * a.W);
    g.ntiles = nb * a.D * g.T;
    g.slab_bytes = (uint32_t)g.R * CIN * 2;
    g.stage_bytes = g.slab_bytes + 9u * COUT * CIN * 2;
    const uint32_t budget = 227u * 1024u - 512u;
    g.S = (int)std::min<uint32_t>(4u, budget / g.stage_bytes);
    if (g.S < 2 || g.ntiles == 0) return false;
    const uint32_t smem = (uint32_t)g.S * g.stage_bytes;
    err = cudaFuncSetAttribute(conv_slab_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return true;
    // prefer the largest shared-memory carveout: several slab CTAs per SM
    err = cudaFuncSetAttribute(conv_slab_kernel<CIN, COUT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                               (int)cudaSharedmemCarveoutMaxShared);
    if (err != cudaSuccess) return true;
    // resident CTAs per SM from the SM's shared memory, registers and TMEM
    // (512 columns); the occupancy calculator answers 1 for this kernel
    int dev = 0, smem_sm = 0, reserved = 0, regs_sm = 0;
    cudaFuncAttributes fa{};
    if ((err = cudaGetDevice(&dev)) != cudaSuccess) return true;
    if ((err = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess)
        return true;
    if ((err = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev)) != cudaSuccess)
        return true;
    if ((err = cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev)) != cudaSuccess)
        return true;
    if ((err = cudaFuncGetAttributes(&fa, conv_slab_kernel<CIN, COUT>)) != cudaSuccess) return true;
    constexpr int TCOLS = 2 * COUT <= 32 ? 32 : (2 * COUT <= 64 ? 64 : (2 * COUT <= 128 ? 128 : 256));
    int per_sm = smem_sm / (int)(smem + fa.sharedSizeBytes + reserved);
    per_sm = std::min(per_sm, regs_sm / (std::max(1, fa.numRegs) * CONV_THREADS));
    per_sm = std::min(per_sm, 512 / TCOLS);
    per_sm = std::min(per_sm, 16);
    const long long grid = std::min<long long>(g.ntiles, (long long)std::max(1, per_sm) * std::max(1, a.sms));
    ++launch_count;
    conv_slab_kernel<CIN, COUT><<<(unsigned)grid, CONV_THREADS, smem, s>>>(a, g);
    err = cudaGetLastError();
    return true;
}

// --------------------------------------------------------------------------
// backend 0 with plain inputs: warp-specialised, TMA-fed tcgen05 convolution.
//
// Same padded-position tiles and slab operands as conv_slab_kernel, but a
// stage is filled by the Tensor Memory Accelerator: one 5-D box (8 channels x
// W+2 columns x NR rows x 1 plane x 1 item, starting at column -1) per
// 8-channel chunk, whose out-of-volume elements (halo columns, rows above and
// below the plane, planes outside the volume) arrive as zeros.  Warp 4 (one
// lane) produces stages, warp 5 (one lane) issues tcgen05.mma, warps 0-3 drain
// the double-buffered TMEM accumulator; the roles meet only at mbarriers
// (full/empty per stage, full/empty per accumulator), every wait bounded.
// NI = 3: warps 5-7 issue, warp 5 + d the stage of dz = d - 1 of every tile
// into its own accumulator, and the epilogue adds the three (a tcgen05.mma
// costs its issuing thread ~150 cycles whatever its shape while the tensor
// pipe accepts one every ~40, so several issuers keep the pipe busy).
// Weights stay resident in shared memory when all 27 taps fit, else each
// stage carries its dz's nine taps (one bulk copy).
// --------------------------------------------------------------------------
struct TmaGeom {
    int Wp, NR;             // padded row length, padded rows per slab
    int T;                  // tiles per plane
    long long ntiles;
    uint32_t plane_bytes;   // one 8-channel chunk of a slab (multiple of 128)
    uint32_t box_bytes;     // bytes one box delivers (16 * Wp * NR)
    uint32_t slab_bytes;    // cin/8 planes
    uint32_t wstage_bytes;  // weights carried per stage (0: resident)
    uint32_t stage_bytes;
    uint32_t wres_bytes;    // shared memory reserved for resident weights (0: per stage)
    uint32_t wcopy_bytes;   // bytes of the resident weights copied
    int S;
    int ZC;                 // z-column kernel: output planes per work item
    long long nitems;       // z-column kernel: nb * T * ceil(D / ZC) work items
};

__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            int c4, uint32_t mbar)
{
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5, %6}], [%7];\n" ::"r"(dst),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(mbar)
        : "memory");
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t mbar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mbar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(mbar) : "memory");
}
// bounded wait that also gives up once another role has flagged an error
__device__ __forceinline__ bool mbar_wait_flag(uint32_t addr, uint32_t parity, volatile int *err)
{
    for (uint32_t i = 0; i < (1u << 20); i++) {
        if (mbar_try_wait(addr, parity)) return true;
        if (*err) return false;
    }
    *err = 1;
    return false;
}

__device__ __forceinline__ int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

constexpr int TMA_THREADS = 192;  // with NI issuing warps: 32 * (5 + NI)

__host__ __device__ constexpr uint32_t tma_tcols(int cols)
{
    return cols <= 32 ? 32 : (cols <= 64 ? 64 : (cols <= 128 ? 128 : (cols <= 256 ? 256 : 512)));
}

template <int CIN, int COUT, int NI>
__global__ void __launch_bounds__(256) conv_tma_kernel(const __grid_constant__ CUtensorMap xmap,
                                                       const ConvArgs a, const TmaGeom g)
{
    static_assert(NI == 1 || NI == 3, "one issuer, or one per dz");
    constexpr uint32_t TCOLS = tma_tcols(2 * NI * COUT);
    constexpr uint32_t IDESC = idesc_bf16(TILE_M, COUT);
    constexpr uint32_t WT_BYTES = COUT * CIN * 2;
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[8], empty[8], accfull[2], accempty[2], wfull;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_err;
    __shared__ long long s_issued, s_last[NI];  // stages loaded by the producer / last multiplied per issuer
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = smem_u32(smem);
    const uint32_t wbase = sbase;                   // resident weights
    const uint32_t stbase = sbase + g.wres_bytes;   // stages
    if (tid == 0) {
        for (int k = 0; k < g.S; k++) {
            mbar_init(smem_u32(&full[k]), 1);
            mbar_init(smem_u32(&empty[k]), 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(smem_u32(&accfull[b]), NI);
            mbar_init(smem_u32(&accempty[b]), 4);
        }
        mbar_init(smem_u32(&wfull), 1);
        fence_mbar_init();
        s_err = 0;
        s_issued = 0;
        for (int i = 0; i < NI; i++) s_last[i] = -1;
    }
    if (warp == 5) {
        tmem_alloc(smem_u32(&s_tmem), TCOLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const long long my_tiles =
        blockIdx.x < g.ntiles ? (g.ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    const long long nst = 3 * my_tiles;
    const int HW = a.H * a.W;

    if (warp == 4) {
        if (lane == 0) {  // producer
            if (g.wres_bytes) {
                mbar_expect_tx(smem_u32(&wfull), g.wcopy_bytes);
                bulk_load(wbase, a.w, g.wcopy_bytes, smem_u32(&wfull));
            }
            for (long long i = 0; i < nst; i++) {
                const int slot = (int)(i % g.S);
                if (i >= g.S && !mbar_wait_flag(smem_u32(&empty[slot]), (uint32_t)(((i / g.S) - 1) & 1), &s_err))
                    break;
                const long long tile = blockIdx.x + (i / 3) * (long long)gridDim.x;
                const int dz = (int)(i % 3) - 1;
                const long long plane = tile / g.T;
                const int q0 = (int)(tile % g.T) * TILE_M;
                const int n = (int)(plane / a.D), z = (int)(plane % a.D) + dz;
                const int y_lo = floor_div(q0 - g.Wp - 1, g.Wp);
                const uint32_t st = stbase + (uint32_t)slot * g.stage_bytes;
                const uint32_t fb = smem_u32(&full[slot]);
                mbar_expect_tx(fb, (CIN / 8) * g.box_bytes + g.wstage_bytes);
#pragma unroll
                for (int c = 0; c < CIN / 8; c++) tma_load_5d(st + c * g.plane_bytes, &xmap, c * 8, -1, y_lo, z, n, fb);
                if (g.wstage_bytes)
                    bulk_load(st + g.slab_bytes, a.w + (size_t)(9 * (dz + 1)) * CIN * COUT, g.wstage_bytes, fb);
                s_issued = i + 1;
            }
        }
    } else if (warp >= 5 && warp < 5 + NI) {
        const int iw = warp - 5;
        if (lane == 0) {  // MMA issuer: every stage (NI = 1) or the stages of dz = iw - 1
            bool ok = !g.wres_bytes || mbar_wait_flag(smem_u32(&wfull), 0, &s_err);
            for (long long i = iw; ok && i < nst; i += NI) {
                const int slot = (int)(i % g.S);
                if (!mbar_wait_flag(smem_u32(&full[slot]), (uint32_t)((i / g.S) & 1), &s_err)) break;
                const long long k = i / 3;
                const int dzi = (int)(i % 3);
                if ((NI == 3 || dzi == 0) && k >= 2 &&
                    !mbar_wait_flag(smem_u32(&accempty[k & 1]), (uint32_t)(((k >> 1) - 1) & 1), &s_err))
                    break;
                tc_fence_after();
                const long long tile = blockIdx.x + k * (long long)gridDim.x;
                const int q0 = (int)(tile % g.T) * TILE_M;
                const int rel = q0 - floor_div(q0 - g.Wp - 1, g.Wp) * g.Wp;  // q0 within the slab
                const uint32_t st = stbase + (uint32_t)slot * g.stage_bytes;
                const uint32_t wt = g.wres_bytes ? wbase + (uint32_t)(9 * dzi) * WT_BYTES : st + g.slab_bytes;
                const uint32_t dcol = tmem + (uint32_t)(((k & 1) * NI + (NI == 3 ? dzi : 0)) * COUT);
#pragma unroll 1
                for (int t = 0; t < 9; t++) {
                    const uint32_t r0 = (uint32_t)(rel + (t / 3 - 1) * g.Wp + (t % 3 - 1));
#pragma unroll
                    for (int kk = 0; kk < CIN / 16; kk++) {
                        const uint64_t da = smem_desc(st + (uint32_t)(2 * kk) * g.plane_bytes + r0 * 16, g.plane_bytes, 128);
                        const uint64_t db = smem_desc(wt + t * WT_BYTES + kk * 2 * (COUT * 16), COUT * 16, 128);
                        umma_bf16(dcol, da, db, IDESC, ((NI == 1 && dzi > 0) || t > 0 || kk > 0) ? 1u : 0u);
                    }
                }
                umma_commit(smem_u32(&empty[slot]));
                if (NI == 3 || dzi == 2) umma_commit(smem_u32(&accfull[k & 1]));
                s_last[iw] = i;
            }
        }
    } else {  // epilogue: warps 0-3 own TMEM lanes 32w .. 32w+31
        for (long long k = 0; k < my_tiles; k++) {
            if (!mbar_wait_flag(smem_u32(&accfull[k & 1]), (uint32_t)((k >> 1) & 1), &s_err)) break;
            __syncwarp();  // converged for the warp-collective TMEM loads
            tc_fence_after();
            const long long tile = blockIdx.x + k * (long long)gridDim.x;
            const long long plane = tile / g.T;
            const int q = (int)(tile % g.T) * TILE_M + tid;
            const int y = q / g.Wp, xp = q - (q / g.Wp) * g.Wp;
            const bool valid = y < a.H && xp >= 1 && xp <= a.W;
            const long long v = plane * HW + (long long)y * a.W + (xp - 1);
            uint32_t r[COUT];
            const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((k & 1) * NI * COUT);
#pragma unroll
            for (int c = 0; c < COUT; c += 16) {
                uint32_t (&rr)[16] = *reinterpret_cast<uint32_t(*)[16]>(&r[c]);
                tmem_ld16(lane_base + (uint32_t)c, rr);
                if constexpr (NI == 3) {  // (dz -1) + (dz 0), then + (dz +1)
                    uint32_t r1[16], r2[16];
                    tmem_ld16(lane_base + (uint32_t)(COUT + c), r1);
                    tmem_ld16(lane_base + (uint32_t)(2 * COUT + c), r2);
                    tmem_wait_ld();
#pragma unroll
                    for (int j = 0; j < 16; j++)
                        rr[j] = __float_as_uint(__fadd_rn(__fadd_rn(__uint_as_float(rr[j]), __uint_as_float(r1[j])),
                                                          __uint_as_float(r2[j])));
                }
            }
            tmem_wait_ld();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&accempty[k & 1]));
            if (valid) {
#pragma unroll
                for (int c = 0; c < COUT; c += 8) {
                    float f[8];
#pragma unroll
                    for (int j = 0; j < 8; j++) f[j] = __uint_as_float(r[c + j]);
                    store8(a, COUT, v, c, f);
                }
            }
        }
    }
    __syncthreads();
    if (s_err) {
        // after an error: let the copies and MMAs already issued finish (bounded)
        // before the shared memory and TMEM are released
        if (tid == 0) {
            note_timeout(a.counters, SITE_CONV_TMA);
            // every copy still in flight: the stages of the last S loads
            for (long long i = s_issued > g.S ? s_issued - g.S : 0; i < s_issued; i++)
                mbar_wait(smem_u32(&full[i % g.S]), (uint32_t)((i / g.S) & 1));
            // every issuer's MMAs: its last commit covers all of them
            for (int w = 0; w < NI; w++) {
                const long long i = s_last[w];
                if (i >= 0) mbar_wait(smem_u32(&empty[i % g.S]), (uint32_t)((i / g.S) & 1));
            }
        }
        __syncthreads();
    }
    if (warp == 5) {
        tc_fence_after();
        tmem_dealloc(tmem, TCOLS);
    }
}

// --------------------------------------------------------------------------
// z-column variant of conv_tma_kernel.  conv_tma_kernel stages the three
// input-plane slabs (dz = -1, 0, +1) of every output tile, so each input row
// crosses L2 -> shared memory about 8 times (3 planes x halo rows) and the
// kernel is bound by that traffic.  Here a work item is one tile position
// (n, q0) over ZC consecutive output planes z0 .. z0+ZC-1: the producer loads
// the slab of each input plane z0-1 .. z0+ZC once, and every slab feeds three
// outputs (planes p+1, p, p-1 as dz = -1, 0, +1).  Warps 5, 6, 7 issue the
// taps of dz = -1, 0, +1 (warp 5 + i uses the stage of plane z - 1 + i for
// output z) into their own accumulators; the epilogue adds the three.  Every
// issuer walks every stage in order (committing the stages it does not use),
// so a slot's parity waits stay in phase order; an issuer at stage k works on
// output k - i, so outputs k-2 .. k are in flight together and the
// accumulators rotate over NB buffers (3 per buffer, 3 * NB * COUT columns).
// Weights are resident (all 27 taps in shared memory).
// --------------------------------------------------------------------------
template <int CIN, int COUT, int NB>
__global__ void __launch_bounds__(256, 1) conv_zcol_kernel(const __grid_constant__ CUtensorMap xmap,
                                                        const ConvArgs a, const TmaGeom g)
{
    constexpr uint32_t TCOLS = tma_tcols(3 * NB * COUT);
    static_assert(3 * NB * COUT <= 512, "TMEM holds 512 columns");
    constexpr uint32_t IDESC = idesc_bf16(TILE_M, COUT);
    constexpr uint32_t WT_BYTES = COUT * CIN * 2;
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[8], empty[8], accfull[NB], accempty[NB], wfull;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_err;
    __shared__ long long s_issued, s_last[3];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = smem_u32(smem);
    const uint32_t wbase = sbase;                   // resident weights
    const uint32_t stbase = sbase + g.wres_bytes;   // stages: one input-plane slab each
    if (tid == 0) {
        for (int k = 0; k < g.S; k++) {
            mbar_init(smem_u32(&full[k]), 1);
            mbar_init(smem_u32(&empty[k]), 3);  // every issuer commits every stage
        }
        for (int b = 0; b < NB; b++) {
            mbar_init(smem_u32(&accfull[b]), 3);
            mbar_init(smem_u32(&accempty[b]), 4);
        }
        mbar_init(smem_u32(&wfull), 1);
        fence_mbar_init();
        s_err = 0;
        s_issued = 0;
        for (int i = 0; i < 3; i++) s_last[i] = -1;
    }
    if (warp == 5) {
        tmem_alloc(smem_u32(&s_tmem), TCOLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const int nzc = (a.D + g.ZC - 1) / g.ZC;  // z-chunks per column
    const int HW = a.H * a.W;
    // work item it -> batch item n, tile q0 of the plane, output planes z0 .. z1-1
    auto item = [&](long long it, int &n, int &q0, int &z0, int &z1) {
        const long long col = it / nzc;
        z0 = (int)(it % nzc) * g.ZC;
        z1 = z0 + g.ZC < a.D ? z0 + g.ZC : a.D;
        n = (int)(col / g.T);
        q0 = (int)(col % g.T) * TILE_M;
    };

    if (warp == 4) {
        if (lane == 0) {  // producer: one slab per input plane z0-1 .. z1 (planes outside the volume arrive as zeros)
            mbar_expect_tx(smem_u32(&wfull), g.wcopy_bytes);
            bulk_load(wbase, a.w, g.wcopy_bytes, smem_u32(&wfull));
            long long j = 0;
            bool ok = true;
            for (long long it = blockIdx.x; ok && it < g.nitems; it += gridDim.x) {
                int n, q0, z0, z1;
                item(it, n, q0, z0, z1);
                const int y_lo = floor_div(q0 - g.Wp - 1, g.Wp);
                for (int pz = z0 - 1; pz <= z1; pz++, j++) {
                    const int slot = (int)(j % g.S);
                    if (j >= g.S && !mbar_wait_flag(smem_u32(&empty[slot]), (uint32_t)(((j / g.S) - 1) & 1), &s_err)) {
                        ok = false;
                        break;
                    }
                    const uint32_t st = stbase + (uint32_t)slot * g.stage_bytes;
                    const uint32_t fb = smem_u32(&full[slot]);
                    mbar_expect_tx(fb, (CIN / 8) * g.box_bytes);
#pragma unroll
                    for (int c = 0; c < CIN / 8; c++)
                        tma_load_5d(st + c * g.plane_bytes, &xmap, c * 8, -1, y_lo, pz, n, fb);
                    s_issued = j + 1;
                }
            }
        }
    } else if (warp >= 5) {
        const int iw = warp - 5;  // taps of dz = iw - 1
        if (lane == 0) {
            bool ok = mbar_wait_flag(smem_u32(&wfull), 0, &s_err);
            long long j = 0, o = 0;  // stages and outputs of this CTA so far
            for (long long it = blockIdx.x; ok && it < g.nitems; it += gridDim.x) {
                int n, q0, z0, z1;
                item(it, n, q0, z0, z1);
                const int nz = z1 - z0;
                const int rel = q0 - floor_div(q0 - g.Wp - 1, g.Wp) * g.Wp;  // q0 within the slab
                for (int k = 0; k < nz + 2; k++, j++) {
                    const int slot = (int)(j % g.S);
                    if (!mbar_wait_flag(smem_u32(&full[slot]), (uint32_t)((j / g.S) & 1), &s_err)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const int ol = k - iw;  // the output this plane feeds as dz = iw - 1
                    if (ol >= 0 && ol < nz) {
                        const long long og = o + ol;
                        const int b = (int)(og % NB);
                        if (og >= NB &&
                            !mbar_wait_flag(smem_u32(&accempty[b]), (uint32_t)(((og / NB) - 1) & 1), &s_err)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t st = stbase + (uint32_t)slot * g.stage_bytes;
                        const uint32_t wt = wbase + (uint32_t)(9 * iw) * WT_BYTES;
                        const uint32_t dcol = tmem + (uint32_t)((b * 3 + iw) * COUT);
#pragma unroll 1
                        for (int t = 0; t < 9; t++) {
                            const uint32_t r0 = (uint32_t)(rel + (t / 3 - 1) * g.Wp + (t % 3 - 1));
#pragma unroll
                            for (int kk = 0; kk < CIN / 16; kk++) {
                                const uint64_t da =
                                    smem_desc(st + (uint32_t)(2 * kk) * g.plane_bytes + r0 * 16, g.plane_bytes, 128);
                                const uint64_t db = smem_desc(wt + t * WT_BYTES + kk * 2 * (COUT * 16), COUT * 16, 128);
                                umma_bf16(dcol, da, db, IDESC, (t > 0 || kk > 0) ? 1u : 0u);
                            }
                        }
                        umma_commit(smem_u32(&accfull[b]));
                    }
                    umma_commit(smem_u32(&empty[slot]));
                    s_last[iw] = j;
                }
                o += nz;
            }
        }
    } else {  // epilogue: warps 0-3 own TMEM lanes 32w .. 32w+31
        long long o = 0;
        bool ok = true;
        for (long long it = blockIdx.x; ok && it < g.nitems; it += gridDim.x) {
            int n, q0, z0, z1;
            item(it, n, q0, z0, z1);
            const int q = q0 + tid;
            const int y = q / g.Wp, xp = q - (q / g.Wp) * g.Wp;
            const bool valid = y < a.H && xp >= 1 && xp <= a.W;
            for (int z = z0; z < z1; z++, o++) {
                const int b = (int)(o % NB);
                if (!mbar_wait_flag(smem_u32(&accfull[b]), (uint32_t)((o / NB) & 1), &s_err)) {
                    ok = false;
                    break;
                }
                __syncwarp();  // converged for the warp-collective TMEM loads
                tc_fence_after();
                uint32_t r[COUT];
                const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(b * 3 * COUT);
#pragma unroll
                for (int c = 0; c < COUT; c += 16) {
                    uint32_t (&rr)[16] = *reinterpret_cast<uint32_t(*)[16]>(&r[c]);
                    uint32_t r1[16], r2[16];
                    tmem_ld16(lane_base + (uint32_t)c, rr);
                    tmem_ld16(lane_base + (uint32_t)(COUT + c), r1);
                    tmem_ld16(lane_base + (uint32_t)(2 * COUT + c), r2);
                    tmem_wait_ld();
#pragma unroll
                    for (int jj = 0; jj < 16; jj++)  // (dz -1) + (dz 0), then + (dz +1)
                        rr[jj] = __float_as_uint(__fadd_rn(__fadd_rn(__uint_as_float(rr[jj]), __uint_as_float(r1[jj])),
                                                           __uint_as_float(r2[jj])));
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(&accempty[b]));
                if (valid) {
                    const long long v = ((long long)n * a.D + z) * HW + (long long)y * a.W + (xp - 1);
#pragma unroll
                    for (int c = 0; c < COUT; c += 8) {
                        float f[8];
#pragma unroll
                        for (int jj = 0; jj < 8; jj++) f[jj] = __uint_as_float(r[c + jj]);
                        store8(a, COUT, v, c, f);
                    }
                }
            }
        }
    }
    __syncthreads();
    if (s_err) {
        // after an error: let the copies and MMAs already issued finish (bounded)
        // before the shared memory and TMEM are released
        if (tid == 0) {
            note_timeout(a.counters, SITE_CONV_ZCOL);
            for (long long i = s_issued > g.S ? s_issued - g.S : 0; i < s_issued; i++)
                mbar_wait(smem_u32(&full[i % g.S]), (uint32_t)((i / g.S) & 1));
            for (int w = 0; w < 3; w++) {
                const long long i = s_last[w];
                if (i >= 0) mbar_wait(smem_u32(&empty[i % g.S]), (uint32_t)((i / g.S) & 1));
            }
        }
        __syncthreads();
    }
    if (warp == 5) {
        tc_fence_after();
        tmem_dealloc(tmem, TCOLS);
    }
}

// --------------------------------------------------------------------------
// z-column convolution with the three dz taps of an in-plane offset in one
// MMA.  conv_zcol_kernel feeds each staged input-plane slab to three output
// planes through three issuers, each multiplying the same shifted A tile
// (128 positions x 16 channels, 4 KB of shared memory per K step) by an
// N = cout weight tile: with N = 16 the tensor pipe spends its time reading A.
// Here B is the concatenation [W(dz=-1) | W(dz=0) | W(dz=+1)] of the in-plane
// tap (dy, dx), N = 3 cout, so each A tile is read once for all three output
// planes: stage k (input plane p = z0 - 1 + k) writes the partial sums
// P_k = A_p x Bcat into TMEM region k % NB, whose block b (dz = b - 1) belongs
// to output plane p + 1 - b.  Output z0 + ol is P_ol[block 0] + P_ol+1[block 1]
// + P_ol+2[block 2], complete once stages ol .. ol + 2 are; the epilogue adds
// the three blocks in the order (dz -1) + (dz 0), then + (dz +1).
// Roles: warps 0-7 drain in two groups of four (group g takes the outputs
// ol = g mod 2, each warp the 32 TMEM lanes of its quadrant, the bias in
// registers), warp 8 loads slabs by TMA, warps 9 .. 8 + NISS issue the MMAs of
// the stages in turn (a tcgen05.mma occupies its issuing thread for longer
// than the tensor pipe needs for it).  A region is reused once both groups
// are done with it: after output ol a group frees the regions of stages ol and
// ol + 1 (its next output starts at stage ol + 2), and at the end of a work
// item the stages it never read.  The regions rotate over NB >= 3 buffers.
// Slabs arrive as one TMA box per 16 channels with the 32-byte swizzle: rows
// of 32 bytes, stage layout [cin/16][position][16 channels], read by the MMAs
// as swizzled K-major tiles from any row.  The TMA unit moves about one box row
// per clock, so 16-byte rows (one box per 8 channels, the unswizzled K-major
// layout) left the issuers waiting on slabs 40 % of the time at 16 -> 16.
// Loading with warp-wide cp.async (16 bytes per thread, coalesced) measured
// 1.6x slower still: too few loads in flight per SM to cover the latency.
// The concatenated weights (27 cin cout bf16) are built in shared memory by
// all threads at the start, from the [tap][cin/8][cout][8] tiles.
// --------------------------------------------------------------------------
constexpr int ZCAT_EPI_WARPS = 8;
constexpr int ZCAT_PRODUCER = 8;  // warp index of the TMA producer
constexpr int ZCAT_ISSUER0 = 9;   // first MMA-issuing warp

template <int CIN, int COUT, int COUTH, int NB, int NISS, int MINB>
__global__ void __launch_bounds__(32 * (ZCAT_ISSUER0 + NISS), MINB)
    conv_zcat_kernel(const __grid_constant__ CUtensorMap xmap, const ConvArgs a, const TmaGeom g)
{
    static_assert(CIN % 16 == 0, "slabs of 16-channel planes");
    constexpr int N3 = 3 * COUTH;  // COUTH of the COUT output channels per CTA: blockIdx.y selects them
    const int c_lo = (int)blockIdx.y * COUTH;
    constexpr uint32_t TCOLS = tma_tcols(NB * N3);
    static_assert(NB >= 3 && NB * N3 <= 512, "three regions in flight within 512 TMEM columns");
    static_assert(N3 % 16 == 0 && N3 <= 256, "M = 128 MMAs take N = 16 .. 256 in steps of 16");
    constexpr uint32_t IDESC = idesc_bf16(TILE_M, N3);
    constexpr uint32_t WT9_BYTES = N3 * CIN * 2;  // one in-plane tap, all three dz
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[8], empty[8], accfull[NB], accempty[NB];
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_err;
    __shared__ int s_issued, s_last[NISS];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = smem_u32(smem);
    const uint32_t wbase = sbase;                   // concatenated weights [t9][cin/8][3 cout][8]
    const uint32_t stbase = sbase + g.wres_bytes;   // stages: one input-plane slab each
    // Bcat(t9)[kc][dzi * COUTH + co][8] = W(tap = 9 dzi + t9)[kc][c_lo + co][8]
    for (int i = tid; i < 27 * CIN * COUTH / 8; i += blockDim.x) {
        const int co = i % COUTH;
        int r = i / COUTH;
        const int dzi = r % 3;
        r /= 3;
        const int kc = r % (CIN / 8), t9 = r / (CIN / 8);
        const uint4 v =
            *reinterpret_cast<const uint4 *>(a.w + (((size_t)(9 * dzi + t9) * (CIN / 8) + kc) * COUT + c_lo + co) * 8);
        *reinterpret_cast<uint4 *>(smem + (size_t)i * 16) = v;
    }
    fence_proxy_async();  // the weights written by threads, read by the tensor core
    if (tid == 0) {
        for (int k = 0; k < g.S; k++) {
            mbar_init(smem_u32(&full[k]), 1);
            mbar_init(smem_u32(&empty[k]), 1);
        }
        for (int b = 0; b < NB; b++) {
            mbar_init(smem_u32(&accfull[b]), 1);
            mbar_init(smem_u32(&accempty[b]), ZCAT_EPI_WARPS);  // both drain groups
        }
        fence_mbar_init();
        s_err = 0;
        s_issued = 0;
        for (int i = 0; i < NISS; i++) s_last[i] = -1;
    }
    if (warp == ZCAT_PRODUCER) {
        tmem_alloc(smem_u32(&s_tmem), TCOLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const int HW = a.H * a.W;
    // work: with g.ZC > 0, items of ZC output planes of a column dealt round
    // robin (g.nitems items); with g.ZC == 0, an equal contiguous share of the
    // g.nitems (column, plane) pairs per CTA, walked as runs within a column.
    // A run of Z planes takes Z + 2 stages; the launcher picks the scheme with
    // the fewer stages on the busiest CTA.
    const bool rr = g.ZC > 0;
    const int nzc = rr ? (a.D + g.ZC - 1) / g.ZC : 1;  // z-chunks per column
    const long long c_begin = rr ? (long long)blockIdx.x : g.nitems * blockIdx.x / gridDim.x;
    const long long c_end = rr ? g.nitems : g.nitems * (blockIdx.x + 1) / gridDim.x;
    auto item = [&](long long &cur, int &n, int &q0, int &z0, int &z1) {
        long long col;
        if (rr) {
            col = cur / nzc;
            z0 = (int)(cur % nzc) * g.ZC;
            z1 = z0 + g.ZC < a.D ? z0 + g.ZC : a.D;
            cur += gridDim.x;
        } else {
            col = cur / a.D;
            z0 = (int)(cur - col * a.D);
            const long long left = c_end - cur;
            z1 = (long long)(a.D - z0) <= left ? a.D : z0 + (int)left;
            cur += z1 - z0;
        }
        n = (int)(col / g.T);
        q0 = (int)(col % g.T) * TILE_M;
    };

    if (warp == ZCAT_PRODUCER) {
        if (lane == 0) {  // one slab per input plane z0-1 .. z1 (planes outside the volume arrive as zeros)
            int j = 0, slot = 0, round = 0;  // slot = j % S, round = j / S
            bool ok = true;
            for (long long cur = c_begin; ok && cur < c_end;) {
                int n, q0, z0, z1;
                item(cur, n, q0, z0, z1);
                const int y_lo = floor_div(q0 - g.Wp - 1, g.Wp);
                for (int pz = z0 - 1; pz <= z1; pz++, j++) {
                    if (j >= g.S && !mbar_wait_flag(smem_u32(&empty[slot]), (uint32_t)((round - 1) & 1), &s_err)) {
                        ok = false;
                        break;
                    }
                    const uint32_t st = stbase + (uint32_t)slot * g.stage_bytes;
                    const uint32_t fb = smem_u32(&full[slot]);
                    mbar_expect_tx(fb, (CIN / 16) * g.box_bytes);
#pragma unroll
                    for (int c = 0; c < CIN / 16; c++)
                        tma_load_5d(st + c * g.plane_bytes, &xmap, c * 16, -1, y_lo, pz, n, fb);
                    s_issued = j + 1;
                    if (++slot == g.S) {
                        slot = 0;
                        round++;
                    }
                }
            }
        }
    } else if (warp >= ZCAT_ISSUER0) {
        const int iw = warp - ZCAT_ISSUER0;  // stages j with j % NISS == iw
        if (lane == 0) {
            int j = 0, slot = 0, round = 0, r = 0, rround = 0;  // slot = j % S, round = j / S, r = j % NB, rround = j / NB
            bool ok = true;
            for (long long cur = c_begin; ok && cur < c_end;) {
                int n, q0, z0, z1;
                item(cur, n, q0, z0, z1);
                const int rel = q0 - floor_div(q0 - g.Wp - 1, g.Wp) * g.Wp;  // q0 within the slab
                for (int k = 0; k < z1 - z0 + 2; k++, j++) {
                    const int cur_slot = slot, cur_round = round, cur_r = r, cur_rround = rround;
                    if (++slot == g.S) {
                        slot = 0;
                        round++;
                    }
                    if (++r == NB) {
                        r = 0;
                        rround++;
                    }
                    if (j % NISS != iw) continue;
                    if (!mbar_wait_flag(smem_u32(&full[cur_slot]), (uint32_t)(cur_round & 1), &s_err) ||
                        (j >= NB && !mbar_wait_flag(smem_u32(&accempty[cur_r]), (uint32_t)((cur_rround - 1) & 1), &s_err))) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t st = stbase + (uint32_t)cur_slot * g.stage_bytes;
                    const uint32_t dcol = tmem + (uint32_t)(cur_r * N3);
                    // descriptors: the start-address field (16-byte units, low 14 bits) moves
                    // by whole units from one MMA to the next and never leaves [0, 2^14), so
                    // each is the stage's base descriptor plus a small (signed) offset
                    const uint64_t da0 = smem_desc_sw32(st + (uint32_t)rel * 32);
                    const uint64_t db0 = smem_desc(wbase, N3 * 16, 128);
#pragma unroll
                    for (int t = 0; t < 9; t++) {
                        const int64_t toff = (int64_t)(2 * ((t / 3 - 1) * g.Wp + (t % 3 - 1)));  // rows of 32 B, in 16 B
#pragma unroll
                        for (int kk = 0; kk < CIN / 16; kk++) {
                            const uint64_t da = da0 + (uint64_t)(toff + (int64_t)((kk * g.plane_bytes) >> 4));
                            const uint64_t db = db0 + (uint64_t)((t * WT9_BYTES + kk * 2 * (N3 * 16)) >> 4);
                            umma_bf16(dcol, da, db, IDESC, (t > 0 || kk > 0) ? 1u : 0u);
                        }
                    }
                    umma_commit(smem_u32(&empty[cur_slot]));
                    umma_commit(smem_u32(&accfull[cur_r]));
                    s_last[iw] = j;
                }
            }
        }
    } else {  // drain: group grp = warp / 4 takes outputs ol = grp mod 2; warp % 4 = its TMEM quadrant
        const int grp = warp >> 2, quad = warp & 3;
        const int row = quad * 32 + lane;  // this thread's position in the tile
        float bias[COUTH];
#pragma unroll
        for (int c = 0; c < COUTH; c++) bias[c] = a.bias ? a.bias[c_lo + c] : 0.0f;
        const uint32_t lb = tmem + ((uint32_t)(quad * 32) << 16);
        auto release = [&](long long stage) {  // this warp is done with the region of `stage`
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&accempty[stage % NB]));
        };
        // a stage this group never reads is released only once its MMAs have
        // completed: an arrival before that could land in the region's previous
        // phase (the release of stage - NB) while a slower warp still reads it,
        // when the warps of a group run at different speeds (tiles whose lower
        // rows are padding store nothing)
        auto release_unread = [&](long long stage) -> bool {
            if (!mbar_wait_flag(smem_u32(&accfull[stage % NB]), (uint32_t)((stage / NB) & 1), &s_err)) return false;
            release(stage);
            return true;
        };
        int j = 0;  // this CTA's stages before the current item
        bool ok = true;
        for (long long cur = c_begin; ok && cur < c_end;) {
            int n, q0, z0, z1;
            item(cur, n, q0, z0, z1);
            const int nz = z1 - z0;
            const int q = q0 + row;
            const int y = q / g.Wp, xp = q - (q / g.Wp) * g.Wp;
            const bool valid = y < a.H && xp >= 1 && xp <= a.W;
            // stages this group never reads: those before its first output
            for (int k = 0; ok && k < grp && k < nz + 2; k++) ok = release_unread(j + k);
            int last = -1;  // this group's last output of the item
            for (int ol = grp; ok && ol < nz; ol += 2) {
                for (int k = 0; k < 3; k++)
                    if (!mbar_wait_flag(smem_u32(&accfull[(j + ol + k) % NB]), (uint32_t)(((j + ol + k) / NB) & 1),
                                        &s_err)) {
                        ok = false;
                        break;
                    }
                if (!ok) break;
                // the warp converges before the warp-collective TMEM loads: the
                // previous output's stores diverge on `valid` and may be slow
                __syncwarp();
                tc_fence_after();
                uint32_t rr[COUTH];
                const uint32_t c0 = (uint32_t)(((j + ol) % NB) * N3);
                const uint32_t c1 = (uint32_t)(((j + ol + 1) % NB) * N3 + COUTH);
                const uint32_t c2 = (uint32_t)(((j + ol + 2) % NB) * N3 + 2 * COUTH);
#pragma unroll
                for (int c = 0; c < COUTH; c += 16) {
                    uint32_t (&r0)[16] = *reinterpret_cast<uint32_t(*)[16]>(&rr[c]);
                    uint32_t r1[16], r2[16];
                    tmem_ld16(lb + c0 + (uint32_t)c, r0);
                    tmem_ld16(lb + c1 + (uint32_t)c, r1);
                    tmem_ld16(lb + c2 + (uint32_t)c, r2);
                    tmem_wait_ld();
#pragma unroll
                    for (int jj = 0; jj < 16; jj++)  // (dz -1) + (dz 0), then + (dz +1)
                        r0[jj] = __float_as_uint(__fadd_rn(__fadd_rn(__uint_as_float(r0[jj]), __uint_as_float(r1[jj])),
                                                           __uint_as_float(r2[jj])));
                }
                tc_fence_before();
                release(j + ol);  // the next output of this group starts at stage ol + 2
                release(j + ol + 1);
                last = ol;
                if (valid) {
                    const long long v = ((long long)n * a.D + z0 + ol) * HW + (long long)y * a.W + (xp - 1);
#pragma unroll
                    for (int c = 0; c < COUTH; c += 8) {
                        float f[8];
#pragma unroll
                        for (int jj = 0; jj < 8; jj++) f[jj] = __uint_as_float(rr[c + jj]);
                        store8_b(a, COUT, v, c_lo + c, f, bias + c);
                    }
                }
            }
            if (!ok) break;
            // the stages after this group's last output (or all but the first grp if it had none);
            // stage last + 2 was read by the last output
            for (int k = last >= 0 ? last + 2 : grp; ok && k < nz + 2; k++)
                ok = (last >= 0 && k == last + 2) ? (release(j + k), true) : release_unread(j + k);
            if (!ok) break;
            j += nz + 2;
        }
    }
    __syncthreads();
    if (s_err) {
        // after an error: let the copies and MMAs already issued finish (bounded)
        // before the shared memory and TMEM are released
        if (tid == 0) {
            note_timeout(a.counters, SITE_CONV_ZCAT);
            for (int i = s_issued > g.S ? s_issued - g.S : 0; i < s_issued; i++)
                mbar_wait(smem_u32(&full[i % g.S]), (uint32_t)((i / g.S) & 1));
            for (int w = 0; w < NISS; w++) {
                const int i = s_last[w];
                if (i >= 0) mbar_wait(smem_u32(&empty[i % g.S]), (uint32_t)((i / g.S) & 1));
            }
        }
        __syncthreads();
    }
    if (warp == ZCAT_PRODUCER) {
        tc_fence_after();
        tmem_dealloc(tmem, TCOLS);
    }
}

// K-major operand with the 64-byte swizzle: rows of 32 bf16 (64 bytes), 8-row
// groups 512 bytes apart (SBO), layout type 4.  The start may sit at any row,
// and at +32 bytes within a row for its second K step (checked for row offsets
// 0 .. 67, base-offset field 0).
__device__ __forceinline__ uint64_t smem_desc_sw64(uint32_t addr)
{
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | (1ull << 16) | ((uint64_t)(512u >> 4) << 32) | (1ull << 46) |
           (4ull << 61);
}

// --------------------------------------------------------------------------
// x-pair z-column convolution for 16 input channels.  conv_zcat_kernel stages
// one 32-byte TMA row per padded position; at 16 channels the TMA unit's row
// rate (about one per clock per SM) bounds it.  Here the 16-channel NDHWC
// tensor is viewed as rows of x-pairs (two voxels, 64 bytes) and staged with
// the 64-byte swizzle: a slab row is a padded pair position q = y Wq + px
// (Wq = W/2 + 2, pair px holding voxels 2px - 2 and 2px - 1, pairs 0 and
// Wq - 1 the zero halo), a tile 128 pair positions = 256 voxel slots, and a
// slab of rows y_lo .. y_lo + NR - 1 reaches every pair a tile's taps need.
// An MMA row is a pair (K = 32: both voxels' 16 channels) and its N = 96
// columns are (dz, output voxel j of the pair, 16 output channels).  Output
// voxel 2p + j takes input voxel 2(p + pdx) + k (k: K step = voxel of the
// input pair) at dx = 2 pdx + k - j, so a pair tap (dy, pdx) multiplies the
// pair row shifted by dy Wq + pdx by B(dy, pdx, k)[n][ci] = W(dz, dy, dx)[co][ci]
// where |dx| <= 1, else 0: the pair taps pdx = -1 and +1 need only their K step
// k = 1 and k = 0 (the other is all zeros), so a stage issues 12 MMAs of
// 128 x 96 x 16 for 256 voxels where conv_zcat_kernel issues 18 of 128 x 48 x 16,
// reads fewer operand bytes, and stages its slab in 2.8x fewer TMA rows.  The
// z-column structure, the TMEM regions (NB of 96 columns), the roles and the
// release protocol are conv_zcat_kernel's; with one CTA per SM (480 TMEM
// columns) the drain runs in three groups of four warps (outputs ol = g mod 3),
// and a drain thread stores its pair's two voxels; a data gradient's ReLU mask
// for them is loaded before the thread waits for the output's MMAs.
// --------------------------------------------------------------------------
constexpr int ZPAIR_NB = 5;
constexpr int ZPAIR_NISS = 3;
constexpr int ZPAIR_GROUPS = 3;                        // drain groups of four warps
constexpr int ZPAIR_DRAIN = 4 * ZPAIR_GROUPS;          // drain warps
constexpr int ZPAIR_PRODUCER = ZPAIR_DRAIN;            // warp index of the TMA producer
constexpr int ZPAIR_ISSUER0 = ZPAIR_DRAIN + 1;         // first MMA-issuing warp
constexpr int ZPAIR_N = 96;                            // 3 dz x 2 voxels x 16 channels
constexpr uint32_t ZPAIR_WBYTES = 9u * 2u * 2u * ZPAIR_N * 16u;  // [pair tap][k][kc][n][8] bf16

template <int COUT>
__global__ void __launch_bounds__(32 * (ZPAIR_ISSUER0 + ZPAIR_NISS), 1)
    conv_zpair_kernel(const __grid_constant__ CUtensorMap xmap, const ConvArgs a, const TmaGeom g)
{
    constexpr int CIN = 16, NB = ZPAIR_NB, NISS = ZPAIR_NISS, N3 = ZPAIR_N;
    const int c_lo = (int)blockIdx.y * 16;
    constexpr uint32_t TCOLS = tma_tcols(NB * N3);
    static_assert(NB * N3 <= 512, "NB regions within 512 TMEM columns");
    constexpr uint32_t IDESC = idesc_bf16(TILE_M, N3);
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[8], empty[8], accfull[NB], accempty[NB];
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_err;
    __shared__ int s_issued, s_last[NISS];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = smem_u32(smem);
    const uint32_t wbase = sbase;                  // pair-tap weights [9][2][2][96][8]
    const uint32_t stbase = sbase + g.wres_bytes;  // stages: one input-plane pair slab each
    // B(pt, k)[kc][n][e], pt = 3 (dy + 1) + pdx + 1, n = 32 dzi + 16 j + co, ci = 8 kc + e
    for (int i = tid; i < 9 * 2 * 2 * N3; i += blockDim.x) {
        const int n = i % N3;
        int r = i / N3;
        const int kc = r % 2;
        r /= 2;
        const int k = r % 2, pt = r / 2;
        const int dzi = n / 32, j = (n / 16) % 2, co = c_lo + n % 16;
        const int dy = pt / 3 - 1, pdx = pt % 3 - 1;
        const int dx = 2 * pdx + k - j;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (dx >= -1 && dx <= 1) {
            const int tap = 9 * dzi + 3 * (dy + 1) + dx + 1;
            v = *reinterpret_cast<const uint4 *>(a.w + (((size_t)tap * (CIN / 8) + kc) * COUT + co) * 8);
        }
        *reinterpret_cast<uint4 *>(smem + (size_t)i * 16) = v;
    }
    fence_proxy_async();  // the weights written by threads, read by the tensor core
    if (tid == 0) {
        for (int k = 0; k < g.S; k++) {
            mbar_init(smem_u32(&full[k]), 1);
            mbar_init(smem_u32(&empty[k]), 1);
        }
        for (int b = 0; b < NB; b++) {
            mbar_init(smem_u32(&accfull[b]), 1);
            mbar_init(smem_u32(&accempty[b]), ZPAIR_DRAIN);  // every drain warp
        }
        fence_mbar_init();
        s_err = 0;
        s_issued = 0;
        for (int i = 0; i < NISS; i++) s_last[i] = -1;
    }
    if (warp == ZPAIR_PRODUCER) {
        tmem_alloc(smem_u32(&s_tmem), TCOLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const int HW = a.H * a.W;
    const int WP = g.Wp;                      // padded pairs per row
    // work: with g.ZC > 0, items of ZC output planes of a column dealt round
    // robin (g.nitems items); with g.ZC == 0, an equal contiguous share of the
    // g.nitems (column, plane) pairs per CTA, walked as runs within a column.
    // A run of Z planes takes Z + 2 stages; the launcher picks the scheme with
    // the fewer stages on the busiest CTA.
    const bool rr = g.ZC > 0;
    const int nzc = rr ? (a.D + g.ZC - 1) / g.ZC : 1;  // z-chunks per column
    const long long c_begin = rr ? (long long)blockIdx.x : g.nitems * blockIdx.x / gridDim.x;
    const long long c_end = rr ? g.nitems : g.nitems * (blockIdx.x + 1) / gridDim.x;
    auto item = [&](long long &cur, int &n, int &q0, int &z0, int &z1) {
        long long col;
        if (rr) {
            col = cur / nzc;
            z0 = (int)(cur % nzc) * g.ZC;
            z1 = z0 + g.ZC < a.D ? z0 + g.ZC : a.D;
            cur += gridDim.x;
        } else {
            col = cur / a.D;
            z0 = (int)(cur - col * a.D);
            const long long left = c_end - cur;
            z1 = (long long)(a.D - z0) <= left ? a.D : z0 + (int)left;
            cur += z1 - z0;
        }
        n = (int)(col / g.T);
        q0 = (int)(col % g.T) * TILE_M;
    };

    if (warp == ZPAIR_PRODUCER) {
        if (lane == 0) {  // one pair slab per input plane z0-1 .. z1 (planes outside the volume arrive as zeros)
            int j = 0, slot = 0, round = 0;
            bool ok = true;
            for (long long cur = c_begin; ok && cur < c_end;) {
                int n, q0, z0, z1;
                item(cur, n, q0, z0, z1);
                const int y_lo = floor_div(q0 - WP - 1, WP);
                for (int pz = z0 - 1; pz <= z1; pz++, j++) {
                    if (j >= g.S && !mbar_wait_flag(smem_u32(&empty[slot]), (uint32_t)((round - 1) & 1), &s_err)) {
                        ok = false;
                        break;
                    }
                    const uint32_t st = stbase + (uint32_t)slot * g.stage_bytes;
                    const uint32_t fb = smem_u32(&full[slot]);
                    mbar_expect_tx(fb, g.box_bytes);
                    tma_load_5d(st, &xmap, 0, -1, y_lo, pz, n, fb);  // pairs -1 .. Wq - 2 of rows y_lo ..
                    s_issued = j + 1;
                    if (++slot == g.S) {
                        slot = 0;
                        round++;
                    }
                }
            }
        }
    } else if (warp >= ZPAIR_ISSUER0) {
        const int iw = warp - ZPAIR_ISSUER0;  // stages j with j % NISS == iw
        if (lane == 0) {
            int j = 0, slot = 0, round = 0, r = 0, rround = 0;
            bool ok = true;
            for (long long cur = c_begin; ok && cur < c_end;) {
                int n, q0, z0, z1;
                item(cur, n, q0, z0, z1);
                const int rel = q0 - floor_div(q0 - WP - 1, WP) * WP;  // q0 within the slab
                for (int k = 0; k < z1 - z0 + 2; k++, j++) {
                    const int cur_slot = slot, cur_round = round, cur_r = r, cur_rround = rround;
                    if (++slot == g.S) {
                        slot = 0;
                        round++;
                    }
                    if (++r == NB) {
                        r = 0;
                        rround++;
                    }
                    if (j % NISS != iw) continue;
                    if (!mbar_wait_flag(smem_u32(&full[cur_slot]), (uint32_t)(cur_round & 1), &s_err) ||
                        (j >= NB && !mbar_wait_flag(smem_u32(&accempty[cur_r]), (uint32_t)((cur_rround - 1) & 1), &s_err))) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t st = stbase + (uint32_t)cur_slot * g.stage_bytes;
                    const uint32_t dcol = tmem + (uint32_t)(cur_r * N3);
                    // descriptors as a base plus offsets in 16-byte units: a pair row is 4 units,
                    // the second K step of a row 2 units in; a (pair tap, k) weight block
                    // 2 N3 units
                    const uint64_t da0 = smem_desc_sw64(st + (uint32_t)rel * 64);
                    const uint64_t db0 = smem_desc(wbase, N3 * 16, 128);
                    bool first = true;
#pragma unroll
                    for (int pt = 0; pt < 9; pt++) {
                        const int dy = pt / 3 - 1, pdx = pt % 3 - 1;
#pragma unroll
                        for (int kk = 0; kk < 2; kk++) {
                            if ((pdx == -1 && kk == 0) || (pdx == 1 && kk == 1)) continue;  // all-zero weights
                            const uint64_t da = da0 + (uint64_t)(int64_t)(4 * (dy * WP + pdx) + 2 * kk);
                            const uint64_t db = db0 + (uint64_t)((uint32_t)((pt * 2 + kk) * 2 * N3));
                            umma_bf16(dcol, da, db, IDESC, first ? 0u : 1u);
                            first = false;
                        }
                    }
                    umma_commit(smem_u32(&empty[cur_slot]));
                    umma_commit(smem_u32(&accfull[cur_r]));
                    s_last[iw] = j;
                }
            }
        }
    } else {  // drain: group grp = warp / 4 takes outputs ol = grp mod ZPAIR_GROUPS; warp % 4 = its TMEM quadrant
        constexpr int NG = ZPAIR_GROUPS;
        const int grp = warp >> 2, quad = warp & 3;
        const int row = quad * 32 + lane;  // this thread's pair position in the tile
        float bias[16];
#pragma unroll
        for (int c = 0; c < 16; c++) bias[c] = a.bias ? a.bias[c_lo + c] : 0.0f;
        const uint32_t lb = tmem + ((uint32_t)(quad * 32) << 16);
        auto release = [&](long long stage) {
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&accempty[stage % NB]));
        };
        // a stage this warp has not read is released only once its MMAs have completed (an
        // earlier arrival could complete the region's previous phase while a slower warp reads it)
        auto release_unread = [&](long long stage) -> bool {
            if (!mbar_wait_flag(smem_u32(&accfull[stage % NB]), (uint32_t)((stage / NB) & 1), &s_err)) return false;
            release(stage);
            return true;
        };
        // every warp releases every stage of an item once: those before its group's first
        // output, after output ol the stages ol .. ol + NG - 1 (the first three read by it), and
        // at the end those after its last output's range
        int j = 0;
        bool ok = true;
        for (long long cur = c_begin; ok && cur < c_end;) {
            int n, q0, z0, z1;
            item(cur, n, q0, z0, z1);
            const int nz = z1 - z0;
            const int q = q0 + row;
            const int y = q / WP, px = q - (q / WP) * WP;
            const bool valid = y < a.H && px >= 1 && 2 * px <= a.W;
            for (int k = 0; ok && k < grp && k < nz + 2; k++) ok = release_unread(j + k);
            int last = -1;
            for (int ol = grp; ok && ol < nz; ol += NG) {
                const long long v = ((long long)n * a.D + z0 + ol) * HW + (long long)y * a.W + (2 * px - 2);
                uint4 mk[4] = {};  // the ReLU mask of the pair's two voxels, loaded ahead of the MMA waits
                if (a.mask_y && valid) {
#pragma unroll
                    for (int m = 0; m < 4; m++)
                        mk[m] = *reinterpret_cast<const uint4 *>(a.mask_y + (v + (m >> 1)) * COUT + c_lo + 8 * (m & 1));
                }
                for (int k = 0; k < 3; k++)
                    if (!mbar_wait_flag(smem_u32(&accfull[(j + ol + k) % NB]), (uint32_t)(((j + ol + k) / NB) & 1),
                                        &s_err)) {
                        ok = false;
                        break;
                    }
                if (!ok) break;
                __syncwarp();  // converged for the warp-collective TMEM loads
                tc_fence_after();
                uint32_t rr[32];
                const uint32_t c0 = (uint32_t)(((j + ol) % NB) * N3);            // dz -1 block of stage ol
                const uint32_t c1 = (uint32_t)(((j + ol + 1) % NB) * N3 + 32);   // dz 0 of stage ol + 1
                const uint32_t c2 = (uint32_t)(((j + ol + 2) % NB) * N3 + 64);   // dz +1 of stage ol + 2
#pragma unroll
                for (int c = 0; c < 32; c += 16) {
                    uint32_t (&r0)[16] = *reinterpret_cast<uint32_t(*)[16]>(&rr[c]);
                    uint32_t t[16];
                    tmem_ld16(lb + c0 + (uint32_t)c, r0);
                    tmem_ld16(lb + c1 + (uint32_t)c, t);
                    tmem_wait_ld();
#pragma unroll
                    for (int jj = 0; jj < 16; jj++)  // (dz -1) + (dz 0)
                        r0[jj] = __float_as_uint(__fadd_rn(__uint_as_float(r0[jj]), __uint_as_float(t[jj])));
                    tmem_ld16(lb + c2 + (uint32_t)c, t);
                    tmem_wait_ld();
#pragma unroll
                    for (int jj = 0; jj < 16; jj++)  // then + (dz +1)
                        r0[jj] = __float_as_uint(__fadd_rn(__uint_as_float(r0[jj]), __uint_as_float(t[jj])));
                }
                tc_fence_before();
                for (int k = 0; k < 3 && ol + k < nz + 2 && k < NG; k++) release(j + ol + k);  // read
                last = ol;
                if (valid) {
#pragma unroll
                    for (int jv = 0; jv < 2; jv++)  // the pair's two voxels
#pragma unroll
                        for (int c = 0; c < 16; c += 8) {
                            float f[8];
#pragma unroll
                            for (int jj = 0; jj < 8; jj++) f[jj] = __uint_as_float(rr[16 * jv + c + jj]);
                            store8_bm(a, COUT, v + jv, c_lo + c, f, bias + c, mk[2 * jv + c / 8]);
                        }
                }
                for (int k = 3; ok && k < NG && ol + k < nz + 2; k++) ok = release_unread(j + ol + k);  // not read
            }
            if (!ok) break;
            for (int k = last >= 0 ? last + NG : grp; ok && k < nz + 2; k++) ok = release_unread(j + k);
            if (!ok) break;
            j += nz + 2;
        }
    }
    __syncthreads();
    if (s_err) {
        if (tid == 0) {
            note_timeout(a.counters, SITE_CONV_ZCAT);
            for (int i = s_issued > g.S ? s_issued - g.S : 0; i < s_issued; i++)
                mbar_wait(smem_u32(&full[i % g.S]), (uint32_t)((i / g.S) & 1));
            for (int w = 0; w < NISS; w++) {
                const int i = s_last[w];
                if (i >= 0) mbar_wait(smem_u32(&empty[i % g.S]), (uint32_t)((i / g.S) & 1));
            }
        }
        __syncthreads();
    }
    if (warp == ZPAIR_PRODUCER) {
        tc_fence_after();
        tmem_dealloc(tmem, TCOLS);
    }
}

// shared-memory attributes of a kernel, set once per process (the largest
// size asked for so far); the attribute calls are host work on every launch
// otherwise
template <typename K>
static cudaError_t smem_attributes(K kernel, uint32_t smem)
{
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, uint32_t> done;  // (device, kernel) -> size set
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    uint32_t &have = done[{dev, reinterpret_cast<const void *>(kernel)}];
    if (smem <= have) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess) have = smem;
    return e;
}

// cuTensorMapEncodeTiled from the driver (no link-time dependency on libcuda)
static PFN_cuTensorMapEncodeTiled tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(p);
    });
    return fn;
}

// accumulator buffers of the z-column kernel, 3 per buffer within 512 TMEM
// columns: 3 or 4 keep the outputs k-2 .. k in flight at stage k apart; 2
// makes the dz = -1 issuer wait for the drain of output k-2, which can pay
// when the smaller allocation admits more CTAs per SM (the launcher picks)
template <int COUT>
struct ZcolNB {
    static constexpr int value = 12 * COUT <= 512 ? 4 : (9 * COUT <= 512 ? 3 : 0);
    static constexpr int small = 6 * COUT <= 128 ? 2 : 0;  // 2 buffers in 128 columns
};

// CTAs per SM and stages of the z-column kernel for a TMEM allocation
static void zcol_fit(const TmaGeom &g, uint32_t budget, uint32_t tcols, int &per_sm, int &S)
{
    per_sm = 0;
    S = 0;
    for (int want = std::min(4, (int)(512 / tcols)); want >= 1; want--) {
        const uint32_t share = std::min(budget, (228u * 1024u) / (uint32_t)want - 2048u);
        if (share <= g.wres_bytes) continue;
        const int st = (int)std::min<uint32_t>(8u, (share - g.wres_bytes) / g.stage_bytes);
        if (st >= 4) {
            per_sm = want;
            S = st;
            return;
        }
    }
}

template <int CIN, int COUT, int NB>
static void launch_zcol_nb(const ConvArgs &a, TmaGeom g, const CUtensorMap &map, int per_sm, int S, cudaStream_t s,
                           cudaError_t &err)
{
    g.S = S;
    const long long nb = a.V / ((long long)a.D * a.H * a.W);
    const long long grid_max = (long long)per_sm * std::max(1, a.sms);
    // output planes per work item: the whole depth unless that leaves SMs idle
    int ZC = a.D;
    while (ZC > 4 && nb * g.T * ((a.D + ZC - 1) / ZC) < 2 * grid_max) ZC = (ZC + 1) / 2;
    g.ZC = ZC;
    g.nitems = nb * g.T * ((a.D + ZC - 1) / ZC);
    const uint32_t smem = g.wres_bytes + (uint32_t)S * g.stage_bytes;
    err = smem_attributes(conv_zcol_kernel<CIN, COUT, NB>, smem);
    if (err != cudaSuccess) return;
    const long long grid = std::min<long long>(g.nitems, grid_max);
    ++launch_count;
    conv_zcol_kernel<CIN, COUT, NB><<<(unsigned)grid, 256, smem, s>>>(map, a, g);
    err = cudaGetLastError();
}

// regions (NB) and issuing warps (NISS) of the concatenated-dz z-column
// kernel per output channel count: N = 3 cout columns per region, NB >= 3
// regions within the TMEM allocation the CTAs of an SM share
template <int CIN, int COUT>
struct ZcatCfg {
    // output channels per CTA: all of them, or a split where the concatenated
    // weights of all would not stay resident in 96 KB (27 cin cout bf16) or N = 3 cout
    // would pass 256 (96 -> 32: 16 per CTA; 32 -> 96: 48; 64 -> 64: 16)
    static constexpr bool FITS_ALL = 3 * COUT <= 256 && CIN * COUT <= 1820;
    static constexpr int COUTH = FITS_ALL ? COUT
                                 : (COUT % 48 == 0 && CIN * 48 <= 1820) ? 48
                                 : (COUT % 16 == 0 && CIN * 16 <= 1820) ? 16 : COUT;
    static constexpr int N3 = 3 * COUTH;
    static constexpr int NB = 5 * N3 <= 256 ? 5 : (5 * N3 <= 512 ? 5 : (3 * N3 <= 512 ? 3 : 0));
    static constexpr int PER_SM = (int)(512 / tma_tcols(NB > 0 ? NB * N3 : 512));  // CTAs per SM by TMEM
    static constexpr int NISS = PER_SM >= 2 ? 2 : 3;
};

// the work split of the z-column kernels (TmaGeom::ZC, nitems): items of ZC
// planes dealt round robin, or equal contiguous shares of the (column, plane)
// pairs; whichever leaves the busiest CTA the fewer stages (a run of Z planes
// of one column takes Z + 2)
static void zcol_work_split(TmaGeom &g, long long ncols, int D, long long grid)
{
    long long best = -1;
    for (int zc = D; zc >= 1; zc = zc > 1 ? (zc + 1) / 2 : 0) {
        const long long items = ncols * ((D + zc - 1) / zc);
        const long long cost = ((items + grid - 1) / grid) * (zc + 2);
        if (best < 0 || cost < best) {
            best = cost;
            g.ZC = zc;
            g.nitems = items;
        }
        if (zc == 1) break;
    }
    const long long total = ncols * D;
    long long worst = 0;
    for (long long b = 0; b < grid; b++) {
        long long cur = total * b / grid, stages = 0;
        const long long end = total * (b + 1) / grid;
        while (cur < end) {
            const long long z0 = cur % D, run = std::min<long long>(D - z0, end - cur);
            stages += run + 2;
            cur += run;
        }
        worst = std::max(worst, stages);
    }
    if (worst < best) {
        g.ZC = 0;
        g.nitems = total;
    }
}

// the concatenated-dz z-column convolution (conv_zcat_kernel) when its
// weights stay resident and 4+ stages fit; false leaves the layer to the
// others.  IAC_DENOISE_ZCAT=0 in the environment turns it off (for comparing
// the kernels).
template <int CIN, int COUT>
static bool launch_zcat(const ConvArgs &a, const TmaGeom &g0, uint32_t budget, cudaStream_t s, cudaError_t &err)
{
    using Z = ZcatCfg<CIN, COUT>;
    if constexpr (Z::NB == 0 || Z::N3 > 256 || COUT % Z::COUTH != 0) {
        return false;
    } else {
        static const bool off = [] {
            const char *e = getenv("IAC_DENOISE_ZCAT");
            return e && e[0] == '0';
        }();
        if (off) return false;
        constexpr int NG = COUT / Z::COUTH;  // output-channel groups (blockIdx.y)
        const uint32_t w27 = 27u * Z::COUTH * CIN * 2;
        if (w27 > 96u * 1024u) return false;
        TmaGeom g = g0;
        g.wcopy_bytes = w27;
        g.wres_bytes = (w27 + 1023u) & ~1023u;
        g.wstage_bytes = 0;
        // slabs as 32-byte swizzled rows: one box of 16 channels x Wp x NR per plane
        g.box_bytes = 32u * (uint32_t)g.Wp * (uint32_t)g.NR;
        g.plane_bytes = (g.box_bytes + 255u) & ~255u;
        g.slab_bytes = g.plane_bytes * (CIN / 16);
        g.stage_bytes = (g.slab_bytes + 1023u) & ~1023u;
        const long long nb = a.V / ((long long)a.D * a.H * a.W);
        PFN_cuTensorMapEncodeTiled enc = tensor_map_encoder();
        if (!enc) return false;
        CUtensorMap map;
        const cuuint64_t dims[5] = {(cuuint64_t)CIN, (cuuint64_t)a.W, (cuuint64_t)a.H, (cuuint64_t)a.D, (cuuint64_t)nb};
        const cuuint64_t strides[4] = {(cuuint64_t)CIN * 2, (cuuint64_t)a.W * CIN * 2,
                                       (cuuint64_t)a.H * a.W * CIN * 2, (cuuint64_t)a.D * a.H * a.W * CIN * 2};
        const cuuint32_t box[5] = {16u, (cuuint32_t)g.Wp, (cuuint32_t)g.NR, 1u, 1u};
        const cuuint32_t estr[5] = {1u, 1u, 1u, 1u, 1u};
        if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16 *>(a.src1), dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
        int per_sm = 0, S = 0;
        for (int want = Z::PER_SM; want >= 1 && per_sm == 0; want--) {
            const uint32_t share = std::min(budget, (228u * 1024u) / (uint32_t)want - 2048u);
            if (share <= g.wres_bytes) continue;
            const int st = (int)std::min<uint32_t>(8u, (share - g.wres_bytes) / g.stage_bytes);
            if (st >= (NG > 1 ? 3 : 4)) {
                per_sm = want;
                S = st;
            }
        }
        if (per_sm == 0) {
            // wide rows (48 or 96 input channels with W >= 64): one CTA per SM
            // with the stages that fit, at least one per issuer; every stage
            // holds one input plane whose MMAs release it, so the pipeline only
            // runs shallower (the other kernels are several times slower here)
            const int st = g.wres_bytes < budget ? (int)std::min<uint32_t>(8u, (budget - g.wres_bytes) / g.stage_bytes)
                                                 : 0;
            if (st >= 2 && st >= Z::NISS) {
                per_sm = 1;
                S = st;
            }
        }
        if (per_sm == 0) return false;
        g.S = S;
        const long long grid_max = ((long long)per_sm * std::max(1, a.sms) + NG - 1) / NG;  // per channel group
        const long long grid0 = std::min<long long>(nb * g.T * a.D, grid_max);
        zcol_work_split(g, nb * g.T, a.D, grid0);
        const long long grid = g.ZC ? std::min<long long>(grid0, g.nitems) : grid0;
        const uint32_t smem = g.wres_bytes + (uint32_t)S * g.stage_bytes;
        auto k = conv_zcat_kernel<CIN, COUT, Z::COUTH, Z::NB, Z::NISS, Z::PER_SM>;
        err = smem_attributes(k, smem);
        if (err != cudaSuccess) return true;
        ++launch_count;
        k<<<dim3((unsigned)grid, NG), 32 * (ZCAT_ISSUER0 + Z::NISS), smem, s>>>(map, a, g);
        err = cudaGetLastError();
        return true;
    }
}

// the x-pair z-column convolution (conv_zpair_kernel) for 16 input channels;
// false leaves the layer to the others.  IAC_DENOISE_ZPAIR=0 in the
// environment turns it off (for comparing the kernels).
template <int CIN, int COUT>
static bool launch_zpair(const ConvArgs &a, cudaStream_t s, cudaError_t &err)
{
    if constexpr (CIN != 16 || COUT != 16) {  // 32 or 48 outputs: re-staging the slab per group loses
        return false;
    } else {
        static const bool off = [] {
            const char *e = getenv("IAC_DENOISE_ZPAIR");
            return e && e[0] == '0';
        }();
        if (off) return false;
        if (a.c0 != 0 || (a.W & 1) || a.W / 2 + 2 > 256 || a.D < 1) return false;
        if (reinterpret_cast<uintptr_t>(a.src1) & 15) return false;
        PFN_cuTensorMapEncodeTiled enc = tensor_map_encoder();
        if (!enc) return false;
        TmaGeom g{};
        g.Wp = a.W / 2 + 2;                      // padded pairs per row
        g.NR = 3 + (130 + g.Wp - 1) / g.Wp;      // covers rows y_lo .. y_lo + NR - 1 of every tile
        if (g.NR > 256) return false;
        g.T = (a.H * g.Wp + TILE_M - 1) / TILE_M;
        const long long nb = a.V / ((long long)a.D * a.H * a.W);
        g.ntiles = nb * a.D * g.T;
        g.box_bytes = 64u * (uint32_t)g.Wp * (uint32_t)g.NR;
        g.plane_bytes = (g.box_bytes + 1023u) & ~1023u;
        g.slab_bytes = g.plane_bytes;
        g.stage_bytes = g.plane_bytes;
        g.wcopy_bytes = ZPAIR_WBYTES;
        g.wres_bytes = (ZPAIR_WBYTES + 1023u) & ~1023u;
        g.wstage_bytes = 0;
        const uint32_t budget = 227u * 1024u - 2048u;
        if (g.wres_bytes + 4u * g.stage_bytes > budget) return false;
        g.S = (int)std::min<uint32_t>(8u, (budget - g.wres_bytes) / g.stage_bytes);
        constexpr int NG = COUT / 16;  // output-channel groups (blockIdx.y)
        const long long grid_max = ((long long)std::max(1, a.sms) + NG - 1) / NG;  // one CTA per SM
        const long long grid0 = std::min<long long>(nb * g.T * a.D, grid_max);
        zcol_work_split(g, nb * g.T, a.D, grid0);
        CUtensorMap map;
        const cuuint64_t dims[5] = {32u, (cuuint64_t)(a.W / 2), (cuuint64_t)a.H, (cuuint64_t)a.D, (cuuint64_t)nb};
        const cuuint64_t strides[4] = {64u, (cuuint64_t)a.W * 32u, (cuuint64_t)a.H * a.W * 32u,
                                       (cuuint64_t)a.D * a.H * a.W * 32u};
        const cuuint32_t box[5] = {32u, (cuuint32_t)g.Wp, (cuuint32_t)g.NR, 1u, 1u};
        const cuuint32_t estr[5] = {1u, 1u, 1u, 1u, 1u};
        if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16 *>(a.src1), dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
        const uint32_t smem = g.wres_bytes + (uint32_t)g.S * g.stage_bytes;
        const long long grid = std::min<long long>(g.nitems, grid_max);
        auto k = conv_zpair_kernel<COUT>;
        err = smem_attributes(k, smem);
        if (err != cudaSuccess) return true;
        ++launch_count;
        k<<<dim3((unsigned)grid, NG), 32 * (ZPAIR_ISSUER0 + ZPAIR_NISS), smem, s>>>(map, a, g);
        err = cudaGetLastError();
        return true;
    }
}

// the z-column convolution when its weights stay resident and 4+ stages fit;
// false leaves the layer to conv_tma_kernel
template <int CIN, int COUT>
static bool launch_zcol(const ConvArgs &a, const TmaGeom &g0, const CUtensorMap &map, uint32_t budget,
                        cudaStream_t s, cudaError_t &err)
{
    constexpr int NB = ZcolNB<COUT>::value, NB2 = ZcolNB<COUT>::small;
    if constexpr (NB == 0) {
        return false;
    } else {
        const uint32_t w27 = 27u * COUT * CIN * 2;
        if (w27 > 64u * 1024u) return false;
        TmaGeom g = g0;
        g.wcopy_bytes = w27;
        g.wres_bytes = (w27 + 1023u) & ~1023u;
        g.wstage_bytes = 0;
        g.stage_bytes = (g.slab_bytes + 1023u) & ~1023u;
        int per_sm = 0, S = 0;
        zcol_fit(g, budget, tma_tcols(3 * NB * COUT), per_sm, S);
        if constexpr (NB2 != 0) {
            int per_sm2 = 0, S2 = 0;
            zcol_fit(g, budget, tma_tcols(3 * NB2 * COUT), per_sm2, S2);
            if (per_sm2 > per_sm) {  // measured: 16 -> 16 at 8 x 64^3 0.110 -> 0.100 ms with 3 CTAs
                launch_zcol_nb<CIN, COUT, NB2>(a, g, map, per_sm2, S2, s, err);
                return true;
            }
        }
        if (per_sm == 0) return false;
        launch_zcol_nb<CIN, COUT, NB>(a, g, map, per_sm, S, s, err);
        return true;
    }
}

template <int CIN, int COUT>
static bool launch_tma(const ConvArgs &a, cudaStream_t s, cudaError_t &err)
{
    if (a.c0 != 0 || a.W + 2 > 256 || a.D < 1) return false;  // TMA boxes: plain input, rows of <= 256
    PFN_cuTensorMapEncodeTiled enc = tensor_map_encoder();
    if (!enc) return false;
    if ((reinterpret_cast<uintptr_t>(a.src1) & 15) || (reinterpret_cast<uintptr_t>(a.w) & 15)) return false;
    TmaGeom g{};
    g.Wp = a.W + 2;
    g.NR = 3 + (130 + g.Wp - 1) / g.Wp;  // covers rows y_lo .. y_lo + NR - 1 of every tile
    if (g.NR > 256) return false;
    g.T = (a.H * g.Wp + TILE_M - 1) / TILE_M;
    const long long nb = a.V / ((long long)a.D * a.H * a.W);
    g.ntiles = nb * a.D * g.T;
    g.box_bytes = 16u * (uint32_t)g.Wp * (uint32_t)g.NR;
    g.plane_bytes = (g.box_bytes + 127u) & ~127u;
    g.slab_bytes = g.plane_bytes * (CIN / 8);
    const uint32_t w27 = 27u * COUT * CIN * 2;
    const uint32_t budget = 227u * 1024u - 1024u;
    g.wcopy_bytes = (w27 <= 64u * 1024u) ? w27 : 0u;
    g.wres_bytes = (g.wcopy_bytes + 1023u) & ~1023u;
    g.wstage_bytes = g.wres_bytes ? 0u : 9u * COUT * CIN * 2;
    g.stage_bytes = (g.slab_bytes + g.wstage_bytes + 1023u) & ~1023u;
    if (g.wres_bytes && g.wres_bytes + 2 * g.stage_bytes > budget) {  // make room for stages
        g.wres_bytes = 0;
        g.wcopy_bytes = 0;
        g.wstage_bytes = 9u * COUT * CIN * 2;
        g.stage_bytes = (g.slab_bytes + g.wstage_bytes + 1023u) & ~1023u;
    }
    // several CTAs per SM and, where TMEM and shared memory allow, three
    // issuing warps per CTA: the count of MMA issuers per SM sets the MMA
    // rate; 4 stages per CTA when they fit
    auto fit = [&](int ni, int &per_sm, int &S) {
        per_sm = 0;
        S = 0;
        for (int want = std::min(4, (int)(512 / tma_tcols(2 * ni * COUT))); want >= 1; want--) {
            const uint32_t share = (228u * 1024u) / (uint32_t)want - 2048u;
            int st = (int)std::min<uint32_t>(want == 1 ? 8u : 4u,
                                             (std::min(share, budget) - g.wres_bytes) / g.stage_bytes);
            // three issuers: a multiple of 3 stages, so every slot always
            // serves the same issuer and its parity waits stay in phase order
            if (ni == 3) st = st >= 3 ? (st >= 6 ? 6 : 3) : 0;
            if (g.wres_bytes < share && st >= 2) {
                per_sm = want;
                S = st;
                return;
            }
        }
    };
    int per_sm = 0, per_sm3 = 0, S1 = 0, S3 = 0;
    fit(1, per_sm, S1);
    if (2 * 3 * COUT <= 512) fit(3, per_sm3, S3);
    const int ni = (S3 >= 2 && per_sm3 >= per_sm) ? 3 : 1;  // more issuers, no fewer CTAs (measured)
    if (ni == 3) per_sm = per_sm3;
    g.S = ni == 3 ? S3 : S1;
    if (g.S < 2 || g.ntiles == 0) return false;
    const uint32_t smem = g.wres_bytes + (uint32_t)g.S * g.stage_bytes;

    CUtensorMap map;
    const cuuint64_t dims[5] = {(cuuint64_t)CIN, (cuuint64_t)a.W, (cuuint64_t)a.H, (cuuint64_t)a.D, (cuuint64_t)nb};
    const cuuint64_t strides[4] = {(cuuint64_t)CIN * 2, (cuuint64_t)a.W * CIN * 2, (cuuint64_t)a.H * a.W * CIN * 2,
                                   (cuuint64_t)a.D * a.H * a.W * CIN * 2};
    const cuuint32_t box[5] = {8u, (cuuint32_t)g.Wp, (cuuint32_t)g.NR, 1u, 1u};
    const cuuint32_t estr[5] = {1u, 1u, 1u, 1u, 1u};
    const CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16 *>(a.src1), dims, strides, box,
                           estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    if (launch_zpair<CIN, COUT>(a, s, err)) return true;
    if (launch_zcat<CIN, COUT>(a, g, budget, s, err)) return true;
    if (launch_zcol<CIN, COUT>(a, g, map, budget, s, err)) return true;
    const long long grid = std::min<long long>(g.ntiles, (long long)per_sm * std::max(1, a.sms));
    if constexpr (2 * 3 * COUT <= 512) {
        if (ni == 3) {
            err = smem_attributes(conv_tma_kernel<CIN, COUT, 3>, smem);
            if (err != cudaSuccess) return true;
            ++launch_count;
            conv_tma_kernel<CIN, COUT, 3><<<(unsigned)grid, 32 * (5 + 3), smem, s>>>(map, a, g);
            err = cudaGetLastError();
            return true;
        }
    }
    err = smem_attributes(conv_tma_kernel<CIN, COUT, 1>, smem);
    if (err != cudaSuccess) return true;
    ++launch_count;
    conv_tma_kernel<CIN, COUT, 1><<<(unsigned)grid, TMA_THREADS, smem, s>>>(map, a, g);
    err = cudaGetLastError();
    return true;
}

template <int CIN, int COUT>
static cudaError_t launch_conv(const ConvArgs &a, int backend, cudaStream_t s)
{
    const unsigned grid = (unsigned)((a.V + TILE_M - 1) / TILE_M);
    if (backend == BACKEND_TC_SLAB) {
        cudaError_t e = cudaSuccess;
        if (launch_tma<CIN, COUT>(a, s, e)) return e;
        if (launch_slab<CIN, COUT>(a, s, e)) return e;
        backend = BACKEND_TC_TAP;  // a slab stage does not fit in shared memory
    }
    if (backend == BACKEND_TC_TAP) {
        const uint32_t smem = TcCfg<CIN, COUT>::SMEM;
        cudaError_t e = cudaFuncSetAttribute(conv_tc_kernel<CIN, COUT>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        ++launch_count;
        conv_tc_kernel<CIN, COUT><<<grid, CONV_THREADS, smem, s>>>(a);
    } else {
        const uint32_t smem = MmaCfg<CIN, COUT>::SMEM;
        cudaError_t e = cudaFuncSetAttribute(conv_mma_kernel<CIN, COUT>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        ++launch_count;
        conv_mma_kernel<CIN, COUT><<<grid, CONV_THREADS, smem, s>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t conv3x3(const ConvArgs &a, int cin, int cout, int backend, cudaStream_t s)
{
#define IAC_CONV_CASE(CI, CO) \
    if (cin == CI && cout == CO) return launch_conv<CI, CO>(a, backend, s);
    IAC_CONV_CASE(16, 16)
    IAC_CONV_CASE(16, 32)
    IAC_CONV_CASE(32, 32)
    IAC_CONV_CASE(32, 64)
    IAC_CONV_CASE(64, 64)
    IAC_CONV_CASE(96, 32)
    IAC_CONV_CASE(48, 16)
    IAC_CONV_CASE(32, 16)
    IAC_CONV_CASE(64, 32)
    IAC_CONV_CASE(32, 96)
    IAC_CONV_CASE(16, 48)
#undef IAC_CONV_CASE
    return cudaErrorInvalidValue;
}

// --------------------------------------------------------------------------
// first layer (1 input channel): 27 x 16 MACs per voxel on the FP32 pipe.
// A thread takes four consecutive voxels of a row: per (dz, dy) it loads the
// six input values the four need and applies the three dx taps to all four
// (the weights of a tap are read from shared memory once for four voxels, as
// four float4), so the kernel is bound by its FMAs, not by shared-memory
// loads.  Taps outside the volume read 0 (zero padding); a voxel's sums run
// over the taps in order.  W is a multiple of 4.
// --------------------------------------------------------------------------
template <bool VEC>  // VEC: x is 16-byte aligned (the middle four of a row's six loads as one float4)
__global__ void __launch_bounds__(256) conv_first_kernel(const float *__restrict__ x, const bf16 *__restrict__ w,
                                                         const float *__restrict__ bias, bf16 *__restrict__ y,
                                                         int D, int H, int W, long long V)
{
    __shared__ float4 ws[27][4];
    __shared__ float bs[16];
    for (int i = threadIdx.x; i < 27 * 16; i += blockDim.x)
        reinterpret_cast<float *>(ws)[i] = __bfloat162float(w[i]);
    if (threadIdx.x < 16) bs[threadIdx.x] = bias[threadIdx.x];
    __syncthreads();
    const long long v0 = 4 * ((long long)blockIdx.x * blockDim.x + threadIdx.x);  // first of four voxels
    if (v0 >= V) return;
    const Vox q = decode(v0, D, H, W, V);
    float acc[4][16];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int c = 0; c < 16; c++) acc[i][c] = bs[c];
    const long long HW = (long long)H * W;
    const bool left = q.x > 0, right = q.x + 4 < W;
#pragma unroll
    for (int dz = 0; dz < 3; dz++) {
        const bool zin = (unsigned)(q.z + dz - 1) < (unsigned)D;
#pragma unroll
        for (int dy = 0; dy < 3; dy++) {
            const bool in = zin && (unsigned)(q.y + dy - 1) < (unsigned)H;
            const float *row = x + v0 + (dz - 1) * HW + (long long)(dy - 1) * W;  // voxel x0 of the row
            float r[6];
            // the four voxels' own column as one 16-byte load (x0, W and H W are multiples of 4)
            const float4 mid = !in ? make_float4(0.0f, 0.0f, 0.0f, 0.0f)
                                   : (VEC ? *reinterpret_cast<const float4 *>(row)
                                          : make_float4(row[0], row[1], row[2], row[3]));
            r[0] = in && left ? row[-1] : 0.0f;
            r[1] = mid.x;
            r[2] = mid.y;
            r[3] = mid.z;
            r[4] = mid.w;
            r[5] = in && right ? row[4] : 0.0f;
#pragma unroll
            for (int dx = 0; dx < 3; dx++) {
                const int t = 9 * dz + 3 * dy + dx;
#pragma unroll
                for (int c4 = 0; c4 < 4; c4++) {
                    const float4 wv = ws[t][c4];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const float xv = r[i + dx];
                        acc[i][4 * c4] = fmaf(wv.x, xv, acc[i][4 * c4]);
                        acc[i][4 * c4 + 1] = fmaf(wv.y, xv, acc[i][4 * c4 + 1]);
                        acc[i][4 * c4 + 2] = fmaf(wv.z, xv, acc[i][4 * c4 + 2]);
                        acc[i][4 * c4 + 3] = fmaf(wv.w, xv, acc[i][4 * c4 + 3]);
                    }
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        uint4 pk[2];
        uint32_t *u = reinterpret_cast<uint32_t *>(pk);
#pragma unroll
        for (int c = 0; c < 16; c += 2) u[c / 2] = pack_bf16(fmaxf(acc[i][c], 0.0f), fmaxf(acc[i][c + 1], 0.0f));
        uint4 *dst = reinterpret_cast<uint4 *>(y + (v0 + i) * 16);
        dst[0] = pk[0];
        dst[1] = pk[1];
    }
}

cudaError_t conv3x3_first(const float *x, const bf16 *w, const float *bias, bf16 *y, int D, int H, int W,
                          long long V, cudaStream_t s)
{
    if (W % 4) return cudaErrorInvalidValue;
    const long long threads = V / 4;
    ++launch_count;
    if ((reinterpret_cast<uintptr_t>(x) & 15) == 0)
        conv_first_kernel<true><<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(x, w, bias, y, D, H, W, V);
    else
        conv_first_kernel<false><<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(x, w, bias, y, D, H, W, V);
    return cudaGetLastError();
}

// --------------------------------------------------------------------------
// weight gradient: per tap, dW_tap[co][ci] = G^T X_tap over the voxels.
// CTA = one tap x a strided set of 128-voxel blocks; operands are staged as in
// the forward ([k-chunk][voxel][8]) and read with ldmatrix.trans, since here
// the voxels are the GEMM K dimension.  Partial sums are reduced in shared
// memory and added to dW with one fp32 atomic per element per CTA.
// --------------------------------------------------------------------------
template <int CIN, int COUT>
struct WgCfg {
    static constexpr int MT = COUT / 16, NT = CIN / 8;
    static constexpr bool SPLIT_K = MT * NT <= 24;  // warps split voxels, else output tiles
    static constexpr int TILES = SPLIT_K ? MT * NT : MT * NT / 4;
    static constexpr uint32_t G_BYTES = TILE_M * COUT * 2;
    static constexpr uint32_t X_BYTES = TILE_M * CIN * 2;
    static constexpr uint32_t STAGE = G_BYTES + X_BYTES;
    static constexpr int S = 2;
    static constexpr uint32_t SMEM = S * STAGE + COUT * CIN * 4;
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(CONV_THREADS) wgrad_kernel(const WgradArgs a)
{
    using Cfg = WgCfg<CIN, COUT>;
    static_assert(Cfg::SPLIT_K || Cfg::NT % 8 == 0, "tile split: an even number of n tiles per warp");
    extern __shared__ __align__(1024) unsigned char smem[];
    float *red = reinterpret_cast<float *>(smem + Cfg::S * Cfg::STAGE);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tap = blockIdx.y;
    const long long nblk = (a.V + TILE_M - 1) / TILE_M;
    const uint32_t sbase = smem_u32(smem);
    for (int i = tid; i < COUT * CIN; i += CONV_THREADS) red[i] = 0.0f;

    float acc[Cfg::TILES][4];
#pragma unroll
    for (int i = 0; i < Cfg::TILES; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.0f;
    float bsum = 0.0f;  // bias gradient (centre tap, thread co < COUT)

    auto stage_load = [&](int st, long long b) {
        const uint32_t sG = sbase + st * Cfg::STAGE, sX = sG + Cfg::G_BYTES;
        const long long v = b * TILE_M + tid;
        const Vox q = decode(v, a.D, a.H, a.W, a.V);
        const bf16 *gp = a.g + (q.ok ? v : 0) * COUT;
#pragma unroll
        for (int c = 0; c < COUT / 8; c++)
            cp_async16(sG + (uint32_t)((c * TILE_M + tid) * 16), gp + c * 8, q.ok ? 16u : 0u);
        gather_rows<CIN>(sX, a.src0, a.src1, a.c0, a.c1, a.up0, a.D, a.H, a.W, q, tid, tap);
    };

    long long b = blockIdx.x;
    if (b < nblk) stage_load(0, b);
    cp_async_commit();
    int st = 0;
    for (; b < nblk; b += gridDim.x) {
        const long long bn = b + gridDim.x;
        if (bn < nblk) stage_load(st ^ 1, bn);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const uint32_t sG = sbase + st * Cfg::STAGE, sX = sG + Cfg::G_BYTES;
        if (tap == 13 && a.db && tid < COUT) {
            const bf16 *gs = reinterpret_cast<const bf16 *>(smem + st * Cfg::STAGE);
            for (int r = 0; r < TILE_M; r++) bsum += __bfloat162float(gs[((tid >> 3) * TILE_M + r) * 8 + (tid & 7)]);
        }
        if (Cfg::SPLIT_K) {
            // warp w: voxels 32w..32w+31 (2 k16 steps), every (m, n) tile
#pragma unroll
            for (int ks = 0; ks < 2; ks++) {
                const int kb = warp * 32 + ks * 16;
#pragma unroll
                for (int m = 0; m < Cfg::MT; m++) {
                    uint32_t a0, a1, a2, a3;
                    const int vr = kb + (lane & 7) + ((lane >> 4) << 3);
                    const int ch = 2 * m + ((lane >> 3) & 1);
                    ldsm_x4_t(sG + (uint32_t)((ch * TILE_M + vr) * 16), a0, a1, a2, a3);
#pragma unroll
                    for (int n2 = 0; n2 < Cfg::NT / 2; n2++) {
                        uint32_t b0, b1, b2, b3;
                        const int vx = kb + (lane & 7) + (((lane >> 3) & 1) << 3);
                        const int cx = 2 * n2 + (lane >> 4);
                        ldsm_x4_t(sX + (uint32_t)((cx * TILE_M + vx) * 16), b0, b1, b2, b3);
                        mma_bf16(acc[m * Cfg::NT + 2 * n2], a0, a1, a2, a3, b0, b1);
                        mma_bf16(acc[m * Cfg::NT + 2 * n2 + 1], a0, a1, a2, a3, b2, b3);
                    }
                }
            }
        } else {
            // warp w: every voxel, n tiles [w*NT/4, (w+1)*NT/4) of every m tile
            constexpr int NW = Cfg::NT / 4;
#pragma unroll
            for (int ks = 0; ks < TILE_M / 16; ks++) {
                const int kb = ks * 16;
#pragma unroll
                for (int m = 0; m < Cfg::MT; m++) {
                    uint32_t a0, a1, a2, a3;
                    const int vr = kb + (lane & 7) + ((lane >> 4) << 3);
                    const int ch = 2 * m + ((lane >> 3) & 1);
                    ldsm_x4_t(sG + (uint32_t)((ch * TILE_M + vr) * 16), a0, a1, a2, a3);
#pragma unroll
                    for (int n2 = 0; n2 < NW / 2; n2++) {
                        uint32_t b0, b1, b2, b3;
                        const int vx = kb + (lane & 7) + (((lane >> 3) & 1) << 3);
                        const int cx = warp * NW + 2 * n2 + (lane >> 4);
                        ldsm_x4_t(sX + (uint32_t)((cx * TILE_M + vx) * 16), b0, b1, b2, b3);
                        mma_bf16(acc[m * NW + 2 * n2], a0, a1, a2, a3, b0, b1);
                        mma_bf16(acc[m * NW + 2 * n2 + 1], a0, a1, a2, a3, b2, b3);
                    }
                }
            }
        }
        __syncthreads();  // the stage is refilled two blocks on
        st ^= 1;
    }
    cp_async_wait_all();
    // reduce: accumulator element j of tile (m, n): co = m*16 + g + 8*(j>>1), ci = n*8 + 2*tq + (j&1)
    const int g = lane >> 2, tq = lane & 3;
    constexpr int NW = Cfg::SPLIT_K ? Cfg::NT : Cfg::NT / 4;
#pragma unroll
    for (int i = 0; i < Cfg::TILES; i++) {
        const int m = i / NW;
        const int n = Cfg::SPLIT_K ? (i % NW) : warp * NW + (i % NW);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int co = m * 16 + g + 8 * (j >> 1), ci = n * 8 + 2 * tq + (j & 1);
            atomicAdd(&red[co * CIN + ci], acc[i][j]);
        }
    }
    __syncthreads();
    for (int i = tid; i < COUT * CIN; i += CONV_THREADS) {
        const int co = i / CIN, ci = i % CIN;
        const float r = red[i];
        if (r != 0.0f) atomicAdd(&a.dw[((size_t)co * 27 + tap) * CIN + ci], r);
    }
    if (tap == 13 && a.db && tid < COUT && bsum != 0.0f) atomicAdd(&a.db[tid], bsum);
}

template <int CIN, int COUT>
static cudaError_t launch_wgrad(const WgradArgs &a, int sms, cudaStream_t s)
{
    using Cfg = WgCfg<CIN, COUT>;
    const long long nblk = (a.V + TILE_M - 1) / TILE_M;
    const int per_tap = (int)std::max<long long>(1, std::min<long long>(nblk, (4LL * sms + 26) / 27 * 2));
    cudaError_t e = cudaFuncSetAttribute(wgrad_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)Cfg::SMEM);
    if (e != cudaSuccess) return e;
    ++launch_count;
    wgrad_kernel<CIN, COUT><<<dim3(per_tap, 27), CONV_THREADS, Cfg::SMEM, s>>>(a);
    return cudaGetLastError();
}

// Weight gradient on slabs.  The 128-position tiles of the forward slab
// kernel are the K dimension here: a CTA owns G taps of one dz (G = 9, 3 or 1,
// as many as its registers hold: G * cout * cin / 32 accumulators per thread)
// and walks tiles; per tile it stages the gradient rows (zero at halo
// columns, so only real voxels count) and the dz slab of X once, and every
// tap of the group reads the slab at its row offset.  Warps split the tile's
// positions; partial sums are reduced in shared memory, then one fp32 atomic
// per weight per CTA.
template <int CIN, int COUT>
struct WgsCfg {
    static constexpr int MT = COUT / 16, NT = CIN / 8;
    static constexpr int G = 9 * MT * NT * 4 <= 96 ? 9 : (3 * MT * NT * 4 <= 96 ? 3 : 1);
    static constexpr uint32_t G_BYTES = TILE_M * COUT * 2;
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(CONV_THREADS) wgrad_slab_kernel(const WgradArgs a, const SlabGeom g)
{
    using Cfg = WgsCfg<CIN, COUT>;
    constexpr int MT = Cfg::MT, NT = Cfg::NT, G = Cfg::G;
    extern __shared__ __align__(1024) unsigned char smem[];
    const uint32_t stage_bytes = g.stage_bytes;  // G tile + slab
    float *red = reinterpret_cast<float *>(smem + 2 * stage_bytes);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tap0 = blockIdx.y * G;
    const int dz = tap0 / 9 - 1;
    const uint32_t sbase = smem_u32(smem);
    for (int i = tid; i < G * COUT * CIN; i += CONV_THREADS) red[i] = 0.0f;
    const bool bias = a.db && tap0 <= 13 && 13 < tap0 + G;
    const int HW = a.H * a.W;

    float acc[G][MT][NT][4];
#pragma unroll
    for (int t = 0; t < G; t++)
#pragma unroll
        for (int m = 0; m < MT; m++)
#pragma unroll
            for (int n = 0; n < NT; n++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[t][m][n][j] = 0.0f;
    float bsum = 0.0f;

    auto load = [&](int st, long long tile) {
        const uint32_t sG = sbase + (uint32_t)st * stage_bytes, sS = sG + Cfg::G_BYTES;
        const long long plane = tile / g.T;
        const int q0 = (int)(tile % g.T) * TILE_M;
        const int n = (int)(plane / a.D), z = (int)(plane % a.D);
        // gradient rows of the tile's positions (zero at halo columns / past the plane)
        {
            const int q = q0 + tid;
            const int y = q / g.Wp, xp = q - (q / g.Wp) * g.Wp;
            const bool ok = y < a.H && xp >= 1 && xp <= a.W;
            const bf16 *gp = a.g + (ok ? ((long long)plane * HW + (long long)y * a.W + (xp - 1)) * COUT : 0);
#pragma unroll
            for (int c = 0; c < COUT / 8; c++)
                cp_async16(sG + (uint32_t)((c * TILE_M + tid) * 16), gp + c * 8, ok ? 16u : 0u);
        }
        slab_rows<CIN>(sS, g, q0, n, z + dz, a.src0, a.src1, a.c0, a.c1, a.up0, a.D, a.H, a.W, tid);
    };

    long long tile = blockIdx.x;
    if (tile < g.ntiles) load(0, tile);
    cp_async_commit();
    int st = 0;
    for (; tile < g.ntiles; tile += gridDim.x) {
        const long long nxt = tile + gridDim.x;
        if (nxt < g.ntiles) load(st ^ 1, nxt);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const uint32_t sG = sbase + (uint32_t)st * stage_bytes, sS = sG + Cfg::G_BYTES;
        if (bias && tid < COUT) {
            const bf16 *gs = reinterpret_cast<const bf16 *>(smem + (size_t)st * stage_bytes);
            for (int r = 0; r < TILE_M; r++) bsum += __bfloat162float(gs[((tid >> 3) * TILE_M + r) * 8 + (tid & 7)]);
        }
#pragma unroll
        for (int ks = 0; ks < 2; ks++) {
            const int kb = warp * 32 + ks * 16;
            uint32_t af[MT][4];
#pragma unroll
            for (int m = 0; m < MT; m++) {
                const int vr = kb + (lane & 7) + ((lane >> 4) << 3);
                const int ch = 2 * m + ((lane >> 3) & 1);
                ldsm_x4_t(sG + (uint32_t)((ch * TILE_M + vr) * 16), af[m][0], af[m][1], af[m][2], af[m][3]);
            }
#pragma unroll
            for (int t = 0; t < G; t++) {
                const int tap = tap0 + t;
                const int r0 = g.Wp + 1 + ((tap / 3) % 3 - 1) * g.Wp + (tap % 3 - 1);
#pragma unroll
                for (int n2 = 0; n2 < NT / 2; n2++) {
                    uint32_t b0, b1, b2, b3;
                    const int vx = r0 + kb + (lane & 7) + (((lane >> 3) & 1) << 3);
                    const int cx = 2 * n2 + (lane >> 4);
                    ldsm_x4_t(sS + (uint32_t)((cx * g.R + vx) * 16), b0, b1, b2, b3);
#pragma unroll
                    for (int m = 0; m < MT; m++) {
                        mma_bf16(acc[t][m][2 * n2], af[m][0], af[m][1], af[m][2], af[m][3], b0, b1);
                        mma_bf16(acc[t][m][2 * n2 + 1], af[m][0], af[m][1], af[m][2], af[m][3], b2, b3);
                    }
                }
            }
        }
        __syncthreads();  // the stage is refilled on the next iteration
        st ^= 1;
    }
    cp_async_wait_all();
    const int gq = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int t = 0; t < G; t++)
#pragma unroll
        for (int m = 0; m < MT; m++)
#pragma unroll
            for (int n = 0; n < NT; n++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int co = m * 16 + gq + 8 * (j >> 1), ci = n * 8 + 2 * tq + (j & 1);
                    atomicAdd(&red[(t * COUT + co) * CIN + ci], acc[t][m][n][j]);
                }
    __syncthreads();
    for (int i = tid; i < G * COUT * CIN; i += CONV_THREADS) {
        const int t = i / (COUT * CIN), co = (i / CIN) % COUT, ci = i % CIN;
        const float r = red[i];
        if (r != 0.0f) atomicAdd(&a.dw[((size_t)co * 27 + tap0 + t) * CIN + ci], r);
    }
    if (bias && tid < COUT && bsum != 0.0f) atomicAdd(&a.db[tid], bsum);
}

template <int CIN, int COUT>
static bool launch_wgrad_slab(const WgradArgs &a, int sms, cudaStream_t s, cudaError_t &err)
{
    using Cfg = WgsCfg<CIN, COUT>;
    SlabGeom g{};
    g.Wp = a.W + 2;
    g.R = TILE_M + 2 * g.Wp + 2;
    g.T = (a.H * g.Wp + TILE_M - 1) / TILE_M;
    const long long nb = a.V / ((long long)a.D * a.H * a.W);
    g.ntiles = nb * a.D * g.T;
    g.slab_bytes = (uint32_t)g.R * CIN * 2;
    g.stage_bytes = Cfg::G_BYTES + g.slab_bytes;
    g.S = 2;
    const uint32_t smem = 2 * g.stage_bytes + (uint32_t)Cfg::G * COUT * CIN * 4;
    // with one tap per CTA a slab (R rows) costs more than the tap's own 128 rows
    if (Cfg::G == 1 || smem > 227u * 1024u - 512u || g.ntiles == 0) return false;
    err = cudaFuncSetAttribute(wgrad_slab_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return true;
    err = cudaFuncSetAttribute(wgrad_slab_kernel<CIN, COUT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                               (int)cudaSharedmemCarveoutMaxShared);
    if (err != cudaSuccess) return true;
    const int groups = 27 / Cfg::G;
    // about 4 CTAs per SM in total, at least 2 tiles per CTA
    const long long per_group = std::max<long long>(
        1, std::min<long long>((g.ntiles + 1) / 2, (4LL * std::max(1, sms) + groups - 1) / groups));
    ++launch_count;
    wgrad_slab_kernel<CIN, COUT><<<dim3((unsigned)per_group, groups), CONV_THREADS, smem, s>>>(a, g);
    err = cudaGetLastError();
    return true;
}

// Weight gradient on tcgen05, fed by TMA.  Per tap, dW_t^T[ci][co] =
// sum_q X[q + off(t)][ci] G[q][co] is a GEMM with M = input channels, N =
// output channels and K = positions.  The staged slab ([chunk][position][8
// channels]) is exactly the canonical MN-major, non-swizzled operand layout
// (8 channels x 8 positions per 128-byte core matrix, channel groups one
// plane apart, position groups 128 B apart), so the tap shift is again a
// descriptor offset.  M = 64 rows per MMA (input channels beyond cin read
// padding and are dropped); the accumulators of every tap of the CTA's group
// live in TMEM for the whole launch and are read once at the end.  Warp 4
// loads stages with TMA, warps 5.. issue the MMAs (each a share of the taps:
// a tcgen05.mma takes its issuing thread ~150 cycles whatever its shape while
// the tensor pipe accepts one every ~40, so several issuers keep it busy),
// warps 0-3 drain TMEM.
struct WTGeom {
    int Wp, NR, NRg, T;
    int KT;                        // positions per tile (wgrad_zs_kernel; TILE_M elsewhere)
    long long ntiles;
    uint32_t planeX, planeG;       // one channel-chunk plane of X / of the gradient in a stage
    uint32_t boxX, boxG;           // bytes one box delivers
    uint32_t stage_bytes;
    int S;
};

constexpr int WT_THREADS = 448;  // at most: warps 0-3 drain, 4 loads, 5.. issue (NI <= 9)

template <int CIN, int COUT>
struct WtcCfg {
    // rows per MMA: 64, or 128 above 64 input channels (an MMA takes one issue
    // slot of the tensor pipe whatever its M, so fewer, taller MMAs pay)
    static constexpr int MR = CIN > 64 ? 128 : 64;
    static constexpr int MB = (CIN + MR - 1) / MR;  // M blocks of MR input channels
    static constexpr int G = 9 * COUT * MB <= 512 ? 9 : (3 * COUT * MB <= 512 ? 3 : 1);
    static constexpr int COLS = G * COUT * MB;
    static constexpr uint32_t TCOLS = COLS <= 32 ? 32 : (COLS <= 64 ? 64 : (COLS <= 128 ? 128 : (COLS <= 256 ? 256 : 512)));
    static constexpr int PAD_PLANES = MB * MR / 8 - CIN / 8;  // planes read past the slab by the padded M rows
    static constexpr int NI = G >= 9 ? 9 : (G >= 3 ? 3 : 1);  // MMA-issuing warps, G / NI taps each
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(WT_THREADS) wgrad_tc_kernel(const __grid_constant__ CUtensorMap xmap,
                                                              const __grid_constant__ CUtensorMap gmap,
                                                              const WgradArgs a, const WTGeom g)
{
    using Cfg = WtcCfg<CIN, COUT>;
    constexpr int G = Cfg::G, MB = Cfg::MB, NI = Cfg::NI;
    constexpr int MR = Cfg::MR;
    constexpr uint32_t IDESC = idesc_bf16(MR, COUT) | (1u << 15) | (1u << 16);  // A and B MN-major
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[8], empty[8], done;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_err;
    __shared__ long long s_issued, s_consumed[NI];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tap0 = blockIdx.y * G;
    const int dz = tap0 / 9 - 1;
    const uint32_t sbase = smem_u32(smem);
    const uint32_t xbytes = (CIN / 8) * g.planeX;
    if (tid == 0) {
        for (int k = 0; k < g.S; k++) {
            mbar_init(smem_u32(&full[k]), 1);
            mbar_init(smem_u32(&empty[k]), NI);  // one commit per issuing warp
        }
        mbar_init(smem_u32(&done), NI);
        fence_mbar_init();
        s_err = 0;
        s_issued = 0;
        for (int i = 0; i < NI; i++) s_consumed[i] = 0;
    }
    if (warp == 5) {
        tmem_alloc(smem_u32(&s_tmem), Cfg::TCOLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const long long my_tiles =
        blockIdx.x < g.ntiles ? (g.ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;

    if (warp == 4) {
        if (lane == 0) {
            for (long long k = 0; k < my_tiles; k++) {
                const int slot = (int)(k % g.S);
                if (k >= g.S && !mbar_wait_flag(smem_u32(&empty[slot]), (uint32_t)(((k / g.S) - 1) & 1), &s_err))
                    break;
                const long long tile = blockIdx.x + k * (long long)gridDim.x;
                const long long plane = tile / g.T;
                const int q0 = (int)(tile % g.T) * TILE_M;
                const int n = (int)(plane / a.D), z = (int)(plane % a.D);
                const int y_lo = floor_div(q0 - g.Wp - 1, g.Wp), yg_lo = q0 / g.Wp;
                const uint32_t st = sbase + (uint32_t)slot * g.stage_bytes;
                const uint32_t fb = smem_u32(&full[slot]);
                mbar_expect_tx(fb, (CIN / 8) * g.boxX + (COUT / 8) * g.boxG);
#pragma unroll
                for (int c = 0; c < CIN / 8; c++) tma_load_5d(st + c * g.planeX, &xmap, c * 8, -1, y_lo, z + dz, n, fb);
#pragma unroll
                for (int c = 0; c < COUT / 8; c++)
                    tma_load_5d(st + xbytes + c * g.planeG, &gmap, c * 8, -1, yg_lo, z, n, fb);
                s_issued = k + 1;
            }
        }
    } else if (warp >= 5 && warp < 5 + NI) {
        const int iw = warp - 5;  // this warp's taps: [iw G / NI, (iw + 1) G / NI)
        if (lane == 0) {
            for (long long k = 0; k < my_tiles; k++) {
                const int slot = (int)(k % g.S);
                if (!mbar_wait_flag(smem_u32(&full[slot]), (uint32_t)((k / g.S) & 1), &s_err)) break;
                tc_fence_after();
                const long long tile = blockIdx.x + k * (long long)gridDim.x;
                const int q0 = (int)(tile % g.T) * TILE_M;
                const int rel = q0 - floor_div(q0 - g.Wp - 1, g.Wp) * g.Wp;
                const int relg = q0 - (q0 / g.Wp) * g.Wp;
                const uint32_t sX = sbase + (uint32_t)slot * g.stage_bytes, sG = sX + xbytes;
#pragma unroll 1
                for (int t = iw * (G / NI); t < (iw + 1) * (G / NI); t++) {
                    const int tap = tap0 + t;
                    const int r0 = rel + ((tap / 3) % 3 - 1) * g.Wp + (tap % 3 - 1);
#pragma unroll
                    for (int mb = 0; mb < MB; mb++) {
                        const uint32_t dcol = tmem + (uint32_t)((t * MB + mb) * COUT);
#pragma unroll
                        for (int ks = 0; ks < TILE_M / 16; ks++) {
                            const uint64_t da = smem_desc(sX + (uint32_t)(mb * (MR / 8)) * g.planeX + (uint32_t)(r0 + 16 * ks) * 16,
                                                          128, g.planeX);
                            const uint64_t db = smem_desc(sG + (uint32_t)(relg + 16 * ks) * 16, 128, g.planeG);
                            umma_bf16(dcol, da, db, IDESC, (k > 0 || ks > 0) ? 1u : 0u);
                        }
                    }
                }
                umma_commit(smem_u32(&empty[slot]));
                s_consumed[iw] = k + 1;
            }
            if (!s_err && my_tiles > 0) umma_commit(smem_u32(&done));
        }
    }
    __syncthreads();
    // drain: warps 0-3 read the accumulators (thread = TMEM lane) and add them to dW
    const bool ok = !s_err && my_tiles > 0;
    if (warp < 4 && ok) {
        if (!mbar_wait(smem_u32(&done), 0)) s_err = 1;
    }
    __syncthreads();
    if (warp < 4 && ok && !s_err) {
        tc_fence_after();
        // an M = 64 accumulator keeps row i in TMEM lane 32 (i / 16) + i % 16:
        // lanes 0-15 of each warp's quadrant
        // (M = 128: row i in lane i)
        const int row = MR == 128 ? warp * 32 + lane : (lane < 16 ? warp * 16 + lane : -1);
#pragma unroll 1
        for (int blk = 0; blk < G * MB; blk++) {
            uint32_t r[COUT];
#pragma unroll
            for (int c = 0; c < COUT; c += 16) {
                uint32_t (&rr)[16] = *reinterpret_cast<uint32_t(*)[16]>(&r[c]);
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(blk * COUT + c), rr);
            }
            tmem_wait_ld();
            const int t = blk / MB, mb = blk % MB;
            const int ci = mb * MR + row;
            if (row >= 0 && ci < CIN) {
#pragma unroll
                for (int co = 0; co < COUT; co++) {
                    const float v = __uint_as_float(r[co]);
                    if (v != 0.0f) atomicAdd(&a.dw[((size_t)co * 27 + tap0 + t) * CIN + ci], v);
                }
            }
        }
        tc_fence_before();
    }
    if (s_err && tid == 0) {
        note_timeout(a.counters, SITE_WGRAD_TC);
        long long consumed = s_consumed[0];
        for (int i = 1; i < NI; i++) consumed = s_consumed[i] < consumed ? s_consumed[i] : consumed;
        for (long long k = consumed; k < s_issued; k++)
            mbar_wait(smem_u32(&full[k % g.S]), (uint32_t)((k / g.S) & 1));
        if (consumed > 0) {
            const long long k = consumed - 1;
            mbar_wait(smem_u32(&empty[k % g.S]), (uint32_t)((k / g.S) & 1));
        }
    }
    __syncthreads();
    if (warp == 5) {
        tc_fence_after();
        tmem_dealloc(tmem, Cfg::TCOLS);
    }
}

// --------------------------------------------------------------------------
// weight gradient with the three dz planes stacked into one MMA operand.
// wgrad_tc_kernel runs one dz per CTA (blockIdx.y), so an MMA has M = cin
// rows (64 for 16 or 48 channels, 25-75 % of them padding) and N = cout = 16
// columns, and each stage's X and gradient slabs are staged three times.
// Here one stage holds all that one tile needs for its 27 taps, laid out so
// that the dz axis becomes part of an MMA dimension (the chunk planes of
// consecutive slabs are equally spaced, so they stack in one descriptor).
// A stage covers ZSTEP gradient planes z0 .. z0 + ZSTEP - 1 and stacks NX X
// slabs (planes z0 + XLO ..) along M and NG gradient slabs (planes z0 + GLO ..)
// along N; the block of X plane p and gradient plane p' holds the dz = p - p'
// term of output plane p', kept where |dz| <= 1:
//   MODE 0: X planes z-1, z, z+1 along M (M = 3 cin), the gradient of plane z
//           as B (N = cout);
//   MODE 1: the X plane z as A (M = cin), gradient planes z-1, z, z+1 along N;
//   MODE 2: X planes z0-1 .. z0+3 along M, gradient planes z0 .. z0+2 along N:
//           three output planes per stage, 9 of the 15 blocks kept, a third
//           of the MMAs (and of the X slab loads) of MODE 0 per output plane.
// Either way a stage yields every tap of the tile: issuer warp 5 + t takes
// the in-plane tap t = 3 (dy + 1) + dx + 1 and accumulates its (M x N) block
// in TMEM for the whole launch.  Where nine such blocks exceed TMEM's 512
// columns (96 -> 32: N = 96; 32 -> 64: N = 64), blockIdx.y splits the nine
// in-plane taps into groups of five and four, each group staging the tiles
// on its own.  Stages of every (item, plane, tile) are
// independent (planes outside the volume arrive as zeros), so the CTAs are
// persistent over all tiles; a tile is KT consecutive padded positions of a
// plane (K = KT per stage: longer tiles stage fewer halo rows per position).
// Slabs arrive as one swizzled TMA box per 32 channels (64-byte rows) where the
// channel count is a multiple of 32, else per 16 (32-byte rows), stage planes
// [position][channels], read as MN-major operands: the TMA unit moves about one
// box row per clock, so wider rows stage a slab in fewer rows than the
// unswizzled layout's 16-byte rows.
// The bias gradient comes with it: the first of the padding rows of A is a
// plane of ones, written once into every stage slot, so its accumulator row
// holds sum_v G[v][co] (the gradient is zero at the padded positions).
// --------------------------------------------------------------------------
template <int CIN, int COUT, int MODE>
struct WzsCfg {
    static constexpr int NX = MODE == 0 ? 3 : (MODE == 1 ? 1 : 5);  // X planes per stage (along M)
    static constexpr int NG = MODE == 0 ? 1 : 3;                     // gradient planes per stage (along N)
    static constexpr int ZSTEP = MODE == 2 ? 3 : 1;                  // gradient planes a stage owns
    static constexpr int XLO = MODE == 1 ? 0 : -1;                   // first X plane - z0
    static constexpr int GLO = MODE == 1 ? -1 : 0;                   // first gradient plane - z0
    static constexpr int MROWS = NX * CIN;              // real M rows
    static constexpr int MR = MROWS > 64 ? 128 : 64;    // rows per MMA
    static constexpr int MB = (MROWS + MR - 1) / MR;    // M blocks
    static constexpr int N = NG * COUT;                 // MMA columns
    // in-plane taps per CTA: all nine, or the fewest groups whose accumulators fit TMEM
    static constexpr int NTG = 9 * N * MB <= 512 ? 1 : (5 * N * MB <= 512 ? 2 : (3 * N * MB <= 512 ? 3 : 9));
    static constexpr int TPG = (9 + NTG - 1) / NTG;     // taps of a group (the last may have fewer)
    static constexpr int COLS = TPG * N * MB;
    static constexpr uint32_t TCOLS = COLS <= 32 ? 32 : (COLS <= 64 ? 64 : (COLS <= 128 ? 128 : (COLS <= 256 ? 256 : 512)));
    // channels per staged plane (a swizzled row of 64 or 32 bytes): 32 where they divide
    static constexpr int XW = CIN % 32 == 0 ? 32 : 16;
    static constexpr int GW = COUT % 32 == 0 ? 32 : 16;
    static constexpr int XREAL = NX * CIN / XW;         // X planes loaded
    static constexpr int XPLANES = MB * MR / XW;        // X planes the MMAs read (padding rows: garbage)
    static constexpr int GPLANES = NG * COUT / GW;
    static constexpr bool OK = COLS <= 512 && N <= 256 && N % (MR == 128 ? 16 : 8) == 0 && XPLANES > XREAL &&
                               NTG <= 3 && CIN % 16 == 0 && COUT % 16 == 0;
};

template <int CIN, int COUT, int MODE>
__global__ void __launch_bounds__(WT_THREADS) wgrad_zs_kernel(const __grid_constant__ CUtensorMap xmap,
                                                              const __grid_constant__ CUtensorMap gmap,
                                                              const WgradArgs a, const WTGeom g)
{
    using Z = WzsCfg<CIN, COUT, MODE>;
    constexpr int MB = Z::MB, MR = Z::MR, N = Z::N;
    constexpr uint32_t IDESC = idesc_bf16(MR, N) | (1u << 15) | (1u << 16);  // A and B MN-major
    constexpr int NI = Z::TPG;  // issuing warps: one per in-plane tap of this CTA's group
    const int tg0 = (int)blockIdx.y * Z::TPG;                     // first in-plane tap of the group
    const int ntap = 9 - tg0 < Z::TPG ? 9 - tg0 : Z::TPG;         // taps of the group
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[8], empty[8], done;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_err;
    __shared__ long long s_issued, s_consumed[NI];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = smem_u32(smem);
    const uint32_t xbytes = (uint32_t)Z::XPLANES * g.planeX;
    static_assert(Z::XPLANES > Z::XREAL, "a padding plane of A carries the ones of the bias gradient");
    // the ones plane of every stage slot (never written by the loads)
    for (int k = 0; k < g.S; k++) {
        uint4 *ones = reinterpret_cast<uint4 *>(smem + (size_t)k * g.stage_bytes + (size_t)Z::XREAL * g.planeX);
        for (uint32_t i = tid; i < g.planeX / 16; i += blockDim.x) ones[i] = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u);
    }
    fence_proxy_async();  // written by threads, read by the tensor core
    if (tid == 0) {
        for (int k = 0; k < g.S; k++) {
            mbar_init(smem_u32(&full[k]), 1);
            mbar_init(smem_u32(&empty[k]), ntap);  // one commit per issuing warp
        }
        mbar_init(smem_u32(&done), ntap);
        fence_mbar_init();
        s_err = 0;
        s_issued = 0;
        for (int i = 0; i < NI; i++) s_consumed[i] = 0;
    }
    if (warp == 5) {
        tmem_alloc(smem_u32(&s_tmem), Z::TCOLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const long long my_tiles =
        blockIdx.x < g.ntiles ? (g.ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;

    if (warp == 4) {
        if (lane == 0) {
            for (long long k = 0; k < my_tiles; k++) {
                const int slot = (int)(k % g.S);
                if (k >= g.S && !mbar_wait_flag(smem_u32(&empty[slot]), (uint32_t)(((k / g.S) - 1) & 1), &s_err))
                    break;
                const long long tile = blockIdx.x + k * (long long)gridDim.x;
                const long long plane = tile / g.T;  // (batch item, group of ZSTEP gradient planes)
                const int q0 = (int)(tile % g.T) * g.KT;
                const int nzg = (a.D + Z::ZSTEP - 1) / Z::ZSTEP;
                const int n = (int)(plane / nzg), z0 = (int)(plane % nzg) * Z::ZSTEP;
                const int y_lo = floor_div(q0 - g.Wp - 1, g.Wp), yg_lo = q0 / g.Wp;
                const uint32_t st = sbase + (uint32_t)slot * g.stage_bytes;
                const uint32_t fb = smem_u32(&full[slot]);
                mbar_expect_tx(fb, (uint32_t)Z::XREAL * g.boxX + (uint32_t)Z::GPLANES * g.boxG);
#pragma unroll
                for (int b = 0; b < Z::NX; b++)
#pragma unroll
                    for (int c = 0; c < CIN / Z::XW; c++)
                        tma_load_5d(st + (uint32_t)(b * (CIN / Z::XW) + c) * g.planeX, &xmap, c * Z::XW, -1, y_lo,
                                    z0 + Z::XLO + b, n, fb);
#pragma unroll
                for (int pg = 0; pg < Z::NG; pg++)
#pragma unroll
                    for (int c = 0; c < COUT / Z::GW; c++)
                        tma_load_5d(st + xbytes + (uint32_t)(pg * (COUT / Z::GW) + c) * g.planeG, &gmap, c * Z::GW, -1,
                                    yg_lo, z0 + Z::GLO + pg, n, fb);
                s_issued = k + 1;
            }
        }
    } else if (warp >= 5 && warp < 5 + ntap) {
        const int tl = warp - 5, t = tg0 + tl;  // in-plane tap 3 (dy + 1) + dx + 1
        if (lane == 0) {
            for (long long k = 0; k < my_tiles; k++) {
                const int slot = (int)(k % g.S);
                if (!mbar_wait_flag(smem_u32(&full[slot]), (uint32_t)((k / g.S) & 1), &s_err)) break;
                tc_fence_after();
                const long long tile = blockIdx.x + k * (long long)gridDim.x;
                const int q0 = (int)(tile % g.T) * g.KT;
                const int rel = q0 - floor_div(q0 - g.Wp - 1, g.Wp) * g.Wp;
                const int relg = q0 - (q0 / g.Wp) * g.Wp;
                const int r0 = rel + (t / 3 - 1) * g.Wp + (t % 3 - 1);
                const uint32_t sX = sbase + (uint32_t)slot * g.stage_bytes, sG = sX + xbytes;
                // descriptors advance by 16 positions (16 rows, RB units of 16 B) per K step
                constexpr uint32_t RBX = 2 * Z::XW, RBG = 2 * Z::GW;  // bytes per staged row
                const uint64_t db0 = smem_desc_swz_mn(sG + (uint32_t)relg * RBG, RBG, g.planeG);
#pragma unroll
                for (int mb = 0; mb < MB; mb++) {
                    const uint32_t dcol = tmem + (uint32_t)((tl * MB + mb) * N);
                    const uint64_t da0 = smem_desc_swz_mn(
                        sX + (uint32_t)(mb * (MR / Z::XW)) * g.planeX + (uint32_t)r0 * RBX, RBX, g.planeX);
                    const int nks = g.KT / 16;
#pragma unroll 8
                    for (int ks = 0; ks < nks; ks++)
                        umma_bf16(dcol, da0 + (uint64_t)(RBX * ks), db0 + (uint64_t)(RBG * ks), IDESC,
                                  (k > 0 || ks > 0) ? 1u : 0u);
                }
                umma_commit(smem_u32(&empty[slot]));
                s_consumed[tl] = k + 1;
            }
            if (!s_err && my_tiles > 0) umma_commit(smem_u32(&done));
        }
    }
    __syncthreads();
    // drain: warps 0-3 read the accumulators (thread = TMEM lane) and add them to dW
    const bool ok = !s_err && my_tiles > 0;
    if (warp < 4 && ok) {
        if (!mbar_wait(smem_u32(&done), 0)) s_err = 1;
    }
    __syncthreads();
    if (warp < 4 && ok && !s_err) {
        tc_fence_after();
        // an M = 64 accumulator keeps row i in TMEM lane 32 (i / 16) + i % 16; M = 128: row i in lane i
        const int row = MR == 128 ? warp * 32 + lane : (lane < 16 ? warp * 16 + lane : -1);
#pragma unroll 1
        for (int blk = 0; blk < ntap * MB; blk++) {
            uint32_t r[N];
#pragma unroll
            for (int c = 0; c < N; c += 16) {
                uint32_t (&rr)[16] = *reinterpret_cast<uint32_t(*)[16]>(&r[c]);
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(blk * N + c), rr);
            }
            tmem_wait_ld();
            const int t = tg0 + blk / MB, mb = blk % MB;
            const int m = mb * MR + row;
            if (a.db && t == 4 && row >= 0 && m == Z::XREAL * Z::XW) {  // the ones row: sum_v G[v][co]
#pragma unroll
                for (int nn = 0; nn < N; nn++) {
                    const int c = nn / COUT;  // gradient plane z0 + GLO + c: counted by the stage that owns it
                    if (Z::GLO + c < 0 || Z::GLO + c >= Z::ZSTEP) continue;
                    const float v = __uint_as_float(r[nn]);
                    if (v != 0.0f) atomicAdd(&a.db[nn % COUT], v);
                }
            }
            if (row >= 0 && m < Z::MROWS) {  // row b cin + ci (X plane b), column c cout + co (gradient plane c)
                const int b = m / CIN, ci = m % CIN;
#pragma unroll
                for (int nn = 0; nn < N; nn++) {
                    const int dz = (Z::XLO + b) - (Z::GLO + nn / COUT);
                    if (dz < -1 || dz > 1) continue;
                    const float v = __uint_as_float(r[nn]);
                    if (v != 0.0f) atomicAdd(&a.dw[((size_t)(nn % COUT) * 27 + 9 * (dz + 1) + t) * CIN + ci], v);
                }
            }
        }
        tc_fence_before();
    }
    if (s_err && tid == 0) {
        note_timeout(a.counters, SITE_WGRAD_ZS);
        long long consumed = s_consumed[0];
        for (int i = 1; i < ntap; i++) consumed = s_consumed[i] < consumed ? s_consumed[i] : consumed;
        for (long long k = consumed; k < s_issued; k++)
            mbar_wait(smem_u32(&full[k % g.S]), (uint32_t)((k / g.S) & 1));
        if (consumed > 0) {
            const long long k = consumed - 1;
            mbar_wait(smem_u32(&empty[k % g.S]), (uint32_t)((k / g.S) & 1));
        }
    }
    __syncthreads();
    if (warp == 5) {
        tc_fence_after();
        tmem_dealloc(tmem, Z::TCOLS);
    }
}

// bias gradient: db[c] += sum_v g[v][c]
__global__ void bias_grad_kernel(const bf16 *__restrict__ g, int C, long long V, float *__restrict__ db)
{
    extern __shared__ float part[];
    const int c = threadIdx.x % C, lanes = blockDim.x / C;
    float s = 0.0f;
    for (long long v = (long long)blockIdx.x * lanes + threadIdx.x / C; v < V; v += (long long)gridDim.x * lanes)
        s += __bfloat162float(g[v * C + c]);
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x < C) {
        float t = 0.0f;
        for (int k = 0; k < lanes; k++) t += part[k * C + threadIdx.x];
        atomicAdd(&db[threadIdx.x], t);
    }
}

template <int CIN, int COUT>
static bool launch_wgrad_tc(const WgradArgs &a, int sms, cudaStream_t s, cudaError_t &err)
{
    using Cfg = WtcCfg<CIN, COUT>;
    if (a.c0 != 0 || a.W + 2 > 256) return false;
    PFN_cuTensorMapEncodeTiled enc = tensor_map_encoder();
    if (!enc) return false;
    if ((reinterpret_cast<uintptr_t>(a.src1) & 15) || (reinterpret_cast<uintptr_t>(a.g) & 15)) return false;
    WTGeom g{};
    g.Wp = a.W + 2;
    g.NR = 3 + (130 + g.Wp - 1) / g.Wp;
    g.NRg = 2 + (TILE_M + g.Wp - 1) / g.Wp;
    if (g.NR > 256 || g.NRg > 256) return false;
    g.T = (a.H * g.Wp + TILE_M - 1) / TILE_M;
    const long long nb = a.V / ((long long)a.D * a.H * a.W);
    g.ntiles = nb * a.D * g.T;
    g.boxX = 16u * (uint32_t)g.Wp * (uint32_t)g.NR;
    g.boxG = 16u * (uint32_t)g.Wp * (uint32_t)g.NRg;
    g.planeX = (g.boxX + 127u) & ~127u;
    g.planeG = (g.boxG + 127u) & ~127u;
    g.stage_bytes = (((CIN / 8) * g.planeX + (COUT / 8) * g.planeG) + 1023u) & ~1023u;
    // the padded M rows of the last stage read up to PAD_PLANES planes past its slab
    const uint32_t pad = (uint32_t)Cfg::PAD_PLANES * g.planeX;
    const uint32_t budget = 227u * 1024u - 2048u;
    int per_sm = std::min(4, (int)(512 / Cfg::TCOLS));
    g.S = 0;
    for (; per_sm >= 1; per_sm--) {
        const uint32_t share = std::min<uint32_t>(budget, (228u * 1024u) / (uint32_t)per_sm - 2048u);
        if (share <= pad) continue;
        const int S = (int)std::min<uint32_t>(4u, (share - pad) / g.stage_bytes);
        if (S >= 2) {
            g.S = S;
            break;
        }
    }
    if (g.S < 2 || g.ntiles == 0) return false;
    const uint32_t smem = (uint32_t)g.S * g.stage_bytes + pad;
    CUtensorMap maps[2];
    const void *bases[2] = {a.src1, a.g};
    const int chans[2] = {CIN, COUT};
    const int rows[2] = {g.NR, g.NRg};
    for (int m = 0; m < 2; m++) {
        const cuuint64_t C = (cuuint64_t)chans[m];
        const cuuint64_t dims[5] = {C, (cuuint64_t)a.W, (cuuint64_t)a.H, (cuuint64_t)a.D, (cuuint64_t)nb};
        const cuuint64_t strides[4] = {C * 2, (cuuint64_t)a.W * C * 2, (cuuint64_t)a.H * a.W * C * 2,
                                       (cuuint64_t)a.D * a.H * a.W * C * 2};
        const cuuint32_t box[5] = {8u, (cuuint32_t)g.Wp, (cuuint32_t)rows[m], 1u, 1u};
        const cuuint32_t estr[5] = {1u, 1u, 1u, 1u, 1u};
        if (enc(&maps[m], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void *>(bases[m]), dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    err = smem_attributes(wgrad_tc_kernel<CIN, COUT>, smem);
    if (err != cudaSuccess) return true;
    const int groups = 27 / Cfg::G;
    const long long per_group = std::max<long long>(
        1, std::min<long long>((g.ntiles + 1) / 2, ((long long)per_sm * std::max(1, sms) + groups - 1) / groups));
    ++launch_count;
    wgrad_tc_kernel<CIN, COUT><<<dim3((unsigned)per_group, groups), 32 * (5 + Cfg::NI), smem, s>>>(maps[0], maps[1], a, g);
    if ((err = cudaGetLastError()) != cudaSuccess) return true;
    if (a.db) {
        const int lanes = 256 / COUT;
        const long long blocks = std::min<long long>((a.V + lanes - 1) / lanes, 4LL * std::max(1, sms));
        ++launch_count;
        bias_grad_kernel<<<(unsigned)blocks, lanes * COUT, lanes * COUT * sizeof(float), s>>>(a.g, COUT, a.V, a.db);
        err = cudaGetLastError();
    }
    return true;
}

// the dz-stacked tcgen05 weight gradient (wgrad_zs_kernel); false when the
// layer's shape has no configuration or a stage does not fit
template <int CIN, int COUT, int MODE>
static bool launch_wgrad_zs(const WgradArgs &a, int sms, cudaStream_t s, cudaError_t &err)
{
    using Z = WzsCfg<CIN, COUT, MODE>;
    if constexpr (!Z::OK) {
        return false;
    } else {
        if (a.c0 != 0 || a.W + 2 > 256) return false;
        PFN_cuTensorMapEncodeTiled enc = tensor_map_encoder();
        if (!enc) return false;
        if ((reinterpret_cast<uintptr_t>(a.src1) & 15) || (reinterpret_cast<uintptr_t>(a.g) & 15)) return false;
        WTGeom g{};
        g.Wp = a.W + 2;
        const long long nb = a.V / ((long long)a.D * a.H * a.W);
        const uint32_t budget = 227u * 1024u - 2048u;
        // positions per tile: 256 (fewer halo rows staged per position) where two stages fit
        // and the tiles still outnumber the CTAs twice, else 128; IAC_DENOISE_WGRAD_KT forces one
        static const int kt_env = [] {
            const char *e = getenv("IAC_DENOISE_WGRAD_KT");
            return e ? atoi(e) : 0;
        }();
        int per_sm = 0;
        for (int KT : {256, 128}) {
            if (kt_env && KT != kt_env) continue;
            g.KT = KT;
            g.NR = 3 + (KT + 2 + g.Wp - 1) / g.Wp;
            g.NRg = 2 + (KT + g.Wp - 1) / g.Wp;
            if (g.NR > 256 || g.NRg > 256) continue;
            g.T = (a.H * g.Wp + KT - 1) / KT;
            g.ntiles = nb * ((a.D + Z::ZSTEP - 1) / Z::ZSTEP) * g.T;
            g.boxX = 2u * Z::XW * (uint32_t)g.Wp * (uint32_t)g.NR;  // planes of XW channels, 2 XW-byte rows
            g.boxG = 2u * Z::GW * (uint32_t)g.Wp * (uint32_t)g.NRg;
            // planes aligned to their swizzle pattern (8 rows)
            g.planeX = (g.boxX + 16u * Z::XW - 1u) & ~(16u * Z::XW - 1u);
            g.planeG = (g.boxG + 16u * Z::GW - 1u) & ~(16u * Z::GW - 1u);
            g.stage_bytes = (((uint32_t)Z::XPLANES * g.planeX + (uint32_t)Z::GPLANES * g.planeG) + 1023u) & ~1023u;
            g.S = 0;
            const int min_stages = 2;
            for (per_sm = std::min(2, (int)(512 / Z::TCOLS)); per_sm >= 1; per_sm--) {
                const uint32_t share = std::min<uint32_t>(budget, (228u * 1024u) / (uint32_t)per_sm - 2048u);
                const int S = (int)std::min<uint32_t>(6u, share / g.stage_bytes);
                if (S >= min_stages) {
                    g.S = S;
                    break;
                }
            }
            if (g.S >= min_stages && g.ntiles >= 2LL * per_sm * std::max(1, sms)) break;
            g.S = 0;
        }
        if (g.S < 2 || g.ntiles == 0) return false;
        const uint32_t smem = (uint32_t)g.S * g.stage_bytes;
        CUtensorMap maps[2];
        const void *bases[2] = {a.src1, a.g};
        const int chans[2] = {CIN, COUT};
        const int rows[2] = {g.NR, g.NRg};
        for (int m = 0; m < 2; m++) {
            const cuuint64_t C = (cuuint64_t)chans[m];
            const cuuint64_t dims[5] = {C, (cuuint64_t)a.W, (cuuint64_t)a.H, (cuuint64_t)a.D, (cuuint64_t)nb};
            const cuuint64_t strides[4] = {C * 2, (cuuint64_t)a.W * C * 2, (cuuint64_t)a.H * a.W * C * 2,
                                           (cuuint64_t)a.D * a.H * a.W * C * 2};
            const cuuint32_t w = m == 0 ? Z::XW : Z::GW;
            const cuuint32_t box[5] = {w, (cuuint32_t)g.Wp, (cuuint32_t)rows[m], 1u, 1u};
            const cuuint32_t estr[5] = {1u, 1u, 1u, 1u, 1u};
            if (enc(&maps[m], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void *>(bases[m]), dims, strides, box,
                    estr, CU_TENSOR_MAP_INTERLEAVE_NONE, w == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
                return false;
        }
        err = smem_attributes(wgrad_zs_kernel<CIN, COUT, MODE>, smem);
        if (err != cudaSuccess) return true;
        // with tap groups every group stages the tiles again: fewer CTAs per group
        const long long grid =
            std::min<long long>(g.ntiles, ((long long)per_sm * std::max(1, sms) + Z::NTG - 1) / Z::NTG);
        ++launch_count;
        wgrad_zs_kernel<CIN, COUT, MODE><<<dim3((unsigned)grid, Z::NTG), 32 * (5 + Z::TPG), smem, s>>>(maps[0], maps[1],
                                                                                                   a, g);
        err = cudaGetLastError();  // the kernel also adds the bias gradient (its ones row)
        return true;
    }
}

// the stage layout of wgrad_zs_kernel per layer: three output planes per stage
// (MODE 2) for 16 -> 16, where one plane's MMAs are 64 x 16 and the issue rate
// bounds the kernel; else the dz axis on the operand whose three planes give
// the fewer MMA rows x columns (X along M for 16 or 32 input channels, the
// gradient along N for 48 -> 16 and 96 -> 32)
template <int CIN, int COUT>
struct WzsPick {
    static constexpr int MODE = (CIN == 16 && COUT == 16)
                                    ? 2
                                    : (((CIN == 48 && COUT == 16) || (CIN == 96 && COUT == 32)) ? 1 : 0);
};

cudaError_t wgrad3x3(const WgradArgs &a, int cin, int sms, cudaStream_t s)
{
#define IAC_WG_CASE(CI, CO)                                               \
    if (cin == CI && a.cout == CO) {                                      \
        cudaError_t e = cudaSuccess;                                      \
        if (a.slabs == 3 && launch_wgrad_zs<CI, CO, WzsPick<CI, CO>::MODE>(a, sms, s, e)) return e; \
        if (a.slabs >= 2 && launch_wgrad_tc<CI, CO>(a, sms, s, e)) return e; \
        if (a.slabs >= 1 && launch_wgrad_slab<CI, CO>(a, sms, s, e)) return e; \
        return launch_wgrad<CI, CO>(a, sms, s);                           \
    }
    IAC_WG_CASE(16, 16)
    IAC_WG_CASE(16, 32)
    IAC_WG_CASE(32, 32)
    IAC_WG_CASE(32, 64)
    IAC_WG_CASE(64, 64)
    IAC_WG_CASE(96, 32)
    IAC_WG_CASE(48, 16)
#undef IAC_WG_CASE
    return cudaErrorInvalidValue;
}

// first layer: dW[co][tap] = sum_v G[v][co] x[v+off(tap)] and db[co] = sum_v G[v][co]
// on mma.sync, warp by warp: a warp takes 128 voxels at a time, a lane four
// consecutive voxels of a row (it loads the six input values per (dz, dy) that
// the four need, as conv_first_kernel).  The lane writes the 27 shifted inputs
// of its voxels, a one for the bias and four zeros as bf16 rows of 32 columns
// into the warp's own shared-memory operand [column chunk][voxel][8], the
// gradient rows as [co chunk][voxel][8] (voxel 4 lane + i in row 32 i + lane:
// the sum over voxels does not depend on their order, and consecutive lanes
// write consecutive rows, free of bank conflicts); M = 16 output channels,
// N = 32 columns, K = 128 voxels.  Only warp barriers inside the loop.
constexpr int WGF_WARPS = 8;
constexpr int WGF_ROWS = 128;  // voxels per warp and iteration
constexpr int WGF_WARP_BYTES = (4 + 2) * WGF_ROWS * 16;
template <bool VEC>  // VEC: x is 16-byte aligned
__global__ void __launch_bounds__(32 * WGF_WARPS, 2) wgrad_first_kernel(const float *__restrict__ x,
                                                                        const bf16 *__restrict__ g,
                                                                        float *__restrict__ dw,
                                                                        float *__restrict__ db, int D, int H,
                                                                        int W, long long V)
{
    extern __shared__ __align__(128) unsigned char wgf_smem[];
    __shared__ float red[16][32];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < 16 * 32; i += blockDim.x) (&red[0][0])[i] = 0.0f;
    float acc[4][4];
#pragma unroll
    for (int n = 0; n < 4; n++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[n][j] = 0.0f;
    unsigned char *mine = wgf_smem + warp * WGF_WARP_BYTES;
    uint4 *xs = reinterpret_cast<uint4 *>(mine);                       // [4][128] rows of 8 bf16
    uint4 *gs = reinterpret_cast<uint4 *>(mine + 4 * WGF_ROWS * 16);   // [2][128]
    const uint32_t sx = smem_u32(xs), sg = smem_u32(gs);
    const long long HW = (long long)H * W;
    const long long ngroups = (V + WGF_ROWS - 1) / WGF_ROWS;
    const long long stride = (long long)gridDim.x * WGF_WARPS;
    for (long long grp = (long long)blockIdx.x * WGF_WARPS + warp; grp < ngroups; grp += stride) {
        const long long v0 = grp * WGF_ROWS + 4 * lane;
        const Vox q = decode(v0, D, H, W, V);
        float r[9][6];
        const bool left = q.x > 0, right = q.x + 4 < W;
#pragma unroll
        for (int dz = 0; dz < 3; dz++) {
            const bool zin = q.ok && (unsigned)(q.z + dz - 1) < (unsigned)D;
#pragma unroll
            for (int dy = 0; dy < 3; dy++) {
                const bool in = zin && (unsigned)(q.y + dy - 1) < (unsigned)H;
                const float *row = x + (q.ok ? v0 : 0) + (dz - 1) * HW + (long long)(dy - 1) * W;
                float *rr = r[3 * dz + dy];
                const float4 mid = !in ? make_float4(0.0f, 0.0f, 0.0f, 0.0f)
                                       : (VEC ? *reinterpret_cast<const float4 *>(row)
                                              : make_float4(row[0], row[1], row[2], row[3]));
                rr[0] = in && left ? row[-1] : 0.0f;
                rr[1] = mid.x;
                rr[2] = mid.y;
                rr[3] = mid.z;
                rr[4] = mid.w;
                rr[5] = in && right ? row[4] : 0.0f;
            }
        }
        uint4 gv[4][2];
        const uint4 z4 = make_uint4(0, 0, 0, 0);
        const uint4 *gp = reinterpret_cast<const uint4 *>(g + (q.ok ? v0 : 0) * 16);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            gv[i][0] = q.ok ? gp[2 * i] : z4;
            gv[i][1] = q.ok ? gp[2 * i + 1] : z4;
        }
        __syncwarp();  // the previous iteration's fragments are read
#pragma unroll
        for (int i = 0; i < 4; i++) {
            float col[32];
#pragma unroll
            for (int t = 0; t < 27; t++) col[t] = r[t / 3][i + t % 3];
            col[27] = q.ok ? 1.0f : 0.0f;
#pragma unroll
            for (int t = 28; t < 32; t++) col[t] = 0.0f;
            const int row = 32 * i + lane;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                uint4 u;
                u.x = pack_bf16(col[8 * c], col[8 * c + 1]);
                u.y = pack_bf16(col[8 * c + 2], col[8 * c + 3]);
                u.z = pack_bf16(col[8 * c + 4], col[8 * c + 5]);
                u.w = pack_bf16(col[8 * c + 6], col[8 * c + 7]);
                xs[c * WGF_ROWS + row] = u;
            }
            gs[row] = gv[i][0];
            gs[WGF_ROWS + row] = gv[i][1];
        }
        __syncwarp();
#pragma unroll
        for (int ks = 0; ks < WGF_ROWS / 16; ks++) {
            const int kb = ks * 16;
            uint32_t a0, a1, a2, a3;
            {
                const int vr = kb + (lane & 7) + ((lane >> 4) << 3);
                const int ch = (lane >> 3) & 1;
                ldsm_x4_t(sg + (uint32_t)((ch * WGF_ROWS + vr) * 16), a0, a1, a2, a3);
            }
#pragma unroll
            for (int n2 = 0; n2 < 2; n2++) {
                uint32_t b0, b1, b2, b3;
                const int vx = kb + (lane & 7) + (((lane >> 3) & 1) << 3);
                const int cx = 2 * n2 + (lane >> 4);
                ldsm_x4_t(sx + (uint32_t)((cx * WGF_ROWS + vx) * 16), b0, b1, b2, b3);
                mma_bf16(acc[2 * n2], a0, a1, a2, a3, b0, b1);
                mma_bf16(acc[2 * n2 + 1], a0, a1, a2, a3, b2, b3);
            }
        }
    }
    __syncthreads();  // red is zeroed
    const int gq = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int n = 0; n < 4; n++)
#pragma unroll
        for (int j = 0; j < 4; j++) atomicAdd(&red[gq + 8 * (j >> 1)][n * 8 + 2 * tq + (j & 1)], acc[n][j]);
    __syncthreads();
    for (int i = tid; i < 16 * 28; i += blockDim.x) {
        const int co = i / 28, t = i % 28;
        const float rv = red[co][t];
        if (rv == 0.0f) continue;
        if (t < 27)
            atomicAdd(&dw[co * 27 + t], rv);
        else
            atomicAdd(&db[co], rv);
    }
}

cudaError_t wgrad3x3_first(const float *x, const bf16 *g, float *dw, float *db, int D, int H, int W, long long V,
                           int sms, cudaStream_t s)
{
    if (W % 4) return cudaErrorInvalidValue;
    const int smem = WGF_WARPS * WGF_WARP_BYTES;
    const bool vec = (reinterpret_cast<uintptr_t>(x) & 15) == 0;
    auto k = vec ? wgrad_first_kernel<true> : wgrad_first_kernel<false>;
    const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const long long ngroups = (V + WGF_ROWS - 1) / WGF_ROWS;
    const long long blocks = (ngroups + WGF_WARPS - 1) / WGF_WARPS;
    const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(blocks, 2LL * sms));
    ++launch_count;
    k<<<grid, 32 * WGF_WARPS, smem, s>>>(x, g, dw, db, D, H, W, V);
    return cudaGetLastError();
}

// --------------------------------------------------------------------------
// pooling, masks and the decoder's concat/upsample gradient
// --------------------------------------------------------------------------
__device__ __forceinline__ void load8(const bf16 *p, float *f)
{
    const uint4 u = *reinterpret_cast<const uint4 *>(p);
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const float2 t = __bfloat1622float2(h[j]);
        f[2 * j] = t.x;
        f[2 * j + 1] = t.y;
    }
}
__device__ __forceinline__ void store8b(bf16 *p, const float *f)
{
    uint4 u;
    u.x = pack_bf16(f[0], f[1]);
    u.y = pack_bf16(f[2], f[3]);
    u.z = pack_bf16(f[4], f[5]);
    u.w = pack_bf16(f[6], f[7]);
    *reinterpret_cast<uint4 *>(p) = u;
}

// y (D/2 x H/2 x W/2) = mean of the 2x2x2 children; thread = (coarse voxel, 8 channels)
__global__ void avgpool2_kernel(const bf16 *__restrict__ x, int x_stride, bf16 *__restrict__ y, int C, int D,
                                int H, int W, long long total)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int nc = C / 8, c = (int)(i % nc) * 8;
    const long long u = i / nc;
    const int D2 = D / 2, H2 = H / 2, W2 = W / 2;
    const Vox q = decode(u, D2, H2, W2, total / nc);
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < 8; k++) {
        const long long v = (((long long)q.n * D + 2 * q.z + (k >> 2)) * H + 2 * q.y + ((k >> 1) & 1)) * W + 2 * q.x + (k & 1);
        float f[8];
        load8(x + v * x_stride + c, f);
#pragma unroll
        for (int j = 0; j < 8; j++) s[j] += f[j];
    }
#pragma unroll
    for (int j = 0; j < 8; j++) s[j] *= 0.125f;
    store8b(y + u * C + c, s);
}

cudaError_t avgpool2(const bf16 *x, int x_stride, bf16 *y, int C, int D, int H, int W, int nb, cudaStream_t s)
{
    const long long total = (long long)nb * (D / 2) * (H / 2) * (W / 2) * (C / 8);
    ++launch_count;
    avgpool2_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(x, x_stride, y, C, D, H, W, total);
    return cudaGetLastError();
}

__global__ void relu_mask_kernel(const bf16 *__restrict__ g, const bf16 *__restrict__ y, bf16 *__restrict__ out,
                                 long long n8)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n8) return;
    float fg[8], fy[8];
    load8(g + i * 8, fg);
    load8(y + i * 8, fy);
#pragma unroll
    for (int j = 0; j < 8; j++) fg[j] = fy[j] > 0.0f ? fg[j] : 0.0f;
    store8b(out + i * 8, fg);
}

cudaError_t relu_mask(const bf16 *g, const bf16 *y, bf16 *out, long long n, cudaStream_t s)
{
    const long long n8 = n / 8;
    ++launch_count;
    relu_mask_kernel<<<(unsigned)((n8 + 255) / 256), 256, 0, s>>>(g, y, out, n8);
    return cudaGetLastError();
}

// gup [V][c0] at full resolution, the gradient of a decoder input's upsampled
// part: g0 (coarse, c0) = mask(y0) * sum of the 8 children (backward of
// nearest upsampling); the skip part's gradient went to its own buffer
__global__ void split_concat_kernel(const bf16 *__restrict__ gup, int c0, const bf16 *__restrict__ y0,
                                    bf16 *__restrict__ g0, int D, int H, int W, long long n_coarse)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_coarse) return;
    const int nc = c0 / 8, c = (int)(i % nc) * 8;
    const long long u = i / nc;
    const Vox q = decode(u, D / 2, H / 2, W / 2, n_coarse / nc);
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < 8; k++) {
        const long long v =
            (((long long)q.n * D + 2 * q.z + (k >> 2)) * H + 2 * q.y + ((k >> 1) & 1)) * W + 2 * q.x + (k & 1);
        float f[8];
        load8(gup + v * c0 + c, f);
#pragma unroll
        for (int j = 0; j < 8; j++) s[j] += f[j];
    }
    float fy[8];
    load8(y0 + u * c0 + c, fy);
#pragma unroll
    for (int j = 0; j < 8; j++) s[j] = fy[j] > 0.0f ? s[j] : 0.0f;
    store8b(g0 + u * c0 + c, s);
}

cudaError_t split_concat_grad(const bf16 *gup, int c0, const bf16 *y0, bf16 *g0, int D, int H, int W, int nb,
                              cudaStream_t s)
{
    const long long V = (long long)nb * D * H * W;
    const long long nco = V / 8 * (c0 / 8);
    ++launch_count;
    split_concat_kernel<<<(unsigned)((nco + 255) / 256), 256, 0, s>>>(gup, c0, y0, g0, D, H, W, nco);
    return cudaGetLastError();
}

// cat[v] = src0[parent(v)] ++ src1[v]: a decoder input, the coarse part
// nearest-upsampled (2x), the skip tensor after it.  The first n_coarse
// threads take (coarse voxel, 8 channels): one load, the 8 children stored;
// the rest copy the skip tensor 16 bytes each.  D, H, W: the full resolution.
__global__ void concat_up_kernel(const bf16 *__restrict__ src0, int c0, const bf16 *__restrict__ src1, int c1,
                                 bf16 *__restrict__ cat, int D, int H, int W, long long n_coarse, long long n_skip)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int C = c0 + c1;
    if (i < n_coarse) {
        const int nc = c0 / 8, c = (int)(i % nc) * 8;
        const long long u = i / nc;
        const Vox q = decode(u, D / 2, H / 2, W / 2, n_coarse / nc);
        const uint4 val = *reinterpret_cast<const uint4 *>(src0 + u * c0 + c);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const long long v =
                (((long long)q.n * D + 2 * q.z + (k >> 2)) * H + 2 * q.y + ((k >> 1) & 1)) * W + 2 * q.x + (k & 1);
            *reinterpret_cast<uint4 *>(cat + v * C + c) = val;
        }
    } else if (i < n_coarse + n_skip) {
        const long long k = i - n_coarse;
        const int nc = c1 / 8, c = (int)(k % nc) * 8;
        const long long v = k / nc;
        *reinterpret_cast<uint4 *>(cat + v * C + c0 + c) = *reinterpret_cast<const uint4 *>(src1 + v * c1 + c);
    }
}

cudaError_t concat_up(const bf16 *src0, int c0, const bf16 *src1, int c1, bf16 *cat, int D, int H, int W, int nb,
                      cudaStream_t s)
{
    const long long V = (long long)nb * D * H * W;
    const long long nco = V / 8 * (c0 / 8), nsk = V * (c1 / 8);
    ++launch_count;
    concat_up_kernel<<<(unsigned)((nco + nsk + 255) / 256), 256, 0, s>>>(src0, c0, src1, c1, cat, D, H, W, nco, nsk);
    return cudaGetLastError();
}

// out = (gskip + gpool(parent) / 8) * (y > 0): gradient of a skip tensor that
// also fed an average pool; gskip and y have gskip_stride and y_stride
// channels per voxel (the skip channels of the decoder input's gradient and
// of the decoder input, read in place)
__global__ void pool_grad_mask_kernel(const bf16 *__restrict__ gskip, int gskip_stride,
                                      const bf16 *__restrict__ gpool, const bf16 *__restrict__ y, int y_stride,
                                      bf16 *__restrict__ out, int C, int D, int H, int W, long long total)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int nc = C / 8, c = (int)(i % nc) * 8;
    const long long v = i / nc;
    const Vox q = decode(v, D, H, W, total / nc);
    const long long u = (((long long)q.n * (D / 2) + q.z / 2) * (H / 2) + q.y / 2) * (W / 2) + q.x / 2;
    float a[8], b[8], fy[8];
    load8(gskip + v * gskip_stride + c, a);
    load8(gpool + u * C + c, b);
    load8(y + v * y_stride + c, fy);
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] = fy[j] > 0.0f ? a[j] + 0.125f * b[j] : 0.0f;
    store8b(out + v * C + c, a);
}

cudaError_t pool_grad_mask(const bf16 *gskip, int gskip_stride, const bf16 *gpool, const bf16 *y, int y_stride,
                           bf16 *out, int C, int D, int H, int W, int nb, cudaStream_t s)
{
    const long long total = (long long)nb * D * H * W * (C / 8);
    ++launch_count;
    pool_grad_mask_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(gskip, gskip_stride, gpool, y, y_stride,
                                                                          out, C, D, H, W, total);
    return cudaGetLastError();
}

// --------------------------------------------------------------------------
// residual 1x1 head with the MSE loss and its gradient
// --------------------------------------------------------------------------
__global__ void __launch_bounds__(256) head_kernel(const HeadArgs a)
{
    __shared__ float red[8][18];
    const float bias = a.w[16];
    float w[16];
#pragma unroll
    for (int c = 0; c < 16; c++) w[c] = a.w[c];
    float pw[17];
#pragma unroll
    for (int c = 0; c < 17; c++) pw[c] = 0.0f;
    float ploss = 0.0f;
    const bool train = a.target != nullptr;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < a.V; v += (long long)gridDim.x * blockDim.x) {
        float d[16];
        load8(a.d + v * 16, d);
        load8(a.d + v * 16 + 8, d + 8);
        float o = bias;
#pragma unroll
        for (int c = 0; c < 16; c++) o = fmaf(w[c], d[c], o);
        o += a.x[v];
        if (a.out) a.out[v] = o;
        if (train) {
            const float wt = a.weight ? a.weight[v] : 1.0f;
            const float diff = o - a.target[v];
            ploss = fmaf(wt * diff, diff, ploss);
            const float go = (float)(2.0 * a.inv_count) * wt * diff;
            float gd[16];
#pragma unroll
            for (int c = 0; c < 16; c++) {
                gd[c] = d[c] > 0.0f ? go * w[c] : 0.0f;
                pw[c] = fmaf(go, d[c], pw[c]);
            }
            pw[16] += go;
            store8b(a.gd + v * 16, gd);
            store8b(a.gd + v * 16 + 8, gd + 8);
        }
    }
    if (!train) return;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 17; c++) {
        float t = pw[c];
        for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) red[wp][c] = t;
    }
    for (int o = 16; o; o >>= 1) ploss += __shfl_xor_sync(0xffffffffu, ploss, o);
    if (lane == 0) red[wp][17] = ploss;
    __syncthreads();
    if (threadIdx.x < 18) {
        float t = 0.0f;
        for (int k = 0; k < (int)(blockDim.x / 32); k++) t += red[k][threadIdx.x];
        if (threadIdx.x < 17)
            atomicAdd(&a.dw[threadIdx.x], t);
        else
            atomicAdd(a.loss + (a.d_step ? a.d_step[0] : 0), (double)t);
    }
}

cudaError_t head(const HeadArgs &a, int sms, cudaStream_t s)
{
    const long long blocks = (a.V + 255) / 256;
    ++launch_count;
    head_kernel<<<(unsigned)std::max<long long>(1, std::min<long long>(blocks, 8LL * sms)), 256, 0, s>>>(a);
    return cudaGetLastError();
}

// --------------------------------------------------------------------------
// AdamW on the fp32 master weights, then the bf16 B tiles
// --------------------------------------------------------------------------
__global__ void adamw_kernel(const AdamArgs a)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    int l = 0;
    while (l + 1 < a.nlayers && i >= a.layers[l + 1].off) l++;
    const AdamLayer L = a.layers[l];
    const long long j = i - L.off;
    const long long nw = L.taps ? (long long)L.cout * L.taps * L.cin : 16;
    const bool is_w = j < nw;
    float p = a.p[i];
    if (a.update) {
        float lr = a.lr, bc1 = a.bc1, bc2 = a.bc2;
        if (a.d_step) {  // graph replay: step index and schedule from device memory
            const float t = (float)(a.d_step[1] + 1);
            lr = a.lrs[a.d_step[0]];
            bc1 = 1.0f - powf(a.beta1, t);
            bc2 = 1.0f - powf(a.beta2, t);
        }
        const float g = a.g[i];
        const float m = a.beta1 * a.m[i] + (1.0f - a.beta1) * g;
        const float v = a.beta2 * a.v[i] + (1.0f - a.beta2) * g * g;
        a.m[i] = m;
        a.v[i] = v;
        const float step = (m / bc1) / (sqrtf(v / bc2) + a.eps);
        p -= lr * (step + (is_w ? a.weight_decay * p : 0.0f));
        a.p[i] = p;
    }
    if (!L.taps || !is_w) return;
    const int co = (int)(j / (L.taps * L.cin));
    const int rem = (int)(j % (L.taps * L.cin));
    const int tap = rem / L.cin, ci = rem % L.cin;
    const bf16 h = __float2bfloat16_rn(p);
    if (L.cin == 1) {
        a.wf[L.wf_off + tap * L.cout + co] = h;
        return;
    }
    a.wf[L.wf_off + (((long long)tap * (L.cin / 8) + ci / 8) * L.cout + co) * 8 + ci % 8] = h;
    a.wd[L.wd_off + (((long long)(26 - tap) * (L.cout / 8) + co / 8) * L.cin + ci) * 8 + co % 8] = h;
}

cudaError_t adamw(const AdamArgs &a, cudaStream_t s)
{
    ++launch_count;
    adamw_kernel<<<(unsigned)((a.n + 255) / 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}

// --------------------------------------------------------------------------
// training patches: plan[b] = {mesh, z0, y0, x0, transform}; out[b] = P^3 crop
// of mesh (E^3, bf16) under one of the 48 axis permutations x reflections
// --------------------------------------------------------------------------
__global__ void crop_kernel(const bf16 *__restrict__ meshes, int nmesh, int E, const int *__restrict__ plan, int P,
                            float *__restrict__ out, long long total, DeviceCounters *counters,
                            const long long *__restrict__ d_step, int nb)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const long long per = (long long)P * P * P;
    const int b = (int)(i / per);
    const long long r = i % per;
    int c[3] = {(int)(r / ((long long)P * P)), (int)((r / P) % P), (int)(r % P)};
    const int *pl = plan + 5 * ((d_step ? d_step[0] * nb : 0) + b);
    if ((unsigned)pl[4] >= 48u || (unsigned)pl[0] >= (unsigned)nmesh) {
        out[i] = 0.0f;  // a plan entry outside the meshes: counted, not read
        if (counters) atomicAdd(&counters->out_of_mesh, 1ull);
        return;
    }
    const int perm = pl[4] % 6, flip = pl[4] / 6;
    const int pa = perm / 2, pb = (perm / 2 + 1 + (perm & 1)) % 3, pc = 3 - pa - pb;
    const int src_axis[3] = {pa, pb, pc};
    int s[3];
    for (int k = 0; k < 3; k++) {
        int t = c[src_axis[k]];
        if (flip & (1 << k)) t = P - 1 - t;
        s[k] = t + pl[1 + k];
    }
    if ((unsigned)s[0] >= (unsigned)E || (unsigned)s[1] >= (unsigned)E || (unsigned)s[2] >= (unsigned)E) {
        out[i] = 0.0f;  // a plan entry outside the meshes: counted, not read
        if (counters) atomicAdd(&counters->out_of_mesh, 1ull);
        return;
    }
    out[i] = __bfloat162float(meshes[(size_t)pl[0] * E * E * E + ((size_t)s[0] * E + s[1]) * E + s[2]]);
}

cudaError_t crop_patches(const bf16 *meshes, int nmesh, int E, const int *plan, int nb, int P, float *out,
                         DeviceCounters *counters, cudaStream_t s, const long long *d_step)
{
    const long long total = (long long)nb * P * P * P;
    ++launch_count;
    crop_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(meshes, nmesh, E, plan, P, out, total, counters,
                                                                d_step, nb);
    return cudaGetLastError();
}

// graph replay bookkeeping: d_step[0] = replay index, d_step[1] = optimizer steps
__global__ void step_kernel(long long *d_step, long long set_opt, int mode)
{
    if (mode == 0) {
        d_step[0] = 0;
        d_step[1] = set_opt;
    } else {
        d_step[0] += 1;
        d_step[1] += 1;
    }
}

cudaError_t step_counter(long long *d_step, long long set_opt, int advance, cudaStream_t s)
{
    ++launch_count;
    step_kernel<<<1, 1, 0, s>>>(d_step, set_opt, advance);
    return cudaGetLastError();
}

// network input from a pair mesh: the leading E^3 corner of the S^3 uint64
// mesh times `scale` (1 / (Multiplicator x frames x normaliser)), as fp32
// and/or bf16
__global__ void mesh_input_kernel(const unsigned long long *__restrict__ full, int S, int E, double scale,
                                  float *__restrict__ o32, bf16 *__restrict__ o16, long long total)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int x = (int)(i % E), y = (int)((i / E) % E), z = (int)(i / ((long long)E * E));
    const float f = (float)((double)full[((size_t)z * S + y) * S + x] * scale);
    if (o32) o32[i] = f;
    if (o16) o16[i] = __float2bfloat16_rn(f);
}

cudaError_t mesh_input(const uint64_t *full, int S, int E, double scale, float *o32, bf16 *o16, cudaStream_t s)
{
    const long long total = (long long)E * E * E;
    ++launch_count;
    mesh_input_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(
        reinterpret_cast<const unsigned long long *>(full), S, E, scale, o32, o16, total);
    return cudaGetLastError();
}

}  // namespace dn
}  // namespace iac
