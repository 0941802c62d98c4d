// cq_merge.cu -- (b') rotate-and-weight merge of the small C(q) mesh into
// the big cubic mesh.
//
// Replaces Merge_CQ (IAC/kernel.cl:189-344) and the device part of
// Detector::Merge_smallCofQ (IAC/Detector.cpp:1321-1573).  For every small-mesh
// voxel with C >= 1e-37 and every frame f, the voxel's q (in voxels) is rotated
// by the frame's RotMatrix and (uint64)(C * w_f * Mult) is added at the
// nearest voxel (or split over 8 corners) of the cubic mesh.
//
// The non-zero voxels are first compacted in mesh order (ordered per block), so
// that consecutive threads hold neighbouring voxels and, for one frame,
// scatter to neighbouring targets of the rotated lattice.  Each CTA stages a
// chunk of frames' rotation+weight rows in shared memory and walks them for
// its voxels.  One 64-bit L2 atomic per (voxel, frame): the merge is bound by
// the atomic rate, with no reuse to exploit (each frame's rotation sends a
// voxel block somewhere else).
//
// Reference quirks kept: the slow index uses the A/B centre (:287, :306) and
// the NN value is (C * w) * Mult while the linear one is (C * Mult) * w * corner.
#include <algorithm>

#include "iac_internal.cuh"

namespace iac {

constexpr int MERGE_THREADS = 256;
constexpr int MERGE_FRAMES = 128;  // frames per shared-memory chunk

struct MergeArgs {
    const double *__restrict__ small;
    const float *__restrict__ rw;  // 10 floats per frame
    const uint32_t *__restrict__ list;  // compacted voxel indices
    const uint32_t *__restrict__ count;
    unsigned long long *__restrict__ big;
    DeviceCounters *counters;
    uint32_t nframes;
    int ab, sc, cab, cc;
    int ka, kb, kc;
    double mult;
};

__global__ void merge_compact_kernel(const double *__restrict__ small, uint32_t n,
                                     uint32_t *__restrict__ list, uint32_t *__restrict__ count)
{
    __shared__ uint32_t s_warp[MERGE_THREADS / 32];
    __shared__ uint32_t s_base;
    const uint32_t i = blockIdx.x * MERGE_THREADS + threadIdx.x;
    const bool keep = i < n && !(small[i] < 1e-37f);  // IAC/kernel.cl:260
    const unsigned ball = __ballot_sync(0xffffffffu, keep);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) s_warp[w] = __popc(ball);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int k = 0; k < MERGE_THREADS / 32; k++) {
            const uint32_t c = s_warp[k];
            s_warp[k] = t;
            t += c;
        }
        s_base = t ? atomicAdd(count, t) : 0;
    }
    __syncthreads();
    if (keep) list[s_base + s_warp[w] + __popc(ball & ((1u << lane) - 1))] = i;
}

__device__ __forceinline__ void big_put(const MergeArgs &a, int fs, int ms, int ss,
                                        unsigned long long v)
{
    if (v == 0) return;
    if ((unsigned)fs >= (unsigned)a.ab || (unsigned)ms >= (unsigned)a.ab ||
        (unsigned)ss >= (unsigned)a.ab) {
        atomicAdd(&a.counters->out_of_mesh, 1ull);
        return;
    }
    atomicAdd(&a.big[(uint64_t)fs + (uint64_t)ms * a.ab + (uint64_t)ss * a.ab * a.ab], v);
}

template <int INTERP>
__global__ void __launch_bounds__(MERGE_THREADS) merge_kernel(const MergeArgs a)
{
    __shared__ float s_rw[MERGE_FRAMES * 10];
    const uint32_t nvox = *a.count;
    const float cabf = (float)a.cab;
    const uint32_t f0 = blockIdx.y * MERGE_FRAMES;
    const uint32_t nf = min((uint32_t)MERGE_FRAMES, a.nframes - f0);
    for (uint32_t k = threadIdx.x; k < nf * 10; k += MERGE_THREADS) s_rw[k] = a.rw[(size_t)f0 * 10 + k];
    __syncthreads();
    const uint32_t AB2 = (uint32_t)a.ab * a.ab;
    for (uint32_t t = blockIdx.x * MERGE_THREADS + threadIdx.x; t < nvox; t += gridDim.x * MERGE_THREADS) {
        const uint32_t ind = a.list[t];
        const int ss_in = (int)(ind / AB2);
        const int ms_in = (int)((ind - ss_in * AB2) / (uint32_t)a.ab);
        const int fs_in = (int)(ind - ss_in * AB2 - ms_in * (uint32_t)a.ab);
        float qi[3];
        qi[a.ka] = (float)(fs_in - a.cab);
        qi[a.kb] = (float)(ms_in - a.cab);
        qi[a.kc] = (float)(ss_in - a.cc);
        const double vin = a.small[ind];
        for (uint32_t f = 0; f < nf; f++) {
            const float *r = &s_rw[10 * f];
            const float o0 = rot_row(qi[0], qi[1], qi[2], r[0], r[1], r[2]);
            const float o1 = rot_row(qi[0], qi[1], qi[2], r[3], r[4], r[5]);
            const float o2 = rot_row(qi[0], qi[1], qi[2], r[6], r[7], r[8]);
            const double w = (double)r[9];
            if (INTERP == 0) {
                const unsigned long long v = d2u64(dmul(dmul(vin, w), a.mult));
                big_put(a, (int)fadd(round_away_f(o0), cabf), (int)fadd(round_away_f(o1), cabf),
                        (int)fadd(round_away_f(o2), cabf), v);
            } else {
                const float f0x = floorf(o0), f1x = floorf(o1), f2x = floorf(o2);
                const double sf = (double)fsub(1.0f, fsub(o0, f0x));
                const double sm = (double)fsub(1.0f, fsub(o1, f1x));
                const double sz = (double)fsub(1.0f, fsub(o2, f2x));
                const int fs = (int)fadd(f0x, cabf), ms = (int)fadd(f1x, cabf), ss = (int)fadd(f2x, cabf);
                const double base = dmul(dmul(vin, a.mult), w);
                const double xf[2] = {sf, dsub(1.0, sf)}, yf[2] = {sm, dsub(1.0, sm)},
                             zf[2] = {sz, dsub(1.0, sz)};
#pragma unroll
                for (int c = 0; c < 8; c++)
                    big_put(a, fs + (c >> 2), ms + ((c >> 1) & 1), ss + (c & 1),
                            d2u64(dmul(base, dmul(dmul(xf[c >> 2], yf[(c >> 1) & 1]), zf[c & 1]))));
            }
        }
    }
}

}  // namespace iac

using namespace iac;

extern "C" iac_status iac_cq_merge(iac_ctx *ctx, const double *d_small_cq, const float *d_rw10,
                                   uint32_t nframes, const iac_mesh_shape *sh, int interp,
                                   double mult, uint64_t *d_big, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx && d_small_cq && sh && d_big, "iac_cq_merge: NULL argument");
    IAC_REQUIRE(interp == 0 || interp == 1, "interpolation must be 0 or 1");
    IAC_REQUIRE(sh->size_ab >= 5 && sh->size_ab % 2 == 1 && sh->size_c % 2 == 1 &&
                    sh->size_c <= sh->size_ab && sh->size_ab <= 1625,
                "iac_cq_merge: bad small mesh %u x %u", sh->size_ab, sh->size_c);
    IAC_REQUIRE(sh->k_a < 3 && sh->k_b < 3 && sh->k_c < 3 &&
                    sh->k_a + sh->k_b + sh->k_c == 3 && sh->k_a != sh->k_b,
                "iac_cq_merge: axis alignment is not a permutation");
    IAC_REQUIRE(mult > 0, "multiplicator must be positive");
    if (nframes == 0) return IAC_OK;
    IAC_REQUIRE(d_rw10 != nullptr, "iac_cq_merge: NULL rotation/weight table");
    DeviceGuard g(ctx->device);
    const uint32_t n = sh->size_ab * sh->size_ab * sh->size_c;
    void *scr = nullptr;
    iac_status st = stream_scratch(ctx, stream, SLOT_AUX1, sizeof(uint32_t) * ((size_t)n + 64), &scr);
    if (st != IAC_OK) return st;
    uint32_t *count = (uint32_t *)scr;
    uint32_t *list = count + 32;
    cudaStream_t s = as_stream(stream);
    IAC_CUDA(cudaMemsetAsync(count, 0, sizeof(uint32_t), s));
    merge_compact_kernel<<<(n + MERGE_THREADS - 1) / MERGE_THREADS, MERGE_THREADS, 0, s>>>(d_small_cq, n,
                                                                                         list, count);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    MergeArgs a;
    a.small = d_small_cq;
    a.rw = d_rw10;
    a.list = list;
    a.count = count;
    a.big = (unsigned long long *)d_big;
    a.counters = ctx->d_counters;
    a.nframes = nframes;
    a.ab = (int)sh->size_ab;
    a.sc = (int)sh->size_c;
    a.cab = (a.ab - 1) / 2;
    a.cc = (a.sc - 1) / 2;
    a.ka = (int)sh->k_a;
    a.kb = (int)sh->k_b;
    a.kc = (int)sh->k_c;
    a.mult = mult;
    const uint32_t chunks = (nframes + MERGE_FRAMES - 1) / MERGE_FRAMES;
    // enough voxel blocks per frame chunk to fill the GPU several times over
    const uint32_t vblocks = std::max<uint32_t>(1, std::min<uint32_t>(
        (n + MERGE_THREADS - 1) / MERGE_THREADS, (uint32_t)(ctx->sm_count * 8 + chunks - 1) / chunks));
    dim3 grid(vblocks, chunks);
    if (interp == 0)
        merge_kernel<0><<<grid, MERGE_THREADS, 0, s>>>(a);
    else
        merge_kernel<1><<<grid, MERGE_THREADS, 0, s>>>(a);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}
