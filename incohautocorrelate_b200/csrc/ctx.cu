// ctx.cu -- context, error reporting, mesh geometry, k-map and the
// scatter-add micro-benchmark of libiac_b200.
#include <dlfcn.h>

#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "iac_internal.cuh"

namespace iac {

static thread_local char g_last_error[512] = "";

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof g_last_error, fmt, ap);
    va_end(ap);
}

iac_status Scratch::ensure(size_t need)
{
    if (need <= bytes) return IAC_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    size_t grow = need + need / 4 + 4096;
    IAC_CUDA(cudaMalloc(&ptr, grow));
    bytes = grow;
    return IAC_OK;
}

// The autotuner's table: tuning/sparse_tuning.tsv next to this library (or the
// file named by IAC_SPARSE_TUNING).  Rows: mesh_edge tile_pairs block_threads
// ctas_per_sm [...]; '#' starts a comment.
static void load_tuning_table(iac_ctx *c)
{
    std::string path;
    if (const char *env = std::getenv("IAC_SPARSE_TUNING")) {
        path = env;
    } else {
        Dl_info info;
        if (dladdr((void *)&load_tuning_table, &info) && info.dli_fname) {
            path = info.dli_fname;
            const size_t slash = path.find_last_of('/');
            path = (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) +
                   "/tuning/sparse_tuning.tsv";
        }
    }
    FILE *fh = path.empty() ? nullptr : std::fopen(path.c_str(), "r");
    if (!fh) return;
    char line[512];
    while (std::fgets(line, sizeof line, fh)) {
        if (line[0] == '#') continue;
        unsigned e, t, b, k, h = 2;
        char rest[256] = "";
        if (std::sscanf(line, "%u %u %u %u %255[^\n]", &e, &t, &b, &k, rest) >= 4 && t >= 64 && b >= 64 &&
            b <= 256 && b % 32 == 0 && k >= 1 && k <= 32) {
            // optional sixth column: cache_hints (the fifth is the measured rate)
            double rate;
            unsigned hh;
            if (std::sscanf(rest, "%lf %*u %u", &rate, &hh) == 2 && (hh == 1 || hh == 2)) h = hh;
            c->tuning_table.push_back({e, t, b, k, h});
        }
    }
    std::fclose(fh);
}

void Scratch::release()
{
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

}  // namespace iac

namespace {
// one thread waits for *flag != 0, at most max_polls polls of ~1 us; a wait that
// runs out is counted in the context's timeout counter (the error path of every
// bounded wait in the library)
__global__ void wait_flag_kernel(const volatile uint32_t *flag, uint32_t max_polls, iac::DeviceCounters *ctr)
{
    for (uint32_t i = 0; i < max_polls; i++) {
        if (*flag != 0u) return;
        __nanosleep(1000);
    }
    iac::note_timeout(ctr, iac::SITE_WAIT_TEST);
}
}  // namespace

using namespace iac;

extern "C" {

const char *iac_status_string(iac_status s)
{
    switch (s) {
    case IAC_OK: return "ok";
    case IAC_ERR_INVALID_ARG: return "invalid argument";
    case IAC_ERR_CUDA: return "CUDA error";
    case IAC_ERR_NO_MEMORY: return "out of memory";
    case IAC_ERR_TIMEOUT: return "device wait timed out";
    case IAC_ERR_OUT_OF_MESH: return "writes outside the mesh were skipped";
    case IAC_ERR_UNSUPPORTED: return "unsupported";
    }
    return "unknown status";
}

const char *iac_last_error(void) { return g_last_error; }

int iac_abi_version(void) { return IAC_ABI_VERSION; }

iac_status iac_ctx_create(int device, iac_ctx **out)
{
    IAC_REQUIRE(out != nullptr, "iac_ctx_create: out is NULL");
    *out = nullptr;
    int n = 0;
    IAC_CUDA(cudaGetDeviceCount(&n));
    IAC_REQUIRE(device >= 0 && device < n, "iac_ctx_create: device %d of %d", device, n);
    cudaDeviceProp prop;
    IAC_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) {
        set_error("iac_ctx_create: device %d is sm_%d%d; this library is built for sm_100a",
                  device, prop.major, prop.minor);
        return IAC_ERR_UNSUPPORTED;
    }
    DeviceGuard g(device);
    iac_ctx *c = new iac_ctx();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    c->cc_major = prop.major;
    c->cc_minor = prop.minor;
    cudaError_t e = cudaMalloc(&c->d_counters, sizeof(DeviceCounters));
    if (e != cudaSuccess) {
        delete c;
        set_error("iac_ctx_create: %s", cudaGetErrorString(e));
        return IAC_ERR_NO_MEMORY;
    }
    cudaMemset(c->d_counters, 0, sizeof(DeviceCounters));
    cudaDeviceSynchronize();
    // device address of the allocation-free entry point's fixed scratch array
    const iac_status st = static_scratch_setup(c);
    if (st != IAC_OK) {
        cudaFree(c->d_counters);
        delete c;
        return st;
    }
    load_tuning_table(c);
    *out = c;
    return IAC_OK;
}

iac_status iac_ctx_destroy(iac_ctx *ctx)
{
    if (!ctx) return IAC_OK;
    {
        DeviceGuard g(ctx->device);
        cudaDeviceSynchronize();
        ctx->sparse_scratch.release();
        for (auto &kv : ctx->stream_scratch) {
            for (auto &s : kv.second.bufs) s.release();
        }
        if (ctx->d_counters) cudaFree(ctx->d_counters);
        for (auto &e : ctx->copy_events)
            if (e) cudaEventDestroy(e);
        for (auto &e : ctx->staging_free)
            if (e) cudaEventDestroy(e);
        if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
        if (ctx->host_stream) cudaStreamDestroy(ctx->host_stream);
    }
    delete ctx;
    return IAC_OK;
}

iac_status iac_ctx_check(iac_ctx *ctx, void *stream, uint64_t *out_of_mesh)
{
    IAC_REQUIRE(ctx != nullptr, "iac_ctx_check: ctx is NULL");
    DeviceGuard g(ctx->device);
    IAC_CUDA(cudaStreamSynchronize(as_stream(stream)));
    DeviceCounters h;
    IAC_CUDA(cudaMemcpy(&h, ctx->d_counters, sizeof h, cudaMemcpyDeviceToHost));
    IAC_CUDA(cudaMemset(ctx->d_counters, 0, sizeof h));
    if (out_of_mesh) *out_of_mesh = h.out_of_mesh;
    if (h.timeouts) {
        char sites[256] = "";
        for (int k = 0; k < SITE_COUNT; k++)
            if (h.timeout_sites & (1ull << k)) {
                if (sites[0]) strncat(sites, ", ", sizeof sites - strlen(sites) - 1);
                strncat(sites, WAIT_SITE_NAMES[k], sizeof sites - strlen(sites) - 1);
            }
        set_error("%llu bounded device waits ran out (%s)", (unsigned long long)h.timeouts, sites);
        return IAC_ERR_TIMEOUT;
    }
    if (h.photon_overflow) {
        set_error("%llu photons did not fit the photon-list capacity and were dropped",
                  (unsigned long long)h.photon_overflow);
        return IAC_ERR_NO_MEMORY;
    }
    if (h.out_of_mesh) {
        set_error("%llu writes fell outside the mesh and were skipped",
                  (unsigned long long)h.out_of_mesh);
        return IAC_ERR_OUT_OF_MESH;
    }
    return IAC_OK;
}

iac_status iac_ctx_set_scratch_limit(iac_ctx *ctx, uint64_t max_bytes)
{
    IAC_REQUIRE(ctx != nullptr, "iac_ctx_set_scratch_limit: ctx is NULL");
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->scratch_limit = max_bytes;
    return IAC_OK;
}

iac_status iac_ctx_wait_flag(iac_ctx *ctx, const uint32_t *d_flag, uint32_t max_polls, void *stream)
{
    IAC_REQUIRE(ctx && d_flag, "iac_ctx_wait_flag: NULL argument");
    IAC_REQUIRE(max_polls <= 10000000u, "iac_ctx_wait_flag: at most 10^7 polls (about 10 s)");
    DeviceGuard g(ctx->device);
    wait_flag_kernel<<<1, 1, 0, as_stream(stream)>>>(d_flag, max_polls, ctx->d_counters);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}

iac_status iac_device_alloc(iac_ctx *ctx, size_t bytes, void **d_ptr)
{
    IAC_REQUIRE(ctx && d_ptr, "iac_device_alloc: NULL argument");
    DeviceGuard g(ctx->device);
    *d_ptr = nullptr;
    if (bytes == 0) return IAC_OK;
    IAC_CUDA(cudaMalloc(d_ptr, bytes));
    return IAC_OK;
}

iac_status iac_device_free(iac_ctx *ctx, void *d_ptr)
{
    IAC_REQUIRE(ctx != nullptr, "iac_device_free: ctx is NULL");
    if (!d_ptr) return IAC_OK;
    DeviceGuard g(ctx->device);
    IAC_CUDA(cudaFree(d_ptr));
    return IAC_OK;
}

iac_status iac_host_alloc_pinned(iac_ctx *ctx, size_t bytes, void **h_ptr)
{
    IAC_REQUIRE(ctx && h_ptr, "iac_host_alloc_pinned: NULL argument");
    DeviceGuard g(ctx->device);
    *h_ptr = nullptr;
    if (bytes == 0) return IAC_OK;
    IAC_CUDA(cudaMallocHost(h_ptr, bytes));
    return IAC_OK;
}

iac_status iac_host_free_pinned(iac_ctx *ctx, void *h_ptr)
{
    IAC_REQUIRE(ctx != nullptr, "iac_host_free_pinned: ctx is NULL");
    if (!h_ptr) return IAC_OK;
    IAC_CUDA(cudaFreeHost(h_ptr));
    return IAC_OK;
}

static iac_status copy(iac_ctx *ctx, void *dst, const void *src, size_t bytes, cudaMemcpyKind k,
                       void *stream)
{
    IAC_REQUIRE(ctx != nullptr, "copy: ctx is NULL");
    if (bytes == 0) return IAC_OK;
    IAC_REQUIRE(dst && src, "copy: NULL pointer");
    DeviceGuard g(ctx->device);
    IAC_CUDA(cudaMemcpyAsync(dst, src, bytes, k, as_stream(stream)));
    return IAC_OK;
}

iac_status iac_memcpy_h2d(iac_ctx *ctx, void *d, const void *h, size_t n, void *stream)
{
    return copy(ctx, d, h, n, cudaMemcpyHostToDevice, stream);
}
iac_status iac_memcpy_d2h(iac_ctx *ctx, void *h, const void *d, size_t n, void *stream)
{
    return copy(ctx, h, d, n, cudaMemcpyDeviceToHost, stream);
}
iac_status iac_memcpy_d2d(iac_ctx *ctx, void *d, const void *s, size_t n, void *stream)
{
    return copy(ctx, d, s, n, cudaMemcpyDeviceToDevice, stream);
}

iac_status iac_memset_device(iac_ctx *ctx, void *d_ptr, int value, size_t bytes, void *stream)
{
    IAC_REQUIRE(ctx != nullptr, "iac_memset_device: ctx is NULL");
    if (bytes == 0) return IAC_OK;
    IAC_REQUIRE(d_ptr != nullptr, "iac_memset_device: NULL pointer");
    DeviceGuard g(ctx->device);
    IAC_CUDA(cudaMemsetAsync(d_ptr, value, bytes, as_stream(stream)));
    return IAC_OK;
}

iac_status iac_stream_create(iac_ctx *ctx, void **stream)
{
    IAC_REQUIRE(ctx && stream, "iac_stream_create: NULL argument");
    DeviceGuard g(ctx->device);
    cudaStream_t s;
    IAC_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    *stream = (void *)s;
    return IAC_OK;
}

iac_status iac_stream_destroy(iac_ctx *ctx, void *stream)
{
    IAC_REQUIRE(ctx != nullptr, "iac_stream_destroy: ctx is NULL");
    if (!stream) return IAC_OK;
    DeviceGuard g(ctx->device);
    IAC_CUDA(cudaStreamSynchronize(as_stream(stream)));
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        auto it = ctx->stream_scratch.find(stream);
        if (it != ctx->stream_scratch.end()) {
            for (auto &b : it->second.bufs) b.release();
            ctx->stream_scratch.erase(it);
        }
    }
    IAC_CUDA(cudaStreamDestroy(as_stream(stream)));
    return IAC_OK;
}

iac_status iac_stream_synchronize(iac_ctx *ctx, void *stream)
{
    IAC_REQUIRE(ctx != nullptr, "iac_stream_synchronize: ctx is NULL");
    DeviceGuard g(ctx->device);
    IAC_CUDA(cudaStreamSynchronize(as_stream(stream)));
    return IAC_OK;
}

uint64_t iac_ctx_launch_count(const iac_ctx *ctx)
{
    return ctx ? ctx->launches.load(std::memory_order_relaxed) : 0;
}

// ---------------------------------------------------------------------------
// mesh geometry (host arithmetic in the reference's float order)
// ---------------------------------------------------------------------------

static void mesh_pitch(iac_mesh_shape *s, float maxq)
{
    s->max_q = maxq;
    s->dq_per_voxel = maxq / (float)(((s->size_ab - 1) / 2) - 2);
    s->voxel_per_dq = (uint32_t)std::floor(1.0f / s->dq_per_voxel);
    s->dq_per_voxel = 1.0f / ((float)s->voxel_per_dq);
}

iac_status iac_big_mesh_shape(const float mq[3], int edge, float q_zoom, iac_mesh_shape *s)
{
    IAC_REQUIRE(mq && s, "iac_big_mesh_shape: NULL argument");
    IAC_REQUIRE(edge % 2 != 0, "Meshsize must be odd for each dimension (got %d)", edge);
    IAC_REQUIRE(edge >= 5, "mesh edge %d too small", edge);
    s->k_a = 0;
    s->k_b = 1;
    s->k_c = 2;
    s->size_ab = (uint32_t)edge + 2;
    s->size_c = s->size_ab;
    s->center[0] = s->center[1] = (s->size_ab - 1) / 2;
    s->center[2] = (s->size_c - 1) / 2;
    float m = std::max(std::max(mq[0], mq[1]), mq[2]);
    mesh_pitch(s, m / q_zoom);
    return IAC_OK;
}

iac_status iac_small_cq_mesh_shape(const float mq[3], int perp, float q_zoom, iac_mesh_shape *s)
{
    IAC_REQUIRE(mq && s, "iac_small_cq_mesh_shape: NULL argument");
    IAC_REQUIRE(perp % 2 != 0, "Meshsize must be odd for each dimension (got %d)", perp);
    IAC_REQUIRE(perp >= 5, "mesh edge %d too small", perp);
    uint32_t a = 0, b = 1, c = 2;
    if (mq[b] > mq[a]) std::swap(a, b);
    if (mq[c] > mq[b]) std::swap(c, b);
    if (mq[b] > mq[a]) std::swap(a, b);
    s->k_a = a;
    s->k_b = b;
    s->k_c = c;
    s->size_ab = (uint32_t)perp + 2;
    if (q_zoom == 1.0f)
        s->size_c = (uint32_t)(int)std::floor((double)((mq[c] / mq[a]) * (float)perp) + 2.5);
    else
        s->size_c = s->size_ab;
    if (s->size_c % 2 == 0) s->size_c += 1;
    s->center[0] = s->center[1] = (s->size_ab - 1) / 2;
    s->center[2] = (s->size_c - 1) / 2;
    mesh_pitch(s, mq[a] / q_zoom);
    return IAC_OK;
}

iac_status iac_ac1d_shape_init(const float mq[3], uint32_t size, float q_zoom, iac_ac1d_shape *s)
{
    IAC_REQUIRE(mq && s, "iac_ac1d_shape_init: NULL argument");
    IAC_REQUIRE(size >= 3, "AC1D array size %u too small", size);
    s->size = size;
    s->max_q = std::sqrt(mq[0] * mq[0] + mq[1] * mq[1] + mq[2] * mq[2]) / q_zoom;
    s->dq_per_step = s->max_q / ((float)(size - 2));
    return IAC_OK;
}

// ---------------------------------------------------------------------------
// host-side multiplicators and the merge weight table
// ---------------------------------------------------------------------------

// ArrayOperators::Min_Max_Mean_Value(float*) mean, IAC/ArrayOperators.h:160-175
static float mean_of(const float *a, uint64_t n)
{
    double t = 0;
    for (uint64_t i = 0; i < n; i++) t += a[i];
    t = t / (double)(int)n;
    return (float)t;
}

iac_status iac_cq_small_multiplicator(const float *h_I, uint64_t npix, double *mult)
{
    IAC_REQUIRE(h_I && mult && npix > 0, "iac_cq_small_multiplicator: bad argument");
    const float m = mean_of(h_I, npix);
    IAC_REQUIRE(m > 0, "No intensity > 0 found in averaged intensity");
    double x = 1e-10;
    for (; 1 > (double)(m * m) * x;) x *= 10;
    *mult = x * 100000;
    return IAC_OK;
}

iac_status iac_ac1d_cq_multiplicator(const float *h_I, uint64_t npix, double *mult)
{
    IAC_REQUIRE(h_I && mult && npix > 0, "iac_ac1d_cq_multiplicator: bad argument");
    const float m = mean_of(h_I, npix);
    IAC_REQUIRE(m > 0, "No intensity > 0 found in averaged intensity");
    double x = 1e-10;
    for (; 1 > (double)(m * m) * x;) x *= 10;
    x = x * 1e5;
    if (x > 1e18) x = 1e18;
    *mult = x;
    return IAC_OK;
}

iac_status iac_cq_merge_weights(const float *R, const float *MI, uint32_t nf, const double *cq,
                                uint64_t small_n, float *rw, double *mult_out)
{
    IAC_REQUIRE(R && MI && cq && rw && mult_out && small_n > 0, "iac_cq_merge_weights: bad argument");
    double maxw = 0.0;
    for (uint32_t i = 0; i < nf; i++) {
        for (int d = 0; d < 9; d++) rw[10 * (size_t)i + d] = R[9 * (size_t)i + d];
        rw[10 * (size_t)i + 9] = (float)((double)MI[i] * (double)MI[i]);
        if (MI[i] > maxw) maxw = MI[i];
    }
    double t = 0;
    for (uint64_t i = 0; i < small_n; i++) t += cq[i];
    const double mean_cq = t / (double)(int)small_n;
    // the reference's search below never ends for an empty C(q) or zero weights
    IAC_REQUIRE(mean_cq > 0 && maxw > 0, "C(q) mesh is empty or every frame weight is zero");
    double m = 1e-12;
    for (; 1 > maxw * maxw * mean_cq * m;) m *= 10;
    uint64_t oom = 1;
    for (; oom < nf;) oom *= 10;
    m = m / (double)oom;
    m *= 1e10;
    if (m > 0.6) m = std::round(m);
    if (m < 1 && m > 0.1) m = 1;
    if (m < 1e-12) m = 1e-12;
    for (uint32_t i = 0; i < nf; i++) {
        float red = (float)m;
        if (m > 0.6) red = std::round((float)m);
        float w = rw[10 * (size_t)i + 9];
        w *= red;
        w = std::floor((float)((double)w + 0.5));
        rw[10 * (size_t)i + 9] = w / red;
    }
    *mult_out = m;
    return IAC_OK;
}

uint64_t iac_half_mesh_words(uint32_t S) { return (uint64_t)S * S * ((S + 1) / 2); }
uint64_t iac_full_mesh_words(uint32_t S) { return (uint64_t)S * S * S; }

}  // extern "C"

// ---------------------------------------------------------------------------
// k-map: unit vectors and the per-block extent of each axis
// ---------------------------------------------------------------------------
__global__ void kmap_kernel(const float *__restrict__ pm, uint64_t npix, float *__restrict__ km,
                            float *__restrict__ block_ext)
{
    float mx[3] = {-100.0f, -100.0f, -100.0f}, mn[3] = {100.0f, 100.0f, 100.0f};
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < npix;
         i += (uint64_t)gridDim.x * blockDim.x) {
        float x = pm[3 * i], y = pm[3 * i + 1], z = pm[3 * i + 2];
        float r = norm3(x, y, z);
        float k[3] = {__fdiv_rn(x, r), __fdiv_rn(y, r), __fdiv_rn(z, r)};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            km[3 * i + d] = k[d];
            mx[d] = fmaxf(mx[d], k[d]);
            mn[d] = fminf(mn[d], k[d]);
        }
    }
    __shared__ float s[6][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        for (int o = 16; o; o >>= 1) {
            mx[d] = fmaxf(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
            mn[d] = fminf(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
        }
    }
    if (lane == 0)
        for (int d = 0; d < 3; d++) {
            s[d][w] = mx[d];
            s[3 + d][w] = mn[d];
        }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int nw = blockDim.x >> 5;
        float v = s[threadIdx.x][0];
        for (int j = 1; j < nw; j++)
            v = threadIdx.x < 3 ? fmaxf(v, s[threadIdx.x][j]) : fminf(v, s[threadIdx.x][j]);
        block_ext[6 * blockIdx.x + threadIdx.x] = v;
    }
}

extern "C" iac_status iac_calc_kmap(iac_ctx *ctx, const float *d_pm, uint64_t npix, float *d_km,
                                    float max_q[3], void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx && d_pm && d_km && max_q, "iac_calc_kmap: NULL argument");
    IAC_REQUIRE(npix > 0, "iac_calc_kmap: empty pixel map");
    DeviceGuard g(ctx->device);
    const int threads = 256;
    int blocks = (int)std::min<uint64_t>((npix + threads - 1) / threads, 4 * (uint64_t)ctx->sm_count);
    float *d_ext = nullptr;
    IAC_CUDA(cudaMallocAsync(&d_ext, sizeof(float) * 6 * blocks, as_stream(stream)));
    kmap_kernel<<<blocks, threads, 0, as_stream(stream)>>>(d_pm, npix, d_km, d_ext);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    std::vector<float> ext(6 * (size_t)blocks);
    IAC_CUDA(cudaMemcpyAsync(ext.data(), d_ext, sizeof(float) * ext.size(), cudaMemcpyDeviceToHost,
                             as_stream(stream)));
    IAC_CUDA(cudaFreeAsync(d_ext, as_stream(stream)));
    IAC_CUDA(cudaStreamSynchronize(as_stream(stream)));
    float mx[3] = {-100.0f, -100.0f, -100.0f}, mn[3] = {100.0f, 100.0f, 100.0f};
    for (int b = 0; b < blocks; b++)
        for (int d = 0; d < 3; d++) {
            mx[d] = std::max(mx[d], ext[6 * b + d]);
            mn[d] = std::min(mn[d], ext[6 * b + 3 + d]);
        }
    for (int d = 0; d < 3; d++) max_q[d] = std::fabs(mx[d] - mn[d]);
    return IAC_OK;
}

// ---------------------------------------------------------------------------
// scatter-add micro-benchmark: the L2 atomic rate that bounds the binning
// kernels.  Each update adds 1 at a pseudo-random word chosen by a 32-bit
// multiplicative hash and a multiply-high range reduction, so the loop body
// is a handful of integer instructions around one RED.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void scatter_add_kernel(T *__restrict__ buf, uint32_t words, uint64_t updates, uint32_t seed)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint32_t h = (uint32_t)u * 2654435761u + seed * 97u;
    for (; u < updates; u += stride) {
        h = h * 1664525u + 1013904223u;
        const uint32_t x = h ^ (h >> 15);
        atomicAdd(&buf[__umulhi(x, words)], (T)1);
    }
}

extern "C" iac_status iac_bench_scatter_add(iac_ctx *ctx, void *d_buffer, uint64_t words,
                                            int word_bits, uint64_t updates, uint32_t seed,
                                            void *stream)
{
    IAC_REQUIRE(ctx && d_buffer && words > 0 && words <= 0xffffffffull,
                "iac_bench_scatter_add: bad argument");
    IAC_REQUIRE(word_bits == 32 || word_bits == 64, "word_bits must be 32 or 64");
    DeviceGuard g(ctx->device);
    const int threads = 256;
    const int blocks = ctx->sm_count * 8;
    if (word_bits == 64)
        scatter_add_kernel<unsigned long long><<<blocks, threads, 0, as_stream(stream)>>>(
            (unsigned long long *)d_buffer, (uint32_t)words, updates, seed);
    else
        scatter_add_kernel<unsigned int><<<blocks, threads, 0, as_stream(stream)>>>(
            (unsigned int *)d_buffer, (uint32_t)words, updates, seed);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}
