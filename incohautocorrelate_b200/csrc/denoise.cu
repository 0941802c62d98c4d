// denoise.cu -- host runtime of the mesh denoiser (no reference counterpart):
// a 3-level 3D U-Net (16/32/64 channels, 3x3x3 convolutions, average
// pooling, nearest upsampling with skip concatenation, residual 1x1 head)
// trained with MSE and AdamW by the kernels of denoise_kernels.cu.
//
//   x (1) -> e1a 16 -> s1 16 --pool--> e2a 32 -> s2 32 --pool--> b1 64 -> b2 64
//   up(b2) ++ s2 (96) -> d2a 32 -> d2b 32 ; up(d2b) ++ s1 (48) -> d1a 16 -> d1b 16
//   out = x + head(d1b)
//
// Parameters live in one flat fp32 array (per 3x3x3 layer: W[cout][27][cin]
// then b[cout]; head: w[16], b), with AdamW moments beside it and the bf16
// operand tiles refreshed after every update.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "denoise_internal.cuh"

using namespace iac;
using namespace iac::dn;

namespace {

struct LayerSpec {
    int cin, cout;
};
// 10 convolutions + head
constexpr LayerSpec SPECS[11] = {{1, 16},  {16, 16}, {16, 32}, {32, 32}, {32, 64}, {64, 64},
                                 {96, 32}, {32, 32}, {48, 16}, {16, 16}, {16, 1}};
constexpr int NCONV = 10;

long long layer_params(int l)
{
    return l < NCONV ? (long long)SPECS[l].cout * 27 * SPECS[l].cin + SPECS[l].cout : 17;
}

}  // namespace

struct iac_denoiser {
    iac_ctx *ctx = nullptr;
    int backend = 0;
    uint32_t max_batch = 0, D = 0, H = 0, W = 0;
    long long nparams = 0;
    long long p_off[11] = {};
    long long wf_off[10] = {}, wd_off[10] = {};
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    bf16 *wf = nullptr, *wd = nullptr;
    long long adam_step = 0;
    double *d_loss = nullptr;
    // activations
    bf16 *e1a = nullptr, *s1 = nullptr, *p1 = nullptr, *e2a = nullptr, *s2 = nullptr, *p2 = nullptr;
    bf16 *b1 = nullptr, *b2 = nullptr, *d2a = nullptr, *d2b = nullptr, *d1a = nullptr, *d1b = nullptr;
    bf16 *cat1 = nullptr, *cat2 = nullptr;  // decoder inputs: up(d2b) ++ s1, up(b2) ++ s2
    uint64_t step_launches = 0;             // kernels in the training-step graph
    // gradients
    bf16 *gA = nullptr, *gB = nullptr, *gup1 = nullptr, *gskip1 = nullptr;  // full resolution
    bf16 *hA = nullptr, *hB = nullptr, *gup2 = nullptr, *gskip2 = nullptr;  // half
    bf16 *qA = nullptr, *qB = nullptr;                                       // quarter
    std::vector<void *> allocs;
    // CUDA graph of one training step (iac_denoise_train_steps)
    long long *d_step = nullptr;  // [0] replay index, [1] optimizer steps so far
    float *px = nullptr, *pt = nullptr;
    double *d_dummy_loss = nullptr;
    cudaGraphExec_t step_exec = nullptr;
    std::vector<uintptr_t> step_key;
    cudaStream_t own_stream = nullptr;  // capture and replay stream of the step graph (highest priority)
    cudaEvent_t own_ev[2] = {nullptr, nullptr};
    cudaStream_t side = nullptr;          // the weight gradients' stream in the backward
    cudaEvent_t ev_g[10] = {}, ev_w[10] = {};  // per layer: its G ready, its weight gradient done

    void *alloc(size_t bytes)
    {
        void *ptr = nullptr;
        if (cudaMalloc(&ptr, bytes) != cudaSuccess) return nullptr;
        allocs.push_back(ptr);
        return ptr;
    }
    ~iac_denoiser()
    {
        if (step_exec) cudaGraphExecDestroy(step_exec);
        for (cudaEvent_t e : own_ev)
            if (e) cudaEventDestroy(e);
        for (int l = 0; l < 10; l++) {
            if (ev_g[l]) cudaEventDestroy(ev_g[l]);
            if (ev_w[l]) cudaEventDestroy(ev_w[l]);
        }
        if (side) cudaStreamDestroy(side);
        if (own_stream) cudaStreamDestroy(own_stream);
        for (void *a : allocs) cudaFree(a);
    }
};

namespace {

iac_status cuda_status(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return IAC_OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return IAC_ERR_CUDA;
}

#define DN_CHECK(expr, what)                                 \
    do {                                                     \
        const iac_status _st = cuda_status((expr), (what)); \
        if (_st != IAC_OK) return _st;                       \
    } while (0)

iac_status check_dims(const iac_denoiser *dn, uint32_t nb, uint32_t D, uint32_t H, uint32_t W)
{
    IAC_REQUIRE(nb >= 1 && nb <= dn->max_batch, "batch %u outside 1..%u", nb, dn->max_batch);
    IAC_REQUIRE(D % 4 == 0 && H % 4 == 0 && W % 4 == 0 && D >= 4 && H >= 4 && W >= 4,
                "volume %ux%ux%u: every edge must be a multiple of 4", D, H, W);
    IAC_REQUIRE((uint64_t)nb * D * H * W <= (uint64_t)dn->max_batch * dn->D * dn->H * dn->W,
                "volume %u x %ux%ux%u exceeds the workspace", nb, D, H, W);
    return IAC_OK;
}

// forward operands of layer l: src1 alone, or the decoder's concatenation of
// src0 (half resolution, upsampled) and the skip tensor src1
ConvArgs conv_args(iac_denoiser *dn, int l, const bf16 *src0, const bf16 *src1, bf16 *y, int D, int H, int W,
                   long long V)
{
    ConvArgs a{};
    const int cin = SPECS[l].cin;
    a.src1 = src1;
    if (src0) {
        a.src0 = src0;
        a.up0 = 1;
        a.c1 = l == 6 ? 32 : 16;  // skip channels of s2 / s1
        a.c0 = cin - a.c1;
    } else {
        a.c1 = cin;
    }
    a.w = dn->wf + dn->wf_off[l];
    a.bias = dn->p + dn->p_off[l] + (long long)SPECS[l].cout * 27 * cin;
    a.y = y;
    a.relu = 1;
    a.D = D;
    a.H = H;
    a.W = W;
    a.V = V;
    a.counters = dn->ctx->d_counters;
    a.sms = dn->ctx->sm_count;
    return a;
}

// data gradient of layer l: G (cout channels) -> dX (cin channels); with
// relu_y (the forward activation dX belongs to) the ReLU derivative is applied
// in the same kernel: dX = 0 where relu_y <= 0
iac_status dgrad(iac_denoiser *dn, int l, const bf16 *gp, bf16 *out, int D, int H, int W, long long V,
                 cudaStream_t s, const bf16 *relu_y = nullptr, bf16 *out2 = nullptr, int split = 0)
{
    ConvArgs a{};
    a.mask_y = relu_y;
    a.src1 = gp;
    a.c1 = SPECS[l].cout;
    a.w = dn->wd + dn->wd_off[l];
    a.y = out;
    a.y2 = out2;  // with out2: channels split.. of dX there, the first split in out
    a.split = split;
    a.D = D;
    a.H = H;
    a.W = W;
    a.V = V;
    a.counters = dn->ctx->d_counters;
    a.sms = dn->ctx->sm_count;
    DN_CHECK(conv3x3(a, SPECS[l].cout, SPECS[l].cin, dn->backend, s), "denoiser data gradient");
    return IAC_OK;
}

// IAC_DENOISE_WGRAD_ZS=0 in the environment keeps the weight gradients on one
// dz per CTA (for comparing the kernels)
static bool wgrad_zs_enabled()
{
    static const bool on = [] {
        const char *e = getenv("IAC_DENOISE_WGRAD_ZS");
        return !(e && e[0] == '0');
    }();
    return on;
}

iac_status wgrad(iac_denoiser *dn, int l, const bf16 *src0, const bf16 *src1, const bf16 *gp, int D, int H,
                 int W, long long V, cudaStream_t s)
{
    WgradArgs a{};
    const int cin = SPECS[l].cin;
    a.src1 = src1;
    if (src0) {
        a.src0 = src0;
        a.up0 = 1;
        a.c1 = l == 6 ? 32 : 16;
        a.c0 = cin - a.c1;
    } else {
        a.c1 = cin;
    }
    a.g = gp;
    a.dw = dn->g + dn->p_off[l];
    a.db = dn->g + dn->p_off[l] + (long long)SPECS[l].cout * 27 * cin;
    a.D = D;
    a.H = H;
    a.W = W;
    a.V = V;
    a.cout = SPECS[l].cout;
    // tcgen05 with the dz planes stacked into one MMA operand where the layer's
    // shape has a configuration (wgrad3x3 falls back to one dz per CTA, then
    // to mma.sync on slabs), mma.sync on slabs for the mma.sync backend
    if (dn->backend == BACKEND_TC_TAP)
        a.slabs = 0;
    else if (dn->backend == BACKEND_TC_SLAB)
        a.slabs = wgrad_zs_enabled() ? 3 : (cin >= 32 ? 2 : 1);
    else
        a.slabs = 1;
    a.counters = dn->ctx->d_counters;
    DN_CHECK(wgrad3x3(a, cin, dn->ctx->sm_count, s), "denoiser weight gradient");
    return IAC_OK;
}

iac_status refresh_tiles(iac_denoiser *dn, const iac_adamw *opt, cudaStream_t s,
                         const long long *d_step = nullptr, const float *lrs = nullptr)
{
    AdamArgs a{};
    a.d_step = d_step;
    a.lrs = lrs;
    a.p = dn->p;
    a.g = dn->g;
    a.m = dn->m;
    a.v = dn->v;
    a.n = dn->nparams;
    a.wf = dn->wf;
    a.wd = dn->wd;
    a.nlayers = 11;
    for (int l = 0; l < 11; l++) {
        a.layers[l].off = dn->p_off[l];
        a.layers[l].cout = SPECS[l].cout;
        a.layers[l].cin = SPECS[l].cin;
        a.layers[l].taps = l < NCONV ? 27 : 0;
        a.layers[l].wf_off = l < NCONV ? dn->wf_off[l] : 0;
        a.layers[l].wd_off = l < NCONV ? dn->wd_off[l] : 0;
    }
    if (opt) {
        if (!d_step) dn->adam_step++;
        a.update = 1;
        a.lr = opt->lr;
        a.beta1 = opt->beta1;
        a.beta2 = opt->beta2;
        a.eps = opt->eps;
        a.weight_decay = opt->weight_decay;
        a.bc1 = (float)(1.0 - std::pow((double)opt->beta1, (double)dn->adam_step));
        a.bc2 = (float)(1.0 - std::pow((double)opt->beta2, (double)dn->adam_step));
    }
    DN_CHECK(adamw(a, s), "denoiser AdamW");
    return IAC_OK;
}

iac_status run_forward(iac_denoiser *dn, const float *x, uint32_t nb, uint32_t D, uint32_t H, uint32_t W,
                       cudaStream_t s)
{
    const long long V = (long long)nb * D * H * W, V2 = V / 8, V4 = V / 64;
    const int D2 = D / 2, H2 = H / 2, W2 = W / 2, D4 = D / 4, H4 = H / 4, W4 = W / 4;
    const int be = dn->backend;
    DN_CHECK(conv3x3_first(x, dn->wf + dn->wf_off[0], dn->p + dn->p_off[0] + 16 * 27, dn->e1a, D, H, W, V, s),
             "denoiser layer 0");
    DN_CHECK(conv3x3(conv_args(dn, 1, nullptr, dn->e1a, dn->s1, D, H, W, V), 16, 16, be, s), "layer 1");
    DN_CHECK(avgpool2(dn->s1, 16, dn->p1, 16, D, H, W, nb, s), "pool 1");
    DN_CHECK(conv3x3(conv_args(dn, 2, nullptr, dn->p1, dn->e2a, D2, H2, W2, V2), 16, 32, be, s), "layer 2");
    DN_CHECK(conv3x3(conv_args(dn, 3, nullptr, dn->e2a, dn->s2, D2, H2, W2, V2), 32, 32, be, s), "layer 3");
    DN_CHECK(avgpool2(dn->s2, 32, dn->p2, 32, D2, H2, W2, nb, s), "pool 2");
    DN_CHECK(conv3x3(conv_args(dn, 4, nullptr, dn->p2, dn->b1, D4, H4, W4, V4), 32, 64, be, s), "layer 4");
    DN_CHECK(conv3x3(conv_args(dn, 5, nullptr, dn->b1, dn->b2, D4, H4, W4, V4), 64, 64, be, s), "layer 5");
    // the decoder inputs (64 + 32 and 32 + 16 channels) are materialised, so the
    // 3x3x3 kernels read plain tensors through TMA: the coarse part upsampled,
    // the skip tensor copied
    DN_CHECK(concat_up(dn->b2, 64, dn->s2, 32, dn->cat2, D2, H2, W2, nb, s), "concat 2");
    DN_CHECK(conv3x3(conv_args(dn, 6, nullptr, dn->cat2, dn->d2a, D2, H2, W2, V2), 96, 32, be, s), "layer 6");
    DN_CHECK(conv3x3(conv_args(dn, 7, nullptr, dn->d2a, dn->d2b, D2, H2, W2, V2), 32, 32, be, s), "layer 7");
    DN_CHECK(concat_up(dn->d2b, 32, dn->s1, 16, dn->cat1, D, H, W, nb, s), "concat 1");
    DN_CHECK(conv3x3(conv_args(dn, 8, nullptr, dn->cat1, dn->d1a, D, H, W, V), 48, 16, be, s), "layer 8");
    DN_CHECK(conv3x3(conv_args(dn, 9, nullptr, dn->d1a, dn->d1b, D, H, W, V), 16, 16, be, s), "layer 9");
    return IAC_OK;
}

uint64_t splitmix(uint64_t &s)
{
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// forward, loss into loss[d_step ? d_step[0] : 0] (accumulated), gradients into dn->g
iac_status run_backward(iac_denoiser *dn, const float *d_in, const float *d_target, const float *d_weight, uint32_t nb,
                        uint32_t D, uint32_t H, uint32_t W, float *d_out, double *loss, const long long *d_step,
                        cudaStream_t s)
{
    iac_status st = IAC_OK;
    const long long V = (long long)nb * D * H * W, V2 = V / 8, V4 = V / 64;
    const int D2 = D / 2, H2 = H / 2, W2 = W / 2, D4 = D / 4, H4 = H / 4, W4 = W / 4;
    DN_CHECK(cudaMemsetAsync(dn->g, 0, dn->nparams * 4, s), "clear gradients");
    st = run_forward(dn, d_in, nb, D, H, W, s);
    if (st != IAC_OK) return st;
    HeadArgs h{};
    h.x = d_in;
    h.d = dn->d1b;
    h.w = dn->p + dn->p_off[10];
    h.target = d_target;
    h.weight = d_weight;
    h.out = d_out;
    h.gd = dn->gA;  // = d loss / d pre-activation of layer 9
    h.dw = dn->g + dn->p_off[10];
    h.loss = loss;
    h.d_step = d_step;
    h.V = V;
    h.inv_count = 1.0 / (double)V;
    DN_CHECK(head(h, dn->ctx->sm_count, s), "denoiser head");
    // The weight gradients run on a side stream beside the chain of data
    // gradients: wgrad(l) needs only the gradient G(l) and its layer's input,
    // and its result is read by AdamW alone. Each wgrad waits for its G (an
    // event on the main stream), and the main stream waits for wgrad(k) before
    // it overwrites a buffer wgrad(k) reads (the gradient buffers are reused
    // down the network); at the end the main stream waits for the side stream.
    cudaStream_t sw = dn->side;
    auto fork_wgrad = [&](int l, const bf16 *x, const bf16 *g, int d, int hh, int ww, long long v) -> iac_status {
        DN_CHECK(cudaEventRecord(dn->ev_g[l], s), "weight-gradient fork");
        DN_CHECK(cudaStreamWaitEvent(sw, dn->ev_g[l], 0), "weight-gradient fork");
        iac_status r = wgrad(dn, l, nullptr, x, g, d, hh, ww, v, sw);
        if (r != IAC_OK) return r;
        DN_CHECK(cudaEventRecord(dn->ev_w[l], sw), "weight-gradient done");
        return IAC_OK;
    };
    auto after_wgrad = [&](int l) -> iac_status {
        DN_CHECK(cudaStreamWaitEvent(s, dn->ev_w[l], 0), "weight-gradient join");
        return IAC_OK;
    };
#define DN_TRY(expr)                    \
    do {                                \
        if ((st = (expr)) != IAC_OK) return st; \
    } while (0)
    // layer 9: X = d1a
    DN_TRY(fork_wgrad(9, dn->d1a, dn->gA, D, H, W, V));
    DN_TRY(dgrad(dn, 9, dn->gA, dn->gB, D, H, W, V, s, dn->d1a));
    // layer 8: X = up(d2b) ++ s1; the decoder input's gradient in two parts: the upsampled 32
    // channels, the skip 16
    DN_TRY(fork_wgrad(8, dn->cat1, dn->gB, D, H, W, V));
    DN_TRY(dgrad(dn, 8, dn->gB, dn->gup1, D, H, W, V, s, nullptr, dn->gskip1, 32));
    DN_CHECK(split_concat_grad(dn->gup1, 32, dn->d2b, dn->hA, D, H, W, nb, s), "split 1");
    // layer 7: X = d2a
    DN_TRY(fork_wgrad(7, dn->d2a, dn->hA, D2, H2, W2, V2));
    DN_TRY(dgrad(dn, 7, dn->hA, dn->hB, D2, H2, W2, V2, s, dn->d2a));
    // layer 6: X = up(b2) ++ s2
    DN_TRY(fork_wgrad(6, dn->cat2, dn->hB, D2, H2, W2, V2));
    DN_TRY(dgrad(dn, 6, dn->hB, dn->gup2, D2, H2, W2, V2, s, nullptr, dn->gskip2, 64));
    DN_CHECK(split_concat_grad(dn->gup2, 64, dn->b2, dn->qA, D2, H2, W2, nb, s), "split 2");
    // layer 5: X = b1
    DN_TRY(fork_wgrad(5, dn->b1, dn->qA, D4, H4, W4, V4));
    DN_TRY(dgrad(dn, 5, dn->qA, dn->qB, D4, H4, W4, V4, s, dn->b1));
    // layer 4: X = p2; its data gradient overwrites qA (wgrad 5's G)
    DN_TRY(fork_wgrad(4, dn->p2, dn->qB, D4, H4, W4, V4));
    DN_TRY(after_wgrad(5));
    DN_TRY(dgrad(dn, 4, dn->qB, dn->qA, D4, H4, W4, V4, s));  // d p2 (32 ch)
    DN_TRY(after_wgrad(7));  // hA (wgrad 7's G) is overwritten next
    DN_CHECK(pool_grad_mask(dn->gskip2, 32, dn->qA, dn->s2, 32, dn->hA, 32, D2, H2, W2, nb, s), "pool grad 2");
    // layer 3: X = e2a
    DN_TRY(fork_wgrad(3, dn->e2a, dn->hA, D2, H2, W2, V2));
    DN_TRY(after_wgrad(6));  // hB
    DN_TRY(dgrad(dn, 3, dn->hA, dn->hB, D2, H2, W2, V2, s, dn->e2a));
    // layer 2: X = p1
    DN_TRY(fork_wgrad(2, dn->p1, dn->hB, D2, H2, W2, V2));
    DN_TRY(after_wgrad(3));  // hA
    DN_TRY(dgrad(dn, 2, dn->hB, dn->hA, D2, H2, W2, V2, s));  // d p1 (16 ch)
    DN_TRY(after_wgrad(9));  // gA
    DN_CHECK(pool_grad_mask(dn->gskip1, 16, dn->hA, dn->s1, 16, dn->gA, 16, D, H, W, nb, s), "pool grad 1");
    // layer 1: X = e1a
    DN_TRY(fork_wgrad(1, dn->e1a, dn->gA, D, H, W, V));
    DN_TRY(after_wgrad(8));  // gB
    DN_TRY(dgrad(dn, 1, dn->gA, dn->gB, D, H, W, V, s, dn->e1a));
#undef DN_TRY
    // layer 0: X = input, on the side stream too; then the main stream waits for all
    DN_CHECK(cudaEventRecord(dn->ev_g[0], s), "weight-gradient fork");
    DN_CHECK(cudaStreamWaitEvent(sw, dn->ev_g[0], 0), "weight-gradient fork");
    DN_CHECK(wgrad3x3_first(d_in, dn->gB, dn->g + dn->p_off[0], dn->g + dn->p_off[0] + 16 * 27, D, H, W, V,
                            dn->ctx->sm_count, sw),
             "layer 0 weight gradient");
    DN_CHECK(cudaEventRecord(dn->ev_w[0], sw), "weight-gradient done");
    DN_CHECK(cudaStreamWaitEvent(s, dn->ev_w[0], 0), "weight-gradient join");
    return IAC_OK;
}

}  // namespace

extern "C" {

uint64_t iac_denoise_param_count(void)
{
    long long n = 0;
    for (int l = 0; l < 11; l++) n += layer_params(l);
    return (uint64_t)n;
}

iac_status iac_denoise_create(iac_ctx *ctx, uint32_t max_batch, uint32_t D, uint32_t H, uint32_t W, int backend,
                              iac_denoiser **out)
{
    IAC_REQUIRE(ctx && out, "null argument");
    IAC_REQUIRE(backend >= 0 && backend <= 2, "backend %d (0 = tcgen05 slabs, 1 = mma.sync, 2 = tcgen05 per tap)",
                backend);
    IAC_REQUIRE(max_batch >= 1 && D % 4 == 0 && H % 4 == 0 && W % 4 == 0 && D && H && W,
                "workspace %u x %ux%ux%u: edges must be multiples of 4", max_batch, D, H, W);
    DeviceGuard guard(ctx->device);
    iac_denoiser *dn = new (std::nothrow) iac_denoiser;
    IAC_REQUIRE(dn, "out of host memory");
    dn->ctx = ctx;
    dn->backend = backend;
    dn->max_batch = max_batch;
    dn->D = D;
    dn->H = H;
    dn->W = W;
    long long off = 0, wf = 0, wd = 0;
    for (int l = 0; l < 11; l++) {
        dn->p_off[l] = off;
        off += layer_params(l);
        if (l < NCONV) {
            dn->wf_off[l] = wf;
            dn->wd_off[l] = wd;
            wf += 27LL * SPECS[l].cin * SPECS[l].cout;
            if (SPECS[l].cin > 1) wd += 27LL * SPECS[l].cin * SPECS[l].cout;
        }
    }
    dn->nparams = off;
    const size_t V = (size_t)max_batch * D * H * W, V2 = V / 8, V4 = V / 64;
    bool ok = true;
    auto A = [&](size_t bytes) {
        void *p = dn->alloc(bytes);
        ok &= p != nullptr;
        return p;
    };
    dn->p = (float *)A(off * 4);
    dn->g = (float *)A(off * 4);
    dn->m = (float *)A(off * 4);
    dn->v = (float *)A(off * 4);
    dn->wf = (bf16 *)A(wf * 2);
    dn->wd = (bf16 *)A(wd * 2);
    dn->d_loss = (double *)A(8);
    const size_t b = 2;
    dn->e1a = (bf16 *)A(V * 16 * b);
    dn->d1a = (bf16 *)A(V * 16 * b);
    dn->d1b = (bf16 *)A(V * 16 * b);
    dn->s1 = (bf16 *)A(V * 16 * b);
    dn->p1 = (bf16 *)A(V2 * 16 * b);
    dn->e2a = (bf16 *)A(V2 * 32 * b);
    dn->s2 = (bf16 *)A(V2 * 32 * b);
    dn->d2a = (bf16 *)A(V2 * 32 * b);
    dn->d2b = (bf16 *)A(V2 * 32 * b);
    dn->p2 = (bf16 *)A(V4 * 32 * b);
    dn->b1 = (bf16 *)A(V4 * 64 * b);
    dn->b2 = (bf16 *)A(V4 * 64 * b);
    dn->cat1 = (bf16 *)A(V * 48 * b);
    dn->cat2 = (bf16 *)A(V2 * 96 * b);
    dn->gA = (bf16 *)A(V * 16 * b);
    dn->gB = (bf16 *)A(V * 16 * b);
    dn->gup1 = (bf16 *)A(V * 32 * b);
    dn->gskip1 = (bf16 *)A(V * 16 * b);
    dn->hA = (bf16 *)A(V2 * 32 * b);
    dn->hB = (bf16 *)A(V2 * 32 * b);
    dn->gup2 = (bf16 *)A(V2 * 64 * b);
    dn->gskip2 = (bf16 *)A(V2 * 32 * b);
    dn->qA = (bf16 *)A(V4 * 64 * b);
    dn->qB = (bf16 *)A(V4 * 64 * b);
    dn->d_step = (long long *)A(16);
    dn->d_dummy_loss = (double *)A(8);
    if (!ok) {
        delete dn;
        set_error("device memory for a %u x %ux%ux%u denoiser workspace", max_batch, D, H, W);
        return IAC_ERR_NO_MEMORY;
    }
    bool evs = cudaStreamCreateWithFlags(&dn->side, cudaStreamNonBlocking) == cudaSuccess;
    for (int l = 0; l < 10 && evs; l++)
        evs = cudaEventCreateWithFlags(&dn->ev_g[l], cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&dn->ev_w[l], cudaEventDisableTiming) == cudaSuccess;
    if (!evs) {
        delete dn;
        set_error("the denoiser's weight-gradient stream and events");
        return IAC_ERR_CUDA;
    }
    cudaMemset(dn->p, 0, off * 4);
    cudaMemset(dn->g, 0, off * 4);
    cudaMemset(dn->m, 0, off * 4);
    cudaMemset(dn->v, 0, off * 4);
    *out = dn;
    return IAC_OK;
}

void iac_denoise_destroy(iac_denoiser *dn)
{
    if (!dn) return;
    DeviceGuard guard(dn->ctx->device);
    cudaDeviceSynchronize();
    delete dn;
}

// He-normal weights (std sqrt(2 / (27 cin))), zero biases, a zero head (the
// network starts as the identity on its input); deterministic in `seed`
iac_status iac_denoise_init_params(iac_denoiser *dn, uint64_t seed)
{
    IAC_REQUIRE(dn, "null denoiser");
    std::vector<float> h((size_t)dn->nparams, 0.0f);
    uint64_t st = seed ^ 0x5DEECE66Dull;
    for (int l = 0; l < NCONV; l++) {
        const long long nw = (long long)SPECS[l].cout * 27 * SPECS[l].cin;
        const double sd = std::sqrt(2.0 / (27.0 * SPECS[l].cin));
        for (long long i = 0; i < nw; i += 2) {
            const double u1 = ((splitmix(st) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
            const double u2 = ((splitmix(st) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
            const double r = std::sqrt(-2.0 * std::log(u1));
            h[dn->p_off[l] + i] = (float)(sd * r * std::cos(6.283185307179586 * u2));
            if (i + 1 < nw) h[dn->p_off[l] + i + 1] = (float)(sd * r * std::sin(6.283185307179586 * u2));
        }
    }
    return iac_denoise_set_params(dn, h.data());
}

iac_status iac_denoise_set_params(iac_denoiser *dn, const float *h_params)
{
    IAC_REQUIRE(dn && h_params, "null argument");
    DeviceGuard guard(dn->ctx->device);
    DN_CHECK(cudaMemcpy(dn->p, h_params, dn->nparams * 4, cudaMemcpyHostToDevice), "set parameters");
    DN_CHECK(cudaMemset(dn->m, 0, dn->nparams * 4), "reset moments");
    DN_CHECK(cudaMemset(dn->v, 0, dn->nparams * 4), "reset moments");
    dn->adam_step = 0;
    iac_status st = refresh_tiles(dn, nullptr, 0);
    if (st != IAC_OK) return st;
    DN_CHECK(cudaDeviceSynchronize(), "set parameters");
    return IAC_OK;
}

iac_status iac_denoise_get_params(iac_denoiser *dn, float *h_params)
{
    IAC_REQUIRE(dn && h_params, "null argument");
    DeviceGuard guard(dn->ctx->device);
    DN_CHECK(cudaDeviceSynchronize(), "get parameters");
    DN_CHECK(cudaMemcpy(h_params, dn->p, dn->nparams * 4, cudaMemcpyDeviceToHost), "get parameters");
    return IAC_OK;
}

iac_status iac_denoise_get_state(iac_denoiser *dn, float *h_m, float *h_v, uint64_t *h_step)
{
    IAC_REQUIRE(dn && h_m && h_v && h_step, "null argument");
    DeviceGuard guard(dn->ctx->device);
    DN_CHECK(cudaDeviceSynchronize(), "get optimizer state");
    DN_CHECK(cudaMemcpy(h_m, dn->m, dn->nparams * 4, cudaMemcpyDeviceToHost), "get first moments");
    DN_CHECK(cudaMemcpy(h_v, dn->v, dn->nparams * 4, cudaMemcpyDeviceToHost), "get second moments");
    *h_step = (uint64_t)dn->adam_step;
    return IAC_OK;
}

iac_status iac_denoise_set_state(iac_denoiser *dn, const float *h_params, const float *h_m, const float *h_v,
                                 uint64_t step)
{
    IAC_REQUIRE(dn && h_params && h_m && h_v, "null argument");
    IAC_REQUIRE(step < (1ull << 62), "optimizer step count %llu out of range", (unsigned long long)step);
    DeviceGuard guard(dn->ctx->device);
    DN_CHECK(cudaMemcpy(dn->p, h_params, dn->nparams * 4, cudaMemcpyHostToDevice), "set parameters");
    DN_CHECK(cudaMemcpy(dn->m, h_m, dn->nparams * 4, cudaMemcpyHostToDevice), "set first moments");
    DN_CHECK(cudaMemcpy(dn->v, h_v, dn->nparams * 4, cudaMemcpyHostToDevice), "set second moments");
    dn->adam_step = (long long)step;
    iac_status st = refresh_tiles(dn, nullptr, 0);
    if (st != IAC_OK) return st;
    DN_CHECK(cudaDeviceSynchronize(), "set optimizer state");
    return IAC_OK;
}

iac_status iac_denoise_get_grads(iac_denoiser *dn, float *h_grads)
{
    IAC_REQUIRE(dn && h_grads, "null argument");
    DeviceGuard guard(dn->ctx->device);
    DN_CHECK(cudaDeviceSynchronize(), "get gradients");
    DN_CHECK(cudaMemcpy(h_grads, dn->g, dn->nparams * 4, cudaMemcpyDeviceToHost), "get gradients");
    return IAC_OK;
}

iac_status iac_denoise_grad_buffer(iac_denoiser *dn, float **d_grads, uint64_t *count)
{
    IAC_REQUIRE(dn && d_grads && count, "null argument");
    *d_grads = dn->g;
    *count = (uint64_t)dn->nparams;
    return IAC_OK;
}

iac_status iac_denoise_forward(iac_denoiser *dn, const float *d_in, uint32_t nb, uint32_t D, uint32_t H,
                               uint32_t W, float *d_out, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(dn && d_in && d_out, "null argument");
    iac_status st = check_dims(dn, nb, D, H, W);
    if (st != IAC_OK) return st;
    DeviceGuard guard(dn->ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    st = run_forward(dn, d_in, nb, D, H, W, s);
    if (st != IAC_OK) return st;
    HeadArgs h{};
    h.x = d_in;
    h.d = dn->d1b;
    h.w = dn->p + dn->p_off[10];
    h.out = d_out;
    h.V = (long long)nb * D * H * W;
    DN_CHECK(head(h, dn->ctx->sm_count, s), "denoiser head");
    dn->ctx->launches += take_launches();
    return IAC_OK;
}

iac_status iac_denoise_backward(iac_denoiser *dn, const float *d_in, const float *d_target, const float *d_weight,
                                uint32_t nb, uint32_t D, uint32_t H, uint32_t W, float *d_out, double *h_loss,
                                void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(dn && d_in && d_target, "null argument");
    iac_status st = check_dims(dn, nb, D, H, W);
    if (st != IAC_OK) return st;
    DeviceGuard guard(dn->ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    DN_CHECK(cudaMemsetAsync(dn->d_loss, 0, 8, s), "clear loss");
    st = run_backward(dn, d_in, d_target, d_weight, nb, D, H, W, d_out, dn->d_loss, nullptr, s);
    dn->ctx->launches += take_launches();
    if (st != IAC_OK) return st;
    if (h_loss) {
        double t = 0;
        DN_CHECK(cudaMemcpyAsync(&t, dn->d_loss, 8, cudaMemcpyDeviceToHost, s), "loss");
        DN_CHECK(cudaStreamSynchronize(s), "loss");
        *h_loss = t / ((double)nb * D * H * W);
    }
    return IAC_OK;
}

iac_status iac_denoise_adamw_step(iac_denoiser *dn, const iac_adamw *opt, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(dn && opt, "null argument");
    IAC_REQUIRE(opt->lr >= 0 && opt->beta1 >= 0 && opt->beta1 < 1 && opt->beta2 >= 0 && opt->beta2 < 1 &&
                    opt->eps > 0,
                "AdamW hyper-parameters out of range");
    DeviceGuard guard(dn->ctx->device);
    const iac_status st = refresh_tiles(dn, opt, (cudaStream_t)stream);
    dn->ctx->launches += take_launches();
    return st;
}

iac_status iac_denoise_train_steps(iac_denoiser *dn, const uint16_t *d_in_meshes, const uint16_t *d_tgt_meshes,
                                   uint32_t nmeshes, uint32_t E, const int32_t *d_plans, const float *d_lrs,
                                   uint32_t nsteps, uint32_t nb, uint32_t P, const iac_adamw *opt, double *d_losses,
                                   void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(dn && d_in_meshes && d_tgt_meshes && d_plans && d_lrs && opt, "null argument");
    IAC_REQUIRE(nsteps >= 1 && nmeshes >= 1 && P >= 4 && P % 4 == 0 && P <= E, "steps %u, meshes %u, patch %u of %u",
                nsteps, nmeshes, P, E);
    IAC_REQUIRE(opt->beta1 >= 0 && opt->beta1 < 1 && opt->beta2 >= 0 && opt->beta2 < 1 && opt->eps > 0,
                "AdamW hyper-parameters out of range");
    iac_status st = check_dims(dn, nb, P, P, P);
    if (st != IAC_OK) return st;
    DeviceGuard guard(dn->ctx->device);
    cudaStream_t caller = (cudaStream_t)stream;
    // the step is captured and replayed on a stream of the denoiser at the highest
    // priority, ordered after and before the caller's work by events: its kernel
    // nodes keep that priority (the chain of data gradients) over the weight
    // gradients' branch, which is captured from the lower-priority side stream
    if (!dn->own_stream) {
        int least = 0, greatest = 0;
        DN_CHECK(cudaDeviceGetStreamPriorityRange(&least, &greatest), "stream priorities");
        DN_CHECK(cudaStreamCreateWithPriority(&dn->own_stream, cudaStreamNonBlocking, greatest), "replay stream");
        DN_CHECK(cudaEventCreateWithFlags(&dn->own_ev[0], cudaEventDisableTiming), "replay event");
        DN_CHECK(cudaEventCreateWithFlags(&dn->own_ev[1], cudaEventDisableTiming), "replay event");
    }
    cudaStream_t s = dn->own_stream;
    DN_CHECK(cudaEventRecord(dn->own_ev[0], caller), "order replay");
    DN_CHECK(cudaStreamWaitEvent(s, dn->own_ev[0], 0), "order replay");
    const size_t vox = (size_t)dn->max_batch * dn->D * dn->H * dn->W;
    if (!dn->px) {
        dn->px = (float *)dn->alloc(vox * 4);
        dn->pt = (float *)dn->alloc(vox * 4);
        IAC_REQUIRE(dn->px && dn->pt, "device memory for the training patches");
    }
    std::vector<uintptr_t> key = {(uintptr_t)d_in_meshes, (uintptr_t)d_tgt_meshes, nmeshes, E,
                                  (uintptr_t)d_plans, (uintptr_t)d_lrs, nb, P, (uintptr_t)d_losses,
                                  (uintptr_t)s};
    const float hp[4] = {opt->beta1, opt->beta2, opt->eps, opt->weight_decay};
    for (float f : hp) {
        uint32_t u;
        std::memcpy(&u, &f, 4);
        key.push_back(u);
    }
    if (!dn->step_exec || key != dn->step_key) {
        if (dn->step_exec) {
            cudaGraphExecDestroy(dn->step_exec);
            dn->step_exec = nullptr;
        }
        // one step, captured once: two patch crops, forward + loss + backward,
        // AdamW (schedule and step count read from device memory), step advance
        DN_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed), "begin capture");
        double *loss = d_losses ? d_losses : dn->d_dummy_loss;
        const long long *step = dn->d_step;
        cudaError_t ce = crop_patches(reinterpret_cast<const bf16 *>(d_in_meshes), (int)nmeshes, (int)E, d_plans,
                                      (int)nb, (int)P, dn->px, dn->ctx->d_counters, s, step);
        if (ce == cudaSuccess)
            ce = crop_patches(reinterpret_cast<const bf16 *>(d_tgt_meshes), (int)nmeshes, (int)E, d_plans, (int)nb,
                              (int)P, dn->pt, dn->ctx->d_counters, s, step);
        if (ce == cudaSuccess) {
            st = run_backward(dn, dn->px, dn->pt, nullptr, nb, P, P, P, nullptr, d_losses ? loss : dn->d_dummy_loss,
                              d_losses ? step : nullptr, s);
            if (st == IAC_OK) st = refresh_tiles(dn, opt, s, step, d_lrs);
            if (st == IAC_OK) ce = step_counter(dn->d_step, 0, 1, s);
        }
        cudaGraph_t graph = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(s, &graph);
        dn->step_launches = take_launches();  // recorded now, launched by every replay
        if (ce != cudaSuccess || st != IAC_OK || ee != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            if (st != IAC_OK) return st;
            DN_CHECK(ce != cudaSuccess ? ce : ee, "capture of the training step");
        }
        const cudaError_t ie = cudaGraphInstantiate(&dn->step_exec, graph, cudaGraphInstantiateFlagUseNodePriority);
        cudaGraphDestroy(graph);
        DN_CHECK(ie, "instantiate the training-step graph");
        dn->step_key = key;
    }
    DN_CHECK(step_counter(dn->d_step, dn->adam_step, 0, s), "reset the step counter");
    if (d_losses) DN_CHECK(cudaMemsetAsync(d_losses, 0, (size_t)nsteps * 8, s), "clear losses");
    for (uint32_t i = 0; i < nsteps; i++) DN_CHECK(cudaGraphLaunch(dn->step_exec, s), "training-step graph");
    DN_CHECK(cudaEventRecord(dn->own_ev[1], s), "order replay");
    DN_CHECK(cudaStreamWaitEvent(caller, dn->own_ev[1], 0), "order replay");
    dn->adam_step += nsteps;
    dn->ctx->launches += (uint64_t)nsteps * dn->step_launches + take_launches();
    return IAC_OK;
}

iac_status iac_denoise_crop_patches(iac_ctx *ctx, const uint16_t *d_meshes, uint32_t nmeshes, uint32_t E,
                                    const int32_t *d_plan, uint32_t nb, uint32_t P, float *d_out, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx && d_meshes && d_plan && d_out, "null argument");
    IAC_REQUIRE(P >= 1 && P <= E, "patch edge %u outside 1..%u", P, E);
    DeviceGuard guard(ctx->device);
    DN_CHECK(crop_patches(reinterpret_cast<const bf16 *>(d_meshes), (int)nmeshes, (int)E, d_plan, (int)nb, (int)P,
                          d_out, ctx->d_counters, (cudaStream_t)stream),
             "crop patches");
    ctx->launches += take_launches();
    return IAC_OK;
}

iac_status iac_denoise_conv3x3(iac_ctx *ctx, int backend, const uint16_t *d_src0, uint32_t c0, int up0,
                               const uint16_t *d_src1, uint32_t c1, const uint16_t *d_wtile, const float *d_bias,
                               uint32_t cout, int relu, uint32_t nb, uint32_t D, uint32_t H, uint32_t W,
                               uint16_t *d_y, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx && d_src1 && d_wtile && d_y && (c0 == 0 || d_src0), "null argument");
    IAC_REQUIRE(backend >= 0 && backend <= 2, "backend %d", backend);
    IAC_REQUIRE(c0 % 16 == 0 && c1 % 8 == 0 && c1 > 0, "channels %u + %u", c0, c1);
    IAC_REQUIRE(D && H && W && nb && (!up0 || (D % 2 == 0 && H % 2 == 0 && W % 2 == 0)), "volume %ux%ux%u", D, H,
                W);
    DeviceGuard guard(ctx->device);
    ConvArgs a{};
    a.src0 = reinterpret_cast<const bf16 *>(d_src0);
    a.src1 = reinterpret_cast<const bf16 *>(d_src1);
    a.c0 = (int)c0;
    a.c1 = (int)c1;
    a.up0 = up0;
    a.w = reinterpret_cast<const bf16 *>(d_wtile);
    a.bias = d_bias;
    a.y = reinterpret_cast<bf16 *>(d_y);
    a.relu = relu;
    a.D = (int)D;
    a.H = (int)H;
    a.W = (int)W;
    a.V = (long long)nb * D * H * W;
    a.counters = ctx->d_counters;
    a.sms = ctx->sm_count;
    const cudaError_t e = conv3x3(a, (int)(c0 + c1), (int)cout, backend, (cudaStream_t)stream);
    IAC_REQUIRE(e != cudaErrorInvalidValue, "no 3x3x3 kernel for %u -> %u channels", c0 + c1, cout);
    DN_CHECK(e, "conv3x3");
    ctx->launches += take_launches();
    return IAC_OK;
}

iac_status iac_denoise_wgrad3x3(iac_ctx *ctx, int slabs, const uint16_t *d_src0, uint32_t c0, int up0,
                                const uint16_t *d_src1, uint32_t c1, const uint16_t *d_grad, uint32_t cout,
                                uint32_t nb, uint32_t D, uint32_t H, uint32_t W, float *d_dw, float *d_db,
                                void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx && d_src1 && d_grad && d_dw && (c0 == 0 || d_src0), "null argument");
    IAC_REQUIRE(D && H && W && nb && (!up0 || (D % 2 == 0 && H % 2 == 0 && W % 2 == 0)), "volume %ux%ux%u", D, H,
                W);
    DeviceGuard guard(ctx->device);
    WgradArgs a{};
    a.src0 = reinterpret_cast<const bf16 *>(d_src0);
    a.src1 = reinterpret_cast<const bf16 *>(d_src1);
    a.c0 = (int)c0;
    a.c1 = (int)c1;
    a.up0 = up0;
    a.g = reinterpret_cast<const bf16 *>(d_grad);
    a.dw = d_dw;
    a.db = d_db;
    a.D = (int)D;
    a.H = (int)H;
    a.W = (int)W;
    a.V = (long long)nb * D * H * W;
    a.cout = (int)cout;
    a.slabs = slabs;
    a.counters = ctx->d_counters;
    const cudaError_t e = wgrad3x3(a, (int)(c0 + c1), ctx->sm_count, (cudaStream_t)stream);
    IAC_REQUIRE(e != cudaErrorInvalidValue, "no 3x3x3 weight-gradient kernel for %u -> %u channels", c0 + c1, cout);
    DN_CHECK(e, "wgrad3x3");
    ctx->launches += take_launches();
    return IAC_OK;
}

iac_status iac_denoise_mesh_input(iac_ctx *ctx, const uint64_t *d_full, uint32_t S, uint32_t E, double scale,
                                  float *d_f32, uint16_t *d_bf16, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx && d_full && (d_f32 || d_bf16), "null argument");
    IAC_REQUIRE(E >= 1 && E <= S, "crop edge %u outside 1..%u", E, S);
    DeviceGuard guard(ctx->device);
    DN_CHECK(mesh_input(d_full, (int)S, (int)E, scale, d_f32, reinterpret_cast<bf16 *>(d_bf16),
                        (cudaStream_t)stream),
             "mesh input");
    ctx->launches += take_launches();
    return IAC_OK;
}

}  // extern "C"
