// denoise_internal.cuh -- shared declarations of the mesh denoiser's kernels
// (a 3-level 3D U-Net, channels 16/32/64, 3x3x3 convolutions) and its host
// runtime.  The denoiser has no counterpart in the reference: it maps a
// few-frame pair-correlation mesh to an estimate of its many-frame mean.
//
// Tensors are NDHWC bf16 with the batch folded into the voxel index
// v = ((n*D + z)*H + y)*W + x.  Weights of a 3x3x3 layer are kept in fp32
// (master copy, [cout][27][cin] + bias[cout]) and in two bf16 copies laid out
// as the implicit-GEMM B tiles are staged in shared memory:
//   forward  Wf[tap][cin/8][cout][8]     (K-major rows of 8 input channels)
//   data-grad Wd[tap][cout/8][cin][8]    with Wd(tap) = Wf(26 - tap)^T
// so every tap's tile is one contiguous block.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "iac_internal.cuh"

namespace iac {
namespace dn {

typedef __nv_bfloat16 bf16;

constexpr int TILE_M = 128;  // voxels per CTA tile (GEMM M)
constexpr int CONV_THREADS = 128;

// 3x3x3 convolution as implicit GEMM: Y[v][co] = sum_{tap,ci} X[v+off(tap)][ci] W[co][tap][ci].
// The input X is the channel concatenation of src0 (c0 channels, nearest
// 2x-upsampled from half resolution when up0) and src1 (c1 channels).
struct ConvArgs {
    const bf16 *src0;
    const bf16 *src1;
    int c0, c1, up0;
    const bf16 *w;       // tiled B operand, [27][cin/8][cout][8]
    const float *bias;   // [cout] or null
    bf16 *y;             // [V][cout]
    float *y32;          // optional fp32 copy of the output
    int relu;
    const bf16 *mask_y;  // optional [V][cout]: outputs where mask_y <= 0 are set to 0 (ReLU derivative)
    // optional split output: channels split .. cout - 1 go to y2 ([V][cout - split]), the
    // first split channels to y ([V][split]) - the decoder input's gradient, coarse and skip parts
    bf16 *y2;
    int split;
    int D, H, W;         // output (= src1) dims per batch item
    long long V;         // nb * D * H * W
    DeviceCounters *counters;
    int sms;             // SMs of the device (persistent grids)
};

// backends of conv3x3
constexpr int BACKEND_TC_SLAB = 0;  // tcgen05, padded-row slabs, persistent (default)
constexpr int BACKEND_MMA = 1;      // mma.sync.m16n8k16
constexpr int BACKEND_TC_TAP = 2;   // tcgen05, one gathered tile per tap

// dW[co][tap][ci] += sum_v G[v][co] X[v+off(tap)][ci], dB[co] += sum_v G[v][co]
struct WgradArgs {
    const bf16 *src0;
    const bf16 *src1;
    int c0, c1, up0;
    const bf16 *g;       // [V][cout]
    float *dw;           // [cout][27][cin] fp32
    float *db;           // [cout] fp32 or null
    int D, H, W;
    long long V;
    int cout;
    int slabs;           // 2: tcgen05 + TMA, 1: slab kernel (mma.sync), 0: one gathered tile per tap
    DeviceCounters *counters;
};

// kernels launched by the calling host thread since the previous call (every
// launch helper below counts its launches)
uint64_t take_launches();

// kernels (denoise_kernels.cu)
cudaError_t conv3x3(const ConvArgs &a, int cin, int cout, int backend, cudaStream_t s);
cudaError_t conv3x3_first(const float *x, const bf16 *w, const float *bias, bf16 *y, int D, int H,
                          int W, long long V, cudaStream_t s);
cudaError_t wgrad3x3(const WgradArgs &a, int cin, int sms, cudaStream_t s);
cudaError_t wgrad3x3_first(const float *x, const bf16 *g, float *dw, float *db, int D, int H, int W,
                           long long V, int sms, cudaStream_t s);
cudaError_t avgpool2(const bf16 *x, int x_stride, bf16 *y, int C, int D, int H, int W, int nb, cudaStream_t s);
cudaError_t relu_mask(const bf16 *g, const bf16 *y, bf16 *out, long long n, cudaStream_t s);
cudaError_t split_concat_grad(const bf16 *gup, int c0, const bf16 *y0, bf16 *g0, int D, int H, int W, int nb,
                              cudaStream_t s);
cudaError_t concat_up(const bf16 *src0, int c0, const bf16 *src1, int c1, bf16 *cat, int D, int H, int W, int nb,
                      cudaStream_t s);
cudaError_t pool_grad_mask(const bf16 *gskip, int gskip_stride, const bf16 *gpool, const bf16 *y, int y_stride,
                           bf16 *out, int C, int D, int H, int W, int nb, cudaStream_t s);

struct HeadArgs {
    const float *x;       // network input (residual), [V]
    const bf16 *d;        // last decoder activation, [V][16]
    const float *w;       // head weights [16] + bias [1] (fp32 master)
    const float *target;  // [V] or null (inference)
    float *out;           // [V] or null
    bf16 *gd;             // d(loss)/d(pre-activation of d), [V][16] (training)
    float *dw;            // head weight grads [17]
    double *loss;         // sum of squared errors (training); + d_step[0] when d_step is set
    const long long *d_step;  // graph replay: d_step[0] = step index
    const float *weight;  // optional per-voxel loss weight [V]
    long long V;
    double inv_count;     // 1 / (number of voxels in the loss)
};
cudaError_t head(const HeadArgs &a, int sms, cudaStream_t s);

struct AdamLayer {
    long long off;  // offset of the layer's weights in the flat parameter array
    int cout, cin, taps;  // taps = 27 for 3x3x3 layers, 0 for the head
    long long wf_off, wd_off;  // offsets of the bf16 tiles (elements)
};
constexpr int MAX_LAYERS = 16;
struct AdamArgs {
    float *p, *g, *m, *v;
    long long n;
    float lr, beta1, beta2, eps, weight_decay;
    float bc1, bc2;  // 1 - beta^t
    bf16 *wf, *wd;
    AdamLayer layers[MAX_LAYERS];
    int nlayers;
    int update;  // 0: only refresh the bf16 tiles from p
    const long long *d_step;  // graph replay: lr = lrs[d_step[0]], bias corrections of step d_step[1] + 1
    const float *lrs;
};
cudaError_t adamw(const AdamArgs &a, cudaStream_t s);

cudaError_t mesh_input(const uint64_t *full, int S, int E, double scale, float *o32, bf16 *o16, cudaStream_t s);
cudaError_t crop_patches(const bf16 *meshes, int nmesh, int E, const int *plan, int nb, int P, float *out,
                         DeviceCounters *counters, cudaStream_t s, const long long *d_step = nullptr);
cudaError_t step_counter(long long *d_step, long long set_opt, int advance, cudaStream_t s);

}  // namespace dn
}  // namespace iac
