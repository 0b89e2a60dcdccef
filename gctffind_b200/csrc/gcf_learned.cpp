// gcf_learned.cpp -- the learned initialiser's network state and passes:
// FP32 master parameters with Adam moments, BF16 copies (row-major for the
// forward products, transposed for the input-gradient products), the
// activations of one batch, and the forward / backward / update sequences
// built from the tensor-core product (gcf_umma.cu) and the layer kernels of
// gcf_nn.cu.  Everything runs on the caller's stream; nothing is read back.
//
// Parameter order in the flat FP32 vector (weights [out][in] row-major, then
// the bias), with in = the im2col column order of gcf_nn.cu:
//   conv1 16 x 16, conv2 32 x 144, conv3 32 x 288, conv4 32 x 288,
//   fc1 256 x 2304, fc2 128 x 256, fc3 3 x 128.
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "gcf_internal.h"

namespace gcf {

namespace {

template <class T>
struct Buf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t ensure(size_t cnt)
    {
        if (cnt <= n && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        note_device_alloc();
        cudaError_t e = cudaMalloc((void**)&p, std::max<size_t>(cnt, 1) * sizeof(T));
        if (e == cudaSuccess) n = cnt;
        return e;
    }
    ~Buf()
    {
        if (p) cudaFree(p);
    }
};

struct Layer {
    int out, in;          // weight matrix out x in
    int ldt;              // pitch of the transposed copy (out rounded up to 8)
    size_t off;           // offset of the weights in the flat vector (bias follows)
};

constexpr int kLayers = 7;
const Layer kNet[kLayers] = {
    {16, 16, 16, 0},   {32, 144, 32, 0},   {32, 288, 32, 0}, {32, 288, 32, 0},
    {256, 2304, 256, 0}, {128, 256, 128, 0}, {3, 128, 8, 0},
};

std::vector<Layer> layers()
{
    std::vector<Layer> v(kNet, kNet + kLayers);
    size_t off = 0;
    for (Layer& l : v) {
        l.off = off;
        off += (size_t)l.out * l.in + l.out;
    }
    return v;
}

}  // namespace

struct NnNet {
    std::vector<Layer> L = layers();
    size_t np = 0;
    Buf<float> w, g, m, v;                 // masters, gradients, Adam moments
    Buf<__nv_bfloat16> wb, wt;             // BF16 copies
    std::vector<size_t> wb_off, wt_off;
    int steps = 0;
    int B = 0;
    // activations (BF16) and products (FP32) of one batch
    Buf<__nv_bfloat16> cols1, y1, cols2, y2, cols3, y3, cols4, y4, h0, h1, h2, dpred;
    Buf<float> pred, fbuf;                 // predictions; FP32 product scratch
    Buf<__nv_bfloat16> dz_a, dz_b;         // BF16 gradients of the current layer
    Buf<int> err;
    const __nv_bfloat16* x1 = nullptr;     // inputs of the last forward
    const __nv_bfloat16* x2 = nullptr;
};

size_t nn_param_count()
{
    size_t n = 0;
    for (const Layer& l : layers()) n += (size_t)l.out * l.in + l.out;
    return n;
}

NnNet* nn_create()
{
    NnNet* n = new NnNet();
    n->np = nn_param_count();
    size_t ob = 0, ot = 0;
    for (const Layer& l : n->L) {
        n->wb_off.push_back(ob);
        n->wt_off.push_back(ot);
        ob += ((size_t)l.out * l.in + 7) / 8 * 8;
        ot += ((size_t)l.in * l.ldt + 7) / 8 * 8;
    }
    if (n->w.ensure(n->np) != cudaSuccess || n->g.ensure(n->np) != cudaSuccess ||
        n->m.ensure(n->np) != cudaSuccess || n->v.ensure(n->np) != cudaSuccess || n->wb.ensure(ob) != cudaSuccess ||
        n->wt.ensure(ot) != cudaSuccess || n->err.ensure(1) != cudaSuccess) {
        delete n;
        return nullptr;
    }
    cudaMemset(n->wt.p, 0, ot * sizeof(__nv_bfloat16));
    cudaMemset(n->m.p, 0, n->np * sizeof(float));
    cudaMemset(n->v.p, 0, n->np * sizeof(float));
    cudaMemset(n->g.p, 0, n->np * sizeof(float));
    cudaMemset(n->err.p, 0, sizeof(int));
    cudaDeviceSynchronize();
    return n;
}

void nn_destroy(NnNet* n) { delete n; }

int* nn_err_flag(NnNet* n) { return n->err.p; }

const float* nn_pred(NnNet* n) { return n->pred.p; }

static cudaError_t refresh_copies(NnNet* n, cudaStream_t st)
{
    for (size_t i = 0; i < n->L.size(); ++i) {
        const Layer& l = n->L[i];
        launch_copy_weights(n->w.p + l.off, l.out, l.in, n->wb.p + n->wb_off[i], n->wt.p + n->wt_off[i], l.ldt, st);
    }
    return cudaGetLastError();
}

cudaError_t nn_set_params(NnNet* n, const float* host, cudaStream_t st)
{
    cudaError_t e = cudaMemcpyAsync(n->w.p, host, n->np * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(n->m.p, 0, n->np * sizeof(float), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(n->v.p, 0, n->np * sizeof(float), st)) != cudaSuccess) return e;
    n->steps = 0;
    e = refresh_copies(n, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);   // the host buffer may go away after return
}

cudaError_t nn_get_params(NnNet* n, float* host, cudaStream_t st)
{
    cudaError_t e = cudaMemcpyAsync(host, n->w.p, n->np * sizeof(float), cudaMemcpyDeviceToHost, st);
    return e != cudaSuccess ? e : cudaStreamSynchronize(st);
}

cudaError_t nn_get_grads(NnNet* n, float* host, cudaStream_t st)
{
    cudaError_t e = cudaMemcpyAsync(host, n->g.p, n->np * sizeof(float), cudaMemcpyDeviceToHost, st);
    return e != cudaSuccess ? e : cudaStreamSynchronize(st);
}

cudaError_t nn_init_random(NnNet* n, unsigned long long seed, cudaStream_t st)
{
    // He-normal: N(0, 2 / fan_in); biases 0.  Drawn on the host (a one-off
    // of 0.65 M numbers).
    std::vector<float> h(n->np, 0.0f);
    std::mt19937_64 rng(seed);
    for (const Layer& l : n->L) {
        std::normal_distribution<float> d(0.0f, std::sqrt(2.0f / (float)l.in));
        for (size_t i = 0; i < (size_t)l.out * l.in; ++i) h[l.off + i] = d(rng);
    }
    return nn_set_params(n, h.data(), st);
}

static cudaError_t ensure_batch(NnNet* n, int B)
{
    if (B <= n->B) return cudaSuccess;
    cudaError_t e;
#define EN(buf, cnt)                                         \
    if ((e = n->buf.ensure((size_t)(cnt))) != cudaSuccess) return e
    EN(cols1, (size_t)B * 4096 * 16);
    EN(y1, (size_t)B * 4096 * 16);
    EN(cols2, (size_t)B * 1024 * 144);
    EN(y2, (size_t)B * 1024 * 32);
    EN(cols3, (size_t)B * 256 * 288);
    EN(y3, (size_t)B * 256 * 32);
    EN(cols4, (size_t)B * 64 * 288);
    EN(y4, (size_t)B * 64 * 32);
    EN(h0, (size_t)B * 2304);
    EN(h1, (size_t)B * 256);
    EN(h2, (size_t)B * 128);
    EN(dpred, (size_t)B * 8);
    EN(pred, (size_t)B * kNnPredPitch);
    EN(fbuf, (size_t)B * 4096 * 16 > (size_t)B * 1024 * 144 ? (size_t)B * 4096 * 16 : (size_t)B * 1024 * 144);
    EN(dz_a, (size_t)B * 4096 * 16);
    EN(dz_b, (size_t)B * 4096 * 16);
#undef EN
    n->B = B;
    return cudaSuccess;
}

// One layer's product: out[rows][l.out] = act(in[rows][l.in] W^T + b).
static cudaError_t layer_fwd(NnNet* n, int li, const __nv_bfloat16* in, int rows, __nv_bfloat16* out_b,
                             float* out_f, long long ldo, bool relu, cudaStream_t st)
{
    const Layer& l = n->L[li];
    GemmArgs g;
    g.M = rows;
    g.N = l.out;
    g.K = l.in;
    g.D = out_f;
    g.Db = out_b;
    g.ldd = ldo;
    g.bias = n->w.p + l.off + (size_t)l.out * l.in;
    g.relu = relu ? 1 : 0;
    g.err = n->err.p;
    // Tile width: the layer's width, narrowed while the product would have
    // fewer than 64 tiles (the MLP's few batch rows would otherwise run on a
    // couple of CTAs); every output element sums the same products in the
    // same order whatever the tile.  Layers of many tiles (the convolutions'
    // im2col rows) take the persistent kernel, one CTA per SM, whose
    // epilogue of one tile overlaps the products of the next.
    const int mt = (rows + 127) / 128;
    int bn = l.out <= 32 ? 32 : (l.out <= 64 ? 64 : (l.out <= 128 ? 128 : 256));
    while (bn > 32 && mt * ((l.out + bn - 1) / bn) < 64) bn /= 2;
    const int stages = bn == 256 ? 3 : 4;
    const __nv_bfloat16* w = n->wb.p + n->wb_off[li];
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    if (mt * ((l.out + bn - 1) / bn) > 2 * sms)
        return launch_umma_gemm_persistent(in, l.in, w, l.in, g, bn, stages, 0, st);
    return launch_umma_gemm(in, l.in, w, l.in, g, bn, stages, 0, st);
}

cudaError_t nn_forward(NnNet* n, const __nv_bfloat16* x1, const __nv_bfloat16* x2, int B, cudaStream_t st)
{
    cudaError_t e = ensure_batch(n, B);
    if (e != cudaSuccess) return e;
    n->x1 = x1;
    n->x2 = x2;
    // the first layer (K = N = 16) on CUDA cores: as a tensor-core product of
    // im2col rows its tiles are too small to keep the pipeline busy
    launch_conv1_direct(x2, B, n->wb.p + n->wb_off[0], n->w.p + n->L[0].off + (size_t)n->L[0].out * n->L[0].in,
                        n->y1.p, st);
    launch_im2col_3s2(n->y1.p, B, 64, 64, 16, n->cols2.p, st);
    if ((e = layer_fwd(n, 1, n->cols2.p, B * 1024, n->y2.p, nullptr, 32, true, st)) != cudaSuccess) return e;
    launch_im2col_3s2(n->y2.p, B, 32, 32, 32, n->cols3.p, st);
    if ((e = layer_fwd(n, 2, n->cols3.p, B * 256, n->y3.p, nullptr, 32, true, st)) != cudaSuccess) return e;
    launch_im2col_3s2(n->y3.p, B, 16, 16, 32, n->cols4.p, st);
    if ((e = layer_fwd(n, 3, n->cols4.p, B * 64, n->y4.p, nullptr, 32, true, st)) != cudaSuccess) return e;
    launch_concat(x1, n->y4.p, B, n->h0.p, st);
    if ((e = layer_fwd(n, 4, n->h0.p, B, n->h1.p, nullptr, 256, true, st)) != cudaSuccess) return e;
    if ((e = layer_fwd(n, 5, n->h1.p, B, n->h2.p, nullptr, 128, true, st)) != cudaSuccess) return e;
    if ((e = layer_fwd(n, 6, n->h2.p, B, nullptr, n->pred.p, kNnPredPitch, false, st)) != cudaSuccess) return e;
    return cudaGetLastError();
}

// d_in[rows][l.in] (FP32) = dz[rows][l.out] W, through the transposed copy.
static cudaError_t layer_dx(NnNet* n, int li, const __nv_bfloat16* dz, long long ldz, int rows, float* dx,
                            cudaStream_t st)
{
    const Layer& l = n->L[li];
    GemmArgs g;
    g.M = rows;
    g.N = l.in;
    g.K = l.out;
    g.D = dx;
    g.ldd = l.in;
    g.err = n->err.p;
    const int bn = l.in <= 32 ? 32 : (l.in <= 64 ? 64 : (l.in <= 128 ? 128 : 256));
    return launch_umma_gemm(dz, ldz, n->wt.p + n->wt_off[li], l.ldt, g, bn, bn == 256 ? 3 : 4, 0, st);
}

static void layer_dw(NnNet* n, int li, const __nv_bfloat16* dz, long long ldz, const __nv_bfloat16* in, int rows,
                     cudaStream_t st)
{
    const Layer& l = n->L[li];
    float* dw = n->g.p + l.off;
    launch_wgrad(dz, ldz, in, l.in, rows, l.out, l.in, dw, dw + (size_t)l.out * l.in, st);
}

cudaError_t nn_backward(NnNet* n, const float* target, int B, float* loss, cudaStream_t st)
{
    if (B > n->B) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(n->g.p, 0, n->np * sizeof(float), st);
    if (e != cudaSuccess) return e;
    launch_mse(n->pred.p, kNnPredPitch, target, B, loss, n->dpred.p, st);
    // fc3 (linear): dz = dpred
    layer_dw(n, 6, n->dpred.p, 8, n->h2.p, B, st);
    if ((e = layer_dx(n, 6, n->dpred.p, 8, B, n->fbuf.p, st)) != cudaSuccess) return e;
    launch_relu_bwd(n->fbuf.p, 128, n->h2.p, 128, B, 128, n->dz_a.p, 128, st);
    // fc2
    layer_dw(n, 5, n->dz_a.p, 128, n->h1.p, B, st);
    if ((e = layer_dx(n, 5, n->dz_a.p, 128, B, n->fbuf.p, st)) != cudaSuccess) return e;
    launch_relu_bwd(n->fbuf.p, 256, n->h1.p, 256, B, 256, n->dz_b.p, 256, st);
    // fc1: the input gradient of its conv4 part only (the profile is an input)
    layer_dw(n, 4, n->dz_b.p, 256, n->h0.p, B, st);
    if ((e = layer_dx(n, 4, n->dz_b.p, 256, B, n->fbuf.p, st)) != cudaSuccess) return e;
    launch_relu_bwd(n->fbuf.p + 256, 2304, n->y4.p, 2048, B, 2048, n->dz_a.p, 2048, st);
    // conv4: dz_a is [B*64][32]
    layer_dw(n, 3, n->dz_a.p, 32, n->cols4.p, B * 64, st);
    if ((e = layer_dx(n, 3, n->dz_a.p, 32, B * 64, n->fbuf.p, st)) != cudaSuccess) return e;
    launch_col2im_3s2_relu(n->fbuf.p, n->y3.p, B, 16, 16, 32, n->dz_b.p, st);
    // conv3
    layer_dw(n, 2, n->dz_b.p, 32, n->cols3.p, B * 256, st);
    if ((e = layer_dx(n, 2, n->dz_b.p, 32, B * 256, n->fbuf.p, st)) != cudaSuccess) return e;
    launch_col2im_3s2_relu(n->fbuf.p, n->y2.p, B, 32, 32, 32, n->dz_a.p, st);
    // conv2
    layer_dw(n, 1, n->dz_a.p, 32, n->cols2.p, B * 1024, st);
    if ((e = layer_dx(n, 1, n->dz_a.p, 32, B * 1024, n->fbuf.p, st)) != cudaSuccess) return e;
    launch_col2im_3s2_relu(n->fbuf.p, n->y1.p, B, 64, 64, 16, n->dz_b.p, st);
    // conv1 (its input needs no gradient): its im2col rows for the weight
    // gradient (the forward reads the input directly)
    launch_im2col_p4(n->x2, B, n->cols1.p, st);
    layer_dw(n, 0, n->dz_b.p, 16, n->cols1.p, B * 4096, st);
    return cudaGetLastError();
}

cudaError_t nn_adam(NnNet* n, float lr, cudaStream_t st)
{
    n->steps += 1;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.0f - std::pow(b1, (float)n->steps), c2 = 1.0f - std::pow(b2, (float)n->steps);
    for (size_t i = 0; i < n->L.size(); ++i) {
        const Layer& l = n->L[i];
        const int cnt = l.out * l.in + l.out;
        launch_adam(n->w.p + l.off, n->g.p + l.off, n->m.p + l.off, n->v.p + l.off, cnt, lr, b1, b2, eps, c1, c2,
                    l.out, l.in, n->wb.p + n->wb_off[i], n->wt.p + n->wt_off[i], l.ldt, st);
    }
    return cudaGetLastError();
}

}  // namespace gcf
