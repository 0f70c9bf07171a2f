// The learned initial guess: a BF16 U-Net whose convolutions, pooling,
// upsampling, loss and Adam update are this library's own kernels. The
// convolutions' forward pass and input gradient run on the tcgen05 tensor
// cores (conv_tc.cu: implicit GEMM, operands staged by TMA, FP32 accumulators
// in tensor memory); the input gradient is the forward convolution of the
// output gradient with the flipped, transposed weights, which are the forward
// weights W[tap][Cin][Cout] read with the taps reversed. The weight gradient
// is a GEMM over the pixels on mma.sync tensor-core instructions (BF16 in,
// FP32 accumulate). Activations are NHWC with channel counts padded to
// multiples of 16.
#include <cuda_bf16.h>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <new>
#include <random>
#include <vector>
#include "incrmt_unet.h"
#include "common.cuh"
#include "conv_tc.cuh"

namespace incrmt {

using bf16 = __nv_bfloat16;

namespace {

constexpr int kBiasSplits = 64;  // pixel ranges of the bias gradient's partial sums

/** Partial bias gradients: partial[split][c] = sum of dY[p][c] over the
 * pixels of split blockIdx.x (every eighth pixel per thread row, then a
 * fixed-order sum over the eight rows), channels blockIdx.y*32 .. +31. */
__global__ void k_bias_partial(const bf16 *dY, float *partial, long P, int C) {
    __shared__ float red[8][33];
    const int c = blockIdx.y * 32 + (threadIdx.x & 31), r = threadIdx.x >> 5;
    const long per = (P + gridDim.x - 1) / gridDim.x;
    const long p0 = blockIdx.x * per, p1 = p0 + per < P ? p0 + per : P;
    float s = 0;
    if (c < C)
        for (long p = p0 + r; p < p1; p += 8) s += __bfloat162float(dY[p * C + c]);
    red[r][threadIdx.x & 31] = s;
    __syncthreads();
    if (r == 0 && c < C) {
        float t = 0;
        for (int q = 0; q < 8; q++) t += red[q][threadIdx.x & 31];
        partial[static_cast<long>(blockIdx.x) * C + c] = t;
    }
}

/** db[c] += the splits' partials in split order. */
__global__ void k_bias_reduce(const float *partial, int splits, int C, float *db) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
        float t = 0;
        for (int sp = 0; sp < splits; sp++) t += partial[static_cast<long>(sp) * C + c];
        db[c] += t;
    }
}

// The elementwise kernels below move eight channels (16 bytes) per thread:
// every channel count of the network is a multiple of 16.

__device__ __forceinline__ uint4 ld8(const bf16 *p) { return *reinterpret_cast<const uint4 *>(p); }
__device__ __forceinline__ void st8(bf16 *p, uint4 v) { *reinterpret_cast<uint4 *>(p) = v; }
__device__ __forceinline__ float bfe(const uint4 &v, int k) {
    const uint32_t w = k < 2 ? v.x : k < 4 ? v.y : k < 6 ? v.z : v.w;
    return __uint_as_float((k & 1) ? (w & 0xFFFF0000u) : (w << 16));
}
__device__ __forceinline__ uint32_t pack2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&h);
}
__device__ __forceinline__ uint4 pack8(const float (&f)[8]) {
    return make_uint4(pack2(f[0], f[1]), pack2(f[2], f[3]), pack2(f[4], f[5]), pack2(f[6], f[7]));
}

/** Gradient through the ReLU: zero where the layer's output is not positive. */
__global__ void k_relu_mask(bf16 *dY, const bf16 *Y, long n) {
    const long n8 = n >> 3;
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n8;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        const uint4 y = ld8(Y + 8 * i);
        uint4 d = ld8(dY + 8 * i);
        uint32_t *dw = reinterpret_cast<uint32_t *>(&d);
#pragma unroll
        for (int k = 0; k < 8; k++)
            if (!(bfe(y, k) > 0.f)) dw[k >> 1] &= (k & 1) ? 0x0000FFFFu : 0xFFFF0000u;
        st8(dY + 8 * i, d);
    }
}

/** 2x2 average pooling, NHWC. */
__global__ void k_pool(const bf16 *X, bf16 *Y, int B, int H, int W, int C) {
    const int Ho = H / 2, Wo = W / 2, C8 = C >> 3;
    const long n = static_cast<long>(B) * Ho * Wo * C8;
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        const int c8 = static_cast<int>(i % C8);
        long r = i / C8;
        const int x = static_cast<int>(r % Wo);
        r /= Wo;
        const int y = static_cast<int>(r % Ho), b = static_cast<int>(r / Ho);
        const long q = ((static_cast<long>(b) * H + 2 * y) * W + 2 * x) * C + 8 * c8;
        const uint4 v0 = ld8(X + q), v1 = ld8(X + q + C), v2 = ld8(X + q + static_cast<long>(W) * C),
                    v3 = ld8(X + q + static_cast<long>(W) * C + C);
        float f[8];
#pragma unroll
        for (int k = 0; k < 8; k++) f[k] = 0.25f * (bfe(v0, k) + bfe(v1, k) + bfe(v2, k) + bfe(v3, k));
        st8(Y + 8 * i, pack8(f));
    }
}

/** Pooling gradient added into dX (which already holds the skip gradient). */
__global__ void k_pool_bwd_add(const bf16 *dY, bf16 *dX, int B, int H, int W, int C) {
    const int C8 = C >> 3;
    const long n = static_cast<long>(B) * H * W * C8;
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        const int c8 = static_cast<int>(i % C8);
        long r = i / C8;
        const int x = static_cast<int>(r % W);
        r /= W;
        const int y = static_cast<int>(r % H), b = static_cast<int>(r / H);
        const long q = ((static_cast<long>(b) * (H / 2) + y / 2) * (W / 2) + x / 2) * C + 8 * c8;
        const uint4 g = ld8(dY + q), d = ld8(dX + 8 * i);
        float f[8];
#pragma unroll
        for (int k = 0; k < 8; k++) f[k] = bfe(d, k) + 0.25f * bfe(g, k);
        st8(dX + 8 * i, pack8(f));
    }
}

/** U = [nearest 2x upsample of L (Cl channels), S (Cs channels)], NHWC. */
__global__ void k_upcat(const bf16 *L, const bf16 *S, bf16 *U, int B, int H, int W, int Cl, int Cs) {
    const int C8 = (Cl + Cs) >> 3, L8 = Cl >> 3;
    const long n = static_cast<long>(B) * H * W * C8;
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        const int c8 = static_cast<int>(i % C8);
        const long pix = i / C8;
        if (c8 < L8) {
            const int x = static_cast<int>(pix % W);
            const long r = pix / W;
            const int y = static_cast<int>(r % H), b = static_cast<int>(r / H);
            st8(U + 8 * i, ld8(L + ((static_cast<long>(b) * (H / 2) + y / 2) * (W / 2) + x / 2) * Cl + 8 * c8));
        } else {
            st8(U + 8 * i, ld8(S + pix * Cs + 8 * (c8 - L8)));
        }
    }
}

/** Gradients of k_upcat: dL summed over the four children, dS written. */
__global__ void k_upcat_bwd(const bf16 *dU, bf16 *dL, bf16 *dS, int B, int H, int W, int Cl, int Cs) {
    const int C = Cl + Cs, L8 = Cl >> 3, S8 = Cs >> 3;
    const long nl = static_cast<long>(B) * (H / 2) * (W / 2) * L8;
    const long ns = static_cast<long>(B) * H * W * S8;
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < nl + ns;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        if (i < nl) {
            const int c8 = static_cast<int>(i % L8);
            long r = i / L8;
            const int x = static_cast<int>(r % (W / 2));
            r /= (W / 2);
            const int y = static_cast<int>(r % (H / 2)), b = static_cast<int>(r / (H / 2));
            float f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int d = 0; d < 4; d++) {
                const long pix = (static_cast<long>(b) * H + 2 * y + (d >> 1)) * W + 2 * x + (d & 1);
                const uint4 v = ld8(dU + pix * C + 8 * c8);
#pragma unroll
                for (int k = 0; k < 8; k++) f[k] += bfe(v, k);
            }
            st8(dL + 8 * i, pack8(f));
        } else {
            const long k = i - nl, pix = k / S8;
            const int c8 = static_cast<int>(k - pix * S8);
            st8(dS + 8 * k, ld8(dU + pix * C + Cl + 8 * c8));
        }
    }
}

/** Network input: 3 FP32 channels into a 16-channel BF16 tensor (rest zero). */
__global__ void k_pack_input(const float *in, bf16 *X, long P) {
    for (long p = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; p < P;
         p += static_cast<long>(gridDim.x) * blockDim.x) {
        const float f[8] = {in[p * 3], in[p * 3 + 1], in[p * 3 + 2], 0.f, 0.f, 0.f, 0.f, 0.f};
        st8(X + 16 * p, pack8(f));
        st8(X + 16 * p + 8, make_uint4(0, 0, 0, 0));
    }
}

/** Output channel 0 of the head as FP32. */
__global__ void k_unpack_output(const bf16 *Y, float *out, long P) {
    for (long p = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; p < P;
         p += static_cast<long>(gridDim.x) * blockDim.x)
        out[p] = __bfloat162float(Y[p * 16]);
}

/** Masked squared error: sums[0] += sum v (o-t)^2, sums[1] += sum v; and the
 * head's output gradient (channel 0; other channels zero), scaled by 2/N
 * with N taken from nvalid. */
__global__ void k_loss(const bf16 *Y, const float *t, const float *valid, long P, double *sums) {
    double s = 0, w = 0;
    for (long p = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; p < P;
         p += static_cast<long>(gridDim.x) * blockDim.x) {
        const float d = __bfloat162float(Y[p * 16]) - t[p];
        s += valid[p] * d * d;
        w += valid[p];
    }
    s = block_sum_256(s);
    __syncthreads();
    w = block_sum_256(w);
    if (threadIdx.x == 0) { atomicAdd(&sums[0], s); atomicAdd(&sums[1], w); }
}

__global__ void k_loss_grad(const bf16 *Y, const float *t, const float *valid, long P, const double *sums, bf16 *dY) {
    const float scale = static_cast<float>(2.0 / (sums[1] > 0 ? sums[1] : 1.0));
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < P * 16;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        const long p = i >> 4;
        float g = 0;
        if ((i & 15) == 0) g = scale * valid[p] * (__bfloat162float(Y[i]) - t[p]);
        dY[i] = __float2bfloat16(g);
    }
}

/** Adam (FP32 master parameters), then the BF16 copies of the weights. */
__global__ void k_adam(float *w, const float *g, float *m, float *v, long n, float lr, float b1, float b2,
                       float c1, float c2, float eps) {
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1 - b1) * gi, vi = b2 * v[i] + (1 - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

/** BF16 weights of one convolution, W[tap][ci][co] (the K-major operand of
 * the input gradient, taps reversed), and its transpose Wt[tap][co][ci] (the
 * K-major operand of the forward pass). */
__global__ void k_weights_bf16(const float *w, bf16 *wb, bf16 *wt, int taps, int Cin, int Cout) {
    const long n = static_cast<long>(taps) * Cin * Cout;
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        const int co = static_cast<int>(i % Cout);
        const long r = i / Cout;
        const int ci = static_cast<int>(r % Cin), tap = static_cast<int>(r / Cin);
        const bf16 v = __float2bfloat16(w[i]);
        wb[i] = v;
        wt[(static_cast<long>(tap) * Cout + co) * Cin + ci] = v;
    }
}

struct Conv {
    int cin, cout, taps;
    bool relu;
    long woff, boff;  // offsets of weights [tap][cin][cout] and biases in the parameter vector
    bf16 *w = nullptr, *wt = nullptr;
};

/** One activation tensor of the forward pass and its gradient. */
struct Act {
    int level, C;
    bf16 *x = nullptr, *g = nullptr;
};

inline int gs(long n) {
    // up to eight 256-thread blocks per SM (all the threads an SM holds), so
    // that the grid-stride loops keep enough loads in flight
    long b = (n + 255) / 256;
    return static_cast<int>(b < 8L * kB200SMs ? (b > 0 ? b : 1) : 8L * kB200SMs);
}

}  // namespace

struct UNet {
    int levels = 4, base = 16;
    std::vector<Conv> convs;
    long nparams = 0;
    float *params = nullptr, *grads = nullptr, *m1 = nullptr, *m2 = nullptr;
    bf16 *wpool = nullptr;
    long adam_t = 0;
    long long launches = 0;
    // Workspace for the current (batch, H, W).
    int wb = 0, wh = 0, ww = 0;
    long long gen = 0;  // activation (re)allocations so far
    std::vector<Act> acts;
    std::vector<void *> work;
    float *part = nullptr;  // weight- and bias-gradient partials
    size_t part_n = 0;
    double *sums = nullptr;

    int C(int l) const { return base << l; }

    int create(int L, int b, unsigned long long seed) {
        levels = L;
        base = b;
        auto add = [&](int cin, int cout, int taps, bool relu) {
            Conv c;
            c.cin = cin; c.cout = cout; c.taps = taps; c.relu = relu;
            c.woff = nparams;
            nparams += static_cast<long>(taps) * cin * cout;
            c.boff = nparams;
            nparams += cout;
            convs.push_back(c);
        };
        // Encoder, bottleneck, decoder, head (the order of the forward pass).
        add(16, C(0), 9, true);
        add(C(0), C(0), 9, true);
        for (int l = 1; l < L; l++) {
            add(C(l - 1), C(l), 9, true);
            add(C(l), C(l), 9, true);
        }
        for (int l = L - 2; l >= 0; l--) {
            add(C(l + 1) + C(l), C(l), 9, true);
            add(C(l), C(l), 9, true);
        }
        add(C(0), 16, 1, false);
        INCRMT_CK(cudaMalloc(&params, sizeof(float) * nparams));
        INCRMT_CK(cudaMalloc(&grads, sizeof(float) * nparams));
        INCRMT_CK(cudaMalloc(&m1, sizeof(float) * nparams));
        INCRMT_CK(cudaMalloc(&m2, sizeof(float) * nparams));
        INCRMT_CK(cudaMemset(m1, 0, sizeof(float) * nparams));
        INCRMT_CK(cudaMemset(m2, 0, sizeof(float) * nparams));
        INCRMT_CK(cudaMalloc(&sums, sizeof(double) * 2));
        long nw = 0;
        for (auto &c : convs) nw += static_cast<long>(c.taps) * c.cin * c.cout;
        INCRMT_CK(cudaMalloc(&wpool, sizeof(bf16) * 2 * nw));
        long o = 0;
        for (auto &c : convs) {
            const long n = static_cast<long>(c.taps) * c.cin * c.cout;
            c.w = wpool + o;
            c.wt = wpool + o + n;
            o += 2 * n;
        }
        // He-uniform weights over the real fan-in (3 input channels in the first
        // layer, the rest being zero padding), zero biases; padded output
        // channels of the head start at zero.
        std::vector<float> h(nparams, 0.f);
        std::mt19937_64 rng(seed);
        for (size_t k = 0; k < convs.size(); k++) {
            const Conv &c = convs[k];
            const int cin_real = k == 0 ? 3 : c.cin;
            const float bound = std::sqrt(6.f / (c.taps * cin_real));
            std::uniform_real_distribution<float> U(-bound, bound);
            for (int tap = 0; tap < c.taps; tap++)
                for (int ci = 0; ci < c.cin; ci++)
                    for (int co = 0; co < c.cout; co++) {
                        const float v = U(rng);
                        const bool live = (k != 0 || ci < 3) && (k + 1 != convs.size() || co == 0);
                        h[c.woff + (static_cast<long>(tap) * c.cin + ci) * c.cout + co] = live ? v : 0.f;
                    }
        }
        INCRMT_CK(cudaMemcpy(params, h.data(), sizeof(float) * nparams, cudaMemcpyHostToDevice));
        return refresh_weights(nullptr);
    }

    int refresh_weights(cudaStream_t s) {
        for (auto &c : convs) {
            const long n = static_cast<long>(c.taps) * c.cin * c.cout;
            k_weights_bf16<<<gs(n), 256, 0, s>>>(params + c.woff, c.w, c.wt, c.taps, c.cin, c.cout);
            launches++;
        }
        INCRMT_CKL("k_weights_bf16");
        return INCRMT_OK;
    }

    void free_work() {
        for (void *p : work) cudaFree(p);
        work.clear();
        cudaFree(part);
        part = nullptr;
        part_n = 0;
        acts.clear();
        wb = wh = ww = 0;
    }

    /** Activation buffers for (B, H, W): the input, then every convolution's
     * output, every pooling's output and every concatenation. */
    int ensure(int B, int H, int W) {
        if (B == wb && H == wh && W == ww) return INCRMT_OK;
        free_work();
        gen++;  // every pointer into the activations changes
        auto alloc = [&](int level, int Cc) -> int {
            Act a;
            a.level = level;
            a.C = Cc;
            const long n = static_cast<long>(B) * (H >> level) * (W >> level) * Cc;
            INCRMT_CK(cudaMalloc(&a.x, sizeof(bf16) * n));
            work.push_back(a.x);
            INCRMT_CK(cudaMalloc(&a.g, sizeof(bf16) * n));
            work.push_back(a.g);
            acts.push_back(a);
            return INCRMT_OK;
        };
        int r;
        if ((r = alloc(0, 16))) return r;  // 0: packed input
        for (int l = 0; l < levels; l++) {
            if (l > 0 && (r = alloc(l, C(l - 1)))) return r;  // pooled input of level l
            if ((r = alloc(l, C(l)))) return r;                // first conv
            if ((r = alloc(l, C(l)))) return r;                // second conv (skip of level l)
        }
        for (int l = levels - 2; l >= 0; l--) {
            if ((r = alloc(l, C(l + 1) + C(l)))) return r;     // concatenation
            if ((r = alloc(l, C(l)))) return r;
            if ((r = alloc(l, C(l)))) return r;
        }
        if ((r = alloc(0, 16))) return r;  // head output
        // partials of the largest weight gradient (and of the bias gradients)
        size_t need = 0;
        {
            int k = 0;
            for (int l = 0; l < levels; l++)
                for (int q = 0; q < 2; q++, k++) {
                    const Conv &c = convs[k];
                    need = std::max(need, conv_tc_wgrad_workspace(B, H >> l, W >> l, c.cin, c.cout, c.taps));
                }
            for (int l = levels - 2; l >= 0; l--)
                for (int q = 0; q < 2; q++, k++) {
                    const Conv &c = convs[k];
                    need = std::max(need, conv_tc_wgrad_workspace(B, H >> l, W >> l, c.cin, c.cout, c.taps));
                }
            const Conv &c = convs[k];
            need = std::max(need, conv_tc_wgrad_workspace(B, H, W, c.cin, c.cout, c.taps));
            need = std::max(need, static_cast<size_t>(kBiasSplits) * (base << (levels - 1)));
        }
        INCRMT_CK(cudaMalloc(&part, sizeof(float) * need));
        part_n = need;
        wb = B; wh = H; ww = W;
        return INCRMT_OK;
    }

    int conv_forward(const Conv &c, const bf16 *X, bf16 *Y, int B, int H, int W, cudaStream_t s) {
        launches++;
        return conv_tc(X, B, H, W, c.cin, c.wt, c.taps, c.cout, false, params + c.boff, c.relu, Y, s);
    }

    /** Gradients of one convolution: its output gradient gY (already masked
     * by the ReLU), input X; accumulates dW, db and writes gX (if given). */
    int conv_backward(const Conv &c, const bf16 *X, const bf16 *gY, bf16 *gX, int B, int H, int W, cudaStream_t s) {
        const long P = static_cast<long>(B) * H * W;
        float *dW = grads + c.woff, *db = grads + c.boff;
        int r = conv_tc_wgrad(X, gY, B, H, W, c.cin, c.cout, c.taps, dW, part, part_n, s);
        if (r) return r;
        k_bias_partial<<<dim3(kBiasSplits, (c.cout + 31) / 32), 256, 0, s>>>(gY, part, P, c.cout);
        k_bias_reduce<<<1, 256, 0, s>>>(part, kBiasSplits, c.cout, db);
        launches += 4;
        INCRMT_CKL("bias gradient");
        if (gX) {
            launches++;
            return conv_tc(gY, B, H, W, c.cout, c.w, c.taps, c.cin, true, nullptr, false, gX, s);
        }
        return INCRMT_OK;
    }

    /** Forward pass; returns the head output activation. Act indices follow
     * ensure(): 0 input; per encoder level [pool,] conv1, conv2; per decoder
     * level cat, conv1, conv2; last the head. */
    int forward(int B, int H, int W, const float *in, cudaStream_t s) {
        int r = ensure(B, H, W);
        if (r) return r;
        const long P = static_cast<long>(B) * H * W;
        k_pack_input<<<gs(P), 256, 0, s>>>(in, acts[0].x, P);
        launches++;
        int a = 1, k = 0;
        bf16 *cur = acts[0].x;
        std::vector<int> skip(levels);
        for (int l = 0; l < levels; l++) {
            const int Hl = H >> l, Wl = W >> l;
            if (l > 0) {
                k_pool<<<gs(static_cast<long>(B) * Hl * Wl * C(l - 1) / 8), 256, 0, s>>>(cur, acts[a].x, B, Hl * 2, Wl * 2, C(l - 1));
                launches++;
                cur = acts[a++].x;
            }
            if ((r = conv_forward(convs[k++], cur, acts[a].x, B, Hl, Wl, s))) return r;
            cur = acts[a++].x;
            if ((r = conv_forward(convs[k++], cur, acts[a].x, B, Hl, Wl, s))) return r;
            skip[l] = a;
            cur = acts[a++].x;
        }
        for (int l = levels - 2; l >= 0; l--) {
            const int Hl = H >> l, Wl = W >> l;
            k_upcat<<<gs(static_cast<long>(B) * Hl * Wl * (C(l + 1) + C(l)) / 8), 256, 0, s>>>(
                cur, acts[skip[l]].x, acts[a].x, B, Hl, Wl, C(l + 1), C(l));
            launches++;
            cur = acts[a++].x;
            if ((r = conv_forward(convs[k++], cur, acts[a].x, B, Hl, Wl, s))) return r;
            cur = acts[a++].x;
            if ((r = conv_forward(convs[k++], cur, acts[a].x, B, Hl, Wl, s))) return r;
            cur = acts[a++].x;
        }
        if ((r = conv_forward(convs[k++], cur, acts[a].x, B, H, W, s))) return r;
        INCRMT_CKL("unet forward");
        return INCRMT_OK;
    }

    /** Backward pass from the head gradient in acts.back().g; accumulates
     * into grads (zeroed by the caller). */
    int backward(int B, int H, int W, cudaStream_t s) {
        int r;
        int a = static_cast<int>(acts.size()) - 1, k = static_cast<int>(convs.size()) - 1;
        // Recover the forward bookkeeping: indices of the skips.
        std::vector<int> skip(levels), pool_idx(levels, -1);
        {
            int q = 1;
            for (int l = 0; l < levels; l++) {
                if (l > 0) pool_idx[l] = q++;
                q++;
                skip[l] = q++;
            }
        }
        // Head.
        if ((r = conv_backward(convs[k], acts[a - 1].x, acts[a].g, acts[a - 1].g, B, H, W, s))) return r;
        k--;
        a--;
        // Decoder, finest first.
        for (int l = 0; l <= levels - 2; l++) {
            const int Hl = H >> l, Wl = W >> l;
            // acts[a] = conv2 output of this decoder level, acts[a-1] = conv1, acts[a-2] = cat
            const long n2 = static_cast<long>(B) * Hl * Wl * C(l);
            k_relu_mask<<<gs(n2 / 8), 256, 0, s>>>(acts[a].g, acts[a].x, n2);
            if ((r = conv_backward(convs[k], acts[a - 1].x, acts[a].g, acts[a - 1].g, B, Hl, Wl, s))) return r;
            k_relu_mask<<<gs(n2 / 8), 256, 0, s>>>(acts[a - 1].g, acts[a - 1].x, n2);
            if ((r = conv_backward(convs[k - 1], acts[a - 2].x, acts[a - 1].g, acts[a - 2].g, B, Hl, Wl, s))) return r;
            launches += 2;
            // Split the concatenation gradient: coarser level's output and the skip.
            const int lower = (l + 1 == levels - 1) ? skip[levels - 1] : a - 3;
            k_upcat_bwd<<<gs(static_cast<long>(B) * Hl * Wl * (C(l + 1) + C(l)) / 8), 256, 0, s>>>(
                acts[a - 2].g, acts[lower].g, acts[skip[l]].g, B, Hl, Wl, C(l + 1), C(l));
            launches++;
            k -= 2;
            a -= 3;
        }
        // Encoder, coarsest first (acts[skip[l]].g now holds the gradient of
        // level l's output, including its skip path).
        for (int l = levels - 1; l >= 0; l--) {
            const int Hl = H >> l, Wl = W >> l;
            const int o2 = skip[l], o1 = o2 - 1, in = (l > 0) ? pool_idx[l] : 0;
            const long n2 = static_cast<long>(B) * Hl * Wl * C(l);
            k_relu_mask<<<gs(n2 / 8), 256, 0, s>>>(acts[o2].g, acts[o2].x, n2);
            if ((r = conv_backward(convs[2 * l + 1], acts[o1].x, acts[o2].g, acts[o1].g, B, Hl, Wl, s))) return r;
            k_relu_mask<<<gs(n2 / 8), 256, 0, s>>>(acts[o1].g, acts[o1].x, n2);
            if ((r = conv_backward(convs[2 * l], acts[in].x, acts[o1].g, l > 0 ? acts[in].g : nullptr, B, Hl, Wl, s))) return r;
            launches += 2;
            if (l > 0) {
                // Pooling gradient into the finer level's output gradient.
                k_pool_bwd_add<<<gs(static_cast<long>(B) * (Hl * 2) * (Wl * 2) * C(l - 1) / 8), 256, 0, s>>>(
                    acts[in].g, acts[skip[l - 1]].g, B, Hl * 2, Wl * 2, C(l - 1));
                launches++;
            }
        }
        INCRMT_CKL("unet backward");
        return INCRMT_OK;
    }

    int loss_and_grad(int B, int H, int W, const float *t, const float *valid, cudaStream_t s) {
        const long P = static_cast<long>(B) * H * W;
        INCRMT_CK(cudaMemsetAsync(sums, 0, sizeof(double) * 2, s));
        k_loss<<<gs(P), 256, 0, s>>>(acts.back().x, t, valid, P, sums);
        k_loss_grad<<<gs(P * 16), 256, 0, s>>>(acts.back().x, t, valid, P, sums, acts.back().g);
        launches += 2;
        INCRMT_CKL("unet loss");
        return INCRMT_OK;
    }

    void destroy() {
        free_work();
        cudaFree(params); cudaFree(grads); cudaFree(m1); cudaFree(m2); cudaFree(wpool); cudaFree(sums);
        params = grads = m1 = m2 = nullptr;
        wpool = nullptr;
        sums = nullptr;
    }
};

}  // namespace incrmt

struct incrmt_unet {
    incrmt::UNet u;
};

namespace incrmt {
long long unet_generation(const incrmt_unet *h) { return h->u.gen; }
}  // namespace incrmt

extern "C" {

int incrmt_unet_create(int levels, int base, unsigned long long seed, incrmt_unet **out) {
    if (!out) { incrmt::set_error("null argument"); return INCRMT_ERR_BADARG; }
    *out = nullptr;
    if (levels < 2 || levels > 5 || base < 16 || base % 16 || base > 128) {
        incrmt::set_error("unet: levels 2..5 and a base of 16..128 channels in steps of 16");
        return INCRMT_ERR_BADARG;
    }
    incrmt_unet *h = new (std::nothrow) incrmt_unet;
    if (!h) { incrmt::set_error("out of host memory"); return INCRMT_ERR_OOM; }
    int r = h->u.create(levels, base, seed);
    if (r) { h->u.destroy(); delete h; return r; }
    *out = h;
    return INCRMT_OK;
}

long long incrmt_unet_num_params(const incrmt_unet *h) { return h ? h->u.nparams : 0; }

int incrmt_unet_get_params(incrmt_unet *h, float *host) {
    if (!h || !host) { incrmt::set_error("null argument"); return INCRMT_ERR_BADARG; }
    INCRMT_CK(cudaMemcpy(host, h->u.params, sizeof(float) * h->u.nparams, cudaMemcpyDeviceToHost));
    return INCRMT_OK;
}

int incrmt_unet_set_params(incrmt_unet *h, const float *host) {
    if (!h || !host) { incrmt::set_error("null argument"); return INCRMT_ERR_BADARG; }
    INCRMT_CK(cudaMemcpy(h->u.params, host, sizeof(float) * h->u.nparams, cudaMemcpyHostToDevice));
    int r = h->u.refresh_weights(nullptr);
    if (r) return r;
    INCRMT_CK(cudaDeviceSynchronize());
    return INCRMT_OK;
}

static int unet_check_shape(const incrmt_unet *h, int batch, int H, int W) {
    const int q = 1 << (h->u.levels - 1);
    if (batch < 1 || H < q || W < q || H % 16 || W % 16 || H % q || W % q) {
        incrmt::set_error("unet: H and W must be positive multiples of 16 and of 2^(levels-1)");
        return INCRMT_ERR_BADARG;
    }
    return INCRMT_OK;
}

int incrmt_unet_forward(incrmt_unet *h, int batch, int H, int W, const float *d_in, float *d_out, void *stream) {
    if (!h || !d_in || !d_out) { incrmt::set_error("null argument"); return INCRMT_ERR_BADARG; }
    int r = unet_check_shape(h, batch, H, W);
    if (r) return r;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if ((r = h->u.forward(batch, H, W, d_in, s))) return r;
    const long P = static_cast<long>(batch) * H * W;
    incrmt::k_unpack_output<<<incrmt::gs(P), 256, 0, s>>>(h->u.acts.back().x, d_out, P);
    h->u.launches++;
    INCRMT_CKL("k_unpack_output");
    return INCRMT_OK;
}

static int unet_grad(incrmt_unet *h, int batch, int H, int W, const float *d_in, const float *d_t,
                     const float *d_valid, float *loss, cudaStream_t s) {
    int r = unet_check_shape(h, batch, H, W);
    if (r) return r;
    incrmt::UNet &u = h->u;
    if ((r = u.forward(batch, H, W, d_in, s))) return r;
    if ((r = u.loss_and_grad(batch, H, W, d_t, d_valid, s))) return r;
    INCRMT_CK(cudaMemsetAsync(u.grads, 0, sizeof(float) * u.nparams, s));
    if ((r = u.backward(batch, H, W, s))) return r;
    double hs[2];
    INCRMT_CK(cudaMemcpyAsync(hs, u.sums, sizeof(hs), cudaMemcpyDeviceToHost, s));
    INCRMT_CK(cudaStreamSynchronize(s));
    if ((r = incrmt::conv_tc_status())) return r;
    if (loss) *loss = static_cast<float>(hs[1] > 0 ? hs[0] / hs[1] : 0.0);
    return INCRMT_OK;
}

int incrmt_unet_train_step(incrmt_unet *h, int batch, int H, int W, const float *d_in, const float *d_target,
                           const float *d_valid, float lr, float *loss, void *stream) {
    if (!h || !d_in || !d_target || !d_valid) { incrmt::set_error("null argument"); return INCRMT_ERR_BADARG; }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int r = unet_grad(h, batch, H, W, d_in, d_target, d_valid, loss, s);
    if (r) return r;
    incrmt::UNet &u = h->u;
    u.adam_t++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, static_cast<float>(u.adam_t)), c2 = 1.f - std::pow(b2, static_cast<float>(u.adam_t));
    incrmt::k_adam<<<incrmt::gs(u.nparams), 256, 0, s>>>(u.params, u.grads, u.m1, u.m2, u.nparams, lr, b1, b2, c1, c2,
                                                        1e-8f);
    u.launches++;
    INCRMT_CKL("k_adam");
    return u.refresh_weights(s);
}

int incrmt_unet_gradients(incrmt_unet *h, int batch, int H, int W, const float *d_in, const float *d_target,
                          const float *d_valid, float *loss, float *host_grad, void *stream) {
    if (!h || !d_in || !d_target || !d_valid || !host_grad) { incrmt::set_error("null argument"); return INCRMT_ERR_BADARG; }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int r = unet_grad(h, batch, H, W, d_in, d_target, d_valid, loss, s);
    if (r) return r;
    INCRMT_CK(cudaMemcpy(host_grad, h->u.grads, sizeof(float) * h->u.nparams, cudaMemcpyDeviceToHost));
    return INCRMT_OK;
}

long long incrmt_unet_launches(const incrmt_unet *h) { return h ? h->u.launches : 0; }

int incrmt_conv_bf16(const void *d_x, int batch, int H, int W, int cin, const void *d_wk, int taps, int cout,
                     int flip, const float *d_bias, int relu, void *d_y, void *stream) {
    return incrmt::conv_tc(static_cast<const incrmt::bf16 *>(d_x), batch, H, W, cin,
                           static_cast<const incrmt::bf16 *>(d_wk), taps, cout, flip != 0, d_bias, relu != 0,
                           static_cast<incrmt::bf16 *>(d_y), static_cast<cudaStream_t>(stream));
}

int incrmt_conv_status(void) { return incrmt::conv_tc_status(); }

int incrmt_conv_set_variant(int variant) { return incrmt::conv_tc_set_variant(variant); }

long long incrmt_conv_wgrad_workspace(int batch, int H, int W, int cin, int cout, int taps) {
    if (batch < 1 || H < 1 || W < 1 || cin < 16 || cout < 16 || (taps != 1 && taps != 9)) return 0;
    return static_cast<long long>(incrmt::conv_tc_wgrad_workspace(batch, H, W, cin, cout, taps));
}

int incrmt_conv_wgrad_bf16(const void *d_x, const void *d_dy, int batch, int H, int W, int cin, int cout, int taps,
                           float *d_dw, float *d_work, long long work_floats, void *stream) {
    if (work_floats < 0) { incrmt::set_error("negative workspace size"); return INCRMT_ERR_BADARG; }
    return incrmt::conv_tc_wgrad(static_cast<const incrmt::bf16 *>(d_x), static_cast<const incrmt::bf16 *>(d_dy),
                                 batch, H, W, cin, cout, taps, d_dw, d_work, static_cast<size_t>(work_floats),
                                 static_cast<cudaStream_t>(stream));
}

void incrmt_unet_destroy(incrmt_unet *h) {
    if (!h) return;
    cudaDeviceSynchronize();
    h->u.destroy();
    delete h;
}

}  // extern "C"
