// 5th-generation tensor-core (tcgen05) convolutions of the learned initial
// guess's U-Net: NHWC BF16 activations, FP32 accumulation in tensor memory.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace incrmt {

/** Y = act(bias + conv(X, weights)) for a 3x3 (taps = 9, zero padding) or
 * 1x1 (taps = 1) convolution on B x H x W images, NHWC BF16, Cin and Cout
 * multiples of 16, as an implicit GEMM on the tcgen05 tensor cores: M = 128
 * pixels (a Wt x Ht tile of one image), N = Cout (split over CTAs above 256),
 * K = taps x Cin. `wk` holds the weights K-major for the GEMM,
 * [tap][Cout][Cin]; with `flip` they are read with the taps reversed, which
 * is how the input gradient (the convolution of the output gradient with the
 * flipped, transposed weights) reuses the same kernel with the forward
 * weights W[tap][Cin][Cout] as its K-major operand.
 * bias may be null. Issued on `s`, not waited for. */
int conv_tc(const __nv_bfloat16 *X, int B, int H, int W, int Cin, const __nv_bfloat16 *wk, int taps, int Cout,
            bool flip, const float *bias, bool relu, __nv_bfloat16 *Y, cudaStream_t s);

/** Weight gradient of such a convolution: dW[tap][Cin][Cout] (FP32) +=
 * sum over the pixels of X[p + off(tap)][ci] dY[p][co], on the tcgen05
 * tensor cores (M = 128 input channels, N = output channels, K = pixels,
 * both operands read as stored, channels fastest). The pixels are split
 * over CTAs; each writes its FP32 partial to `part` (at least
 * conv_tc_wgrad_workspace() floats) and one more kernel adds the partials
 * to dW in a fixed order, so the result does not depend on scheduling. */
int conv_tc_wgrad(const __nv_bfloat16 *X, const __nv_bfloat16 *dY, int B, int H, int W, int Cin, int Cout, int taps,
                  float *dW, float *part, size_t part_floats, cudaStream_t s);
size_t conv_tc_wgrad_workspace(int B, int H, int W, int Cin, int Cout, int taps);

/** Kernel choice of conv_tc for 3x3 convolutions: 0 automatic (two halves up
 * to 32 outputs, or up to 64 from at most 32 inputs; resident weights where
 * they fit with 64 to 128 outputs; else row reuse up to 128 outputs), 1 one
 * tap per pipeline stage, 2 row reuse always, 3 resident weights where they
 * fit (else as 2), 4 row reuse with two 128-pixel halves per CTA up to 64
 * outputs (else as 2).
 * Both form the same products; the FP32 accumulation visits the taps in
 * another order. A check and tuning knob. */
int conv_tc_set_variant(int v);

/** INCRMT_OK, or INCRMT_ERR_CUDA if a tensor-core convolution gave up a wait
 * (its one-second limit on a pipeline barrier) since the last call; clears
 * the flag. Synchronises the device. */
int conv_tc_status();

}  // namespace incrmt
