/* C ABI of the learned initial guess for the pressure solves: a BF16
 * convolutional U-Net trained on the GPU by this library's own kernels.
 *
 * It has no counterpart in the reference, whose projections start from the
 * previous solution (mgs_common.cc:15-21). The network maps three channels on
 * a grid restricted from the solve grid -- the residual b - A z0 normalised by
 * its RMS, the reciprocal density, and a zero channel -- to a field d; the
 * solver then uses z0 + alpha d with alpha = (d . r0) / (d . A d), the step
 * that minimises the error along d in the energy norm of the (definite)
 * system, the norm that weighs the smooth error multigrid removes slowest.
 *
 * Layout: activations NHWC (channel fastest) in BF16 with FP32 accumulation;
 * master weights FP32 with BF16 copies; Adam in FP32. Images are processed at
 * H x W with H, W multiples of 16 (inputs are zero-padded by the caller).
 * All functions return INCRMT_OK (0) or a negative INCRMT_ERR_* code. */
#ifndef INCRMT_UNET_H
#define INCRMT_UNET_H

#include <stddef.h>
#include "incrmt.h"
#include "incrmt_sim.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct incrmt_unet incrmt_unet;

/** Creates a U-Net with `levels` resolutions (2..5) and `base` channels at the
 * finest (a multiple of 16; doubled per level), 3 input channels and one
 * output, weights initialised from `seed` (He-uniform, zero biases). */
int incrmt_unet_create(int levels, int base, unsigned long long seed, incrmt_unet **out);

/** Number of FP32 parameters (all weights and biases). */
long long incrmt_unet_num_params(const incrmt_unet *h);

/** Copies the FP32 parameters out of / into the network (host arrays of
 * incrmt_unet_num_params floats, the layer order of the forward pass; each
 * convolution's weights as [tap][in][out], then its biases). */
int incrmt_unet_get_params(incrmt_unet *h, float *host);
int incrmt_unet_set_params(incrmt_unet *h, const float *host);

/** Forward pass on device arrays: `in` is batch x H x W x 3 FP32 (NHWC),
 * `out` batch x H x W FP32; work on `stream` (0 = default), not waited for. */
int incrmt_unet_forward(incrmt_unet *h, int batch, int H, int W, const float *d_in, float *d_out, void *stream);

/** One training step on device arrays: forward, loss = mean over the
 * `valid` mask (batch x H x W FP32, 1 inside the image, 0 in padding) of
 * (out - target)^2, backward, Adam (lr, beta1 0.9, beta2 0.999, eps 1e-8).
 * The loss before the update is written to *loss (synchronises the stream). */
int incrmt_unet_train_step(incrmt_unet *h, int batch, int H, int W, const float *d_in, const float *d_target,
                           const float *d_valid, float lr, float *loss, void *stream);

/** Gradient check support: forward + backward without the update; the
 * FP32 parameter gradients (incrmt_unet_num_params floats) go to `host_grad`
 * and the loss to *loss. */
int incrmt_unet_gradients(incrmt_unet *h, int batch, int H, int W, const float *d_in, const float *d_target,
                          const float *d_valid, float *loss, float *host_grad, void *stream);

/** Result of a learned guess: the residual 2-norms before and after (the
 * energy-optimal step may raise the residual while lowering the smooth
 * error), the scale alpha, and whether the guess was applied (alpha > 0). */
typedef struct incrmt_learned_stats {
    double res_before, res_after, alpha;
    int used;
} incrmt_learned_stats;

/** Learned initial guess of the solve of `h` (a MAC or FEM solver whose
 * density is set; not x-periodic): from the iterate d_z, forms r0 = b - A z, runs the
 * network on the r0 and 1/rho features restricted by `factor` (block
 * averages; the network grid is ceil(m/factor) x ceil(n/factor) rounded up to
 * multiples of 16), prolongs the output d bilinearly and sets
 * z += alpha d with alpha = (d . r0) / (d . A d) (unchanged if alpha <= 0). Runs on the solver's stream; synchronises only when st is
 * given. No counterpart in the reference (it starts from the previous
 * solution, mgs_common.cc:15-21). */
int incrmt_mg_learned_guess(incrmt_mg *h, incrmt_unet *net, const double *d_b, double *d_z, int factor,
                            incrmt_learned_stats *st);

/** The network input the guess would use (for training data): 3 x H x W
 * floats (NHWC) into d_in, H x W the network grid of `factor`. */
int incrmt_mg_learned_input(incrmt_mg *h, const double *d_b, const double *d_z, int factor, float *d_in, int H,
                            int W);

/** Learned warm start of a simulation's projections (no counterpart in the
 * reference, whose projections start from the previous solution,
 * mgs_common.cc:15-21). For system sys (INCRMT_SYS_MAC: the MAC projection,
 * INCRMT_SYS_FEM: the FEM projection), before every solve the guess above is
 * applied to the warm start (the previous step's solution) with the network
 * net at restriction factor `factor`. rule 0 keeps the previous solution
 * whenever the step would raise the residual's 2-norm (the network's initial
 * residual is worse); rule 1 only when alpha <= 0 (the step lowers the error
 * in the energy norm whenever alpha > 0). The solve then iterates to the same
 * tolerance as without it. net = NULL turns it off. The network stays owned
 * by the caller and must outlive its use. x-periodic systems are rejected. */
int incrmt_sim_set_learned(incrmt_sim *h, int sys, incrmt_unet *net, int factor, int rule);

/** Network grid H x W of system sys at restriction factor `factor`. */
int incrmt_sim_learned_grid(const incrmt_sim *h, int sys, int factor, int *H, int *W);

/** Training samples from the simulation's own projections: each of the next
 * `cap` solves of system sys writes, before solving, the network input of its
 * warm start (H x W x 3 floats, the layout of incrmt_mg_learned_input) to
 * d_in + k*H*W*3 and, after solving, the block averages of (solution - warm
 * start) over factor x factor unknowns (H x W floats, zero outside the image)
 * to d_target + k*H*W, k = 0, 1, ... Captured solves run without the learned
 * guess. cap = 0 stops the capture. Device buffers owned by the caller. */
int incrmt_sim_learned_capture(incrmt_sim *h, int sys, int factor, float *d_in, float *d_target, int cap);

/** Counts of system sys since the simulation was created: guesses applied,
 * guesses rejected by the rule (the solve then starts from the previous
 * solution), samples captured by the current capture, and projections that
 * skipped the guess: after 8 rejected guesses in a row the next 32
 * projections of that system start from the warm start without computing a
 * guess (the network's cost would buy nothing), then guessing resumes. */
typedef struct incrmt_sim_learned_stats {
    long long applied, fallback, captured, skipped;
} incrmt_sim_learned_stats;
int incrmt_sim_get_learned_stats(incrmt_sim *h, int sys, incrmt_sim_learned_stats *st);

/** One convolution of the U-Net's kind on the tcgen05 tensor cores (no
 * reference counterpart): d_y = act(bias + conv(d_x, weights)) for a 3x3
 * (taps 9, zero padding) or 1x1 (taps 1) kernel over batch x H x W images,
 * NHWC BF16 activations (cin and cout multiples of 16), the weights BF16 as
 * [tap][cout][cin] (K-major for the implicit GEMM), d_bias (cout FP32) may
 * be null, relu 0 or 1. With flip set the taps are read in reverse order,
 * so that the forward weights W[tap][cin][cout] of a layer, passed as
 * [tap][cout'=cin][cin'=cout], give the input gradient of that layer from
 * its output gradient. Issued on `stream`, not waited for. */
int incrmt_conv_bf16(const void *d_x, int batch, int H, int W, int cin, const void *d_wk, int taps, int cout,
                     int flip, const float *d_bias, int relu, void *d_y, void *stream);

/** Weight gradient of such a convolution on the tcgen05 tensor cores:
 * d_dw[tap][cin][cout] (FP32) += sum over the pixels of
 * x[p + offset(tap)][ci] * dy[p][co] (x the layer's input, dy the gradient
 * of its output, NHWC BF16). The pixels are split over CTAs whose FP32
 * partial sums go to d_work (incrmt_conv_wgrad_workspace floats) and are
 * then added to d_dw in a fixed order: the result is the same on every run.
 * Issued on `stream`, not waited for. */
long long incrmt_conv_wgrad_workspace(int batch, int H, int W, int cin, int cout, int taps);
int incrmt_conv_wgrad_bf16(const void *d_x, const void *d_dy, int batch, int H, int W, int cin, int cout, int taps,
                           float *d_dw, float *d_work, long long work_floats, void *stream);

/** INCRMT_OK, or INCRMT_ERR_CUDA when a tensor-core convolution gave up one
 * of its pipeline waits (each is limited to one second) since the last call;
 * clears that record. Synchronises the device. */
int incrmt_conv_status(void);

/** Kernel choice of incrmt_conv_bf16 (and of the networks' 3x3 layers) for
 * the whole process: 0 automatic (default), 1 one tap per pipeline stage,
 * 2 row reuse (each stage holds one column offset of the tile's rows -1..8
 * and the weights of that column's three taps), 3 row reuse in persistent
 * CTAs with the layer's weights resident in shared memory (layers of at most
 * 128 outputs whose weights fit; others fall back to 2), 4 row reuse with two
 * 128-pixel halves per CTA sharing each stage's weights (up to 64 outputs;
 * others fall back to 2). All compute the same products; the FP32 sums visit
 * the taps in other orders. No reference counterpart (a check and tuning
 * knob); INCRMT_ERR_BADARG outside 0..4. */
int incrmt_conv_set_variant(int variant);

/** Kernel launches issued by this network so far. */
long long incrmt_unet_launches(const incrmt_unet *h);

void incrmt_unet_destroy(incrmt_unet *h);

#ifdef __cplusplus
}
#endif

#endif
