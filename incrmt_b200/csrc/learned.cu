// The learned initial guess of a MAC or FEM pressure solve. From the current iterate
// z0 the residual r0 = b - A z0 is formed; its restriction to the network's
// grid (block averages over factor x factor cells), normalised by its RMS,
// and the restricted reciprocal density are the network's input; the output
// d is prolonged back bilinearly and the iterate becomes z0 + alpha d with
// alpha = (d . r0) / (d . A d), the step that minimises the error in the
// energy norm of the (definite) system along d. That norm weighs the smooth
// error the multigrid cycles remove slowest; a residual-minimising step would
// instead be dominated by the high-frequency part of d's error, which the
// smoother removes anyway. With alpha <= 0 the iterate is left unchanged, and
// under the residual rule also when the step would raise the residual's
// 2-norm (the iterate then stays the previous solution). Everything runs on
// the solver's stream; no host synchronisation unless statistics are
// requested.
#include <cmath>
#include "incrmt.h"
#include "incrmt_unet.h"
#include "mg.cuh"

namespace incrmt {

void LearnedWork::release() {
    cudaFree(r0); cudaFree(ad); cudaFree(dfine); cudaFree(dots); cudaFree(in); cudaFree(out);
    r0 = ad = dfine = dots = nullptr;
    in = out = nullptr;
    n_fine = n_net = 0;
}

namespace {

__global__ void k_sub(const double *b, const double *az, double *r, long n) {
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x)
        r[i] = b[i] - az[i];
}

/** Partial sums of x.y (one per block), deterministic order. */
__global__ void k_dot_partial(const double *x, const double *y, long n, double *partial) {
    double acc = 0;
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x)
        acc += x[i] * y[i];
    acc = block_sum_256(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

__global__ void k_sum_into(const double *partial, int nb, double *out) {
    double acc = 0;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) acc += partial[q];
    acc = block_sum_256(acc);
    if (threadIdx.x == 0) *out = acc;
}

/** Network input on an H x W grid (NHWC, 3 channels): block averages of the
 * residual over factor x factor unknowns divided by its RMS (rr = sum r^2 over
 * the N unknowns), the block average of the reciprocal density at the
 * unknowns (MAC: mean of a cell's left and right edge coefficients ex, an
 * (m+1) x n array; FEM: the cell coefficient array c, m x n like the nodes),
 * and zero. Outside the m x n image: zero. */
__global__ void k_learned_input(const double *r, const double *dens, int fem, int m, int n, int f, const double *rr,
                                int H, int W, float *in) {
    const int X = blockIdx.x * blockDim.x + threadIdx.x, Y = blockIdx.y * blockDim.y + threadIdx.y;
    if (X >= W || Y >= H) return;
    float c0 = 0, c1 = 0;
    const int i0 = X * f, j0 = Y * f;
    if (i0 < m && j0 < n) {
        double sr = 0, se = 0;
        int cnt = 0;
        for (int j = j0; j < j0 + f && j < n; j++)
            for (int i = i0; i < i0 + f && i < m; i++) {
                sr += r[static_cast<long>(j) * m + i];
                se += fem ? dens[static_cast<long>(j) * m + i]
                          : 0.5 * (dens[static_cast<long>(j) * (m + 1) + i] + dens[static_cast<long>(j) * (m + 1) + i + 1]);
                cnt++;
            }
        const double rms = sqrt(*rr / (static_cast<double>(m) * n));
        c0 = rms > 0 ? static_cast<float>(sr / cnt / rms) : 0.f;
        c1 = static_cast<float>(se / cnt);
    }
    float *o = in + (static_cast<long>(Y) * W + X) * 3;
    o[0] = c0;
    o[1] = c1;
    o[2] = 0.f;
}

/** Bilinear prolongation of the network output (cell-centred on the coarse
 * grid) to the m x n cells; clamped at the image edge. */
__global__ void k_learned_prolong(const float *out, int H, int W, int m, int n, int f, double *d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= m || j >= n) return;
    const int mc = (m + f - 1) / f, nc = (n + f - 1) / f;
    double x = (i + 0.5) / f - 0.5, y = (j + 0.5) / f - 0.5;
    x = fmin(fmax(x, 0.0), mc - 1.0);
    y = fmin(fmax(y, 0.0), nc - 1.0);
    const int x0 = static_cast<int>(x), y0 = static_cast<int>(y);
    const int x1 = x0 + 1 < mc ? x0 + 1 : x0, y1 = y0 + 1 < nc ? y0 + 1 : y0;
    const double fx = x - x0, fy = y - y0;
    const double v = (1 - fy) * ((1 - fx) * out[static_cast<long>(y0) * W + x0] + fx * out[static_cast<long>(y0) * W + x1]) +
                     fy * ((1 - fx) * out[static_cast<long>(y1) * W + x0] + fx * out[static_cast<long>(y1) * W + x1]);
    d[static_cast<long>(j) * m + i] = v;
}

/** z += alpha d with alpha = dots[0] / dots[1] (d.r0 over d.Ad) when
 * positive and finite and, under the residual rule (rule 0), when the new
 * residual |r0 - alpha Ad|^2 = dots[2] - 2 alpha dots[3] + alpha^2 dots[4]
 * is no larger than |r0|^2 = dots[2]. cnt (optional) counts the applied
 * guesses in cnt[0] and the fallbacks in cnt[1]. */
__global__ void k_learned_update(double *z, const double *d, long n, const double *dots, int rule,
                                 unsigned long long *cnt) {
    const double a = dots[1] != 0 ? dots[0] / dots[1] : 0.0;
    bool ok = a > 0 && isfinite(a);
    if (ok && rule == 0) ok = dots[2] - 2 * a * dots[3] + a * a * dots[4] <= dots[2];
    if (cnt && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&cnt[ok ? 0 : 1], 1ull);
    if (!ok) return;
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x)
        z[i] += a * d[i];
}

/** Training target on the network grid: block averages of znew - zold over
 * factor x factor unknowns (zero outside the m x n image). */
__global__ void k_learned_target(const double *znew, const double *zold, int m, int n, int f, int H, int W,
                                 float *tgt) {
    const int X = blockIdx.x * blockDim.x + threadIdx.x, Y = blockIdx.y * blockDim.y + threadIdx.y;
    if (X >= W || Y >= H) return;
    const int i0 = X * f, j0 = Y * f;
    float v = 0.f;
    if (i0 < m && j0 < n) {
        double s = 0;
        int cnt = 0;
        for (int j = j0; j < j0 + f && j < n; j++)
            for (int i = i0; i < i0 + f && i < m; i++) {
                const long q = static_cast<long>(j) * m + i;
                s += znew[q] - zold[q];
                cnt++;
            }
        v = static_cast<float>(s / cnt);
    }
    tgt[static_cast<long>(Y) * W + X] = v;
}

constexpr int kRed = 2 * kB200SMs;

int ensure(LearnedWork &w, long nf, long nn) {
    if (nf > w.n_fine) {
        cudaFree(w.r0); cudaFree(w.ad); cudaFree(w.dfine);
        w.r0 = w.ad = w.dfine = nullptr;
        w.n_fine = 0;
        INCRMT_CK(cudaMalloc(&w.r0, sizeof(double) * nf));
        INCRMT_CK(cudaMalloc(&w.ad, sizeof(double) * nf));
        INCRMT_CK(cudaMalloc(&w.dfine, sizeof(double) * nf));
        w.n_fine = nf;
    }
    if (nn > w.n_net) {
        cudaFree(w.in); cudaFree(w.out);
        w.in = w.out = nullptr;
        w.n_net = 0;
        INCRMT_CK(cudaMalloc(&w.in, sizeof(float) * 3 * nn));
        INCRMT_CK(cudaMalloc(&w.out, sizeof(float) * nn));
        w.n_net = nn;
    }
    if (!w.dots) INCRMT_CK(cudaMalloc(&w.dots, sizeof(double) * (8 + kRed)));
    return INCRMT_OK;
}

int dot(const double *x, const double *y, long n, double *partial, double *out, cudaStream_t s) {
    k_dot_partial<<<kRed, 256, 0, s>>>(x, y, n, partial);
    k_sum_into<<<1, 256, 0, s>>>(partial, kRed, out);
    INCRMT_CKL("learned dot");
    return INCRMT_OK;
}

}  // namespace

void learned_grid(int m, int n, int f, int &H, int &W) {
    W = ((m + f - 1) / f + 15) / 16 * 16;
    H = ((n + f - 1) / f + 15) / 16 * 16;
}

int learned_supported(const Multigrid &mg) {
    if (mg.px) { set_error("learned guess: x-periodic systems are not supported"); return INCRMT_ERR_BADARG; }
    return INCRMT_OK;
}

int learned_input(Multigrid &mg, LearnedWork &w, const double *d_b, const double *d_z, int f, int H, int W) {
    const long N = static_cast<long>(mg.m) * mg.n;
    int r = ensure(w, N, static_cast<long>(H) * W);
    if (r) return r;
    if ((r = mg.effective_rhs(d_b, &d_b))) return r;
    if ((r = mg.apply_device(d_z, w.ad))) return r;
    cudaStream_t s = mg.stream;
    k_sub<<<kRed, 256, 0, s>>>(d_b, w.ad, w.r0, N);
    if ((r = dot(w.r0, w.r0, N, w.dots + 8, w.dots + 2, s))) return r;
    const bool fem = mg.sys == INCRMT_SYS_FEM;
    k_learned_input<<<dim3(cdiv(W, 32), cdiv(H, 8)), dim3(32, 8), 0, s>>>(w.r0, fem ? mg.c : mg.ex, fem ? 1 : 0, mg.m,
                                                                          mg.n, f, w.dots + 2, H, W, w.in);
    mg.launches += 4;
    INCRMT_CKL("k_learned_input");
    return INCRMT_OK;
}

int learned_guess(Multigrid &mg, LearnedWork &w, incrmt_unet *net, const double *d_b, double *d_z, int f, int rule,
                  unsigned long long *cnt) {
    int H, W;
    learned_grid(mg.m, mg.n, f, H, W);
    int r = learned_input(mg, w, d_b, d_z, f, H, W);
    if (r) return r;
    cudaStream_t s = mg.stream;
    if ((r = incrmt_unet_forward(net, 1, H, W, w.in, w.out, s))) return r;
    const long N = static_cast<long>(mg.m) * mg.n;
    k_learned_prolong<<<dim3(cdiv(mg.m, 32), cdiv(mg.n, 8)), dim3(32, 8), 0, s>>>(w.out, H, W, mg.m, mg.n, f,
                                                                                  w.dfine);
    mg.launches++;
    if ((r = mg.apply_device(w.dfine, w.ad))) return r;
    // dots: [0] d.r0, [1] d.Ad, [2] r0.r0, [3] Ad.r0, [4] Ad.Ad
    if ((r = dot(w.dfine, w.r0, N, w.dots + 8, w.dots, s))) return r;
    if ((r = dot(w.dfine, w.ad, N, w.dots + 8, w.dots + 1, s))) return r;
    if ((r = dot(w.ad, w.r0, N, w.dots + 8, w.dots + 3, s))) return r;
    if ((r = dot(w.ad, w.ad, N, w.dots + 8, w.dots + 4, s))) return r;
    k_learned_update<<<kRed, 256, 0, s>>>(d_z, w.dfine, N, w.dots, rule, cnt);
    mg.launches += 10;
    INCRMT_CKL("k_learned_update");
    return INCRMT_OK;
}

int learned_target(Multigrid &mg, const double *znew, const double *zold, int f, int H, int W, float *tgt) {
    k_learned_target<<<dim3(cdiv(W, 32), cdiv(H, 8)), dim3(32, 8), 0, mg.stream>>>(znew, zold, mg.m, mg.n, f, H, W,
                                                                                   tgt);
    mg.launches++;
    INCRMT_CKL("k_learned_target");
    return INCRMT_OK;
}

}  // namespace incrmt

extern "C" {

int incrmt_mg_learned_input(incrmt_mg *h, const double *d_b, const double *d_z, int factor, float *d_in, int H,
                            int W) {
    if (!h || !d_b || !d_z || !d_in) { incrmt::set_error("null argument"); return INCRMT_ERR_BADARG; }
    incrmt::Multigrid &mg = h->mg;
    if (int r = incrmt::learned_supported(mg)) return r;
    int Hn, Wn;
    incrmt::learned_grid(mg.m, mg.n, factor, Hn, Wn);
    if (factor < 1 || H != Hn || W != Wn) {
        incrmt::set_error("learned guess: factor %d needs a %d x %d network grid", factor, Hn, Wn);
        return INCRMT_ERR_BADARG;
    }
    int r = incrmt::learned_input(mg, h->learned, d_b, d_z, factor, H, W);
    if (r) return r;
    INCRMT_CK(cudaMemcpyAsync(d_in, h->learned.in, sizeof(float) * 3 * H * W, cudaMemcpyDeviceToDevice, mg.stream));
    INCRMT_CK(cudaStreamSynchronize(mg.stream));
    return INCRMT_OK;
}

int incrmt_mg_learned_guess(incrmt_mg *h, incrmt_unet *net, const double *d_b, double *d_z, int factor,
                            incrmt_learned_stats *st) {
    if (!h || !net || !d_b || !d_z) { incrmt::set_error("null argument"); return INCRMT_ERR_BADARG; }
    incrmt::Multigrid &mg = h->mg;
    if (int r = incrmt::learned_supported(mg)) return r;
    if (factor < 1) { incrmt::set_error("bad factor %d", factor); return INCRMT_ERR_BADARG; }
    incrmt::LearnedWork &w = h->learned;
    int r = incrmt::learned_guess(mg, w, net, d_b, d_z, factor, 1, nullptr);
    if (r) return r;
    if (st) {
        double hd[5];
        INCRMT_CK(cudaMemcpyAsync(hd, w.dots, sizeof(hd), cudaMemcpyDeviceToHost, mg.stream));
        INCRMT_CK(cudaStreamSynchronize(mg.stream));
        const double a = hd[1] != 0 ? hd[0] / hd[1] : 0.0;
        const bool used = a > 0 && std::isfinite(a);
        st->alpha = used ? a : 0.0;
        st->used = used ? 1 : 0;
        st->res_before = std::sqrt(hd[2]);
        const double after2 = used ? hd[2] - 2 * a * hd[3] + a * a * hd[4] : hd[2];
        st->res_after = std::sqrt(after2 > 0 ? after2 : 0.0);
    }
    return INCRMT_OK;
}

}  // extern "C"
