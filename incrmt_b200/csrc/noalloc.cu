// Allocation-free variant of the pressure-operator application
// (incrmt_mg_apply). Some callers cannot allocate device memory: code that
// runs inside a memory arena whose owner forbids further cudaMalloc calls
// (a framework's caching allocator, a real-time loop that must not take the
// driver's allocation locks), or a host that has already handed all free
// device memory to its own pools. For them this entry point takes device
// input and output pointers and keeps its only scratch -- the edge or cell
// reciprocal densities -- in a fixed array compiled into the library.
#include <cstdint>
#include "incrmt.h"
#include "common.cuh"
#include "mg_ops.cuh"

namespace incrmt {

namespace {

/** Largest grid the allocation-free entry point accepts (cells per side). */
constexpr int kNoAllocMaxCells = 256;
/** Scratch words: the MAC edge arrays ex ((m+1) x n) and ey (m x (n+1)), or
 * the FEM cell array ((m+1) x (n+1)), at the largest grid. */
constexpr long kNoAllocScratch = 2L * (kNoAllocMaxCells + 1) * kNoAllocMaxCells;

/** The scratch. Every GPU that loads the library holds these ~1 MB until the
 * process exits. In host code the symbol is a host-side stand-in, not a
 * device address; its device address comes from cudaGetSymbolAddress. */
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratch];

/** Device addresses of the scratch, looked up once per device. */
constexpr int kMaxDevices = 64;
void *g_scratch_addr[kMaxDevices] = {nullptr};

__global__ void k_na_mac_coef(const double *rho, int m, int n, double *ex, double *ey) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    const int ml = m + 4;
    if (j < n && i <= m) {
        const int q = (i + 2) + ml * (j + 2);
        ex[j * (m + 1) + i] = 0.5 / rho[q] + 0.5 / rho[q - 1];
    }
    if (j <= n && i < m) {
        const int q = (i + 2) + ml * (j + 2);
        ey[j * m + i] = 0.5 / rho[q] + 0.5 / rho[q - ml];
    }
}

__global__ void k_na_fem_coef(const double *rho, int m, int mf, int nf, double *c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= mf || j >= nf) return;
    c[j * mf + i] = 1. / rho[(i + 1) + (m + 4) * (j + 1)];
}

template <class Op>
__global__ void k_na_apply(Op op, const double *z, double *out, int m, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= m || j >= n) return;
    double diag;
    const double off = op.offdiag(i, j, z, diag);
    out[i + m * j] = fma_rn(diag, z[i + m * j], off);
}

/** Device address of the scratch on the current device; the first call on a
 * device looks it up (the device must be current, as it is here). */
int scratch_address(double **out) {
    int dev = 0;
    INCRMT_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) { set_error("device index %d out of range", dev); return INCRMT_ERR_BADARG; }
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
        g_scratch_addr[dev] = p;
    }
    *out = static_cast<double *>(g_scratch_addr[dev]);
    return INCRMT_OK;
}

}  // namespace
}  // namespace incrmt

extern "C" int incrmt_mg_apply_noalloc(int sys, int m, int n, double ax, double bx, double ay, double by,
                                       int zpr, const double *d_rho, const double *d_z, double *d_out,
                                       void *stream) {
    using namespace incrmt;
    if (!d_rho || !d_z || !d_out) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    if (sys != INCRMT_SYS_MAC && sys != INCRMT_SYS_FEM) { set_error("unknown system %d", sys); return INCRMT_ERR_BADARG; }
    if (m < 2 || n < 2 || !(bx > ax) || !(by > ay)) { set_error("bad grid %dx%d", m, n); return INCRMT_ERR_BADARG; }
    if (m > kNoAllocMaxCells || n > kNoAllocMaxCells) {
        set_error("incrmt_mg_apply_noalloc: grid %dx%d exceeds the %dx%d cells its fixed scratch holds",
                  m, n, kNoAllocMaxCells, kNoAllocMaxCells);
        return INCRMT_ERR_BADARG;
    }
    double *scratch = nullptr;
    int r = scratch_address(&scratch);
    if (r) return r;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const double dx = (bx - ax) / m, dy = (by - ay) / n, xsp = 1 / dx, ysp = 1 / dy;
    const dim3 blk(32, 8);
    // Every scratch word read below is written first in this call, so the
    // previous call's contents never leak into the result.
    if (sys == INCRMT_SYS_MAC) {
        double *ex = scratch, *ey = scratch + static_cast<long>(m + 1) * n;
        k_na_mac_coef<<<dim3(cdiv(m + 1, 32), cdiv(n + 1, 8)), blk, 0, s>>>(d_rho, m, n, ex, ey);
        MacOp<double> op;
        op.m = m; op.n = n; op.px = 0; op.py = 0; op.zpr = zpr ? 1 : 0;
        op.xxsp = xsp * xsp; op.yysp = ysp * ysp; op.ex = ex; op.ey = ey;
        k_na_apply<<<dim3(cdiv(m, 32), cdiv(n, 8)), blk, 0, s>>>(op, d_z, d_out, m, n);
    } else {
        const int mf = m + 1, nf = n + 1;
        double *c = scratch;
        k_na_fem_coef<<<dim3(cdiv(mf, 32), cdiv(nf, 8)), blk, 0, s>>>(d_rho, m, mf, nf, c);
        const double dydx = dy / dx, dxdy = dx / dy;
        FemOp<double> op;
        op.m = mf; op.n = nf; op.px = 0; op.py = 0; op.zpr = zpr ? 1 : 0;
        op.fm = 1. / 3. * (dxdy + dydx);
        op.hey = 0.5 * (1. / 3. * (-2 * dxdy + dydx));
        op.hex = 0.5 * (1. / 3. * (-2 * dydx + dxdy));
        op.fc = -1. / 6. * (dxdy + dydx);
        op.c = c;
        k_na_apply<<<dim3(cdiv(mf, 32), cdiv(nf, 8)), blk, 0, s>>>(op, d_z, d_out, mf, nf);
    }
    INCRMT_CKL("incrmt_mg_apply_noalloc");
    return INCRMT_OK;
}
