// Geometric multigrid kernels and driver (see mg.cuh for the method).
#include <cmath>
#include <cstring>
#include <type_traits>
#include "mg.cuh"

namespace incrmt {

namespace {

constexpr int kNu1 = 2, kNu2 = 2, kCoarseSweeps = 64, kCoarsestSize = 16, kMaxLevels = 24;
/** Coupling ratio beyond which only the strongly coupled direction is
 * coarsened (semi-coarsening). */
constexpr double kSemiRatio = 2.0;
/** Largest residual ratio an FP32 defect-correction step may reach before the
 * solve continues in FP64. */
constexpr double kMixedContraction = 0.5;

// ---------------------------------------------------------------------------
// Transfer-operator index helpers (identical rules to the CPU oracle's shim).

__host__ __device__ __forceinline__ int wrap_idx(int i, int m, int p, bool &ok) {
    if (i < 0) { if (p) i += m; else ok = false; }
    else if (i >= m) { if (p) i -= m; else ok = false; }
    return i;
}

/** t + a*b with the product rounded before the sum (no fused multiply-add),
 * as the CPU oracle evaluates it: with the operator-dependent weights the
 * products are not exact, and a fused form would round them differently. The
 * FP32 V-cycles are not compared bit for bit and keep the fused form. */
__device__ __forceinline__ double add_prod(double t, double a, double b) { return __dadd_rn(t, __dmul_rn(a, b)); }
__device__ __forceinline__ float add_prod(float t, float a, float b) { return t + a * b; }

/** Floor of a/2 for any sign of a. */
__host__ __device__ __forceinline__ int half_floor(int a) { return a >= 0 ? a / 2 : -((1 - a) / 2); }

/** Coarse base index of fine index i along a direction: i/2 rounded down
 * when the direction is coarsened, else i. */
__host__ __device__ __forceinline__ int base_of(int i, bool k) { return k ? half_floor(i) : i; }

/** Coarse index of corner q (0 or 1) above base B along a direction of
 * coarse size mc, or -1 outside a non-periodic grid (and for q=1 when the
 * direction is not coarsened). */
__host__ __device__ __forceinline__ int corner_of(int B, int q, int mc, int p, bool k) {
    if (!k && q) return -1;
    int c = B + q;
    if (c < 0 || c >= mc) {
        if (!p) return -1;
        c = (c % mc + mc) % mc;
    }
    return c;
}

/** Prolongation weight of fine point (fi,fj) (unwrapped indices) for coarse
 * point (I,J): entry qx+2qy of the point's four stored weights, with (qx,qy)
 * the coarse point's offset from the point's base; 0 when it is not one of
 * its corners or the point is outside a non-periodic grid. */
template <class W>
__device__ __forceinline__ double pweight(const W *P, int fm, int fn, int px, int py, bool kx, bool ky, int fi,
                                          int fj, int I, int J) {
    const int qx = I - base_of(fi, kx), qy = J - base_of(fj, ky);
    if (qx < 0 || qx > 1 || qy < 0 || qy > 1) return 0;
    bool ok = true;
    const int i = wrap_idx(fi, fm, px, ok), j = wrap_idx(fj, fn, py, ok);
    if (!ok) return 0;
    return static_cast<double>(P[4 * (static_cast<long>(i) + static_cast<long>(fm) * j) + qx + 2 * qy]);
}

inline bool can_coarsen(int m, int p) { return p ? (m % 2 == 0 && m / 2 >= 4) : m >= 5; }

// ---------------------------------------------------------------------------
// Coefficient set-up kernels.

/** Edge reciprocal densities of the MAC system from the ghosted cell density
 * (fluid_2d::set_edge_irho, fluid_2d.cc:1140-1160). */
__global__ void k_mac_coef(const double *rho, int ml, int cm, int cn, double *ex, double *ey,
                           float *exf, float *eyf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (j < cn && i <= cm) {
        const int q = (i + 2) + ml * (j + 2);
        double v = 0.5 / rho[q] + 0.5 / rho[q - 1];
        ex[j * (cm + 1) + i] = v;
        exf[j * (cm + 1) + i] = static_cast<float>(v);
    }
    if (j <= cn && i < cm) {
        const int q = (i + 2) + ml * (j + 2);
        double v = 0.5 / rho[q] + 0.5 / rho[q - ml];
        ey[j * cm + i] = v;
        eyf[j * cm + i] = static_cast<float>(v);
    }
}

/** Cell reciprocal density at each FEM node, the cell below-left of the node
 * (fluid_2d::set_corner_irho, fluid_2d.cc:1163-1170). */
__global__ void k_fem_coef(const double *rho, int ml, int mf, int nf, double *c, float *cf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= mf || j >= nf) return;
    double v = 1. / rho[(i + 1) + ml * (j + 1)];
    c[j * mf + i] = v;
    cf[j * mf + i] = static_cast<float>(v);
}


/** Operator-dependent prolongation of a level (black-box multigrid:
 * Dendy, J. Comput. Phys. 48 (1982) 366-386): four weights per fine point,
 * P[4f+qx+2qy] for the coarse point at offset (qx,qy) from the point's base
 * (base_of). A point on a coarse point takes it with weight 1; a point
 * between two coarse points along x takes L/(-C) and R/(-C), L, C, R its
 * stencil summed over the columns left of, through and right of it (the
 * operator collapsed along y), and along y likewise with the rows; a point
 * between four coarse points takes -(its stencil entries times its eight
 * neighbours' weights)/(its diagonal), so pass 1 runs after pass 0 has set
 * the others. Constant coefficients give the bilinear 1, 1/2, 1/4; across a
 * density jump the weights follow the flux; at the zero-pressure edge of the
 * MAC system the last point's weight drops to about 1/3. Weights stay in
 * double precision so that constants map onto constants exactly and the
 * coarse operators of a pure-Neumann problem keep their null space. */
template <class Op>
__global__ void k_build_p(Op op, int fm, int fn, int px, int py, bool kx, bool ky, int cm, int cn, double *P,
                          int pass) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= fm || j >= fn) return;
    const bool xo = kx && (i & 1), yo = ky && (j & 1);
    if ((pass == 1) != (xo && yo)) return;
    double a[9];
    op.coef9(i, j, a);
    double *q = P + 4 * (static_cast<long>(i) + static_cast<long>(fm) * j);
    double w[4] = {0, 0, 0, 0};
    const int bx = base_of(i, kx), by = base_of(j, ky);
    const bool v1 = corner_of(bx, 1, cm, px, kx) >= 0, v2 = corner_of(by, 1, cn, py, ky) >= 0;
    if (!xo && !yo) {
        w[0] = 1;
    } else if (xo && !yo) {
        const double L = a[0] + a[3] + a[6], C = a[1] + a[4] + a[7], R = a[2] + a[5] + a[8];
        w[0] = L / (-C);
        if (v1) w[1] = R / (-C);
    } else if (!xo && yo) {
        const double D = a[0] + a[1] + a[2], M = a[3] + a[4] + a[5], U = a[6] + a[7] + a[8];
        w[0] = D / (-M);
        if (v2) w[2] = U / (-M);
    } else {
        double acc[4] = {0, 0, 0, 0};
        for (int dj = -1; dj <= 1; dj++)
            for (int di = -1; di <= 1; di++) {
                const double av = a[3 * (dj + 1) + di + 1];
                if ((di == 0 && dj == 0) || av == 0) continue;
                bool ok = true;
                const int gi = wrap_idx(i + di, fm, px, ok), gj = wrap_idx(j + dj, fn, py, ok);
                if (!ok) continue;
                const double *g = P + 4 * (static_cast<long>(gi) + static_cast<long>(fm) * gj);
                const int ox = base_of(i + di, kx) - bx, oy = base_of(j + dj, ky) - by;
                for (int r = 0; r < 4; r++) {
                    const int cx = ox + (r & 1), cy = oy + (r >> 1);
                    if (g[r] != 0 && cx <= 1 && cy <= 1) acc[cx + 2 * cy] = add_prod(acc[cx + 2 * cy], av, g[r]);
                }
            }
        for (int r = 0; r < 4; r++)
            if (((r & 1) == 0 || v1) && ((r >> 1) == 0 || v2)) w[r] = -acc[r] / a[4];
    }
    q[0] = w[0]; q[1] = w[1]; q[2] = w[2]; q[3] = w[3];
}

/** Galerkin coarse stencil A_c = P^T A P, one thread per coarse unknown
 * (I,J): over the fine points f of its support (the 3 x 3 fine points about
 * (2I,2J)) and the stencil neighbours g of f, P(f,(I,J)) A(f,g) P(g,K) is
 * added to the entry of K - (I,J), K running over g's corners. */
template <class Op>
__global__ void k_galerkin(Op op, int fm, int fn, int px, int py, bool kx, bool ky, int cm, int cn, double *st,
                           const double *P) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x, J = blockIdx.y * blockDim.y + threadIdx.y;
    if (I >= cm || J >= cn) return;
    double q[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int x0 = kx ? 2 * I - 1 : I, x1 = kx ? 2 * I + 1 : I, y0 = ky ? 2 * J - 1 : J, y1 = ky ? 2 * J + 1 : J;
    for (int fj = y0; fj <= y1; fj++)
        for (int fi = x0; fi <= x1; fi++) {
            const double w = pweight(P, fm, fn, px, py, kx, ky, fi, fj, I, J);
            if (w == 0) continue;
            bool ok = true;
            const int i = wrap_idx(fi, fm, px, ok), j = wrap_idx(fj, fn, py, ok);
            double a[9];
            op.coef9(i, j, a);
            for (int dj = -1; dj <= 1; dj++)
                for (int di = -1; di <= 1; di++) {
                    const double av = a[3 * (dj + 1) + di + 1];
                    if (av == 0) continue;
                    bool okg = true;
                    const int gi = wrap_idx(fi + di, fm, px, okg), gj = wrap_idx(fj + dj, fn, py, okg);
                    if (!okg) continue;
                    const double *g = P + 4 * (static_cast<long>(gi) + static_cast<long>(fm) * gj);
                    const int ox = base_of(fi + di, kx) - I, oy = base_of(fj + dj, ky) - J;
                    for (int r = 0; r < 4; r++) {
                        const int kx_ = ox + (r & 1), ky_ = oy + (r >> 1);
                        if (g[r] == 0 || kx_ < -1 || kx_ > 1 || ky_ < -1 || ky_ > 1) continue;
                        double &qe = q[3 * (ky_ + 1) + kx_ + 1];
                        qe = add_prod(qe, __dmul_rn(w, av), g[r]);
                    }
                }
        }
    const long N = static_cast<long>(cm) * cn;
    for (int e = 0; e < 9; e++) st[e * N + colour_index(cm, cn, I, J)] = q[e];
}

/** k_galerkin for a 32 x 8 tile of coarse unknowns per 256-thread block,
 * with every input staged in shared memory first: the nine stencil entries
 * of the fine points of the tile's supports (coef9; the fine region
 * 2X0-1 .. 2(X0+31)+1 in a coarsened direction, X0 .. X0+31 otherwise) and
 * the four prolongation weights of that region grown by one point (the
 * stencil neighbours), zero outside a non-periodic grid. The sums then run
 * exactly as in k_galerkin, in the same order: the same values, without
 * each thread re-reading some four hundred entries from global memory.
 * Dynamic shared memory: galerkin_tile_smem(kx, ky) bytes. */
template <class Op, bool KX, bool KY>
__global__ void __launch_bounds__(256) k_galerkin_tile(Op op, int fm, int fn, int px, int py, int cm, int cn,
                                                       double *st, const double *P) {
    // The coarsening flags are template parameters: with them every loop
    // below has fixed bounds and every offset of a support point or stencil
    // neighbour relative to the coarse point is a constant, so the nine sums
    // stay in registers (indexed at run time they would live in local memory).
    extern __shared__ __align__(16) double gal_smem[];
    constexpr int CTW = 32, CTH = 8;
    constexpr bool kx = KX, ky = KY;
    const int X0 = blockIdx.x * CTW, Y0 = blockIdx.y * CTH;
    const int SX0 = kx ? 2 * X0 - 1 : X0, SY0 = ky ? 2 * Y0 - 1 : Y0;
    constexpr int SW = kx ? 2 * CTW + 1 : CTW, SH = ky ? 2 * CTH + 1 : CTH, SA = SW * SH;
    const int NX0 = SX0 - 1, NY0 = SY0 - 1;
    constexpr int NW = SW + 2, NH = SH + 2;
    double *As = gal_smem;          // entry k of support point t at As[k * SA + t]
    double *Ps = gal_smem + 9 * SA;  // weights of region point t at Ps[4 * t .. 4 * t + 3]
    // Only the supports of coarse points I < cm, J < cn (fine x up to sxmax)
    // and their stencil neighbours (one further) are read below. Beyond them
    // the region of a level smaller than the tile would reach more than one
    // period past a periodic grid, where one wrap does not bring an index
    // back inside it: such points are not staged.
    const int sxmax = kx ? 2 * cm - 1 : cm - 1, symax = ky ? 2 * cn - 1 : cn - 1;
    for (int t = threadIdx.x; t < NW * NH; t += blockDim.x) {
        const int xu = NX0 + t % NW, yu = NY0 + t / NW;
        bool ok = xu <= sxmax + 1 && yu <= symax + 1;
        const int i = wrap_idx(xu, fm, px, ok), j = wrap_idx(yu, fn, py, ok);
        double w[4] = {0, 0, 0, 0};
        if (ok) {
            const double *q = P + 4 * (static_cast<long>(i) + static_cast<long>(fm) * j);
            w[0] = q[0]; w[1] = q[1]; w[2] = q[2]; w[3] = q[3];
        }
        Ps[4 * t] = w[0]; Ps[4 * t + 1] = w[1]; Ps[4 * t + 2] = w[2]; Ps[4 * t + 3] = w[3];
    }
    for (int t = threadIdx.x; t < SA; t += blockDim.x) {
        const int xu = SX0 + t % SW, yu = SY0 + t / SW;
        bool ok = xu <= sxmax && yu <= symax;
        const int i = wrap_idx(xu, fm, px, ok), j = wrap_idx(yu, fn, py, ok);
        if (!ok) continue;  // outside the grid (weight zero) or no support of the tile: never read
        double a[9];
        op.coef9(i, j, a);
#pragma unroll
        for (int k = 0; k < 9; k++) As[k * SA + t] = a[k];
    }
    __syncthreads();
    const int I = X0 + (threadIdx.x & 31), J = Y0 + (threadIdx.x >> 5);
    if (I >= cm || J >= cn) return;
    double q[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    // Support points fi = 2I-1+u (u = 0..2) in a coarsened direction, fi = I
    // otherwise; visited in the order of k_galerkin (rows, then columns).
    // Relative to I: base_of(fi) - I = floor((u-1)/2) there, 0 otherwise.
    const int x0 = kx ? 2 * I - 1 : I, y0 = ky ? 2 * J - 1 : J;
#pragma unroll
    for (int v = 0; v <= (ky ? 2 : 0); v++)
#pragma unroll
        for (int u = 0; u <= (kx ? 2 : 0); u++) {
            const int fi = x0 + u, fj = y0 + v;
            // pweight(fi, fj, I, J) from the staged weights
            const int qx = kx ? -((u - 1) >> 1) : 0, qy = ky ? -((v - 1) >> 1) : 0;
            if (qx < 0 || qx > 1 || qy < 0 || qy > 1) continue;
            const double w = Ps[4 * ((fi - NX0) + NW * (fj - NY0)) + qx + 2 * qy];
            if (w == 0) continue;
            const int ls = (fi - SX0) + SW * (fj - SY0);
#pragma unroll
            for (int dj = -1; dj <= 1; dj++)
#pragma unroll
                for (int di = -1; di <= 1; di++) {
                    const double av = As[(3 * (dj + 1) + di + 1) * SA + ls];
                    if (av == 0) continue;
                    const double *g = Ps + 4 * ((fi + di - NX0) + NW * (fj + dj - NY0));
                    const int ox = kx ? ((u - 1 + di) >> 1) : di, oy = ky ? ((v - 1 + dj) >> 1) : dj;
#pragma unroll
                    for (int r = 0; r < 4; r++) {
                        const int kx_ = ox + (r & 1), ky_ = oy + (r >> 1);
                        if (kx_ < -1 || kx_ > 1 || ky_ < -1 || ky_ > 1) continue;
                        if (g[r] == 0) continue;
                        double &qe = q[3 * (ky_ + 1) + kx_ + 1];
                        qe = add_prod(qe, __dmul_rn(w, av), g[r]);
                    }
                }
        }
    const long N = static_cast<long>(cm) * cn;
    const long qi = colour_index(cm, cn, I, J);
#pragma unroll
    for (int e = 0; e < 9; e++) st[e * N + qi] = q[e];
}

/** The shared-memory limit of every k_galerkin_tile instance of Op. */
template <class Op>
cudaError_t set_galerkin_attr(int bytes) {
    cudaError_t e = cudaFuncSetAttribute(k_galerkin_tile<Op, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_galerkin_tile<Op, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_galerkin_tile<Op, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return e;
}

/** Shared memory of k_galerkin_tile for the coarsening flags. */
inline size_t galerkin_tile_smem(bool kx, bool ky) {
    const int SW = kx ? 65 : 32, SH = ky ? 17 : 8;
    return sizeof(double) * (9 * SW * SH + 4 * (SW + 2) * (SH + 2));
}

/** Single-precision copy of a level's Galerkin stencils (entry k of unknown
 * q at k*N+q) for the centred FP32 cycles: entry 4 holds the row sum of the
 * FP64 stencil, summed in FP64, instead of the diagonal. */
__global__ void k_cast_stencil(const double *st, float *stf, long N) {
    for (long q = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; q < N;
         q += static_cast<long>(gridDim.x) * blockDim.x) {
        double rs = 0;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const double v = st[k * N + q];
            rs += v;
            if (k != 4) stf[k * N + q] = static_cast<float>(v);
        }
        stf[4 * N + q] = static_cast<float>(rs);
    }
}

// ---------------------------------------------------------------------------
// V-cycle kernels.

/** One colour (pi,pj) of a Gauss-Seidel sweep: z = (b - offdiag)/diag. */
template <class Op, class T>
__global__ void k_smooth(Op op, T *z, const T *b, int m, int n, int pi, int pj) {
    const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + pi;
    const int j = 2 * (blockIdx.y * blockDim.y + threadIdx.y) + pj;
    if (i >= m || j >= n) return;
    const int ij = i + m * j;
    z[ij] = gs_update(op, i, j, z, b[ij]);
}

/** Index i of a periodic direction of size m brought into [0, m). */
__device__ __forceinline__ int wrap_index(int i, int m) {
    i %= m;
    return i < 0 ? i + m : i;
}

/** Tile-fused Gauss-Seidel: SWEEPS complete four-colour sweeps in one launch.
 * The block stages its TW x TH tile of the iterate zin plus a halo of
 * 4*SWEEPS cells in shared memory and runs the colour phases there, phase p
 * updating the tile grown by 4*SWEEPS-1-p cells, so that every value a later
 * phase reads is already final; the tile is then written to zout. zin is not
 * written during the launch, so every block stages the values from before the
 * sweeps and each point sees exactly the neighbour values of the
 * one-launch-per-colour schedule: the result is identical to it. In a
 * periodic direction (even size) the halo holds periodic images, updated like
 * the points they copy (the colouring is consistent across the seam).
 * Coefficients and the right-hand side are read from global memory (L1/L2). */
template <class Op, class T, int SWEEPS, int TW, int TH>
__global__ void __launch_bounds__(256) k_smooth_tile(Op op, const T *zin, T *zout, const T *b, int m, int n) {
    constexpr int H = 4 * SWEEPS, LW = TW + 2 * H, LH = TH + 2 * H;
    __shared__ T zs[LW * LH];
    const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
    const int gx0 = x0 - H, gy0 = y0 - H;
    const bool px = op.px, py = op.py;
    for (int t = threadIdx.x; t < LW * LH; t += blockDim.x) {
        int i = gx0 + t % LW, j = gy0 + t / LW;
        if (px) i = wrap_index(i, m);
        if (py) j = wrap_index(j, n);
        if (i >= 0 && i < m && j >= 0 && j < n) zs[t] = zin[i + static_cast<long>(m) * j];
    }
    __syncthreads();
    const int pis[4] = {0, 1, 1, 0}, pjs[4] = {0, 1, 0, 1};
    constexpr int P = 4 * SWEEPS;
#pragma unroll 1
    for (int p = 0; p < P; p++) {
        const int e = P - 1 - p, c = p & 3;
        int ilo = x0 - e, ihi = x0 + TW - 1 + e, jlo = y0 - e, jhi = y0 + TH - 1 + e;
        if (!px) {
            if (ilo < 0) ilo = 0;
            if (ihi > m - 1) ihi = m - 1;
        }
        if (!py) {
            if (jlo < 0) jlo = 0;
            if (jhi > n - 1) jhi = n - 1;
        }
        // first index of the colour's parity at or above the low bound
        const int i0 = ilo + ((ilo & 1) != pis[c]), j0 = jlo + ((jlo & 1) != pjs[c]);
        const int ni = i0 <= ihi ? (ihi - i0) / 2 + 1 : 0, nj = j0 <= jhi ? (jhi - j0) / 2 + 1 : 0;
        for (int t = threadIdx.x; t < ni * nj; t += blockDim.x) {
            const int i = i0 + 2 * (t % ni), j = j0 + 2 * (t / ni);
            const int lz = (i - gx0) + LW * (j - gy0);
            const int ir = px ? wrap_index(i, m) : i, jr = py ? wrap_index(j, n) : j;
            zs[lz] = gs_update_s(op, ir, jr, zs, lz, LW, b[ir + static_cast<long>(m) * jr]);
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < TW * TH; t += blockDim.x) {
        const int i = x0 + t % TW, j = y0 + t / TW;
        if (i < m && j < n) zout[i + static_cast<long>(m) * j] = zs[(i - gx0) + LW * (j - gy0)];
    }
}

/** k_smooth_tile for the Galerkin levels' nine-point stencils with every
 * input staged up front: the nine coefficients and the right-hand side of the
 * whole halo region go to shared memory with the iterate before the first
 * phase, so the colour phases run on shared memory alone instead of waiting
 * on L2 for the coefficients in each of them (the small coarse levels are
 * latency-bound). The arithmetic, and so the result, is that of
 * k_smooth_tile. Dynamic shared memory: (11 * LW * LH) elements. */
template <class T, int SWEEPS, int TW, int TH>
__global__ void __launch_bounds__(256) k_smooth_tile_gen(GenOp<T> op, const T *zin, T *zout, const T *b, int m,
                                                         int n) {
    constexpr int H = 4 * SWEEPS, LW = TW + 2 * H, LH = TH + 2 * H, LA = LW * LH;
    extern __shared__ __align__(16) unsigned char gen_smem[];
    T *zs = reinterpret_cast<T *>(gen_smem);
    T *bs = zs + LA;
    T *cs = bs + LA;  // coefficient k of local point t at cs[k * LA + t]
    const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
    const int gx0 = x0 - H, gy0 = y0 - H;
    const bool px = op.px, py = op.py;
    const long N = op.N;
    for (int t = threadIdx.x; t < LA; t += blockDim.x) {
        int i = gx0 + t % LW, j = gy0 + t / LW;
        if (px) i = wrap_index(i, m);
        if (py) j = wrap_index(j, n);
        if (i >= 0 && i < m && j >= 0 && j < n) {
            const long ij = i + static_cast<long>(m) * j;
            zs[t] = zin[ij];
            bs[t] = b[ij];
            const long q = op.at(i, j);
#pragma unroll
            for (int k = 0; k < 9; k++) cs[k * LA + t] = op.st[k * N + q];
        }
    }
    __syncthreads();
    const int pis[4] = {0, 1, 1, 0}, pjs[4] = {0, 1, 0, 1};
    constexpr int P = 4 * SWEEPS;
#pragma unroll 1
    for (int p = 0; p < P; p++) {
        const int e = P - 1 - p, c = p & 3;
        int ilo = x0 - e, ihi = x0 + TW - 1 + e, jlo = y0 - e, jhi = y0 + TH - 1 + e;
        if (!px) {
            if (ilo < 0) ilo = 0;
            if (ihi > m - 1) ihi = m - 1;
        }
        if (!py) {
            if (jlo < 0) jlo = 0;
            if (jhi > n - 1) jhi = n - 1;
        }
        const int i0 = ilo + ((ilo & 1) != pis[c]), j0 = jlo + ((jlo & 1) != pjs[c]);
        const int ni = i0 <= ihi ? (ihi - i0) / 2 + 1 : 0, nj = j0 <= jhi ? (jhi - j0) / 2 + 1 : 0;
        for (int t = threadIdx.x; t < ni * nj; t += blockDim.x) {
            const int i = i0 + 2 * (t % ni), j = j0 + 2 * (t / ni);
            const int lz = (i - gx0) + LW * (j - gy0);
            const int ir = px ? wrap_index(i, m) : i, jr = py ? wrap_index(j, n) : j;
            // gs_update_s of GenOp with the coefficients read from shared
            // memory (in single precision entry 4 is the row sum and the
            // neighbours enter centred)
            const bool l = px || ir > 0, r = px || ir < m - 1, d = py || jr > 0, u = py || jr < n - 1;
            const T zc = sizeof(T) == 8 ? T(0) : zs[lz];
            T diag = cs[4 * LA + lz];
            const T rs = diag;  // the row sum in single precision
            const T s = GenOp<T>::template gen_sum<sizeof(T) == 4>(l, r, d, u, cs + lz, LA, zs + lz, 1, LW, zc, diag);
            zs[lz] = gs_value(bs[lz], s, diag, zc, rs);
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < TW * TH; t += blockDim.x) {
        const int i = x0 + t % TW, j = y0 + t / TW;
        if (i < m && j < n) zout[i + static_cast<long>(m) * j] = zs[(i - gx0) + LW * (j - gy0)];
    }
}

/** Shared memory of k_smooth_tile_gen<T, SWEEPS, TW, TH>. */
template <class T, int SWEEPS = 2, int TW = 16, int TH = 16>
constexpr int gen_tile_smem() {
    return 11 * (TW + 8 * SWEEPS) * (TH + 8 * SWEEPS) * static_cast<int>(sizeof(T));
}

/** Tile-fused red-black Gauss-Seidel for a five-point operator (the fine MAC
 * system): the colours (0,0),(1,1) share no stencil edge, nor do (1,0),(0,1),
 * so the four-colour sweep is exactly two half-sweeps over (i+j) even, then
 * odd, with bitwise the same results. SWEEPS sweeps take 2*SWEEPS phases, so
 * the halo is 2*SWEEPS cells. Threads walk the tile as 32 x 8 (x fastest),
 * each row of a phase holding every second point. Reads zin, writes zout, and
 * handles periodic directions (even sizes) like k_smooth_tile. */
template <class Op, class T, int SWEEPS, int TW, int TH>
__global__ void __launch_bounds__(256) k_smooth_rb(Op op, const T *zin, T *zout, const T *b, int m, int n) {
    constexpr int H = 2 * SWEEPS, LW = TW + 2 * H, LH = TH + 2 * H, NP = 2 * SWEEPS;
    __shared__ T zs[LW * LH];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
    const int gx0 = x0 - H, gy0 = y0 - H;
    const bool px = op.px, py = op.py;
    for (int lj = ty; lj < LH; lj += 8) {
        int j = gy0 + lj;
        if (py) j = wrap_index(j, n);
        if (j < 0 || j >= n) continue;
        for (int li = tx; li < LW; li += 32) {
            int i = gx0 + li;
            if (px) i = wrap_index(i, m);
            if (i >= 0 && i < m) zs[li + LW * lj] = zin[i + static_cast<long>(m) * j];
        }
    }
    __syncthreads();
#pragma unroll 1
    for (int p = 0; p < NP; p++) {
        const int e = NP - 1 - p, parity = p & 1;
        int ilo = x0 - e, ihi = x0 + TW - 1 + e, jlo = y0 - e, jhi = y0 + TH - 1 + e;
        if (!px) {
            if (ilo < 0) ilo = 0;
            if (ihi > m - 1) ihi = m - 1;
        }
        if (!py) {
            if (jlo < 0) jlo = 0;
            if (jhi > n - 1) jhi = n - 1;
        }
        for (int j = jlo + ty; j <= jhi; j += 8) {
            const int i0 = ilo + (((ilo + j) & 1) != parity);
            const int jr = py ? wrap_index(j, n) : j;
            for (int i = i0 + 2 * tx; i <= ihi; i += 64) {
                const int lz = (i - gx0) + LW * (j - gy0);
                const int ir = px ? wrap_index(i, m) : i;
                zs[lz] = gs_update_s(op, ir, jr, zs, lz, LW, b[ir + static_cast<long>(m) * jr]);
            }
        }
        __syncthreads();
    }
    for (int lj = H + ty; lj < H + TH; lj += 8) {
        const int j = gy0 + lj;
        if (j >= n) break;
        for (int li = H + tx; li < H + TW; li += 32) {
            const int i = gx0 + li;
            if (i < m) zout[i + static_cast<long>(m) * j] = zs[li + LW * lj];
        }
    }
}

/** Coarse right-hand side b_c = P^T (b - A z), the fine residual formed on
 * the fly; also clears the coarse iterate. */
template <class Op, class T>
__global__ void k_restrict(Op op, const T *z, const T *b, int fm, int fn, int px, int py,
                           bool kx, bool ky, int cm, int cn, T *bc, T *zc, const double *P) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x, J = blockIdx.y * blockDim.y + threadIdx.y;
    if (I >= cm || J >= cn) return;
    const int x0 = kx ? 2 * I - 1 : I, x1 = kx ? 2 * I + 1 : I, y0 = ky ? 2 * J - 1 : J, y1 = ky ? 2 * J + 1 : J;
    T t = 0;
    for (int fj = y0; fj <= y1; fj++)
        for (int fi = x0; fi <= x1; fi++) {
            const T w = static_cast<T>(pweight(P, fm, fn, px, py, kx, ky, fi, fj, I, J));
            if (w == 0) continue;
            bool ok = true;
            const int i = wrap_idx(fi, fm, px, ok), j = wrap_idx(fj, fn, py, ok);
            const int f = i + fm * j;
            t = add_prod(t, w, residual_at(op, i, j, z, b[f]));
        }
    bc[I + cm * J] = t;
    zc[I + cm * J] = 0;
}

/** k_restrict for a 32 x 8 tile of coarse unknowns per 256-thread block,
 * each fine residual computed once: the block first evaluates b - A z at
 * every fine unknown of its coarse points' supports (the fine region
 * 2X0-1 .. 2(X0+31)+1 in a coarsened direction, X0 .. X0+31 otherwise) into
 * shared memory, then every coarse point sums its support's residuals with
 * the weights and in the order of k_restrict: the same values. */
template <class Op, class T, bool KX, bool KY>
__global__ void __launch_bounds__(256) k_restrict_tile(Op op, const T *z, const T *b, int fm, int fn, int px, int py,
                                                       int cm, int cn, T *bc, T *zc, const double *P) {
    // The coarsening flags are template parameters, so the region's width
    // (the divisor of the staging loop's index) is a constant.
    constexpr bool kx = KX, ky = KY;
    constexpr int CTW = 32, CTH = 8, RW = 2 * CTW + 1, RH = 2 * CTH + 1;
    __shared__ T rs[RW * RH];
    __shared__ double ps[4 * RW * RH];  // the region's prolongation weights (zero outside the grid)
    const int X0 = blockIdx.x * CTW, Y0 = blockIdx.y * CTH;
    const int FX0 = kx ? 2 * X0 - 1 : X0, FY0 = ky ? 2 * Y0 - 1 : Y0;
    constexpr int FW = kx ? RW : CTW, FH = ky ? RH : CTH;
    // Only fine unknowns in the support of a coarse point I < cm, J < cn are
    // needed (and beyond them a periodic index could wrap past the grid).
    const int fxmax = kx ? 2 * cm - 1 : cm - 1, fymax = ky ? 2 * cn - 1 : cn - 1;
    for (int t = threadIdx.x; t < FW * FH; t += blockDim.x) {
        const int fxu = FX0 + t % FW, fyu = FY0 + t / FW;
        bool ok = fxu <= fxmax && fyu <= fymax;
        const int fx = wrap_idx(fxu, fm, px, ok), fy = wrap_idx(fyu, fn, py, ok);
        T r = 0;
        double w0 = 0, w1 = 0, w2 = 0, w3 = 0;
        if (ok) {
            const int f = fx + fm * fy;
            r = residual_at(op, fx, fy, z, b[f]);
            // four weights per fine point: 32-byte aligned, two 16-byte loads
            const double2 *q = reinterpret_cast<const double2 *>(P + 4 * static_cast<long>(f));
            const double2 q01 = q[0], q23 = q[1];
            w0 = q01.x; w1 = q01.y; w2 = q23.x; w3 = q23.y;
        }
        rs[t] = r;
        ps[4 * t] = w0; ps[4 * t + 1] = w1; ps[4 * t + 2] = w2; ps[4 * t + 3] = w3;
    }
    __syncthreads();
    const int I = X0 + (threadIdx.x & 31), J = Y0 + (threadIdx.x >> 5);
    if (I >= cm || J >= cn) return;
    // The support in k_restrict's order, each fine point read from its
    // (unwrapped) position in the staged region.
    const int x0 = kx ? 2 * I - 1 : I, x1 = kx ? 2 * I + 1 : I, y0 = ky ? 2 * J - 1 : J, y1 = ky ? 2 * J + 1 : J;
    T t = 0;
    for (int fj = y0; fj <= y1; fj++)
        for (int fi = x0; fi <= x1; fi++) {
            // pweight(fi, fj, I, J) from the staged weights
            const int qx = I - base_of(fi, kx), qy = J - base_of(fj, ky);
            if (qx < 0 || qx > 1 || qy < 0 || qy > 1) continue;
            const int lt = (fi - FX0) + FW * (fj - FY0);
            const T w = static_cast<T>(ps[4 * lt + qx + 2 * qy]);
            if (w == 0) continue;
            t = add_prod(t, w, rs[lt]);
        }
    bc[I + cm * J] = t;
    zc[I + cm * J] = 0;
}

/** Fine correction z_f += P z_c, from the point's four stored weights. */
template <class T>
__global__ void k_prolong(T *zf, int fm, int fn, int px, int py, bool kx, bool ky,
                          const T *zc, int cm, int cn, const double *P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= fm || j >= fn) return;
    const long f = i + static_cast<long>(fm) * j;
    const double2 *q2 = reinterpret_cast<const double2 *>(P + 4 * f);  // 32-byte aligned
    const double2 q01 = q2[0], q23 = q2[1];
    const double q[4] = {q01.x, q01.y, q23.x, q23.y};
    const int bx = base_of(i, kx), by = base_of(j, ky);
    T t = 0;
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const double w = q[r];
        if (w == 0) continue;
        const int I = corner_of(bx, r & 1, cm, px, kx), J = corner_of(by, r >> 1, cn, py, ky);
        if (I < 0 || J < 0) continue;  // k_build_p leaves such corners at 0
        t = add_prod(t, static_cast<T>(w), zc[I + cm * J]);
    }
    zf[f] += t;
}

/** Coarsest-level solve: `sweeps` four-colour Gauss-Seidel sweeps by one
 * block, with a block barrier between colours. */
template <class Op, class T>
__global__ void k_coarse(Op op, T *z, const T *b, int m, int n, int sweeps) {
    const int pis[4] = {0, 1, 1, 0}, pjs[4] = {0, 1, 0, 1};
    for (int s = 0; s < sweeps; s++) {
        for (int c = 0; c < 4; c++) {
            const int mc = (m - pis[c] + 1) / 2, nc = (n - pjs[c] + 1) / 2;
            for (int p = threadIdx.x; p < mc * nc; p += blockDim.x) {
                const int i = 2 * (p % mc) + pis[c], j = 2 * (p / mc) + pjs[c];
                z[i + m * j] = gs_update(op, i, j, z, b[i + m * j]);
            }
            __syncthreads();
        }
    }
}

/** Coarse levels with at most this many unknowns are solved exactly. */
constexpr int kDirectMax = 96;

/** Dense inverse of the coarsest Galerkin operator, one block, Gauss-Jordan
 * with partial pivoting on [A | I] in shared memory. The singular
 * pure-Neumann operator (zero row sums) is regularised by c e e^T, c the
 * mean |diagonal| / N, which gives the zero-mean solution of a compatible
 * system. Writes the FP64 inverse and an FP32 copy. */
__global__ void k_coarse_inverse(const double *st, int m, int n, int px, int py, double *ginv, float *ginvf) {
    extern __shared__ __align__(16) double gj[];
    const int N = m * n, W = 2 * N;
    double *a = gj, *f = gj + static_cast<long>(N) * W;
    __shared__ double red[32];
    __shared__ int piv;
    __shared__ bool singular;
    __shared__ double creg;
    for (int q = threadIdx.x; q < N * W; q += blockDim.x) a[q] = 0;
    __syncthreads();
    double rsmax = 0, dsum = 0;
    for (int r = threadIdx.x; r < N; r += blockDim.x) {
        const int i = r % m, j = r / m;
        double rs = 0;
        for (int dj = -1; dj <= 1; dj++) {
            bool oky = true;
            const int jj = wrap_idx(j + dj, n, py, oky);
            if (!oky) continue;
            for (int di = -1; di <= 1; di++) {
                bool okx = true;
                const int ii = wrap_idx(i + di, m, px, okx);
                if (!okx) continue;
                const double v = st[(3 * (dj + 1) + di + 1) * static_cast<long>(N) + colour_index(m, n, i, j)];
                a[static_cast<long>(r) * W + ii + m * jj] += v;
                rs += v;
            }
        }
        rsmax = fmax(rsmax, fabs(rs));
        dsum += fabs(st[4 * static_cast<long>(N) + colour_index(m, n, i, j)]);
        a[static_cast<long>(r) * W + N + r] = 1;
    }
    // block max / sum (1024 threads = 32 warps)
    for (int o = 16; o > 0; o >>= 1) {
        rsmax = fmax(rsmax, __shfl_down_sync(0xffffffffu, rsmax, o));
        dsum += __shfl_down_sync(0xffffffffu, dsum, o);
    }
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    if (lane == 0) red[wp] = rsmax;
    __syncthreads();
    if (threadIdx.x == 0) {
        double mx = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) mx = fmax(mx, red[w]);
        creg = mx;
    }
    __syncthreads();
    if (lane == 0) red[wp] = dsum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double sm = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) sm += red[w];
        singular = creg <= 1e-10 * sm / N;
        creg = sm / N / N;
    }
    __syncthreads();
    if (singular)
        for (int q = threadIdx.x; q < N * N; q += blockDim.x) a[static_cast<long>(q / N) * W + q % N] += creg;
    __syncthreads();
    for (int k = 0; k < N; k++) {
        if (threadIdx.x < 32) {
            // warp argmax of |a(r,k)|, r >= k; ties go to the lower row
            int p = -1;
            double best = -1;
            for (int r = k + threadIdx.x; r < N; r += 32) {
                const double v = fabs(a[static_cast<long>(r) * W + k]);
                if (v > best) { best = v; p = r; }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_down_sync(0xffffffffu, best, o);
                const int op_ = __shfl_down_sync(0xffffffffu, p, o);
                if (ob > best || (ob == best && op_ >= 0 && (p < 0 || op_ < p))) { best = ob; p = op_; }
            }
            // no candidate compares (a NaN column): keep row k, so the
            // inverse comes out NaN and the solve reports it, and no row
            // outside the matrix is touched
            if (threadIdx.x == 0) piv = p < 0 ? k : p;
        }
        __syncthreads();
        const int p = piv;
        if (p != k)
            for (int q = threadIdx.x; q < W; q += blockDim.x) {
                const double t = a[static_cast<long>(k) * W + q];
                a[static_cast<long>(k) * W + q] = a[static_cast<long>(p) * W + q];
                a[static_cast<long>(p) * W + q] = t;
            }
        __syncthreads();
        const double iv = 1.0 / a[static_cast<long>(k) * W + k];
        __syncthreads();
        for (int q = threadIdx.x; q < W; q += blockDim.x) a[static_cast<long>(k) * W + q] *= iv;
        for (int r = threadIdx.x; r < N; r += blockDim.x) f[r] = a[static_cast<long>(r) * W + k];
        __syncthreads();
        for (long q = threadIdx.x; q < static_cast<long>(N) * W; q += blockDim.x) {
            const int r = static_cast<int>(q / W);
            if (r == k || f[r] == 0) continue;
            a[q] -= f[r] * a[static_cast<long>(k) * W + q % W];
        }
        __syncthreads();
    }
    for (int q = threadIdx.x; q < N * N; q += blockDim.x) {
        const double v = a[static_cast<long>(q / N) * W + N + q % N];
        ginv[q] = v;
        ginvf[q] = static_cast<float>(v);
    }
}

/** Coarsest solve by the dense inverse: z = G b. */
template <class T>
__device__ __forceinline__ void coarse_direct(const T *G, const T *b, T *z, int N) {
    for (int r = threadIdx.x; r < N; r += blockDim.x) {
        T t = 0;
        for (int q = 0; q < N; q++) t += G[static_cast<long>(r) * N + q] * b[q];
        z[r] = t;
    }
}

template <class T>
__global__ void k_coarse_direct(const T *G, const T *b, T *z, int N) {
    coarse_direct(G, b, z, N);
}

/** Levels handled by the one-block tail kernel. */
constexpr int kTailMaxLevels = 12;
constexpr int kTailMaxSize = 1024;  // unknowns of the first tail level at most
constexpr size_t kTailSmemBudget = 160 * 1024;  // shared memory for the smallest tail levels

template <class T>
struct TailLevels {
    int first, count, px, py;
    const double *P[kTailMaxLevels]; // prolongation weights of each tail level but the last
    int smem_from;                 // levels >= smem_from live in shared memory
    const T *ginv;                 // dense inverse of the coarsest level, or null
    long smem_off[kTailMaxLevels]; // element offsets of st, then z, then b
    int m[kTailMaxLevels], n[kTailMaxLevels];
    long N[kTailMaxLevels];
    bool kx[kTailMaxLevels], ky[kTailMaxLevels];
    T *z[kTailMaxLevels];
    T *b[kTailMaxLevels];
    const T *st[kTailMaxLevels];
};

template <class T>
__device__ __forceinline__ GenOp<T> tail_op(const TailLevels<T> &L, int l) {
    GenOp<T> g; g.m = L.m[l]; g.n = L.n[l]; g.px = L.px; g.py = L.py; g.N = L.N[l]; g.st = L.st[l];
    return g;
}

/** Smoothing of one tail level. Levels of at most kWarpLevel unknowns are
 * swept by the first warp alone with warp barriers (a block barrier per
 * colour phase would dominate there); the block waits once at the end. */
constexpr int kWarpLevel = 256;

template <class T>
__device__ void tail_smooth(const TailLevels<T> &L, int l, int sweeps) {
    const int pis[4] = {0, 1, 1, 0}, pjs[4] = {0, 1, 0, 1};
    const GenOp<T> op = tail_op(L, l);
    const int m = L.m[l], n = L.n[l];
    T *z = L.z[l];
    const T *b = L.b[l];
    const bool warp_only = m * n <= kWarpLevel;
    if (warp_only && threadIdx.x >= 32) { __syncthreads(); return; }
    const int nth = warp_only ? 32 : blockDim.x;
    for (int s = 0; s < sweeps; s++)
        for (int c = 0; c < 4; c++) {
            const int mc = (m - pis[c] + 1) / 2, nc = (n - pjs[c] + 1) / 2;
            for (int p = threadIdx.x; p < mc * nc; p += nth) {
                const int i = 2 * (p % mc) + pis[c], j = 2 * (p / mc) + pjs[c];
                z[i + m * j] = gs_update(op, i, j, z, b[i + m * j]);
            }
            if (warp_only) __syncwarp();
            else __syncthreads();
        }
    if (warp_only) __syncthreads();
}

/** The V-cycle below (and including) level L.first in one block: smoothing,
 * restriction and prolongation of every tail level with block barriers
 * between phases, and the coarsest solve. The levels are small enough to sit
 * in L2, so the cost is the barriers rather than launches. */
template <class T>
__global__ void __launch_bounds__(1024) k_tail(TailLevels<T> Lp, int nu1, int nu2, int coarse_sweeps) {
    // The smallest levels are moved into shared memory: stencils copied in,
    // iterate and right-hand side written there by the restriction.
    extern __shared__ __align__(16) unsigned char tail_smem[];
    T *sbase = reinterpret_cast<T *>(tail_smem);
    TailLevels<T> L = Lp;
    for (int l = L.smem_from; l < L.count; l++) {
        T *st = sbase + L.smem_off[l];
        const long n9 = 9 * L.N[l];
        for (long q = threadIdx.x; q < n9; q += blockDim.x) st[q] = L.st[l][q];
        if (l == 0) {
            // the first tail level's right-hand side and iterate come from the
            // restriction before the tail; its iterate goes back at the end
            for (long q = threadIdx.x; q < L.N[0]; q += blockDim.x) {
                st[n9 + q] = L.z[0][q];
                st[n9 + L.N[0] + q] = L.b[0][q];
            }
        }
        L.st[l] = st;
        L.z[l] = st + n9;
        L.b[l] = st + n9 + L.N[l];
    }
    __syncthreads();
    const int last = L.count - 1;
    for (int l = 0; l < last; l++) {
        tail_smooth(L, l, nu1);
        const GenOp<T> op = tail_op(L, l);
        const int fm = L.m[l], fn = L.n[l], cm = L.m[l + 1], cn = L.n[l + 1];
        const bool kx = L.kx[l], ky = L.ky[l];
        for (int q = threadIdx.x; q < cm * cn; q += blockDim.x) {
            const int I = q % cm, J = q / cm;
            const int x0 = kx ? 2 * I - 1 : I, x1 = kx ? 2 * I + 1 : I, y0 = ky ? 2 * J - 1 : J,
                      y1 = ky ? 2 * J + 1 : J;
            T t = 0;
            for (int fj = y0; fj <= y1; fj++)
                for (int fi = x0; fi <= x1; fi++) {
                    const T w = static_cast<T>(pweight(L.P[l], fm, fn, L.px, L.py, kx, ky, fi, fj, I, J));
                    if (w == 0) continue;
                    bool ok = true;
                    const int i = wrap_idx(fi, fm, L.px, ok), j = wrap_idx(fj, fn, L.py, ok);
                    const int f = i + fm * j;
                    t = add_prod(t, w, residual_at(op, i, j, static_cast<const T *>(L.z[l]), L.b[l][f]));
                }
            L.b[l + 1][q] = t;
            L.z[l + 1][q] = 0;
        }
        __syncthreads();
    }
    if (L.ginv) {
        coarse_direct(L.ginv, L.b[last], L.z[last], static_cast<int>(L.N[last]));
        __syncthreads();
    } else {
        tail_smooth(L, last, coarse_sweeps);
    }
    for (int l = last - 1; l >= 0; l--) {
        const int fm = L.m[l], fn = L.n[l], cm = L.m[l + 1], cn = L.n[l + 1];
        for (int q = threadIdx.x; q < fm * fn; q += blockDim.x) {
            const int i = q % fm, j = q / fm;
            const double *w = L.P[l] + 4 * static_cast<long>(q);
            const int bx = base_of(i, L.kx[l]), by = base_of(j, L.ky[l]);
            T t = 0;
            for (int r = 0; r < 4; r++) {
                if (w[r] == 0) continue;
                const int I = corner_of(bx, r & 1, cm, L.px, L.kx[l]), J = corner_of(by, r >> 1, cn, L.py, L.ky[l]);
                if (I < 0 || J < 0) continue;
                t = add_prod(t, static_cast<T>(w[r]), L.z[l + 1][I + cm * J]);
            }
            L.z[l][q] += t;
        }
        __syncthreads();
        tail_smooth(L, l, nu2);
    }
    if (L.smem_from == 0)
        for (long q = threadIdx.x; q < L.N[0]; q += blockDim.x) Lp.z[0][q] = L.z[0][q];
}

/** FP64 residual r = b - A z, optionally stored in FP32, with per-block sums
 * of r^2 in partial[blockIdx.x]. Each block takes every gridDim.x-th row,
 * its threads the row's unknowns (coalesced, no index division). */
template <class Op>
__global__ void k_resnorm(Op op, const double *z, const double *b, int m, int n, float *rf,
                          double *partial) {
    double acc = 0;
    for (int j = blockIdx.x; j < n; j += gridDim.x)
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            const long q = i + static_cast<long>(m) * j;
            double diag;
            const double off = op.offdiag(i, j, z, diag);
            const double r = fma_rn(-diag, z[q], sub_rn(b[q], off));
            if (rf) rf[q] = static_cast<float>(r);
            acc += r * r;
        }
    acc = block_sum_256(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

/** out = A z. */
template <class Op>
__global__ void k_apply(Op op, const double *z, double *out, int m, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= m || j >= n) return;
    double diag;
    const double off = op.offdiag(i, j, z, diag);
    out[i + m * j] = fma_rn(diag, z[i + m * j], off);
}

__global__ void k_sumsq(const double *b, long N, double *partial) {
    double acc = 0;
    for (long q = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; q < N;
         q += static_cast<long>(gridDim.x) * blockDim.x)
        acc += b[q] * b[q];
    acc = block_sum_256(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

/** Sums nb partials in a fixed order (one block), so results are reproducible. */
__global__ void k_reduce(const double *partial, int nb, double *out) {
    double acc = 0;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) acc += partial[q];
    acc = block_sum_256(acc);
    if (threadIdx.x == 0) *out = acc;
}

/** Per-block sums of an FP32 array, accumulated in FP64. */
__global__ void k_sum_f32(const float *a, long N, double *partial) {
    double acc = 0;
    for (long q = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; q < N;
         q += static_cast<long>(gridDim.x) * blockDim.x)
        acc += static_cast<double>(a[q]);
    acc = block_sum_256(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

/** z += e - mean(e), the mean from the sum in *sum (a correction of a
 * singular system, defined up to a constant). */
__global__ void k_add_f32_centred(double *z, const float *e, long N, const double *sum) {
    const double mean = *sum / static_cast<double>(N);
    for (long q = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; q < N;
         q += static_cast<long>(gridDim.x) * blockDim.x)
        z[q] += static_cast<double>(e[q]) - mean;
}

__global__ void k_add_f32(double *z, const float *e, long N) {
    for (long q = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; q < N;
         q += static_cast<long>(gridDim.x) * blockDim.x)
        z[q] += static_cast<double>(e[q]);
}

template <class T>
__global__ void k_fill(T *a, long N, T v) {
    for (long q = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; q < N;
         q += static_cast<long>(gridDim.x) * blockDim.x)
        a[q] = v;
}

/** Zeroes the right-hand side on the fixed right column (mgs_fem.cc:112). */
__global__ void k_zero_column(double *b, int m, int n) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) b[m - 1 + m * j] = 0;
}

// ---------------------------------------------------------------------------
// Flexible conjugate gradients (FCG(1), Notay, SIAM J. Sci. Comput. 22 (2000)
// 1444-1460) with one V-cycle as the preconditioner e = M r:
//   p_k = e_k - (e_k . q_{k-1} / p_{k-1} . q_{k-1}) p_{k-1},  q_k = A p_k,
//   alpha_k = p_k . r_k / p_k . q_k,  z += alpha_k p_k,  r -= alpha_k q_k.
// The explicit orthogonalisation against the previous direction keeps the
// iteration convergent although the V-cycle (the same colour order before and
// after the coarse correction, FP32 in mixed precision) is not a symmetric
// linear operator. The scalars live on the device (ks), so an iteration needs
// no host round trip besides the residual norm. For the singular systems (no
// zero-pressure edge) e is made mean-free, so every direction, and the
// iterate's mean, stay in the range of A.

/** Per-block sums of e, e.q and q (part[b], part[nb + b], part[2 nb + b]). */
template <class Te>
__global__ void k_cg_dots(const Te *e, const double *q, long N, double *part) {
    double s0 = 0, s1 = 0, s2 = 0;
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < N;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        const double ev = static_cast<double>(e[i]), qv = q[i];
        s0 += ev;
        s1 += ev * qv;
        s2 += qv;
    }
    s0 = block_sum_256(s0);
    s1 = block_sum_256(s1);
    s2 = block_sum_256(s2);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = s0;
        part[gridDim.x + blockIdx.x] = s1;
        part[2 * gridDim.x + blockIdx.x] = s2;
    }
}

/** out[k] = sum of part[k nb .. k nb + nb - 1] for k < K, in a fixed order. */
template <int K>
__global__ void k_reduce_n(const double *part, int nb, double *out) {
#pragma unroll 1
    for (int k = 0; k < K; k++) {
        double acc = 0;
        for (int q = threadIdx.x; q < nb; q += blockDim.x) acc += part[k * nb + q];
        acc = block_sum_256(acc);
        if (threadIdx.x == 0) out[k] = acc;
    }
}

/** The new direction p = (e - mu) - beta p, mu the mean of e on a singular
 * system (else 0), beta = (e - mu).q / p.q of the previous direction (0 for
 * the first direction, ks[3] == 0, when p is not read). */
template <class Te>
__global__ void k_cg_direction(const Te *e, double *p, long N, const double *ks, int singular) {
    const double mu = singular ? ks[0] / static_cast<double>(N) : 0.0;
    const double pq = ks[3];
    const double beta = pq != 0 ? (ks[1] - mu * ks[2]) / pq : 0.0;
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < N;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        const double em = static_cast<double>(e[i]) - mu;
        p[i] = beta != 0 ? em - beta * p[i] : em;
    }
}

/** q = A p with per-block sums of p.q and p.r (part[b], part[nb + b]); rows
 * strided over the blocks as in k_resnorm. */
template <class Op>
__global__ void k_cg_apply(Op op, const double *p, double *q, const double *r, int m, int n, double *part) {
    double s0 = 0, s1 = 0;
    for (int j = blockIdx.x; j < n; j += gridDim.x)
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            const long k = i + static_cast<long>(m) * j;
            double diag;
            const double off = op.offdiag(i, j, p, diag);
            const double pv = p[k], qv = fma_rn(diag, pv, off);
            q[k] = qv;
            s0 += pv * qv;
            s1 += pv * r[k];
        }
    s0 = block_sum_256(s0);
    s1 = block_sum_256(s1);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = s0;
        part[gridDim.x + blockIdx.x] = s1;
    }
}

/** z += alpha p, r -= alpha q (alpha = p.r / p.q from ks[5], ks[4]), the
 * FP32 copy of r for the next mixed cycle, per-block sums of r^2. */
__global__ void k_cg_update(double *z, double *r, const double *p, const double *q, float *rf, long N,
                            const double *ks, double *part) {
    const double pq = ks[4], alpha = pq != 0 ? ks[5] / pq : 0.0;
    double acc = 0;
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < N;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        z[i] = fma_rn(alpha, p[i], z[i]);
        const double rn = fma_rn(-alpha, q[i], r[i]);
        r[i] = rn;
        if (rf) rf[i] = static_cast<float>(rn);
        acc += rn * rn;
    }
    acc = block_sum_256(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

/** ||r||^2 into *norm from the update's partials; the direction's p.q
 * becomes the previous one for the next iteration. */
__global__ void k_cg_finish(const double *part, int nb, double *norm, double *ks) {
    double acc = 0;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) acc += part[q];
    acc = block_sum_256(acc);
    if (threadIdx.x == 0) {
        *norm = acc;
        ks[3] = ks[4];
    }
}

/** r = b - A z in FP64 (and FP32 into rf if given), per-block sums of r^2. */
template <class Op>
__global__ void k_cg_residual(Op op, const double *z, const double *b, int m, int n, double *r, float *rf,
                              double *part) {
    double acc = 0;
    for (int j = blockIdx.x; j < n; j += gridDim.x)
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            const long k = i + static_cast<long>(m) * j;
            double diag;
            const double off = op.offdiag(i, j, z, diag);
            const double rv = fma_rn(-diag, z[k], sub_rn(b[k], off));
            r[k] = rv;
            if (rf) rf[k] = static_cast<float>(rv);
            acc += rv * rv;
        }
    acc = block_sum_256(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

constexpr int kRedBlocks = 4 * kB200SMs;  // reduction grid: 4 x 148 blocks of 256

inline dim3 grid2(int m, int n) { return dim3(cdiv(m, 32), cdiv(n, 8)); }
const dim3 kBlk2(32, 8);

/** Runs `sweeps` four-colour sweeps on the iterate z. Two sweeps on a grid
 * whose periodic directions have even sizes run as one tile-fused launch that
 * reads z and writes zalt (*res = zalt); otherwise one launch per colour
 * updates z in place (*res = z). When prof is given, each launch is bracketed
 * by CUDA events and credited with its algorithmic bytes: (units updated) x
 * bytes_per_unit. */
template <class Op, class T>
int smooth(Op op, T *z, T *zalt, const T *b, int m, int n, int sweeps, cudaStream_t s, long long &nl, T **res,
           Multigrid *prof = nullptr, double bytes_per_unit = 0) {
    *res = z;
    if (sweeps == 2 && zalt && (!op.px || m % 2 == 0) && (!op.py || n % 2 == 0)) {
        // Two sweeps per launch with shared-memory tiles (identical results);
        // the largest tile that still gives every SM work, else the smallest.
        const dim3 b64(cdiv(m, 64), cdiv(n, 32)), b32(cdiv(m, 32), cdiv(n, 16)), b16(cdiv(m, 16), cdiv(n, 16));
        if (prof) { int r = prof->prof_begin(static_cast<double>(m) * n * 2 * bytes_per_unit); if (r) return r; }
        bool done = false;
        if constexpr (Op::kFivePoint) {
            if (static_cast<int>(b64.x * b64.y) >= 2 * kB200SMs) {
                k_smooth_rb<Op, T, 2, 64, 32><<<b64, 256, 0, s>>>(op, z, zalt, b, m, n);
                done = true;
            }
        }
        if (done) {
        } else if (static_cast<int>(b64.x * b64.y) >= 2 * kB200SMs)
            k_smooth_tile<Op, T, 2, 64, 32><<<b64, 256, 0, s>>>(op, z, zalt, b, m, n);
        else if (static_cast<int>(b32.x * b32.y) >= kB200SMs)
            k_smooth_tile<Op, T, 2, 32, 16><<<b32, 256, 0, s>>>(op, z, zalt, b, m, n);
        else if constexpr (std::is_same<Op, GenOp<T>>::value)
            k_smooth_tile_gen<T, 2, 16, 16><<<b16, 256, gen_tile_smem<T>(), s>>>(op, z, zalt, b, m, n);
        else
            k_smooth_tile<Op, T, 2, 16, 16><<<b16, 256, 0, s>>>(op, z, zalt, b, m, n);
        nl++;
        if (prof) { int r = prof->prof_end(); if (r) return r; }
        INCRMT_CKL("k_smooth_tile");
        *res = zalt;
        return INCRMT_OK;
    }
    const int pis[4] = {0, 1, 1, 0}, pjs[4] = {0, 1, 0, 1};
    for (int q = 0; q < sweeps; q++)
        for (int c = 0; c < 4; c++) {
            const int mc = (m - pis[c] + 1) / 2, nc = (n - pjs[c] + 1) / 2;
            if (mc <= 0 || nc <= 0) continue;
            if (prof) { int r = prof->prof_begin(static_cast<double>(mc) * nc * bytes_per_unit); if (r) return r; }
            k_smooth<Op, T><<<grid2(mc, nc), kBlk2, 0, s>>>(op, z, b, m, n, pis[c], pjs[c]);
            nl++;
            if (prof) { int r = prof->prof_end(); if (r) return r; }
        }
    INCRMT_CKL("k_smooth");
    return INCRMT_OK;
}

/** Coarse right-hand side and cleared coarse iterate: the tiled restriction,
 * or k_restrict when tiles are off (the identity check of
 * incrmt_mg_set_tiles covers both). */
template <class Op, class T>
void restrict_launch(bool tiles, Op op, cudaStream_t s, const T *z, const T *b, int fm, int fn, int px, int py,
                     bool kx, bool ky, int cm, int cn, T *bc, T *zc, const double *we) {
    if (!tiles) {
        k_restrict<<<grid2(cm, cn), kBlk2, 0, s>>>(op, z, b, fm, fn, px, py, kx, ky, cm, cn, bc, zc, we);
        return;
    }
    const dim3 g(cdiv(cm, 32), cdiv(cn, 8));
    if (kx && ky)
        k_restrict_tile<Op, T, true, true><<<g, 256, 0, s>>>(op, z, b, fm, fn, px, py, cm, cn, bc, zc, we);
    else if (kx)
        k_restrict_tile<Op, T, true, false><<<g, 256, 0, s>>>(op, z, b, fm, fn, px, py, cm, cn, bc, zc, we);
    else
        k_restrict_tile<Op, T, false, true><<<g, 256, 0, s>>>(op, z, b, fm, fn, px, py, cm, cn, bc, zc, we);
}

}  // namespace

MacOp<double> Multigrid::mac64() const {
    MacOp<double> o; o.m = m; o.n = n; o.px = px; o.py = py; o.zpr = zpr;
    o.xxsp = xxsp; o.yysp = yysp; o.ex = ex; o.ey = ey; return o;
}
MacOp<float> Multigrid::mac32() const {
    MacOp<float> o; o.m = m; o.n = n; o.px = px; o.py = py; o.zpr = zpr;
    o.xxsp = static_cast<float>(xxsp); o.yysp = static_cast<float>(yysp); o.ex = exf; o.ey = eyf; return o;
}
FemOp<double> Multigrid::fem64() const {
    FemOp<double> o; o.m = m; o.n = n; o.px = px; o.py = py; o.zpr = zpr;
    o.fm = fm; o.fc = fc; o.hex = hex; o.hey = hey; o.c = c; return o;
}
FemOp<float> Multigrid::fem32() const {
    FemOp<float> o; o.m = m; o.n = n; o.px = px; o.py = py; o.zpr = zpr;
    o.fm = static_cast<float>(fm); o.fc = static_cast<float>(fc);
    o.hex = static_cast<float>(hex); o.hey = static_cast<float>(hey); o.c = cf; return o;
}

int Multigrid::create(int sys_, int cm_, int cn_, double ax, double bx, double ay, double by,
                      int px_, int py_, int zpr_, cudaStream_t ext) {
    if (sys_ != INCRMT_SYS_MAC && sys_ != INCRMT_SYS_FEM) { set_error("unknown system %d", sys_); return INCRMT_ERR_BADARG; }
    if (cm_ < 2 || cn_ < 2 || !(bx > ax) || !(by > ay)) { set_error("bad grid %dx%d", cm_, cn_); return INCRMT_ERR_BADARG; }
    sys = sys_; cm = cm_; cn = cn_; px = px_ ? 1 : 0; py = py_ ? 1 : 0; zpr = zpr_ ? 1 : 0;
    dx = (bx - ax) / cm; dy = (by - ay) / cn;
    const double xsp = 1 / dx, ysp = 1 / dy;
    xxsp = xsp * xsp; yysp = ysp * ysp;
    if (sys == INCRMT_SYS_MAC) { m = cm; n = cn; }
    else { m = px ? cm : cm + 1; n = py ? cn : cn + 1; }
    if ((px && m % 2) || (py && n % 2)) {
        set_error("a periodic direction needs an even number of unknowns (got %dx%d)", m, n);
        return INCRMT_ERR_BADARG;
    }
    // Finite-element stencil constants (mgs_fem.cc:12-21).
    const double dydx = dy / dx, dxdy = dx / dy;
    fm = 1. / 3. * (dxdy + dydx);
    const double fey = 1. / 3. * (-2 * dxdy + dydx), fex = 1. / 3. * (-2 * dydx + dxdy);
    hey = 0.5 * fey; hex = 0.5 * fex;
    fc = -1. / 6. * (dxdy + dydx);
    if (ext) { stream = ext; own_stream = false; }
    else INCRMT_CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    INCRMT_CK(cudaEventCreate(&ev0));
    INCRMT_CK(cudaEventCreate(&ev1));
    const long N = static_cast<long>(m) * n;
    if (sys == INCRMT_SYS_MAC) {
        INCRMT_CK(cudaMalloc(&ex, sizeof(double) * (cm + 1) * cn));
        INCRMT_CK(cudaMalloc(&ey, sizeof(double) * cm * (cn + 1)));
        INCRMT_CK(cudaMalloc(&exf, sizeof(float) * (cm + 1) * cn));
        INCRMT_CK(cudaMalloc(&eyf, sizeof(float) * cm * (cn + 1)));
    } else {
        INCRMT_CK(cudaMalloc(&c, sizeof(double) * N));
        INCRMT_CK(cudaMalloc(&cf, sizeof(float) * N));
    }
    INCRMT_CK(cudaMalloc(&rho, sizeof(double) * (cm + 4) * (cn + 4)));
    INCRMT_CK(cudaMalloc(&bbuf, sizeof(double) * N));
    INCRMT_CK(cudaMalloc(&zbuf, sizeof(double) * N));
    INCRMT_CK(cudaMalloc(&partial, sizeof(double) * kRedBlocks));
    INCRMT_CK(cudaMalloc(&dnorm, sizeof(double) * 4));
    INCRMT_CK(cudaMallocHost(&hnorm, sizeof(double) * 4));
    return build_hierarchy();
}

int Multigrid::build_hierarchy() {
    lev.clear();
    MgLevel L0; L0.m = m; L0.n = n; L0.N = static_cast<long>(m) * n;
    INCRMT_CK(cudaMalloc(&L0.zf, sizeof(float) * L0.N));
    INCRMT_CK(cudaMalloc(&L0.bf, sizeof(float) * L0.N));
    INCRMT_CK(cudaMalloc(&L0.z2, sizeof(double) * L0.N));
    INCRMT_CK(cudaMalloc(&L0.zf2, sizeof(float) * L0.N));
    lev.push_back(L0);
    int mm = m, nn = n;
    // Semi-coarsening on anisotropic grids: r is the ratio of the operator's
    // y coupling to its x coupling, (dx/dy)^2 on the fine level of both
    // systems. Point Gauss-Seidel smooths only along the strong direction, so
    // while one direction's coupling is more than twice the other's only
    // that direction is halved, which divides (or multiplies) r by 4.
    double r = yysp / xxsp;
    while (static_cast<int>(lev.size()) < kMaxLevels && mm * nn > kCoarsestSize) {
        bool kx = can_coarsen(mm, px), ky = can_coarsen(nn, py);
        if (kx && ky) {
            if (r > kSemiRatio) kx = false;
            else if (r < 1 / kSemiRatio) ky = false;
        }
        if (!kx && !ky) break;
        if (kx && !ky) r *= 4;
        else if (ky && !kx) r /= 4;
        const int mc = kx ? (px ? mm / 2 : (mm + 1) / 2) : mm, nc = ky ? (py ? nn / 2 : (nn + 1) / 2) : nn;
        lev.back().kx = kx; lev.back().ky = ky;
        MgLevel L; L.m = mc; L.n = nc; L.N = static_cast<long>(mc) * nc;
        INCRMT_CK(cudaMalloc(&L.z, sizeof(double) * L.N));
        INCRMT_CK(cudaMalloc(&L.b, sizeof(double) * L.N));
        INCRMT_CK(cudaMalloc(&L.st, sizeof(double) * 9 * L.N));
        INCRMT_CK(cudaMalloc(&L.zf, sizeof(float) * L.N));
        INCRMT_CK(cudaMalloc(&L.bf, sizeof(float) * L.N));
        INCRMT_CK(cudaMalloc(&L.stf, sizeof(float) * 9 * L.N));
        INCRMT_CK(cudaMalloc(&L.z2, sizeof(double) * L.N));
        INCRMT_CK(cudaMalloc(&L.zf2, sizeof(float) * L.N));
        lev.push_back(L);
        mm = mc; nn = nc;
    }
    // Prolongation weights of every level but the coarsest (k_build_p).
    for (size_t l = 0; l + 1 < lev.size(); l++) {
        INCRMT_CK(cudaMalloc(&lev[l].P, sizeof(double) * 4 * lev[l].N));
        INCRMT_CK(cudaMemsetAsync(lev[l].P, 0, sizeof(double) * 4 * lev[l].N, stream));
    }
    if (lev.size() > 1 && lev.back().N <= kDirectMax) {
        const long N = lev.back().N;
        INCRMT_CK(cudaMalloc(&ginv, sizeof(double) * N * N));
        INCRMT_CK(cudaMalloc(&ginvf, sizeof(float) * N * N));
        // The attribute is per kernel, shared by every solver: set the maximum.
        INCRMT_CK(cudaFuncSetAttribute(k_coarse_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(sizeof(double) * (2 * kDirectMax * kDirectMax + kDirectMax))));
    }
    INCRMT_CK(cudaFuncSetAttribute(k_tail<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(kTailSmemBudget)));
    INCRMT_CK(cudaFuncSetAttribute(k_smooth_tile_gen<double, 2, 16, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   gen_tile_smem<double>()));
    INCRMT_CK(cudaFuncSetAttribute(k_smooth_tile_gen<float, 2, 16, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   gen_tile_smem<float>()));
    INCRMT_CK(cudaFuncSetAttribute(k_tail<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(kTailSmemBudget)));

    const int gal_smem = static_cast<int>(galerkin_tile_smem(true, true));
    INCRMT_CK(set_galerkin_attr<MacOp<double>>(gal_smem));
    INCRMT_CK(set_galerkin_attr<FemOp<double>>(gal_smem));
    INCRMT_CK(set_galerkin_attr<GenOp<double>>(gal_smem));
    // First level small enough for the one-block tail kernel (never level 0).
    tail_level = -1;
    for (int l = 1; l < static_cast<int>(lev.size()); l++)
        if (lev[l].N <= kTailMaxSize && static_cast<int>(lev.size()) - l <= kTailMaxLevels) { tail_level = l; break; }
    return INCRMT_OK;
}

void Multigrid::destroy() {
    for (auto &L : lev) {
        cudaFree(L.z); cudaFree(L.b); cudaFree(L.st); cudaFree(L.zf); cudaFree(L.bf); cudaFree(L.stf);
        cudaFree(L.z2); cudaFree(L.zf2); cudaFree(L.P);
    }
    lev.clear();
    cudaFree(ex); cudaFree(ey); cudaFree(exf); cudaFree(eyf); cudaFree(c); cudaFree(cf);
    cudaFree(rho); cudaFree(bbuf); cudaFree(zbuf); cudaFree(partial); cudaFree(dnorm);
    cudaFree(ginv); cudaFree(ginvf); ginv = nullptr; ginvf = nullptr;

    if (hnorm) cudaFreeHost(hnorm);
    if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
    if (setup_exec) { cudaGraphExecDestroy(setup_exec); setup_exec = nullptr; }
    if (kexec) { cudaGraphExecDestroy(kexec); kexec = nullptr; }
    cudaFree(kr); cudaFree(kp); cudaFree(kq); cudaFree(ke); cudaFree(kpart); cudaFree(ks);
    kr = kp = kq = ke = kpart = ks = nullptr;
    for (auto e : prof_ev) cudaEventDestroy(e);
    prof_ev.clear();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream && own_stream) cudaStreamDestroy(stream);
    stream = nullptr;
}

int Multigrid::set_density_device(const double *d_rho, int ld) {
    if (ld <= 0) ld = cm + 4;
    if (sys == INCRMT_SYS_MAC) {
        k_mac_coef<<<grid2(cm + 1, cn + 1), kBlk2, 0, stream>>>(d_rho, ld, cm, cn, ex, ey, exf, eyf);
    } else {
        k_fem_coef<<<grid2(m, n), kBlk2, 0, stream>>>(d_rho, ld, m, n, c, cf);
    }
    launches++;
    INCRMT_CKL("coefficients");
    int r = galerkin_graph();
    if (r == INCRMT_OK) ready = true;
    coarse_builds++;
    coarse_age = 0;
    coarse_vc0 = -1;
    coarse_stale = false;
    return r;
}

int Multigrid::set_density_lagged(const double *d_rho, int ld) {
    lag_rho = d_rho;
    lag_ld = ld;
    if (!ready || coarse_stale || coarse_every <= 1 || coarse_age + 1 >= coarse_every)
        return set_density_device(d_rho, ld);
    if (ld <= 0) ld = cm + 4;
    if (sys == INCRMT_SYS_MAC) {
        k_mac_coef<<<grid2(cm + 1, cn + 1), kBlk2, 0, stream>>>(d_rho, ld, cm, cn, ex, ey, exf, eyf);
    } else {
        k_fem_coef<<<grid2(m, n), kBlk2, 0, stream>>>(d_rho, ld, m, n, c, cf);
    }
    launches++;
    INCRMT_CKL("coefficients");
    coarse_age++;
    return INCRMT_OK;
}

void Multigrid::note_vcycles(int vc) {
    if (coarse_vc0 < 0) coarse_vc0 = vc;
    else if (vc > coarse_vc0 + 1) coarse_stale = true;
}

int Multigrid::solve_lagged(const double *d_b, double *d_z, const incrmt_mg_opts *o, incrmt_mg_stats *st,
                            bool time_it) {
    incrmt_mg_stats s1{};
    int r = solve_device(d_b, d_z, o, &s1, time_it);
    if (r == INCRMT_OK) {
        note_vcycles(s1.vcycles);
        if (st) *st = s1;
        return r;
    }
    coarse_stale = true;
    if ((r == INCRMT_ERR_NOCONV || r == INCRMT_ERR_NONFINITE) && coarse_age > 0 && lag_rho) {
        if (r == INCRMT_ERR_NONFINITE)
            INCRMT_CK(cudaMemsetAsync(d_z, 0, sizeof(double) * static_cast<size_t>(m) * n, stream));
        int rr = set_density_device(lag_rho, lag_ld);
        if (rr) return rr;
        coarse_retries++;
        incrmt_mg_stats s2{};
        r = solve_device(d_b, d_z, o, &s2, time_it);
        s1.vcycles += s2.vcycles;
        s1.rel_res = s2.rel_res;
        s1.device_ms += s2.device_ms;
        if (r == INCRMT_OK) note_vcycles(s2.vcycles);
        else coarse_stale = true;
    }
    if (st) *st = s1;
    return r;
}

int Multigrid::set_unit_density() {
    const long N = static_cast<long>(cm + 4) * (cn + 4);
    double *ones = nullptr;
    INCRMT_CK(cudaMalloc(&ones, sizeof(double) * N));
    k_fill<<<cdiv(N, 256) < kRedBlocks ? cdiv(N, 256) : kRedBlocks, 256, 0, stream>>>(ones, N, 1.0);
    launches++;
    int r = set_density_device(ones, cm + 4);
    cudaError_t e = cudaStreamSynchronize(stream);
    cudaFree(ones);
    if (r) return r;
    INCRMT_CK(e);
    return INCRMT_OK;
}

int Multigrid::galerkin_all() {
    for (size_t l = 1; l < lev.size(); l++) {
        MgLevel &F = lev[l - 1], &C = lev[l];
        const dim3 gf = grid2(F.m, F.n), gc = grid2(C.m, C.n), gt(cdiv(C.m, 32), cdiv(C.n, 8));
        const size_t gsm = galerkin_tile_smem(F.kx, F.ky);
        auto build = [&](auto op) {
            for (int pass = 0; pass < 2; pass++)
                k_build_p<<<gf, kBlk2, 0, stream>>>(op, F.m, F.n, px, py, F.kx, F.ky, C.m, C.n, F.P, pass);
            using OpT = decltype(op);
            if (tiles && F.kx && F.ky)
                k_galerkin_tile<OpT, true, true><<<gt, 256, gsm, stream>>>(op, F.m, F.n, px, py, C.m, C.n, C.st, F.P);
            else if (tiles && F.kx)
                k_galerkin_tile<OpT, true, false><<<gt, 256, gsm, stream>>>(op, F.m, F.n, px, py, C.m, C.n, C.st, F.P);
            else if (tiles)
                k_galerkin_tile<OpT, false, true><<<gt, 256, gsm, stream>>>(op, F.m, F.n, px, py, C.m, C.n, C.st, F.P);
            else
                k_galerkin<<<gc, kBlk2, 0, stream>>>(op, F.m, F.n, px, py, F.kx, F.ky, C.m, C.n, C.st, F.P);
        };
        if (l == 1 && sys == INCRMT_SYS_MAC) {
            build(mac64());
        } else if (l == 1) {
            build(fem64());
        } else {
            GenOp<double> g; g.m = F.m; g.n = F.n; g.px = px; g.py = py; g.N = F.N; g.st = F.st;
            build(g);
        }
        launches += 3;
        INCRMT_CKL("galerkin");
    }
    f32_stale = true;
    if (ginv) {
        const MgLevel &C = lev.back();
        const size_t sm = sizeof(double) * (2 * C.N * C.N + C.N);
        k_coarse_inverse<<<1, 1024, sm, stream>>>(C.st, C.m, C.n, px, py, ginv, ginvf);
        launches++;
        INCRMT_CKL("k_coarse_inverse");
    }
    return INCRMT_OK;
}

int Multigrid::galerkin_graph() {
    // The hierarchy's arrays never move, so the whole rebuild (weights,
    // Galerkin products, the coarsest inverse: dozens of launches, most on
    // small levels) is captured once and replayed; profiling runs it
    // directly.
    if (prof) return galerkin_all();
    if (!setup_exec) {
        const long long l0 = launches;
        cudaGraph_t graph = nullptr;
        INCRMT_CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        int rc = galerkin_all();
        cudaError_t ce = cudaStreamEndCapture(stream, &graph);
        if (rc == INCRMT_OK && ce == cudaSuccess) ce = cudaGraphInstantiate(&setup_exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (rc != INCRMT_OK || ce != cudaSuccess) {
            setup_exec = nullptr;
            cudaGetLastError();
            launches = l0;
            return galerkin_all();
        }
        setup_launches = launches - l0;
        launches = l0;
    }
    INCRMT_CK(cudaGraphLaunch(setup_exec, stream));
    launches += setup_launches;
    f32_stale = true;
    return INCRMT_OK;
}

int Multigrid::cast_levels() {
    if (!f32_stale) return INCRMT_OK;
    for (size_t l = 1; l < lev.size(); l++) {
        MgLevel &C = lev[l];
        k_cast_stencil<<<cdiv(C.N, 256) < kRedBlocks ? cdiv(C.N, 256) : kRedBlocks, 256, 0, stream>>>(C.st, C.stf, C.N);
        launches++;
    }
    INCRMT_CKL("k_cast_stencil");
    f32_stale = false;
    return INCRMT_OK;
}

int Multigrid::cycle64(int l, const double *b0, double *z0) {
    if (l > 0 && l == tail_level) return tail64();
    const MgLevel &L = lev[l];
    const double *b = l == 0 ? b0 : L.b;
    double *z = l == 0 ? z0 : L.z;
    GenOp<double> g; g.m = L.m; g.n = L.n; g.px = px; g.py = py; g.N = L.N; g.st = L.st;
    const bool last = l == static_cast<int>(lev.size()) - 1;
    if (last) {
        if (l == 0) {
            if (sys == INCRMT_SYS_MAC) k_coarse<<<1, 256, 0, stream>>>(mac64(), z, b, L.m, L.n, kCoarseSweeps);
            else k_coarse<<<1, 256, 0, stream>>>(fem64(), z, b, L.m, L.n, kCoarseSweeps);
        } else if (ginv) k_coarse_direct<double><<<1, 256, 0, stream>>>(ginv, b, z, static_cast<int>(L.N));
        else k_coarse<<<1, 256, 0, stream>>>(g, z, b, L.m, L.n, kCoarseSweeps);
        launches++;
        INCRMT_CKL("k_coarse");
        return INCRMT_OK;
    }
    const MgLevel &C = lev[l + 1];
    int r;
    Multigrid *pf = prof ? this : nullptr;
    // Algorithmic bytes per updated unknown of a fine FP64 sweep: read z,b
    // and the coefficient words, write z (3+c words; c=2 MAC, c=1 FEM).
    const double bpu = 8.0 * (sys == INCRMT_SYS_MAC ? 5 : 4);
    // Pre-smoothing may leave the iterate in the level's second buffer; the
    // restriction, prolongation and post-smoothing follow it, and the
    // post-smoothing brings it back (both smoothings use the same kind of
    // launch, so the two moves cancel).
    double *cur = z;
    if (l == 0 && sys == INCRMT_SYS_MAC) {
        auto op = mac64();
        if ((r = smooth(op, z, tiles ? L.z2 : nullptr, b, L.m, L.n, kNu1, stream, launches, &cur, pf, bpu))) return r;
        restrict_launch(tiles, op, stream, cur, b, L.m, L.n, px, py, L.kx, L.ky, C.m, C.n, C.b, C.z, L.P);
    } else if (l == 0) {
        auto op = fem64();
        if ((r = smooth(op, z, tiles ? L.z2 : nullptr, b, L.m, L.n, kNu1, stream, launches, &cur, pf, bpu))) return r;
        restrict_launch(tiles, op, stream, cur, b, L.m, L.n, px, py, L.kx, L.ky, C.m, C.n, C.b, C.z, L.P);
    } else {
        if ((r = smooth(g, z, tiles ? L.z2 : nullptr, b, L.m, L.n, kNu1, stream, launches, &cur))) return r;
        restrict_launch(tiles, g, stream, cur, b, L.m, L.n, px, py, L.kx, L.ky, C.m, C.n, C.b, C.z, L.P);
    }
    launches++;
    INCRMT_CKL("k_restrict");
    if ((r = cycle64(l + 1, b0, z0))) return r;
    k_prolong<<<grid2(L.m, L.n), kBlk2, 0, stream>>>(cur, L.m, L.n, px, py, L.kx, L.ky, static_cast<const double *>(C.z), C.m, C.n, L.P);
    launches++;
    INCRMT_CKL("k_prolong");
    double *alt = !tiles ? nullptr : cur == z ? L.z2 : z, *out = cur;
    if (l == 0 && sys == INCRMT_SYS_MAC) r = smooth(mac64(), cur, alt, b, L.m, L.n, kNu2, stream, launches, &out, pf, bpu);
    else if (l == 0) r = smooth(fem64(), cur, alt, b, L.m, L.n, kNu2, stream, launches, &out, pf, bpu);
    else r = smooth(g, cur, alt, b, L.m, L.n, kNu2, stream, launches, &out);
    if (r) return r;
    if (out != z) INCRMT_CK(cudaMemcpyAsync(z, out, sizeof(double) * L.N, cudaMemcpyDeviceToDevice, stream));
    return INCRMT_OK;
}

int Multigrid::prof_begin(double bytes) {
    constexpr int kMaxEvents = 4096;
    if (prof_used + 2 > kMaxEvents) {
        int r = prof_collect();
        if (r) return r;
    }
    while (prof_used + 2 > static_cast<int>(prof_ev.size())) {
        cudaEvent_t e;
        INCRMT_CK(cudaEventCreate(&e));
        prof_ev.push_back(e);
    }
    INCRMT_CK(cudaEventRecord(prof_ev[prof_used], stream));
    pending_bytes = bytes;
    prof_bytes += bytes;
    return INCRMT_OK;
}

int Multigrid::prof_end() {
    INCRMT_CK(cudaEventRecord(prof_ev[prof_used + 1], stream));
    prof_used += 2;
    prof_launches++;
    return INCRMT_OK;
}

/** Folds the recorded event pairs into prof_ms (synchronises the stream).
 * \return 0 (the number of pairs still pending) or an error status. */
int Multigrid::prof_collect() {
    if (prof_used == 0) return 0;
    INCRMT_CK(cudaStreamSynchronize(stream));
    for (int k = 0; k + 1 < prof_used; k += 2) {
        float ms = 0;
        INCRMT_CK(cudaEventElapsedTime(&ms, prof_ev[k], prof_ev[k + 1]));
        prof_ms += ms;
    }
    prof_used = 0;
    return 0;
}

int Multigrid::cycle32(int l) {
    if (l > 0 && l == tail_level) return tail32();
    const MgLevel &L = lev[l];
    const float *b = L.bf;
    float *z = L.zf;
    GenOp<float> g; g.m = L.m; g.n = L.n; g.px = px; g.py = py; g.N = L.N; g.st = L.stf;
    const bool last = l == static_cast<int>(lev.size()) - 1;
    if (last) {
        if (l == 0) {
            if (sys == INCRMT_SYS_MAC) k_coarse<<<1, 256, 0, stream>>>(mac32(), z, b, L.m, L.n, kCoarseSweeps);
            else k_coarse<<<1, 256, 0, stream>>>(fem32(), z, b, L.m, L.n, kCoarseSweeps);
        } else if (ginvf) k_coarse_direct<float><<<1, 256, 0, stream>>>(ginvf, b, z, static_cast<int>(L.N));
        else k_coarse<<<1, 256, 0, stream>>>(g, z, b, L.m, L.n, kCoarseSweeps);
        launches++;
        INCRMT_CKL("k_coarse");
        return INCRMT_OK;
    }
    const MgLevel &C = lev[l + 1];
    int r;
    float *cur = z;  // as in cycle64
    Multigrid *pf = prof ? this : nullptr;
    const double bpu = 4.0 * (sys == INCRMT_SYS_MAC ? 5 : 4);  // FP32 words: z, b, coefficients in; z out
    if (l == 0 && sys == INCRMT_SYS_MAC) {
        auto op = mac32();
        if ((r = smooth(op, z, tiles ? L.zf2 : nullptr, b, L.m, L.n, kNu1, stream, launches, &cur, pf, bpu))) return r;
        restrict_launch(tiles, op, stream, static_cast<const float *>(cur), b, L.m, L.n, px, py, L.kx, L.ky, C.m, C.n, C.bf, C.zf, L.P);
    } else if (l == 0) {
        auto op = fem32();
        if ((r = smooth(op, z, tiles ? L.zf2 : nullptr, b, L.m, L.n, kNu1, stream, launches, &cur, pf, bpu))) return r;
        restrict_launch(tiles, op, stream, static_cast<const float *>(cur), b, L.m, L.n, px, py, L.kx, L.ky, C.m, C.n, C.bf, C.zf, L.P);
    } else {
        if ((r = smooth(g, z, tiles ? L.zf2 : nullptr, b, L.m, L.n, kNu1, stream, launches, &cur))) return r;
        restrict_launch(tiles, g, stream, static_cast<const float *>(cur), b, L.m, L.n, px, py, L.kx, L.ky, C.m, C.n, C.bf, C.zf, L.P);
    }
    launches++;
    INCRMT_CKL("k_restrict");
    if ((r = cycle32(l + 1))) return r;
    k_prolong<<<grid2(L.m, L.n), kBlk2, 0, stream>>>(cur, L.m, L.n, px, py, L.kx, L.ky, static_cast<const float *>(C.zf), C.m, C.n, L.P);
    launches++;
    INCRMT_CKL("k_prolong");
    float *alt = !tiles ? nullptr : cur == z ? L.zf2 : z, *out = cur;
    if (l == 0 && sys == INCRMT_SYS_MAC) r = smooth(mac32(), cur, alt, b, L.m, L.n, kNu2, stream, launches, &out, pf, bpu);
    else if (l == 0) r = smooth(fem32(), cur, alt, b, L.m, L.n, kNu2, stream, launches, &out, pf, bpu);
    else r = smooth(g, cur, alt, b, L.m, L.n, kNu2, stream, launches, &out);
    if (r) return r;
    if (out != z) INCRMT_CK(cudaMemcpyAsync(z, out, sizeof(float) * L.N, cudaMemcpyDeviceToDevice, stream));
    return INCRMT_OK;
}

/** Shared-memory layout of the tail: the coarsest levels, from the bottom
 * up, while their stencils, iterates and right-hand sides fit in the budget.
 * \return the dynamic shared memory in bytes. */
template <class T>
size_t tail_layout(TailLevels<T> &L, size_t budget) {
    long off = 0;
    L.smem_from = L.count;
    for (int k = L.count - 1; k >= 0; k--) {
        const long need = 11 * L.N[k];
        if (static_cast<size_t>(off + need) * sizeof(T) > budget) break;
        L.smem_from = k;
        off += need;
    }
    long o = 0;
    for (int k = L.smem_from; k < L.count; k++) { L.smem_off[k] = o; o += 11 * L.N[k]; }
    return static_cast<size_t>(o) * sizeof(T);
}

int Multigrid::tail64() {
    TailLevels<double> T{};
    T.first = tail_level; T.count = static_cast<int>(lev.size()) - tail_level; T.px = px; T.py = py;
    for (int k = 0; k < T.count; k++) {
        const MgLevel &L = lev[tail_level + k];
        T.m[k] = L.m; T.n[k] = L.n; T.N[k] = L.N; T.kx[k] = L.kx; T.ky[k] = L.ky;
        T.z[k] = L.z; T.b[k] = L.b; T.st[k] = L.st; T.P[k] = L.P;
    }
    T.ginv = ginv;
    const size_t sm = tail_layout(T, kTailSmemBudget);
    k_tail<double><<<1, 1024, sm, stream>>>(T, kNu1, kNu2, kCoarseSweeps);
    launches++;
    INCRMT_CKL("k_tail");
    return INCRMT_OK;
}

int Multigrid::tail32() {
    TailLevels<float> T{};
    T.first = tail_level; T.count = static_cast<int>(lev.size()) - tail_level; T.px = px; T.py = py;
    for (int k = 0; k < T.count; k++) {
        const MgLevel &L = lev[tail_level + k];
        T.m[k] = L.m; T.n[k] = L.n; T.N[k] = L.N; T.kx[k] = L.kx; T.ky[k] = L.ky;
        T.z[k] = L.zf; T.b[k] = L.bf; T.st[k] = L.stf; T.P[k] = L.P;
    }
    T.ginv = ginvf;
    const size_t sm = tail_layout(T, kTailSmemBudget);
    k_tail<float><<<1, 1024, sm, stream>>>(T, kNu1, kNu2, kCoarseSweeps);
    launches++;
    INCRMT_CKL("k_tail");
    return INCRMT_OK;
}

int Multigrid::norm2_rhs(const double *b, double *out_dev) {
    const long N = static_cast<long>(m) * n;
    const int nb = cdiv(N, 256) < kRedBlocks ? cdiv(N, 256) : kRedBlocks;
    k_sumsq<<<nb, 256, 0, stream>>>(b, N, partial);
    k_reduce<<<1, 256, 0, stream>>>(partial, nb, out_dev);
    launches += 2;
    INCRMT_CKL("norm");
    return INCRMT_OK;
}

int Multigrid::residual_norm(const double *b, const double *z, float *rf, double *out_dev) {
    const int nb = n < kRedBlocks ? n : kRedBlocks;  // blocks over the rows
    if (sys == INCRMT_SYS_MAC) k_resnorm<<<nb, 256, 0, stream>>>(mac64(), z, b, m, n, rf, partial);
    else k_resnorm<<<nb, 256, 0, stream>>>(fem64(), z, b, m, n, rf, partial);
    k_reduce<<<1, 256, 0, stream>>>(partial, nb, out_dev);
    launches += 2;
    INCRMT_CKL("residual norm");
    return INCRMT_OK;
}

int Multigrid::fetch_norm(double *v) {
    INCRMT_CK(cudaMemcpyAsync(hnorm, dnorm, sizeof(double), cudaMemcpyDeviceToHost, stream));
    INCRMT_CK(cudaStreamSynchronize(stream));
    *v = hnorm[0];
    return INCRMT_OK;
}

/** One V-cycle (FP64, or one FP32 defect-correction step in mixed mode),
 * the FP64 residual norm of the new iterate, and its copy to hnorm[0]. */
int Multigrid::vcycle_and_norm(int prec, const double *b, double *d_z, long N) {
    int r;
    const long long l0 = launches;
    if (prec == INCRMT_PREC_FP64) {
        if ((r = cycle64(0, b, d_z))) return r;
        if ((r = residual_norm(b, d_z, nullptr, dnorm))) return r;
    } else {
        const int nbk = cdiv(N, 256) < kRedBlocks ? cdiv(N, 256) : kRedBlocks;
        k_fill<float><<<nbk, 256, 0, stream>>>(lev[0].zf, N, 0.f);
        launches++;
        if ((r = cycle32(0))) return r;
        if (zpr) {
            k_add_f32<<<nbk, 256, 0, stream>>>(d_z, lev[0].zf, N);
            launches++;
        } else {
            // Without the zero-pressure edge both systems are singular (the
            // constants): the FP32 cycle's correction comes back with a
            // constant part thousands of times its variation on the finest
            // grids, which the iterate would accumulate; it is removed.
            k_sum_f32<<<nbk, 256, 0, stream>>>(lev[0].zf, N, partial);
            k_reduce<<<1, 256, 0, stream>>>(partial, nbk, dnorm + 1);
            k_add_f32_centred<<<nbk, 256, 0, stream>>>(d_z, lev[0].zf, N, dnorm + 1);
            launches += 3;
        }
        INCRMT_CKL("defect correction");
        if ((r = residual_norm(b, d_z, lev[0].bf, dnorm))) return r;
    }
    INCRMT_CK(cudaMemcpyAsync(hnorm, dnorm, sizeof(double), cudaMemcpyDeviceToHost, stream));
    graph_launches = launches - l0;
    return INCRMT_OK;
}

int Multigrid::krylov_alloc() {
    if (kr) return INCRMT_OK;
    const size_t N = static_cast<size_t>(m) * n;
    INCRMT_CK(cudaMalloc(&kr, sizeof(double) * N));
    INCRMT_CK(cudaMalloc(&kp, sizeof(double) * N));
    INCRMT_CK(cudaMalloc(&kq, sizeof(double) * N));
    INCRMT_CK(cudaMalloc(&ke, sizeof(double) * N));
    INCRMT_CK(cudaMalloc(&kpart, sizeof(double) * 3 * kRedBlocks));
    INCRMT_CK(cudaMalloc(&ks, sizeof(double) * 8));
    // q enters the first iteration's dot products (whose results the first
    // direction does not use): keep it finite
    INCRMT_CK(cudaMemsetAsync(kq, 0, sizeof(double) * N, stream));
    INCRMT_CK(cudaMemsetAsync(kp, 0, sizeof(double) * N, stream));
    INCRMT_CK(cudaMemsetAsync(ks, 0, sizeof(double) * 8, stream));
    return INCRMT_OK;
}

int Multigrid::krylov_residual(int prec, const double *b, const double *d_z) {
    const int nb = n < kRedBlocks ? n : kRedBlocks;  // blocks over the rows
    float *rf = prec == INCRMT_PREC_MIXED ? lev[0].bf : nullptr;
    if (sys == INCRMT_SYS_MAC) k_cg_residual<<<nb, 256, 0, stream>>>(mac64(), d_z, b, m, n, kr, rf, kpart);
    else k_cg_residual<<<nb, 256, 0, stream>>>(fem64(), d_z, b, m, n, kr, rf, kpart);
    k_reduce<<<1, 256, 0, stream>>>(kpart, nb, dnorm);
    launches += 2;
    INCRMT_CKL("krylov residual");
    return INCRMT_OK;
}

int Multigrid::krylov_iteration(int prec, double *d_z, long N) {
    int r;
    const long long l0 = launches;
    const int nbk = cdiv(N, 256) < kRedBlocks ? cdiv(N, 256) : kRedBlocks;
    const int nbr = n < kRedBlocks ? n : kRedBlocks;
    const int singular = zpr ? 0 : 1;
    if (prec == INCRMT_PREC_FP64) {
        k_fill<double><<<nbk, 256, 0, stream>>>(ke, N, 0.0);
        launches++;
        if ((r = cycle64(0, kr, ke))) return r;
        k_cg_dots<double><<<nbk, 256, 0, stream>>>(ke, kq, N, kpart);
        k_reduce_n<3><<<1, 256, 0, stream>>>(kpart, nbk, ks);
        k_cg_direction<double><<<nbk, 256, 0, stream>>>(ke, kp, N, ks, singular);
    } else {
        k_fill<float><<<nbk, 256, 0, stream>>>(lev[0].zf, N, 0.f);
        launches++;
        if ((r = cycle32(0))) return r;
        k_cg_dots<float><<<nbk, 256, 0, stream>>>(lev[0].zf, kq, N, kpart);
        k_reduce_n<3><<<1, 256, 0, stream>>>(kpart, nbk, ks);
        k_cg_direction<float><<<nbk, 256, 0, stream>>>(lev[0].zf, kp, N, ks, singular);
    }
    if (sys == INCRMT_SYS_MAC) k_cg_apply<<<nbr, 256, 0, stream>>>(mac64(), kp, kq, kr, m, n, kpart);
    else k_cg_apply<<<nbr, 256, 0, stream>>>(fem64(), kp, kq, kr, m, n, kpart);
    k_reduce_n<2><<<1, 256, 0, stream>>>(kpart, nbr, ks + 4);
    k_cg_update<<<nbk, 256, 0, stream>>>(d_z, kr, kp, kq, prec == INCRMT_PREC_MIXED ? lev[0].bf : nullptr, N, ks,
                                         kpart);
    k_cg_finish<<<1, 256, 0, stream>>>(kpart, nbk, dnorm, ks);
    launches += 7;
    INCRMT_CKL("krylov iteration");
    INCRMT_CK(cudaMemcpyAsync(hnorm, dnorm, sizeof(double), cudaMemcpyDeviceToHost, stream));
    kexec_launches = launches - l0;
    return INCRMT_OK;
}

int Multigrid::krylov_solve(int prec, const double *b, double *d_z, long N, double tol, int maxc, int &k,
                            double &rn2, bool &conv, bool &finite, bool &fell) {
    int r;
    conv = false;
    finite = true;
    fell = false;
    if ((r = krylov_alloc())) return r;
    if (prec == INCRMT_PREC_MIXED && (r = cast_levels())) return r;
    // The fixed column's rows of the FEM system with the zero-pressure edge
    // hold the diagonal alone and a zero right-hand side: their solution is
    // 0, set here, so that the iteration stays on the symmetric remainder.
    if (sys == INCRMT_SYS_FEM && zpr) {
        k_zero_column<<<cdiv(n, 256), 256, 0, stream>>>(d_z, m, n);
        launches++;
        INCRMT_CKL("zero column");
    }
    if ((r = krylov_residual(prec, b, d_z))) return r;
    if ((r = fetch_norm(&rn2))) return r;
    double rn_prev = std::sqrt(rn2);
    if (!std::isfinite(rn_prev)) { finite = false; return INCRMT_OK; }
    if (rn_prev <= tol) { conv = true; return INCRMT_OK; }
    INCRMT_CK(cudaMemsetAsync(ks, 0, sizeof(double) * 8, stream));
    const bool use_graph = !prof;
    if (use_graph && (!kexec || kkey_prec != prec || kkey_b != b || kkey_z != d_z)) {
        if (kexec) { cudaGraphExecDestroy(kexec); kexec = nullptr; }
        cudaGraph_t graph = nullptr;
        INCRMT_CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        const int rc = krylov_iteration(prec, d_z, N);
        cudaError_t ce = cudaStreamEndCapture(stream, &graph);
        if (rc || ce != cudaSuccess) {
            if (ce == cudaSuccess && graph) cudaGraphDestroy(graph);
            if (rc) return rc;
            return cuda_status(ce, "capture", __FILE__, __LINE__);
        }
        ce = cudaGraphInstantiate(&kexec, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) { kexec = nullptr; return cuda_status(ce, "instantiate", __FILE__, __LINE__); }
        kkey_prec = prec; kkey_b = b; kkey_z = d_z;
    }
    while (k < maxc) {
        if (use_graph) {
            INCRMT_CK(cudaGraphLaunch(kexec, stream));
            launches += kexec_launches;
        } else if ((r = krylov_iteration(prec, d_z, N))) {
            return r;
        }
        INCRMT_CK(cudaStreamSynchronize(stream));
        rn2 = hnorm[0];
        k++;
        const double rn = std::sqrt(rn2);
        if (!std::isfinite(rn)) { finite = false; return INCRMT_OK; }
        if (rn <= tol) {
            // The recurrence's residual has converged: confirm it on b - A z
            // itself, else restart from that residual.
            if ((r = krylov_residual(prec, b, d_z))) return r;
            if ((r = fetch_norm(&rn2))) return r;
            const double rt = std::sqrt(rn2);
            if (!std::isfinite(rt)) { finite = false; return INCRMT_OK; }
            if (rt <= tol) { conv = true; return INCRMT_OK; }
            INCRMT_CK(cudaMemsetAsync(ks, 0, sizeof(double) * 8, stream));
            rn_prev = rt;
            continue;
        }
        // An iteration that does not halve the residual: the preconditioned
        // iteration is not working on this system; the caller finishes with
        // plain FP64 V-cycles from the current iterate.
        if (rn > kMixedContraction * rn_prev) {
            fell = true;
            krylov_fallbacks++;
            return INCRMT_OK;
        }
        rn_prev = rn;
    }
    return INCRMT_OK;
}

int Multigrid::vcycle64(const double *d_b, double *d_z) {
    if (!ready) { set_error("density not set"); return INCRMT_ERR_BADARG; }
    return cycle64(0, d_b, d_z);
}

int Multigrid::effective_rhs(const double *d_b, const double **out) {
    *out = d_b;
    if (sys != INCRMT_SYS_FEM || !zpr) return INCRMT_OK;
    const long N = static_cast<long>(m) * n;
    if (d_b != bbuf) INCRMT_CK(cudaMemcpyAsync(bbuf, d_b, sizeof(double) * N, cudaMemcpyDeviceToDevice, stream));
    k_zero_column<<<cdiv(n, 256), 256, 0, stream>>>(bbuf, m, n);
    launches++;
    INCRMT_CKL("zero column");
    *out = bbuf;
    return INCRMT_OK;
}

int Multigrid::apply_device(const double *d_z, double *d_out) {
    if (!ready) { set_error("density not set"); return INCRMT_ERR_BADARG; }
    if (sys == INCRMT_SYS_MAC) k_apply<<<grid2(m, n), kBlk2, 0, stream>>>(mac64(), d_z, d_out, m, n);
    else k_apply<<<grid2(m, n), kBlk2, 0, stream>>>(fem64(), d_z, d_out, m, n);
    launches++;
    INCRMT_CKL("k_apply");
    return INCRMT_OK;
}

int Multigrid::solve_device(const double *d_b, double *d_z, const incrmt_mg_opts *o,
                            incrmt_mg_stats *st, bool time_it) {
    if (!ready) { set_error("density not set"); return INCRMT_ERR_BADARG; }
    const double rtol = (o && o->rel_tol > 0) ? o->rel_tol : 1e-9;
    const int maxc = (o && o->max_vcycles > 0) ? o->max_vcycles : 200;
    int prec = o ? o->precision : INCRMT_PREC_FP64;
    if (prec != INCRMT_PREC_FP64 && prec != INCRMT_PREC_MIXED) { set_error("bad precision %d", prec); return INCRMT_ERR_BADARG; }
    // After kMixedStrikes consecutive mixed solves that fell back to FP64,
    // the next kMixedRest solves run FP64 from the start (the FP32 cycle
    // only cost time on this system), then mixed precision is tried again.
    if (prec == INCRMT_PREC_MIXED && mixed_rest > 0) {
        mixed_rest--;
        mixed_rested++;
        prec = INCRMT_PREC_FP64;
    }
    const long N = static_cast<long>(m) * n;
    // The solve reads a residual norm back to the host after every V-cycle,
    // which a stream under capture cannot do.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    INCRMT_CK(cudaStreamIsCapturing(stream, &cap));
    if (cap != cudaStreamCaptureStatusNone) {
        set_error("a solve cannot run while its stream is being captured into a CUDA graph");
        return INCRMT_ERR_BADARG;
    }
    if (time_it) INCRMT_CK(cudaEventRecord(ev0, stream));
    const double *b = d_b;
    if (sys == INCRMT_SYS_FEM && zpr) {
        if (d_b != bbuf) INCRMT_CK(cudaMemcpyAsync(bbuf, d_b, sizeof(double) * N, cudaMemcpyDeviceToDevice, stream));
        k_zero_column<<<cdiv(n, 256), 256, 0, stream>>>(bbuf, m, n);
        launches++;
        INCRMT_CKL("zero column");
        b = bbuf;
    }
    int r;
    double nb2, rn2 = 0;
    if ((r = norm2_rhs(b, dnorm))) return r;
    if ((r = fetch_norm(&nb2))) return r;
    const double nb = std::sqrt(nb2), tol = rtol * nb;
    int k = 0;
    if (nb == 0) {
        // A zero right-hand side: z = 0 solves A z = 0 exactly (for the
        // singular pure-Neumann systems it is the zero-mean solution), and the
        // warm start need not, so the iterate is cleared.
        INCRMT_CK(cudaMemsetAsync(d_z, 0, sizeof(double) * N, stream));
        if (time_it) {
            INCRMT_CK(cudaEventRecord(ev1, stream));
            INCRMT_CK(cudaEventSynchronize(ev1));
        }
        if (st) {
            st->vcycles = 0;
            st->rel_res = 0;
            float ms = 0;
            if (time_it) cudaEventElapsedTime(&ms, ev0, ev1);
            st->device_ms = ms;
        }
        return INCRMT_OK;
    }
    bool conv = false, finite = true, plain = true;
    double rn_prev = 0;
    int cur = prec;
    if (krylov) {
        // Flexible CG around the V-cycle; plain FP64 V-cycles finish the
        // solve only if an iteration fails to halve the residual.
        bool fell = false;
        if ((r = krylov_solve(prec, b, d_z, N, tol, maxc, k, rn2, conv, finite, fell))) return r;
        plain = fell;
        if (fell) {
            cur = INCRMT_PREC_FP64;
            if (prec == INCRMT_PREC_MIXED) mixed_fallbacks++;
        }
    } else if (prec == INCRMT_PREC_MIXED) {
        if ((r = cast_levels())) return r;
        if ((r = residual_norm(b, d_z, lev[0].bf, dnorm))) return r;
        if ((r = fetch_norm(&rn2))) return r;
        rn_prev = std::sqrt(rn2);
    }
    // One V-cycle, its residual norm and the read-back of that norm, captured
    // once into a CUDA graph per (precision, b, z) and replayed per cycle.
    const bool use_graph = !prof;
    auto capture = [&]() -> int {
        if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
        cudaGraph_t graph = nullptr;
        INCRMT_CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        int rc = vcycle_and_norm(cur, b, d_z, N);
        cudaError_t ce = cudaStreamEndCapture(stream, &graph);
        if (rc || ce != cudaSuccess) {
            if (ce == cudaSuccess && graph) cudaGraphDestroy(graph);
            if (rc) return rc;
            return cuda_status(ce, "capture", __FILE__, __LINE__);
        }
        ce = cudaGraphInstantiate(&gexec, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) { gexec = nullptr; return cuda_status(ce, "instantiate", __FILE__, __LINE__); }
        gkey_prec = cur; gkey_b = b; gkey_z = d_z;
        return INCRMT_OK;
    };
    if (plain && use_graph && (!gexec || gkey_prec != cur || gkey_b != b || gkey_z != d_z) && (r = capture()))
        return r;
    while (plain && k < maxc) {
        if (use_graph) {
            INCRMT_CK(cudaGraphLaunch(gexec, stream));
            launches += graph_launches;
            INCRMT_CK(cudaStreamSynchronize(stream));
            rn2 = hnorm[0];
        } else {
            if ((r = vcycle_and_norm(cur, b, d_z, N))) return r;
            INCRMT_CK(cudaStreamSynchronize(stream));
            rn2 = hnorm[0];
        }
        k++;
        const double rn = std::sqrt(rn2);
        if (!std::isfinite(rn)) { finite = false; break; }
        if (rn <= tol) { conv = true; break; }
        // An FP32 correction that does not halve the FP64 residual means the
        // single-precision cycle no longer approximates the system's inverse
        // well enough for defect correction to converge: the rest of the
        // solve runs FP64 V-cycles from the current iterate.
        if (cur == INCRMT_PREC_MIXED && rn > kMixedContraction * rn_prev) {
            cur = INCRMT_PREC_FP64;
            mixed_fallbacks++;
            if (use_graph && (r = capture())) return r;
        }
        rn_prev = rn;
    }
    if (prec == INCRMT_PREC_MIXED) {
        if (cur != prec) {
            if (++mixed_streak >= kMixedStrikes) {
                mixed_streak = 0;
                mixed_rest = kMixedRest;
            }
        } else {
            mixed_streak = 0;
        }
    }
    if (time_it) {
        INCRMT_CK(cudaEventRecord(ev1, stream));
        INCRMT_CK(cudaEventSynchronize(ev1));
    }
    if (prof && (r = prof_collect())) return r;
    if (st) {
        st->vcycles = k;
        st->rel_res = nb > 0 ? std::sqrt(rn2) / nb : std::sqrt(rn2);
        float ms = 0;
        if (time_it) cudaEventElapsedTime(&ms, ev0, ev1);
        st->device_ms = ms;
    }
    if (!finite) { set_error("non-finite residual after %d V-cycles", k); return INCRMT_ERR_NONFINITE; }
    if (!conv && nb > 0) { set_error("V-cycle failed to converge in %d cycles", k); return INCRMT_ERR_NOCONV; }
    return INCRMT_OK;
}

}  // namespace incrmt
