// Device-side stencil operators of the two pressure systems and of the
// Galerkin coarse levels, in the form the multigrid kernels consume.
//
// Every operator offers, for an unknown (i,j):
//   offdiag(i,j,z,diag) -> sum of the off-diagonal stencil entries times z,
//                          writing the diagonal entry to diag;
//   coef9(i,j,a)        -> the nine stencil entries in the order
//                          dl,dc,dr,cl,cc,cr,ul,uc,ur, zero where the
//                          neighbour lies outside a non-periodic grid.
// A Gauss-Seidel update is z = (b - offdiag)/diag, the residual
// b - offdiag - diag*z, exactly the reference's inv_cc/mul_a/a_cc callbacks.
//
// Single precision uses the centred (difference) form of the same operator:
//   offdiag<true>(i,j,z,diag,zc) = sum_k a_k (z_k - zc), rowsum(i,j) = s,
//   (A z)(i,j) = offdiag<true> + s zc,
// with s the stencil's row sum, which is exactly zero except in rows touched
// by a Dirichlet condition. Rounding each FP32 entry separately would leave
// row sums of about one ulp of the diagonal, as large as the smallest
// eigenvalues of the pure-Neumann systems on fine grids (relative to the
// diagonal, (pi h / L)^2 / 4, about 1e-7 at 2048 x 4096), which the FP32
// cycles would then no longer resolve; in the centred form the row sum is
// exact and the smooth error is resolved to FP32 relative accuracy.
#pragma once
#include <cuda_runtime.h>

namespace incrmt {

// Every product and sum of the stencil arithmetic is written as an explicit
// operation (a fused multiply-add where a product is added, a rounded product
// or sum otherwise): left to itself the compiler contracts some products and
// sums into FMAs, and which ones can depend on the code around an inlined
// expression, so that kernels computing the same update in the same order
// could round it differently. With every rounding fixed in the source, the
// smoothers (one launch per colour, tiled) agree bit for bit.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
/** t + a*b, fused. */
template <class T>
__device__ __forceinline__ T acc_rn(T t, T a, T b) { return fma_rn(a, b, t); }
/** z - zc in the centred form, z itself otherwise. */
template <bool CEN, class T>
__device__ __forceinline__ T cen(T z, T zc) {
    if constexpr (CEN) return sub_rn(z, zc);
    else return z;
}

/** a - b*c with the product rounded before the difference in double (the
 * reference's a_cc, mgs_mac.hh:93-97, evaluated as the CPU does, without a
 * fused multiply-add), so that the MAC diagonal and the prolongation weights
 * built from it agree with the oracle's to the last bit; fused in single. */
__device__ __forceinline__ double mac_diag(double a, double b, double c) { return __dsub_rn(a, __dmul_rn(b, c)); }
__device__ __forceinline__ float mac_diag(float a, float b, float c) { return __fmaf_rn(-b, c, a); }

/** Variable-density MAC system (mgs_mac_varying_rho, mgs_mac.hh:64-102,
 * mgs_mac.cc:49-54). Unknowns are the m x n cells. The edge reciprocal
 * densities are stored as ex[(m+1)*n], the x-edge left of cell (i,j) at
 * ex[j*(m+1)+i] (i=m is the right boundary edge), and ey[m*(n+1)], the y-edge
 * below cell (i,j) at ey[j*m+i] (j=n is the top edge); each is
 * 0.5/rho+0.5/rho of the two adjacent cells (fluid_2d.cc:1140-1160). */
template <class T>
struct MacOp {
    /** Five-point stencil: red-black ordering equals the four-colour one. */
    static constexpr bool kFivePoint = true;
    int m, n, px, py, zpr;
    T xxsp, yysp;
    const T *ex, *ey;

    template <bool CEN = false>
    __device__ __forceinline__ T offdiag(int i, int j, const T *z, T &diag, T zc = T(0)) const {
        const int ij = i + m * j;
        const T el = ex[j * (m + 1) + i], er = ex[j * (m + 1) + i + 1];
        const T ed = ey[j * m + i], eu = ey[(j + 1) * m + i];
        const bool l = px || i > 0, r = px || i < m - 1, d = py || j > 0, u = py || j < n - 1;
        // neighbour indices wrap, so every load is in range (see GenOp::gen_sum)
        const T zl = z[i > 0 ? ij - 1 : ij + m - 1], zr = z[i < m - 1 ? ij + 1 : ij + 1 - m];
        const T zd = z[j > 0 ? ij - m : ij + m * (n - 1)], zu = z[j < n - 1 ? ij + m : ij - m * (n - 1)];
        diag = diag_of(i, l, r, d, u, el, er, ed, eu);
        return mac_terms<CEN>(l, r, d, u, el, er, ed, eu, zl, zr, zd, zu, zc);
    }

    /** xxsp (el zl + er zr) + yysp (ed zd + eu zu), terms outside the grid
     * skipped (centred: each z minus zc). */
    template <bool CEN>
    __device__ __forceinline__ T mac_terms(bool l, bool r, bool d, bool u, T el, T er, T ed, T eu, T zl, T zr, T zd,
                                           T zu, T zc) const {
        T sx = l ? mul_rn(el, cen<CEN>(zl, zc)) : T(0);
        sx = r ? acc_rn(sx, er, cen<CEN>(zr, zc)) : sx;
        T sy = d ? mul_rn(ed, cen<CEN>(zd, zc)) : T(0);
        sy = u ? acc_rn(sy, eu, cen<CEN>(zu, zc)) : sy;
        return fma_rn(xxsp, sx, mul_rn(yysp, sy));
    }

    /** The diagonal a_cc (mgs_mac.hh:93-97): the zero-pressure edge's ghost
     * value -z doubles the right coefficient. */
    __device__ __forceinline__ T diag_of(int i, bool l, bool r, bool d, bool u, T el, T er, T ed, T eu) const {
        (void)r;
        return mac_diag(mul_rn(-xxsp, add_rn(l ? el : T(0), px ? er : (i < m - 1 ? er : (zpr ? 2 * er : T(0))))),
                        yysp, add_rn(d ? ed : T(0), u ? eu : T(0)));
    }

    /** Row sum of the stencil: zero except at the zero-pressure edge, whose
     * ghost value is -z (the 2 er of a_cc, mgs_mac.hh:93-97). */
    __device__ __forceinline__ T rowsum(int i, int j) const {
        if (!zpr || px || i != m - 1) return T(0);
        return -2 * xxsp * ex[j * (m + 1) + i + 1];
    }

    /** offdiag with the iterate in a shared-memory tile (lz: local index of
     * (i,j), ldz: tile row stride). The tile holds the neighbours at lz+-1,
     * lz+-ldz, across a periodic edge too (as periodic images). */
    template <bool CEN = false>
    __device__ __forceinline__ T offdiag_s(int i, int j, const T *zs, int lz, int ldz, T &diag) const {
        return offdiag_v<CEN>(i, j, ex[j * (m + 1) + i], ex[j * (m + 1) + i + 1], ey[j * m + i], ey[(j + 1) * m + i],
                              zs, lz, ldz, diag);
    }

    /** offdiag_s with the four edge coefficients of (i,j) given (left, right,
     * below, above), e.g. staged in shared memory. */
    template <bool CEN = false>
    __device__ __forceinline__ T offdiag_v(int i, int j, T el, T er, T ed, T eu, const T *zs, int lz, int ldz,
                                           T &diag) const {
        const bool l = px || i > 0, r = px || i < m - 1, d = py || j > 0, u = py || j < n - 1;
        const T zc = CEN ? zs[lz] : T(0);
        diag = diag_of(i, l, r, d, u, el, er, ed, eu);
        return mac_terms<CEN>(l, r, d, u, el, er, ed, eu, zs[lz - 1], zs[lz + 1], zs[lz - ldz], zs[lz + ldz], zc);
    }

    __device__ __forceinline__ void coef9(int i, int j, T a[9]) const {
        T diag;
        const T el = ex[j * (m + 1) + i], er = ex[j * (m + 1) + i + 1];
        const T ed = ey[j * m + i], eu = ey[(j + 1) * m + i];
        const bool l = px || i > 0, r = px || i < m - 1, d = py || j > 0, u = py || j < n - 1;
        diag = diag_of(i, l, r, d, u, el, er, ed, eu);
        a[0] = 0; a[1] = d ? yysp * ed : T(0); a[2] = 0;
        a[3] = l ? xxsp * el : T(0); a[4] = diag; a[5] = r ? xxsp * er : T(0);
        a[6] = 0; a[7] = u ? yysp * eu : T(0); a[8] = 0;
    }
};

/** Variable-density finite-element system (mgs_fem_varying_rho,
 * mgs_fem.hh:86-136, mgs_fem.cc:126-162). Unknowns are the m x n corner nodes
 * (m=m_fem, n=n_fem); c[j*m+i] is 1/rho of the cell below-left of node (i,j)
 * (fluid_2d.cc:1163-1170). With zpr the right column is a fixed (Dirichlet)
 * node whose off-diagonal entries vanish (mgs_fem.cc:19-20). */
template <class T>
struct FemOp {
    static constexpr bool kFivePoint = false;
    int m, n, px, py, zpr;
    T fm, fc, hex, hey;
    const T *c;

    /** Cell reciprocal densities around node (i,j) (cp(), mgs_fem.hh:99-106).
     * Cells outside a non-periodic grid read as zero; their entries are zero. */
    __device__ __forceinline__ void cells(int i, int j, T &cdl, T &cdr, T &cul, T &cur) const {
        const int ij = i + m * j;
        const bool r = px || i < m - 1, u = py || j < n - 1;
        const int di = (px && i == m - 1) ? 1 - m : 1;
        const int dj = (py && j == n - 1) ? m - m * n : m;
        cdl = c[ij];
        cdr = r ? c[ij + di] : T(0);
        cul = u ? c[ij + dj] : T(0);
        cur = (r && u) ? c[ij + di + dj] : T(0);
    }

    __device__ __forceinline__ void coef9(int i, int j, T a[9]) const {
        T cdl, cdr, cul, cur;
        cells(i, j, cdl, cdr, cul, cur);
        const bool l = px || i > 0, r = px || i < m - 1, d = py || j > 0, u = py || j < n - 1;
        const bool fix = zpr && i == m - 1;
        a[4] = fm * (!d ? ((l ? cul : T(0)) + (r ? cur : T(0)))
                        : (!u ? ((l ? cdl : T(0)) + (r ? cdr : T(0)))
                              : ((l ? (cul + cdl) : T(0)) + (r ? (cur + cdr) : T(0)))));
        if (fix) {
            a[0] = a[1] = a[2] = a[3] = a[5] = a[6] = a[7] = a[8] = 0;
            return;
        }
        a[0] = (d && l) ? fc * cdl : T(0);
        a[2] = (d && r) ? fc * cdr : T(0);
        a[6] = (u && l) ? fc * cul : T(0);
        a[8] = (u && r) ? fc * cur : T(0);
        a[1] = d ? ((l ? cdl : T(0)) + (r ? cdr : T(0))) * hey : T(0);
        a[7] = u ? ((l ? cul : T(0)) + (r ? cur : T(0))) * hey : T(0);
        a[3] = l ? ((d ? cdl : T(0)) + (u ? cul : T(0))) * hex : T(0);
        a[5] = r ? ((d ? cdr : T(0)) + (u ? cur : T(0))) * hex : T(0);
    }

    template <bool CEN = false>
    __device__ __forceinline__ T offdiag_s(int i, int j, const T *zs, int lz, int ldz, T &diag) const {
        const int ij = i + m * j;
        if (i > 0 && i < m - 1 && j > 0 && j < n - 1)
            return offdiag_int<CEN>(c[ij], c[ij + 1], c[ij + m], c[ij + m + 1], zs, lz, ldz, diag);
        return offdiag_edge<CEN>(i, j, zs, lz, ldz, diag);
    }

    /** offdiag_s at an interior node, the four cell values around it given
     * (below-left, below-right, above-left, above-right). */
    template <bool CEN = false>
    __device__ __forceinline__ T offdiag_int(T cdl, T cdr, T cul, T cur, const T *zs, int lz, int ldz,
                                             T &diag) const {
        const T zc = CEN ? zs[lz] : T(0);
        diag = mul_rn(fm, add_rn(add_rn(cul, cdl), add_rn(cur, cdr)));
        const T *w = zs + lz;
        // each cell's three neighbours: x-edge (hex), corner (fc), y-edge (hey)
        auto cell = [&](int ox, int oy) {
            return fma_rn(cen<CEN>(w[oy], zc), hey,
                          fma_rn(cen<CEN>(w[ox + oy], zc), fc, mul_rn(cen<CEN>(w[ox], zc), hex)));
        };
        return fma_rn(cdr, cell(1, -ldz), fma_rn(cur, cell(1, ldz), fma_rn(cdl, cell(-1, -ldz), mul_rn(cul, cell(-1, ldz)))));
    }

    /** offdiag_s at a node on an edge of the grid (the cells from c). */
    template <bool CEN = false>
    __device__ __forceinline__ T offdiag_edge(int i, int j, const T *zs, int lz, int ldz, T &diag) const {
        const T zc = CEN ? zs[lz] : T(0);
        T a[9];
        coef9(i, j, a);
        diag = a[4];
        const bool l = px || i > 0, r = px || i < m - 1, d = py || j > 0, u = py || j < n - 1;
        T t = 0;
        if (d) {
            if (l) t = acc_rn(t, a[0], cen<CEN>(zs[lz - ldz - 1], zc));
            t = acc_rn(t, a[1], cen<CEN>(zs[lz - ldz], zc));
            if (r) t = acc_rn(t, a[2], cen<CEN>(zs[lz - ldz + 1], zc));
        }
        if (l) t = acc_rn(t, a[3], cen<CEN>(zs[lz - 1], zc));
        if (r) t = acc_rn(t, a[5], cen<CEN>(zs[lz + 1], zc));
        if (u) {
            if (l) t = acc_rn(t, a[6], cen<CEN>(zs[lz + ldz - 1], zc));
            t = acc_rn(t, a[7], cen<CEN>(zs[lz + ldz], zc));
            if (r) t = acc_rn(t, a[8], cen<CEN>(zs[lz + ldz + 1], zc));
        }
        return t;
    }

    template <bool CEN = false>
    __device__ __forceinline__ T offdiag(int i, int j, const T *z, T &diag, T zc = T(0)) const {
        const int ij = i + m * j;
        // (zc is the iterate at (i,j) in the centred form: z[ij] itself)
        if (i > 0 && i < m - 1 && j > 0 && j < n - 1)
            return offdiag_int<CEN>(c[ij], c[ij + 1], c[ij + m], c[ij + m + 1], z, ij, m, diag);
        if (!CEN) zc = T(0);
        T a[9];
        coef9(i, j, a);
        diag = a[4];
        const int il = i > 0 ? -1 : m - 1, ir = i < m - 1 ? 1 : 1 - m;
        const int jd = j > 0 ? -m : m * (n - 1), ju = j < n - 1 ? m : -m * (n - 1);
        const bool l = px || i > 0, r = px || i < m - 1, d = py || j > 0, u = py || j < n - 1;
        T t = 0;
        if (d) {
            if (l) t = acc_rn(t, a[0], cen<CEN>(z[ij + jd + il], zc));
            t = acc_rn(t, a[1], cen<CEN>(z[ij + jd], zc));
            if (r) t = acc_rn(t, a[2], cen<CEN>(z[ij + jd + ir], zc));
        }
        if (l) t = acc_rn(t, a[3], cen<CEN>(z[ij + il], zc));
        if (r) t = acc_rn(t, a[5], cen<CEN>(z[ij + ir], zc));
        if (u) {
            if (l) t = acc_rn(t, a[6], cen<CEN>(z[ij + ju + il], zc));
            t = acc_rn(t, a[7], cen<CEN>(z[ij + ju], zc));
            if (r) t = acc_rn(t, a[8], cen<CEN>(z[ij + ju + ir], zc));
        }
        return t;
    }

    /** Row sum: zero (the bilinear basis functions sum to one, so every
     * Neumann row annihilates constants) except in the fixed column, whose
     * row is its diagonal alone (mgs_fem.cc:19-20). */
    __device__ __forceinline__ T rowsum(int i, int j) const {
        if (!(zpr && i == m - 1)) return T(0);
        T a[9];
        coef9(i, j, a);
        return a[4];
    }
};

/** Position of unknown (i,j) of an m x n level in the colour-split layout
 * of the Galerkin stencils: the four Gauss-Seidel colours (i mod 2, j mod 2)
 * each hold a contiguous row-major block, in the order (0,0), (1,0), (0,1),
 * (1,1). A colour phase of the smoothers then reads its points' entries
 * contiguously (every byte of each 32-byte sector, once per sweep) instead
 * of every second entry of a row in each of the two phases that share the
 * row's sectors. */
__host__ __device__ __forceinline__ long colour_index(int m, int n, int i, int j) {
    const int pi = i & 1, pj = j & 1;
    const long m0 = (m + 1) >> 1, m1 = m >> 1, n0 = (n + 1) >> 1;
    const long base = (pj ? static_cast<long>(m) * n0 : 0) + (pi ? (pj ? m0 * (n >> 1) : m0 * n0) : 0);
    return base + static_cast<long>(j >> 1) * (pi ? m1 : m0) + (i >> 1);
}

/** A Galerkin coarse level: explicit 9-point stencil stored structure-of-
 * arrays, entry k of unknown (i,j) at st[k*N + colour_index(m, n, i, j)]. */
template <class T>
struct GenOp {
    static constexpr bool kFivePoint = false;
    int m, n, px, py;
    long N;
    const T *st;

    __device__ __forceinline__ long at(int i, int j) const { return colour_index(m, n, i, j); }

    __device__ __forceinline__ void coef9(int i, int j, T a[9]) const {
        const long q = at(i, j);
#pragma unroll
        for (int k = 0; k < 9; k++) a[k] = st[k * N + q];
    }

    /** With CEN (the single-precision stencils, whose entry 4 holds the row
     * sum, see galerkin_all), the centred off-diagonal sum; diag is then the
     * row sum minus the off-diagonal entries. */
    template <bool CEN = false>
    __device__ __forceinline__ T offdiag_s(int i, int j, const T *zs, int lz, int ldz, T &diag) const {
        const long q = at(i, j);
        const T zc = CEN ? zs[lz] : T(0);
        diag = st[4 * N + q];
        return gen_sum<CEN>(px || i > 0, px || i < m - 1, py || j > 0, py || j < n - 1, st + q, N, zs + lz, 1, ldz,
                            zc, diag);
    }

    /** The off-diagonal sum over the entries c[k*ldc] (k = 0..8, in the
     * order dl,dc,dr,cl,cr,ul,uc,ur) of a point whose iterate is w[0],
     * neighbours at w[+-dx], w[+-dy]; diag holds entry 4 on entry and, with
     * CEN, the row sum minus the off-diagonal entries on return. Shared by
     * every nine-point smoother so that all of them round alike. */
    template <bool CEN, class C>
    static __device__ __forceinline__ T gen_sum(bool l, bool r, bool d, bool u, const C *c, long ldc, const T *w,
                                                int dx, int dy, T zc, T &diag) {
        // Every entry and neighbour is read unconditionally (the point's own
        // entries, and neighbours inside the caller's array: a shared-memory
        // tile with a halo, or a wrapped global index), so that all eighteen
        // loads can be in flight at once; the terms outside the grid are then
        // skipped by selection, which leaves the sum as the branches would.
        const T k0 = c[0], k1 = c[ldc], k2 = c[2 * ldc], k3 = c[3 * ldc], k5 = c[5 * ldc], k6 = c[6 * ldc],
                k7 = c[7 * ldc], k8 = c[8 * ldc];
        const T z0 = w[-dy - dx], z1 = w[-dy], z2 = w[-dy + dx], z3 = w[-dx], z5 = w[dx], z6 = w[dy - dx],
                z7 = w[dy], z8 = w[dy + dx];
        return gen_terms<CEN>(l, r, d, u, k0, k1, k2, k3, k5, k6, k7, k8, z0, z1, z2, z3, z5, z6, z7, z8, zc, diag);
    }

    /** The off-diagonal sum from the eight entries and neighbour values
     * (order dl,dc,dr,cl,cr,ul,uc,ur), terms outside the grid skipped. */
    template <bool CEN>
    static __device__ __forceinline__ T gen_terms(bool l, bool r, bool d, bool u, T k0, T k1, T k2, T k3, T k5, T k6,
                                                  T k7, T k8, T z0, T z1, T z2, T z3, T z5, T z6, T z7, T z8, T zc,
                                                  T &diag) {
        T t = 0, a = 0;
        auto term = [&](bool on, T ck, T zk) {
            t = on ? acc_rn(t, ck, cen<CEN>(zk, zc)) : t;
            if constexpr (CEN) a = on ? add_rn(a, ck) : a;
        };
        term(d && l, k0, z0);
        term(d, k1, z1);
        term(d && r, k2, z2);
        term(l, k3, z3);
        term(r, k5, z5);
        term(u && l, k6, z6);
        term(u, k7, z7);
        term(u && r, k8, z8);
        if constexpr (CEN) diag = sub_rn(diag, a);
        return t;
    }

    template <bool CEN = false>
    __device__ __forceinline__ T offdiag(int i, int j, const T *z, T &diag, T zc = T(0)) const {
        const int ij = i + m * j;
        const int il = i > 0 ? -1 : m - 1, ir = i < m - 1 ? 1 : 1 - m;
        const int jd = j > 0 ? -m : m * (n - 1), ju = j < n - 1 ? m : -m * (n - 1);
        const bool l = px || i > 0, r = px || i < m - 1, d = py || j > 0, u = py || j < n - 1;
        if (!CEN) zc = T(0);
        const T *c = st + at(i, j);
        diag = c[4 * N];
        const T *w = z + ij;
        return gen_terms<CEN>(l, r, d, u, c[0], c[N], c[2 * N], c[3 * N], c[5 * N], c[6 * N], c[7 * N], c[8 * N],
                              w[jd + il], w[jd], w[jd + ir], w[il], w[ir], w[ju + il], w[ju], w[ju + ir], zc, diag);
    }

    /** Row sum, stored in entry 4 of the single-precision stencils. */
    __device__ __forceinline__ T rowsum(int i, int j) const { return st[4 * N + at(i, j)]; }
};

/** A Gauss-Seidel update of unknown (i,j) with the iterate in global memory:
 * (b - offdiag)/diag in double precision, exactly the reference's
 * inv_cc; in single precision the centred form zc + (b - A z)/diag. */
/** The new value of a Gauss-Seidel update from the off-diagonal sum and the
 * diagonal: (b - off)/diag in double; zc + (b - off - rs zc)/diag in the
 * centred single-precision form (rs: the row sum). */
__device__ __forceinline__ double gs_value(double b, double off, double diag, double, double) {
    return sub_rn(b, off) / diag;
}
__device__ __forceinline__ float gs_value(float b, float off, float diag, float zc, float rs) {
    return add_rn(zc, fma_rn(-rs, zc, sub_rn(b, off)) / diag);
}

template <class Op, class T>
__device__ __forceinline__ T gs_update(const Op &op, int i, int j, const T *z, T b) {
    T diag;
    if constexpr (sizeof(T) == 8) {
        const T off = op.offdiag(i, j, z, diag);
        return gs_value(b, off, diag, T(0), T(0));
    } else {
        const T zc = z[i + static_cast<long>(op.m) * j];
        const T off = op.template offdiag<true>(i, j, z, diag, zc);
        return gs_value(b, off, diag, zc, op.rowsum(i, j));
    }
}

/** gs_update with the iterate in a shared-memory tile. */
template <class Op, class T>
__device__ __forceinline__ T gs_update_s(const Op &op, int i, int j, const T *zs, int lz, int ldz, T b) {
    T diag;
    if constexpr (sizeof(T) == 8) {
        const T off = op.offdiag_s(i, j, zs, lz, ldz, diag);
        return gs_value(b, off, diag, T(0), T(0));
    } else {
        const T zc = zs[lz];
        const T off = op.template offdiag_s<true>(i, j, zs, lz, ldz, diag);
        return gs_value(b, off, diag, zc, op.rowsum(i, j));
    }
}

/** The residual b - (A z)(i,j): b - offdiag - diag*z in double precision
 * (the reference's mul_a/a_cc), the centred form in single. */
template <class Op, class T>
__device__ __forceinline__ T residual_at(const Op &op, int i, int j, const T *z, T b) {
    T diag;
    const T zc = z[i + static_cast<long>(op.m) * j];
    if constexpr (sizeof(T) == 8) {
        const T off = op.offdiag(i, j, z, diag);
        return fma_rn(-diag, zc, sub_rn(b, off));
    } else {
        const T off = op.template offdiag<true>(i, j, z, diag, zc);
        return fma_rn(-op.rowsum(i, j), zc, sub_rn(b, off));
    }
}

}  // namespace incrmt
