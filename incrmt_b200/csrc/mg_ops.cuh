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

/** a - b*c with the product rounded before the difference in double (the
 * reference's a_cc, mgs_mac.hh:93-97, evaluated as the CPU does, without a
 * fused multiply-add), so that the MAC diagonal and the prolongation weights
 * built from it agree with the oracle's to the last bit; fused in single. */
__device__ __forceinline__ double mac_diag(double a, double b, double c) { return __dsub_rn(a, __dmul_rn(b, c)); }
__device__ __forceinline__ float mac_diag(float a, float b, float c) { return a - b * c; }

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
        T sx = 0, sy = 0;
        if (l) sx = el * (z[i > 0 ? ij - 1 : ij + m - 1] - (CEN ? zc : T(0)));
        if (r) sx += er * (z[i < m - 1 ? ij + 1 : ij + 1 - m] - (CEN ? zc : T(0)));
        if (d) sy = ed * (z[j > 0 ? ij - m : ij + m * (n - 1)] - (CEN ? zc : T(0)));
        if (u) sy += eu * (z[j < n - 1 ? ij + m : ij - m * (n - 1)] - (CEN ? zc : T(0)));
        diag = mac_diag(-xxsp * ((l ? el : T(0)) + (px ? er : (i < m - 1 ? er : (zpr ? 2 * er : T(0))))),
                        yysp, (d ? ed : T(0)) + (u ? eu : T(0)));
        return xxsp * sx + yysp * sy;
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
        T sx = 0, sy = 0;
        if (l) sx = el * (zs[lz - 1] - zc);
        if (r) sx += er * (zs[lz + 1] - zc);
        if (d) sy = ed * (zs[lz - ldz] - zc);
        if (u) sy += eu * (zs[lz + ldz] - zc);
        diag = mac_diag(-xxsp * ((l ? el : T(0)) + (px ? er : (i < m - 1 ? er : (zpr ? 2 * er : T(0))))),
                        yysp, (d ? ed : T(0)) + (u ? eu : T(0)));
        return xxsp * sx + yysp * sy;
    }

    __device__ __forceinline__ void coef9(int i, int j, T a[9]) const {
        T diag;
        const T el = ex[j * (m + 1) + i], er = ex[j * (m + 1) + i + 1];
        const T ed = ey[j * m + i], eu = ey[(j + 1) * m + i];
        const bool l = px || i > 0, r = px || i < m - 1, d = py || j > 0, u = py || j < n - 1;
        diag = mac_diag(-xxsp * ((l ? el : T(0)) + (px ? er : (i < m - 1 ? er : (zpr ? 2 * er : T(0))))),
                        yysp, (d ? ed : T(0)) + (u ? eu : T(0)));
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
        diag = fm * ((cul + cdl) + (cur + cdr));
        const T *w = zs + lz;
        return cul * ((w[-1] - zc) * hex + (w[ldz - 1] - zc) * fc + (w[ldz] - zc) * hey)
             + cdl * ((w[-1] - zc) * hex + (w[-ldz - 1] - zc) * fc + (w[-ldz] - zc) * hey)
             + cur * ((w[1] - zc) * hex + (w[ldz + 1] - zc) * fc + (w[ldz] - zc) * hey)
             + cdr * ((w[1] - zc) * hex + (w[-ldz + 1] - zc) * fc + (w[-ldz] - zc) * hey);
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
            if (l) t += a[0] * (zs[lz - ldz - 1] - zc);
            t += a[1] * (zs[lz - ldz] - zc);
            if (r) t += a[2] * (zs[lz - ldz + 1] - zc);
        }
        if (l) t += a[3] * (zs[lz - 1] - zc);
        if (r) t += a[5] * (zs[lz + 1] - zc);
        if (u) {
            if (l) t += a[6] * (zs[lz + ldz - 1] - zc);
            t += a[7] * (zs[lz + ldz] - zc);
            if (r) t += a[8] * (zs[lz + ldz + 1] - zc);
        }
        return t;
    }

    template <bool CEN = false>
    __device__ __forceinline__ T offdiag(int i, int j, const T *z, T &diag, T zc = T(0)) const {
        const int ij = i + m * j;
        if (!CEN) zc = T(0);
        if (i > 0 && i < m - 1 && j > 0 && j < n - 1) {
            const T cdl = c[ij], cdr = c[ij + 1], cul = c[ij + m], cur = c[ij + m + 1];
            diag = fm * ((cul + cdl) + (cur + cdr));
            if (zpr && i == m - 1) return 0;
            const T *w = z + ij;
            return cul * ((w[-1] - zc) * hex + (w[m - 1] - zc) * fc + (w[m] - zc) * hey)
                 + cdl * ((w[-1] - zc) * hex + (w[-m - 1] - zc) * fc + (w[-m] - zc) * hey)
                 + cur * ((w[1] - zc) * hex + (w[m + 1] - zc) * fc + (w[m] - zc) * hey)
                 + cdr * ((w[1] - zc) * hex + (w[-m + 1] - zc) * fc + (w[-m] - zc) * hey);
        }
        T a[9];
        coef9(i, j, a);
        diag = a[4];
        const int il = i > 0 ? -1 : m - 1, ir = i < m - 1 ? 1 : 1 - m;
        const int jd = j > 0 ? -m : m * (n - 1), ju = j < n - 1 ? m : -m * (n - 1);
        const bool l = px || i > 0, r = px || i < m - 1, d = py || j > 0, u = py || j < n - 1;
        T t = 0;
        if (d) {
            if (l) t += a[0] * (z[ij + jd + il] - zc);
            t += a[1] * (z[ij + jd] - zc);
            if (r) t += a[2] * (z[ij + jd + ir] - zc);
        }
        if (l) t += a[3] * (z[ij + il] - zc);
        if (r) t += a[5] * (z[ij + ir] - zc);
        if (u) {
            if (l) t += a[6] * (z[ij + ju + il] - zc);
            t += a[7] * (z[ij + ju] - zc);
            if (r) t += a[8] * (z[ij + ju + ir] - zc);
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

/** A Galerkin coarse level: explicit 9-point stencil stored structure-of-
 * arrays, entry k of unknown ij at st[k*N+ij]. */
template <class T>
struct GenOp {
    static constexpr bool kFivePoint = false;
    int m, n, px, py;
    long N;
    const T *st;

    __device__ __forceinline__ void coef9(int i, int j, T a[9]) const {
        const int ij = i + m * j;
#pragma unroll
        for (int k = 0; k < 9; k++) a[k] = st[k * N + ij];
    }

    /** With CEN (the single-precision stencils, whose entry 4 holds the row
     * sum, see galerkin_all), the centred off-diagonal sum; diag is then the
     * row sum minus the off-diagonal entries. */
    template <bool CEN = false>
    __device__ __forceinline__ T offdiag_s(int i, int j, const T *zs, int lz, int ldz, T &diag) const {
        const int ij = i + m * j;
        const bool l = px || i > 0, r = px || i < m - 1, d = py || j > 0, u = py || j < n - 1;
        const T zc = CEN ? zs[lz] : T(0);
        diag = st[4 * N + ij];
        T t = 0, a = 0;
        if (d) {
            if (l) { t += st[ij] * (zs[lz - ldz - 1] - zc); a += st[ij]; }
            t += st[N + ij] * (zs[lz - ldz] - zc); a += st[N + ij];
            if (r) { t += st[2 * N + ij] * (zs[lz - ldz + 1] - zc); a += st[2 * N + ij]; }
        }
        if (l) { t += st[3 * N + ij] * (zs[lz - 1] - zc); a += st[3 * N + ij]; }
        if (r) { t += st[5 * N + ij] * (zs[lz + 1] - zc); a += st[5 * N + ij]; }
        if (u) {
            if (l) { t += st[6 * N + ij] * (zs[lz + ldz - 1] - zc); a += st[6 * N + ij]; }
            t += st[7 * N + ij] * (zs[lz + ldz] - zc); a += st[7 * N + ij];
            if (r) { t += st[8 * N + ij] * (zs[lz + ldz + 1] - zc); a += st[8 * N + ij]; }
        }
        if (CEN) diag -= a;
        return t;
    }

    template <bool CEN = false>
    __device__ __forceinline__ T offdiag(int i, int j, const T *z, T &diag, T zc = T(0)) const {
        const int ij = i + m * j;
        const int il = i > 0 ? -1 : m - 1, ir = i < m - 1 ? 1 : 1 - m;
        const int jd = j > 0 ? -m : m * (n - 1), ju = j < n - 1 ? m : -m * (n - 1);
        const bool l = px || i > 0, r = px || i < m - 1, d = py || j > 0, u = py || j < n - 1;
        if (!CEN) zc = T(0);
        diag = st[4 * N + ij];
        T t = 0, a = 0;
        if (d) {
            if (l) { t += st[ij] * (z[ij + jd + il] - zc); a += st[ij]; }
            t += st[N + ij] * (z[ij + jd] - zc); a += st[N + ij];
            if (r) { t += st[2 * N + ij] * (z[ij + jd + ir] - zc); a += st[2 * N + ij]; }
        }
        if (l) { t += st[3 * N + ij] * (z[ij + il] - zc); a += st[3 * N + ij]; }
        if (r) { t += st[5 * N + ij] * (z[ij + ir] - zc); a += st[5 * N + ij]; }
        if (u) {
            if (l) { t += st[6 * N + ij] * (z[ij + ju + il] - zc); a += st[6 * N + ij]; }
            t += st[7 * N + ij] * (z[ij + ju] - zc); a += st[7 * N + ij];
            if (r) { t += st[8 * N + ij] * (z[ij + ju + ir] - zc); a += st[8 * N + ij]; }
        }
        if (CEN) diag -= a;
        return t;
    }

    /** Row sum, stored in entry 4 of the single-precision stencils. */
    __device__ __forceinline__ T rowsum(int i, int j) const { return st[4 * N + i + static_cast<long>(m) * j]; }
};

/** A Gauss-Seidel update of unknown (i,j) with the iterate in global memory:
 * (b - offdiag)/diag in double precision, exactly the reference's
 * inv_cc; in single precision the centred form zc + (b - A z)/diag. */
template <class Op, class T>
__device__ __forceinline__ T gs_update(const Op &op, int i, int j, const T *z, T b) {
    T diag;
    if constexpr (sizeof(T) == 8) {
        const T off = op.offdiag(i, j, z, diag);
        return (b - off) / diag;
    } else {
        const T zc = z[i + static_cast<long>(op.m) * j];
        const T off = op.template offdiag<true>(i, j, z, diag, zc);
        return zc + (b - off - op.rowsum(i, j) * zc) / diag;
    }
}

/** gs_update with the iterate in a shared-memory tile. */
template <class Op, class T>
__device__ __forceinline__ T gs_update_s(const Op &op, int i, int j, const T *zs, int lz, int ldz, T b) {
    T diag;
    if constexpr (sizeof(T) == 8) {
        const T off = op.offdiag_s(i, j, zs, lz, ldz, diag);
        return (b - off) / diag;
    } else {
        const T zc = zs[lz];
        const T off = op.template offdiag_s<true>(i, j, zs, lz, ldz, diag);
        return zc + (b - off - op.rowsum(i, j) * zc) / diag;
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
        return b - off - diag * zc;
    } else {
        const T off = op.template offdiag<true>(i, j, z, diag, zc);
        return b - off - op.rowsum(i, j) * zc;
    }
}

}  // namespace incrmt
