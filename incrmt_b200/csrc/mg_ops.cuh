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

    __device__ __forceinline__ T offdiag(int i, int j, const T *z, T &diag) const {
        const int ij = i + m * j;
        const T el = ex[j * (m + 1) + i], er = ex[j * (m + 1) + i + 1];
        const T ed = ey[j * m + i], eu = ey[(j + 1) * m + i];
        const bool l = px || i > 0, r = px || i < m - 1, d = py || j > 0, u = py || j < n - 1;
        T sx = 0, sy = 0;
        if (l) sx = el * z[i > 0 ? ij - 1 : ij + m - 1];
        if (r) sx += er * z[i < m - 1 ? ij + 1 : ij + 1 - m];
        if (d) sy = ed * z[j > 0 ? ij - m : ij + m * (n - 1)];
        if (u) sy += eu * z[j < n - 1 ? ij + m : ij - m * (n - 1)];
        diag = mac_diag(-xxsp * ((l ? el : T(0)) + (px ? er : (i < m - 1 ? er : (zpr ? 2 * er : T(0))))),
                        yysp, (d ? ed : T(0)) + (u ? eu : T(0)));
        return xxsp * sx + yysp * sy;
    }

    /** offdiag with the iterate in a shared-memory tile (lz: local index of
     * (i,j), ldz: tile row stride). The tile holds the neighbours at lz+-1,
     * lz+-ldz, across a periodic edge too (as periodic images). */
    __device__ __forceinline__ T offdiag_s(int i, int j, const T *zs, int lz, int ldz, T &diag) const {
        const T el = ex[j * (m + 1) + i], er = ex[j * (m + 1) + i + 1];
        const T ed = ey[j * m + i], eu = ey[(j + 1) * m + i];
        const bool l = px || i > 0, r = px || i < m - 1, d = py || j > 0, u = py || j < n - 1;
        T sx = 0, sy = 0;
        if (l) sx = el * zs[lz - 1];
        if (r) sx += er * zs[lz + 1];
        if (d) sy = ed * zs[lz - ldz];
        if (u) sy += eu * zs[lz + ldz];
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

    __device__ __forceinline__ T offdiag_s(int i, int j, const T *zs, int lz, int ldz, T &diag) const {
        const int ij = i + m * j;
        if (i > 0 && i < m - 1 && j > 0 && j < n - 1) {
            const T cdl = c[ij], cdr = c[ij + 1], cul = c[ij + m], cur = c[ij + m + 1];
            diag = fm * ((cul + cdl) + (cur + cdr));
            const T *w = zs + lz;
            return cul * (w[-1] * hex + w[ldz - 1] * fc + w[ldz] * hey)
                 + cdl * (w[-1] * hex + w[-ldz - 1] * fc + w[-ldz] * hey)
                 + cur * (w[1] * hex + w[ldz + 1] * fc + w[ldz] * hey)
                 + cdr * (w[1] * hex + w[-ldz + 1] * fc + w[-ldz] * hey);
        }
        T a[9];
        coef9(i, j, a);
        diag = a[4];
        const bool l = px || i > 0, r = px || i < m - 1, d = py || j > 0, u = py || j < n - 1;
        T t = 0;
        if (d) {
            if (l) t += a[0] * zs[lz - ldz - 1];
            t += a[1] * zs[lz - ldz];
            if (r) t += a[2] * zs[lz - ldz + 1];
        }
        if (l) t += a[3] * zs[lz - 1];
        if (r) t += a[5] * zs[lz + 1];
        if (u) {
            if (l) t += a[6] * zs[lz + ldz - 1];
            t += a[7] * zs[lz + ldz];
            if (r) t += a[8] * zs[lz + ldz + 1];
        }
        return t;
    }

    __device__ __forceinline__ T offdiag(int i, int j, const T *z, T &diag) const {
        const int ij = i + m * j;
        if (i > 0 && i < m - 1 && j > 0 && j < n - 1) {
            const T cdl = c[ij], cdr = c[ij + 1], cul = c[ij + m], cur = c[ij + m + 1];
            diag = fm * ((cul + cdl) + (cur + cdr));
            if (zpr && i == m - 1) return 0;
            const T *w = z + ij;
            return cul * (w[-1] * hex + w[m - 1] * fc + w[m] * hey)
                 + cdl * (w[-1] * hex + w[-m - 1] * fc + w[-m] * hey)
                 + cur * (w[1] * hex + w[m + 1] * fc + w[m] * hey)
                 + cdr * (w[1] * hex + w[-m + 1] * fc + w[-m] * hey);
        }
        T a[9];
        coef9(i, j, a);
        diag = a[4];
        const int il = i > 0 ? -1 : m - 1, ir = i < m - 1 ? 1 : 1 - m;
        const int jd = j > 0 ? -m : m * (n - 1), ju = j < n - 1 ? m : -m * (n - 1);
        const bool l = px || i > 0, r = px || i < m - 1, d = py || j > 0, u = py || j < n - 1;
        T t = 0;
        if (d) {
            if (l) t += a[0] * z[ij + jd + il];
            t += a[1] * z[ij + jd];
            if (r) t += a[2] * z[ij + jd + ir];
        }
        if (l) t += a[3] * z[ij + il];
        if (r) t += a[5] * z[ij + ir];
        if (u) {
            if (l) t += a[6] * z[ij + ju + il];
            t += a[7] * z[ij + ju];
            if (r) t += a[8] * z[ij + ju + ir];
        }
        return t;
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

    __device__ __forceinline__ T offdiag_s(int i, int j, const T *zs, int lz, int ldz, T &diag) const {
        const int ij = i + m * j;
        const bool l = px || i > 0, r = px || i < m - 1, d = py || j > 0, u = py || j < n - 1;
        diag = st[4 * N + ij];
        T t = 0;
        if (d) {
            if (l) t += st[ij] * zs[lz - ldz - 1];
            t += st[N + ij] * zs[lz - ldz];
            if (r) t += st[2 * N + ij] * zs[lz - ldz + 1];
        }
        if (l) t += st[3 * N + ij] * zs[lz - 1];
        if (r) t += st[5 * N + ij] * zs[lz + 1];
        if (u) {
            if (l) t += st[6 * N + ij] * zs[lz + ldz - 1];
            t += st[7 * N + ij] * zs[lz + ldz];
            if (r) t += st[8 * N + ij] * zs[lz + ldz + 1];
        }
        return t;
    }

    __device__ __forceinline__ T offdiag(int i, int j, const T *z, T &diag) const {
        const int ij = i + m * j;
        const int il = i > 0 ? -1 : m - 1, ir = i < m - 1 ? 1 : 1 - m;
        const int jd = j > 0 ? -m : m * (n - 1), ju = j < n - 1 ? m : -m * (n - 1);
        const bool l = px || i > 0, r = px || i < m - 1, d = py || j > 0, u = py || j < n - 1;
        diag = st[4 * N + ij];
        T t = 0;
        if (d) {
            if (l) t += st[ij] * z[ij + jd + il];
            t += st[N + ij] * z[ij + jd];
            if (r) t += st[2 * N + ij] * z[ij + jd + ir];
        }
        if (l) t += st[3 * N + ij] * z[ij + il];
        if (r) t += st[5 * N + ij] * z[ij + ir];
        if (u) {
            if (l) t += st[6 * N + ij] * z[ij + ju + il];
            t += st[7 * N + ij] * z[ij + ju];
            if (r) t += st[8 * N + ij] * z[ij + ju + ir];
        }
        return t;
    }
};

}  // namespace incrmt
