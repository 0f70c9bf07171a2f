// Narrow-band level-set reinitialisation (levelset::build_band,
// levelset.cc:199-335) and reference-map extrapolation
// (levelset::extrapolate_fields, traverse.hh:169-260) on the GPU.
//
// The level-set grid is the ghosted fluid grid: mL=m+4 by nL=n+4 points,
// origin ax-1.5dx (obj_field.cc:18), stored with the fluid row pitch P, so
// level-set point (i,j) is at j*P+i.
//
// Reinitialisation. The reference (1) classifies each point by the sign of
// phi and of its four neighbours, (2) moves the points next to the interface
// to the signed distance of the closest zero of a bicubic interpolant
// (Newton), and (3) fast-marches outwards on each side with a second-order
// upwind stencil (heap.cc:177-376), accepting points in increasing |phi|
// until the band limit. The march is sequential; here step (3) is the
// fixed point of the same stencil: a point's value is the stencil evaluated
// with "in" neighbours = interface points plus same-side points whose
// current value is smaller, iterated (Jacobi, double-buffered) until no value
// changes. In exact arithmetic this is the value the march assigns, since a
// marched point's final value is the stencil over the points accepted before
// it, which are those with smaller values.
//
// Extrapolation. The reference visits the band in increasing phi and fits
// each point outside the solid by weighted least squares over already-visited
// neighbours with smaller phi; the result depends only on phi, so it is
// computed as a wavefront (Jacobi) iteration over the outside band points
// that stops when no value changes; the dependency depth is ~65 for the
// ~7-cell-wide band, independent of the grid size.
#pragma once
#include <cooperative_groups.h>
#include "sim.cuh"

namespace incrmt {

struct LsGrid {
    int mL, nL, P;
    double axl, ayl, dx, dy, xsp, ysp;
    double phi_up, phi_down;
};

/** Level-set arrays of one object. The batched kernels below take an array
 * of these and treat blockIdx.z as the object index; the cooperative ones
 * take a combined point list whose entries carry their object index, so
 * every object's band is rebuilt (or extrapolated) in the same launches. */
struct LsObj {
    double *phi;             // level set (ghosted grid, pitch P)
    int *s;                  // status
    double *phi_new;         // Newton distances of the interface points
    double *a, *b;           // march values, or extrapolated X (ping-pong)
    double *c, *d;           // extrapolated Y (ping-pong)
    unsigned char *ca, *cb;  // change marks of the previous / current sweep
    int *ia, *ib;            // dilation masks; trial statuses
    double *nX, *nY;         // reference map being extrapolated
};

// Status values (levelset.cc:211-263, heap.cc): 0/7 far negative/positive,
// 1/6 trial, 2/5 accepted by the march, 3/4 next to the interface.

/** Point (i,j) of thread (x,y) in object blockIdx.z's window; false
 * outside it. */
__device__ __forceinline__ bool ls_point(const LsGrid &g, const LsWin *win, int &i, int &j) {
    const LsWin w = win[blockIdx.z];
    i = w.x0 + blockIdx.x * blockDim.x + threadIdx.x;
    j = w.y0 + blockIdx.y * blockDim.y + threadIdx.y;
    return i < w.x1 && j < w.y1 && i < g.mL && j < g.nL;
}

/** Sign classification (levelset.cc:209-263): s=4 for phi>0 with a 4-neighbour
 * phi<=0, s=3 for phi<=0 with a neighbour phi>0, else 7 / 0. */
__global__ void k_ls_scan(LsGrid g, const LsObj *ob, const LsWin *win, int *box) {
    __shared__ int sb[4];
    if (threadIdx.x == 0 && threadIdx.y == 0) sb[0] = sb[1] = sb[2] = sb[3] = 0x7fffffff;
    __syncthreads();
    int i, j;
    const bool live = ls_point(g, win, i, j);
    bool keep = false;
    if (live) {
        const double *phi = ob[blockIdx.z].phi;
        int *s = ob[blockIdx.z].s;
        const int ij = j * g.P + i;
        const bool pos = phi[ij] > 0;
        bool diff = false;
        if (i > 0) diff |= (phi[ij - 1] > 0) != pos;
        if (i < g.mL - 1) diff |= (phi[ij + 1] > 0) != pos;
        if (j > 0) diff |= (phi[ij - g.P] > 0) != pos;
        if (j < g.nL - 1) diff |= (phi[ij + g.P] > 0) != pos;
        const int st = pos ? (diff ? 4 : 7) : (diff ? 3 : 0);
        s[ij] = st;
        keep = st != 7;
    }
    // Bounding box of the points inside the solid or next to its interface:
    // a warp is one row, so its extent comes from the ballot; the block's
    // warps meet in shared memory and one thread updates the object's box
    // (minima of x, y, -x, -y).
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    if (bal && (threadIdx.x & 31) == 0) {
        const int xb = i - static_cast<int>(threadIdx.x & 31);
        atomicMin(&sb[0], xb + __ffs(bal) - 1);
        atomicMin(&sb[1], j);
        atomicMin(&sb[2], -(xb + 31 - __clz(bal)));
        atomicMin(&sb[3], -j);
    }
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0 && sb[0] != 0x7fffffff) {
        int *b = box + 4 * blockIdx.z;
        atomicMin(&b[0], sb[0]);
        atomicMin(&b[1], sb[1]);
        atomicMin(&b[2], sb[2]);
        atomicMin(&b[3], sb[3]);
    }
}

/** One-dimensional Hermite weights of the reference's bicubic
 * (levelset/built/bicubic.cc): value weights for the two nodes (a0,a1) and
 * for their slopes (b0,b1), and their derivatives. kind 1 is the cubic
 * interior patch, 0 the quadratic patch at the low edge (no slope at node 0),
 * 2 the quadratic patch at the high edge (no slope at node 1). */
__device__ __forceinline__ void hermite_w(int kind, double e, double &a0, double &a1, double &b0, double &b1,
                                          double &da0, double &da1, double &db0, double &db1) {
    const double me = 1 - e;
    if (kind == 1) {
        a0 = me * me * (1 + 2 * e); a1 = e * e * (3 - 2 * e); b0 = e * me * me; b1 = -e * e * me;
        da0 = -6 * e * me; da1 = 6 * e * me; db0 = me * (1 - 3 * e); db1 = e * (3 * e - 2);
    } else if (kind == 0) {
        a0 = me * me; a1 = e * (2 - e); b0 = 0; b1 = -e * me;
        da0 = -2 * me; da1 = 2 * me; db0 = 0; db1 = 2 * e - 1;
    } else {
        a0 = 1 - e * e; a1 = e * e; b0 = e * me; b1 = 0;
        da0 = -2 * e; da1 = 2 * e; db0 = 1 - 2 * e; db1 = 0;
    }
}

/** Bicubic interpolation of phi with its gradient (levelset::bicubic,
 * levelset.cc:67-79, built/bicubic.cc): a tensor-product Hermite patch whose
 * nodal slopes are central differences (and the cross slope a central second
 * difference), with quadratic one-sided patches in the first and last cell of
 * each direction. Points outside the grid use the nearest edge patch. */
__device__ double ls_bicubic(const LsGrid &g, const double *phi, double x, double y, double &phix, double &phiy) {
    double e = (x - g.axl) * g.xsp, f = (y - g.ayl) * g.ysp;
    const int i = static_cast<int>(e), j = static_cast<int>(f);
    int kx, ky, ci, cj;
    if (i < 1) { kx = 0; ci = 0; }
    else if (i >= g.mL - 2) { kx = 2; ci = g.mL - 2; e -= static_cast<double>(g.mL - 2); }
    else { kx = 1; ci = i; e -= static_cast<double>(i); }
    if (j < 1) { ky = 0; cj = 0; }
    else if (j >= g.nL - 2) { ky = 2; cj = g.nL - 2; f -= static_cast<double>(g.nL - 2); }
    else { ky = 1; cj = j; f -= static_cast<double>(j); }
    double a0, a1, b0, b1, da0, da1, db0, db1;
    hermite_w(kx, e, a0, a1, b0, b1, da0, da1, db0, db1);
    double c0, c1, d0, d1, dc0, dc1, dd0, dd1;
    hermite_w(ky, f, c0, c1, d0, d1, dc0, dc1, dd0, dd1);
    const int P = g.P;
    // Row values V (and d/de) and row y-slopes W at rows cj, cj+1.
    double V[2], Vd[2], W[2], Wd[2];
    for (int r = 0; r < 2; r++) {
        const int rr = cj + r;
        const bool needW = (r == 0) ? (ky != 0) : (ky != 2);
        const int q0 = rr * P + ci, q1 = q0 + 1;
        double sx0 = 0, sx1 = 0;
        if (kx != 0) sx0 = (phi[q0 + 1] - phi[q0 - 1]) * 0.5;
        if (kx != 2) sx1 = (phi[q1 + 1] - phi[q1 - 1]) * 0.5;
        V[r] = a0 * phi[q0] + a1 * phi[q1] + b0 * sx0 + b1 * sx1;
        Vd[r] = da0 * phi[q0] + da1 * phi[q1] + db0 * sx0 + db1 * sx1;
        W[r] = Wd[r] = 0;
        if (needW) {
            const double sy0 = (phi[q0 + P] - phi[q0 - P]) * 0.5, sy1 = (phi[q1 + P] - phi[q1 - P]) * 0.5;
            double sxy0 = 0, sxy1 = 0;
            if (kx != 0) sxy0 = (phi[q0 + P + 1] - phi[q0 - P + 1] - phi[q0 + P - 1] + phi[q0 - P - 1]) * 0.25;
            if (kx != 2) sxy1 = (phi[q1 + P + 1] - phi[q1 - P + 1] - phi[q1 + P - 1] + phi[q1 - P - 1]) * 0.25;
            W[r] = a0 * sy0 + a1 * sy1 + b0 * sxy0 + b1 * sxy1;
            Wd[r] = da0 * sy0 + da1 * sy1 + db0 * sxy0 + db1 * sxy1;
        }
    }
    phix = g.xsp * (c0 * Vd[0] + c1 * Vd[1] + d0 * Wd[0] + d1 * Wd[1]);
    phiy = g.ysp * (dc0 * V[0] + dc1 * V[1] + dd0 * W[0] + dd1 * W[1]);
    return c0 * V[0] + c1 * V[1] + d0 * W[0] + d1 * W[1];
}

/** First-order fallback closest point (levelset::newton_failsafe,
 * levelset.cc:138-195), from the straight-line zero crossings to the
 * opposite-side interface neighbours. */
__device__ bool ls_failsafe(const LsGrid &g, const double *phi, const int *s, int i, int j, double x0, double y0,
                            double &x, double &y) {
    const int P = g.P, ij = j * P + i, ts = 7 - s[ij];
    const double cphi = phi[ij];
    bool hf, vf;
    double tdis;
    if (i > 0 && s[ij - 1] == ts) {
        x = cphi / (phi[ij - 1] - cphi);
        if (i < g.mL - 1 && s[ij + 1] == ts) {
            tdis = cphi / (cphi - phi[ij + 1]);
            if (tdis < -x) x = tdis;
        }
        hf = true;
    } else {
        if (i < g.mL - 1 && s[ij + 1] == ts) { x = cphi / (cphi - phi[ij + 1]); hf = true; }
        else hf = false;
    }
    if (j > 0 && s[ij - P] == ts) {
        y = cphi / (phi[ij - P] - cphi);
        if (j < g.nL - 1 && s[ij + P] == ts) {
            tdis = cphi / (cphi - phi[ij + P]);
            if (tdis < -y) y = tdis;
        }
        vf = true;
    } else {
        if (j < g.nL - 1 && s[ij + P] == ts) { y = cphi / (cphi - phi[ij + P]); vf = true; }
        else vf = false;
    }
    if (hf) {
        if (vf) {
            y *= g.dy;
            tdis = x * g.dx;
            const double c = tdis * y / (tdis * tdis + y * y);
            x = y * c + x0;
            y = tdis * c + y0;
        } else { x = x * g.dx + x0; y = y0; }
        return true;
    }
    if (vf) { x = x0; y = y * g.dy + y0; return true; }
    return false;
}

/** The reference's |v| as compiled: its unqualified abs() on a double binds to
 * int abs(int) (levelset.cc:124,126), i.e. |trunc(v)|. */
__device__ __forceinline__ double int_abs(double v) {
    int t = static_cast<int>(v);
    return static_cast<double>(t < 0 ? -t : t);
}

/** Closest-point Newton iteration of Chopp (levelset::newton,
 * levelset.cc:107-127) for the points next to the interface. Because of the
 * integer abs the loop ends after eight steps whose |phi| < 1 and the
 * closeness test is |x0-x| < 1, exactly as the reference runs. Writes the
 * signed distance to phi_new; sets *err on a failure (levelset.cc:275). */
__global__ void k_ls_newton(LsGrid g, const LsObj *ob, const LsWin *win, int *err) {
    int i, j;
    if (!ls_point(g, win, i, j)) return;
    const double *phi = ob[blockIdx.z].phi;
    const int *s = ob[blockIdx.z].s;
    double *phi_new = ob[blockIdx.z].phi_new;
    const int ij = j * g.P + i, st = s[ij];
    if (st != 3 && st != 4) return;
    const double dyy = g.dy / static_cast<double>(g.mL), step_limit = sqrt(g.dx * g.dx + g.dy * g.dy);
    const double x0 = g.axl + i * g.dx, y0 = g.ayl + static_cast<double>(j * g.mL) * dyy;
    double x = x0, y = y0, px, py;
    double ph = ls_bicubic(g, phi, x, y, px, py);
    int iter = 0, cutoff = 0;
    bool ok = true, fallback = false;
    do {
        const double delx = x0 - x, dely = y0 - y;
        double m0 = delx * px + dely * py + ph;
        const double m1 = px * px + py * py;
        iter++;
        m0 /= m1;
        if (iter > 100 || !isfinite(m0) || m0 > step_limit) { fallback = true; break; }
        x += delx - m0 * px;
        y += dely - m0 * py;
        ph = ls_bicubic(g, phi, x, y, px, py);
        if (int_abs(ph) < 1e-10) cutoff++; else cutoff = 0;
    } while (cutoff < 8);
    if (!fallback && !(int_abs(x0 - x) < 3 * g.dx && int_abs(y0 - y) < 3 * g.dy)) fallback = true;
    if (fallback) ok = ls_failsafe(g, phi, s, i, j, x0, y0, x, y);
    if (!ok) { atomicExch(err, INCRMT_ERR_NEWTON); phi_new[ij] = phi[ij]; return; }
    x -= x0;
    y -= y0;
    const double d = sqrt(x * x + y * y);
    phi_new[ij] = st == 4 ? d : -d;
}

__global__ void k_ls_copy_interface(LsGrid g, const LsObj *ob, const LsWin *win) {
    int i, j;
    if (!ls_point(g, win, i, j)) return;
    const LsObj &o = ob[blockIdx.z];
    const int ij = j * g.P + i;
    if (o.s[ij] == 3 || o.s[ij] == 4) o.phi[ij] = o.phi_new[ij];
}

/** Marching direction: positive side (dir_positive) or negative side
 * (dir_negative), heap.hh:56-80. */
template <bool POS>
struct MarchDir {
    __device__ static __forceinline__ bool cm(double a, double b) { return POS ? a < b : a > b; }
    __device__ static __forceinline__ double ct(double a, double b) { return POS ? a + b : a - b; }
};

/** The second-order upwind stencil of the fast march for one point
 * (heap<d_option>::calc and helpers, heap.cc:177-376, 390-435), with the
 * "in" predicate supplied by the caller. */
template <bool POS>
struct March {
    using D = MarchDir<POS>;
    const LsGrid &g;
    const double *phi;
    const int *s0;        // status after the sign scan
    const double *cur;    // current values of this side's candidates
    double pv;            // current value of the point being evaluated
    int lim_i, lim_j;
    double dx, dy, dx2, dy2, dxbydy, dx2bydy2;

    __device__ March(const LsGrid &g_, const double *phi_, const int *s0_, const double *cur_, double pv_)
        : g(g_), phi(phi_), s0(s0_), cur(cur_), pv(pv_) {
        dx = g.dx; dy = g.dy; dx2 = dx * dx; dy2 = dy * dy;
        dxbydy = dx / dy; dx2bydy2 = dxbydy * dxbydy;
    }
    /** Value of a point as seen by the stencil: fixed points keep phi, this
     * side's candidates their current value. */
    __device__ __forceinline__ double val(int ij) const {
        const int st = s0[ij];
        return (POS ? st == 7 : st == 0) ? cur[ij] : phi[ij];
    }
    /** Whether a point counts as accepted before the one being evaluated:
     * every point of the other side or of the interface, or a candidate of
     * this side with a smaller current value. */
    __device__ __forceinline__ bool in(int ij) const {
        const int st = s0[ij];
        if (POS ? st != 7 : st != 0) return true;
        return D::cm(cur[ij], pv);
    }
    __device__ bool look(int ij, int o, bool ok2, double &e) const {
        if (ok2 && in(ij + 2 * o)) {
            const double f2 = val(ij + 2 * o), f1 = val(ij + o);
            if (D::cm(f2, f1)) { e = 2 * f1 - 0.5 * f2; return true; }
        }
        e = val(ij + o);
        return false;
    }
    __device__ double corner_bail(bool h, bool v, double a, double b) const {
        const double ti = 2.0 / 3.0;
        double ht = h ? D::ct(a, dx) * ti : D::ct(a, dx);
        double vt = v ? D::ct(b, dy) * ti : D::ct(b, dy);
        return D::cm(ht, vt) ? ht : vt;
    }
    __device__ double corner(bool h, bool v, double a, double b) const {
        const double f2a = 2.25 * (dy2 + dx2), f2b = 2.25 * dy2 + dx2, f2c = dy2 + 2.25 * dx2, f2d = dy2 + dx2;
        const double b1 = 2.25 * dx2 > dy2 ? 1 + 2.25 * dx2bydy2 : 1 + dy2 / (2.25 * dx2);
        const double b2 = dx2 > dy2 ? 1 + dx2bydy2 : 1 + dy2 / dx2;
        const double b3 = dx2 > 2.25 * dy2 ? 1 + dx2bydy2 / 2.25 : 1 + 2.25 * dy2 / dx2;
        const double i2a = dy2 / f2a, i2b = dy2 / f2b, i2c = dy2 / f2c, i2d = dy2 / f2d;
        double f;
        if (h) {
            if (v) {
                f = 1.5 * (a - b); f *= f;
                return f * b2 < f2a ? D::ct(a * 1.5 + b * 1.5 * dx2bydy2, dxbydy * sqrt(f2a - f)) * i2a
                                    : corner_bail(true, true, a, b);
            }
            f = a - 1.5 * b; f *= f;
            return f * b3 < f2b ? D::ct(a * 1.5 + b * dx2bydy2, dxbydy * sqrt(f2b - f)) * i2b
                                : corner_bail(true, false, a, b);
        }
        if (v) {
            f = 1.5 * a - b; f *= f;
            return f * b1 < f2c ? D::ct(a + b * 1.5 * dx2bydy2, dxbydy * sqrt(f2c - f)) * i2c
                                : corner_bail(false, true, a, b);
        }
        f = a - b; f *= f;
        return f * b2 < f2d ? D::ct(a + b * dx2bydy2, dxbydy * sqrt(f2d - f)) * i2d
                            : corner_bail(false, false, a, b);
    }
    __device__ double fourway(double a, double b, double c, double d) const {
        double e = 2 * (c - a), f = 2 * (d - b), gg, h;
        if (D::cm(e, f)) {
            gg = e - a; h = e - b;
            if (D::cm(gg, 0)) gg = 0;
            if (D::cm(h, 0)) h = 0;
            if (gg * gg + h * h * dx2bydy2 < dx2) {
                gg = 1.5 * f - c; h = f - b;
                if (D::cm(gg, 0)) gg = 0;
                if (D::cm(h, 0)) h = 0;
                if (gg * gg + h * h * dx2bydy2 < dx2) return corner(true, true, c, d);
                return corner(true, false, c, b);
            }
            return corner(false, false, a, b);
        }
        gg = f - a; h = f - b;
        if (D::cm(gg, 0)) gg = 0;
        if (D::cm(h, 0)) h = 0;
        if (gg * gg + h * h * dx2bydy2 < dx2) {
            gg = e - a; h = 1.5 * e - d;
            if (D::cm(gg, 0)) gg = 0;
            if (D::cm(h, 0)) h = 0;
            if (gg * gg + h * h * dx2bydy2 < dx2) return corner(true, true, c, d);
            return corner(false, true, a, d);
        }
        return corner(false, false, a, b);
    }
    __device__ double threeway1(bool h1, bool h2, bool v, double a, double c, double b) const {
        double d;
        if (h1) {
            if (h2) { d = D::cm(a, c) ? a : c; return corner(true, v, d, b); }
            d = 2 * (a - c);
            double e = d - c, f = (v ? 1.5 * d : d) - b;
            if (D::cm(e, 0)) e = 0;
            if (D::cm(f, 0)) f = 0;
            return e * e + f * f * dx2bydy2 < dx2 ? corner(true, v, a, b) : corner(false, v, c, b);
        }
        if (h2) {
            d = 2 * (c - a);
            double e = d - a, f = (v ? 1.5 * d : d) - b;
            if (D::cm(e, 0)) e = 0;
            if (D::cm(f, 0)) f = 0;
            return e * e + f * f * dx2bydy2 < dx2 ? corner(true, v, c, b) : corner(false, v, a, b);
        }
        d = D::cm(a, c) ? a : c;
        return corner(false, v, d, b);
    }
    __device__ double threeway2(bool h, bool v1, bool v2, double b, double a, double c) const {
        double d;
        if (v1) {
            if (v2) { d = D::cm(a, c) ? a : c; return corner(h, true, b, d); }
            d = 2 * (a - c);
            double e = d - c, f = (h ? 1.5 * d : d) - b;
            if (D::cm(e, 0)) e = 0;
            if (D::cm(f, 0)) f = 0;
            return f * f + e * e * dx2bydy2 < dx2 ? corner(h, true, b, a) : corner(h, false, b, c);
        }
        if (v2) {
            d = 2 * (c - a);
            double e = d - a, f = (h ? 1.5 * d : d) - b;
            if (D::cm(e, 0)) e = 0;
            if (D::cm(f, 0)) f = 0;
            return f * f + e * e * dx2bydy2 < dx2 ? corner(h, true, b, c) : corner(h, false, b, a);
        }
        d = D::cm(a, c) ? a : c;
        return corner(h, false, b, d);
    }
    /** heap::calc (heap.cc:177-263) at point (i,j). */
    __device__ double calc(int i, int j) const {
        const int P = g.P, ij = j * P + i, m = g.mL, n = g.nL;
        const int L = -1, R = 1, Dn = -P, U = P;
        double a, b, c, d;
        const double ti = 2.0 / 3.0;
        auto look_l = [&](double &e) { return look(ij, L, i > 1, e); };
        auto look_r = [&](double &e) { return look(ij, R, i < m - 2, e); };
        auto look_d = [&](double &e) { return look(ij, Dn, j > 1, e); };
        auto look_u = [&](double &e) { return look(ij, U, j < n - 2, e); };
        if (j > 0 && in(ij - P)) {
            if (j < n - 1 && in(ij + P)) {
                if (i < m - 1 && in(ij + 1)) {
                    if (i > 0 && in(ij - 1)) {
                        if (look_d(a)) {
                            if (look_u(c)) {
                                d = D::cm(a, c) ? a : c;
                                bool hl = look_l(a), hr = look_r(c);
                                return threeway1(hl, hr, true, a, c, d);
                            } else {
                                if (look_l(b)) {
                                    if (look_r(d)) { b = D::cm(b, d) ? b : d; return threeway2(true, true, false, b, a, c); }
                                    return fourway(d, c, b, a);
                                } else {
                                    if (look_r(d)) return fourway(b, c, d, a);
                                    b = D::cm(b, d) ? b : d;
                                    return threeway2(false, true, false, b, a, c);
                                }
                            }
                        } else {
                            if (look_u(c)) {
                                if (look_l(b)) {
                                    if (look_r(d)) { b = D::cm(b, d) ? b : d; return threeway2(true, true, false, b, c, a); }
                                    return fourway(d, a, b, c);
                                } else {
                                    if (look_r(d)) return fourway(b, a, d, c);
                                    b = D::cm(b, d) ? b : d;
                                    return threeway2(false, true, false, b, c, a);
                                }
                            } else {
                                d = D::cm(a, c) ? a : c;
                                bool hl = look_l(a), hr = look_r(c);
                                return threeway1(hl, hr, false, a, c, d);
                            }
                        }
                    } else {
                        bool h = look_r(b), v1 = look_u(a), v2 = look_d(c);
                        return threeway2(h, v1, v2, b, a, c);
                    }
                } else {
                    if (i > 0 && in(ij - 1)) {
                        bool h = look_l(b), v1 = look_u(a), v2 = look_d(c);
                        return threeway2(h, v1, v2, b, a, c);
                    }
                    c = look_d(a) ? D::ct(a, dy) * ti : D::ct(a, dy);
                    d = look_u(b) ? D::ct(b, dy) * ti : D::ct(b, dy);
                    return D::cm(c, d) ? c : d;
                }
            } else {
                if (i < m - 1 && in(ij + 1)) {
                    if (i > 0 && in(ij - 1)) {
                        bool hl = look_l(a), hr = look_r(c), v = look_d(b);
                        return threeway1(hl, hr, v, a, c, b);
                    }
                    bool h = look_r(a), v = look_d(b);
                    return corner(h, v, a, b);
                } else {
                    if (i > 0 && in(ij - 1)) { bool h = look_l(a), v = look_d(b); return corner(h, v, a, b); }
                    return look_d(a) ? D::ct(a, dy) * ti : D::ct(a, dy);
                }
            }
        } else {
            if (j < n - 1 && in(ij + P)) {
                if (i < m - 1 && in(ij + 1)) {
                    if (i > 0 && in(ij - 1)) {
                        bool hl = look_l(a), hr = look_r(c), v = look_u(b);
                        return threeway1(hl, hr, v, a, c, b);
                    }
                    bool h = look_r(a), v = look_u(b);
                    return corner(h, v, a, b);
                } else {
                    if (i > 0 && in(ij - 1)) { bool h = look_l(a), v = look_u(b); return corner(h, v, a, b); }
                    return look_u(a) ? D::ct(a, dy) * ti : D::ct(a, dy);
                }
            } else {
                if (i < m - 1 && in(ij + 1)) {
                    if (i > 0 && in(ij - 1)) {
                        c = look_l(a) ? D::ct(a, dx) * ti : D::ct(a, dx);
                        d = look_r(b) ? D::ct(b, dx) * ti : D::ct(b, dx);
                        return D::cm(c, d) ? c : d;
                    }
                    return look_r(a) ? D::ct(a, dx) * ti : D::ct(a, dx);
                } else {
                    if (i > 0 && in(ij - 1)) return look_l(a) ? D::ct(a, dx) * ti : D::ct(a, dx);
                    return 0;
                }
            }
        }
    }
};

/** Whether a point has at least one 4-neighbour that counts as "in". */
template <bool POS>
__device__ __forceinline__ bool any_in(const March<POS> &mr, int i, int j) {
    const int P = mr.g.P, ij = j * P + i;
    return (i > 0 && mr.in(ij - 1)) || (i < mr.g.mL - 1 && mr.in(ij + 1)) ||
           (j > 0 && mr.in(ij - P)) || (j < mr.g.nL - 1 && mr.in(ij + P));
}

constexpr double kUnset = 1e300;

/** Initialises both march buffers (+/-kUnset for this side's far points)
 * and clears both change marks. */
__global__ void k_ls_fim_init(LsGrid g, const LsObj *ob, const LsWin *win) {
    int i, j;
    if (!ls_point(g, win, i, j)) return;
    const LsObj &o = ob[blockIdx.z];
    const int ij = j * g.P + i, st = o.s[ij];
    const double v = st == 7 ? kUnset : (st == 0 ? -kUnset : 0.0);
    o.a[ij] = v;
    o.b[ij] = v;
    o.ca[ij] = 0;
    o.cb[ij] = 0;
}

/** Final values and clean-up (heap::march acceptance, levelset::clean,
 * levelset.cc:408-413): far points whose value fell inside the band limit are
 * accepted (5 / 2); every point outside the band is set to the band limit. */
__global__ void k_ls_finish(LsGrid g, const LsObj *ob, const LsWin *win) {
    int i, j;
    if (!ls_point(g, win, i, j)) return;
    // After the last (unchanging) sweep both buffers hold the final values.
    const double *cur = ob[blockIdx.z].a;
    int *s = ob[blockIdx.z].s;
    double *phi = ob[blockIdx.z].phi;
    const int ij = j * g.P + i, st = s[ij];
    const double v = cur[ij];
    if (st == 7) {
        if (v < g.phi_up) { s[ij] = 5; phi[ij] = v; }
        else phi[ij] = g.phi_up;
    } else if (st == 0) {
        if (v > g.phi_down) { s[ij] = 2; phi[ij] = v; }
        else phi[ij] = g.phi_down;
    }
}

/** Trial statuses (heap::check_gridpoint / update, heap.cc:38-44,159-167):
 * a far point next to an interface or accepted point of its side was put on
 * the heap and, not being accepted, stays trial (6 / 1). */
__global__ void k_ls_trial(LsGrid g, const LsObj *ob, const LsWin *win) {
    int i, j;
    if (!ls_point(g, win, i, j)) return;
    const int *s = ob[blockIdx.z].s;
    int *s_out = ob[blockIdx.z].ia;
    const int ij = j * g.P + i, st = s[ij];
    int out = st;
    if (st == 7 || st == 0) {
        const int lo = st == 7 ? 4 : 2, hi = st == 7 ? 5 : 3;
        bool nb = false;
        if (i > 0) nb |= s[ij - 1] >= lo && s[ij - 1] <= hi;
        if (i < g.mL - 1) nb |= s[ij + 1] >= lo && s[ij + 1] <= hi;
        if (j > 0) nb |= s[ij - g.P] >= lo && s[ij - g.P] <= hi;
        if (j < g.nL - 1) nb |= s[ij + g.P] >= lo && s[ij + g.P] <= hi;
        if (nb) out = st == 7 ? 6 : 1;
    }
    s_out[ij] = out;
}

/** Copies the trial statuses back into the status array. */
__global__ void k_ls_store_status(LsGrid g, const LsObj *ob, const LsWin *win) {
    int i, j;
    if (!ls_point(g, win, i, j)) return;
    const int ij = j * g.P + i;
    ob[blockIdx.z].s[ij] = ob[blockIdx.z].ia[ij];
}

/** Weighted least-squares extrapolation of (nX,nY) at one band point outside
 * the solid (traverse::extrapolate, traverse.hh:169-231): linear fit over the
 * band neighbours with smaller phi inside a (2r+1)^2 window, weighted by the
 * phi difference; the window grows from r=3 to r=7 while the system is
 * singular. Values of points inside the solid come from nX/nY, of points
 * outside from the current iterate (cx,cy). Returns false when singular. */
__device__ bool ls_extrap_point(const LsGrid &g, const int *s, const double *phi, const double *nX, const double *nY,
                                const double *cx, const double *cy, int i, int j, double &ox, double &oy) {
    const int P = g.P, ij = j * P + i;
    const double pp = phi[ij];
    double sw, sx, sy, sxx, sxy, syy, det, acc[6];
    if (i >= 3 && j >= 3 && i + 3 < g.mL && j + 3 < g.nL) {
        // The radius-3 window lies inside the grid: unrolled, so the status
        // and phi loads of all 49 points issue together. Same sums, same order.
        sw = sx = sy = sxx = sxy = syy = 0;
#pragma unroll
        for (int k = 0; k < 6; k++) acc[k] = 0;
#pragma unroll
        for (int dj = -3; dj <= 3; dj++) {
            int sq[7];
            double w[7];
#pragma unroll
            for (int di = -3; di <= 3; di++) {
                const int q = ij + dj * P + di;
                sq[di + 3] = s[q];
                w[di + 3] = phi[q];
            }
#pragma unroll
            for (int di = -3; di <= 3; di++) {
                const int q = ij + dj * P + di, st = sq[di + 3];
                if (st < 2 || st > 5 || !(w[di + 3] < pp)) continue;
                const double ww = pp - w[di + 3];
                sw += ww;
                sx += di * ww;
                sy += dj * ww;
                sxx += di * di * ww;
                sxy += di * dj * ww;
                syy += dj * dj * ww;
                const double vx = st <= 3 ? nX[q] : cx[q], vy = st <= 3 ? nY[q] : cy[q];
                acc[0] += ww * vx; acc[1] += ww * di * vx; acc[2] += ww * dj * vx;
                acc[3] += ww * vy; acc[4] += ww * di * vy; acc[5] += ww * dj * vy;
            }
        }
        det = sw * (sxy * sxy - sxx * syy) + sx * sx * syy - 2 * sx * sxy * sy + sy * sy * sxx;
        if (!(fabs(det) < 1e-10)) {
            det = 1 / det;
            const double al = (sxy * sxy - sxx * syy) * det, be = (sx * syy - sxy * sy) * det,
                         ga = (sxx * sy - sxy * sx) * det;
            ox = acc[0] * al + acc[1] * be + acc[2] * ga;
            oy = acc[3] * al + acc[4] * be + acc[5] * ga;
            return true;
        }
    }
    int r = 3;
    do {
        const int ilo = i <= r ? -i : -r, ihi = i + r >= g.mL ? g.mL - 1 - i : r;
        const int jlo = j <= r ? -j : -r, jhi = j + r >= g.nL ? g.nL - 1 - j : r;
        sw = sx = sy = sxx = sxy = syy = 0;
        for (int k = 0; k < 6; k++) acc[k] = 0;
        for (int dj = jlo; dj <= jhi; dj++)
            for (int di = ilo; di <= ihi; di++) {
                const int q = ij + dj * P + di, sq = s[q];
                if (sq < 2 || sq > 5) continue;
                double w = phi[q];
                if (!(w < pp)) continue;
                w = pp - w;
                sw += w;
                sx += di * w;
                sy += dj * w;
                sxx += di * di * w;
                sxy += di * dj * w;
                syy += dj * dj * w;
                const double vx = sq <= 3 ? nX[q] : cx[q], vy = sq <= 3 ? nY[q] : cy[q];
                acc[0] += w * vx; acc[1] += w * di * vx; acc[2] += w * dj * vx;
                acc[3] += w * vy; acc[4] += w * di * vy; acc[5] += w * dj * vy;
            }
        det = sw * (sxy * sxy - sxx * syy) + sx * sx * syy - 2 * sx * sxy * sy + sy * sy * sxx;
        r++;
    } while (fabs(det) < 1e-10 && r <= 7);
    if (fabs(det) < 1e-10) return false;
    det = 1 / det;
    const double al = (sxy * sxy - sxx * syy) * det, be = (sx * syy - sxy * sy) * det, ga = (sxx * sy - sxy * sx) * det;
    ox = acc[0] * al + acc[1] * be + acc[2] * ga;
    oy = acc[3] * al + acc[4] * be + acc[5] * ga;
    return true;
}

/** Appends (ij, object) to the combined point list if it has room;
 * flags an overflow otherwise (the list is sized for every point of every
 * object, so this only guards the bound). */
__device__ __forceinline__ void ls_list_push(int *list, int *list_k, int *count, int cap, int *overflow, int ij,
                                             int k) {
    const int t = atomicAdd(count, 1);
    if (t < cap) { list[t] = ij; list_k[t] = k; }
    else atomicExch(overflow, 1);
}

/** Lists the band points outside each solid (status 4 or 5). */
__global__ void k_ls_collect_outside(LsGrid g, const LsObj *ob, const LsWin *win, int *list, int *list_k, int *count, int cap,
                                     int *overflow) {
    int i, j;
    if (!ls_point(g, win, i, j)) return;
    const int ij = j * g.P + i, st = ob[blockIdx.z].s[ij];
    if (st == 4 || st == 5) ls_list_push(list, list_k, count, cap, overflow, ij, blockIdx.z);
}

/** Starts the extrapolation: both buffers of every listed point hold its
 * current reference map. Only listed points are ever read as iterates. */
__global__ void k_ls_extrap_init(const LsObj *ob, const int *list, const int *list_k, const int *countp, int cap) {
    const int count = min(*countp, cap);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        const LsObj &o = ob[list_k[t]];
        const int ij = list[t];
        o.a[ij] = o.b[ij] = o.nX[ij];
        o.c[ij] = o.d[ij] = o.nY[ij];
    }
}

/** Stores the extrapolated values of the listed points into nX, nY. */
__global__ void k_ls_extrap_store(const LsObj *ob, const int *list, const int *list_k, const int *countp, int cap) {
    const int count = min(*countp, cap);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        const LsObj &o = ob[list_k[t]];
        const int ij = list[t];
        o.nX[ij] = o.a[ij];
        o.nY[ij] = o.c[ij];
    }
}

}  // namespace incrmt

namespace incrmt {

/** Marks the points next to the interface (status 3 or 4) as 1 in mark. */
__global__ void k_ls_mark_interface(LsGrid g, const LsObj *ob, const LsWin *win) {
    int i, j;
    if (!ls_point(g, win, i, j)) return;
    const int ij = j * g.P + i, st = ob[blockIdx.z].s[ij];
    ob[blockIdx.z].ia[ij] = (st == 3 || st == 4) ? 1 : 0;
}

/** One direction of a separable dilation by radius R (max over a window):
 * along x from ia into ib, along y from ib back into ia. */
template <bool ALONG_X>
__global__ void k_ls_dilate(LsGrid g, const LsObj *ob, const LsWin *win, int R) {
    int i, j;
    if (!ls_point(g, win, i, j)) return;
    const int *in = ALONG_X ? ob[blockIdx.z].ia : ob[blockIdx.z].ib;
    int *out = ALONG_X ? ob[blockIdx.z].ib : ob[blockIdx.z].ia;
    // Every marked point lies inside the window, and only the window's
    // marks are current: the reach is clipped to it.
    const LsWin w = win[blockIdx.z];
    int v = 0;
    if (ALONG_X) {
        const int lo = i - R < w.x0 ? w.x0 : i - R, hi = i + R >= w.x1 ? w.x1 - 1 : i + R;
        for (int a = lo; a <= hi && !v; a++) v = in[j * g.P + a];
    } else {
        const int lo = j - R < w.y0 ? w.y0 : j - R, hi = j + R >= w.y1 ? w.y1 - 1 : j + R;
        for (int b = lo; b <= hi && !v; b++) v = in[b * g.P + i];
    }
    out[j * g.P + i] = v;
}

/** Lists the far points (status 0 or 7) inside the dilated interface region:
 * the only points the march can reach within the band limit. */
__global__ void k_ls_collect_candidates(LsGrid g, const LsObj *ob, const LsWin *win, int *list, int *list_k, int *count, int cap,
                                        int *overflow) {
    int i, j;
    if (!ls_point(g, win, i, j)) return;
    const LsObj &o = ob[blockIdx.z];
    const int ij = j * g.P + i, st = o.s[ij];
    if ((st == 0 || st == 7) && o.ia[ij]) ls_list_push(list, list_k, count, cap, overflow, ij, blockIdx.z);
}

/** Threads per block of the cooperative sweeps: one block per SM (the grid
 * barrier costs more with more blocks), as many threads as the registers
 * allow, so that a candidate list of ~1e5 points takes about one pass per
 * sweep and each SM has many warps to hide the stencil's dependent loads. */
constexpr int kFimThreads = 1024;
constexpr int kExtrapThreads = 512;

/** Whether any point the stencil of (i,j) reads (up to two cells along
 * each axis) changed in the previous sweep. */
__device__ __forceinline__ bool stencil_changed(const LsGrid &g, const unsigned char *chg, int i, int j) {
    const int P = g.P, ij = j * P + i;
    if (chg[ij]) return true;
    for (int d = 1; d <= 2; d++) {
        if (i - d >= 0 && chg[ij - d]) return true;
        if (i + d < g.mL && chg[ij + d]) return true;
        if (j - d >= 0 && chg[ij - d * P]) return true;
        if (j + d < g.nL && chg[ij + d * P]) return true;
    }
    return false;
}

/** All sweeps of the march fixed point in one cooperative launch: every
 * sweep evaluates the stencil at the listed candidates (Jacobi, reading cur,
 * writing nxt), a grid barrier follows, and the loop ends after the first
 * sweep that changed nothing. A candidate whose stencil inputs did not change
 * in the previous sweep keeps its value (its stencil would return it again),
 * so later sweeps only touch the moving front; each object's ca/cb are
 * per-point change marks of the previous and the current sweep (cleared by
 * k_ls_fim_init) and a/b its values, swapped every sweep. The list holds the
 * candidates of every object, so all bands settle in the same launch.
 * flags[0..2] rotate as per-sweep change flags; flags[3] receives the number
 * of sweeps and flags[4] 1 if converged. */
__global__ void __launch_bounds__(kFimThreads, 1) k_ls_fim_coop(LsGrid g, const LsObj *ob, const int *list, const int *list_k, const int *countp,
                              int cap, int *flags, int max_sweeps) {
    namespace cg = cooperative_groups;
    cg::grid_group grid = cg::this_grid();
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    const int count = min(*countp, cap);
    int it = 0;
    bool done = false;
    for (; it < max_sweeps; it++) {
        if (tid == 0) flags[(it + 1) % 3] = 0;
        const bool odd = it & 1;
        // Where the second-order stencil is not monotone, the plain sweeps can
        // cycle between two states instead of settling (seen on thin solids at
        // fine grids). After half the sweep budget each value may then only
        // move towards the interface, which settles; flags[12] records it.
        const bool monotone = it >= max_sweeps / 2;
        if (monotone && tid == 0) flags[12] = 1;
        bool ch = false;
        for (int t = tid; t < count; t += nth) {
            const LsObj &o = ob[list_k[t]];
            const double *cur = odd ? o.b : o.a;
            double *nxt = odd ? o.a : o.b;
            const unsigned char *cprev = odd ? o.cb : o.ca;
            unsigned char *cnow = odd ? o.ca : o.cb;
            const int ij = list[t], i = ij % g.P, j = ij / g.P, st = o.s[ij];
            const double old = cur[ij];
            double v = old;
            if (it == 0 || stencil_changed(g, cprev, i, j)) {
                if (st == 7) {
                    March<true> mr(g, o.phi, o.s, cur, old);
                    if (any_in(mr, i, j)) v = mr.calc(i, j);
                    if (monotone && v > old) v = old;
                } else {
                    March<false> mr(g, o.phi, o.s, cur, old);
                    if (any_in(mr, i, j)) v = mr.calc(i, j);
                    if (monotone && v < old) v = old;
                }
            }
            nxt[ij] = v;
            // Changes in the last bits (the tail of the fixed point) do not
            // count: the sweeps end once every value is settled to 1e-13.
            const bool c = fabs(v - old) > 1e-13 * fabs(v);
            cnow[ij] = c;
            if (c) ch = true;
        }
        if (__syncthreads_or(ch) && threadIdx.x == 0) flags[it % 3] = 1;
        grid.sync();
        const int c = *reinterpret_cast<volatile int *>(&flags[it % 3]);
        if (!c) { done = true; break; }
    }
    if (tid == 0) { flags[3] = done ? it + 1 : it; flags[4] = done ? 1 : 0; }
}

/** All sweeps of the extrapolation wavefront in one cooperative launch (same
 * scheme as k_ls_fim_coop); flags[5] is raised for a singular fit. */
__global__ void __launch_bounds__(kExtrapThreads, 1) k_ls_extrap_coop(LsGrid g, const LsObj *ob, const int *list, const int *list_k,
                                 const int *countp, int cap, int *flags, int max_sweeps) {
    namespace cg = cooperative_groups;
    cg::grid_group grid = cg::this_grid();
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    const int count = min(*countp, cap);
    int it = 0;
    bool done = false;
    for (; it < max_sweeps; it++) {
        if (tid == 0) flags[(it + 1) % 3] = 0;
        const bool odd = it & 1;
        bool ch = false;
        for (int t = tid; t < count; t += nth) {
            const LsObj &o = ob[list_k[t]];
            const double *cx = odd ? o.b : o.a, *cy = odd ? o.d : o.c;
            double *tx = odd ? o.a : o.b, *ty = odd ? o.c : o.d;
            const int ij = list[t], i = ij % g.P, j = ij / g.P;
            double ox, oy;
            if (!ls_extrap_point(g, o.s, o.phi, o.nX, o.nY, cx, cy, i, j, ox, oy)) {
                atomicExch(&flags[5], INCRMT_ERR_EXTRAP_SINGULAR);
                ox = cx[ij]; oy = cy[ij];
            }
            if (ox != cx[ij] || oy != cy[ij]) ch = true;
            tx[ij] = ox;
            ty[ij] = oy;
        }
        if (__syncthreads_or(ch) && threadIdx.x == 0) flags[it % 3] = 1;
        grid.sync();
        const int c = *reinterpret_cast<volatile int *>(&flags[it % 3]);
        if (!c) { done = true; break; }
    }
    if (tid == 0) { flags[3] = done ? it + 1 : it; flags[4] = done ? 1 : 0; }
}

}  // namespace incrmt
