// Output frames assembled on the GPU: the float32 gnuplot binary matrices of
// fluid_2d::output (fluid_2d_io.cc:123-179), so that a frame crosses PCIe as
// 4-byte values of the requested box only, and the solid bounding box used
// for cropped solid output (obj_field::bound, obj_field.cc:102-106).
#pragma once
#include <cfloat>
#include <climits>
#include "sim.cuh"

namespace incrmt {

/** Whether an output mode is a cell-corner field (pressure, vorticity,
 * volume change, pressure difference): fluid_2d_io.cc:133,113. */
__host__ __device__ inline bool frame_corner_mode(int mode) {
    return ((1 << mode) & (8 | 16 | 512 | 2048)) != 0;
}

/** Sum of the four phi values around the lower-left corner of cell q
 * (fluid_2d::corner_phi, fluid_2d.hh:268-270), in the reference's order. */
__device__ __forceinline__ double frame_corner_phi(const double *phi, int q, int P) {
    return __dadd_rn(__dadd_rn(__dadd_rn(phi[q - P - 1], phi[q - P]), phi[q - 1]), phi[q]);
}

/** Value of output mode `mode` at ghosted point q. Products and sums use
 * explicit round-to-nearest operations so that no fused multiply-add changes
 * the double value before its conversion to float. */
__device__ double frame_value(const GridDev &g, const FluidDev &f, const SolidDev *sol, int nobj, int mode,
                              int q) {
    const int P = g.P;
    switch (mode) {
        case 0: return f.u[q];
        case 1: return f.v[q];
        case 2: return sqrt(__dadd_rn(__dmul_rn(f.u[q], f.u[q]), __dmul_rn(f.v[q], f.v[q])));  // fields.hh:27-29
        case 3: return f.p[q];
        case 4: {  // fluid_2d::vorticity (fluid_2d.hh:252-255)
            const double *u = f.u, *v = f.v;
            double a = __dadd_rn(__dadd_rn(__dadd_rn(v[q], -v[q - 1]), v[q - P]), -v[q - P - 1]);
            double b = __dadd_rn(__dadd_rn(__dadd_rn(u[q], u[q - 1]), -u[q - P]), -u[q - P - 1]);
            return __dmul_rn(0.5, __dadd_rn(__dmul_rn(g.xsp, a), -__dmul_rn(g.ysp, b)));
        }
        case 5: return f.rho[q];
        case 10: return f.c0[q];
        case 11: return f.c1[q];
        case 12: {  // fluid_2d::divergence (fluid_2d.hh:259-262)
            const double *u = f.u, *v = f.v;
            double a = __dadd_rn(__dadd_rn(__dadd_rn(u[q], -u[q - 1]), u[q - P]), -u[q - P - 1]);
            double b = __dadd_rn(__dadd_rn(__dadd_rn(v[q], v[q - 1]), -v[q - P]), -v[q - P - 1]);
            return __dmul_rn(0.5, __dadd_rn(__dmul_rn(g.xsp, a), __dmul_rn(g.ysp, b)));
        }
        case 6:
        case 7: {  // reference map of the object of least phi (fluid_2d::min_phi_obj, fluid_2d.cc:1504-1511)
            int ks = 0;
            double mphi = sol[0].phi[q];
            for (int k = 1; k < nobj; k++)
                if (sol[k].phi[q] < mphi) { mphi = sol[k].phi[q]; ks = k; }
            return mode == 6 ? sol[ks].X[q] : sol[ks].Y[q];
        }
        case 8: {  // fluid_2d::min_phi (fluid_2d.cc:1490-1495)
            double mphi = DBL_MAX;
            for (int k = 0; k < nobj; k++)
                if (sol[k].phi[q] < mphi) mphi = sol[k].phi[q];
            return mphi;
        }
        case 9: {  // fluid_2d::vol_change (fluid_2d_io.cc:303-317) with min_corner_phi_obj
            // (fluid_2d.cc:1519-1526), which compares a point value against a corner sum.
            int ks = 0;
            double mphi = frame_corner_phi(sol[0].phi, q, P);
            for (int k = 1; k < nobj; k++)
                if (sol[k].phi[q] < mphi) { mphi = frame_corner_phi(sol[k].phi, q, P); ks = k; }
            if (frame_corner_phi(sol[ks].phi, q, P) > 0) return 0;
            const double *X = sol[ks].X, *Y = sol[ks].Y;
            const double hx = __dmul_rn(0.5, g.xsp), hy = __dmul_rn(0.5, g.ysp);
            double Xx = __dmul_rn(hx, __dadd_rn(__dadd_rn(__dadd_rn(X[q], X[q - P]), -X[q - 1]), -X[q - P - 1]));
            double Xy = __dmul_rn(hy, __dadd_rn(__dadd_rn(__dadd_rn(X[q], X[q - 1]), -X[q - P]), -X[q - P - 1]));
            double Yx = __dmul_rn(hx, __dadd_rn(__dadd_rn(__dadd_rn(Y[q], Y[q - P]), -Y[q - 1]), -Y[q - P - 1]));
            double Yy = __dmul_rn(hy, __dadd_rn(__dadd_rn(__dadd_rn(Y[q], Y[q - 1]), -Y[q - P]), -Y[q - P - 1]));
            return __dadd_rn(__ddiv_rn(1.0, __dadd_rn(__dmul_rn(Xx, Yy), -__dmul_rn(Xy, Yx))), -1.0);
        }
    }
    return 0;
}

/** Fills the (sj+1) x (si+1) float matrix of one frame: row 0 holds si and
 * the x coordinates, row 1+j the y coordinate and the values of row lj+j of
 * the box. One thread per output float, rows coalesced. */
__global__ void k_frame(GridDev g, FluidDev f, const SolidDev *sol, int nobj, int mode, int li, int lj, int si,
                        int sj, double lx, double ly, float *out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y * blockDim.y + threadIdx.y;
    if (c > si || r > sj) return;
    float val;
    if (r == 0) val = c == 0 ? static_cast<float>(si) : static_cast<float>(__dadd_rn(lx, __dmul_rn(c - 1, g.dx)));
    else if (c == 0) val = static_cast<float>(__dadd_rn(ly, __dmul_rn(r - 1, g.dy)));
    else val = static_cast<float>(frame_value(g, f, sol, nobj, mode, (lj + r - 1) * g.P + li + c - 1));
    out[static_cast<long>(r) * (si + 1) + c] = val;
}

/** Extends box = {li, ui, lj, uj} to every ghosted point whose level-set
 * status is below 4 in any object (obj_field::bound). */
__global__ void k_solid_bound(GridDev g, const SolidDev *sol, int nobj, int *box) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    bool in = false;
    if (i < g.ml && j < g.nl)
        for (int k = 0; k < nobj; k++) in |= sol[k].s[j * g.P + i] < 4;
    // Warp-level reduction first, one atomic per warp and bound.
    const unsigned mask = __ballot_sync(0xffffffffu, in);
    if (!mask) return;
    int li = in ? i : INT_MAX, ui = in ? i + 1 : INT_MIN, lj = in ? j : INT_MAX, uj = in ? j + 1 : INT_MIN;
    for (int o = 16; o > 0; o >>= 1) {
        li = min(li, __shfl_xor_sync(0xffffffffu, li, o));
        ui = max(ui, __shfl_xor_sync(0xffffffffu, ui, o));
        lj = min(lj, __shfl_xor_sync(0xffffffffu, lj, o));
        uj = max(uj, __shfl_xor_sync(0xffffffffu, uj, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(box, li);
        atomicMax(box + 1, ui);
        atomicMin(box + 2, lj);
        atomicMax(box + 3, uj);
    }
}

}  // namespace incrmt

namespace incrmt {

/** Smallest level set over the objects at ghosted index q (fluid_2d::min_phi,
 * fluid_2d.cc:1490-1495): the largest double when there is none. */
__device__ __forceinline__ double min_phi_at(const SolidDev *sol, int nobj, int q) {
    double m = 1.7976931348623157e308;
    for (int k = 0; k < nobj; k++) {
        const double v = sol[k].phi[q];
        if (v < m) m = v;
    }
    return m;
}

/** Accumulators of l_comparison, in the reference's order: [0..2] velocity
 * counts (fluid, solid, blur), [3..5] pressure counts, [6..8] velocity sums
 * of squares, [9..11] pressure sums of squares, [12..14] velocity sums,
 * [15..17] pressure sums, [18..20] velocity maxima, [21..23] pressure
 * maxima. */
constexpr int kLcmp = 24;

/** fluid_2d::l_comparison (fluid_2d_io.cc:186-281) of the coarse grid g
 * against the fine grid gf (dm, dn its refinement factors): per block the 24
 * accumulators into part[block*24 + k]; the velocity and pressure
 * differences of each coarse cell are also stored in the coarse c0 and c1,
 * as the reference does. */
__global__ void k_l_comparison(GridDev g, FluidDev f, const SolidDev *sol, int nobj, FluidDev ff, int fP, int dm,
                               int dn, double *part) {
    const double ste[5] = {1, -1. / 16., 9. / 16, 9. / 16., -1 / 16.};
    const int mm = g.xp ? g.m : g.m + 1, nn = g.yp ? g.n : g.n + 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[kLcmp];
#pragma unroll
    for (int k = 0; k < kLcmp; k++) acc[k] = 0;
    if (t < mm * nn) {
        const int i = t % mm, j = t / mm;
        const double tf = g.yp || (j > 0 && j < g.n) ? 1 : 0.5;
        const double tf2 = g.xp || (i > 0 && i < g.m) ? tf : 0.5 * tf;
        const int q = g.idx(i, j);
        const int qf = (dn * j + 2) * fP + (dm * i + 2);  // fine cell (dm i, dn j)
        int li, ui, lj, uj;
        const double *stx, *sty;
        if (dm & 1) { ui = (li = dm / 2) + 1; stx = ste; }
        else { ui = (li = dm / 2 - 2) + 4; stx = ste + 1; }
        if (dn & 1) { uj = (lj = dn / 2) + 1; sty = ste; }
        else { uj = (lj = dn / 2 - 2) + 4; sty = ste + 1; }
        if (j < g.n && i < g.m) {
            double delu = 0, delv = 0;
            const double *sy = sty;
            for (int jj = lj; jj < uj; jj++, sy++) {
                const double *sx = stx;
                for (int ii = li; ii < ui; ii++, sx++) {
                    const int q3 = qf + jj * fP + ii;
                    delu += *sy * (*sx) * ff.u[q3];
                    delv += *sy * (*sx) * ff.v[q3];
                }
            }
            delu -= f.u[q];
            delv -= f.v[q];
            const double mphi = min_phi_at(sol, nobj, q);
            const int c = mphi > g.eps ? 0 : (mphi < -g.eps ? 1 : 2);
            const double delsq = delu * delu + delv * delv, del = sqrt(delsq);
            f.c0[q] = del;
            acc[c] += 1.;
            acc[6 + c] += delsq;
            acc[12 + c] += del;
            if (acc[18 + c] < del) acc[18 + c] = del;
        }
        // material at this cell corner, from the four-by-four neighbourhood;
        // at the last corner of a non-periodic direction it reaches one cell
        // past the ghosted grid (the reference reads beyond its array there),
        // which is clamped to the last ghost cell
        double mphi = 0;
        for (int jj = -1; jj < 3; jj++) {
            const int cj = min(j + jj, g.n + 1);
            for (int ii = -1; ii < 3; ii++) {
                const int ci = min(i + ii, g.m + 1);
                mphi += ste[jj + 2] * ste[ii + 2] * min_phi_at(sol, nobj, g.idx(ci, cj));
            }
        }
        const int c = mphi > g.eps ? 0 : (mphi < -g.eps ? 1 : 2);
        const double delp = ff.p[qf] - f.p[q];
        f.c1[q] = delp;
        acc[3 + c] += 1.;
        acc[9 + c] += delp * delp * tf2;
        acc[15 + c] += fabs(delp) * tf2;
        if (acc[21 + c] < delp) acc[21 + c] = delp;
    }
    // block reduction (256 threads): sums for [0..18), maxima for [18..24)
    __shared__ double red[kLcmp][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kLcmp; k++) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) {
            const double u = __shfl_down_sync(0xffffffffu, v, o);
            v = k < 18 ? v + u : fmax(v, u);
        }
        if (lane == 0) red[k][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < kLcmp) {
        const int k = threadIdx.x;
        double v = red[k][0];
        for (int q = 1; q < 8; q++) v = k < 18 ? v + red[k][q] : fmax(v, red[k][q]);
        part[blockIdx.x * kLcmp + k] = v;
    }
}

/** Combines the block accumulators in block order into the 32 norms of
 * l_comparison: err[4a+l] for quantity a and category l, err[4a+3] the total
 * (sums for a < 6, maxima for a = 6, 7), the L2 rows square-rooted; sums are
 * scaled by 1/(m n). One thread. */
__global__ void k_l_comparison_final(const double *part, int nb, double fac, double *err) {
    double o[kLcmp];
    for (int k = 0; k < kLcmp; k++) o[k] = 0;
    for (int b = 0; b < nb; b++)
        for (int k = 0; k < kLcmp; k++) o[k] = k < 18 ? o[k] + part[b * kLcmp + k] : fmax(o[k], part[b * kLcmp + k]);
    for (int a = 0; a < 6; a++) {
        for (int l = 0; l < 3; l++) err[4 * a + l] = o[3 * a + l] * fac;
        err[4 * a + 3] = err[4 * a] + err[4 * a + 1] + err[4 * a + 2];
    }
    for (int a = 6; a < 8; a++) {
        for (int l = 0; l < 3; l++) err[4 * a + l] = o[3 * a + l];
        double mx = err[4 * a] > err[4 * a + 1] ? err[4 * a] : err[4 * a + 1];
        err[4 * a + 3] = err[4 * a + 2] > mx ? err[4 * a + 2] : mx;
    }
    for (int k = 8; k < 16; k++) err[k] = sqrt(err[k]);
}

}  // namespace incrmt
