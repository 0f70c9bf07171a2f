// Time-step kernels of fluid_2d::step_forward (fluid_2d.cc:298-369) for
// grids with walls in x (optionally the zero-pressure right edge and the
// horizontal inflow of sim_horiz_flow) and walls or periodicity in y. One
// thread per cell or edge; every kernel reads the fields it needs straight
// from HBM (SoA, coalesced along x) and writes each output once.
#pragma once
#include "sim.cuh"

namespace incrmt {

__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }

/** delta_lim (fluid_2d.cc:629-634). */
__device__ __forceinline__ double delta_lim(double f0, double f1, double f2) {
    double drm = f1 - f0, drp = f2 - f1;
    return drm > 0 ? (drp > 0 ? 2 * dmin(drm, drp) : 0) : (drp > 0 ? 0 : -2 * dmax(drm, drp));
}
/** delta_f (fluid_2d.cc:617-621). */
__device__ __forceinline__ double delta_f(double f0, double f1, double f2) {
    double drc = 0.5 * (f2 - f0);
    return drc > 0 ? dmin(drc, delta_lim(f0, f1, f2)) : dmax(drc, -delta_lim(f0, f1, f2));
}
/** Fourth-order monotonicity-limited slope (fluid_2d.cc:604-609). */
__device__ __forceinline__ double mono_diff(double f0, double f1, double f2, double f3, double f4) {
    double tdrc = f3 - f1;
    double s = (1 / 6.) * (4 * tdrc - delta_f(f0, f1, f2) - delta_f(f2, f3, f4));
    double t = delta_lim(f1, f2, f3);
    return tdrc > 0 ? dmin(s, t) : dmax(s, -t);
}

/** normal_derivatives_velocity + normal_derivatives_refmap
 * (fluid_2d.cc:877-950): limited slopes and edge extrapolations of u,v and
 * of every object's X,Y. */
__global__ void k_normal_derivatives(GridDev g, FluidDev f, const SolidDev *sol, TileObjs to, double dt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.m || j >= g.n) return;
    const int q = g.idx(i, j), P = g.P;
    const double u = f.u[q], v = f.v[q];
    const double ux = g.xsp * mono_diff(f.u[q - 2], f.u[q - 1], u, f.u[q + 1], f.u[q + 2]);
    const double vx = g.xsp * mono_diff(f.v[q - 2], f.v[q - 1], v, f.v[q + 1], f.v[q + 2]);
    const double uy = g.ysp * mono_diff(f.u[q - 2 * P], f.u[q - P], u, f.u[q + P], f.u[q + 2 * P]);
    const double vy = g.ysp * mono_diff(f.v[q - 2 * P], f.v[q - P], v, f.v[q + P], f.v[q + 2 * P]);
    f.ux[q] = ux; f.vx[q] = vx; f.uy[q] = uy; f.vy[q] = vy;
    f.ul[q] = u - 0.5 * (g.dx + dt * u) * ux;
    f.vl[q] = v - 0.5 * (g.dx + dt * u) * vx;
    f.ur[q] = u + 0.5 * (g.dx - dt * u) * ux;
    f.vr[q] = v + 0.5 * (g.dx - dt * u) * vx;
    f.ud[q] = u - 0.5 * (g.dy + dt * v) * uy;
    f.vd[q] = v - 0.5 * (g.dy + dt * v) * vy;
    f.uu[q] = u + 0.5 * (g.dy - dt * v) * uy;
    f.vu[q] = v + 0.5 * (g.dy - dt * v) * vy;
    int kb, ke;
    to.range(i, j, kb, ke);
    for (int p = kb; p < ke; p++) {
        const SolidDev s = sol[to.at(p)];
        const double X = s.X[q], Y = s.Y[q];
        const double Xx = g.xsp * mono_diff(s.X[q - 2], s.X[q - 1], X, s.X[q + 1], s.X[q + 2]);
        const double Yx = g.xsp * mono_diff(s.Y[q - 2], s.Y[q - 1], Y, s.Y[q + 1], s.Y[q + 2]);
        const double Xy = g.ysp * mono_diff(s.X[q - 2 * P], s.X[q - P], X, s.X[q + P], s.X[q + 2 * P]);
        const double Yy = g.ysp * mono_diff(s.Y[q - 2 * P], s.Y[q - P], Y, s.Y[q + P], s.Y[q + 2 * P]);
        s.Xx[q] = Xx; s.Yx[q] = Yx; s.Xy[q] = Xy; s.Yy[q] = Yy;
        s.Xl[q] = X - 0.5 * (g.dx + dt * u) * Xx;
        s.Yl[q] = Y - 0.5 * (g.dx + dt * u) * Yx;
        s.Xr[q] = X + 0.5 * (g.dx - dt * u) * Xx;
        s.Yr[q] = Y + 0.5 * (g.dx - dt * u) * Yx;
        s.Xd[q] = X - 0.5 * (g.dy + dt * v) * Xy;
        s.Yd[q] = Y - 0.5 * (g.dy + dt * v) * Yy;
        s.Xu[q] = X + 0.5 * (g.dy - dt * v) * Xy;
        s.Yu[q] = Y + 0.5 * (g.dy - dt * v) * Yy;
    }
}

/** godunov_upwinding_set<tang> (fluid_2d.cc:1112-1121, godunov_set_lr/du
 * :642-686) fused with edge_boundary_conditions for walls
 * (fluid_2d.cc:743-756, 770-777). Each thread owns the right and top edge of
 * its cell; the boundary edges it writes are disjoint from the Godunov
 * writes, so the two passes fuse without a race. */
template <bool tang>
__global__ void k_godunov(GridDev g, FluidDev f, const SolidDev *sol, TileObjs to) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.m || j >= g.n) return;
    const int q = g.idx(i, j), P = g.P;
    int kb, ke;
    to.range(i, j, kb, ke);
    if (i < g.m - 1 || g.xp) {
        // With x periodicity the right edge of the last column is the left
        // edge of column 0; the reference selects it with
        // godunov_set_lr<true> on the ghost column -1, which holds column
        // m-1's fluid edge values but the (never written) ghost solid values
        // (fluid_2d.cc:733-741); qs is that column for the solids.
        const bool wrap = i == g.m - 1;
        const bool tg = tang || wrap;
        const int r = wrap ? q - (g.m - 1) : q + 1, qs = wrap ? r - 1 : q;
        const double fur = f.ur[q], frul = f.ul[r];
        if (fur + frul > 0 && fur > 0) {
            f.ul[r] = fur;
            f.vl[r] = f.vr[q];
            for (int p = kb; p < ke; p++) {
                const SolidDev &s = sol[to.at(p)];
                s.Xl[r] = s.Xr[qs];
                s.Yl[r] = s.Yr[qs];
            }
        } else if (fur + frul < 0 && frul < 0) {
            if (tg) f.ur[q] = frul;
        } else {
            if (tg) f.ur[q] = 0.5 * (fur + frul);
            f.ul[r] = 0;
            f.vl[r] = 0.5 * (f.vr[q] + f.vl[r]);
            for (int p = kb; p < ke; p++) {
                const SolidDev &s = sol[to.at(p)];
                s.Xl[r] = 0.5 * (s.Xr[qs] + s.Xl[r]);
                s.Yl[r] = 0.5 * (s.Yr[qs] + s.Yl[r]);
            }
        }
    }
    if (j < g.n - 1 || g.yp) {
        // With y periodicity the top edge of the last row is the bottom edge
        // of row 0. The reference selects it in edge_boundary_conditions with
        // godunov_set_du<true> on the ghost row -1, which holds row n-1's
        // fluid edge values but the (never written) ghost solid values
        // (fluid_2d.cc:760-768); qs is that row for the solids.
        const bool wrap = j == g.n - 1;
        const bool tg = tang || wrap;
        const int t = wrap ? q - (g.n - 1) * P : q + P, qs = wrap ? t - P : q;
        const double fvu = f.vu[q], ftvd = f.vd[t];
        if (fvu + ftvd > 0 && fvu > 0) {
            f.vd[t] = fvu;
            f.ud[t] = f.uu[q];
            for (int p = kb; p < ke; p++) {
                const SolidDev &s = sol[to.at(p)];
                s.Xd[t] = s.Xu[qs];
                s.Yd[t] = s.Yu[qs];
            }
        } else if (fvu + ftvd < 0 && ftvd < 0) {
            if (tg) f.vu[q] = ftvd;
        } else {
            if (tg) f.vu[q] = 0.5 * (fvu + ftvd);
            f.vd[t] = 0;
            f.ud[t] = 0.5 * (f.uu[q] + f.ud[t]);
            for (int p = kb; p < ke; p++) {
                const SolidDev &s = sol[to.at(p)];
                s.Xd[t] = 0.5 * (s.Xu[qs] + s.Xd[t]);
                s.Yd[t] = 0.5 * (s.Yu[qs] + s.Yd[t]);
            }
        }
    }
    // Wall edge conditions.
    if (!g.xp) {
        if (i == 0) {
            if (g.zpr) f.ur[q - 1] = f.ul[q];
            else { f.ul[q] = 0; f.vl[q] = 0; f.ur[q - 1] = 0; }
        }
        if (i == g.m - 1) {
            if (g.zpr) { f.ul[q + 1] = f.ur[q]; f.vl[q + 1] = f.vr[q]; }
            else { f.ul[q + 1] = 0; f.vl[q + 1] = 0; f.ur[q] = 0; }
        }
    }
    if (!g.yp) {
        if (j == 0) { f.ud[q] = 0; f.vd[q] = 0; f.vu[q - P] = 0; }
        if (j == g.n - 1) { f.ud[q + P] = 0; f.vd[q + P] = 0; f.vu[q] = 0; }
    }
}

/** Ghost rows of the edge values under y periodicity, after k_godunov
 * (fluid_2d::edge_boundary_conditions, fluid_2d.cc:760-768): row -1 takes
 * row n-1's top values, row n row 0's bottom values. */
__global__ void k_wrap_edges_y(GridDev g, FluidDev f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.m) return;
    const int q0 = g.idx(i, 0), qt = g.idx(i, g.n - 1);
    f.vu[q0 - g.P] = f.vu[qt];
    f.uu[q0 - g.P] = f.uu[qt];
    f.vd[qt + g.P] = f.vd[q0];
    f.ud[qt + g.P] = f.ud[q0];
}

/** Ghost columns of the edge values under x periodicity, after k_godunov
 * (fluid_2d::edge_boundary_conditions, fluid_2d.cc:733-741): column -1 takes
 * column m-1's right values, column m column 0's left values. */
__global__ void k_wrap_edges_x(GridDev g, FluidDev f) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= g.n) return;
    const int q0 = g.idx(0, j), qt = g.idx(g.m - 1, j);
    f.ur[q0 - 1] = f.ur[qt];
    f.vr[q0 - 1] = f.vr[qt];
    f.ul[qt + 1] = f.ul[q0];
    f.vl[qt + 1] = f.vl[q0];
}

/** fluid_2d::set_boundaries_solid (fluid_2d.cc:818-835): under periodic
 * reference-map boundary conditions the ghost columns and rows of every
 * object's X, Y copy the opposite side shifted by the box length (columns
 * first, then rows including the corners). One block. */
__global__ void k_set_boundaries_solid(GridDev g, const SolidDev *sol, int nobj) {
    const double lx = g.bx - g.ax, ly = g.by - g.ay;
    const int P = g.P, G = g.n * P;
    for (int k = 0; k < nobj; k++) {
        double *X = sol[k].X, *Y = sol[k].Y;
        for (int j = threadIdx.x; j < g.n; j += blockDim.x) {
            const int q = g.idx(0, j), r = q + g.m;
            X[q - 2] = X[r - 2] - lx; Y[q - 2] = Y[r - 2];
            X[q - 1] = X[r - 1] - lx; Y[q - 1] = Y[r - 1];
            X[r] = X[q] + lx; Y[r] = Y[q];
            X[r + 1] = X[q + 1] + lx; Y[r + 1] = Y[q + 1];
        }
        __syncthreads();
        for (int i = threadIdx.x - 2; i < g.m + 2; i += blockDim.x) {
            const int q = g.idx(i, 0);
            X[q - 2 * P] = X[q + G - 2 * P]; Y[q - 2 * P] = Y[q + G - 2 * P] - ly;
            X[q - P] = X[q + G - P]; Y[q - P] = Y[q + G - P] - ly;
            X[q + G] = X[q]; Y[q + G] = Y[q] + ly;
            X[q + G + P] = X[q + P]; Y[q + G + P] = Y[q + P] + ly;
        }
        __syncthreads();
    }
}

/** fluid_2d::edge_boundary_conditions_solid_pre / _post (fluid_2d.cc:784-815):
 * before the Godunov selection (post = 0) the ghost column -1's right and the
 * ghost row -1's top reference-map edge values copy column m-1's and row
 * n-1's, shifted; after it (post = 1) the ghost column m's left and row n's
 * bottom values copy column 0's and row 0's, shifted. One block. */
__global__ void k_solid_edges_prd(GridDev g, const SolidDev *sol, int nobj, int post) {
    const double lx = g.bx - g.ax, ly = g.by - g.ay;
    for (int k = 0; k < nobj; k++) {
        const SolidDev &s = sol[k];
        for (int j = threadIdx.x; j < g.n; j += blockDim.x) {
            const int q0 = g.idx(0, j), qt = g.idx(g.m - 1, j);
            if (!post) { s.Xr[q0 - 1] = s.Xr[qt] - lx; s.Yr[q0 - 1] = s.Yr[qt]; }
            else { s.Xl[qt + 1] = s.Xl[q0] + lx; s.Yl[qt + 1] = s.Yl[q0]; }
        }
        for (int i = threadIdx.x; i < g.m; i += blockDim.x) {
            const int q0 = g.idx(i, 0), qt = g.idx(i, g.n - 1);
            if (!post) { s.Xu[q0 - g.P] = s.Xu[qt]; s.Yu[q0 - g.P] = s.Yu[qt] - ly; }
            else { s.Xd[qt + g.P] = s.Xd[q0]; s.Yd[qt + g.P] = s.Yd[q0] + ly; }
        }
        __syncthreads();
    }
}

/** compute_tangential_stability_derivatives (fluid_2d.cc:953-975), without
 * the dead r0..r3 writes. */
__global__ void k_tangential(GridDev g, FluidDev f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.m || j >= g.n) return;
    const int q = g.idx(i, j), P = g.P;
    const double u_adv = 0.5 * g.xsp * (f.ul[q + 1] + f.ul[q]), v_adv = 0.5 * g.ysp * (f.vd[q + P] + f.vd[q]);
    f.c0[q] = u_adv * (f.ur[q] - f.ur[q - 1]);
    f.c1[q] = u_adv * (f.vl[q + 1] - f.vl[q]);
    f.c2[q] = v_adv * (f.ud[q + P] - f.ud[q]);
    f.c3[q] = v_adv * (f.vu[q] - f.vu[q - P]);
}

/** Wall repulsion (fluid_2d::wall_force, fluid_2d.cc:1056-1078). */
__device__ __forceinline__ void wall_force(const GridDev &g, double x, double y, double phiv, double &fx, double &fy) {
    const double w = g.w_scale * g.eps, winv = 1 / w, k_rep = g.w_force * winv;
    if (x <= g.ax + w) {
        double t = (x - g.ax) * winv;
        fx += k_rep * ((1. - t) / t) * (phiv > -g.dx ? (phiv > g.dx ? 0 : 0.5 * (1 - phiv * g.xsp)) : 1);
    } else if (x >= g.bx - w) {
        double t = (g.bx - x) * winv;
        fx -= k_rep * ((1. - t) / t) * (phiv > -g.dx ? (phiv > g.dx ? 0 : 0.5 * (1 - phiv * g.xsp)) : 1);
    }
    if (y <= g.ay + w) {
        double t = (y - g.ay) * winv;
        fy += k_rep * ((1. - t) / t) * (phiv > -g.dy ? (phiv > g.dy ? 0 : 0.5 * (1 - phiv * g.ysp)) : 1);
    } else if (y >= g.by - w) {
        double t = (g.by - y) * winv;
        fy -= k_rep * ((1. - t) / t) * (phiv > -g.dy ? (phiv > g.dy ? 0 : 0.5 * (1 - phiv * g.ysp)) : 1);
    }
}

/** fluid_2d::acceleration (fluid_2d.cc:1019-1050). */
__device__ __forceinline__ void acceleration(const GridDev &g, const FluidDev &f, const ObjDev *obj,
                                             const SolidDev *sol, const TileObjs &to, int i, int j, int q,
                                             double x, double y, bool pressure, double &accx, double &accy) {
    const int P = g.P;
    double ax_ = 0, ay_ = 0;
    accx = g.xsp * (f.s11[q + 1] - f.s11[q]) + g.ysp * (f.s12[q + P] - f.s12[q]);
    accy = g.xsp * (f.s21[q + 1] - f.s21[q]) + g.ysp * (f.s22[q + P] - f.s22[q]);
    if (pressure) {
        accx -= 0.5 * g.xsp * (f.p[q + P + 1] + f.p[q + 1] - f.p[q + P] - f.p[q]);
        accy -= 0.5 * g.ysp * (f.p[q + P + 1] - f.p[q + 1] + f.p[q + P] - f.p[q]);
    }
    int kb, ke;
    to.range(i, j, kb, ke);
    for (int p = kb; p < ke; p++) {
        const int k = to.at(p);
        const double phiv = sol[k].phi[q];
        if (phiv < obj[k].eps && !g.solid_prd) {
            wall_force(g, x, y, phiv, accx, accy);
            obj_accel(obj[k], x, y, sol[k].X[q], sol[k].Y[q], phiv, ax_, ay_);
        }
    }
    const double rho = f.rho[q];
    accx /= rho;
    accy /= rho;
    accx += ax_;
    accy += ay_;
}

/** compute_half_time_edge_velocities (fluid_2d.cc:979-1008) fused with
 * compute_half_time_edge_reference_map (fluid_2d.cc:1082-1108). */
__global__ void k_half_time(GridDev g, FluidDev f, const ObjDev *obj, const SolidDev *sol, TileObjs to, double dt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.m || j >= g.n) return;
    const int q = g.idx(i, j);
    const double x = g.ax + g.dx * (0.5 + i), y = g.ay + g.dy * (0.5 + j);
    double accx, accy;
    acceleration(g, f, obj, sol, to, i, j, q, x, y, true, accx, accy);
    const double u = f.u[q], v = f.v[q], ux = f.ux[q], vx = f.vx[q], uy = f.uy[q], vy = f.vy[q];
    const double c0 = f.c0[q], c1 = f.c1[q], c2 = f.c2[q], c3 = f.c3[q];
    f.ul[q] = u + 0.5 * (-g.dx * ux + dt * (-u * ux - c2 + accx));
    f.vl[q] = v + 0.5 * (-g.dx * vx + dt * (-u * vx - c3 + accy));
    f.ur[q] = u + 0.5 * (g.dx * ux + dt * (-u * ux - c2 + accx));
    f.vr[q] = v + 0.5 * (g.dx * vx + dt * (-u * vx - c3 + accy));
    f.ud[q] = u + 0.5 * (-g.dy * uy + dt * (-v * uy - c0 + accx));
    f.vd[q] = v + 0.5 * (-g.dy * vy + dt * (-v * vy - c1 + accy));
    f.uu[q] = u + 0.5 * (g.dy * uy + dt * (-v * uy - c0 + accx));
    f.vu[q] = v + 0.5 * (g.dy * vy + dt * (-v * vy - c1 + accy));
    int kb, ke;
    to.range(i, j, kb, ke);
    for (int p = kb; p < ke; p++) {
        const SolidDev s = sol[to.at(p)];
        const double X = s.X[q], Y = s.Y[q], Xx = s.Xx[q], Xy = s.Xy[q], Yx = s.Yx[q], Yy = s.Yy[q];
        const double Xdt = dt * (-u * Xx - v * Xy), Ydt = dt * (-u * Yx - v * Yy);
        s.Xl[q] = X + 0.5 * (-g.dx * Xx + Xdt);
        s.Yl[q] = Y + 0.5 * (-g.dx * Yx + Ydt);
        s.Xr[q] = X + 0.5 * (g.dx * Xx + Xdt);
        s.Yr[q] = Y + 0.5 * (g.dx * Yx + Ydt);
        s.Xd[q] = X + 0.5 * (-g.dy * Xy + Xdt);
        s.Yd[q] = Y + 0.5 * (-g.dy * Yy + Ydt);
        s.Xu[q] = X + 0.5 * (g.dy * Xy + Xdt);
        s.Yu[q] = Y + 0.5 * (g.dy * Yy + Ydt);
    }
}

/** MAC source: discrete divergence of the edge velocities
 * (fluid_2d.cc:1179-1187), row-major m x n. */
__global__ void k_mac_source(GridDev g, FluidDev f, double *src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.m || j >= g.n) return;
    const int q = g.idx(i, j);
    src[j * g.m + i] = g.xsp * (f.ul[q + 1] - f.ul[q]) + g.ysp * (f.vd[q + g.P] - f.vd[q]);
}

/** Variable-density MAC correction of the edge velocities
 * (fluid_2d.cc:1214-1234); ex/ey are the edge 1/rho arrays of the MAC
 * system (left edge of (i,j) at ex[j*(m+1)+i], bottom edge at ey[j*m+i]). */
__global__ void k_mac_correct(GridDev g, FluidDev f, const double *z, const double *ex, const double *ey) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.m || j >= g.n) return;
    const int q = g.idx(i, j), ij = j * g.m + i;
    if (j > 0) f.vd[q] -= ey[j * g.m + i] * (z[ij] - z[ij - g.m]) * g.ysp;
    else if (g.yp) {
        f.vd[q] -= ey[i] * (z[ij] - z[ij + (g.n - 1) * g.m]) * g.ysp;
        f.vd[q + g.n * g.P] = f.vd[q];
    }
    if (i > 0) f.ul[q] -= ex[j * (g.m + 1) + i] * (z[ij] - z[ij - 1]) * g.xsp;
    else if (g.xp) {
        f.ul[q] -= ex[j * (g.m + 1)] * (z[ij] - z[ij + g.m - 1]) * g.xsp;
        f.ul[q + g.m] = f.ul[q];
    }
}

/** Cell (i,j) of thread (x,y) of a launch over object blockIdx.z's window
 * (level-set coordinates, so cell = point - 2); false outside the window or
 * outside the cells lo <= i < m+hi, lo <= j < n+hi. */
__device__ __forceinline__ bool win_cell(const GridDev &g, const LsWin *win, int lo, int hi, int &i, int &j) {
    const LsWin w = win[blockIdx.z];
    const int li = w.x0 + blockIdx.x * blockDim.x + threadIdx.x, lj = w.y0 + blockIdx.y * blockDim.y + threadIdx.y;
    i = li - 2;
    j = lj - 2;
    return li < w.x1 && lj < w.y1 && i >= lo && j >= lo && i < g.m + hi && j < g.n + hi;
}

/** First part of update_reference_map (fluid_2d.cc:1246-1258): the end-of-
 * step reference map nX,nY at points with status < 4, for object blockIdx.z
 * within its window (status < 4 holds only inside it). */
__global__ void k_refmap_update(GridDev g, FluidDev f, const SolidDev *sol, const LsWin *win, double dt) {
    int i, j;
    if (!win_cell(g, win, 0, 0, i, j)) return;
    const SolidDev &s = sol[blockIdx.z];
    const int q = g.idx(i, j), P = g.P;
    if (s.s[q] >= 4) return;
    const double hx = 0.5 * dt * g.xsp, hy = 0.5 * dt * g.ysp;
    const double a = f.ul[q + 1] + f.ul[q], b = f.vd[q + P] + f.vd[q];
    s.nX[q] = s.X[q] + (-hx * a * (s.Xl[q + 1] - s.Xl[q]) - hy * b * (s.Xd[q + P] - s.Xd[q]));
    s.nY[q] = s.Y[q] + (-hx * a * (s.Yl[q + 1] - s.Yl[q]) - hy * b * (s.Yd[q + P] - s.Yd[q]));
}

/** Last part of update_reference_map (fluid_2d.cc:1266-1272):
 * X = (X+nX)/2 where status < 6 (s_field::set_half_timestep), object
 * blockIdx.z within its window. */
__global__ void k_refmap_half(GridDev g, const SolidDev *sol, const LsWin *win) {
    int i, j;
    if (!win_cell(g, win, 0, 0, i, j)) return;
    const SolidDev &s = sol[blockIdx.z];
    const int q = g.idx(i, j);
    if (s.s[q] < 6) {
        s.X[q] = 0.5 * (s.X[q] + s.nX[q]);
        s.Y[q] = 0.5 * (s.Y[q] + s.nY[q]);
    }
}

/** Density from the level sets (fluid_2d::set_rho, fluid_2d.cc:1124-1137),
 * over the whole ghosted grid. */
__global__ void k_set_rho(GridDev g, FluidDev f, const ObjDev *obj, const SolidDev *sol, TileObjs to) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x - 2, j = blockIdx.y * blockDim.y + threadIdx.y - 2;
    if (i >= g.m + 2 || j >= g.n + 2) return;
    const int q = g.idx(i, j);
    double rho = 0, sfrac = 0;
    int kb, ke;
    to.range(i, j, kb, ke);
    for (int p = kb; p < ke; p++) {
        const int k = to.at(p);
        double tf = trans_func(obj[k], sol[k].phi[q]);
        sfrac += tf;
        rho += tf * obj[k].rhos;
    }
    f.rho[q] = sfrac >= 1 ? rho / sfrac : (1 - sfrac) * g.rhof + rho;
}

/** Ghost velocities (fluid_2d::set_boundaries, fluid_2d.cc:689-725): one
 * block; first the left/right ghosts of every row (periodic, walls, or linear
 * extrapolation at a zero-pressure right edge), then the bottom/top ghost
 * rows including the corners (walls or periodic), then the inflow of
 * sim_horiz_flow::boundary (sim_type.cc:51-56) on the two left ghost columns. */
__global__ void k_set_boundaries(GridDev g, FluidDev f) {
    const int P = g.P;
    double *u = f.u, *v = f.v;
    for (int j = threadIdx.x; j < g.n; j += blockDim.x) {
        const int q = g.idx(0, j);
        const int r = q + g.m;
        if (g.xp) {
            u[q - 2] = u[r - 2]; v[q - 2] = v[r - 2];
            u[q - 1] = u[r - 1]; v[q - 1] = v[r - 1];
            u[r] = u[q]; v[r] = v[q];
            u[r + 1] = u[q + 1]; v[r + 1] = v[q + 1];
            continue;
        }
        u[q - 2] = -u[q + 1]; v[q - 2] = -v[q + 1];
        u[q - 1] = -u[q]; v[q - 1] = -v[q];
        if (g.zpr) {
            u[r] = 2 * u[r - 1] - u[r - 2]; v[r] = 2 * v[r - 1] - v[r - 2];
            u[r + 1] = 2 * u[r] - u[r - 1]; v[r + 1] = 2 * v[r] - v[r - 1];
        } else {
            u[r] = -u[r - 1]; v[r] = -v[r - 1];
            u[r + 1] = -u[r - 2]; v[r + 1] = -v[r - 2];
        }
    }
    __syncthreads();
    const int G = g.n * P;
    for (int i = threadIdx.x - 2; i < g.m + 2; i += blockDim.x) {
        const int q = g.idx(i, 0);
        if (g.yp) {
            u[q - 2 * P] = u[q + G - 2 * P]; v[q - 2 * P] = v[q + G - 2 * P];
            u[q - P] = u[q + G - P]; v[q - P] = v[q + G - P];
            u[q + G] = u[q]; v[q + G] = v[q];
            u[q + G + P] = u[q + P]; v[q + G + P] = v[q + P];
        } else {
            u[q - 2 * P] = -u[q + P]; v[q - 2 * P] = -v[q + P];
            u[q - P] = -u[q]; v[q - P] = -v[q];
            u[q + G] = -u[q + G - P]; v[q + G] = -v[q + G - P];
            u[q + G + P] = -u[q + G - 2 * P]; v[q + G + P] = -v[q + G - 2 * P];
        }
    }
    if (!g.hflow) return;
    __syncthreads();
    for (int j = threadIdx.x - 2; j < g.n + 2; j += blockDim.x) {
        const int q = g.idx(0, j);
        u[q - 1] = u[q - 2] = g.flow_u;
        v[q - 1] = v[q - 2] = 0;
    }
}

/** Solid stress of one object at a left (left=true) or bottom edge
 * (fluid_2d::solid_stress, fluid_2d.cc:510-560). Returns false when the edge
 * is outside the object's blur zone. */
template <bool left>
__device__ __forceinline__ bool solid_stress(const GridDev &g, const FluidDev &f, const ObjDev &o,
                                             const SolidDev &s, int q, double &s1s, double &s2s,
                                             double &sfrac) {
    const int P = g.P, o1 = left ? 1 : P;
    const double phiv = 0.5 * (s.phi[q] + s.phi[q - o1]);
    if (phiv > o.eps) return false;
    double Xx, Yx, Xy, Yy;
    if (left) {
        Xx = g.xsp * (s.X[q] - s.X[q - 1]);
        Yx = g.xsp * (s.Y[q] - s.Y[q - 1]);
        Xy = 0.25 * g.ysp * (s.X[q + P] + s.X[q + P - 1] - s.X[q - P] - s.X[q - P - 1]);
        Yy = 0.25 * g.ysp * (s.Y[q + P] + s.Y[q + P - 1] - s.Y[q - P] - s.Y[q - P - 1]);
    } else {
        Xx = 0.25 * g.xsp * (s.X[q + 1] + s.X[q - P + 1] - s.X[q - 1] - s.X[q - P - 1]);
        Yx = 0.25 * g.xsp * (s.Y[q + 1] + s.Y[q - P + 1] - s.Y[q - 1] - s.Y[q - P - 1]);
        Xy = g.ysp * (s.X[q] - s.X[q - P]);
        Yy = g.ysp * (s.Y[q] - s.Y[q - P]);
    }
    // F=[[Yy,-Xy],[-Yx,Xx]], the object's actuation applied at the edge's
    // reference map, sigma=F F^T (mat::AAT, mat.hh:159-161).
    double Fa = Yy, Fb = -Xy, Fc = -Yx, Fd = Xx;
    if (o.type == OBJ_FLAPPER || o.type == OBJ_LAMPREY) {
        const double X = left ? 0.5 * (s.X[q] + s.X[q - 1]) : 0.5 * (s.X[q] + s.X[q - P]),
                     Y = left ? 0.5 * (s.Y[q] + s.Y[q - 1]) : 0.5 * (s.Y[q] + s.Y[q - P]);
        obj_actuate(o, X, Y, Fa, Fb, Fc, Fd);
    }
    const double sa = Fa * Fa + Fb * Fb, sb = Fa * Fc + Fb * Fd, sd = Fc * Fc + Fd * Fd;
    const double sfac = (1 / 3.0) * ((sa + sd) + 1);
    const double tf = trans_func_in(o, phiv), G = o.G * tf,
                 ex_visc = o.ex_visc * tf * (1 + o.ev_trans_mult * tderiv_func_in(o, phiv));
    sfrac += tf;
    if (left) {
        s1s += G * (sa - sfac);
        s2s += G * sb;
        s1s += ex_visc * g.xsp * (f.u[q] - f.u[q - 1]);
        s2s += ex_visc * g.xsp * (f.v[q] - f.v[q - 1]);
    } else {
        s1s += G * sb;
        s2s += G * (sd - sfac);
        s1s += ex_visc * g.ysp * (f.u[q] - f.u[q - P]);
        s2s += ex_visc * g.ysp * (f.v[q] - f.v[q - P]);
    }
    return true;
}

/** Level set of one object and its gradient at an edge (collision_stress,
 * fluid_2d.cc:457-468). */
template <bool left>
__device__ __forceinline__ void edge_phi(const GridDev &g, const double *phi, int q, double &p, double &px, double &py) {
    const int P = g.P;
    if (left) {
        p = 0.5 * (phi[q] + phi[q - 1]);
        px = g.xsp * (phi[q] - phi[q - 1]);
        py = 0.25 * g.ysp * (phi[q + P] + phi[q + P - 1] - phi[q - P] - phi[q - P - 1]);
    } else {
        p = 0.5 * (phi[q] + phi[q - P]);
        px = 0.25 * g.xsp * (phi[q + 1] + phi[q - P + 1] - phi[q - 1] - phi[q - P - 1]);
        py = g.ysp * (phi[q] - phi[q - P]);
    }
}

/** Stress at one edge: solids, fluid remainder, collisions
 * (compute_stress body, fluid_2d.cc:395-441). */
template <bool left>
__device__ __forceinline__ void edge_stress(const GridDev &g, const FluidDev &f, const ObjDev *obj,
                                            const SolidDev *sol, const TileObjs &to, int i, int j, int q,
                                            double &o1, double &o2) {
    const int P = g.P;
    double s1s = 0, s2s = 0, sfrac = 0;
    unsigned long long present = 0;
    int k = 0;
    int kb, ke;
    to.range(i, j, kb, ke);
    for (int pa = kb; pa < ke; pa++) {
        const int a = to.at(pa);
        if (solid_stress<left>(g, f, obj[a], sol[a], q, s1s, s2s, sfrac)) { present |= 1ull << (pa - kb); k++; }
    }
    if (sfrac >= 1) {
        o1 = s1s / sfrac;
        o2 = s2s / sfrac;
    } else {
        double s1f, s2f;
        if (left) {
            const double ux = g.xsp * (f.u[q] - f.u[q - 1]), vx = g.xsp * (f.v[q] - f.v[q - 1]),
                         uy = 0.25 * g.ysp * (f.u[q + P] + f.u[q + P - 1] - f.u[q - P] - f.u[q - P - 1]);
            s1f = 2 * g.visc * ux;
            s2f = g.visc * (vx + uy);
        } else {
            const double vx = 0.25 * g.xsp * (f.v[q + 1] + f.v[q - P + 1] - f.v[q - 1] - f.v[q - P - 1]),
                         uy = g.ysp * (f.u[q] - f.u[q - P]), vy = g.ysp * (f.v[q] - f.v[q - P]);
            s1f = g.visc * (vx + uy);
            s2f = 2 * g.visc * vy;
        }
        o1 = (1 - sfrac) * s1f + s1s;
        o2 = (1 - sfrac) * s2f + s2s;
    }
    if (k > 1) {
        const double small_number = 100. * 2.220446049250313e-16;
        for (int pa = kb; pa < ke; pa++) {
            if (!(present >> (pa - kb) & 1)) continue;
            const int a = to.at(pa);
            double p1, p1x, p1y;
            edge_phi<left>(g, sol[a].phi, q, p1, p1x, p1y);
            for (int pb = pa + 1; pb < ke; pb++) {
                if (!(present >> (pb - kb) & 1)) continue;
                const int b = to.at(pb);
                double p2, p2x, p2y;
                edge_phi<left>(g, sol[b].phi, q, p2, p2x, p2y);
                const double norx = (p2x - p1x), nory = (p2y - p1y), nn = norx * norx + nory * nory;
                double fac = 4. * dmin(coll_func(obj[a], p1), coll_func(obj[b], p2)) * (obj[a].G + obj[b].G);
                fac = nn < small_number ? 0. : fac / nn;
                if (left) {
                    o1 -= fac * 0.5 * (norx * norx - nory * nory);
                    o2 -= fac * norx * nory;
                } else {
                    o1 -= fac * norx * nory;
                    o2 -= fac * 0.5 * (nory * nory - norx * norx);
                }
            }
        }
    }
}

/** fluid_2d::compute_stress (fluid_2d.cc:381-445) over the (m+1) x (n+1)
 * left and bottom edges. */
__global__ void k_stress(GridDev g, FluidDev f, const ObjDev *obj, const SolidDev *sol, TileObjs to) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i > g.m || j > g.n) return;
    const int q = g.idx(i, j);
    double a, b;
    edge_stress<true>(g, f, obj, sol, to, i, j, q, a, b);
    f.s11[q] = a;
    f.s21[q] = b;
    edge_stress<false>(g, f, obj, sol, to, i, j, q, a, b);
    f.s12[q] = a;
    f.s22[q] = b;
}

/** Intermediate velocity u* (fluid_2d::compute_ustar, fluid_2d.cc:1278-1291)
 * into c0,c1. */
__global__ void k_ustar(GridDev g, FluidDev f, const ObjDev *obj, const SolidDev *sol, TileObjs to, double dt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.m || j >= g.n) return;
    const int q = g.idx(i, j), P = g.P;
    const double x = g.ax + 0.5 * g.dx + i * g.dx, y = g.ay + g.dy * (.5 + j);
    double accx, accy;
    acceleration(g, f, obj, sol, to, i, j, q, x, y, false, accx, accy);
    const double hx = 0.5 * dt * g.xsp, hy = 0.5 * dt * g.ysp;
    const double a = f.ul[q + 1] + f.ul[q], b = f.vd[q + P] + f.vd[q];
    f.c0[q] = f.u[q] - hx * a * (f.ul[q + 1] - f.ul[q]) - hy * b * (f.ud[q + P] - f.ud[q]) + dt * accx;
    f.c1[q] = f.v[q] - hx * a * (f.vl[q + 1] - f.vl[q]) - hy * b * (f.vd[q + P] - f.vd[q]) + dt * accy;
}

/** u* at cell (i,j) for the FEM source, with the ghost values that
 * fem_source_term_conditions sets for walls, the zero-pressure edge and y
 * periodicity (fluid_2d.cc:837-871). */
__device__ __forceinline__ void ustar_bc(const GridDev &g, const FluidDev &f, int i, int j, double &c0, double &c1) {
    if (i < 0 && g.xp) i = g.m - 1;  // ghost column -1 copies column m-1 (fluid_2d.cc:841-845)
    if (j < 0 && g.yp) j = g.n - 1;  // ghost row -1 copies row n-1 (fluid_2d.cc:861-865)
    if (j < 0 || j >= g.n || i >= g.m) { c0 = 0; c1 = 0; return; }
    const int q = g.idx(i, j);
    if (i < 0) {
        if (g.zpr) { c0 = f.u[q]; c1 = f.v[q]; } else { c0 = 0; c1 = 0; }
        return;
    }
    c0 = f.c0[q];
    c1 = f.c1[q];
}

/** The ghost values of u* that fem_source_term_conditions stores
 * (fluid_2d.cc:837-871), written back into c0/c1 so that the state matches
 * the reference's: left ghost column u (zero-pressure edge) or 0, right ghost
 * column 0, then the bottom ghost row copying row n-1 (y periodic) or the
 * bottom and top ghost rows 0. One block; k_fem_source computes the same
 * values on the fly (ustar_bc). */
__global__ void k_fem_ghosts(GridDev g, FluidDev f) {
    for (int j = threadIdx.x; j < g.n; j += blockDim.x) {
        const int q = g.idx(0, j), r = g.idx(g.m, j);
        if (g.xp) {  // column -1 copies column m-1; column m is left as it is
            f.c0[q - 1] = f.c0[r - 1];
            f.c1[q - 1] = f.c1[r - 1];
            continue;
        }
        f.c0[q - 1] = g.zpr ? f.u[q - 1] : 0.;
        f.c1[q - 1] = g.zpr ? f.v[q - 1] : 0.;
        f.c0[r] = 0;
        f.c1[r] = 0;
    }
    __syncthreads();
    const int G = g.n * g.P;
    // the bottom/top rows from column -1 to m (x periodic: to m-1)
    for (int i = threadIdx.x - 1; i <= (g.xp ? g.m - 1 : g.m); i += blockDim.x) {
        const int q = g.idx(i, 0);
        if (g.yp) {
            f.c0[q - g.P] = f.c0[q + G - g.P];
            f.c1[q - g.P] = f.c1[q + G - g.P];
        } else {
            f.c0[q - g.P] = f.c0[q + G] = 0;
            f.c1[q - g.P] = f.c1[q + G] = 0;
        }
    }
}

/** FEM source at the (m+1) x (n+1) corners (finite_element_projection,
 * fluid_2d.cc:1298-1309). */
__global__ void k_fem_source(GridDev g, FluidDev f, double *src, double dt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.mf || j >= g.nf) return;
    const double hx = 0.5 * g.dy / dt, hy = 0.5 * g.dx / dt;
    double a0, a1, b0, b1, c0, c1, d0, d1;  // cells (i-1,j-1), (i-1,j), (i,j-1), (i,j)
    ustar_bc(g, f, i - 1, j - 1, a0, a1);
    ustar_bc(g, f, i - 1, j, b0, b1);
    ustar_bc(g, f, i, j - 1, c0, c1);
    ustar_bc(g, f, i, j, d0, d1);
    src[j * g.mf + i] = hx * (a0 + b0 - c0 - d0) + hy * (a1 - b1 + c1 - d1);
}

/** Partial sums of the trapezoid-weighted FEM pressure
 * (fluid_2d::average_pressure, fluid_2d.cc:1333-1348). */
__global__ void k_pressure_sum(GridDev g, const double *z, double *partial) {
    double acc = 0;
    const long N = static_cast<long>(g.mf) * g.nf;
    for (long t = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; t < N;
         t += static_cast<long>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(t % g.mf), j = static_cast<int>(t / g.mf);
        double w = !g.xp && (i == 0 || i == g.mf - 1) ? 0.5 : 1.0;
        if (!g.yp && (j == 0 || j == g.nf - 1)) w *= 0.5;
        acc += w * z[t];
    }
    acc = block_sum_256(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

/** Sums nb partials in a fixed order (one block of 256). */
__global__ void k_reduce_partials(const double *partial, int nb, double *out) {
    double acc = 0;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) acc += partial[q];
    acc = block_sum_256(acc);
    if (threadIdx.x == 0) *out = acc;
}

/** p = z - mean (copy_pressure, fluid_2d.cc:1317-1328); pavg[0] holds the
 * sum, scaled by 1/mn here, or is ignored when zpr. */
__global__ void k_copy_pressure(GridDev g, FluidDev f, const double *z, const double *psum) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i > g.m || j > g.n) return;
    const double pavg = g.zpr ? 0. : psum[0] * (1. / (static_cast<double>(g.m) * g.n));
    const int jz = g.yp && j == g.n ? 0 : j;  // the last row repeats row 0 (fluid_2d.cc:1323)
    const int iz = g.xp && i == g.m ? 0 : i;  // the last column repeats column 0 (fluid_2d.cc:1326)
    f.p[g.idx(i, j)] = z[jz * g.mf + iz] - pavg;
}

/** End-of-step velocity (update_velocity, fluid_2d.cc:1354-1374); the
 * reference-map part is k_refmap_commit. */
__global__ void k_update_velocity(GridDev g, FluidDev f, double dt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.m || j >= g.n) return;
    const int q = g.idx(i, j), P = g.P;
    const double rhoinv = 1. / f.rho[q];
    f.u[q] = f.c0[q] - 0.5 * dt * rhoinv * g.xsp * (f.p[q + P + 1] + f.p[q + 1] - f.p[q + P] - f.p[q]);
    f.v[q] = f.c1[q] - 0.5 * dt * rhoinv * g.ysp * (f.p[q + P + 1] - f.p[q + 1] + f.p[q + P] - f.p[q]);
}

/** The reference map part of update_velocity (fluid_2d.cc:1366-1373):
 * X = nX for object blockIdx.z, over the window where this step's
 * reference-map update changed X or nX (everywhere else they are equal). */
__global__ void k_refmap_commit(GridDev g, const SolidDev *sol, const LsWin *win) {
    int i, j;
    if (!win_cell(g, win, 0, 0, i, j)) return;
    const SolidDev &s = sol[blockIdx.z];
    const int q = g.idx(i, j);
    s.X[q] = s.nX[q];
    s.Y[q] = s.nY[q];
}

/** Pins the level set to the reference map within the pinning width
 * (obj_field::pin, obj_field.cc:92-97), object blockIdx.z over its window of
 * the ghosted grid (|phi| < pinw only inside it). */
__global__ void k_pin(GridDev g, const ObjDev *obj, const SolidDev *sol, const LsWin *win) {
    int i, j;
    if (!win_cell(g, win, -2, 2, i, j)) return;
    const ObjDev &o = obj[blockIdx.z];
    const SolidDev &s = sol[blockIdx.z];
    const int q = g.idx(i, j);
    const double p = s.phi[q];
    if (p < o.pinw && p > -o.pinw) s.phi[q] = obj_phi(o, s.X[q], s.Y[q]);
}

/** Initial reference map and level set of object blockIdx.z over the
 * ghosted grid (obj_field::init via fluid_2d::init_fields, fluid_2d.cc:198-205). */
__global__ void k_init_object(GridDev g, const ObjDev *obj, const SolidDev *sol) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x - 2, j = blockIdx.y * blockDim.y + threadIdx.y - 2;
    if (i >= g.m + 2 || j >= g.n + 2) return;
    const ObjDev &o = obj[blockIdx.z];
    const SolidDev &s = sol[blockIdx.z];
    const int q = g.idx(i, j);
    double X, Y;
    obj_transform(o, g.ax + g.dx * (0.5 + i), g.ay + g.dy * (0.5 + j), X, Y);
    s.X[q] = X;
    s.Y[q] = Y;
    s.phi[q] = obj_phi(o, X, Y);
}

/** sim_velocity_pulses::velocity (sim_type.cc:43-47, sim_type.hh:109-113):
 * six incompressible Gaussian pulses of alternating sign and growing inverse
 * square length along the diagonal. */
__device__ __forceinline__ void pulses_velocity(double x, double y, double &u, double &v) {
    u = v = 0;
    for (double k = 2, s = 1, z = -5 / 6.; z < 1; z += 1 / 3., k += 2, s = -s) {
        const double px = x - z, py = y - z;
        const double f = s * exp(-k * (2 - cos(px * M_PI) - cos(py * M_PI)));
        u -= sin(py * M_PI) * f;
        v += sin(px * M_PI) * f;
    }
}

/** Initial velocity from the solids' momenta and the scenario's fluid
 * velocity (fluid_2d::init_fields, fluid_2d.cc:213-239). */
__global__ void k_init_velocity(GridDev g, FluidDev f, const ObjDev *obj, const SolidDev *sol, int nobj) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.m || j >= g.n) return;
    const int q = g.idx(i, j);
    double mu = 0, mv = 0, rho = 0, sfrac = 0;
    for (int k = 0; k < nobj; k++) {
        if (!obj[k].set_velocity) continue;
        double tf = trans_func(obj[k], sol[k].phi[q]), uu, vv;
        obj_velocity(obj[k], sol[k].X[q], sol[k].Y[q], uu, vv);
        sfrac += tf;
        rho += tf * obj[k].rhos;
        mu += tf * obj[k].rhos * uu;
        mv += tf * obj[k].rhos * vv;
    }
    if (sfrac >= 1) {
        f.u[q] = mu / rho;
        f.v[q] = mv / rho;
    } else {
        // sim_type::velocity: at rest, (U, 0) for sim_horiz_flow
        // (sim_type.hh:132-135), or the pulses of sim_velocity_pulses
        double uf = g.hflow ? g.flow_u : 0., vf = 0.;
        if (g.pulses) pulses_velocity(g.ax + g.dx * (0.5 + i), g.ay + g.dy * (0.5 + j), uf, vf);
        double irho = 1 / ((1 - sfrac) * g.rhof + rho);
        f.u[q] = ((1 - sfrac) * g.rhof * uf + mu) * irho;
        f.v[q] = ((1 - sfrac) * g.rhof * vf + mv) * irho;
    }
}

}  // namespace incrmt
