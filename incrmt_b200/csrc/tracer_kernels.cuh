// Passive tracers and object-tracked points (fluid_2d::update_tracers,
// fluid_2d.cc:1445-1484; obj_track, object.cc:313-417) with the reference's
// bicubic interpolation of a two-component field (bicubic_interp,
// bi_interp.cc:18-194).
#pragma once
#include "sim.cuh"

namespace incrmt {

/** A two-component field on the ghosted grid: (u,v) or (X,Y). */
struct Field2 {
    const double *a, *b;
};

/** Cubic-in-x coefficients (1,x,x^2,x^3) of one grid row around column i
 * (bicubic_interp::compute_x, bi_interp.cc:90-146): cubic in the bulk,
 * quadratic in the first and last column. */
__device__ __forceinline__ void bic_row(const double *f, int i, int ij, int mL, double c[4]) {
    const double f0 = f[ij];
    c[0] = f0;
    if (i == 0) {
        const double f1 = f[ij + 1], f2 = f[ij + 2];
        c[1] = -1.5 * f0 + 2.0 * f1 - 0.5 * f2;
        c[2] = 0.5 * f0 - f1 + 0.5 * f2;
        c[3] = 0;
    } else if (i == mL - 2) {
        const double fm = f[ij - 1], f1 = f[ij + 1];
        c[1] = -0.5 * fm + 0.5 * f1;
        c[2] = 0.5 * fm - f0 + 0.5 * f1;
        c[3] = 0;
    } else {
        const double fm = f[ij - 1], f1 = f[ij + 1], f2 = f[ij + 2];
        c[1] = -0.5 * fm + 0.5 * f1;
        c[2] = fm - 2.5 * f0 + 2.0 * f1 - 0.5 * f2;
        c[3] = -0.5 * fm + 1.5 * f0 - 1.5 * f1 + 0.5 * f2;
    }
}

/** Bicubic interpolation of one component at fractional grid position
 * (bicubic_interp::grid_index/table_setup/f/f_grad_f, bi_interp.cc:26-162).
 * Returns the value and, if grad, the derivatives in grid units. */
__device__ double bic_eval(const double *f, int mL, int nL, int P, int i, int j, double x, double y,
                           bool grad, double &fx, double &fy) {
    const int ij = j * P + i;
    double c1[4], c2[4], c0[4], c3[4], a[16];
    bic_row(f, i, ij, mL, c1);
    bic_row(f, i, ij + P, mL, c2);
    for (int k = 0; k < 4; k++) {
        double *ap = a + 4 * k;
        if (j == 0) {
            if (k == 0) bic_row(f, i, ij + 2 * P, mL, c3);
            ap[0] = c1[k];
            ap[1] = -1.5 * c1[k] + 2.0 * c2[k] - 0.5 * c3[k];
            ap[2] = 0.5 * c1[k] - c2[k] + 0.5 * c3[k];
            ap[3] = 0;
        } else if (j == nL - 2) {
            if (k == 0) bic_row(f, i, ij - P, mL, c0);
            ap[0] = c1[k];
            ap[1] = -0.5 * c0[k] + 0.5 * c2[k];
            ap[2] = 0.5 * c0[k] - c1[k] + 0.5 * c2[k];
            ap[3] = 0;
        } else {
            if (k == 0) { bic_row(f, i, ij - P, mL, c0); bic_row(f, i, ij + 2 * P, mL, c3); }
            ap[0] = c1[k];
            ap[1] = -0.5 * c0[k] + 0.5 * c2[k];
            ap[2] = c0[k] - 2.5 * c1[k] + 2.0 * c2[k] - 0.5 * c3[k];
            ap[3] = -0.5 * c0[k] + 1.5 * c1[k] - 1.5 * c2[k] + 0.5 * c3[k];
        }
    }
    auto yl = [&](int o) { return a[o] + y * (a[o + 1] + y * (a[o + 2] + y * a[o + 3])); };
    auto dyl = [&](int o) { return a[o + 1] + y * (2.0 * a[o + 2] + 3.0 * y * a[o + 3]); };
    if (grad) {
        fx = yl(4) + x * (2.0 * yl(8) + 3 * x * yl(12));
        fy = dyl(0) + x * (dyl(4) + x * (dyl(8) + x * dyl(12)));
    }
    return yl(0) + x * (yl(4) + x * (yl(8) + x * yl(12)));
}

/** Cell and fractional position for interpolation on the ghosted grid
 * (bicubic_interp::grid_index); the grid spans ax-1.5dx .. bx+1.5dx. */
__device__ __forceinline__ void bic_index(const GridDev &g, double &x, double &y, int &i, int &j) {
    const double xsp = (g.ml - 1) / ((g.bx + 1.5 * g.dx) - (g.ax - 1.5 * g.dx));
    const double ysp = (g.nl - 1) / ((g.by + 1.5 * g.dy) - (g.ay - 1.5 * g.dy));
    x = (x - (g.ax - 1.5 * g.dx)) * xsp;
    y = (y - (g.ay - 1.5 * g.dy)) * ysp;
    i = static_cast<int>(x);
    j = static_cast<int>(y);
    if (i < 0) i = 0; else if (i > g.ml - 2) i = g.ml - 2;
    if (j < 0) j = 0; else if (j > g.nl - 2) j = g.nl - 2;
    x -= i;
    y -= j;
}

__device__ __forceinline__ void bic_vec(const GridDev &g, Field2 F, double x, double y, double &va, double &vb) {
    int i, j;
    bic_index(g, x, y, i, j);
    double d0, d1;
    va = bic_eval(F.a, g.ml, g.nl, g.P, i, j, x, y, false, d0, d1);
    vb = bic_eval(F.b, g.ml, g.nl, g.P, i, j, x, y, false, d0, d1);
}

/** Tracer stages (fluid_2d::tracer_update_1/2, fluid_2d.cc:1445-1459):
 * stage 1 stores the velocity at the position in slots 2,3; stage 2 completes
 * the improved Euler step. Records have `stride` doubles. For passive tracers
 * (remap=1) the indices of the tracers that left the box are appended to
 * list (*remapped counts them): the host applies sim_type::tracer_remap
 * (sim_type.cc:12-17) to them in index order, since its redraw of the other
 * coordinate uses the C library's rand() sequence. */
__global__ void k_tracers(GridDev g, Field2 vel, double *tm, int count, int stride, int stage, double dt,
                          int remap, int *remapped, int *list) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    double *tp = tm + static_cast<long>(t) * stride;
    if (stage == 1) {
        bic_vec(g, vel, tp[0], tp[1], tp[2], tp[3]);
        return;
    }
    const double tx = tp[0] + dt * tp[2], ty = tp[1] + dt * tp[3];
    double vx, vy;
    bic_vec(g, vel, tx, ty, vx, vy);
    tp[0] += 0.5 * dt * (tp[2] + vx);
    tp[1] += 0.5 * dt * (tp[3] + vy);
    if (remap && (tp[0] < g.ax || tp[0] > g.bx || tp[1] < g.ay || tp[1] > g.by)) {
        const int k = atomicAdd(remapped, 1);
        if (k < count) list[k] = t;
    }
}

/** Newton correction of a tracked point onto the solid's reference map
 * (obj_track::correct_tracer, object.cc:388-417): finds x with X(x)=X_ref
 * using the bicubic interpolant of (X,Y) and its Jacobian. Record layout
 * (obj_track tm): x, y, stage velocity (2), X_ref, Y_ref. On failure the
 * position keeps the partial update and *failed is set. */
__global__ void k_correct_tracers(GridDev g, Field2 refmap, double *tm, int count, int *failed) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    double *tp = tm + 6 * t;
    const double small_number = 100. * 2.220446049250313e-16, tolnewt = small_number * small_number * 100,
                 bigstep = 1;
    const double xsp = (g.ml - 1) / ((g.bx + 1.5 * g.dx) - (g.ax - 1.5 * g.dx));
    const double ysp = (g.nl - 1) / ((g.by + 1.5 * g.dy) - (g.ay - 1.5 * g.dy));
    double xx = tp[0], yy = tp[1];
    int cnt = 0, iter = 0;
    bool ok = true;
    while (cnt < 4) {
        if (iter > 100) { ok = false; break; }
        double x = xx, y = yy;
        int i, j;
        bic_index(g, x, y, i, j);
        double Xx, Xy, Yx, Yy;
        double X = bic_eval(refmap.a, g.ml, g.nl, g.P, i, j, x, y, true, Xx, Xy);
        double Y = bic_eval(refmap.b, g.ml, g.nl, g.P, i, j, x, y, true, Yx, Yy);
        Xx *= xsp; Xy *= ysp; Yx *= xsp; Yy *= ysp;
        const double fxv = X - tp[4], fyv = Y - tp[5];
        if (fxv * fxv + fyv * fyv < tolnewt) cnt++;
        const double det = Xx * Yy - Xy * Yx;
        if (det < small_number && det > -small_number) { ok = false; break; }
        const double delx = (Yy * fxv - Xy * fyv) / det, dely = (-Yx * fxv + Xx * fyv) / det;
        if (delx * delx + dely * dely > bigstep) { ok = false; break; }
        xx -= delx;
        yy -= dely;
        iter++;
    }
    tp[0] = xx;
    tp[1] = yy;
    if (!ok) atomicExch(failed, 1);
}

}  // namespace incrmt
