// Device state and per-point helpers of the time-step kernels.
//
// Layout in HBM: structure of arrays, FP64, one array per field of the
// reference's struct field / struct s_field (fields.hh:7-79), each covering
// the ghosted (m+4) x (n+4) grid with a row pitch P (>= m+4, a multiple of 32
// doubles = 256 B so rows start aligned). Cell (i,j), -2 <= i < m+2,
// -2 <= j < n+2, lives at (j+2)*P + (i+2). The level-set status of each
// object is an int array with the same layout. The reference's dead r0..r3
// temporaries (written at fluid_2d.cc:968-971, never read) are not stored.
#pragma once
#include <cuda_runtime.h>
#include <cmath>
#include "common.cuh"

namespace incrmt {

constexpr int kMaxObjects = 64;

/** Object geometry / forcing kinds (the object subclasses of object.hh). */
enum ObjType : int {
    OBJ_SIMPLE_SPIN = 0,  // obj_simple_spin (object.hh:422-467, object.cc:152-219)
    OBJ_CIRCLE = 1,       // obj_circle (object.hh:128-138, object.cc:22-34)
    OBJ_ROUNDED_ROD = 2,  // obj_rounded_rod (object.hh:218-241, object.cc:75-78, 275-278)
    OBJ_ELLIPSE = 3,      // rotated ellipse under gravity (no reference counterpart)
    OBJ_FLAG = 4,         // obj_flag (object.hh:471-505, object.cc:420-496)
    OBJ_SQUARE = 5,       // obj_square (object.hh:142-152, object.cc:41-44, 83-87)
    OBJ_SEVEN_POINT = 6,  // obj_seven_point (object.hh:176-213, object.cc:100-147)
    OBJ_FLAPPER = 7,      // obj_flapper (object.hh:245-285, object.cc:284-308)
    OBJ_PISTON = 8,       // obj_piston (object.hh:369-418, object.cc:224-269)
    OBJ_FULL = 9,         // obj_full: solid everywhere (object.hh:83-86)
    OBJ_TRIANGLE = 10,    // obj_triangle (object.hh:155-172, object.cc:52-70, 93-95)
    OBJ_LAMPREY = 11,     // obj_lamprey (object.hh:542-595, object.cc:554-581)
    OBJ_HOOP = 12,        // obj_hoop (object.hh:598-611, object.cc:586-588)
};

/** Device description of one solid: material constants (mat_const,
 * obj_field.hh:15-29), transition-function constants (obj_field.cc:14-20),
 * geometry parameters and the per-step state of pre_stress_setup. */
struct ObjDev {
    int type;
    int set_velocity;
    double G, rhos, ev_trans_mult;
    double eps, pinw, ex_visc;
    double tf1, tf2, tf3;
    // Geometry: simple spin {c0, c1, c2, piv_r, th_max, omega, piv_thresh,
    // K_stiff}; circle and square {cx, cy, cr, grav, uu, vv, omega}; rounded rod
    // {cx, cy, cr, grav, 0, 0, 0, cl}; ellipse {cx, cy, a, grav, 0, 0, 0, b,
    // cos theta, sin theta}; flag {cx, cy, flag_l, 0, 0, 0, 0, flag_w, flag_a,
    // perturb_v, flag_thresh, K_stiff}; seven-point star {cx, cy, cr, piv_r,
    // th_max, omega, piv_thresh, K_stiff}; flapper {cx, cy, cr, 0, cos theta,
    // sin theta, 0, cl, ar, al, amp, omega}; piston {0, y_start, lx, 0, idur,
    // anch_r, 0, ly, cx, len, anch_thresh, K_stiff}; triangle {cx, cy, cr/2,
    // grav, 0, 0, 0, 0, n0x, n0y, n1x, n1y} with n2 in nor2; lamprey {cx, cy,
    // dis, la, cos theta, sin theta, w1, w2, T, log(mlam)}; hoop {0, 0, cr,
    // 0, 0, 0, 0, cc}.
    double g[12];
    double nor2[2];
    // Per-step state set on the host before each stress evaluation: the
    // rotation of the spinner's and the star's anchors, the flapper's or the
    // lamprey's contraction or the piston anchor's height, and the shift of
    // the lamprey's contraction wave.
    double cth, sth, act, shift;
};

/** Smoothed Heaviside inside the solid or blur zone (obj_field.hh:110-112). */
__device__ __forceinline__ double trans_func_in(const ObjDev &o, double x) {
    return x < -o.eps ? 1 : 0.5 - x * o.tf1 - o.tf2 * sin(o.tf3 * x);
}
__device__ __forceinline__ double trans_func(const ObjDev &o, double x) {
    return x > o.eps ? 0 : trans_func_in(o, x);
}
/** eps times the transition derivative (obj_field.hh:118-120). */
__device__ __forceinline__ double tderiv_func_in(const ObjDev &o, double x) {
    return x < -o.eps ? 0 : 0.5 * (1 + cos(M_PI * x / o.eps));
}
__device__ __forceinline__ double coll_func(const ObjDev &o, double x) {
    return x > o.eps ? 0 : 0.5 - x * o.tf1;
}

/** Level-set function of the object at reference-map position (X,Y). */
__device__ __forceinline__ double obj_phi(const ObjDev &o, double X, double Y) {
    if (o.type == OBJ_SIMPLE_SPIN) {  // object.cc:177-180
        double th = atan2(Y, X), c = cos(3 * th);
        return sqrt(X * X + Y * Y) - o.g[0] - c * (o.g[1] + o.g[2] * c);
    }
    if (o.type == OBJ_ROUNDED_ROD) {  // obj_rounded_rod::phi, object.cc:275-278
        double fY = fabs(Y) - o.g[7];
        return (fY < 0 ? fabs(X) : sqrt(fY * fY + X * X)) - o.g[2];
    }
    if (o.type == OBJ_FLAG) {  // obj_flag::phi, object.cc:446-449
        const double L = o.g[2];
        return (X < 0 ? sqrt(X * X + Y * Y) : (X > L ? sqrt((X - L) * (X - L) + Y * Y) : fabs(Y))) - 0.5 * o.g[7];
    }
    if (o.type == OBJ_ELLIPSE) {
        // Semi-axes a=g[2], b=g[7] at angle th (g[8]=cos th, g[9]=sin th).
        // With r = |(X'/a, Y'/b)| in the body frame, (r-1)/|grad r| is the
        // signed distance to first order in the distance, which is all the
        // pinning band uses; the band rebuild makes it exact.
        const double xb = o.g[8] * X + o.g[9] * Y, yb = -o.g[9] * X + o.g[8] * Y;
        const double ia = 1 / o.g[2], ib = 1 / o.g[7];
        const double r = sqrt(xb * xb * ia * ia + yb * yb * ib * ib);
        const double gr = sqrt(xb * xb * ia * ia * ia * ia + yb * yb * ib * ib * ib * ib);
        if (gr == 0) return -fmin(o.g[2], o.g[7]);
        return (r - 1) * r / gr;
    }
    if (o.type == OBJ_FULL) return -1;  // obj_full::phi (object.hh:85)
    if (o.type == OBJ_TRIANGLE) {  // obj_triangle::phi, object.cc:93-95
        // the side whose normal selects the distance, then that normal turned
        // by -90 degrees applied to (X, Y)
        const double s0 = X * o.g[8] + Y * o.g[9], s1 = X * o.g[10] + Y * o.g[11],
                     s2 = X * o.nor2[0] + Y * o.nor2[1];
        const int k = s0 > 0 ? (s1 > 0 ? 0 : 2) : (s2 > 0 ? 1 : 0);
        const double nx = k == 0 ? o.g[8] : (k == 1 ? o.g[10] : o.nor2[0]),
                     ny = k == 0 ? o.g[9] : (k == 1 ? o.g[11] : o.nor2[1]);
        return Y * nx + -X * ny - o.g[2];
    }
    if (o.type == OBJ_LAMPREY) {  // obj_lamprey::phi, object.cc:554-558
        if (X > 0) return o.g[2] * Y * Y / (o.g[6] * o.g[6]) + X - o.g[2];
        const double wl = o.g[6] - (o.g[7] - o.g[6]) * X / o.g[3];
        return fmax(-o.g[3] - X, Y * Y / (wl * wl) - 1);
    }
    if (o.type == OBJ_HOOP) return fabs(sqrt(X * X + Y * Y) - o.g[7]) - o.g[2];  // object.cc:586-588
    if (o.type == OBJ_SEVEN_POINT) {  // obj_seven_point::phi, object.cc:117-124
        const double fac = 2 * M_PI / 7.;
        double theta = fabs(atan2(Y, X)), R = sqrt(X * X + Y * Y);
        theta = fabs(theta - fac * int(theta / fac + 0.5));
        X = R * cos(theta) - o.g[2];
        Y = R * sin(theta);
        return X * cos(0.25 * fac) - Y * sin(0.25 * fac) > 0 ? sqrt(X * X + Y * Y)
                                                             : Y * cos(0.25 * fac) + X * sin(0.25 * fac);
    }
    if (o.type == OBJ_FLAPPER) {  // obj_flapper::phi, object.cc:284-287
        const double fX = fabs(X) - o.g[7];
        return (fX < 0 ? fabs(Y) : sqrt(fX * fX + Y * Y)) - o.g[2];
    }
    if (o.type == OBJ_PISTON) {  // obj_piston::phi, object.cc:243-246
        const double gx = fabs(X) - o.g[2], gy = fabs(Y) - o.g[7];
        return gx > gy ? gx : gy;
    }
    if (o.type == OBJ_SQUARE) {  // obj_square::phi, object.cc:83-87
        X = fabs(X) - o.g[2];
        Y = fabs(Y) - o.g[2];
        return X < 0 || Y < 0 ? fmax(X, Y) : sqrt(X * X + Y * Y);
    }
    return sqrt(X * X + Y * Y) - o.g[2];  // obj_circle::phi, object.cc:22-24
}

/** Initial reference map (object::transform / obj_standard::transform). */
__device__ __forceinline__ void obj_transform(const ObjDev &o, double x, double y, double &X, double &Y) {
    if (o.type == OBJ_SIMPLE_SPIN || o.type == OBJ_FULL || o.type == OBJ_HOOP) { X = x; Y = y; }  // object::transform
    else if (o.type == OBJ_FLAPPER || o.type == OBJ_LAMPREY) {
        // translation, then rotation (object.hh:272-276, 573-577)
        x -= o.g[0];
        y -= o.g[1];
        X = x * o.g[4] + y * o.g[5];
        Y = -x * o.g[5] + y * o.g[4];
    } else { X = x - o.g[0]; Y = y - o.g[1]; }  // the piston's g[0] = 0 (object.hh:406-408)
}

/** Initial solid velocity (object::velocity / obj_standard::velocity,
 * object.cc:13-16). */
__device__ __forceinline__ void obj_velocity(const ObjDev &o, double X, double Y, double &u, double &v) {
    if (o.type == OBJ_FLAG) {  // obj_flag::velocity, object.cc:489-496
        X -= o.g[2];
        const double rsq = X * X + Y * Y;
        u = 0;
        v = rsq < o.g[10] ? o.g[9] * trans_func_in(o, sqrt(rsq) - o.g[8]) : 0.;
    } else if (o.type == OBJ_CIRCLE || o.type == OBJ_SQUARE || o.type == OBJ_ROUNDED_ROD ||
               o.type == OBJ_ELLIPSE) {
        u = o.g[4] - o.g[6] * Y;
        v = o.g[5] + o.g[6] * X;
    } else { u = 0; v = 0; }  // object::velocity (object.hh:32-34)
}

/** Extra accelerations (object::accel overrides): the simple spinner's
 * rotating pivot (object.cc:189-197), the flag's anchor (object.cc:476-484)
 * and the gravity of the circle, the square, the triangle, the rounded rod
 * and the ellipse (object.cc:31-34, 41-44, 65-70, 75-78). */
__device__ __forceinline__ void obj_accel(const ObjDev &o, double x, double y, double X, double Y,
                                          double phiv, double &ax, double &ay) {
    if (o.type == OBJ_SIMPLE_SPIN) {
        double rsq = x * x + y * y;
        if (rsq < o.g[6]) {
            double rx = X * o.cth - Y * o.sth, ry = X * o.sth + Y * o.cth,
                   K = o.g[7] * trans_func_in(o, sqrt(rsq) - o.g[3]);
            ax -= K * (x - rx);
            ay -= K * (y - ry);
        }
    } else if (o.type == OBJ_FLAG) {  // obj_flag::accel, object.cc:476-484
        const double delx = x - o.g[0], dely = y - o.g[1], rsq = delx * delx + dely * dely;
        if (rsq < o.g[10]) {
            const double K = o.g[11] * trans_func_in(o, sqrt(rsq) - o.g[8]);
            ax -= K * (x - X);
            ay -= K * (y - Y);
        }
    } else if (o.type == OBJ_SEVEN_POINT) {  // obj_seven_point::accel, object.cc:138-147
        const double delx = x - o.g[0], dely = y - o.g[1], rsq = delx * delx + dely * dely;
        if (rsq < o.g[6]) {
            const double rx = X * o.cth - Y * o.sth, ry = X * o.sth + Y * o.cth,
                         K = o.g[7] * trans_func_in(o, sqrt(rsq) - o.g[3]);
            ax -= K * (x - rx);
            ay -= K * (y - ry);
        }
    } else if (o.type == OBJ_PISTON) {  // obj_piston::accel, object.cc:260-269
        const double delx = x - o.g[8], dely = y - o.act, rsq = delx * delx + dely * dely;
        if (rsq < o.g[10]) {
            const double K = o.g[11] * trans_func_in(o, sqrt(rsq) - o.g[5]);
            ax -= K * (x - X);
            ay -= K * (dely - Y);
        }
    } else if (o.type == OBJ_FLAPPER || o.type == OBJ_FULL || o.type == OBJ_LAMPREY || o.type == OBJ_HOOP) {
        // no acceleration (object::accel, object.hh:73-74; obj_hoop keeps
        // its grav but does not override accel)
    } else {
        ay -= o.g[3] * trans_func_in(o, phiv);
    }
}

/** object::actuate overrides: scale the deformation gradient F = [[a, b],
 * [c, d]] at reference-map position (X, Y). obj_lamprey (object.cc:573-581):
 * a contraction wave of amplitude o.act travelling down the body, shifted by
 * o.shift; obj_flapper (object.cc:301-308): the current contraction o.act
 * inside the actuated region. */
__device__ __forceinline__ void obj_actuate(const ObjDev &o, double X, double Y, double &a, double &b, double &c,
                                            double &d) {
    if (o.type == OBJ_LAMPREY) {
        const double la = o.g[3], w1 = o.g[6], w2 = o.g[7];
        const double dx = X + (Y > 0 ? 1.5 * la : la) + o.shift, wl = w1 - (w2 - w1) * X / la, fac = fabs(Y) / wl;
        const double band = fmin(-X, la * 0.15 - fabs(dx - la * (static_cast<int>(dx / la) + 0.5)));
        const double st = exp(o.act * (fac < 1 ? fac * (2 - fac) : 1) * trans_func(o, -band));
        a *= st;
        b *= 1. / st;
        c *= st;
        d *= 1. / st;
        return;
    }
    if (o.type != OBJ_FLAPPER) return;
    const double fX = fabs(X) - o.g[9], ph = (fX < 0 ? fabs(Y) : sqrt(fX * fX + Y * Y)) - o.g[8];
    if (ph < o.eps) {
        const double fac = exp(o.act * Y * trans_func_in(o, ph));
        a *= fac;
        b *= 1. / fac;
        c *= fac;
        d *= 1. / fac;
    }
}

/** Grid constants (fluid_2d.hh:32-99). */
struct GridDev {
    int m, n, ml, nl, P;
    int mf, nf;  // FEM nodes
    int zpr;
    int xp;         // x-periodic (sim_type::x_prd)
    int yp;         // y-periodic (sim_type::y_prd)
    int pulses;     // initial fluid velocity of sim_velocity_pulses
    int solid_prd;  // periodic reference-map boundary conditions (fluid_2d::solid_prd_bc)
    int hflow;      // sim_horiz_flow inflow at the left edge
    double flow_u;  // its speed
    double ax, bx, ay, by, dx, dy, xsp, ysp, xxsp, yysp;
    double visc, rhof, eps, epsinv, w_scale, w_force;
    __device__ __forceinline__ int idx(int i, int j) const { return (j + 2) * P + (i + 2); }
};

/** Fluid fields (struct field, fields.hh:7-49). */
struct FluidDev {
    double *u, *v, *p, *rho;
    double *ux, *uy, *vx, *vy;
    double *ud, *vd, *ul, *vl, *ur, *vr, *uu, *vu;
    double *c0, *c1, *c2, *c3;
    double *s11, *s12, *s21, *s22;
};

/** Fields of one solid (struct s_field, fields.hh:51-79, plus the level set). */
struct SolidDev {
    double *X, *Y, *nX, *nY;
    double *Xx, *Xy, *Yx, *Yy;
    double *Xd, *Yd, *Xl, *Yl, *Xr, *Yr, *Xu, *Yu;
    double *phi, *phi_tmp;
    int *s;
};

// Per-object windows.
//
// The reference sweeps every object's arrays over the whole grid in every
// level-set and reference-map pass, but after the first band rebuild an
// object only differs from "far away" (status 7, phi at the positive band
// limit, no stress, no density, no acceleration) inside a box around its
// band and interior. The simulation keeps, per object, the bounding box B of
// the points that are inside it or next to its interface (status != 7 after
// the sign scan of the last rebuild) and derives:
//  - the rebuild window B + 2R + 4 (R the candidate radius): everything the
//    next rebuild can change, with the two-cell reach of the march stencil;
//  - the presence window B + R + 3: every point whose phi is below the band
//    limit, with a cell of stencil reach around it.
// Outside these the kernels below skip the object; the skipped work leaves
// every value the reference's computation reads unchanged. Before the first
// rebuild, and after a state upload, the windows are the whole grid.

/** Half-open window [x0,x1) x [y0,y1) on the level-set grid (ghosted
 * coordinates: level-set point (li,lj) is cell (li-2, lj-2)). */
struct LsWin {
    int x0, y0, x1, y1;
};

/** Which objects each 32 x 8 tile of the ghosted grid has to visit: those
 * whose presence window meets the tile, in increasing object order (so the
 * per-point sums over objects add the same terms in the same order). A null
 * start means every object everywhere. Tile (tx,ty) covers cells
 * 32(tx-1) <= i < 32tx and 8(ty-1) <= j < 8ty, so ghost cells i,j >= -2 fall
 * in tile 0 and the 32-wide rows of the cell kernels are never split. */
struct TileObjs {
    const int *start;  // ntiles + 1 offsets into obj
    const int *obj;
    int ntx;           // tiles per row
    int nobj;
    __device__ __forceinline__ void range(int i, int j, int &b, int &e) const {
        if (!start) { b = 0; e = nobj; return; }
        const int t = ((j + 8) >> 3) * ntx + ((i + 32) >> 5);
        b = start[t];
        e = start[t + 1];
    }
    __device__ __forceinline__ int at(int p) const { return start ? obj[p] : p; }
};

}  // namespace incrmt
