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
