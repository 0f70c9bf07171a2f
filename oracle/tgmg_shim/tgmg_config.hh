/* Clean-room configuration for the TGMG-API shim.
 *
 * TEST INFRASTRUCTURE ONLY: this directory is part of the oracle. Only the
 * test suite, the smoke check and bench.py's CPU-baseline leg may build or
 * run it. The product (incrmt_b200) never links against it.
 *
 * IncRMT includes "tgmg.hh" from an external library (chr1shr/tgmg, no pinned
 * version: the reference expects it at ../tgmg, Makefile:4,14). That library
 * is absent, so this shim restates the published geometric-multigrid method
 * (Briggs, Henson & McCormick, "A Multigrid Tutorial", 2nd ed., ch. 3-4 and
 * 8: Galerkin coarse operators, Gauss-Seidel smoothing, V-cycles; the
 * operator-dependent prolongation of black-box multigrid, Dendy, J. Comput.
 * Phys. 48 (1982) 366-386) behind exactly the API used at the reference's call
 * sites (mgs_mac.cc:10-34,40-71; mgs_fem.cc:25-120; mgs_common.cc:70-74;
 * mg_test.cc:21-43; fluid_2d.cc:284-290). The GPU multigrid in incrmt_b200
 * implements the same V-cycle so that V-cycle counts are comparable. */
#ifndef TGMG_CONFIG_HH
#define TGMG_CONFIG_HH

#include <cstdlib>

/** Gauss-Seidel sweeps before the coarse-grid correction. */
const int tgmg_nu1=2;
/** Gauss-Seidel sweeps after the coarse-grid correction. */
const int tgmg_nu2=2;
/** Gauss-Seidel sweeps used as the solve on the coarsest level when that
 * level is the finest one (a grid too small to coarsen). */
const int tgmg_coarse_sweeps=64;
/** Coarse levels with at most this many unknowns are solved exactly, by a
 * dense inverse built at setup. */
const int tgmg_direct_max=96;
/** Coarsening stops once a level has at most this many unknowns. */
const int tgmg_coarsest_size=16;
/** Semi-coarsening: while the operator's coupling along one direction is
 * more than this many times that along the other, only the strongly coupled
 * direction is halved (point Gauss-Seidel smooths only along it). */
const double tgmg_semi_ratio=2.0;
/** Maximum number of levels in a hierarchy. */
const int tgmg_max_levels=24;
/** Maximum number of V-cycles in one solve before reporting failure. */
const int tgmg_max_vcycles=200;

/** Relative residual target ||b-Az||_2 <= rtol*||b||_2 of every solve. The
 * default 1e-9 is the tolerance both the CPU and GPU solvers use; the
 * environment variable INCRMT_MG_RTOL overrides it. */
inline double tgmg_rel_tol() {
    static double r=-1;
    if(r<0) {
        const char *e=getenv("INCRMT_MG_RTOL");
        r=e!=NULL?atof(e):1e-9;
        if(!(r>0)) r=1e-9;
    }
    return r;
}

/** Absolute residual floor. The reference computes it per system from a
 * stencil scale and a multiplier (mgs_mac.hh:32, mgs_fem.cc:17); here it is
 * that scale times the multiplier times machine epsilon, so a solve whose
 * right-hand side is already (numerically) zero terminates. */
inline double tgmg_accuracy(double scale,double mult) {
    return scale*mult*2.220446049250313e-16;
}

#endif
