// Geometric multigrid for the MAC and FEM pressure systems on one B200.
//
// Same method as the CPU oracle's TGMG-API shim, so that V-cycle counts are
// comparable: vertex-style coarsening (coarse I on fine 2I), an
// operator-dependent prolongation P (black-box multigrid weights from the
// collapsed stencil: bilinear for constant coefficients, following the flux
// across density jumps and Dirichlet edges), restriction P^T, Galerkin coarse
// operators P^T A P rebuilt on every density change, four-colour Gauss-Seidel smoothing visited as
// (0,0),(1,1),(1,0),(0,1) (red-black for the 5-point MAC stencil), V(2,2)
// cycles, and a one-block Gauss-Seidel solve on the coarsest level.
//
// Precision. FP64 mode runs everything in double. Mixed mode keeps the outer
// residual r = b - A z and the update z += e in FP64 and solves A e = r with
// one FP32 V-cycle per outer iteration (FP32 copies of the fine coefficients
// and of the Galerkin stencils).
//
// Optionally (krylov) the outer iteration is a flexible conjugate gradient
// method, FCG(1), with one V-cycle of either precision as its preconditioner
// and the residual, direction and iterate in FP64.
#pragma once
#include <vector>
#include "common.cuh"
#include "incrmt_unet.h"
#include "mg_ops.cuh"

namespace incrmt {

struct MgLevel {
    int m = 0, n = 0;
    long N = 0;
    bool kx = false, ky = false;  // whether the next level halves x / y
    double *z = nullptr, *b = nullptr, *st = nullptr;  // FP64 arrays (level >= 1)
    float *zf = nullptr, *bf = nullptr, *stf = nullptr;  // FP32 arrays (all levels)
    double *z2 = nullptr;  // second FP64 iterate buffer of the tile smoothers (all levels)
    double *P = nullptr;   // prolongation to the next level: four weights per unknown (all but the last)
    float *zf2 = nullptr;  // and the FP32 one
};

class Multigrid {
public:
    int sys = INCRMT_SYS_MAC;
    int cm = 0, cn = 0;           // cell grid of the simulation
    int m = 0, n = 0;             // unknowns of the system
    int px = 0, py = 0, zpr = 0;
    double dx = 0, dy = 0, xxsp = 0, yysp = 0;
    double fm = 0, fc = 0, hex = 0, hey = 0;  // FEM stencil constants
    cudaStream_t stream = nullptr;
    std::vector<MgLevel> lev;
    // Fine-level coefficients: MAC ex/ey, FEM cell array c, FP64 and FP32.
    double *ex = nullptr, *ey = nullptr, *c = nullptr;
    float *exf = nullptr, *eyf = nullptr, *cf = nullptr;
    double *rho = nullptr;          // device copy of a host density array
    double *bbuf = nullptr;          // device right-hand side (host solves, FEM zpr masking)
    double *zbuf = nullptr;          // device iterate for host solves
    double *partial = nullptr;       // reduction partials
    double *ginv = nullptr;          // dense inverse of the coarsest level (FP64)
    float *ginvf = nullptr;          // and its FP32 copy
    double *hnorm = nullptr;         // pinned host scalars
    double *dnorm = nullptr;         // device scalars
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    long long launches = 0;
    bool ready = false;              // coefficients and hierarchy built
    // Lagged coarse operators: set_density_lagged recomputes the fine
    // coefficients every time but the Galerkin levels only every
    // coarse_every calls, when marked stale, or after a solve that took more
    // than one V-cycle over the first solve since the last rebuild.
    int coarse_every = 1;
    int coarse_age = 0;
    int coarse_vc0 = -1;
    bool coarse_stale = true;
    long long coarse_builds = 0;
    long long coarse_retries = 0;    // solves repeated after rebuilding lagged coarse levels
    long long mixed_fallbacks = 0;   // mixed-precision solves finished with FP64 V-cycles
    // Mixed solves that fell back in a row, the FP64 solves still to run
    // before mixed precision is tried again, and the solves run that way.
    static constexpr int kMixedStrikes = 3, kMixedRest = 50;
    int mixed_streak = 0, mixed_rest = 0;
    long long mixed_rested = 0;
    const double *lag_rho = nullptr; // density of the last set_density_lagged (read again on a retry)
    int lag_ld = 0;
    bool f32_stale = true;           // FP32 Galerkin stencils not cast since the last rebuild
    bool tiles = true;               // tile-fused smoothing where it applies
    int tail_level = -1;             // first level run by the one-block tail kernel
    cudaGraphExec_t gexec = nullptr; // captured V-cycle + norm
    cudaGraphExec_t setup_exec = nullptr;  // captured rebuild of the coarse levels
    long long setup_launches = 0;
    int gkey_prec = -1;
    const double *gkey_b = nullptr;
    const double *gkey_z = nullptr;
    long long graph_launches = 0;    // kernels in the captured graph
    // Flexible conjugate gradients with the V-cycle as preconditioner
    // (incrmt_mg_set_krylov; off by default). kr: FP64 residual, kp: search
    // direction, kq: A kp, ke: FP64 preconditioned residual (FP64 cycles;
    // mixed cycles leave it in lev[0].zf), kpart: 3 x kRedBlocks partial
    // sums, ks: device scalars (sum e, e.q, sum q, the previous direction's
    // p.q, p.q, p.r).
    bool krylov = false;
    double *kr = nullptr, *kp = nullptr, *kq = nullptr, *ke = nullptr;
    double *kpart = nullptr, *ks = nullptr;
    cudaGraphExec_t kexec = nullptr; // captured iteration (V-cycle, direction, step, norm)
    int kkey_prec = -1;
    const double *kkey_b = nullptr;
    const double *kkey_z = nullptr;
    long long kexec_launches = 0;
    long long krylov_fallbacks = 0;  // solves finished with plain FP64 V-cycles
    // Optional timing of the fine-level smoothing launches (the dominant
    // kernel): CUDA events around each launch on the handle's stream.
    bool prof = false;
    std::vector<cudaEvent_t> prof_ev;
    int prof_used = 0;
    double prof_ms = 0, prof_bytes = 0;
    long long prof_launches = 0;
    double pending_bytes = 0;
    int prof_begin(double bytes);
    int prof_end();
    int prof_collect();

    bool own_stream = true;
    int create(int sys, int cm, int cn, double ax, double bx, double ay, double by,
               int px, int py, int zpr, cudaStream_t ext = nullptr);
    void destroy();
    int set_density_device(const double *d_rho, int ld = 0);
    /** Unit density everywhere: the constant-density operators
     * (mgs_mac_const_rho, mgs_fem_const_rho; mgs_mac.hh, mgs_fem.cc:27-80),
     * which are the varying-density ones with every 1/rho equal to 1. */
    int set_unit_density();
    /** The fine-level coefficients from d_rho, with the coarse levels
     * rebuilt per the lag policy above. The converged solution depends on
     * the fine operator alone; the coarse levels only steer convergence. */
    int set_density_lagged(const double *d_rho, int ld);
    /** Records a solve's V-cycle count for the lag policy. */
    void note_vcycles(int vc);
    /** solve_device after set_density_lagged. If the solve fails (V-cycle cap
     * or a non-finite residual) while the coarse levels are lagged, i.e.
     * built for an earlier density, they are rebuilt from the density given
     * to set_density_lagged (which must still hold it) and the solve is
     * repeated once, from a zero iterate if the failed one is not finite.
     * The reference rebuilds its solver for every projection
     * (mgs_mac.cc:62-63, mgs_fem.cc:108-109), so a system it converges on
     * must not fail here for want of a rebuild. Any failure marks the coarse
     * levels stale. The statistics count the V-cycles of both attempts. */
    int solve_lagged(const double *d_b, double *d_z, const incrmt_mg_opts *o, incrmt_mg_stats *st, bool time_it);
    int solve_device(const double *d_b, double *d_z, const incrmt_mg_opts *o,
                     incrmt_mg_stats *st, bool time_it);
    int vcycle64(const double *d_b, double *d_z);
    int apply_device(const double *d_z, double *d_out);
    /** The right-hand side the solve uses: d_b itself, or for the FEM system
     * with the zero-pressure column a copy in bbuf with that column zeroed. */
    int effective_rhs(const double *d_b, const double **out);

    MacOp<double> mac64() const;
    MacOp<float> mac32() const;
    FemOp<double> fem64() const;
    FemOp<float> fem32() const;

private:
    int build_hierarchy();
    int galerkin_all();
    /** galerkin_all as a CUDA graph captured on first use and replayed. */
    int galerkin_graph();
    /** FP32 copies of the Galerkin stencils, made on the first mixed solve
     * after a rebuild (FP64 solves never read them). */
    int cast_levels();
    int cycle64(int l, const double *b0, double *z0);
    int cycle32(int l);
    int tail64();
    int vcycle_and_norm(int prec, const double *b, double *d_z, long N);
    int tail32();
    int norm2_rhs(const double *b, double *out_dev);
    int residual_norm(const double *b, const double *z, float *rf, double *out_dev);
    int fetch_norm(double *v);
    int krylov_alloc();
    /** kr = b - A z (and its FP32 copy into lev[0].bf in mixed precision),
     * ||kr||^2 into dnorm[0]. */
    int krylov_residual(int prec, const double *b, const double *d_z);
    /** One flexible-CG iteration: e = V-cycle(kr), the new direction, the
     * step along it, and ||kr||^2 into dnorm[0] and hnorm[0]. */
    int krylov_iteration(int prec, double *d_z, long N);
    /** Iterations of the flexible CG from d_z until the residual reaches
     * tol (*conv), fails to halve (*fell, the caller continues with plain
     * FP64 V-cycles) or is not finite (*finite false); *k counts them. */
    int krylov_solve(int prec, const double *b, double *d_z, long N, double tol, int maxc, int &k, double &rn2,
                     bool &conv, bool &finite, bool &fell);
};

/** Workspace of the learned initial guess (learned.cu), per solver. */
struct LearnedWork {
    double *r0 = nullptr, *ad = nullptr, *dfine = nullptr, *dots = nullptr;
    float *in = nullptr, *out = nullptr;
    long n_fine = 0, n_net = 0;
    void release();
};

/** Network grid of a solve: the m x n unknowns restricted by f, rounded up to
 * multiples of 16. */
void learned_grid(int m, int n, int f, int &H, int &W);
/** INCRMT_OK, or an error for systems the guess does not handle (x-periodic). */
int learned_supported(const Multigrid &mg);
/** r0 = b - A z and the network input features into w.in (H x W x 3). */
int learned_input(Multigrid &mg, LearnedWork &w, const double *d_b, const double *d_z, int f, int H, int W);
/** The whole guess: features, network, prolongation, step along d (rule 0:
 * residual rule, 1: energy rule only), optional applied/fallback counters. */
int learned_guess(Multigrid &mg, LearnedWork &w, incrmt_unet *net, const double *d_b, double *d_z, int f, int rule,
                  unsigned long long *cnt);
/** How many times the network's activation buffers have been (re)allocated
 * (a captured forward pass is valid only while this stays the same). */
long long unet_generation(const incrmt_unet *h);
/** Block averages of znew - zold on the network grid (training targets). */
int learned_target(Multigrid &mg, const double *znew, const double *zold, int f, int H, int W, float *tgt);

}  // namespace incrmt

/** The solver handle of the C ABI (include/incrmt.h). */
struct incrmt_mg {
    incrmt::Multigrid mg;
    incrmt::LearnedWork learned;
};
