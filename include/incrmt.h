/* incrmt_b200: C ABI of the B200 implementation of IncRMT's per-timestep hot
 * path (libincrmt_gpu.so). Plain pointers and sizes only; every function
 * returns an int status (INCRMT_OK or a negative INCRMT_ERR_* code) and never
 * exits the process. Host buffers are caller-owned and complete on return.
 * One handle per host thread; each handle owns its device memory and one
 * CUDA stream. The reference interface each entry point replaces is cited
 * as file:line within the chr1shr/incrmt tree. */
#ifndef INCRMT_H
#define INCRMT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define INCRMT_OK                    0
#define INCRMT_ERR_NOCONV           -1  /* V-cycle cap reached ("V-cycle failed to converge", mgs_mac.cc:31-34) */
#define INCRMT_ERR_NONFINITE        -2  /* NaN/Inf in a residual or input */
#define INCRMT_ERR_NEWTON           -3  /* level-set closest-point failure (levelset.cc:275) */
#define INCRMT_ERR_EXTRAP_SINGULAR  -4  /* singular extrapolation fit (traverse.hh:211-222) */
#define INCRMT_ERR_OOM              -5  /* device allocation failed */
#define INCRMT_ERR_BADARG           -6  /* invalid argument */
#define INCRMT_ERR_CUDA             -7  /* other CUDA runtime error */

/* ---- linear systems ------------------------------------------------------ */
/** Which pressure system a solver handle holds. */
#define INCRMT_SYS_MAC 0  /* mgs_mac_varying_rho: cell-centred 5-point, edge 1/rho (mgs_mac.hh:64-102) */
#define INCRMT_SYS_FEM 1  /* mgs_fem_varying_rho: corner-node bilinear FE 9-point, cell 1/rho (mgs_fem.hh:86-136) */

/** Arithmetic of the V-cycles. */
#define INCRMT_PREC_FP64  0  /* smoothing, transfers and residuals in FP64 */
#define INCRMT_PREC_MIXED 1  /* FP32 V-cycles on the correction equation inside FP64 defect correction;
                                 a solve continues in FP64 once an FP32 step fails to halve the
                                 residual (incrmt_mg_mixed_fallbacks counts those solves) */

typedef struct incrmt_mg incrmt_mg;

typedef struct incrmt_mg_opts {
    double rel_tol;    /* stop once ||b-Az||_2 <= rel_tol*||b||_2 (default 1e-9 when <= 0) */
    int max_vcycles;   /* cap (default 200 when <= 0); reaching it returns INCRMT_ERR_NOCONV */
    int precision;     /* INCRMT_PREC_FP64 or INCRMT_PREC_MIXED */
} incrmt_mg_opts;

typedef struct incrmt_mg_stats {
    int vcycles;        /* V-cycles (outer iterations in mixed precision) of this solve */
    double rel_res;     /* final ||b-Az||_2/||b||_2 */
    double device_ms;   /* device time of setup + solve, CUDA events on the handle's stream */
} incrmt_mg_stats;

/** Creates a solver for the MAC or FEM system of an m x n cell grid on
 * [ax,bx]x[ay,by] with the given periodicity and right-edge zero-pressure flag.
 * Replaces the mgs_mac_varying_rho / mgs_fem_varying_rho constructors
 * (mgs_mac.cc:40-43, mgs_fem.cc:98-100). The FEM system has
 * (x_prd?m:m+1) x (y_prd?n:n+1) unknowns (fluid_2d.cc:30-31). A periodic
 * direction needs an even size. */
int incrmt_mg_create(int sys, int m, int n, double ax, double bx, double ay, double by,
                     int x_prd, int y_prd, int zpr, incrmt_mg **out);

/** Number of unknowns of the handle's system (m*n for MAC, m_fem*n_fem for FEM). */
int incrmt_mg_size(const incrmt_mg *h, int *m_sys, int *n_sys);

/** Sets the density from a host array of (m+4)*(n+4) ghosted cell values
 * (row-major, the fluid_2d field layout, fluid_2d.cc:37) and rebuilds the
 * coefficients and the multigrid hierarchy. Replaces
 * fluid_2d::set_edge_irho / set_corner_irho + tgmg::setup
 * (fluid_2d.cc:1140-1170, mgs_mac.cc:62-63, mgs_fem.cc:108-109). */
int incrmt_mg_set_density(incrmt_mg *h, const double *rho);

/** Same with a device array of (m+4)*(n+4) doubles. */
int incrmt_mg_set_density_device(incrmt_mg *h, const double *d_rho);

/** Solves A z = b from host buffers: b (read; for FEM with zpr its fixed
 * column is treated as zero, mgs_fem.cc:112), z (initial guess in, solution
 * out). Replaces mgs_*::solve_internal's tgmg::solve_v_cycle call
 * (mgs_mac.cc:66-70, mgs_fem.cc:115-119). Copies run on the handle's stream. */
int incrmt_mg_solve(incrmt_mg *h, const double *b, double *z,
                    const incrmt_mg_opts *opts, incrmt_mg_stats *stats);

/** Same with device pointers (b read-only, z in/out), on the handle's stream.
 * A solve reads each V-cycle's residual norm back to the host, so it must not
 * be called while the handle's stream is being captured into a CUDA graph
 * (that call returns INCRMT_ERR_BADARG). A right-hand side of zero norm
 * returns z = 0. */
int incrmt_mg_solve_device(incrmt_mg *h, const double *d_b, double *d_z,
                           const incrmt_mg_opts *opts, incrmt_mg_stats *stats);

/** Applies the system operator: out = A z (host buffers). For tests. */
int incrmt_mg_apply(incrmt_mg *h, const double *z, double *out);

/** Runs exactly one FP64 V-cycle on device arrays (b read, z in/out); the
 * mg_test timing mode (mg_test.cc:32-41). */
int incrmt_mg_vcycle_device(incrmt_mg *h, const double *d_b, double *d_z);

/** Turns on (1) or off (0) CUDA-event timing of the fine-level smoothing
 * launches, the dominant kernel, and clears the accumulated profile. No
 * reference counterpart (instrumentation). */
int incrmt_mg_set_profiling(incrmt_mg *h, int on);

/** Tile-fused smoothing (on by default; no reference counterpart): two
 * Gauss-Seidel sweeps per launch in shared-memory tiles wherever the level's
 * periodic directions have even sizes, with results identical to one launch
 * per colour in the V-cycle's four-colour order. Off (0) runs one launch per
 * colour everywhere; it exists to check that identity. */
int incrmt_mg_set_tiles(incrmt_mg *h, int on);

/** Flexible conjugate gradients around the V-cycle (no reference
 * counterpart; off by default). On (1), each solve iterates FCG(1) (Notay,
 * SIAM J. Sci. Comput. 22 (2000) 1444-1460) with one V-cycle of the
 * requested precision as the preconditioner: the direction is the
 * preconditioned residual made A-orthogonal to the previous direction, the
 * step minimises the energy norm along it, and the residual is updated in
 * FP64 (confirmed on b - A z when it reaches the tolerance). The tolerance,
 * the statistics (vcycles counts iterations, one V-cycle each) and the
 * result's accuracy are those of the plain solve; an iteration that fails to
 * halve the residual hands the solve to plain FP64 V-cycles from the current
 * iterate (counted by incrmt_mg_krylov_fallbacks). Off, the solve is the
 * reference's plain V-cycle iteration (mg.solve_v_cycle, mgs_mac.cc:67,
 * mgs_fem.cc:116). */
int incrmt_mg_set_krylov(incrmt_mg *h, int on);

/** Solves since creation in which the flexible CG handed over to plain FP64
 * V-cycles. */
long long incrmt_mg_krylov_fallbacks(const incrmt_mg *h);

/** Lagged coarse operators (no reference counterpart; default 1). With
 * every > 1 a density change recomputes the fine-level coefficients, which
 * define the system solved, but rebuilds the Galerkin coarse levels only on
 * every `every`-th change; the reference rebuilds on each one
 * (mgs_mac.cc:62-63, mgs_fem.cc:108-109). Stale coarse levels only steer
 * convergence: every solve still reaches its tolerance on the current
 * operator. If a solve fails (V-cycle cap or a non-finite residual) while its
 * coarse levels are lagged, they are rebuilt from the last density and the
 * solve is repeated once, from zero if the iterate is not finite. With
 * every > 1, incrmt_mg_set_density_device copies the density into the
 * handle, so the caller's array need not outlive the call. */
int incrmt_mg_set_coarse_refresh(incrmt_mg *h, int every);

/** Mixed-precision solves (INCRMT_PREC_MIXED) since creation that finished
 * with FP64 V-cycles: a solve switches once an FP32 defect-correction step
 * fails to halve the FP64 residual norm, so it converges as the FP64 solve
 * would. After three such solves in a row the handle runs the next 50
 * mixed-precision requests as FP64 solves (not counted here), then tries
 * FP32 cycles again. */
long long incrmt_mg_mixed_fallbacks(const incrmt_mg *h);

/** Galerkin hierarchy rebuilds since creation; *retries (if not null)
 * receives the number of solves repeated after rebuilding lagged levels. */
long long incrmt_mg_coarse_builds(const incrmt_mg *h, long long *retries);

/** Accumulated profile since incrmt_mg_set_profiling: total device time (ms)
 * of the timed launches, their algorithmic bytes (updated unknowns x (3+c)
 * words) and their number. */
int incrmt_mg_profile(incrmt_mg *h, double *ms, double *bytes, long long *launches);

/** The handle's CUDA stream (a cudaStream_t), on which every kernel and copy
 * of the handle is issued; lets a caller time or order work against it. */
void *incrmt_mg_stream(const incrmt_mg *h);

/** Number of levels in the handle's hierarchy. */
int incrmt_mg_levels(const incrmt_mg *h);

/** Kernel launches issued by the handle since creation (for accounting). */
long long incrmt_mg_launches(const incrmt_mg *h);

void incrmt_mg_destroy(incrmt_mg *h);

/** Allocation-free out = A z for the MAC (sys 0) or FEM (sys 1) system of a
 * non-periodic m x n cell grid built from the ghosted density, all pointers
 * device pointers, work issued on `stream` (a cudaStream_t, 0 = default) and
 * not waited for. It has no counterpart in the reference. It is for callers
 * that cannot allocate device memory (a framework arena that forbids
 * cudaMalloc, a real-time loop that must not take allocation locks): it calls
 * no allocator, and its only scratch, the edge or cell reciprocal densities,
 * lives in a ~1 MB array compiled into the library (held by every GPU that
 * loads the library until exit). Grids larger than 256 x 256 cells are
 * rejected with INCRMT_ERR_BADARG. The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress); make that first call before
 * any stream capture. The address is cached per device for the process's
 * primary context: after cudaDeviceReset, or from a context other than the
 * primary one, it is not valid (a failed lookup is not cached). All calls share the array, so calls that overlap on the
 * GPU (other streams, other host threads) race; each call writes every
 * scratch word it reads. */
int incrmt_mg_apply_noalloc(int sys, int m, int n, double ax, double bx, double ay, double by,
                            int zpr, const double *d_rho, const double *d_z, double *d_out, void *stream);

/** Last error message of the calling thread (empty if none). */
const char *incrmt_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
