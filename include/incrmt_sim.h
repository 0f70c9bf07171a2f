/* incrmt_b200: C ABI of the simulation handle, the B200 replacement of
 * IncRMT's fluid_2d time integrator (fluid_2d.hh:131-177). Same conventions
 * as incrmt.h: int status returns, no exit, caller-owned host buffers. The
 * time step supports walls on all sides (simple spin, sediment), walls in x
 * with the inflow and zero-pressure outlet of sim_horiz_flow and periodic y
 * (flag), and periodicity in both directions (conv_test's
 * sim_velocity_pulses). Other combinations (periodic in one direction with
 * walls and no outlet in the other, or the outlet with x periodicity) and odd
 * sizes in a periodic direction are rejected with INCRMT_ERR_BADARG. */
#ifndef INCRMT_SIM_H
#define INCRMT_SIM_H

#include "incrmt.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct incrmt_sim incrmt_sim;

/** Grid and domain (fluid_2d ctor arguments m, n and sim_type's
 * ax,bx,ay,by,x_prd,y_prd; fluid_2d.cc:26-43, sim_type.hh:51-55). */
typedef struct incrmt_grid {
    int m, n;
    double ax, bx, ay, by;
    int x_prd, y_prd;
} incrmt_grid;

/** Physical and numerical parameters (fluid_2d ctor: visc, rhof, tw, pinw,
 * ntrace; sim_type w_scale/w_force, default 3 and 20 when <= 0; fluid_2d::zpr;
 * plus the projection tolerance and precision of this implementation).
 * horiz_flow selects sim_horiz_flow (sim_type.hh:117-141, sim_type.cc:51-64):
 * a uniform inflow of speed flow_u through the left edge (its two ghost
 * columns hold (flow_u, 0)), the zero-pressure right edge (zpr is set) and
 * the fluid initialised to (flow_u, 0). */
typedef struct incrmt_phys {
    double visc, rhof, tw, pinw;
    double w_scale, w_force;
    int ntrace;
    int zpr;
    int precision;       /* INCRMT_PREC_FP64 or INCRMT_PREC_MIXED for both projections */
    double mg_rel_tol;   /* relative residual of each projection (default 1e-9 when <= 0) */
    int horiz_flow;      /* 1: sim_horiz_flow boundary and initial conditions */
    double flow_u;       /* its inflow speed U */
    int pulses;          /* 1: sim_velocity_pulses' initial fluid velocity (sim_type.cc:43-47) on
                            the doubly periodic [-1,1]^2 of that scenario */
} incrmt_phys;

/** Object kinds (subclasses of object, object.hh). */
#define INCRMT_OBJ_SIMPLE_SPIN 0  /* params: r_scale, a1, a2, piv_r, th_max, omega (object.hh:447) */
#define INCRMT_OBJ_CIRCLE      1  /* params: cx, cy, cr, uu, vv, omega, grav (object.hh:128-138) */
#define INCRMT_OBJ_ROUNDED_ROD 2  /* params: cx, cy, cr, cl, grav (object.hh:218-241) */
#define INCRMT_OBJ_ELLIPSE     3  /* params: cx, cy, a, b, theta, grav: an ellipse with semi-axes a, b
                                     rotated by theta, falling under grav like obj_circle; it has no
                                     counterpart in the reference */
#define INCRMT_OBJ_FLAG        4  /* params: cx, cy, flag_l, flag_w, flag_a, perturb_v, ntrace: a flag
                                     anchored at its leading end (obj_flag, object.hh:471-505,
                                     object.cc:420-496), tracking ntrace points along its length */
#define INCRMT_OBJ_SQUARE      5  /* params: cx, cy, cr, uu, vv, omega, grav: a square of half side cr
                                     (obj_square, object.hh:142-152, object.cc:41-44, 83-87) */
#define INCRMT_OBJ_SEVEN_POINT 6  /* params: cx, cy, cr, piv_r, th_max, omega: a seven-pointed star
                                     spun by a stiff anchor of radius piv_r (obj_seven_point,
                                     object.hh:176-213, object.cc:100-147) */
#define INCRMT_OBJ_FLAPPER     7  /* params: cx, cy, cr, cl, ar, al, theta, m_stretch, T: a rod that
                                     swims by periodically contracting its actuated core
                                     (obj_flapper, object.hh:245-285, object.cc:284-308) */
#define INCRMT_OBJ_PISTON      8  /* params: lx, ly, cx, y_start, y_end, duration, anch_r: a block
                                     dragged by an anchor moving from y_start to y_end, tracking the
                                     point (-cx, y_start) (obj_piston, object.hh:369-418,
                                     object.cc:224-269) */
#define INCRMT_OBJ_CIRCLE_TRACK 9 /* params: cx, cy, cr, uu, vv, omega: a circle tracking the points
                                     (cx -+ cr/2, cy) (obj_circle_track, object.hh:509-538,
                                     object.cc:504-549) */
#define INCRMT_OBJ_FULL        10 /* no params: a solid filling the whole domain (obj_full,
                                     object.hh:83-86), used with incrmt_set_solid_prd_bc */
#define INCRMT_OBJ_TRIANGLE    11 /* params: cx, cy, cr, theta, grav: an equilateral triangle with
                                     vertices cr from its centre, rotated by theta, falling under grav
                                     (obj_triangle, object.hh:155-172, object.cc:52-70, 93-95) */
#define INCRMT_OBJ_LAMPREY     12 /* params: cx, cy, theta, le, dis, w1, w2, T, mlam: a swimmer of
                                     length le (head dis) and half-widths w1, w2, actuated by a
                                     contraction wave of period T and maximum mlam (obj_lamprey,
                                     object.hh:542-595, object.cc:554-581) */
#define INCRMT_OBJ_HOOP        13 /* params: r_in, r_out, grav: a hoop about the origin; grav is
                                     kept but, as in the reference, never applied (obj_hoop,
                                     object.hh:598-611, object.cc:586-588) */

/** An object plus its material constants (object*, mat_const;
 * fluid_2d::add_object, fluid_2d.cc:74-90; obj_field.hh:15-29). */
typedef struct incrmt_object_desc {
    int type;
    double G, rhos, ev_trans_mult;
    int set_velocity;
    double params[12];
} incrmt_object_desc;

/** Field ids for get/set: 0..23 the members of struct field in order
 * (u,v,p,rho,ux,uy,vx,vy,ud,vd,ul,vl,ur,vr,uu,vu,c0,c1,c2,c3,s11,s12,s21,s22;
 * fields.hh:7-49); 100..115 the members of struct s_field of object k
 * (X,Y,nX,nY,Xx,Xy,Yx,Yy,Xd,Yd,Xl,Yl,Xr,Yr,Xu,Yu; fields.hh:51-79). */
#define INCRMT_FIELD_PHI    200  /* level set of object k */
#define INCRMT_FIELD_STATUS 201  /* level-set status of object k (as doubles) */

typedef struct incrmt_sim_stats {
    long long steps;
    long long vcycles_mac, vcycles_fem;   /* V-cycles summed over all projections */
    long long solves_mac, solves_fem;
    long long march_sweeps, extrap_sweeps;
    long long launches;                    /* kernels issued by this handle */
    double dt_reg, time;
    long long march_monotone;              /* band rebuilds that needed the monotone march sweeps */
    long long window_points;               /* level-set points in the objects' current rebuild
                                              windows (all objects' whole grids when off) */
    long long coarse_builds;               /* Galerkin hierarchy rebuilds, MAC plus FEM */
    long long coarse_retries;              /* projections solved again after a failed solve on lagged
                                              coarse levels, with the levels rebuilt */
    long long mixed_fallbacks;             /* mixed-precision projections finished with FP64 V-cycles
                                              (an FP32 correction did not halve the residual) */
    long long krylov_fallbacks;            /* projections whose flexible CG handed over to plain FP64
                                              V-cycles (incrmt_sim_set_krylov) */
} incrmt_sim_stats;

/** Creates the simulation (fluid_2d::fluid_2d, fluid_2d.cc:26-43). */
int incrmt_create(const incrmt_grid *g, const incrmt_phys *p, incrmt_sim **out);

/** Adds a solid (fluid_2d::add_object, fluid_2d.cc:74-90). */
int incrmt_add_object(incrmt_sim *h, const incrmt_object_desc *d);

/** Chooses the extra viscosity and time step and initialises every field
 * (fluid_2d::initialize, fluid_2d.cc:101-122, without the tracer placement;
 * see incrmt_set_tracers). dt_reg receives fluid_2d::dt_reg. */
int incrmt_initialize(incrmt_sim *h, double ev_mult, double dt_pad, double dt_ev_pad, double *dt_reg);

/** Places the ntrace passive tracers at host positions (x,y pairs);
 * fluid_2d::init_tracers (fluid_2d.cc:1377-1386) draws them on the host. */
int incrmt_set_tracers(incrmt_sim *h, const double *xy);

/** One time step (fluid_2d::step_forward, fluid_2d.cc:298-369). */
int incrmt_step(incrmt_sim *h, double dt);

/** nsteps time steps, then waits for the device. */
int incrmt_steps(incrmt_sim *h, double dt, int nsteps);

/** Runs one step function on the current state (for parity tests): 0 tracer
 * stage 1, 1/2 normal derivatives, 3 Godunov (tangential), 5 tangential
 * derivatives, 6/7 half-time edge values, 8 Godunov, 9 MAC projection,
 * 10 update_reference_map, 11 pin, 12 set_boundaries, 13 compute_stress,
 * 14 compute_ustar, 15 finite_element_projection + copy_pressure,
 * 17 update_velocity, 18 tracer stage 2, 19 set_rho, 20 a whole step,
 * 21 build_band, 22 extrapolation. Edge boundary conditions (4) and
 * copy_pressure (16) are fused into their neighbours and do nothing alone. */
int incrmt_stage(incrmt_sim *h, int stage, double dt);

/** Copies a ghosted (m+4)x(n+4) field to / from a host array (row-major). */
int incrmt_get_field(incrmt_sim *h, int id, int k, double *host);
int incrmt_set_field(incrmt_sim *h, int id, int k, const double *host);

/** Projection arrays (m*n MAC, (m+1)*(n+1) FEM): which = 0 MAC solution
 * (mgs_base::z of ms_mac, the warm start of the next solve), 1 FEM solution,
 * 2 MAC right-hand side, 3 FEM right-hand side (fluid_2d::src). */
int incrmt_get_mg(incrmt_sim *h, int which, double *host);
int incrmt_set_mg(incrmt_sim *h, int which, const double *host);

int incrmt_get_time(const incrmt_sim *h, double *t);
/** Sets the simulation time; also re-evaluates the objects' time-dependent
 * state (object::pre_stress_setup) at that time. */
int incrmt_set_time(incrmt_sim *h, double t);

/** Passive tracers: ntrace records of 4 doubles (x, y, stage velocity). */
int incrmt_get_tracers(incrmt_sim *h, double *host);

/** Object-tracked points: records of 6 doubles (x, y, stage velocity, X, Y). */
int incrmt_get_object_tracers(incrmt_sim *h, double *host, int *count);

/** Sets the object-tracked points (count records of 6 doubles, the layout of
 * incrmt_get_object_tracers; count must equal the number of tracked points)
 * and the step counter of their recording (obj_track::count: steps since the
 * last record, 1 after one), as when restarting from a saved state. */
int incrmt_set_object_tracers(incrmt_sim *h, const double *host, int count, int track_count);

/** Tracked-point records collected so far, 1 + 4*K doubles each for the K
 * object tracers of incrmt_get_object_tracers: the time, then for every
 * tracer its position before and after the correction onto the reference map
 * (obj_track::file_output, object.cc:202-219, 339-347). clear=1 empties the
 * list. */
int incrmt_track_records(incrmt_sim *h, double *host, int cap, int *count, int clear);

/** Adds a tracked-point record now (obj_track::write at frame output,
 * object.cc:333-336). */
int incrmt_record_track(incrmt_sim *h);

/** Bounding box of the solids for cropped output (obj_field::bound,
 * obj_field.cc:102-106, as fluid_2d::write_files uses it, fluid_2d_io.cc:74-79):
 * box = {li, ui, lj, uj} in ghosted indices, starting from {ml, 0, nl, 0} and
 * extended to every point whose level-set status is below 4 in any object. */
int incrmt_solid_bound(incrmt_sim *h, int box[4]);

/** One output frame as fluid_2d::output writes it (fluid_2d_io.cc:123-179),
 * assembled on the GPU: mode is the reference's field code (0 u, 1 v, 2 speed,
 * 3 p, 4 vorticity, 5 rho, 6 X, 7 Y, 8 phi, 9 volume change, 10 c0, 11 c1,
 * 12 divergence), box = {li, ui, lj, uj} the ghosted index box [li,ui)x[lj,uj).
 * host receives (uj-lj+1) x (ui-li+1) floats: row 0 = [ui-li, x coordinates],
 * then one row per j = [y, values], the gnuplot binary matrix layout. Modes
 * 4, 9 and 12 read the points below and to the left, so they need li, lj >= 1. */
int incrmt_frame(incrmt_sim *h, int mode, const int box[4], float *host);

int incrmt_get_stats(const incrmt_sim *h, incrmt_sim_stats *st);

/** Phases of a step timed by the profiler (device milliseconds). */
#define INCRMT_PHASE_TRACERS   0  /* tracer stages */
#define INCRMT_PHASE_ADVECTION 1  /* normal derivatives, Godunov, half-time edge values */
#define INCRMT_PHASE_MAC       2  /* MAC source, V-cycles, correction */
#define INCRMT_PHASE_REFMAP    3  /* reference-map update (without the extrapolation) */
#define INCRMT_PHASE_EXTRAP    4  /* reference-map extrapolation */
#define INCRMT_PHASE_PIN       5  /* pinning, band rebuild, density */
#define INCRMT_PHASE_STRESS    6  /* boundaries, stress, u*, velocity update */
#define INCRMT_PHASE_FEM       7  /* FEM source, V-cycles, pressure copy */
#define INCRMT_PHASE_MG_SETUP  8  /* coefficients and Galerkin hierarchy of both projections */
#define INCRMT_PHASES          9

/** fluid_2d::l_comparison (fluid_2d_io.cc:186-281): the error norms of
 * this (coarse) simulation against `fine`, whose m and n must be multiples of
 * this one's, into err[32]. For a = 0..7 (velocity count fraction, pressure
 * count fraction, velocity L2, pressure L2, velocity L1, pressure L1,
 * velocity max, pressure max) err[4a+l] holds the fluid (l=0), solid (1) and
 * blur-zone (2) parts and err[4a+3] their total (their maximum for the
 * maxima). The fine velocity is interpolated to the coarse cell centres, the
 * pressures compared at coinciding corners; like the reference it leaves the
 * differences in this simulation's c0 (velocity) and c1 (pressure) fields.
 * Synchronises both simulations' streams. */
int incrmt_l_comparison(incrmt_sim *h, incrmt_sim *fine, double *err);

/** Per-object windows (no reference counterpart; on by default). The
 * reference sweeps every object's level set and reference map over the whole
 * grid in every pass. With windows on, after the first band rebuild each
 * object's level-set, pinning and reference-map passes cover only a box
 * around its band and interior, and the per-cell passes over all objects
 * (stress, density, accelerations, advection) visit only the objects whose
 * box meets the cell's 32x8 tile. Every value the reference's step reads is
 * the same either way; what differs is only the never-read edge and slope
 * values of the reference map far outside each solid. Off (0) runs the
 * whole-grid passes throughout; a state upload (incrmt_set_field) returns
 * to whole-grid passes until the next rebuild. */
int incrmt_sim_set_windows(incrmt_sim *h, int on);

/** Warm start of the two projections' solves (no reference counterpart;
 * default 0): 0 the previous step's solution, as the reference's
 * fluid_2d::mac_projection and finite_element_projection solve from the
 * pressure left in place (fluid_2d.cc:1175-1236, 1297-1328); 1 from the
 * third solve on, the linear extrapolation 2 z(n-1) - z(n-2) of the last two
 * solutions (one extra array per system); 2 from the fourth solve on, the
 * quadratic 3 z(n-1) - 3 z(n-2) + z(n-3) (two extra arrays per system).
 * Every solve still stops at the same
 * relative residual; the start only changes how many V-cycles that takes. A
 * learned guess (incrmt_sim_set_learned) corrects whichever start this
 * gives. Setting the mode, and incrmt_set_field, restart the history.
 * INCRMT_ERR_BADARG for another mode. */
int incrmt_sim_set_guess(incrmt_sim *h, int mode);

/** How often the projections rebuild their Galerkin coarse operators: every
 * `every` projections (1: on every density change, as the reference's solver
 * setup does), sooner when a solve takes more than one V-cycle over the first
 * solve after the last rebuild, and always after incrmt_set_field. The fine
 * operator always uses the current density, so every solve still reaches the
 * same relative residual; stale coarse levels only steer convergence.
 * Default 1 (the reference's policy); the C++ host's fluid_2d and the
 * benchmark use 16, which on the rotor and sediment scenes keeps the V-cycle
 * counts and removes most of the setup time. */
int incrmt_sim_set_coarse_refresh(incrmt_sim *h, int every);

/** Flexible conjugate gradients around the V-cycle in both projections
 * (incrmt_mg_set_krylov; off by default, the reference's plain V-cycles).
 * Every projection still reaches the same relative residual. */
int incrmt_sim_set_krylov(incrmt_sim *h, int on);

/** fluid_2d::solid_prd_bc (fluid_2d.hh:124), set before incrmt_initialize on
 * a doubly periodic domain: every object's reference map is periodic up to
 * the box lengths (set_boundaries_solid and edge_boundary_conditions_solid_pre
 * / _post, fluid_2d.cc:784-835) and the wall force and object accelerations
 * are off (fluid_2d.cc:1037). ftest's "full" scenario and conv_test's type 2
 * pair it with INCRMT_OBJ_FULL. */
int incrmt_set_solid_prd_bc(incrmt_sim *h, int on);

/** Turns timing on or off (CUDA events on the handle's stream; no reference
 * counterpart) and clears the accumulated times: bit 0 times the phases,
 * bit 1 times every fine-level smoothing launch of both projections (their
 * V-cycles then run without CUDA graphs). */
int incrmt_sim_set_profiling(incrmt_sim *h, int on);

/** Fine-level smoothing launches of the MAC (which = INCRMT_SYS_MAC) or FEM
 * projection timed since bit 1 of the profiling flags was set: total device
 * milliseconds, algorithmic bytes (updated unknowns x (3+c) x 8, c = 2 MAC,
 * 1 FEM) and launches. */
int incrmt_sim_mg_profile(incrmt_sim *h, int which, double *ms, double *bytes, long long *launches);

/** Accumulated device time per phase since profiling was turned on
 * (INCRMT_PHASES doubles, milliseconds). */
int incrmt_sim_profile(incrmt_sim *h, double *ms);

/** The handle's CUDA stream (a cudaStream_t). */
void *incrmt_sim_stream(const incrmt_sim *h);

void incrmt_destroy(incrmt_sim *h);

#ifdef __cplusplus
}
#endif

#endif
