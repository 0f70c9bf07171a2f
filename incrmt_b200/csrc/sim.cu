// The simulation handle: device state of one fluid_2d, its time step
// (fluid_2d::step_forward, fluid_2d.cc:298-369) as a sequence of kernels on
// one stream, and the C ABI that replaces the fluid_2d interface.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <utility>
#include <vector>
#include "incrmt_sim.h"
#include "incrmt_unet.h"
#include "mg.cuh"
#include "step_kernels.cuh"
#include "ls_kernels.cuh"
#include "tracer_kernels.cuh"
#include "frame_kernels.cuh"

namespace incrmt {

namespace {
const dim3 kB2(32, 8);
inline dim3 g2(int m, int n) { return dim3(cdiv(m, 32), cdiv(n, 8)); }
constexpr int kLsMaxSweeps = 400;       // cap of the fixed-point sweeps of one march
constexpr int kExtrapMaxSweeps = 1000;  // cap of the extrapolation wavefront sweeps
constexpr int kLearnedStrikes = 8;      // rejected learned guesses in a row ...
constexpr int kLearnedRest = 32;        // ... after which this many projections skip the guess
}  // namespace

struct Sim {
    GridDev g{};
    LsGrid lg{};
    cudaStream_t stream = nullptr;
    FluidDev f{};
    std::vector<double *> allocs;
    std::vector<ObjDev> obj;
    std::vector<SolidDev> sol;
    std::vector<incrmt_object_desc> desc;
    ObjDev *d_obj = nullptr;
    SolidDev *d_sol = nullptr;
    double *src_mac = nullptr, *z_mac = nullptr, *src_fem = nullptr, *z_fem = nullptr;
    std::vector<LsObj> lso;                         // level-set working arrays per object
    LsObj *d_lso = nullptr;
    int *d_list = nullptr, *d_list_k = nullptr;     // combined point list of all objects
    int list_cap = 0;
    std::vector<void *> raw_allocs;                 // non-double per-object arrays
    int coop_blocks_fim = 0, coop_blocks_ext = 0;   // co-resident grid sizes
    int *d_flags = nullptr;  // [0..2] sweep change flags, [3] sweeps, [4] converged, [5] fit error,
                           // [6] Newton error, [7] list length, [8] tracer remaps, [9] correction failure
    int *h_flags = nullptr;                         // pinned
    double *partial = nullptr;
    double *tm = nullptr, *otm = nullptr;          // passive and object tracers
    int *d_remap = nullptr;                         // indices of tracers that left the box
    long long remapped_tracers = 0;
    int ntrace = 0, nobjtr = 0;
    Multigrid mac, fem;
    // Learned warm start of each projection (0 MAC, 1 FEM) and the capture of
    // training samples (network input and target per projection).
    struct Learned {
        incrmt_unet *net = nullptr;
        int factor = 0, rule = 0;
        LearnedWork w;
        float *cap_in = nullptr, *cap_tgt = nullptr;
        int cap = 0, cap_factor = 0;
        long long captured = 0;
        double *z0 = nullptr;  // the warm start, kept for the capture's target
        long z0_n = 0;
        // The guess (features, network, step along its output) captured into
        // a CUDA graph for one (net, b, z), replayed on later projections:
        // some sixty small launches, most of them the network's layers on a
        // 256-square grid, whose host-side launch cost was a good part of the
        // guess's time.
        cudaGraphExec_t gexec = nullptr;
        const incrmt_unet *gkey_net = nullptr;
        long long gkey_gen = -1;
        const double *gkey_b = nullptr;
        const double *gkey_z = nullptr;
        long long glaunches = 0;
        const incrmt_unet *warm_net = nullptr;  // network and allocation generation
        long long warm_gen = -1;                // after the last direct guess
        bool gfail = false;
        // Rejected guesses in a row, projections still to skip, the rejection
        // count last read, whether this projection computed a guess, and the
        // projections skipped so far.
        int fb_streak = 0, skip = 0;
        unsigned long long fb_seen = 0;
        bool ran = false;
        long long skipped = 0;
        void release_graph() {
            if (gexec) cudaGraphExecDestroy(gexec);
            gexec = nullptr;
            gkey_net = nullptr;
        }
    } learn[2];
    unsigned long long *d_lcnt = nullptr;  // [sys][applied, fallback]
    // Warm start of the projections: 0 the previous solution (the
    // reference's), 1 its linear extrapolation 2 z(n-1) - z(n-2) once two
    // solutions exist, 2 the quadratic one 3 z(n-1) - 3 z(n-2) + z(n-3) once
    // three exist; zold[sys] holds z(n-2), zold2[sys] z(n-3), nsol[sys] the
    // solves since the history was last reset.
    int guess = 0;
    double *zold[2] = {nullptr, nullptr}, *zold2[2] = {nullptr, nullptr};
    long long nsol[2] = {0, 0};
    int extrapolate_guess(int sys, double *z);
    incrmt_mg_opts mgo{1e-9, 200, INCRMT_PREC_FP64};
    double dt_reg = 0, time = 0;
    double w_scale = 3, w_force = 20, tw = 2.5, pinw = 2.5;
    bool initialized = false;
    // fluid_2d::const_rho (fluid_2d.cc:126-137): every solid's density within
    // small_number of the fluid's; the projections then use the constant-
    // density operators, set once, and pin leaves rho alone.
    bool const_rho = false;
    long long steps = 0;
    long long vc_mac = 0, vc_fem = 0, solves_mac = 0, solves_fem = 0;
    long long ls_sweeps = 0, ex_sweeps = 0;
    long long ls_monotone = 0;                      // band rebuilds that needed the monotone sweeps
    long long launches = 0;
    int track_count = 1;                            // obj_track step counter
    int track_every = 10;                           // steps between its records
    int trk = -1;                                   // object whose points are tracked
    int t_correction = 1;
    int pre_stress_objects = 0;
    std::vector<double> track;                      // records: time, xpre, ypre, x, y
    float *d_frame = nullptr;                       // output frame staging (grown on demand)
    size_t frame_cap = 0;
    int *d_box = nullptr;                           // solid bounding box reduction
    // Per-object windows (sim.cuh). d_win holds kMaxObjects windows of each
    // kind: 0 rebuild, 1 presence, 2 presence at the last reference-map
    // update, 3 the whole grid. d_tiles holds the tile object lists of the
    // presence windows (ntx*nty+1 offsets, then the lists).
    LsWin *d_win = nullptr, *h_win = nullptr;       // device / pinned host
    int *d_lsbox = nullptr, *h_lsbox = nullptr;     // box of the last sign scan, per object
    int *d_tiles = nullptr, *h_tiles = nullptr;
    size_t tiles_cap = 0;
    int ntx = 0, nty = 0;
    bool win_enable = true;   // windows after the first rebuild (else the whole grid always)
    bool win_valid = false;   // windows derived from a rebuild since the last state change
    bool x_synced = false;    // X == nX outside the window of the last reference-map update
    bool pref_valid = false;  // that window is recorded (kind 2)
    int wmax[4][2] = {};      // largest window of each kind (width, height)
    // Optional phase timing: CUDA events on the stream at phase boundaries.
    bool prof = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<int> ev_phase;                      // phase of each recorded (start,end) pair
    int ev_used = 0;
    double phase_ms[INCRMT_PHASES] = {0};
    long long phase_n[INCRMT_PHASES] = {0};
    int cur_phase = -1;
    int phase_begin(int ph) {
        if (!prof) return INCRMT_OK;
        if (ev_used + 2 > static_cast<int>(ev_pool.size())) {
            if (ev_used + 2 > 8192) { int r = phase_collect(); if (r) return r; }
            while (ev_used + 2 > static_cast<int>(ev_pool.size())) {
                cudaEvent_t e;
                INCRMT_CK(cudaEventCreate(&e));
                ev_pool.push_back(e);
            }
        }
        INCRMT_CK(cudaEventRecord(ev_pool[ev_used], stream));
        cur_phase = ph;
        return INCRMT_OK;
    }
    int phase_end() {
        if (!prof || cur_phase < 0) return INCRMT_OK;
        INCRMT_CK(cudaEventRecord(ev_pool[ev_used + 1], stream));
        if (static_cast<int>(ev_phase.size()) <= ev_used / 2) ev_phase.resize(ev_used / 2 + 1);
        ev_phase[ev_used / 2] = cur_phase;
        ev_used += 2;
        cur_phase = -1;
        return INCRMT_OK;
    }
    int phase_collect() {
        if (ev_used == 0) return INCRMT_OK;
        INCRMT_CK(cudaStreamSynchronize(stream));
        for (int k = 0; k + 1 < ev_used; k += 2) {
            float ms = 0;
            INCRMT_CK(cudaEventElapsedTime(&ms, ev_pool[k], ev_pool[k + 1]));
            phase_ms[ev_phase[k / 2]] += ms;
            phase_n[ev_phase[k / 2]]++;
        }
        ev_used = 0;
        return INCRMT_OK;
    }

    int alloc(double **p, size_t n) {
        INCRMT_CK(cudaMalloc(p, sizeof(double) * n));
        INCRMT_CK(cudaMemsetAsync(*p, 0, sizeof(double) * n, stream));
        allocs.push_back(*p);
        return INCRMT_OK;
    }
    size_t cells() const { return static_cast<size_t>(g.P) * g.nl; }

    int create(const incrmt_grid *gr, const incrmt_phys *ph);
    int add_object(const incrmt_object_desc *d);
    int initialize(double ev_mult, double dt_pad, double dt_ev_pad);
    int step(double dt);
    int stage(int s, double dt);
    void destroy();

    // pieces
    int upload_objects();
    void pre_stress_setup(double t);
    int compute_stress();
    int set_boundaries();
    int set_rho();
    int pin();
    int build_bands();
    int godunov(bool tang);
    int extrapolate_all();
    int mac_projection();
    int fem_projection(double dt);
    int update_reference_map(double dt);
    int tracers(int stage, double dt);
    int record_track();
    int remap_tracers();
    int fetch_flags();
    int update_velocity(double dt);
    int learned_pre(int sys, const double *b, double *z);
    int learned_post(int sys, const double *z);
    int win_reset();
    int win_update();
    TileObjs tiles() const {
        const int no = static_cast<int>(obj.size());
        if (!win_valid) return TileObjs{nullptr, nullptr, ntx, no};
        return TileObjs{d_tiles, d_tiles + static_cast<size_t>(ntx) * nty + 1, ntx, no};
    }
    dim3 wgrid(int kind) const {
        const int w = wmax[kind][0] > 0 ? wmax[kind][0] : 1, h = wmax[kind][1] > 0 ? wmax[kind][1] : 1;
        return dim3(cdiv(w, 32), cdiv(h, 8), static_cast<unsigned>(obj.size()));
    }
    const LsWin *win(int kind) const { return d_win + static_cast<size_t>(kind) * kMaxObjects; }
};

int Sim::create(const incrmt_grid *gr, const incrmt_phys *ph) {
    if (gr->m < 8 || gr->n < 8 || !(gr->bx > gr->ax) || !(gr->by > gr->ay)) {
        set_error("bad grid %dx%d", gr->m, gr->n);
        return INCRMT_ERR_BADARG;
    }
    if ((gr->y_prd && (gr->n & 1)) || (gr->x_prd && (gr->m & 1))) {
        set_error("a periodic direction needs an even size (multigrid coarsening)");
        return INCRMT_ERR_BADARG;
    }
    const bool outlet = ph->zpr || ph->horiz_flow;
    if (gr->x_prd && (outlet || !gr->y_prd)) {
        // The zero-pressure outlet is the right edge; x periodicity comes only
        // with y periodicity, as in sim_velocity_pulses (sim_type.hh:99-101).
        set_error("an x-periodic domain must be periodic in y too and have no zero-pressure outlet");
        return INCRMT_ERR_BADARG;
    }
    if (gr->y_prd && !gr->x_prd && !outlet) {
        // Walls in x with y periodicity and no outlet: the reference's drivers
        // use y periodicity with walls in x only with sim_horiz_flow's outlet
        // (ftest.cc:362), and the projections were not shown to converge on
        // that singular combination.
        set_error("a y-periodic domain with walls in x needs the zero-pressure outlet (zpr or horiz_flow)");
        return INCRMT_ERR_BADARG;
    }
    INCRMT_CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    g.m = gr->m; g.n = gr->n; g.ml = g.m + 4; g.nl = g.n + 4;
    g.P = (g.ml + 31) / 32 * 32;
    g.xp = gr->x_prd ? 1 : 0;
    g.yp = gr->y_prd ? 1 : 0;
    g.pulses = ph->pulses ? 1 : 0;
    g.solid_prd = 0;  // incrmt_set_solid_prd_bc
    g.mf = g.xp ? g.m : g.m + 1; g.nf = g.yp ? g.n : g.n + 1;  // m_fem, n_fem (fluid_2d.cc:30-31)
    g.hflow = ph->horiz_flow ? 1 : 0;
    g.flow_u = ph->flow_u;
    g.zpr = (ph->zpr || g.hflow) ? 1 : 0;  // sim_horiz_flow::start sets zpr (sim_type.cc:59-64)
    g.ax = gr->ax; g.bx = gr->bx; g.ay = gr->ay; g.by = gr->by;
    g.dx = (g.bx - g.ax) / g.m; g.dy = (g.by - g.ay) / g.n;  // fluid_2d.cc:33-34
    g.xsp = 1 / g.dx; g.ysp = 1 / g.dy; g.xxsp = g.xsp * g.xsp; g.yysp = g.ysp * g.ysp;
    g.visc = ph->visc; g.rhof = ph->rhof;
    tw = ph->tw > 0 ? ph->tw : 2.5;
    pinw = ph->pinw > 0 ? ph->pinw : 2.5;
    g.eps = tw * (g.dx < g.dy ? g.dx : g.dy);
    g.epsinv = 1 / g.eps;
    g.w_scale = ph->w_scale > 0 ? ph->w_scale : 3.;   // sim_type.hh:13-16
    g.w_force = ph->w_force > 0 ? ph->w_force : 20.;
    if (ph->mg_rel_tol > 0) mgo.rel_tol = ph->mg_rel_tol;
    mgo.precision = ph->precision;
    ntrace = ph->ntrace > 0 ? ph->ntrace : 0;
    // Level-set grid (obj_field.cc:18): ghosted grid, origin at cell (-2,-2)'s centre.
    lg.mL = g.ml; lg.nL = g.nl; lg.P = g.P;
    lg.axl = g.ax - 1.5 * g.dx; lg.ayl = g.ay - 1.5 * g.dy;
    lg.dx = g.dx; lg.dy = g.dy; lg.xsp = 1 / g.dx; lg.ysp = 1 / g.dy;
    lg.phi_up = g.eps + 4.5 * g.dx; lg.phi_down = -g.eps - 4.5 * g.dx;
    double **fp[] = {&f.u, &f.v, &f.p, &f.rho, &f.ux, &f.uy, &f.vx, &f.vy, &f.ud, &f.vd, &f.ul, &f.vl,
                     &f.ur, &f.vr, &f.uu, &f.vu, &f.c0, &f.c1, &f.c2, &f.c3, &f.s11, &f.s12, &f.s21, &f.s22};
    for (double **q : fp) { int r = alloc(q, cells()); if (r) return r; }
    int r;
    if ((r = alloc(&src_mac, static_cast<size_t>(g.m) * g.n))) return r;
    if ((r = alloc(&z_mac, static_cast<size_t>(g.m) * g.n))) return r;
    if ((r = alloc(&src_fem, static_cast<size_t>(g.mf) * g.nf))) return r;
    if ((r = alloc(&z_fem, static_cast<size_t>(g.mf) * g.nf))) return r;
    if ((r = alloc(&partial, 4 * kB200SMs))) return r;
    INCRMT_CK(cudaMalloc(&d_lso, sizeof(LsObj) * kMaxObjects));
    {
        int dev = 0, sms = 0, nb = 0;
        INCRMT_CK(cudaGetDevice(&dev));
        INCRMT_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        // One block per SM: the grid barrier of the cooperative sweeps costs
        // more with more blocks, and the candidate lists are ~1e4-1e5 points.
        INCRMT_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ls_fim_coop, kFimThreads, 0));
        coop_blocks_fim = sms * (nb > 0 ? 1 : 0);
        INCRMT_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ls_extrap_coop, kExtrapThreads, 0));
        coop_blocks_ext = sms * (nb > 0 ? 1 : 0);
        if (coop_blocks_fim == 0 || coop_blocks_ext == 0) {
            set_error("level-set kernels cannot be co-resident");
            return INCRMT_ERR_CUDA;
        }
    }
    INCRMT_CK(cudaMalloc(&d_flags, sizeof(int) * 16));
    INCRMT_CK(cudaMemsetAsync(d_flags, 0, sizeof(int) * 16, stream));
    INCRMT_CK(cudaMallocHost(&h_flags, sizeof(int) * 16));
    INCRMT_CK(cudaMalloc(&d_lcnt, sizeof(unsigned long long) * 4));
    INCRMT_CK(cudaMemsetAsync(d_lcnt, 0, sizeof(unsigned long long) * 4, stream));
    INCRMT_CK(cudaMalloc(&d_win, sizeof(LsWin) * 4 * kMaxObjects));
    INCRMT_CK(cudaMallocHost(&h_win, sizeof(LsWin) * 4 * kMaxObjects));
    INCRMT_CK(cudaMalloc(&d_lsbox, sizeof(int) * 4 * kMaxObjects));
    INCRMT_CK(cudaMallocHost(&h_lsbox, sizeof(int) * 4 * kMaxObjects));
    ntx = ((g.m + 1 + 32) >> 5) + 1;
    nty = ((g.n + 1 + 8) >> 3) + 1;
    if (ntrace > 0 && (r = alloc(&tm, 4 * static_cast<size_t>(ntrace)))) return r;
    if (ntrace > 0) INCRMT_CK(cudaMalloc(&d_remap, sizeof(int) * ntrace));
    if ((r = mac.create(INCRMT_SYS_MAC, g.m, g.n, g.ax, g.bx, g.ay, g.by, g.xp, g.yp, g.zpr, stream))) return r;
    if ((r = fem.create(INCRMT_SYS_FEM, g.m, g.n, g.ax, g.bx, g.ay, g.by, g.xp, g.yp, g.zpr, stream))) return r;
    return INCRMT_OK;
}

int Sim::add_object(const incrmt_object_desc *d) {
    if (initialized) { set_error("objects must be added before initialize"); return INCRMT_ERR_BADARG; }
    if (static_cast<int>(obj.size()) >= kMaxObjects) { set_error("too many objects"); return INCRMT_ERR_BADARG; }
    if (d->type < INCRMT_OBJ_SIMPLE_SPIN || d->type > INCRMT_OBJ_HOOP) {
        set_error("unknown object type %d", d->type);
        return INCRMT_ERR_BADARG;
    }
    ObjDev o{};
    o.type = d->type == INCRMT_OBJ_SIMPLE_SPIN   ? OBJ_SIMPLE_SPIN
             : d->type == INCRMT_OBJ_CIRCLE      ? OBJ_CIRCLE
             : d->type == INCRMT_OBJ_ROUNDED_ROD ? OBJ_ROUNDED_ROD
             : d->type == INCRMT_OBJ_ELLIPSE     ? OBJ_ELLIPSE
             : d->type == INCRMT_OBJ_SQUARE      ? OBJ_SQUARE
             : d->type == INCRMT_OBJ_SEVEN_POINT ? OBJ_SEVEN_POINT
             : d->type == INCRMT_OBJ_FLAPPER     ? OBJ_FLAPPER
             : d->type == INCRMT_OBJ_PISTON      ? OBJ_PISTON
             : d->type == INCRMT_OBJ_CIRCLE_TRACK ? OBJ_CIRCLE
             : d->type == INCRMT_OBJ_FULL        ? OBJ_FULL
             : d->type == INCRMT_OBJ_TRIANGLE    ? OBJ_TRIANGLE
             : d->type == INCRMT_OBJ_LAMPREY     ? OBJ_LAMPREY
             : d->type == INCRMT_OBJ_HOOP        ? OBJ_HOOP
                                                 : OBJ_FLAG;
    o.set_velocity = d->set_velocity;
    o.G = d->G; o.rhos = d->rhos; o.ev_trans_mult = d->ev_trans_mult;
    o.eps = g.eps; o.pinw = pinw * g.dx;  // obj_field.cc:16
    o.tf1 = 0.5 / g.eps; o.tf2 = 0.5 / M_PI; o.tf3 = M_PI / g.eps;
    const double *p = d->params;
    if (o.type == OBJ_SIMPLE_SPIN) {
        // obj_simple_spin(r_scale,a1,a2,piv_r,th_max,omega) (object.hh:447-453)
        const double scf = p[0] / (1 + p[1] + p[2]);
        o.g[0] = scf * (1 - p[2]); o.g[1] = scf * p[1]; o.g[2] = 2 * scf * p[2];
        o.g[3] = p[3]; o.g[4] = p[4]; o.g[5] = p[5];
    } else if (d->type == INCRMT_OBJ_CIRCLE_TRACK) {
        // obj_circle_track(cx,cy,cr,uu,vv,omega) (object.hh:526-527): a circle
        // without gravity whose tracked points are set up at initialize
        o.g[0] = p[0]; o.g[1] = p[1]; o.g[2] = p[2]; o.g[3] = 0;
        o.g[4] = p[3]; o.g[5] = p[4]; o.g[6] = p[5];
    } else if (o.type == OBJ_SEVEN_POINT) {
        // obj_seven_point(cx,cy,cr,piv_r,th_max,omega) (object.hh:192-194)
        for (int k = 0; k < 6; k++) o.g[k] = p[k];
    } else if (o.type == OBJ_FLAPPER) {
        // obj_flapper(cx,cy,cr,cl,ar,al,theta,m_stretch,T) (object.hh:263-267)
        if (!(p[4] > 0) || !(p[7] > 0) || !(p[8] > 0)) {
            set_error("flapper needs ar > 0, m_stretch > 0, T > 0");
            return INCRMT_ERR_BADARG;
        }
        o.g[0] = p[0]; o.g[1] = p[1]; o.g[2] = p[2]; o.g[3] = 0;
        o.g[4] = cos(p[6]); o.g[5] = sin(p[6]); o.g[7] = p[3]; o.g[8] = p[4]; o.g[9] = p[5];
        o.g[10] = log(p[7]) / p[4];
        o.g[11] = 2 * M_PI / p[8];
    } else if (o.type == OBJ_PISTON) {
        // obj_piston(lx,ly,cx,y_start,y_end,duration,anch_r) (object.hh:390-401)
        if (!(p[5] > 0)) { set_error("piston needs a positive duration"); return INCRMT_ERR_BADARG; }
        o.g[0] = 0; o.g[1] = p[3]; o.g[2] = p[0]; o.g[4] = 1. / p[5]; o.g[5] = p[6];
        o.g[7] = p[1]; o.g[8] = p[2]; o.g[9] = p[4] - p[3];
    } else if (o.type == OBJ_CIRCLE || o.type == OBJ_SQUARE) {
        // obj_circle / obj_square(cx,cy,cr,uu,vv,omega,grav) (object.hh:128-152)
        o.g[0] = p[0]; o.g[1] = p[1]; o.g[2] = p[2]; o.g[3] = p[6];
        o.g[4] = p[3]; o.g[5] = p[4]; o.g[6] = p[5];
    } else if (o.type == OBJ_ROUNDED_ROD) {
        // obj_rounded_rod(cx,cy,cr,cl,grav) (object.hh:229-230); at rest initially
        if (!(p[2] > 0) || !(p[3] >= 0)) { set_error("rounded rod needs cr > 0, cl >= 0"); return INCRMT_ERR_BADARG; }
        o.g[0] = p[0]; o.g[1] = p[1]; o.g[2] = p[2]; o.g[3] = p[4]; o.g[7] = p[3];
    } else if (o.type == OBJ_FULL) {
        // obj_full() (object.hh:83-86): no parameters
    } else if (o.type == OBJ_TRIANGLE) {
        // obj_triangle(cx,cy,cr,theta,grav) (object.cc:52-58): an equilateral
        // triangle whose side normals point at theta + 2 pi k / 3, at rest
        o.g[0] = p[0]; o.g[1] = p[1]; o.g[2] = p[2] * 0.5; o.g[3] = p[4];
        double nor[6];
        for (int i = 0; i < 3; i++) {
            nor[2 * i] = cos(p[3] + 2 * M_PI / 3 * i);
            nor[2 * i + 1] = sin(p[3] + 2 * M_PI / 3 * i);
        }
        o.g[8] = nor[0]; o.g[9] = nor[1]; o.g[10] = nor[2]; o.g[11] = nor[3];
        o.nor2[0] = nor[4]; o.nor2[1] = nor[5];
    } else if (o.type == OBJ_LAMPREY) {
        // obj_lamprey(cx,cy,theta,le,dis,w1,w2,T,mlam) (object.hh:568-571)
        if (!(p[7] > 0) || !(p[8] > 0) || !(p[5] > 0) || !(p[3] > p[4])) {
            set_error("lamprey needs T > 0, mlam > 0, w1 > 0 and le > dis");
            return INCRMT_ERR_BADARG;
        }
        o.g[0] = p[0]; o.g[1] = p[1]; o.g[2] = p[4]; o.g[3] = p[3] - p[4];
        o.g[4] = cos(p[2]); o.g[5] = sin(p[2]); o.g[6] = p[5]; o.g[7] = p[6]; o.g[8] = p[7];
        o.g[9] = log(p[8]);
    } else if (o.type == OBJ_HOOP) {
        // obj_hoop(r_in,r_out,grav) (object.hh:608-609): centred on the
        // origin; its grav is stored but never applied (no accel override)
        if (!(p[1] > p[0])) { set_error("hoop needs r_out > r_in"); return INCRMT_ERR_BADARG; }
        o.g[2] = (p[1] - p[0]) * 0.5; o.g[7] = 0.5 * (p[0] + p[1]);
    } else if (o.type == OBJ_FLAG) {
        // obj_flag(cx,cy,flag_l,flag_w,flag_a,perturb_v,ntrace) (object.cc:420-441)
        if (!(p[2] > 0) || !(p[3] > 0) || !(p[4] >= 0)) { set_error("flag needs positive length and width"); return INCRMT_ERR_BADARG; }
        if (p[4] >= 0.5 * p[3]) {
            set_error("flag_a should be smaller than 0.5*flag_w to avoid cutting off its influence");
            return INCRMT_ERR_BADARG;
        }
        if (!(p[6] >= 1) || p[6] > 4096) { set_error("flag needs 1..4096 tracked points"); return INCRMT_ERR_BADARG; }
        o.g[0] = p[0]; o.g[1] = p[1]; o.g[2] = p[2]; o.g[7] = p[3]; o.g[8] = p[4]; o.g[9] = p[5];
    } else {
        // ellipse (cx,cy,a,b,theta,grav); at rest initially
        if (!(p[2] > 0) || !(p[3] > 0)) { set_error("ellipse needs positive semi-axes"); return INCRMT_ERR_BADARG; }
        o.g[0] = p[0]; o.g[1] = p[1]; o.g[2] = p[2]; o.g[3] = p[5]; o.g[7] = p[3];
        o.g[8] = cos(p[4]); o.g[9] = sin(p[4]);
    }
    SolidDev s{};
    double **sp[] = {&s.X, &s.Y, &s.nX, &s.nY, &s.Xx, &s.Xy, &s.Yx, &s.Yy, &s.Xd, &s.Yd, &s.Xl, &s.Yl,
                     &s.Xr, &s.Yr, &s.Xu, &s.Yu, &s.phi, &s.phi_tmp};
    for (double **q : sp) { int r = alloc(q, cells()); if (r) return r; }
    INCRMT_CK(cudaMalloc(&s.s, sizeof(int) * cells()));
    INCRMT_CK(cudaMemsetAsync(s.s, 0, sizeof(int) * cells(), stream));
    LsObj l{};
    l.phi = s.phi; l.s = s.s; l.phi_new = s.phi_tmp; l.nX = s.nX; l.nY = s.nY;
    for (double **q : {&l.a, &l.b, &l.c, &l.d}) { int r = alloc(q, cells()); if (r) return r; }
    void *raw = nullptr;
    INCRMT_CK(cudaMalloc(&raw, 2 * cells() + 2 * sizeof(int) * cells()));
    raw_allocs.push_back(raw);
    INCRMT_CK(cudaMemsetAsync(raw, 0, 2 * cells() + 2 * sizeof(int) * cells(), stream));
    l.ia = static_cast<int *>(raw);
    l.ib = l.ia + cells();
    l.ca = reinterpret_cast<unsigned char *>(l.ib + cells());
    l.cb = l.ca + cells();
    lso.push_back(l);
    obj.push_back(o);
    sol.push_back(s);
    desc.push_back(*d);
    return INCRMT_OK;
}

int Sim::upload_objects() {
    if (!d_obj) {
        INCRMT_CK(cudaMalloc(&d_obj, sizeof(ObjDev) * kMaxObjects));
        INCRMT_CK(cudaMalloc(&d_sol, sizeof(SolidDev) * kMaxObjects));
    }
    if (obj.empty()) return INCRMT_OK;
    INCRMT_CK(cudaMemcpyAsync(d_obj, obj.data(), sizeof(ObjDev) * obj.size(), cudaMemcpyHostToDevice, stream));
    INCRMT_CK(cudaMemcpyAsync(d_sol, sol.data(), sizeof(SolidDev) * sol.size(), cudaMemcpyHostToDevice, stream));
    INCRMT_CK(cudaMemcpyAsync(d_lso, lso.data(), sizeof(LsObj) * lso.size(), cudaMemcpyHostToDevice, stream));
    // Room for every point of every object in the combined level-set list.
    const size_t need = cells() * obj.size();
    if (need > static_cast<size_t>(list_cap)) {
        if (need > 0x7fffffffu) { set_error("level-set point list too large"); return INCRMT_ERR_BADARG; }
        cudaFree(d_list);
        cudaFree(d_list_k);
        d_list = d_list_k = nullptr;
        list_cap = 0;
        INCRMT_CK(cudaMalloc(&d_list, sizeof(int) * need));
        INCRMT_CK(cudaMalloc(&d_list_k, sizeof(int) * need));
        list_cap = static_cast<int>(need);
    }
    return INCRMT_OK;
}

/** Per-object state before a stress evaluation (object::pre_stress_setup;
 * obj_simple_spin, object.cc:185-188). */
void Sim::pre_stress_setup(double t) {
    for (auto &o : obj) {
        if (o.type == OBJ_SIMPLE_SPIN) {
            double ang = t * o.g[5], theta = ang > 2 * M_PI ? 0 : o.g[4] * (1 - cos(ang));
            o.cth = cos(theta);
            o.sth = sin(theta);
        } else if (o.type == OBJ_SEVEN_POINT) {  // object.cc:128-131
            double theta = o.g[4] * (1 - cos(t * o.g[5]));
            o.cth = cos(theta);
            o.sth = sin(theta);
        } else if (o.type == OBJ_FLAPPER) {  // object.cc:291-295
            double a = sin(o.g[11] * t);
            a *= a * a;
            a *= a;
            a *= a;
            o.act = -o.g[10] * a;
        } else if (o.type == OBJ_PISTON) {  // object.cc:250-253
            t *= o.g[4];
            o.act = o.g[1] + (t >= 1 ? o.g[9] : o.g[9] * t * t * (3 - 2 * t));
        } else if (o.type == OBJ_LAMPREY) {  // object.cc:563-568
            double sh = t / o.g[8], a = 2 * sh;
            o.act = a < 1 ? o.g[9] * a * a * (3 - 2 * a) : o.g[9];
            o.shift = sh * o.g[3];
        }
    }
}

int Sim::fetch_flags() {
    INCRMT_CK(cudaMemcpyAsync(h_flags, d_flags, sizeof(int) * 16, cudaMemcpyDeviceToHost, stream));
    INCRMT_CK(cudaStreamSynchronize(stream));
    return INCRMT_OK;
}

/** Windows of every kind set to the whole grid; objects are visited
 * everywhere until the next rebuild, and the next reference-map commit covers
 * the whole grid. Used before the first rebuild and after a state upload. */
int Sim::win_reset() {
    INCRMT_CK(cudaStreamSynchronize(stream));  // h_win may still feed an earlier copy
    win_valid = false;
    x_synced = false;
    pref_valid = false;
    const LsWin full{0, 0, g.ml, g.nl};
    for (int kind = 0; kind < 4; kind++) {
        for (int k = 0; k < kMaxObjects; k++) h_win[kind * kMaxObjects + k] = full;
        wmax[kind][0] = g.ml;
        wmax[kind][1] = g.nl;
    }
    INCRMT_CK(cudaMemcpyAsync(d_win, h_win, sizeof(LsWin) * 4 * kMaxObjects, cudaMemcpyHostToDevice, stream));
    return INCRMT_OK;
}

/** New rebuild and presence windows from the boxes of the rebuild that just
 * ran (h_lsbox, fetched with its flags), and the tile object lists. Called
 * after that rebuild's last kernel is queued: the uploads follow it on the
 * stream. The windows stay the whole grid when they are switched off, or
 * when the pinning width reaches the band limit (pin would then rewrite far
 * points). */
int Sim::win_update() {
    const int no = static_cast<int>(obj.size());
    if (!win_enable || no == 0 || !(obj[0].pinw < lg.phi_up)) return INCRMT_OK;
    const int R = static_cast<int>(std::ceil((lg.phi_up) / (g.dx < g.dy ? g.dx : g.dy))) + 2;
    auto grow = [&](const int *b, int e) {
        if (b[0] >= 0x7f7f7f7f) return LsWin{0, 0, 0, 0};  // no point inside or at the interface
        LsWin w{b[0] - e, b[1] - e, -b[2] + e + 1, -b[3] + e + 1};
        w.x0 = w.x0 < 0 ? 0 : w.x0 & ~31;  // rows of 32 start on a 256-byte boundary
        w.y0 = w.y0 < 0 ? 0 : w.y0;
        w.x1 = w.x1 > g.ml ? g.ml : w.x1;
        w.y1 = w.y1 > g.nl ? g.nl : w.y1;
        return w;
    };
    for (int kind = 0; kind < 2; kind++) wmax[kind][0] = wmax[kind][1] = 0;
    LsWin *wl = h_win, *wp = h_win + kMaxObjects;
    size_t entries = 0;
    for (int k = 0; k < no; k++) {
        wl[k] = grow(h_lsbox + 4 * k, 2 * R + 4);
        wp[k] = grow(h_lsbox + 4 * k, R + 3);
        // Under y periodicity the Godunov pass of the last row writes the
        // bottom edges of row 0: a window near either end spans the height
        // (and likewise the width under x periodicity).
        if (g.yp && wp[k].y1 > wp[k].y0 && (wp[k].y0 <= 3 || wp[k].y1 >= g.nl - 3)) {
            wp[k].y0 = 0;
            wp[k].y1 = g.nl;
        }
        if (g.xp && wp[k].x1 > wp[k].x0 && (wp[k].x0 <= 3 || wp[k].x1 >= g.ml - 3)) {
            wp[k].x0 = 0;
            wp[k].x1 = g.ml;
        }
        for (int kind = 0; kind < 2; kind++) {
            const LsWin &w = h_win[kind * kMaxObjects + k];
            if (w.x1 - w.x0 > wmax[kind][0]) wmax[kind][0] = w.x1 - w.x0;
            if (w.y1 - w.y0 > wmax[kind][1]) wmax[kind][1] = w.y1 - w.y0;
        }
        if (wp[k].x1 > wp[k].x0 && wp[k].y1 > wp[k].y0)
            entries += static_cast<size_t>(((wp[k].x1 + 29) >> 5) - ((wp[k].x0 + 30) >> 5) + 1) *
                       (((wp[k].y1 + 5) >> 3) - ((wp[k].y0 + 6) >> 3) + 1);
    }
    // Tile lists: tile (tx,ty) holds cells 32(tx-1) <= i < 32tx,
    // 8(ty-1) <= j < 8ty; level-set point li is cell li-2.
    const size_t ntiles = static_cast<size_t>(ntx) * nty, need = ntiles + 1 + entries;
    if (need > tiles_cap) {
        cudaFreeHost(h_tiles);
        cudaFree(d_tiles);
        h_tiles = nullptr;
        d_tiles = nullptr;
        tiles_cap = 0;
        INCRMT_CK(cudaMallocHost(&h_tiles, sizeof(int) * need));
        INCRMT_CK(cudaMalloc(&d_tiles, sizeof(int) * need));
        tiles_cap = need;
    }
    int *start = h_tiles, *list = h_tiles + ntiles + 1;
    std::fill(start, start + ntiles + 1, 0);
    auto each_tile = [&](const LsWin &w, auto &&fn) {
        if (w.x1 <= w.x0 || w.y1 <= w.y0) return;
        const int tx0 = (w.x0 + 30) >> 5, tx1 = (w.x1 + 29) >> 5, ty0 = (w.y0 + 6) >> 3, ty1 = (w.y1 + 5) >> 3;
        for (int ty = ty0; ty <= ty1; ty++)
            for (int tx = tx0; tx <= tx1; tx++) fn(static_cast<size_t>(ty) * ntx + tx);
    };
    for (int k = 0; k < no; k++) each_tile(wp[k], [&](size_t t) { start[t + 1]++; });
    for (size_t t = 0; t < ntiles; t++) start[t + 1] += start[t];
    std::vector<int> fill(start, start + ntiles);
    for (int k = 0; k < no; k++) each_tile(wp[k], [&](size_t t) { list[fill[t]++] = k; });
    INCRMT_CK(cudaMemcpyAsync(d_win, h_win, sizeof(LsWin) * 2 * kMaxObjects, cudaMemcpyHostToDevice, stream));
    INCRMT_CK(cudaMemcpyAsync(d_tiles, h_tiles, sizeof(int) * need, cudaMemcpyHostToDevice, stream));
    win_valid = true;
    return INCRMT_OK;
}

int Sim::compute_stress() {
    pre_stress_setup(time);
    int r = upload_objects();
    if (r) return r;
    k_stress<<<g2(g.m + 1, g.n + 1), kB2, 0, stream>>>(g, f, d_obj, d_sol, tiles());
    launches++;
    INCRMT_CKL("k_stress");
    return INCRMT_OK;
}

int Sim::set_boundaries() {
    if (g.solid_prd && !obj.empty()) {  // fluid_2d::set_boundaries (fluid_2d.cc:690)
        k_set_boundaries_solid<<<1, 1024, 0, stream>>>(g, d_sol, static_cast<int>(obj.size()));
        launches++;
        INCRMT_CKL("k_set_boundaries_solid");
    }
    k_set_boundaries<<<1, 1024, 0, stream>>>(g, f);
    launches++;
    INCRMT_CKL("k_set_boundaries");
    return INCRMT_OK;
}

int Sim::set_rho() {
    k_set_rho<<<g2(g.ml, g.nl), kB2, 0, stream>>>(g, f, d_obj, d_sol, tiles());
    launches++;
    INCRMT_CKL("k_set_rho");
    return INCRMT_OK;
}

/** levelset::build_band for every object (levelset.cc:199-335): each kernel
 * runs over all objects at once (blockIdx.z), each over its rebuild window,
 * and one cooperative launch settles every object's march, the objects being
 * independent. The sign scan also records each object's box, from which the
 * next windows follow. */
int Sim::build_bands() {
    const int no = static_cast<int>(obj.size());
    if (no == 0) return INCRMT_OK;
    INCRMT_CK(cudaMemsetAsync(d_flags, 0, sizeof(int) * 13, stream));
    INCRMT_CK(cudaMemsetAsync(d_lsbox, 0x7f, sizeof(int) * 4 * no, stream));
    const dim3 gg = wgrid(0);
    const LsWin *wl = win(0);
    k_ls_scan<<<gg, kB2, 0, stream>>>(lg, d_lso, wl, d_lsbox);
    k_ls_newton<<<gg, kB2, 0, stream>>>(lg, d_lso, wl, d_flags + 6);
    k_ls_copy_interface<<<gg, kB2, 0, stream>>>(lg, d_lso, wl);
    // Candidates: far points within the band radius of the interface.
    const int R = static_cast<int>(std::ceil((lg.phi_up) / (g.dx < g.dy ? g.dx : g.dy))) + 2;
    k_ls_mark_interface<<<gg, kB2, 0, stream>>>(lg, d_lso, wl);
    k_ls_dilate<true><<<gg, kB2, 0, stream>>>(lg, d_lso, wl, R);
    k_ls_dilate<false><<<gg, kB2, 0, stream>>>(lg, d_lso, wl, R);
    k_ls_collect_candidates<<<gg, kB2, 0, stream>>>(lg, d_lso, wl, d_list, d_list_k, d_flags + 7, list_cap,
                                                    d_flags + 10);
    k_ls_fim_init<<<gg, kB2, 0, stream>>>(lg, d_lso, wl);
    launches += 8;
    INCRMT_CKL("level-set scan/newton/candidates");
    int maxs = kLsMaxSweeps, cap = list_cap;
    const int *countp = d_flags + 7;
    const LsObj *ob = d_lso;
    void *args[] = {&lg, &ob, &d_list, &d_list_k, &countp, &cap, &d_flags, &maxs};
    INCRMT_CK(cudaLaunchCooperativeKernel(reinterpret_cast<void *>(k_ls_fim_coop), dim3(coop_blocks_fim), dim3(kFimThreads),
                                          args, 0, stream));
    launches++;
    INCRMT_CK(cudaMemcpyAsync(h_lsbox, d_lsbox, sizeof(int) * 4 * no, cudaMemcpyDeviceToHost, stream));
    int r = fetch_flags();
    if (r) return r;
    if (h_flags[6]) { set_error("level++: Newton iteration failed."); return h_flags[6]; }
    if (h_flags[10]) { set_error("level-set candidate list overflow"); return INCRMT_ERR_BADARG; }
    ls_sweeps += h_flags[3];
    if (h_flags[12]) ls_monotone++;
    if (!h_flags[4]) { set_error("level-set march did not settle in %d sweeps", h_flags[3]); return INCRMT_ERR_NOCONV; }
    k_ls_finish<<<gg, kB2, 0, stream>>>(lg, d_lso, wl);
    k_ls_trial<<<gg, kB2, 0, stream>>>(lg, d_lso, wl);
    k_ls_store_status<<<gg, kB2, 0, stream>>>(lg, d_lso, wl);
    launches += 3;
    INCRMT_CKL("k_ls_finish");
    return win_update();
}

/** obj_field::pin for every object, then set_rho (fluid_2d::pin,
 * fluid_2d.cc:373-377). */
int Sim::pin() {
    int r;
    if (!obj.empty()) {
        k_pin<<<wgrid(1), kB2, 0, stream>>>(g, d_obj, d_sol, win(1));
        launches++;
        INCRMT_CKL("k_pin");
    }
    if ((r = build_bands())) return r;
    return const_rho ? INCRMT_OK : set_rho();
}

/** levelset::extrapolate_fields for every object (traverse.hh:235-260),
 * the objects' wavefronts settling together in one cooperative launch. */
int Sim::extrapolate_all() {
    const int no = static_cast<int>(obj.size());
    if (no == 0) return INCRMT_OK;
    INCRMT_CK(cudaMemsetAsync(d_flags, 0, sizeof(int) * 11, stream));
    k_ls_collect_outside<<<wgrid(1), kB2, 0, stream>>>(lg, d_lso, win(1), d_list, d_list_k, d_flags + 7,
                                                       list_cap, d_flags + 10);
    k_ls_extrap_init<<<4 * kB200SMs, 256, 0, stream>>>(d_lso, d_list, d_list_k, d_flags + 7, list_cap);
    launches += 2;
    INCRMT_CKL("collect");
    int maxs = kExtrapMaxSweeps, cap = list_cap;
    const int *countp = d_flags + 7;
    const LsObj *ob = d_lso;
    void *args[] = {&lg, &ob, &d_list, &d_list_k, &countp, &cap, &d_flags, &maxs};
    INCRMT_CK(cudaLaunchCooperativeKernel(reinterpret_cast<void *>(k_ls_extrap_coop), dim3(coop_blocks_ext),
                                          dim3(kExtrapThreads), args, 0, stream));
    launches++;
    int r = fetch_flags();
    if (r) return r;
    if (h_flags[5]) { set_error("singular extrapolation fit"); return h_flags[5]; }
    if (h_flags[10]) { set_error("extrapolation list overflow"); return INCRMT_ERR_BADARG; }
    ex_sweeps += h_flags[3];
    if (!h_flags[4]) { set_error("extrapolation did not settle in %d sweeps", h_flags[3]); return INCRMT_ERR_NOCONV; }
    // After the last sweep both buffers hold the same values.
    k_ls_extrap_store<<<4 * kB200SMs, 256, 0, stream>>>(d_lso, d_list, d_list_k, d_flags + 7, list_cap);
    launches++;
    INCRMT_CKL("k_ls_extrap_store");
    return INCRMT_OK;
}

/** fluid_2d::update_reference_map (fluid_2d.cc:1242-1273), every object
 * over its presence window, which is recorded for the commit in
 * update_velocity. */
int Sim::update_reference_map(double dt) {
    const int no = static_cast<int>(obj.size());
    if (no > 0) {
        k_refmap_update<<<wgrid(1), kB2, 0, stream>>>(g, f, d_sol, win(1), dt);
        launches++;
        INCRMT_CKL("k_refmap_update");
        INCRMT_CK(cudaMemcpyAsync(d_win + 2 * kMaxObjects, win(1), sizeof(LsWin) * no, cudaMemcpyDeviceToDevice,
                                  stream));
        wmax[2][0] = wmax[1][0];
        wmax[2][1] = wmax[1][1];
        pref_valid = true;
    }
    int r, outer = cur_phase;
    if ((r = phase_end())) return r;
    if ((r = phase_begin(INCRMT_PHASE_EXTRAP))) return r;
    if ((r = extrapolate_all())) return r;
    if ((r = phase_end())) return r;
    if ((r = phase_begin(outer))) return r;
    if (no > 0) {
        k_refmap_half<<<wgrid(1), kB2, 0, stream>>>(g, d_sol, win(1));
        launches++;
        INCRMT_CKL("k_refmap_half");
    }
    return INCRMT_OK;
}

/** The extrapolated start of order `order` at one unknown (0: z, 1:
 * 2 z - zo, 2: 3 (z - zo) + zo2). */
__device__ __forceinline__ double extrapolated(int order, double v, double o, const double *zo2, long q) {
    if (order == 1) return __dsub_rn(2.0 * v, o);
    if (order == 2) return __dadd_rn(3.0 * __dsub_rn(v, o), zo2[q]);
    return v;
}

/** Block sums of the extrapolation's increment (extrapolated - z). */
__global__ void k_extrapolate_increment(const double *z, const double *zo, const double *zo2, long N, int order,
                                        double *partial) {
    double acc = 0;
    for (long q = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; q < N;
         q += static_cast<long>(gridDim.x) * blockDim.x) {
        const double v = z[q];
        acc += __dsub_rn(extrapolated(order, v, zo[q], zo2, q), v);
    }
    acc = block_sum_256(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

/** The extrapolated start, less the mean of its increment when `isum` (the
 * sum of the increments) is given, and the history shifted: zo2 = zo (zo2
 * not null), zo = the old z. */
__global__ void k_extrapolate_guess(double *z, double *zo, double *zo2, long N, int order, const double *isum) {
    const double shift = isum ? *isum / static_cast<double>(N) : 0.0;
    for (long q = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; q < N;
         q += static_cast<long>(gridDim.x) * blockDim.x) {
        const double v = z[q], o = zo[q];
        if (order) z[q] = __dsub_rn(extrapolated(order, v, o, zo2, q), shift);
        if (zo2) zo2[q] = o;
        zo[q] = v;
    }
}

/** The extrapolated warm start of a projection (guess 1): from the third
 * solve on, z(n-1) becomes 2 z(n-1) - z(n-2), a second-order prediction of
 * a pressure that varies smoothly in time; the solve then reaches the same
 * relative residual from a closer start. Guess 2 uses the quadratic
 * 3 z(n-1) - 3 z(n-2) + z(n-3) from the fourth solve on (linear for the
 * third). The first two solves keep the previous solution, as the reference
 * does always (fluid_2d.cc:1175-1236, 1297-1328 solve from the pressure
 * left in place). */
int Sim::extrapolate_guess(int sys, double *z) {
    if (!guess) return INCRMT_OK;
    const long N = sys == INCRMT_SYS_MAC ? static_cast<long>(g.m) * g.n : static_cast<long>(g.mf) * g.nf;
    if (!zold[sys]) {
        int r = alloc(&zold[sys], static_cast<size_t>(N));
        if (r) return r;
    }
    if (guess == 2 && !zold2[sys]) {
        int r = alloc(&zold2[sys], static_cast<size_t>(N));
        if (r) return r;
    }
    const int order = guess == 2 && nsol[sys] >= 3 ? 2 : nsol[sys] >= 2 ? 1 : 0;
    const int nb = cdiv(N, 256) < 4 * kB200SMs ? cdiv(N, 256) : 4 * kB200SMs;
    double *zo2 = guess == 2 ? zold2[sys] : nullptr;
    // Without a Dirichlet condition (no zero-pressure column) the system is
    // singular and its solutions differ by constants, which the solves
    // neither fix nor use. Extrapolated, a constant drift between steps would
    // grow without bound (quadratically for the quadratic start) until the
    // residual drowns in the rounding of a huge constant; the increment's
    // mean is therefore removed.
    const double *isum = nullptr;
    if (order && !g.zpr) {
        // partial holds 4 x kB200SMs doubles: block sums, then their total
        const int nbs = nb < 2 * kB200SMs ? nb : 2 * kB200SMs;
        k_extrapolate_increment<<<nbs, 256, 0, stream>>>(z, zold[sys], zo2, N, order, partial);
        k_reduce_partials<<<1, 256, 0, stream>>>(partial, nbs, partial + nbs);
        launches += 2;
        isum = partial + nbs;
    }
    k_extrapolate_guess<<<nb, 256, 0, stream>>>(z, zold[sys], zo2, N, order, isum);
    launches++;
    INCRMT_CKL("k_extrapolate_guess");
    return INCRMT_OK;
}

/** fluid_2d::mac_projection (fluid_2d.cc:1175-1236). */
int Sim::mac_projection() {
    k_mac_source<<<g2(g.m, g.n), kB2, 0, stream>>>(g, f, src_mac);
    launches++;
    INCRMT_CKL("k_mac_source");
    int outer = cur_phase, r;
    if ((r = phase_end())) return r;
    if ((r = phase_begin(INCRMT_PHASE_MG_SETUP))) return r;
    r = const_rho ? INCRMT_OK : mac.set_density_lagged(f.rho, g.P);
    if (r) return r;
    if ((r = phase_end())) return r;
    if ((r = phase_begin(outer))) return r;
    incrmt_mg_stats st{};
    long long l0 = mac.launches;
    if ((r = extrapolate_guess(INCRMT_SYS_MAC, z_mac))) return r;
    if ((r = learned_pre(INCRMT_SYS_MAC, src_mac, z_mac))) return r;
    r = const_rho ? mac.solve_device(src_mac, z_mac, &mgo, &st, false) : mac.solve_lagged(src_mac, z_mac, &mgo, &st, false);
    if (!r) r = learned_post(INCRMT_SYS_MAC, z_mac);
    if (!r) nsol[INCRMT_SYS_MAC]++;
    launches += mac.launches - l0;
    vc_mac += st.vcycles;
    solves_mac++;
    if (r) return r;
    k_mac_correct<<<g2(g.m, g.n), kB2, 0, stream>>>(g, f, z_mac, mac.ex, mac.ey);
    launches++;
    INCRMT_CKL("k_mac_correct");
    return INCRMT_OK;
}

/** fluid_2d::finite_element_projection + copy_pressure
 * (fluid_2d.cc:1297-1328). */
/** Before a projection's solve: a training capture (the network input of
 * the warm start, which is kept), or the learned guess applied to the warm
 * start, counted as applied or fallen back in d_lcnt. */
int Sim::learned_pre(int sys, const double *b, double *z) {
    Learned &L = learn[sys];
    Multigrid &mg = sys == INCRMT_SYS_MAC ? mac : fem;
    if (L.cap > 0 && L.captured < L.cap) {
        int H, W;
        learned_grid(mg.m, mg.n, L.cap_factor, H, W);
        const long N = static_cast<long>(mg.m) * mg.n;
        if (L.z0_n < N) {
            cudaFree(L.z0);
            L.z0 = nullptr;
            L.z0_n = 0;
            INCRMT_CK(cudaMalloc(&L.z0, sizeof(double) * N));
            L.z0_n = N;
        }
        INCRMT_CK(cudaMemcpyAsync(L.z0, z, sizeof(double) * N, cudaMemcpyDeviceToDevice, stream));
        int r = learned_input(mg, L.w, b, z, L.cap_factor, H, W);
        if (r) return r;
        INCRMT_CK(cudaMemcpyAsync(L.cap_in + static_cast<size_t>(L.captured) * H * W * 3, L.w.in,
                                  sizeof(float) * H * W * 3, cudaMemcpyDeviceToDevice, stream));
        return INCRMT_OK;
    }
    if (!L.net) return INCRMT_OK;
    if (L.skip > 0) {
        L.skip--;
        L.skipped++;
        return INCRMT_OK;
    }
    L.ran = true;
    unsigned long long *cnt = d_lcnt + 2 * sys;
    if (L.gexec && L.gkey_net == L.net && L.gkey_gen == unet_generation(L.net) && L.gkey_b == b && L.gkey_z == z) {
        INCRMT_CK(cudaGraphLaunch(L.gexec, stream));
        mg.launches += L.glaunches;
        return INCRMT_OK;
    }
    // A guess runs directly while the network's buffers may still be
    // (re)allocated for this grid: the first one, and the first after the
    // network was used at another size; the next one is captured (nothing is
    // allocated then) and replayed from then on.
    if (L.gfail || L.warm_net != L.net || L.warm_gen != unet_generation(L.net)) {
        const int rd = learned_guess(mg, L.w, L.net, b, z, L.factor, L.rule, cnt);
        L.warm_net = L.net;
        L.warm_gen = unet_generation(L.net);
        return rd;
    }
    L.release_graph();
    const long long l0 = mg.launches;
    INCRMT_CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    int rc = learned_guess(mg, L.w, L.net, b, z, L.factor, L.rule, cnt);
    cudaGraph_t graph = nullptr;
    cudaError_t ce = cudaStreamEndCapture(stream, &graph);
    if (rc == INCRMT_OK && ce == cudaSuccess) {
        ce = cudaGraphInstantiate(&L.gexec, graph, 0);
        if (ce != cudaSuccess) L.gexec = nullptr;
    }
    if (graph) cudaGraphDestroy(graph);
    if (rc != INCRMT_OK || ce != cudaSuccess || !L.gexec) {
        // not capturable here: run the guess directly from now on
        cudaGetLastError();
        L.release_graph();
        L.gfail = true;
        mg.launches = l0;
        return learned_guess(mg, L.w, L.net, b, z, L.factor, L.rule, cnt);
    }
    L.gkey_net = L.net;
    L.gkey_gen = unet_generation(L.net);
    L.gkey_b = b;
    L.gkey_z = z;
    L.glaunches = mg.launches - l0;
    INCRMT_CK(cudaGraphLaunch(L.gexec, stream));
    return INCRMT_OK;
}

/** After a solve under capture: the target (block averages of the solution
 * minus the warm start). */
int Sim::learned_post(int sys, const double *z) {
    Learned &L = learn[sys];
    if (L.ran) {
        // the solve has synchronised the stream: reading the rejection count
        // costs one small copy
        L.ran = false;
        unsigned long long fb = 0;
        INCRMT_CK(cudaMemcpyAsync(&fb, d_lcnt + 2 * sys + 1, sizeof(fb), cudaMemcpyDeviceToHost, stream));
        INCRMT_CK(cudaStreamSynchronize(stream));
        if (fb > L.fb_seen) {
            if (++L.fb_streak >= kLearnedStrikes) {
                L.fb_streak = 0;
                L.skip = kLearnedRest;
            }
        } else {
            L.fb_streak = 0;
        }
        L.fb_seen = fb;
    }
    if (!(L.cap > 0 && L.captured < L.cap)) return INCRMT_OK;
    Multigrid &mg = sys == INCRMT_SYS_MAC ? mac : fem;
    int H, W;
    learned_grid(mg.m, mg.n, L.cap_factor, H, W);
    int r = learned_target(mg, z, L.z0, L.cap_factor, H, W, L.cap_tgt + static_cast<size_t>(L.captured) * H * W);
    if (r) return r;
    L.captured++;
    return INCRMT_OK;
}

int Sim::fem_projection(double dt) {
    k_fem_ghosts<<<1, 1024, 0, stream>>>(g, f);
    k_fem_source<<<g2(g.mf, g.nf), kB2, 0, stream>>>(g, f, src_fem, dt);
    launches += 2;
    INCRMT_CKL("k_fem_source");
    int outer = cur_phase, r;
    if ((r = phase_end())) return r;
    if ((r = phase_begin(INCRMT_PHASE_MG_SETUP))) return r;
    r = const_rho ? INCRMT_OK : fem.set_density_lagged(f.rho, g.P);
    if (r) return r;
    if ((r = phase_end())) return r;
    if ((r = phase_begin(outer))) return r;
    incrmt_mg_stats st{};
    long long l0 = fem.launches;
    if ((r = extrapolate_guess(INCRMT_SYS_FEM, z_fem))) return r;
    if ((r = learned_pre(INCRMT_SYS_FEM, src_fem, z_fem))) return r;
    r = const_rho ? fem.solve_device(src_fem, z_fem, &mgo, &st, false) : fem.solve_lagged(src_fem, z_fem, &mgo, &st, false);
    if (!r) r = learned_post(INCRMT_SYS_FEM, z_fem);
    if (!r) nsol[INCRMT_SYS_FEM]++;
    launches += fem.launches - l0;
    vc_fem += st.vcycles;
    solves_fem++;
    if (r) return r;
    const int nb = 2 * kB200SMs;
    k_pressure_sum<<<nb, 256, 0, stream>>>(g, z_fem, partial);
    k_reduce_partials<<<1, 256, 0, stream>>>(partial, nb, partial + nb);
    k_copy_pressure<<<g2(g.m + 1, g.n + 1), kB2, 0, stream>>>(g, f, z_fem, partial + nb);
    launches += 3;
    INCRMT_CKL("copy_pressure");
    return INCRMT_OK;
}

int Sim::tracers(int st, double dt) {
    Field2 vel{f.u, f.v};
    if (ntrace > 0) {
        if (st == 2) INCRMT_CK(cudaMemsetAsync(d_flags + 8, 0, sizeof(int), stream));
        k_tracers<<<cdiv(ntrace, 128), 128, 0, stream>>>(g, vel, tm, ntrace, 4, st, dt, 1, d_flags + 8, d_remap);
        launches++;
    }
    if (nobjtr > 0) {
        k_tracers<<<cdiv(nobjtr, 128), 128, 0, stream>>>(g, vel, otm, nobjtr, 6, st, dt, 0, nullptr, nullptr);
        launches++;
    }
    INCRMT_CKL("k_tracers");
    if (st == 2 && ntrace > 0) {
        int r = remap_tracers();
        if (r) return r;
    }
    if (st == 2 && nobjtr > 0) {
        // obj_track::update_tracers (object.cc:358-366): a record every 10 steps.
        if (track_count == track_every) return record_track();
        track_count++;
    }
    return INCRMT_OK;
}

/** sim_type::tracer_remap (sim_type.cc:12-17) for the tracers that left the
 * box in the last stage-2 update, in index order as fluid_2d::update_tracers
 * visits them (fluid_2d.cc:1476-1479): the wrapped coordinate moves by the box
 * length and the other is redrawn with the C library's rand() (common.hh:
 * 28-30), so a host that seeded its tracers with rand() continues the same
 * sequence. */
int Sim::remap_tracers() {
    int n = 0;
    INCRMT_CK(cudaMemcpyAsync(&n, d_flags + 8, sizeof(int), cudaMemcpyDeviceToHost, stream));
    INCRMT_CK(cudaStreamSynchronize(stream));
    if (n == 0) return INCRMT_OK;
    if (n > ntrace) n = ntrace;
    std::vector<int> idx(n);
    std::vector<double> t(4 * static_cast<size_t>(ntrace));
    INCRMT_CK(cudaMemcpyAsync(idx.data(), d_remap, sizeof(int) * n, cudaMemcpyDeviceToHost, stream));
    INCRMT_CK(cudaMemcpyAsync(t.data(), tm, sizeof(double) * t.size(), cudaMemcpyDeviceToHost, stream));
    INCRMT_CK(cudaStreamSynchronize(stream));
    std::sort(idx.begin(), idx.end());
    auto rnd = [](double a, double b) { return a + ((b - a) / RAND_MAX) * static_cast<double>(rand()); };
    for (int k : idx) {
        double &x = t[4 * static_cast<size_t>(k)], &y = t[4 * static_cast<size_t>(k) + 1];
        if (x < g.ax) x += (g.bx - g.ax), y = rnd(g.ay, g.by);
        if (x > g.bx) x -= (g.bx - g.ax), y = rnd(g.ay, g.by);
        if (y < g.ay) y += (g.by - g.ay), x = rnd(g.ax, g.bx);
        if (y > g.by) y -= (g.by - g.ay), x = rnd(g.ax, g.bx);
    }
    INCRMT_CK(cudaMemcpyAsync(tm, t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice, stream));
    INCRMT_CK(cudaStreamSynchronize(stream));
    remapped_tracers += n;
    return INCRMT_OK;
}

/** obj_track::file_output / obj_simple_spin::file_output (object.cc:202-219,
 * 339-347): the point before and after its correction onto the reference
 * map, stored with the time; the host writes track.dat from these. */
int Sim::record_track() {
    std::vector<double> pre(6 * static_cast<size_t>(nobjtr)), post(pre.size());
    INCRMT_CK(cudaMemcpyAsync(pre.data(), otm, sizeof(double) * pre.size(), cudaMemcpyDeviceToHost, stream));
    if (t_correction) {
        Field2 rm{sol[trk].X, sol[trk].Y};
        INCRMT_CK(cudaMemsetAsync(d_flags + 9, 0, sizeof(int), stream));
        k_correct_tracers<<<cdiv(nobjtr, 128), 128, 0, stream>>>(g, rm, otm, nobjtr, d_flags + 9);
        launches++;
        INCRMT_CKL("k_correct_tracers");
    }
    INCRMT_CK(cudaMemcpyAsync(post.data(), otm, sizeof(double) * post.size(), cudaMemcpyDeviceToHost, stream));
    int r = fetch_flags();
    if (r) return r;
    if (h_flags[9]) t_correction = 0;
    track.push_back(time);
    for (int k = 0; k < nobjtr; k++) {
        track.push_back(pre[6 * k]); track.push_back(pre[6 * k + 1]);
        track.push_back(post[6 * k]); track.push_back(post[6 * k + 1]);
    }
    track_count = 1;
    return INCRMT_OK;
}

int Sim::initialize(double ev_mult, double dt_pad, double dt_ev_pad) {
    if (initialized) { set_error("already initialized"); return INCRMT_ERR_BADARG; }
    // fluid_2d::choose_ev_and_dt (fluid_2d.cc:152-192) and obj_field::set_ex_visc
    // (obj_field.cc:35-49).
    const double hmax = g.dx > g.dy ? g.dx : g.dy, hmin = g.dx > g.dy ? g.dy : g.dx;
    double sws_max = 0, ex_visc_max = 0, rdev_min = 1.7976931348623157e308;
    for (auto &o : obj) {
        const double tfac = ev_mult * hmax, sws = sqrt(o.G / o.rhos);
        if (sws > sws_max) sws_max = sws;
        o.ex_visc = tfac * o.rhos * sws;
        if (o.ex_visc > ex_visc_max) ex_visc_max = o.ex_visc;
        const double r = o.rhos / (o.ex_visc * (o.ev_trans_mult + 1));
        if (r < rdev_min) rdev_min = r;
    }
    const double dt0 = hmin / sws_max * dt_pad, dt1 = 0.5 * rdev_min / (g.xxsp + g.yysp) * dt_ev_pad,
                 dt2 = 0.5 * g.rhof / (g.visc * (g.xxsp + g.yysp)) * dt_pad;
    if (dt0 < dt1) dt_reg = dt0 < dt2 ? dt0 : dt2;
    else dt_reg = dt1 < dt2 ? dt1 : dt2;
    // object::start (obj_simple_spin::start_extra, object.cc:152-165;
    // obj_flag::start_extra, object.cc:455-469).
    for (auto &o : obj) {
        if (o.type == OBJ_SIMPLE_SPIN) {
            double t = o.g[3] + o.eps;
            o.g[6] = t * t;
            o.g[7] = 0.1 / (dt_reg * dt_reg);
        } else if (o.type == OBJ_FLAG) {
            double t = o.g[8] + o.eps;
            o.g[10] = t * t;
            o.g[11] = 0.01 / (dt_reg * dt_reg);
        } else if (o.type == OBJ_SEVEN_POINT) {  // obj_seven_point::start_extra, object.cc:100-111
            double t = o.g[3] + o.eps;
            o.g[6] = t * t;
            o.g[7] = 0.01 / (dt_reg * dt_reg);
        } else if (o.type == OBJ_PISTON) {  // obj_piston::start_extra, object.cc:224-237
            double t = o.g[5] + o.eps;
            o.g[10] = t * t;
            o.g[11] = 0.01 / (dt_reg * dt_reg);
        }
    }
    // Object tracers (obj_track) of the first tracking object: the simple
    // spinner's point at 0.9*r_scale on the x axis, recorded every 10 steps
    // (object.hh:444-453); the flag's points evenly spaced along its length
    // from the tail, every 100 steps (object.cc:427-434); the piston's point
    // at (-cx, y_start), every 100 steps (object.hh:390-401); the circle
    // tracker's points at (cx -+ cr/2, cy), every 32 steps (object.cc:504-512).
    nobjtr = 0;
    trk = -1;
    for (size_t k = 0; k < obj.size() && trk < 0; k++)
        if (obj[k].type == OBJ_SIMPLE_SPIN || obj[k].type == OBJ_FLAG || obj[k].type == OBJ_PISTON ||
            desc[k].type == INCRMT_OBJ_CIRCLE_TRACK)
            trk = static_cast<int>(k);
    if (trk >= 0) {
        const ObjDev &o = obj[trk];
        std::vector<double> h;
        if (o.type == OBJ_SIMPLE_SPIN) {
            const double x = 0.9 * desc[trk].params[0];
            h = {x, 0, 0, 0, x, 0};
            track_every = 10;
        } else if (o.type == OBJ_PISTON) {
            const double x = -o.g[8], y = o.g[1];
            h = {x, y, 0, 0, x, y - o.g[1]};  // transform: X = x, Y = y - y_start
            track_every = 100;
        } else if (o.type == OBJ_CIRCLE) {
            const double x0 = o.g[0] - 0.5 * o.g[2], x1 = o.g[0] + 0.5 * o.g[2], y = o.g[1];
            h = {x0, y, 0, 0, x0 - o.g[0], y - o.g[1], x1, y, 0, 0, x1 - o.g[0], y - o.g[1]};
            track_every = 32;
        } else {
            const int nt = static_cast<int>(desc[trk].params[6]);
            const double step = nt == 1 ? 0. : o.g[2] / (nt - 1);
            double ex = o.g[2];
            for (int k = 0; k < nt; k++, ex -= step) {
                const double t[6] = {ex, 0, 0, 0, ex - o.g[0], 0 - o.g[1]};
                h.insert(h.end(), t, t + 6);
            }
            track_every = 100;
        }
        nobjtr = static_cast<int>(h.size() / 6);
        int r = alloc(&otm, h.size());
        if (r) return r;
        INCRMT_CK(cudaMemcpyAsync(otm, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, stream));
        INCRMT_CK(cudaStreamSynchronize(stream));
    }
    int r = upload_objects();
    if (r) return r;
    if ((r = win_reset())) return r;
    // fluid_2d::init_fields (fluid_2d.cc:195-254).
    if (!obj.empty()) {
        k_init_object<<<dim3(cdiv(g.ml, 32), cdiv(g.nl, 8), obj.size()), kB2, 0, stream>>>(g, d_obj, d_sol);
        launches++;
        INCRMT_CKL("k_init_object");
    }
    if ((r = build_bands())) return r;
    k_init_velocity<<<g2(g.m, g.n), kB2, 0, stream>>>(g, f, d_obj, d_sol, static_cast<int>(obj.size()));
    launches++;
    INCRMT_CKL("k_init_velocity");
    if ((r = set_boundaries())) return r;
    if ((r = compute_stress())) return r;
    if ((r = set_rho())) return r;
    // fluid_2d::setup_multigrid with same_rho (fluid_2d.cc:126-137,
    // fluid_2d.hh:244-248; small_number = 100 DBL_EPSILON, common.hh:16).
    const_rho = true;
    for (const auto &o : obj)
        if (fabs(o.rhos - g.rhof) > 100 * DBL_EPSILON) const_rho = false;
    if (const_rho && ((r = mac.set_unit_density()) || (r = fem.set_unit_density()))) return r;
    initialized = true;
    INCRMT_CK(cudaStreamSynchronize(stream));
    return INCRMT_OK;
}

/** fluid_2d::update_velocity (fluid_2d.cc:1354-1374): the velocity, then
 * X = nX over the window of the last reference-map update (the whole grid
 * when X and nX may differ elsewhere: before the first step, after a state
 * upload, or without a recorded update). */
int Sim::update_velocity(double dt) {
    k_update_velocity<<<g2(g.m, g.n), kB2, 0, stream>>>(g, f, dt);
    launches++;
    INCRMT_CKL("k_update_velocity");
    if (obj.empty()) return INCRMT_OK;
    const int kind = x_synced && pref_valid ? 2 : 3;
    k_refmap_commit<<<wgrid(kind), kB2, 0, stream>>>(g, d_sol, win(kind));
    launches++;
    INCRMT_CKL("k_refmap_commit");
    x_synced = true;
    pref_valid = false;
    return INCRMT_OK;
}

/** godunov_upwinding_set<tang> followed by edge_boundary_conditions
 * (fluid_2d.cc:1112-1121, 689-777). */
int Sim::godunov(bool tang) {
    const int no = static_cast<int>(obj.size());
    if (g.solid_prd && no > 0) {
        // edge_boundary_conditions_solid_pre (fluid_2d.cc:730): it runs after
        // the interior Godunov pass in the reference, which writes no right
        // or top solid edge value, so running it first is the same.
        k_solid_edges_prd<<<1, 1024, 0, stream>>>(g, d_sol, no, 0);
        launches++;
    }
    if (tang) k_godunov<true><<<g2(g.m, g.n), kB2, 0, stream>>>(g, f, d_sol, tiles());
    else k_godunov<false><<<g2(g.m, g.n), kB2, 0, stream>>>(g, f, d_sol, tiles());
    launches++;
    if (g.xp) {
        k_wrap_edges_x<<<cdiv(g.n, 256), 256, 0, stream>>>(g, f);
        launches++;
    }
    if (g.yp) {
        k_wrap_edges_y<<<cdiv(g.m, 256), 256, 0, stream>>>(g, f);
        launches++;
    }
    if (g.solid_prd && no > 0) {  // edge_boundary_conditions_solid_post (fluid_2d.cc:778)
        k_solid_edges_prd<<<1, 1024, 0, stream>>>(g, d_sol, no, 1);
        launches++;
    }
    INCRMT_CKL("k_godunov");
    return INCRMT_OK;
}

/** fluid_2d::step_forward (fluid_2d.cc:298-369). */
int Sim::step(double dt) {
    if (!initialized) { set_error("not initialized"); return INCRMT_ERR_BADARG; }
    const double ntime = time + dt;
    int r;
#define INCRMT_PHASE(ph, ...) do { if ((r = phase_begin(ph))) return r; __VA_ARGS__; if ((r = phase_end())) return r; } while (0)
    INCRMT_PHASE(INCRMT_PHASE_TRACERS, if ((r = tracers(1, dt))) return r);
    INCRMT_PHASE(INCRMT_PHASE_ADVECTION, {
        k_normal_derivatives<<<g2(g.m, g.n), kB2, 0, stream>>>(g, f, d_sol, tiles(), dt);
        if ((r = godunov(true))) return r;
        k_tangential<<<g2(g.m, g.n), kB2, 0, stream>>>(g, f);
        k_half_time<<<g2(g.m, g.n), kB2, 0, stream>>>(g, f, d_obj, d_sol, tiles(), dt);
        if ((r = godunov(false))) return r;
        launches += 3;
        INCRMT_CKL("advection");
    });
    time += 0.5 * dt;
    INCRMT_PHASE(INCRMT_PHASE_MAC, if ((r = mac_projection())) return r);
    INCRMT_PHASE(INCRMT_PHASE_REFMAP, if ((r = update_reference_map(dt))) return r);
    INCRMT_PHASE(INCRMT_PHASE_PIN, if ((r = pin())) return r);
    INCRMT_PHASE(INCRMT_PHASE_STRESS, {
        if ((r = set_boundaries())) return r;
        if ((r = compute_stress())) return r;
        k_ustar<<<g2(g.m, g.n), kB2, 0, stream>>>(g, f, d_obj, d_sol, tiles(), dt);
        launches++;
        INCRMT_CKL("k_ustar");
    });
    time = ntime;
    INCRMT_PHASE(INCRMT_PHASE_FEM, if ((r = fem_projection(dt))) return r);
    INCRMT_PHASE(INCRMT_PHASE_STRESS, if ((r = update_velocity(dt))) return r);
    INCRMT_PHASE(INCRMT_PHASE_PIN, if ((r = pin())) return r);
    INCRMT_PHASE(INCRMT_PHASE_STRESS, {
        if ((r = set_boundaries())) return r;
        if ((r = compute_stress())) return r;
    });
    INCRMT_PHASE(INCRMT_PHASE_TRACERS, if ((r = tracers(2, dt))) return r);
#undef INCRMT_PHASE
    steps++;
    return INCRMT_OK;
}

/** Runs one reference step function on the current state (same numbering as
 * the oracle's ref_stage). */
int Sim::stage(int s, double dt) {
    switch (s) {
        case 0: return tracers(1, dt);
        case 1:
        case 2: k_normal_derivatives<<<g2(g.m, g.n), kB2, 0, stream>>>(g, f, d_sol, tiles(), dt); break;
        case 3: return godunov(true);
        case 4: break;  // fused into the Godunov kernels
        case 5: k_tangential<<<g2(g.m, g.n), kB2, 0, stream>>>(g, f); break;
        case 6:
        case 7: k_half_time<<<g2(g.m, g.n), kB2, 0, stream>>>(g, f, d_obj, d_sol, tiles(), dt); break;
        case 8: return godunov(false);
        case 9: return mac_projection();
        case 10: return update_reference_map(dt);
        case 11: return pin();
        case 12: return set_boundaries();
        case 13: return compute_stress();
        case 14: k_ustar<<<g2(g.m, g.n), kB2, 0, stream>>>(g, f, d_obj, d_sol, tiles(), dt); break;
        case 15: return fem_projection(dt);
        case 16: return INCRMT_OK;  // fused into fem_projection
        case 17: return update_velocity(dt);
        case 18: return tracers(2, dt);
        case 19: return set_rho();
        case 20: return step(dt);
        case 21: return build_bands();
        case 22: return extrapolate_all();
        default: set_error("unknown stage %d", s); return INCRMT_ERR_BADARG;
    }
    launches++;
    INCRMT_CKL("stage");
    return INCRMT_OK;
}

void Sim::destroy() {
    if (stream) cudaStreamSynchronize(stream);
    mac.destroy();
    fem.destroy();
    for (double *p : allocs) cudaFree(p);
    allocs.clear();
    for (auto &s : sol) cudaFree(s.s);
    cudaFree(d_frame); cudaFree(d_box);
    d_frame = nullptr; d_box = nullptr; frame_cap = 0;
    cudaFree(d_win); cudaFree(d_lsbox); cudaFree(d_tiles); cudaFree(d_lcnt); cudaFree(d_remap);
    d_remap = nullptr;
    d_lcnt = nullptr;
    for (Learned &L : learn) {
        L.release_graph();
        L.w.release();
        cudaFree(L.z0);
        L.z0 = nullptr;
        L.z0_n = 0;
    }
    if (h_win) cudaFreeHost(h_win);
    if (h_lsbox) cudaFreeHost(h_lsbox);
    if (h_tiles) cudaFreeHost(h_tiles);
    d_win = h_win = nullptr; d_lsbox = h_lsbox = nullptr; d_tiles = h_tiles = nullptr; tiles_cap = 0;
    for (void *p : raw_allocs) cudaFree(p);
    raw_allocs.clear();
    lso.clear();
    cudaFree(d_obj); cudaFree(d_sol); cudaFree(d_lso); cudaFree(d_list); cudaFree(d_list_k); cudaFree(d_flags);
    d_obj = nullptr; d_sol = nullptr; d_lso = nullptr; d_list = d_list_k = nullptr; d_flags = nullptr; list_cap = 0;
    if (h_flags) cudaFreeHost(h_flags);
    for (auto e : ev_pool) cudaEventDestroy(e);
    ev_pool.clear();
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
}

}  // namespace incrmt

struct incrmt_sim {
    incrmt::Sim s;
};

using incrmt::set_error;

namespace {

/** Device array of field id (include/incrmt_sim.h) for object k. */
double *field_ptr(incrmt::Sim &S, int id, int k) {
    incrmt::FluidDev &f = S.f;
    double *fl[] = {f.u, f.v, f.p, f.rho, f.ux, f.uy, f.vx, f.vy, f.ud, f.vd, f.ul, f.vl,
                    f.ur, f.vr, f.uu, f.vu, f.c0, f.c1, f.c2, f.c3, f.s11, f.s12, f.s21, f.s22};
    if (id >= 0 && id < 24) return fl[id];
    if (k < 0 || k >= static_cast<int>(S.sol.size())) return nullptr;
    incrmt::SolidDev &s = S.sol[k];
    double *sl[] = {s.X, s.Y, s.nX, s.nY, s.Xx, s.Xy, s.Yx, s.Yy, s.Xd, s.Yd, s.Xl, s.Yl, s.Xr, s.Yr, s.Xu, s.Yu};
    if (id >= 100 && id < 116) return sl[id - 100];
    if (id == INCRMT_FIELD_PHI) return s.phi;
    return nullptr;
}

}  // namespace

extern "C" {

int incrmt_create(const incrmt_grid *g, const incrmt_phys *p, incrmt_sim **out) {
    if (!g || !p || !out) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    *out = nullptr;
    incrmt_sim *h = new (std::nothrow) incrmt_sim;
    if (!h) { set_error("host allocation failed"); return INCRMT_ERR_OOM; }
    int r = h->s.create(g, p);
    if (r) { h->s.destroy(); delete h; return r; }
    *out = h;
    return INCRMT_OK;
}

int incrmt_add_object(incrmt_sim *h, const incrmt_object_desc *d) {
    if (!h || !d) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    return h->s.add_object(d);
}

int incrmt_initialize(incrmt_sim *h, double ev_mult, double dt_pad, double dt_ev_pad, double *dt_reg) {
    if (!h) { set_error("null handle"); return INCRMT_ERR_BADARG; }
    int r = h->s.initialize(ev_mult, dt_pad, dt_ev_pad);
    if (dt_reg) *dt_reg = h->s.dt_reg;
    return r;
}

int incrmt_set_tracers(incrmt_sim *h, const double *xy) {
    if (!h || !xy) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    incrmt::Sim &S = h->s;
    if (S.ntrace == 0) return INCRMT_OK;
    std::vector<double> t(4 * static_cast<size_t>(S.ntrace), 0.0);
    for (int k = 0; k < S.ntrace; k++) { t[4 * k] = xy[2 * k]; t[4 * k + 1] = xy[2 * k + 1]; }
    INCRMT_CK(cudaMemcpyAsync(S.tm, t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice, S.stream));
    INCRMT_CK(cudaStreamSynchronize(S.stream));
    return INCRMT_OK;
}

int incrmt_step(incrmt_sim *h, double dt) {
    if (!h) { set_error("null handle"); return INCRMT_ERR_BADARG; }
    return h->s.step(dt);
}

int incrmt_steps(incrmt_sim *h, double dt, int nsteps) {
    if (!h) { set_error("null handle"); return INCRMT_ERR_BADARG; }
    for (int k = 0; k < nsteps; k++) { int r = h->s.step(dt); if (r) return r; }
    INCRMT_CK(cudaStreamSynchronize(h->s.stream));
    return INCRMT_OK;
}

int incrmt_stage(incrmt_sim *h, int stage, double dt) {
    if (!h) { set_error("null handle"); return INCRMT_ERR_BADARG; }
    int r = h->s.stage(stage, dt);
    if (r) return r;
    INCRMT_CK(cudaStreamSynchronize(h->s.stream));
    return INCRMT_OK;
}

int incrmt_get_field(incrmt_sim *h, int id, int k, double *host) {
    if (!h || !host) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    incrmt::Sim &S = h->s;
    const size_t w = S.g.ml, rows = S.g.nl;
    if (id == INCRMT_FIELD_STATUS) {
        if (k < 0 || k >= static_cast<int>(S.sol.size())) { set_error("bad object"); return INCRMT_ERR_BADARG; }
        std::vector<int> tmp(w * rows);
        INCRMT_CK(cudaMemcpy2DAsync(tmp.data(), w * sizeof(int), S.sol[k].s, S.g.P * sizeof(int), w * sizeof(int),
                                    rows, cudaMemcpyDeviceToHost, S.stream));
        INCRMT_CK(cudaStreamSynchronize(S.stream));
        for (size_t q = 0; q < w * rows; q++) host[q] = tmp[q];
        return INCRMT_OK;
    }
    double *p = field_ptr(S, id, k);
    if (!p) { set_error("bad field id %d", id); return INCRMT_ERR_BADARG; }
    INCRMT_CK(cudaMemcpy2DAsync(host, w * sizeof(double), p, S.g.P * sizeof(double), w * sizeof(double), rows,
                                cudaMemcpyDeviceToHost, S.stream));
    INCRMT_CK(cudaStreamSynchronize(S.stream));
    return INCRMT_OK;
}

int incrmt_set_field(incrmt_sim *h, int id, int k, const double *host) {
    if (!h || !host) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    incrmt::Sim &S = h->s;
    const size_t w = S.g.ml, rows = S.g.nl;
    // An uploaded state may have anything anywhere: whole-grid passes until
    // the next band rebuild, and coarse operators rebuilt at the next solve.
    if (int r = S.win_reset()) return r;
    S.mac.coarse_stale = true;
    S.fem.coarse_stale = true;
    S.nsol[0] = S.nsol[1] = 0;  // the warm start's history no longer applies
    if (id == INCRMT_FIELD_STATUS) {
        if (k < 0 || k >= static_cast<int>(S.sol.size())) { set_error("bad object"); return INCRMT_ERR_BADARG; }
        std::vector<int> tmp(w * rows);
        for (size_t q = 0; q < w * rows; q++) tmp[q] = static_cast<int>(host[q]);
        INCRMT_CK(cudaMemcpy2DAsync(S.sol[k].s, S.g.P * sizeof(int), tmp.data(), w * sizeof(int), w * sizeof(int),
                                    rows, cudaMemcpyHostToDevice, S.stream));
        INCRMT_CK(cudaStreamSynchronize(S.stream));
        return INCRMT_OK;
    }
    double *p = field_ptr(S, id, k);
    if (!p) { set_error("bad field id %d", id); return INCRMT_ERR_BADARG; }
    INCRMT_CK(cudaMemcpy2DAsync(p, S.g.P * sizeof(double), host, w * sizeof(double), w * sizeof(double), rows,
                                cudaMemcpyHostToDevice, S.stream));
    INCRMT_CK(cudaStreamSynchronize(S.stream));
    return INCRMT_OK;
}

namespace {
double *mg_ptr(incrmt::Sim &S, int which, size_t &n) {
    const size_t nm = static_cast<size_t>(S.g.m) * S.g.n, nf = static_cast<size_t>(S.g.mf) * S.g.nf;
    switch (which) {
        case 0: n = nm; return S.z_mac;
        case 1: n = nf; return S.z_fem;
        case 2: n = nm; return S.src_mac;
        case 3: n = nf; return S.src_fem;
    }
    n = 0;
    return nullptr;
}
}  // namespace

int incrmt_get_mg(incrmt_sim *h, int which, double *host) {
    if (!h || !host) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    size_t n;
    double *p = mg_ptr(h->s, which, n);
    if (!p) { set_error("bad array %d", which); return INCRMT_ERR_BADARG; }
    INCRMT_CK(cudaMemcpyAsync(host, p, sizeof(double) * n, cudaMemcpyDeviceToHost, h->s.stream));
    INCRMT_CK(cudaStreamSynchronize(h->s.stream));
    return INCRMT_OK;
}

int incrmt_set_mg(incrmt_sim *h, int which, const double *host) {
    if (!h || !host) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    size_t n;
    double *p = mg_ptr(h->s, which, n);
    if (!p) { set_error("bad array %d", which); return INCRMT_ERR_BADARG; }
    INCRMT_CK(cudaMemcpyAsync(p, host, sizeof(double) * n, cudaMemcpyHostToDevice, h->s.stream));
    INCRMT_CK(cudaStreamSynchronize(h->s.stream));
    return INCRMT_OK;
}

int incrmt_get_time(const incrmt_sim *h, double *t) {
    if (!h || !t) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    *t = h->s.time;
    return INCRMT_OK;
}

int incrmt_set_time(incrmt_sim *h, double t) {
    if (!h) { set_error("null handle"); return INCRMT_ERR_BADARG; }
    h->s.time = t;
    // The per-object state of the last stress evaluation follows the clock
    // (object::pre_stress_setup is called at every compute_stress).
    h->s.pre_stress_setup(t);
    return h->s.upload_objects();
}

int incrmt_get_tracers(incrmt_sim *h, double *host) {
    if (!h || !host) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    incrmt::Sim &S = h->s;
    if (S.ntrace > 0)
        INCRMT_CK(cudaMemcpyAsync(host, S.tm, sizeof(double) * 4 * S.ntrace, cudaMemcpyDeviceToHost, S.stream));
    INCRMT_CK(cudaStreamSynchronize(S.stream));
    return INCRMT_OK;
}

int incrmt_get_object_tracers(incrmt_sim *h, double *host, int *count) {
    if (!h || !count) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    incrmt::Sim &S = h->s;
    *count = S.nobjtr;
    if (host && S.nobjtr > 0)
        INCRMT_CK(cudaMemcpyAsync(host, S.otm, sizeof(double) * 6 * S.nobjtr, cudaMemcpyDeviceToHost, S.stream));
    INCRMT_CK(cudaStreamSynchronize(S.stream));
    return INCRMT_OK;
}

int incrmt_set_object_tracers(incrmt_sim *h, const double *host, int count, int track_count) {
    if (!h || !host) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    incrmt::Sim &S = h->s;
    if (count != S.nobjtr) { set_error("%d tracked points given, the simulation has %d", count, S.nobjtr); return INCRMT_ERR_BADARG; }
    if (track_count < 1) { set_error("bad track counter %d", track_count); return INCRMT_ERR_BADARG; }
    if (count > 0)
        INCRMT_CK(cudaMemcpyAsync(S.otm, host, sizeof(double) * 6 * count, cudaMemcpyHostToDevice, S.stream));
    S.track_count = track_count;
    INCRMT_CK(cudaStreamSynchronize(S.stream));
    return INCRMT_OK;
}

int incrmt_track_records(incrmt_sim *h, double *host, int cap, int *count, int clear) {
    if (!h || !count) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    incrmt::Sim &S = h->s;
    const size_t rec = 1 + 4 * static_cast<size_t>(S.nobjtr);
    const int n = static_cast<int>(S.track.size() / rec);
    *count = n;
    if (host) memcpy(host, S.track.data(), sizeof(double) * rec * (n < cap ? n : cap));
    if (clear) S.track.clear();
    return INCRMT_OK;
}

int incrmt_record_track(incrmt_sim *h) {
    if (!h) { set_error("null handle"); return INCRMT_ERR_BADARG; }
    if (h->s.nobjtr == 0) return INCRMT_OK;
    return h->s.record_track();
}

int incrmt_get_stats(const incrmt_sim *h, incrmt_sim_stats *st) {
    if (!h || !st) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    const incrmt::Sim &S = h->s;
    st->steps = S.steps;
    st->vcycles_mac = S.vc_mac;
    st->vcycles_fem = S.vc_fem;
    st->solves_mac = S.solves_mac;
    st->solves_fem = S.solves_fem;
    st->march_sweeps = S.ls_sweeps;
    st->march_monotone = S.ls_monotone;
    st->window_points = 0;
    for (size_t k = 0; k < S.obj.size(); k++) {
        const incrmt::LsWin &w = S.win_valid ? S.h_win[k] : incrmt::LsWin{0, 0, S.g.ml, S.g.nl};
        st->window_points += static_cast<long long>(w.x1 - w.x0) * (w.y1 - w.y0);
    }
    st->extrap_sweeps = S.ex_sweeps;
    st->coarse_builds = S.mac.coarse_builds + S.fem.coarse_builds;
    st->coarse_retries = S.mac.coarse_retries + S.fem.coarse_retries;
    st->mixed_fallbacks = S.mac.mixed_fallbacks + S.fem.mixed_fallbacks;
    st->krylov_fallbacks = S.mac.krylov_fallbacks + S.fem.krylov_fallbacks;
    st->launches = S.launches;
    st->dt_reg = S.dt_reg;
    st->time = S.time;
    return INCRMT_OK;
}

int incrmt_sim_set_learned(incrmt_sim *h, int sys, incrmt_unet *net, int factor, int rule) {
    if (!h) { set_error("null handle"); return INCRMT_ERR_BADARG; }
    if (sys != INCRMT_SYS_MAC && sys != INCRMT_SYS_FEM) { set_error("bad system %d", sys); return INCRMT_ERR_BADARG; }
    if (net && (factor < 1 || (rule != 0 && rule != 1))) {
        set_error("learned warm start needs factor >= 1 and rule 0 or 1");
        return INCRMT_ERR_BADARG;
    }
    incrmt::Sim &S = h->s;
    if (net) {
        if (int r = incrmt::learned_supported(sys == INCRMT_SYS_MAC ? S.mac : S.fem)) return r;
    }
    if (S.stream) INCRMT_CK(cudaStreamSynchronize(S.stream));
    S.learn[sys].release_graph();
    S.learn[sys].warm_net = nullptr;
    S.learn[sys].gfail = false;
    S.learn[sys].fb_streak = 0;
    S.learn[sys].skip = 0;
    S.learn[sys].net = net;
    S.learn[sys].factor = factor;
    S.learn[sys].rule = rule;
    return INCRMT_OK;
}

int incrmt_sim_learned_grid(const incrmt_sim *h, int sys, int factor, int *H, int *W) {
    if (!h || !H || !W) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    if (sys != INCRMT_SYS_MAC && sys != INCRMT_SYS_FEM) { set_error("bad system %d", sys); return INCRMT_ERR_BADARG; }
    if (factor < 1) { set_error("bad factor %d", factor); return INCRMT_ERR_BADARG; }
    const incrmt::Multigrid &mg = sys == INCRMT_SYS_MAC ? h->s.mac : h->s.fem;
    incrmt::learned_grid(mg.m, mg.n, factor, *H, *W);
    return INCRMT_OK;
}

int incrmt_sim_learned_capture(incrmt_sim *h, int sys, int factor, float *d_in, float *d_target, int cap) {
    if (!h) { set_error("null handle"); return INCRMT_ERR_BADARG; }
    if (sys != INCRMT_SYS_MAC && sys != INCRMT_SYS_FEM) { set_error("bad system %d", sys); return INCRMT_ERR_BADARG; }
    if (cap > 0 && (!d_in || !d_target || factor < 1)) {
        set_error("capture needs device buffers and factor >= 1");
        return INCRMT_ERR_BADARG;
    }
    incrmt::Sim &S = h->s;
    if (cap > 0) {
        if (int r = incrmt::learned_supported(sys == INCRMT_SYS_MAC ? S.mac : S.fem)) return r;
    }
    incrmt::Sim::Learned &L = S.learn[sys];
    L.cap_in = cap > 0 ? d_in : nullptr;
    L.cap_tgt = cap > 0 ? d_target : nullptr;
    L.cap = cap > 0 ? cap : 0;
    L.cap_factor = factor;
    L.captured = 0;
    return INCRMT_OK;
}

int incrmt_sim_get_learned_stats(incrmt_sim *h, int sys, incrmt_sim_learned_stats *st) {
    if (!h || !st) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    if (sys != INCRMT_SYS_MAC && sys != INCRMT_SYS_FEM) { set_error("bad system %d", sys); return INCRMT_ERR_BADARG; }
    incrmt::Sim &S = h->s;
    unsigned long long c[2];
    INCRMT_CK(cudaMemcpyAsync(c, S.d_lcnt + 2 * sys, sizeof(c), cudaMemcpyDeviceToHost, S.stream));
    INCRMT_CK(cudaStreamSynchronize(S.stream));
    st->applied = static_cast<long long>(c[0]);
    st->fallback = static_cast<long long>(c[1]);
    st->captured = S.learn[sys].captured;
    st->skipped = S.learn[sys].skipped;
    return INCRMT_OK;
}

int incrmt_l_comparison(incrmt_sim *h, incrmt_sim *fine, double *err) {
    if (!h || !fine || !err) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    incrmt::Sim &S = h->s, &F = fine->s;
    if (F.g.m % S.g.m != 0 || F.g.n % S.g.n != 0) {
        set_error("Grid dimension is not a multiple of the finer grid");
        return INCRMT_ERR_BADARG;
    }
    if (F.g.xp != S.g.xp || F.g.yp != S.g.yp) { set_error("the two grids differ in periodicity"); return INCRMT_ERR_BADARG; }
    INCRMT_CK(cudaStreamSynchronize(F.stream));
    const int mm = S.g.xp ? S.g.m : S.g.m + 1, nn = S.g.yp ? S.g.n : S.g.n + 1;
    const int nb = incrmt::cdiv(mm * nn, 256);
    double *part = nullptr;
    INCRMT_CK(cudaMallocAsync(&part, sizeof(double) * (incrmt::kLcmp * static_cast<size_t>(nb) + 32), S.stream));
    incrmt::k_l_comparison<<<nb, 256, 0, S.stream>>>(S.g, S.f, S.d_sol, static_cast<int>(S.obj.size()), F.f, F.g.P,
                                                    F.g.m / S.g.m, F.g.n / S.g.n, part);
    const double fac = 1. / (static_cast<double>(S.g.m) * S.g.n);
    double *dev_err = part + incrmt::kLcmp * static_cast<size_t>(nb);
    incrmt::k_l_comparison_final<<<1, 1, 0, S.stream>>>(part, nb, fac, dev_err);
    S.launches += 2;
    INCRMT_CK(cudaGetLastError());
    INCRMT_CK(cudaMemcpyAsync(err, dev_err, sizeof(double) * 32, cudaMemcpyDeviceToHost, S.stream));
    INCRMT_CK(cudaFreeAsync(part, S.stream));
    INCRMT_CK(cudaStreamSynchronize(S.stream));
    return INCRMT_OK;
}

int incrmt_sim_set_guess(incrmt_sim *h, int mode) {
    if (!h || mode < 0 || mode > 2) { set_error("bad argument"); return INCRMT_ERR_BADARG; }
    h->s.guess = mode;
    h->s.nsol[0] = h->s.nsol[1] = 0;
    return INCRMT_OK;
}

int incrmt_sim_set_coarse_refresh(incrmt_sim *h, int every) {
    if (!h || every < 1) { set_error("bad argument"); return INCRMT_ERR_BADARG; }
    h->s.mac.coarse_every = every;
    h->s.fem.coarse_every = every;
    h->s.mac.coarse_stale = true;
    h->s.fem.coarse_stale = true;
    return INCRMT_OK;
}

int incrmt_sim_set_krylov(incrmt_sim *h, int on) {
    if (!h) { set_error("null handle"); return INCRMT_ERR_BADARG; }
    h->s.mac.krylov = on != 0;
    h->s.fem.krylov = on != 0;
    return INCRMT_OK;
}

int incrmt_set_solid_prd_bc(incrmt_sim *h, int on) {
    if (!h) { set_error("null handle"); return INCRMT_ERR_BADARG; }
    incrmt::Sim &S = h->s;
    if (S.initialized) { set_error("solid_prd_bc must be set before initialize"); return INCRMT_ERR_BADARG; }
    if (on && !(S.g.xp && S.g.yp)) {
        set_error("periodic reference-map boundaries need a doubly periodic domain");
        return INCRMT_ERR_BADARG;
    }
    S.g.solid_prd = on ? 1 : 0;
    return INCRMT_OK;
}

int incrmt_sim_set_windows(incrmt_sim *h, int on) {
    if (!h) { set_error("null handle"); return INCRMT_ERR_BADARG; }
    h->s.win_enable = on != 0;
    return on ? INCRMT_OK : h->s.win_reset();
}

int incrmt_sim_set_profiling(incrmt_sim *h, int on) {
    if (!h) { set_error("null handle"); return INCRMT_ERR_BADARG; }
    incrmt::Sim &S = h->s;
    int r = S.phase_collect();
    if (r) return r;
    S.prof = (on & 1) != 0;
    for (int k = 0; k < INCRMT_PHASES; k++) { S.phase_ms[k] = 0; S.phase_n[k] = 0; }
    for (incrmt::Multigrid *mg : {&S.mac, &S.fem}) {
        r = mg->prof_collect();
        if (r) return r;
        mg->prof = (on & 2) != 0;
        mg->prof_ms = 0; mg->prof_bytes = 0; mg->prof_launches = 0;
    }
    return INCRMT_OK;
}

int incrmt_sim_mg_profile(incrmt_sim *h, int which, double *ms, double *bytes, long long *launches) {
    if (!h || (which != INCRMT_SYS_MAC && which != INCRMT_SYS_FEM)) { set_error("bad argument"); return INCRMT_ERR_BADARG; }
    incrmt::Multigrid &mg = which == INCRMT_SYS_MAC ? h->s.mac : h->s.fem;
    int r = mg.prof_collect();
    if (r) return r;
    if (ms) *ms = mg.prof_ms;
    if (bytes) *bytes = mg.prof_bytes;
    if (launches) *launches = mg.prof_launches;
    return INCRMT_OK;
}

int incrmt_sim_profile(incrmt_sim *h, double *ms) {
    if (!h || !ms) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    int r = h->s.phase_collect();
    if (r) return r;
    for (int k = 0; k < INCRMT_PHASES; k++) ms[k] = h->s.phase_ms[k];
    return INCRMT_OK;
}

void *incrmt_sim_stream(const incrmt_sim *h) { return h ? static_cast<void *>(h->s.stream) : nullptr; }

void incrmt_destroy(incrmt_sim *h) {
    if (!h) return;
    h->s.destroy();
    delete h;
}

}  // extern "C"

int incrmt_solid_bound(incrmt_sim *h, int box[4]) {
    if (!h || !box) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    incrmt::Sim &S = h->s;
    const int nobj = static_cast<int>(S.sol.size());
    int init[4] = {S.g.ml, 0, S.g.nl, 0};
    if (nobj == 0) { std::memcpy(box, init, sizeof(init)); return INCRMT_OK; }
    if (!S.d_box) INCRMT_CK(cudaMalloc(&S.d_box, 4 * sizeof(int)));
    INCRMT_CK(cudaMemcpyAsync(S.d_box, init, sizeof(init), cudaMemcpyHostToDevice, S.stream));
    incrmt::k_solid_bound<<<incrmt::g2(S.g.ml, S.g.nl), dim3(32, 8), 0, S.stream>>>(S.g, S.d_sol, nobj, S.d_box);
    S.launches++;
    INCRMT_CKL("k_solid_bound");
    INCRMT_CK(cudaMemcpyAsync(box, S.d_box, 4 * sizeof(int), cudaMemcpyDeviceToHost, S.stream));
    INCRMT_CK(cudaStreamSynchronize(S.stream));
    return INCRMT_OK;
}

int incrmt_frame(incrmt_sim *h, int mode, const int box[4], float *host) {
    if (!h || !box || !host) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    incrmt::Sim &S = h->s;
    const int nobj = static_cast<int>(S.sol.size());
    const int li = box[0], ui = box[1], lj = box[2], uj = box[3], si = ui - li, sj = uj - lj;
    if (mode < 0 || mode > 12) { set_error("bad output mode %d", mode); return INCRMT_ERR_BADARG; }
    if (mode >= 6 && mode <= 9 && nobj == 0) { set_error("output mode %d needs a solid", mode); return INCRMT_ERR_BADARG; }
    const bool stencil = mode == 4 || mode == 9 || mode == 12;
    if (si <= 0 || sj <= 0 || li < (stencil ? 1 : 0) || lj < (stencil ? 1 : 0) || ui > S.g.ml || uj > S.g.nl) {
        set_error("bad output box [%d,%d)x[%d,%d) for mode %d", li, ui, lj, uj, mode);
        return INCRMT_ERR_BADARG;
    }
    const size_t need = static_cast<size_t>(si + 1) * (sj + 1);
    if (need > S.frame_cap) {
        cudaFree(S.d_frame);
        S.d_frame = nullptr;
        S.frame_cap = 0;
        INCRMT_CK(cudaMalloc(&S.d_frame, need * sizeof(float)));
        S.frame_cap = need;
    }
    const double off = incrmt::frame_corner_mode(mode) ? 2.0 : 1.5;
    const double lx = S.g.ax + S.g.dx * (li - off), ly = S.g.ay + S.g.dy * (lj - off);
    incrmt::k_frame<<<incrmt::g2(si + 1, sj + 1), dim3(32, 8), 0, S.stream>>>(S.g, S.f, S.d_sol, nobj, mode, li, lj,
                                                                             si, sj, lx, ly, S.d_frame);
    S.launches++;
    INCRMT_CKL("k_frame");
    INCRMT_CK(cudaMemcpyAsync(host, S.d_frame, need * sizeof(float), cudaMemcpyDeviceToHost, S.stream));
    INCRMT_CK(cudaStreamSynchronize(S.stream));
    return INCRMT_OK;
}
