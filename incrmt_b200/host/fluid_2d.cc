/* fluid_2d and the object classes over the C ABI (see incrmt_host.hh). */
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>

#include "incrmt_host.hh"

void incrmt_check(int r, const char *what) {
    if (r == INCRMT_OK) return;
    fprintf(stderr, "%s failed (%d): %s\n", what, r, incrmt_last_error());
    exit(1);
}

namespace {

/** Wall-clock seconds (the reference's wtime with OpenMP, common.hh:35-36). */
double wtime() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

/** Uniform random number in [a,b] from the C library generator, the
 * reference's rnd (common.hh:28-30), so tracer seeding follows the same
 * sequence. */
inline double rnd(double a, double b) {
    return a + ((b - a) / RAND_MAX) * static_cast<double>(rand());
}

FILE *open_or_die(const char *fn, const char *mode) {
    FILE *f = fopen(fn, mode);
    if (f == nullptr) {
        fprintf(stderr, "Can't open file %s\n", fn);
        exit(1);
    }
    return f;
}

const double small_number = 100. * std::numeric_limits<double>::epsilon();

}  // namespace

// ---------------------------------------------------------------- objects

obj_simple_spin::~obj_simple_spin() {
    if (fp != nullptr) fclose(fp);
}

void obj_simple_spin::describe(incrmt_object_desc &d) const {
    d.type = INCRMT_OBJ_SIMPLE_SPIN;
    const double p[8] = {r_scale, a1, a2, piv_r, th_max, omega, 0, 0};
    memcpy(d.params, p, sizeof(p));
}

/** obj_simple_spin::start_extra (object.cc:152-165): opens the track file and
 * reports the anchor stiffness the library derives from dt_reg. */
void obj_simple_spin::start(fluid_2d &f) {
    std::vector<char> fn(strlen(filename) + 16);
    snprintf(fn.data(), fn.size(), "%s.odr/track.dat", filename);
    fp = open_or_die(fn.data(), "wb");
    K_stiff = 0.1 / (f.dt_reg * f.dt_reg);
    printf("# Anchoring K_stiff       : %g (1/T^2)\n", K_stiff);
}

/** obj_simple_spin::file_output (object.cc:202-219): the angle of the
 * tracked point before its correction, unwrapped by the winding count, and
 * the corrected position. */
void obj_simple_spin::track_record(const double *rec) {
    const double ang = atan2(rec[2], rec[1]);
    const int q = fabs(ang) > 0.5 * M_PI ? (ang > 0 ? 1 : -1) : 0;
    if (q == 1 && prev_q == -1) wind--;
    else if (q == -1 && prev_q == 1) wind++;
    prev_q = q;
    const double out[4] = {rec[0], rec[3], rec[4], ang + 2 * M_PI * wind};
    fwrite(out, sizeof(double), 4, fp);
}

void obj_simple_spin::write(int k, double time) {
    if (fp != nullptr) fflush(fp);
}

obj_flag::~obj_flag() {
    if (fp != nullptr) fclose(fp);
}

void obj_flag::describe(incrmt_object_desc &d) const {
    d.type = INCRMT_OBJ_FLAG;
    const double p[8] = {cx, cy, flag_l, flag_w, flag_a, perturb_v, static_cast<double>(ntrace), 0};
    memcpy(d.params, p, sizeof(p));
}

/** obj_flag::start_extra (object.cc:455-469). */
void obj_flag::start(fluid_2d &f) {
    std::vector<char> fn(strlen(filename) + 16);
    snprintf(fn.data(), fn.size(), "%s.odr/track.dat", filename);
    fp = open_or_die(fn.data(), "wb");
    printf("# Anchoring K_stiff       : %g (1/T^2)\n", 0.01 / (f.dt_reg * f.dt_reg));
}

/** obj_track::file_output (object.cc:344-351): time and the corrected
 * positions of the tracked points. */
void obj_flag::track_record(const double *rec) {
    std::vector<double> out(1 + 2 * static_cast<size_t>(ntrace));
    out[0] = rec[0];
    for (int k = 0; k < ntrace; k++) {
        out[1 + 2 * k] = rec[1 + 4 * k + 2];
        out[2 + 2 * k] = rec[1 + 4 * k + 3];
    }
    fwrite(out.data(), sizeof(double), out.size(), fp);
}

void obj_flag::write(int k, double time) {
    if (fp != nullptr) fflush(fp);
}

void obj_circle::describe(incrmt_object_desc &d) const {
    d.type = INCRMT_OBJ_CIRCLE;
    const double p[8] = {cx, cy, cr, uu, vv, omega, grav, 0};
    memcpy(d.params, p, sizeof(p));
}

void obj_square::describe(incrmt_object_desc &d) const {
    d.type = INCRMT_OBJ_SQUARE;
    const double p[8] = {cx, cy, cr, uu, vv, omega, grav, 0};
    memcpy(d.params, p, sizeof(p));
}

void obj_seven_point::describe(incrmt_object_desc &d) const {
    d.type = INCRMT_OBJ_SEVEN_POINT;
    const double p[6] = {cx, cy, cr, piv_r, th_max, omega};
    memcpy(d.params, p, sizeof(p));
}

/** obj_seven_point::start_extra (object.cc:100-111). */
void obj_seven_point::start(fluid_2d &f) {
    printf("# Anchoring K_stiff       : %g (1/T^2)\n", 0.01 / (f.dt_reg * f.dt_reg));
}

void obj_flapper::describe(incrmt_object_desc &d) const {
    d.type = INCRMT_OBJ_FLAPPER;
    const double p[9] = {cx, cy, cr, cl, ar, al, theta, m_stretch, T};
    memcpy(d.params, p, sizeof(p));
}

void obj_triangle::describe(incrmt_object_desc &d) const {
    d.type = INCRMT_OBJ_TRIANGLE;
    const double p[5] = {cx, cy, cr, theta, grav};
    memcpy(d.params, p, sizeof(p));
}

void obj_lamprey::describe(incrmt_object_desc &d) const {
    d.type = INCRMT_OBJ_LAMPREY;
    const double p[9] = {cx, cy, theta, le, dis, w1, w2, T, mlam};
    memcpy(d.params, p, sizeof(p));
}

void obj_hoop::describe(incrmt_object_desc &d) const {
    d.type = INCRMT_OBJ_HOOP;
    const double p[3] = {r_in, r_out, grav};
    memcpy(d.params, p, sizeof(p));
}

obj_piston::~obj_piston() {
    if (fp != nullptr) fclose(fp);
}

void obj_piston::describe(incrmt_object_desc &d) const {
    d.type = INCRMT_OBJ_PISTON;
    const double p[7] = {lx, ly, cx, y_start, y_end, duration, anch_r};
    memcpy(d.params, p, sizeof(p));
}

/** obj_piston::start_extra (object.cc:224-237). */
void obj_piston::start(fluid_2d &f) {
    std::vector<char> fn(strlen(filename) + 16);
    snprintf(fn.data(), fn.size(), "%s.odr/track.dat", filename);
    fp = open_or_die(fn.data(), "wb");
    printf("# Anchoring K_stiff       : %g (1/T^2)\n", 0.01 / (f.dt_reg * f.dt_reg));
}

/** obj_track::file_output (object.cc:344-351) for the piston's point. */
void obj_piston::track_record(const double *rec) {
    const double out[3] = {rec[0], rec[3], rec[4]};
    fwrite(out, sizeof(double), 3, fp);
}

void obj_piston::write(int k, double time) {
    if (fp != nullptr) fflush(fp);
}

obj_circle_track::~obj_circle_track() {
    if (fp != nullptr) fclose(fp);
}

void obj_circle_track::describe(incrmt_object_desc &d) const {
    d.type = INCRMT_OBJ_CIRCLE_TRACK;
    const double p[6] = {cx, cy, cr, uu, vv, omega};
    memcpy(d.params, p, sizeof(p));
}

/** obj_track::start_extra (object.cc:313-316): the track file. */
void obj_circle_track::start(fluid_2d &f) {
    std::vector<char> fn(strlen(filename) + 16);
    snprintf(fn.data(), fn.size(), "%s.odr/track.dat", filename);
    fp = open_or_die(fn.data(), "wb");
}

/** obj_circle_track::file_output (object.cc:532-549): the angle from the
 * first point's position before its correction to its reference position
 * (-cr/2, 0), unwrapped by the winding count, and its corrected position. */
void obj_circle_track::track_record(const double *rec) {
    const double ang = atan2(0. - rec[2], -0.5 * cr - rec[1]);
    const int q = fabs(ang) > 0.5 * M_PI ? (ang > 0 ? 1 : -1) : 0;
    if (q == 1 && prev_q == -1) wind--;
    else if (q == -1 && prev_q == 1) wind++;
    prev_q = q;
    const double out[4] = {rec[0], rec[3], rec[4], ang + 2 * M_PI * wind};
    fwrite(out, sizeof(double), 4, fp);
}

void obj_circle_track::write(int k, double time) {
    if (fp != nullptr) fflush(fp);
}

// ---------------------------------------------------------------- fluid_2d

void fluid_2d::l_comparison(fluid_2d &f2d, double *err) {
    if (f2d.m % m != 0 || f2d.n % n != 0) {
        fputs("Grid dimension is not a multiple of the finer grid\n", stderr);
        exit(1);
    }
    incrmt_check(incrmt_l_comparison(h, f2d.h, err), "incrmt_l_comparison");
}

double fluid_2d::avg_v_cycles_mac() {
    incrmt_sim_stats st;
    incrmt_check(incrmt_get_stats(h, &st), "incrmt_get_stats");
    const long long dv = st.vcycles_mac - vc_read[0], ds = st.solves_mac - vc_read[1];
    vc_read[0] = st.vcycles_mac;
    vc_read[1] = st.solves_mac;
    return ds ? static_cast<double>(dv) / ds : 0;
}

double fluid_2d::avg_v_cycles_fem() {
    incrmt_sim_stats st;
    incrmt_check(incrmt_get_stats(h, &st), "incrmt_get_stats");
    const long long dv = st.vcycles_fem - vc_read[2], ds = st.solves_fem - vc_read[3];
    vc_read[2] = st.vcycles_fem;
    vc_read[3] = st.solves_fem;
    return ds ? static_cast<double>(dv) / ds : 0;
}

fluid_2d::fluid_2d(int m_, int n_, sim_type &sim_t_, double visc_, double rhof_, double tw_, double pinw_,
                   int ntrace_, unsigned int fflags_, const char *filename_)
    : m(m_), n(n_), ml(m_ + 4), nl(n_ + 4), x_prd(sim_t_.x_prd), y_prd(sim_t_.y_prd), ax(sim_t_.ax),
      bx(sim_t_.bx), ay(sim_t_.ay), by(sim_t_.by), dx((bx - ax) / m_), dy((by - ay) / n_), xsp(1 / dx),
      ysp(1 / dy), visc(visc_), rhof(rhof_), tw(tw_), pinw(pinw_), eps(tw_ * (dx < dy ? dx : dy)),
      ntrace(ntrace_), fflags(fflags_), filename(filename_), dt_reg(0), time(0), f_num(0), zpr(false),
      precision(INCRMT_PREC_FP64), solid_prd_bc(false), coarse_refresh(16), sim_t(sim_t_), h(nullptr), const_rho(true), created(false) {}

/** Objects may already be deleted here (the reference's drivers delete them
 * first), so records not handed out by write_files are dropped. */
fluid_2d::~fluid_2d() {
    if (h != nullptr) incrmt_destroy(h);
}

/** The library handle is made on first use, so that zpr and precision can
 * be set after construction as the reference's public members are. */
void fluid_2d::create() {
    if (created) return;
    incrmt_grid g = {m, n, ax, bx, ay, by, x_prd, y_prd};
    const double U = sim_t.flow_speed();
    if (U != 0) zpr = true;  // sim_horiz_flow::start (sim_type.cc:59-64)
    incrmt_phys p = {visc, rhof, tw, pinw, sim_t.w_scale, sim_t.w_force, ntrace, zpr ? 1 : 0, precision, 1e-9,
                     U != 0 ? 1 : 0, U, sim_t.velocity_pulses() ? 1 : 0};
    incrmt_check(incrmt_create(&g, &p, &h), "incrmt_create");
    created = true;
}

void fluid_2d::add_object(object *o, mat_const &mc) {
    create();
    incrmt_object_desc d;
    memset(&d, 0, sizeof(d));
    o->describe(d);
    d.G = mc.G;
    d.rhos = mc.rhos;
    d.ev_trans_mult = mc.ev_trans_mult;
    d.set_velocity = mc.set_velocity ? 1 : 0;
    incrmt_check(incrmt_add_object(h, &d), "incrmt_add_object");
    olist.push_back(o);
    rhos.push_back(mc.rhos);
}

/** fluid_2d::initialize (fluid_2d.cc:101-122). */
void fluid_2d::initialize(double ev_mult, double dt_pad, double dt_ev_pad) {
    create();
    incrmt_check(incrmt_set_solid_prd_bc(h, solid_prd_bc ? 1 : 0), "incrmt_set_solid_prd_bc");
    incrmt_check(incrmt_sim_set_coarse_refresh(h, coarse_refresh), "incrmt_sim_set_coarse_refresh");
    incrmt_check(incrmt_initialize(h, ev_mult, dt_pad, dt_ev_pad, &dt_reg), "incrmt_initialize");
    printf("# Ex. visc. multiplier    : %g\n"
           "# dt padding (phys)       : %g\n"
           "# dt padding (EV)         : %g\n"
           "# Chosen dtmax            : %g (T)\n",
           ev_mult, dt_pad, dt_ev_pad, dt_reg);
    for (object *o : olist) o->start(*this);
    // fluid_2d::setup_multigrid / same_rho (fluid_2d.cc:126-137, fluid_2d.hh:244-249)
    const_rho = true;
    for (double r : rhos)
        if (fabs(r - rhof) > small_number) const_rho = false;
    puts(const_rho ? "# Constant density" : "# Non-constant density");
    if (ntrace > 0) init_tracers();
    incrmt_check(incrmt_get_time(h, &time), "incrmt_get_time");
}

/** fluid_2d::init_tracers / inside_object / tracer_cell
 * (fluid_2d.cc:1377-1429): uniform random positions outside every solid,
 * judged by the bilinear interpolation of each level set against eps. */
void fluid_2d::init_tracers() {
    std::vector<std::vector<double>> phis(olist.size(), std::vector<double>(static_cast<size_t>(ml) * nl));
    for (size_t k = 0; k < olist.size(); k++)
        incrmt_check(incrmt_get_field(h, INCRMT_FIELD_PHI, static_cast<int>(k), phis[k].data()), "incrmt_get_field");
    std::vector<double> xy(2 * static_cast<size_t>(ntrace));
    for (int t = 0; t < ntrace;) {
        const double tx = rnd(ax, bx), ty = rnd(ay, by);
        double x = (tx - ax) * xsp - 0.5, y = (ty - ay) * ysp - 0.5;
        int i = static_cast<int>(x), j = static_cast<int>(y);
        if (i < -1) i = -1;
        else if (i > m - 1) i = m - 1;
        if (j < -1) j = -1;
        else if (j > n - 1) j = n - 1;
        x -= i;
        y -= j;
        const double fx = 1 - x, fy = 1 - y;
        bool inside = false;
        for (auto &ph : phis) {
            const double *p = ph.data() + (i + 2) + static_cast<size_t>(ml) * (j + 2);
            if (fy * (*p * fx + p[1] * x) + y * (p[ml] * fx + p[ml + 1] * x) < eps) { inside = true; break; }
        }
        if (!inside) { xy[2 * t] = tx; xy[2 * t + 1] = ty; t++; }
    }
    incrmt_check(incrmt_set_tracers(h, xy.data()), "incrmt_set_tracers");
}

void fluid_2d::step_forward(double dt) {
    incrmt_check(incrmt_step(h, dt), "incrmt_step");
    incrmt_check(incrmt_get_time(h, &time), "incrmt_get_time");
}

/** fluid_2d::save_header (fluid_2d_io.cc:13-19). */
void fluid_2d::save_header(double duration, int frames) {
    std::vector<char> fn(strlen(filename) + 16);
    snprintf(fn.data(), fn.size(), "%s/header", filename);
    FILE *f = open_or_die(fn.data(), f_num == 0 ? "w" : "a");
    fprintf(f, "%g %g %d\n", time, time + duration, frames);
    fclose(f);
}

/** fluid_2d::solve (fluid_2d.cc:254-295): the steps of each frame run on the
 * GPU back to back; only the frame's output crosses to the host. */
void fluid_2d::solve(double duration, int frames) {
    double adt;
    const int l = timestep_select(duration / frames, adt);
    const bool timing = (fflags & 8192) != 0;
    incrmt_check(incrmt_sim_set_profiling(h, timing ? 1 : 0), "incrmt_sim_set_profiling");
    save_header(duration, frames);
    if (f_num == 0) write_files(0), puts("# Output frame 0");
    double t0 = wtime();
    incrmt_sim_stats s0;
    incrmt_check(incrmt_get_stats(h, &s0), "incrmt_get_stats");
    for (int k = 1; k <= frames; k++) {
        incrmt_check(incrmt_steps(h, adt, l), "incrmt_steps");
        incrmt_check(incrmt_get_time(h, &time), "incrmt_get_time");
        const double t1 = wtime();
        write_files(k + f_num);
        const double t2 = wtime();
        incrmt_sim_stats s1;
        incrmt_check(incrmt_get_stats(h, &s1), "incrmt_get_stats");
        const long long vm = s1.vcycles_mac - s0.vcycles_mac, vf = s1.vcycles_fem - s0.vcycles_fem;
        const long long nm = s1.solves_mac - s0.solves_mac, nf = s1.solves_fem - s0.solves_fem;
        if (timing) {
            // Projection seconds from CUDA events on the simulation stream.
            double ms[INCRMT_PHASES];
            incrmt_check(incrmt_sim_profile(h, ms), "incrmt_sim_profile");
            printf("%d %d %.8g %.8g  %lld %.8g %lld %.8g\n", k + f_num, l, t1 - t0, t2 - t1, vm,
                   1e-3 * ms[INCRMT_PHASE_MAC], vf, 1e-3 * ms[INCRMT_PHASE_FEM]);
            incrmt_check(incrmt_sim_set_profiling(h, 1), "incrmt_sim_set_profiling");
        } else {
            printf("# Output frame %d [%d, %.8g s, %.8g s] {MAC %.2f, FEM %.2f}\n", k + f_num, l, t1 - t0, t2 - t1,
                   nm > 0 ? static_cast<double>(vm) / nm : 0., nf > 0 ? static_cast<double>(vf) / nf : 0.);
        }
        fflush(stdout);
        s0 = s1;
        t0 = t2;
    }
    f_num += frames;
}

/** Hands the library's tracked-point records to their object. */
void fluid_2d::drain_track_records() {
    int count = 0;
    incrmt_check(incrmt_track_records(h, nullptr, 0, &count, 0), "incrmt_track_records");
    if (count == 0) return;
    object *trk = nullptr;
    for (object *o : olist)
        if (o->tracks()) { trk = o; break; }
    int ntr = 0;
    incrmt_check(incrmt_get_object_tracers(h, nullptr, &ntr), "incrmt_get_object_tracers");
    const size_t rec = 1 + 4 * static_cast<size_t>(ntr);
    dbuf.resize(rec * count);
    incrmt_check(incrmt_track_records(h, dbuf.data(), count, &count, 1), "incrmt_track_records");
    if (trk != nullptr)
        for (int r = 0; r < count; r++) trk->track_record(dbuf.data() + rec * r);
}

/** fluid_2d::write_files (fluid_2d_io.cc:60-110). */
void fluid_2d::write_files(int sn) {
    if (fflags & 1) output("u", 0, sn);
    if (fflags & 2) output("v", 1, sn);
    if (fflags & 4) output("spd", 2, sn);
    if (fflags & 8) output("p", 3, sn);
    if (fflags & 16) output("w", 4, sn);
    if (!const_rho && (fflags & 32)) output("rho", 5, sn);
    if (fflags & 4096) output("div", 12, sn);
    if (!olist.empty() && (fflags & 8640)) {
        if (fflags & 512) {
            int box[4];
            incrmt_check(incrmt_solid_bound(h, box), "incrmt_solid_bound");
            box[0] -= 2; box[1] += 2; box[2] -= 2; box[3] += 2;
            if (box[0] < 0) box[0] = 0;
            if (box[1] > ml) box[1] = ml;
            if (box[2] < 0) box[2] = 0;
            if (box[3] > nl) box[3] = nl;
            if (fflags & 64) output("X", 6, sn, box);
            if (fflags & 128) output("Y", 7, sn, box);
            if (fflags & 256) output("phi", 8, sn, box);
        } else {
            if (fflags & 64) output("X", 6, sn);
            if (fflags & 128) output("Y", 7, sn);
            if (fflags & 256) output("phi", 8, sn);
        }
        if (fflags & 8192) output("J", 9, sn);
    }
    if (fflags & 2048) {
        output("ds", 10, sn);
        output("dp", 11, sn);
    }
    if (ntrace > 0) output_tracers(sn);
    // The tracked point's record at the frame (obj_track::write, object.cc:333-336).
    if (!olist.empty()) {
        incrmt_check(incrmt_record_track(h), "incrmt_record_track");
        drain_track_records();
    }
    for (object *o : olist) o->write(sn, time);
}

/** fluid_2d::output with the default box (fluid_2d_io.cc:108-117). */
void fluid_2d::output(const char *prefix, int mode, int sn) {
    int box[4];
    if (fflags & 1024) {
        const int lo = mode == 4 ? 1 : 0;
        box[0] = lo; box[1] = ml; box[2] = lo; box[3] = nl;
    } else {
        const int dis = ((1 << mode) & (8 | 16 | 512 | 2048)) ? 1 : 2;
        box[0] = 2; box[1] = ml - dis; box[2] = 2; box[3] = nl - dis;
    }
    output(prefix, mode, sn, box);
}

/** fluid_2d::output over a box (fluid_2d_io.cc:123-179): the frame is
 * assembled on the GPU and written as one block of floats. */
void fluid_2d::output(const char *prefix, int mode, int sn, const int box[4]) {
    const int si = box[1] - box[0], sj = box[3] - box[2];
    if (si <= 0 || sj <= 0) return;
    fbuf.resize(static_cast<size_t>(si + 1) * (sj + 1));
    incrmt_check(incrmt_frame(h, mode, box, fbuf.data()), "incrmt_frame");
    std::vector<char> fn(strlen(filename) + strlen(prefix) + 32);
    snprintf(fn.data(), fn.size(), "%s/%s.%d", filename, prefix, sn);
    FILE *f = open_or_die(fn.data(), "wb");
    fwrite(fbuf.data(), sizeof(float), fbuf.size(), f);
    fclose(f);
}

/** fluid_2d::output_tracers (fluid_2d_io.cc:24-57): tracer positions as
 * float pairs. */
void fluid_2d::output_tracers(int sn) {
    dbuf.resize(4 * static_cast<size_t>(ntrace));
    incrmt_check(incrmt_get_tracers(h, dbuf.data()), "incrmt_get_tracers");
    fbuf.resize(2 * static_cast<size_t>(ntrace));
    for (int t = 0; t < ntrace; t++) {
        fbuf[2 * t] = static_cast<float>(dbuf[4 * t]);
        fbuf[2 * t + 1] = static_cast<float>(dbuf[4 * t + 1]);
    }
    std::vector<char> fn(strlen(filename) + 32);
    snprintf(fn.data(), fn.size(), "%s/trace.%d", filename, sn);
    FILE *f = open_or_die(fn.data(), "wb");
    fwrite(fbuf.data(), sizeof(float), fbuf.size(), f);
    fclose(f);
}
