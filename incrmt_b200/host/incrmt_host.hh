/* Host-side classes with the names, constructor arguments, call sequence,
 * stdout lines and output files of IncRMT's simulation classes (fluid_2d,
 * sim_type, mat_const and the object types; fluid_2d.hh:29-178,
 * sim_type.hh:22-81, obj_field.hh:15-29, object.hh), driving the GPU through
 * the C ABI of libincrmt_gpu.so. A program written against the reference's
 * fluid_2d (such as its ftest driver) builds against these classes unchanged
 * for the scenarios they cover: walled domains with simple-spin rotors and
 * circles. Errors from the library print the library's message to stderr and
 * exit with status 1, the reference's own convention (mgs_mac.cc:31-34). */
#ifndef INCRMT_HOST_HH
#define INCRMT_HOST_HH

#include <cstdio>
#include <vector>

#include "incrmt.h"
#include "incrmt_sim.h"

class fluid_2d;

/** Default size of the boundary repulsion region, in multiples of eps
 * (sim_type.hh:14). */
const double w_scale_default = 3.;
/** Default boundary repulsion force (sim_type.hh:17). */
const double w_force_default = 20.;

/** Simulation geometry and boundary periodicity (sim_type.hh:22-81). */
struct sim_type {
    const double ax, bx, ay, by;
    const double w_scale, w_force;
    const bool x_prd, y_prd;
    sim_type() : ax(-1), bx(1), ay(-1), by(1), w_scale(w_scale_default), w_force(w_force_default),
                 x_prd(true), y_prd(true) {}
    sim_type(double ax_, double bx_, double ay_, double by_, bool x_prd_, bool y_prd_)
        : ax(ax_), bx(bx_), ay(ay_), by(by_), w_scale(w_scale_default), w_force(w_force_default),
          x_prd(x_prd_), y_prd(y_prd_) {}
    sim_type(double ax_, double bx_, double ay_, double by_, bool x_prd_, bool y_prd_, double w_scale_,
             double w_force_)
        : ax(ax_), bx(bx_), ay(ay_), by(by_), w_scale(w_scale_), w_force(w_force_), x_prd(x_prd_), y_prd(y_prd_) {}
    virtual ~sim_type() {}
    /** Horizontal inflow speed of sim_horiz_flow, or 0. */
    virtual double flow_speed() const { return 0; }
    /** Whether the fluid starts with sim_velocity_pulses' velocity. */
    virtual bool velocity_pulses() const { return false; }
};

/** Six incompressible Gaussian velocity pulses on the doubly periodic
 * [-1,1]^2 (sim_velocity_pulses, sim_type.hh:99-114, sim_type.cc:43-47);
 * the scenario of conv_test. */
struct sim_velocity_pulses : public sim_type {
    sim_velocity_pulses() : sim_type(-1, 1, -1, 1, true, true) {}
    bool velocity_pulses() const override { return true; }
};

/** Uniform flow entering through the left edge of a y-periodic channel with
 * zero pressure on the right edge (sim_horiz_flow, sim_type.hh:117-141). */
struct sim_horiz_flow : public sim_type {
    const double U;
    sim_horiz_flow(double U_, double ax_, double bx_, double ay_, double by_)
        : sim_type(ax_, bx_, ay_, by_, false, true), U(U_) {}
    double flow_speed() const override { return U; }
};

/** Material constants of a solid (obj_field.hh:15-29). */
struct mat_const {
    double G, rhos, ev_trans_mult;
    bool set_velocity;
    mat_const(double G_, double rhos_, double ev_trans_mult_, bool set_velocity_ = true)
        : G(G_), rhos(rhos_), ev_trans_mult(ev_trans_mult_), set_velocity(set_velocity_) {}
};

/** A solid's geometry and forcing, described to the GPU as a plain record. */
struct object {
    virtual ~object() {}
    /** Fills the type and geometry fields of the library's object record. */
    virtual void describe(incrmt_object_desc &d) const = 0;
    /** Called by fluid_2d::initialize after the time step is chosen
     * (object::start, fluid_2d.cc:114-115). */
    virtual void start(fluid_2d &f) {}
    /** Whether the object tracks points (obj_track); the library tracks the
     * points of the first such object. */
    virtual bool tracks() const { return false; }
    /** Called with each tracked-point record the library collected: the
     * time, then per point its position before and after the correction. */
    virtual void track_record(const double *rec) {}
    /** Flushes per-object output at a frame (object::write, fluid_2d_io.cc:107). */
    virtual void write(int k, double time) {}
};

/** Three-pronged rotor pinned at its centre, spun by a stiff anchor
 * (object.hh:418-470). Writes <filename>.odr/track.dat: records of four
 * doubles (time, x, y, unwrapped angle) for the tracked point
 * (obj_simple_spin::file_output, object.cc:202-219). */
struct obj_simple_spin : public object {
    const double r_scale, a1, a2, piv_r, th_max, omega;
    const char *filename;
    FILE *fp;
    int prev_q, wind;
    double K_stiff;
    obj_simple_spin(double r_scale_, double a1_, double a2_, double piv_r_, double th_max_, double omega_,
                    const char *filename_)
        : r_scale(r_scale_), a1(a1_), a2(a2_), piv_r(piv_r_), th_max(th_max_), omega(omega_),
          filename(filename_), fp(nullptr), prev_q(0), wind(0), K_stiff(0) {}
    ~obj_simple_spin();
    void describe(incrmt_object_desc &d) const override;
    void start(fluid_2d &f) override;
    bool tracks() const override { return true; }
    void track_record(const double *rec) override;
    void write(int k, double time) override;
};

/** Flag of length flag_l and width flag_w anchored around (cx, cy), tracking
 * ntrace points along its length (obj_flag, object.hh:471-505). Writes
 * <filename>.odr/track.dat: records of 1+2*ntrace doubles (time, then each
 * point's corrected position; obj_track::file_output, object.cc:344-351). */
struct obj_flag : public object {
    const double cx, cy, flag_l, flag_w, flag_a, perturb_v;
    const int ntrace;
    const char *filename;
    FILE *fp;
    obj_flag(double cx_, double cy_, double flag_l_, double flag_w_, double flag_a_, double perturb_v_,
             int ntrace_, const char *filename_)
        : cx(cx_), cy(cy_), flag_l(flag_l_), flag_w(flag_w_), flag_a(flag_a_), perturb_v(perturb_v_),
          ntrace(ntrace_), filename(filename_), fp(nullptr) {}
    ~obj_flag();
    void describe(incrmt_object_desc &d) const override;
    void start(fluid_2d &f) override;
    bool tracks() const override { return true; }
    void track_record(const double *rec) override;
    void write(int k, double time) override;
};

/** Circle of radius cr centred at (cx, cy) with an initial velocity and
 * spin and a downward acceleration grav (object.hh:124-137). */
struct obj_circle : public object {
    const double cx, cy, cr, uu, vv, omega, grav;
    obj_circle(double cx_, double cy_, double cr_, double grav_ = 0)
        : cx(cx_), cy(cy_), cr(cr_), uu(0), vv(0), omega(0), grav(grav_) {}
    obj_circle(double cx_, double cy_, double cr_, double uu_, double vv_, double omega_, double grav_ = 0)
        : cx(cx_), cy(cy_), cr(cr_), uu(uu_), vv(vv_), omega(omega_), grav(grav_) {}
    void describe(incrmt_object_desc &d) const override;
};

/** Square of half side cr centred at (cx, cy) with an initial velocity and
 * spin and a downward acceleration grav (obj_square, object.hh:142-152). */
struct obj_square : public object {
    const double cx, cy, cr, uu, vv, omega, grav;
    obj_square(double cx_, double cy_, double cr_, double grav_ = 0)
        : cx(cx_), cy(cy_), cr(cr_), uu(0), vv(0), omega(0), grav(grav_) {}
    obj_square(double cx_, double cy_, double cr_, double uu_, double vv_, double omega_, double grav_ = 0)
        : cx(cx_), cy(cy_), cr(cr_), uu(uu_), vv(vv_), omega(omega_), grav(grav_) {}
    void describe(incrmt_object_desc &d) const override;
};

/** A solid filling the whole domain (obj_full, object.hh:83-86), used with
 * fluid_2d::solid_prd_bc. */
struct obj_full : public object {
    void describe(incrmt_object_desc &d) const override { d.type = INCRMT_OBJ_FULL; }
};

/** Equilateral triangle with vertices cr from (cx, cy), rotated by theta,
 * falling under grav (obj_triangle, object.hh:155-172). */
struct obj_triangle : public object {
    const double cx, cy, cr, theta, grav;
    obj_triangle(double cx_, double cy_, double cr_, double theta_, double grav_)
        : cx(cx_), cy(cy_), cr(cr_), theta(theta_), grav(grav_) {}
    void describe(incrmt_object_desc &d) const override;
};

/** Swimmer of length le (head dis, half-widths w1 at the neck and w2 at the
 * tail) at (cx, cy) rotated by theta, driven by a contraction wave of period
 * T and maximum contraction mlam (obj_lamprey, object.hh:542-595). */
struct obj_lamprey : public object {
    const double cx, cy, theta, le, dis, w1, w2, T, mlam;
    obj_lamprey(double cx_, double cy_, double theta_, double le_, double dis_, double w1_, double w2_, double T_,
                double mlam_)
        : cx(cx_), cy(cy_), theta(theta_), le(le_), dis(dis_), w1(w1_), w2(w2_), T(T_), mlam(mlam_) {}
    void describe(incrmt_object_desc &d) const override;
};

/** Hoop of radii r_in, r_out about the origin (obj_hoop, object.hh:598-611);
 * grav is kept and, as in the reference, never applied. */
struct obj_hoop : public object {
    const double r_in, r_out, grav;
    obj_hoop(double r_in_, double r_out_, double grav_ = 0) : r_in(r_in_), r_out(r_out_), grav(grav_) {}
    void describe(incrmt_object_desc &d) const override;
};

/** Seven-pointed star of tip radius cr centred at (cx, cy), spun back and
 * forth by a stiff anchor of radius piv_r (obj_seven_point,
 * object.hh:176-213). */
struct obj_seven_point : public object {
    const double cx, cy, cr, piv_r, th_max, omega;
    obj_seven_point(double cx_, double cy_, double cr_, double piv_r_, double th_max_, double omega_)
        : cx(cx_), cy(cy_), cr(cr_), piv_r(piv_r_), th_max(th_max_), omega(omega_) {}
    void describe(incrmt_object_desc &d) const override;
    void start(fluid_2d &f) override;
};

/** Rounded rod that swims by periodically contracting its core
 * (obj_flapper, object.hh:245-285): caps of radius cr, half-length cl, an
 * actuated region of caps ar and half-length al, rotated by theta, a maximum
 * stretch m_stretch and a period T. */
struct obj_flapper : public object {
    const double cx, cy, cr, cl, ar, al, theta, m_stretch, T;
    obj_flapper(double cx_, double cy_, double cr_, double cl_, double ar_, double al_, double theta_,
                double m_stretch_, double T_)
        : cx(cx_), cy(cy_), cr(cr_), cl(cl_), ar(ar_), al(al_), theta(theta_), m_stretch(m_stretch_), T(T_) {}
    void describe(incrmt_object_desc &d) const override;
};

/** Flexible block of half-size lx x ly dragged by an anchor of radius anch_r
 * at x = cx that moves from y_start to y_end over the duration, tracking the
 * point (-cx, y_start) (obj_piston, object.hh:369-418). Writes
 * <filename>.odr/track.dat: records of three doubles (time, corrected x, y;
 * obj_track::file_output, object.cc:344-351). */
struct obj_piston : public object {
    const double lx, ly, cx, y_start, y_end, duration, anch_r;
    const char *filename;
    FILE *fp;
    obj_piston(double lx_, double ly_, double cx_, double y_start_, double y_end_, double duration_, double anch_r_,
               const char *filename_)
        : lx(lx_), ly(ly_), cx(cx_), y_start(y_start_), y_end(y_end_), duration(duration_), anch_r(anch_r_),
          filename(filename_), fp(nullptr) {}
    ~obj_piston();
    void describe(incrmt_object_desc &d) const override;
    void start(fluid_2d &f) override;
    bool tracks() const override { return true; }
    void track_record(const double *rec) override;
    void write(int k, double time) override;
};

/** Circle of radius cr centred at (cx, cy) moving and spinning, tracking the
 * points (cx -+ cr/2, cy) (obj_circle_track, object.hh:509-538). Writes
 * <filename>.odr/track.dat: records of four doubles (time, the first point's
 * corrected position, the unwrapped angle from that point to its reference
 * position; obj_circle_track::file_output, object.cc:532-549). */
struct obj_circle_track : public object {
    const double cx, cy, cr, uu, vv, omega;
    const char *filename;
    FILE *fp;
    int prev_q, wind;
    obj_circle_track(double cx_, double cy_, double cr_, double uu_, double vv_, double omega_,
                     const char *filename_)
        : cx(cx_), cy(cy_), cr(cr_), uu(uu_), vv(vv_), omega(omega_), filename(filename_), fp(nullptr), prev_q(0),
          wind(0) {}
    ~obj_circle_track();
    void describe(incrmt_object_desc &d) const override;
    void start(fluid_2d &f) override;
    bool tracks() const override { return true; }
    void track_record(const double *rec) override;
    void write(int k, double time) override;
};

/** The fluid-structure simulation (fluid_2d.hh:29-178): same constructor,
 * add_object / initialize / solve / step_forward / write_files sequence and
 * output directory layout. The state lives on the GPU. */
class fluid_2d {
    public:
        const int m, n, ml, nl;
        const bool x_prd, y_prd;
        const double ax, bx, ay, by, dx, dy, xsp, ysp;
        const double visc, rhof, tw, pinw, eps;
        const int ntrace;
        const unsigned int fflags;
        const char *filename;
        /** Time step limit chosen by initialize (fluid_2d.hh:107). */
        double dt_reg;
        /** Simulation time (fluid_2d.hh:105), updated after every step. */
        double time;
        /** Frames written so far by solve (fluid_2d.hh:83). */
        int f_num;
        /** Right-edge zero-pressure condition (fluid_2d.hh:117-121). */
        bool zpr;
        /** Precision of the projections' V-cycles: INCRMT_PREC_FP64 (the
         * reference's) or INCRMT_PREC_MIXED; set before initialize. */
        int precision;
        /** Periodic reference maps up to the box lengths, with no wall force
         * (fluid_2d.hh:124); set before initialize. */
        bool solid_prd_bc;
        /** Projections between rebuilds of the multigrid's Galerkin coarse
         * operators (incrmt_sim_set_coarse_refresh); 1 rebuilds them on every
         * density change as the reference does. Set before initialize. */
        int coarse_refresh;
        fluid_2d(int m_, int n_, sim_type &sim_t_, double visc_, double rhof_, double tw_, double pinw_,
                 int ntrace_, unsigned int fflags_, const char *filename_);
        ~fluid_2d();
        void add_object(object *o, mat_const &mc);
        void initialize(double ev_mult, double dt_pad, double dt_ev_pad);
        void solve(double duration, int frames);
        void step_forward(double dt);
        void write_files(int sn);
        void save_header(double duration, int frames);
        /** Error norms against the finer simulation f2d (fluid_2d::l_comparison,
         * fluid_2d_io.cc:186-281): 32 doubles into err. */
        void l_comparison(fluid_2d &f2d, double *err);
        /** Mean V-cycles per MAC / FEM projection since the previous call
         * (mgs_base::avg_v_cycles resets its counters when read,
         * mgs_common.hh:59-65). */
        double avg_v_cycles_mac();
        double avg_v_cycles_fem();
        /** Steps of size adt <= dt_reg that cover interval (fluid_2d.hh:173-177). */
        inline int timestep_select(double interval, double &adt) {
            int l = static_cast<int>(interval / dt_reg) + 1;
            adt = interval / l;
            return l;
        }
        /** The library handle, for callers that need the rest of the C ABI. */
        incrmt_sim *handle() { return h; }
    private:
        sim_type &sim_t;
        incrmt_sim *h;
        std::vector<object *> olist;
        std::vector<double> rhos;
        std::vector<float> fbuf;
        std::vector<double> dbuf;
        bool const_rho;
        bool created;
        long long vc_read[4] = {0, 0, 0, 0};  // MAC V-cycles, solves, FEM V-cycles, solves at the last read
        void create();
        void output(const char *prefix, int mode, int sn);
        void output(const char *prefix, int mode, int sn, const int box[4]);
        void output_tracers(int sn);
        void init_tracers();
        void drain_track_records();
};

/** Prints the library's last error and exits when r is not INCRMT_OK. */
void incrmt_check(int r, const char *what);

#endif
