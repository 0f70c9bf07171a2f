/* Driver for the GPU simulation with the reference ftest's command line and
 * output (ftest.cc:52-99, 116-143, 380-415) for the scenarios the library
 * covers:
 *
 *   ftest_gpu simple-spin <grid resolution> [<transition width>]
 *   ftest_gpu circ-move | square | seven-star | fluid | flapper | flappers | full
 *             <grid resolution>
 *   ftest_gpu piston <shear modulus> [-grid <m>]
 *   ftest_gpu multi-drop <grid resolution> <type: 0 circles, 1 squares>
 *   ftest_gpu circles <grid resolution> <count> <seed>
 *   ftest_gpu flag <mu> <k_B> <Re> <ar> [<perturb_v>] [-grid <n>]
 *   (each with [-d <duration>] [-n <frames>] [-mixed])
 *
 * circ-move, square, seven-star, piston, fluid, flapper, flappers,
 * multi-drop and full are ftest's scenarios of those names (ftest.cc:144-333) with its
 * parameters, output directory (<scenario>.odr, piston_G<G>.odr) and the C
 * library's rand() drawing the flappers' and drops' placements in the same
 * order; square, seven-star and fluid run in ftest's default doubly periodic
 * box (sim_type(), fluid starting at rest or, for fluid, with
 * sim_velocity_pulses). The reference's multi-drop checks for three
 * arguments and then reads a fourth (ftest.cc:294-296), so it cannot run as
 * written; here it takes the documented <grid resolution> <type>. -grid m
 * runs the piston on m x 5m/2 instead of ftest's 320 x 800. full fills the
 * pulses' doubly periodic box with one solid whose reference map is periodic
 * up to the box lengths (fluid_2d::solid_prd_bc).
 *
 * simple-spin is the reference's three-pronged rotor scenario: output in
 * sspin_<m>.odr (or sspin_<m>_tw<tw>.odr), 240 frames over 4 pi. circles
 * drops <count> seeded non-overlapping circles (radii 0.03-0.06, densities
 * 1.5-3, G 1) under gravity in a walled [-0.75,0.75]x[-1.5,1.5] box of
 * m x 2m cells (the geometry of the reference's sediment driver,
 * sediment.cc:22,124), output in circles_<m>_<count>.odr. flag is the
 * reference's flapping flag in a uniform inflow (ftest.cc:335-378): mass
 * ratio, bending rigidity, Reynolds number, aspect ratio and an optional tip
 * velocity perturbation, on 3n x n cells of [-1,5]x[-1,1] (n = 608 unless
 * -grid is given), output in fl_<mu>_<k_B>_<Re>_<ar>[_<perturb_v>].odr.
 * -d and -n shorten a run; -mixed runs the projections' V-cycles in FP32
 * inside FP64 defect correction. */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <sys/stat.h>
#include <sys/types.h>
#include <vector>

#include "incrmt_host.hh"

namespace {

bool se(const char *p1, const char *p2) { return strcmp(p1, p2) == 0; }

/** Random number in [a, b] from the C library's rand() (common.hh:28-30). */
double rnd(double a, double b) { return a + ((b - a) / RAND_MAX) * static_cast<double>(rand()); }

void check_grid(int m) {
    if (m < 20 || m > 65536) {
        fprintf(stderr, "Supplied grid resolution of %d is too %s\n", m, m < 20 ? "small" : "large");
        exit(1);
    }
}

void usage() {
    fputs("Syntax: ./ftest_gpu <sim_type> {extra options} [-d <duration>] [-n <frames>] [-grid <n>] [-mixed]\n\n"
          "Simulation types:\n"
          "simple-spin     simple three-pronged rotor: <grid resolution> [<transition width>]\n"
          "circ-move       circle moving through fluid: <grid resolution>\n"
          "square          rotating square: <grid resolution>\n"
          "seven-star      rotating seven-pointed star: <grid resolution>\n"
          "piston          flexible paddle moving through cavity: <shear modulus>\n"
          "fluid           fluid only: <grid resolution>\n"
          "flapper         single flapping swimmer: <grid resolution>\n"
          "flappers        multiple flapping swimmers: <grid resolution>\n"
          "multi-drop      multiple objects sedimenting: <grid resolution> <type>\n"
          "full            full solid with periodic boundaries: <grid resolution>\n"
          "circles         seeded circles settling under gravity: <grid resolution> <count> <seed>\n"
          "flag            flapping flag: <mu> <k_B> <Re> <ar> [<perturb_v>]\n",
          stderr);
    exit(1);
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) usage();

    // Trailing options of this driver
    double T_opt = -1;
    int frames_opt = -1, grid_opt = -1;
    bool mixed = false, solid_prd_bc = false;
    std::vector<char *> pos;
    for (int k = 1; k < argc; k++) {
        if (se(argv[k], "-d") && k + 1 < argc) T_opt = atof(argv[++k]);
        else if (se(argv[k], "-n") && k + 1 < argc) frames_opt = atoi(argv[++k]);
        else if (se(argv[k], "-grid") && k + 1 < argc) grid_opt = atoi(argv[++k]);
        else if (se(argv[k], "-mixed")) mixed = true;
        else pos.push_back(argv[k]);
    }
    const int np = static_cast<int>(pos.size());
    if (np == 0) usage();

    // Defaults of the reference driver (ftest.cc:70-99)
    int m = 200, n = 200;
    double T = 4;
    int num_frames = 200;
    double tw = 2.5, pinw = 2.5;
    int ntrace = 512;
    unsigned int fflags = 8 | 16 | 64 | 128 | 256 | 512;
    double rhof = 1, rhos = 1, visc = 1e-3, G = 24;
    double ev_mult = 0.8, ev_trans_mult = 1, dt_pad = 0.4, dt_ev_pad = 0.8;

    sim_type *sim_t = nullptr;
    std::string fn;
    std::vector<object *> obj;
    std::vector<mat_const> mats;

    if (se(pos[0], "simple-spin")) {
        if (np < 2 || np > 3) usage();
        if (np == 2) {
            fn = std::string("sspin_") + pos[1];
            num_frames = 240;
        } else {
            fn = std::string("sspin_") + pos[1] + "_tw" + pos[2];
            tw = atof(pos[2]);
            fflags |= 8192 | 4096;
        }
        m = n = atoi(pos[1]);
        check_grid(m);
        G = 48; visc = 1e-2; rhos = 3;
        T = 4 * M_PI;
        obj.push_back(new obj_simple_spin(0.8, 0.5, 0.125, 0.2, M_PI, 1, strdup(fn.c_str())));
        mats.emplace_back(G, rhos, ev_trans_mult, true);
        sim_t = new sim_type(-1, 1, -1, 1, false, false);
    } else if (se(pos[0], "circ-move")) {
        if (np != 2) usage();
        m = n = atoi(pos[1]);
        check_grid(m);
        rhos = 4; visc = 1e-3;
        T = 3.; num_frames = 300;
        fn = pos[0];
        obj.push_back(new obj_circle_track(-0.5, -0.5, 0.25, 2, 4, 24, strdup(fn.c_str())));
        sim_t = new sim_type(-1, 1, -1, 1, false, false);
    } else if (se(pos[0], "square")) {
        if (np != 2) usage();
        m = n = atoi(pos[1]);
        check_grid(m);
        rhos = 3;
        fn = pos[0];
        obj.push_back(new obj_square(-0.02, 0, 0.5, 0.01, 0, 2));
    } else if (se(pos[0], "seven-star")) {
        if (np != 2) usage();
        m = n = atoi(pos[1]);
        check_grid(m);
        rhos = 3;
        T = 4 * M_PI; num_frames = 600;
        fn = pos[0];
        obj.push_back(new obj_seven_point(0, 0, 0.62, 0.16, M_PI, 1));
    } else if (se(pos[0], "piston")) {
        if (np != 2) usage();
        fn = std::string("piston_G") + pos[1];
        G = atof(pos[1]);
        if (G <= 0) {
            fputs("The shear modulus must be positive\n", stderr);
            return 1;
        }
        m = 320; n = 800;
        if (grid_opt > 0) { m = grid_opt; n = grid_opt * 5 / 2; }
        T = 20; num_frames = 1000;
        rhos = 2.;
        obj.push_back(new obj_piston(0.8, 0.2, 0.6, 0.4, 4.6, 10, 0.15, strdup(fn.c_str())));
        sim_t = new sim_type(-1, 1, 0, 5, false, false);
    } else if (se(pos[0], "fluid")) {
        if (np != 2) usage();
        m = n = atoi(pos[1]);
        check_grid(m);
        visc = 1e-3;
        T = 20; num_frames = 200;
        ntrace = 256;
        fn = pos[0];
        sim_t = new sim_velocity_pulses;
    } else if (se(pos[0], "flapper")) {
        if (np != 2) usage();
        m = n = atoi(pos[1]);
        check_grid(m);
        rhos = 4; G = 10; visc = 5e-4;
        T = 30; num_frames = 600;
        fn = pos[0];
        obj.push_back(new obj_flapper(0, -0.8, 0.026, 0.25, 0.021, 0.14, 0, 2.2, 8));
        sim_t = new sim_type(-1.5, 1.5, -1.5, 1.5, false, false);
    } else if (se(pos[0], "flappers")) {
        if (np != 2) usage();
        m = n = atoi(pos[1]);
        check_grid(m);
        rhos = 4; G = 10; visc = 5e-4;
        T = 30; num_frames = 1200;
        fn = pos[0];
        // 28 non-overlapping flappers at random positions (ftest.cc:262-288)
        const int cnum = 28;
        const double wx = 0.25 + 0.026 + 0.01, wy = 0.026 + 0.01;
        std::vector<double> px, py;
        while (static_cast<int>(px.size()) < cnum) {
            const double x = rnd(-1, 1), y = rnd(-1, 1);
            if (x + wx > 0.98 || x - wx < -0.98 || y + wy > 0.98 || y - wy < -0.98) continue;
            bool good = true;
            for (size_t j = 0; j < px.size(); j++)
                if (fabs(x - px[j]) < 2 * wx && fabs(y - py[j]) < 2 * wy) { good = false; break; }
            if (good) {
                px.push_back(x);
                py.push_back(y);
                obj.push_back(new obj_flapper(x, y, 0.026, 0.25, 0.021, 0.14, 0, 2.2, rnd(7, 9)));
            }
        }
        sim_t = new sim_type(-1, 1, -1, 1, false, false);
    } else if (se(pos[0], "multi-drop")) {
        if (np != 3) usage();
        const bool square = atoi(pos[2]) == 1;
        m = n = atoi(pos[1]);
        check_grid(m);
        rhos = 3; G = 2; visc = 1e-3;
        T = 25; num_frames = 1200;
        fn = pos[0];
        // 42 non-overlapping circles or squares at random positions
        // (ftest.cc:305-330); the stored radius is r - 0.05
        const int cnum = 42;
        std::vector<double> px, py, pr;
        while (static_cast<int>(px.size()) < cnum) {
            const double x = rnd(-1, 1), y = rnd(-1, 1), r = rnd(0.1, 0.25);
            if (x + r > 1 || x - r < -1 || y + r > 1 || y - r < -1) continue;
            bool good = true;
            for (size_t j = 0; j < px.size(); j++) {
                const double dr = pr[j] + r;
                if (fabs(x - px[j]) < dr && fabs(y - py[j]) < dr) { good = false; break; }
            }
            if (good) {
                px.push_back(x);
                py.push_back(y);
                pr.push_back(r - 0.05);
                if (square) obj.push_back(new obj_square(x, y, r - 0.05, 0, 0, rnd(-5, 5)));
                else obj.push_back(new obj_circle(x, y, r - 0.05, 0, 0, rnd(-5, 5)));
            }
        }
        sim_t = new sim_type(-1, 1, -1, 1, false, false);
    } else if (se(pos[0], "full")) {
        // A solid filling the doubly periodic box, starting with the pulses'
        // velocity; no tracers, periodic reference maps (ftest.cc:218-237)
        if (np != 2) usage();
        m = n = atoi(pos[1]);
        check_grid(m);
        rhos = 1; G = 3; visc = 1e-3;
        T = 1; num_frames = 200;
        ntrace = 0;
        solid_prd_bc = true;
        fn = pos[0];
        obj.push_back(new obj_full());
        mats.emplace_back(G, rhos, ev_trans_mult, false);
        sim_t = new sim_velocity_pulses;
    } else if (se(pos[0], "circles")) {
        if (np != 4) usage();
        m = atoi(pos[1]);
        n = 2 * m;
        check_grid(m);
        const int count = atoi(pos[2]);
        const unsigned long seed = strtoul(pos[3], nullptr, 10);
        fn = std::string("circles_") + pos[1] + "_" + pos[2];
        visc = 1e-2; T = 2; num_frames = 100;
        ntrace = 0;
        // Rejection-sampled non-overlapping circles (as sediment.cc:91-121
        // places its bodies): each new centre keeps a gap of 0.02 from the
        // others and from the walls.
        std::mt19937_64 rng(seed);
        std::uniform_real_distribution<double> U(0, 1);
        const double lx = 0.75, ly = 1.5, gap = 0.02;
        std::vector<double> cx, cy, cr;
        int tries = 0;
        while (static_cast<int>(cx.size()) < count) {
            if (++tries > 1000000) { fputs("Could not place the circles\n", stderr); return 1; }
            const double r = 0.03 + 0.03 * U(rng);
            const double x = -lx + r + gap + (2 * (lx - r - gap)) * U(rng);
            const double y = -ly + r + gap + (2 * (ly - r - gap)) * U(rng);
            bool ok = true;
            for (size_t q = 0; q < cx.size() && ok; q++)
                ok = std::hypot(x - cx[q], y - cy[q]) > r + cr[q] + gap;
            if (!ok) continue;
            cx.push_back(x); cy.push_back(y); cr.push_back(r);
            const double rs = 1.5 + 1.5 * U(rng);
            obj.push_back(new obj_circle(x, y, r, (rs - 1) / rs));
            mats.emplace_back(1.0, rs, ev_trans_mult, true);
        }
        sim_t = new sim_type(-lx, lx, -ly, ly, false, false);
    } else if (se(pos[0], "flag")) {
        if (np < 5 || np > 6) {
            fprintf(stderr, "Selected option requires 4 or 5 arguments (%d supplied)\n", np - 1);
            return 1;
        }
        const double mu = atof(pos[1]), k_B = atof(pos[2]), Re = atof(pos[3]), ar = atof(pos[4]),
                     perturb_v = np == 6 ? atof(pos[5]) : 0;
        n = grid_opt > 0 ? grid_opt : 608;
        m = 3 * n;
        const double flag_L = 1, flag_w = 1. / ar, U = 1, flag_a = flag_w * 0.25;
        const int flag_ntrace = 17;
        fn = std::string("fl_") + pos[1] + "_" + pos[2] + "_" + pos[3] + "_" + pos[4];
        if (np == 6) fn += std::string("_") + pos[5];
        sim_t = new sim_horiz_flow(U, -1, 5, -1, 1);
        obj.push_back(new obj_flag(0, 0, flag_L, flag_w, flag_a, perturb_v, flag_ntrace, strdup(fn.c_str())));
        rhof = 1;
        rhos = mu * rhof * flag_L / flag_w;
        visc = U * flag_L * rhof / Re;
        if (np == 6) { T = 160; num_frames = 80; } else { T = 30; num_frames = 900; }
        G = 4 * k_B / (flag_w * flag_w * flag_w);
        mats.emplace_back(G, rhos, ev_trans_mult, true);
        printf("# Shear modulus                : %g (M/LT^2)\n"
               "# Flag width                   : %g dy\n"
               "# Solid density                : %g\n#\n",
               G, 0.5 * flag_w * n, rhos);
    } else {
        fprintf(stderr, "Simulation type '%s' not recognized\n", pos[0]);
        return 1;
    }
    if (sim_t == nullptr) sim_t = new sim_type();  // ftest's default: doubly periodic [-1,1]^2
    // ftest's one mat_const for every object (ftest.cc:395)
    while (mats.size() < obj.size()) mats.emplace_back(G, rhos, ev_trans_mult, true);
    if (T_opt > 0) T = T_opt;
    if (frames_opt > 0) num_frames = frames_opt;

    // Output directory (ftest.cc:385-388)
    const std::string fout = fn + ".odr";
    mkdir(fout.c_str(), S_IRWXU | S_IRWXG | S_IROTH | S_IXOTH);

    fluid_2d f2d(m, n, *sim_t, visc, rhof, tw, pinw, ntrace, fflags, fout.c_str());
    if (mixed) f2d.precision = INCRMT_PREC_MIXED;
    f2d.solid_prd_bc = solid_prd_bc;
    for (size_t k = 0; k < obj.size(); k++) f2d.add_object(obj[k], mats[k]);
    f2d.initialize(ev_mult, dt_pad, dt_ev_pad);
    f2d.solve(T, num_frames);

    delete sim_t;
    for (object *o : obj) delete o;
    return 0;
}
