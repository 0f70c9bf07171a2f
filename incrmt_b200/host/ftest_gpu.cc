/* Driver for the GPU simulation with the reference ftest's command line and
 * output (ftest.cc:52-99, 116-143, 380-415) for the scenarios the library
 * covers:
 *
 *   ftest_gpu simple-spin <grid resolution> [<transition width>]
 *             [-d <duration>] [-n <frames>] [-mixed]
 *   ftest_gpu circles <grid resolution> <count> <seed>
 *             [-d <duration>] [-n <frames>] [-mixed]
 *   ftest_gpu flag <mu> <k_B> <Re> <ar> [<perturb_v>]
 *             [-grid <n>] [-d <duration>] [-n <frames>] [-mixed]
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
    bool mixed = false;
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
    if (T_opt > 0) T = T_opt;
    if (frames_opt > 0) num_frames = frames_opt;

    // Output directory (ftest.cc:385-388)
    const std::string fout = fn + ".odr";
    mkdir(fout.c_str(), S_IRWXU | S_IRWXG | S_IROTH | S_IXOTH);

    fluid_2d f2d(m, n, *sim_t, visc, rhof, tw, pinw, ntrace, fflags, fout.c_str());
    if (mixed) f2d.precision = INCRMT_PREC_MIXED;
    for (size_t k = 0; k < obj.size(); k++) f2d.add_object(obj[k], mats[k]);
    f2d.initialize(ev_mult, dt_pad, dt_ev_pad);
    f2d.solve(T, num_frames);

    delete sim_t;
    for (object *o : obj) delete o;
    return 0;
}
