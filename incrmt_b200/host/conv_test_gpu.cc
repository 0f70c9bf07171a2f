/* Grid-convergence study on the GPU with the reference conv_test's command
 * line, scenario and output (conv_test.cc:16-194):
 *
 *   conv_test_gpu <test_number> [-res r0,r1,...] [-n <intervals>] [-mixed]
 *
 * Test types (low three bits): 0/1 fluid only (mu 1e-3 / 4e-3), 2 a solid
 * filling the box with periodic reference maps (fluid_2d::solid_prd_bc, no
 * tracers), 3 solid square (rho_s 1), 4-7 solid circle (rho_s 3, 1, 1, 1; mu
 * 1e-3, 1e-3, 4e-3, 1.6e-2), all in sim_velocity_pulses' doubly periodic
 * [-1,1]^2; bits 8, 16, 32 select the reference's extra-viscosity variants and
 * 64 the longer resolution list.
 *
 * All resolutions are stepped together over 50 intervals of 0.02; after every
 * interval each coarser simulation is compared with the finest
 * (fluid_2d::l_comparison) and its 32 norms are appended to cnv_<type>.dat,
 * one line per interval: "<interval> <time>" then, per coarser grid, the
 * norms in groups of eight (%.14g), as the reference writes them; every
 * coarser grid also writes its frames (pressure and difference fields, plus
 * X, Y, phi with a solid) to cnv_<type>_<k>.odr.
 *
 * Resolutions. The reference's lists (2520, 1260, 840, 630, 504, 420, 360,
 * 315, 280 and a doubled list) contain odd sizes, and sizes whose halving
 * stops at large odd grids; the GPU multigrid halves periodic directions and
 * solves its coarsest level exactly only when it is small. The default lists
 * here keep the reference's shape (every size divides the finest, refinement
 * ratios both odd and even) with sizes that halve down to a few cells:
 * 1536, 768, 512, 384, 256, 192, 128, 96, 64 (bit 64: 3072 first and 48
 * added). -res overrides the list (the first entry the finest; every entry
 * even and dividing it), -n the number of intervals; -mixed runs the
 * projections' V-cycles in FP32 inside FP64 defect correction. */
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <sys/types.h>
#include <vector>

#include "incrmt_host.hh"

namespace {

double wtime() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void usage() {
    fputs("Syntax: ./conv_test_gpu <test_number> [-res r0,r1,...] [-n <intervals>] [-mixed]\n\n"
          "Test type:\n"
          "0: fluid only (mu=1e-3)\n"
          "1: fluid only (mu=4e-3)\n"
          "3: solid square (rho_s=1, mu=1e-3)\n"
          "4: solid circle (rho_s=3, mu=1e-3)\n"
          "5: solid circle (rho_s=1, mu=1e-3)\n"
          "6: solid circle (rho_s=1, mu=4e-3)\n"
          "7: solid circle (rho_s=1, mu=1.6e-2)\n\n"
          "Additional options, assembled bitwise:\n"
          "8: constant extra viscosity\n"
          "16: extra viscosity timestep multiplier halved\n"
          "32: extra viscosity x1.5\n"
          "64: increase max resolution from 1536 to 3072\n",
          stderr);
    exit(1);
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) usage();
    const int type = atoi(argv[1]), ctype = type & 7;
    if (type < 0 || type > 127) {
        fputs("Test number out of range\n", stderr);
        return 1;
    }
    std::vector<int> mtab;
    int nsteps = 50;
    bool mixed = false;
    for (int k = 2; k < argc; k++) {
        if (!strcmp(argv[k], "-res") && k + 1 < argc) {
            for (char *t = strtok(argv[++k], ","); t; t = strtok(nullptr, ",")) mtab.push_back(atoi(t));
        } else if (!strcmp(argv[k], "-n") && k + 1 < argc) nsteps = atoi(argv[++k]);
        else if (!strcmp(argv[k], "-mixed")) mixed = true;
        else usage();
    }
    if (mtab.empty()) {
        mtab = {1536, 768, 512, 384, 256, 192, 128, 96, 64};
        if (type & 64) mtab = {3072, 1536, 1024, 768, 512, 384, 256, 192, 128, 96, 64, 48};
    }
    const int nsim = static_cast<int>(mtab.size());
    if (nsim < 2 || nsteps < 1) usage();
    for (int v : mtab)
        if (v < 8 || (v & 1) || mtab[0] % v) {
            fprintf(stderr, "Resolution %d must be even and divide %d\n", v, mtab[0]);
            return 1;
        }

    // Parameters of conv_test.cc:41-75
    const double tw = 2.5, pinw = 2.5;
    const int ntrace = 512;
    const unsigned int fflags = 8 | 2048 | (ctype == 0 || ctype == 1 ? 0 : 64 | 128 | 256);
    const double rhof = 1, rhos[8] = {1, 1, 1, 1, 3, 1, 1, 1},
                 visc[8] = {1e-3, 4e-3, 1e-20, 1e-3, 1e-3, 1e-3, 4e-3, 16e-3}, G = 1, ev_trans_mult = 1;
    double ev_mult = 0.4, dt_pad = 0.4, dt_ev_pad = 0.8;
    if (type & 16) dt_ev_pad = 0.4;
    if (type & 32) ev_mult = 0.6;
    std::vector<object *> obj;
    if (ctype == 2) obj.push_back(new obj_full());
    else if (ctype == 3) obj.push_back(new obj_square(-0.1, 0, 0.6, 0, 0, 0));
    else if (ctype >= 4) obj.push_back(new obj_circle(-0.1, 0, 0.6, 0, 0, 0));
    const double interval = 0.02;

    sim_velocity_pulses sim_t;
    mat_const mc(G, rhos[ctype], ev_trans_mult, false);
    std::vector<fluid_2d *> f2d(nsim);
    std::vector<std::string> dirs(nsim);
    std::vector<int> l(nsim);
    std::vector<double> adt(nsim);
    for (int k = 0; k < nsim; k++) {
        char buf[64];
        snprintf(buf, sizeof(buf), "cnv_%02d_%d.odr", type, k);
        dirs[k] = buf;
        mkdir(buf, S_IRWXU | S_IRWXG | S_IROTH | S_IXOTH);
        // The full solid runs without tracers and with periodic solid
        // boundary conditions (conv_test.cc:116-120)
        f2d[k] = new fluid_2d(mtab[k], mtab[k], sim_t, visc[ctype], rhof, tw, pinw, ctype == 2 ? 0 : ntrace, fflags,
                              dirs[k].c_str());
        if (mixed) f2d[k]->precision = INCRMT_PREC_MIXED;
        for (object *o : obj) f2d[k]->add_object(o, mc);
        if (ctype == 2) f2d[k]->solid_prd_bc = true;
        f2d[k]->initialize(type & 8 ? (ev_mult * mtab[k] / mtab[nsim - 1]) : ev_mult,
                           dt_pad * mtab[nsim - 1] / mtab[k], dt_ev_pad * mtab[nsim - 1] / mtab[k]);
        l[k] = f2d[k]->timestep_select(interval, adt[k]);
        f2d[k]->save_header(interval * nsteps, nsteps);
        printf("# m=%d, steps=%d, dt=%g\n#\n", mtab[k], l[k], adt[k]);
    }

    char cbuf[32];
    snprintf(cbuf, sizeof(cbuf), "cnv_%02d.dat", type);
    FILE *fp = fopen(cbuf, "w");
    if (!fp) {
        fprintf(stderr, "Can't open file '%s'\n", cbuf);
        return 1;
    }
    std::vector<double> err(32);
    double t0, t1;
    for (int i = 0;; i++) {
        fprintf(fp, "%d %g", i, i * interval);
        for (int k = 1; k < nsim; k++) {
            f2d[k]->l_comparison(*f2d[0], err.data());
            for (int e = 0; e < 32; e += 8)
                fprintf(fp, " %.14g %.14g %.14g %.14g %.14g %.14g %.14g %.14g", err[e], err[e + 1], err[e + 2],
                        err[e + 3], err[e + 4], err[e + 5], err[e + 6], err[e + 7]);
            f2d[k]->write_files(i);
        }
        fputc('\n', fp);
        fflush(fp);
        printf("Timestep %d\n", i);
        if (i == nsteps) break;
        t0 = wtime();
        for (int k = 0; k < nsim; k++) {
            int j0 = 0;
            for (int j = 0; j < l[k]; j++) {
                printf("Grid %d, step %d of %d\r", mtab[k], j, l[k]);
                fflush(stdout);
                f2d[k]->step_forward(adt[k]);
                if (j > 0 && (j % 8 == 0 || j == l[k] - 1)) {
                    t1 = wtime();
                    printf("Grid %d, step %d of %d [%.6g s/step] {MAC %.2f,FEM %.2f}\n", mtab[k], j, l[k],
                           (t1 - t0) / (j - j0), f2d[k]->avg_v_cycles_mac(), f2d[k]->avg_v_cycles_fem());
                    t0 = t1;
                    j0 = j;
                }
            }
        }
    }
    fclose(fp);
    for (fluid_2d *f : f2d) delete f;
    for (object *o : obj) delete o;
    return 0;
}
