/* Times the reference's own CPU step (fluid_2d::step_forward,
 * fluid_2d.cc:298-369) on the simple-spin scenario (ftest.cc:116-143):
 *   ref_run <m> <steps> <warmup> <output base path>
 * and prints one line "steps seconds vcycles_mac vcycles_fem threads dt".
 *
 * TEST INFRASTRUCTURE ONLY (the oracle / CPU baseline); never the product. */
#include <cstdio>
#include <cstdlib>
#include <omp.h>

extern "C" {
void* ref_sspin_create(int m,int ntrace,const char *base);
void ref_destroy(void *h);
void ref_scalars(void *h,double *out);
void ref_steps(void *h,int steps,double dt);
int ref_vcycles(void *h,int which,int reset);
}

int main(int argc,char **argv) {
    if(argc!=5) {
        fputs("Syntax: ref_run <m> <steps> <warmup> <output base path>\n",stderr);
        return 1;
    }
    int m=atoi(argv[1]),steps=atoi(argv[2]),warm=atoi(argv[3]);
    void *h=ref_sspin_create(m,512,argv[4]);
    double sc[6];
    ref_scalars(h,sc);
    // The step size that solve(2*pi,120) would choose (fluid_2d.hh:173-177)
    double interval=2*3.14159265358979323846/120;
    int l=static_cast<int>(interval/sc[0])+1;
    double dt=interval/l;
    ref_steps(h,warm,dt);
    ref_vcycles(h,0,1);ref_vcycles(h,1,1);
    double t0=omp_get_wtime();
    ref_steps(h,steps,dt);
    double t1=omp_get_wtime();
    int vm=ref_vcycles(h,0,1),vf=ref_vcycles(h,1,1);
    printf("%d %.9g %d %d %d %.12g\n",steps,t1-t0,vm,vf,omp_get_max_threads(),dt);
    ref_destroy(h);
    return 0;
}
