/* The reference's ftest simple-spin run (ftest.cc:116-143, 383-400) with a
 * chosen duration and frame count, so that its output directory can be
 * compared file by file with the GPU driver's:
 *   ref_ftest <m> <duration> <frames> <output base path>
 * writes <output base path>.odr/{header,p.K,w.K,X.K,Y.K,phi.K,trace.K,track.dat}.
 * A process of its own, so the C library's rand() sequence that seeds the
 * tracers starts from its default state as in ftest.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle); never the product. */
#include <cstdio>
#include <cstdlib>

extern "C" {
void* ref_sspin_create(int m,int ntrace,const char *base);
void ref_destroy(void *h);
void ref_solve(void *h,double duration,int frames);
}

int main(int argc,char **argv) {
    if(argc!=5) {
        fputs("Syntax: ref_ftest <m> <duration> <frames> <output base path>\n",stderr);
        return 1;
    }
    void *h=ref_sspin_create(atoi(argv[1]),512,argv[4]);
    ref_solve(h,atof(argv[2]),atoi(argv[3]));
    ref_destroy(h);
    return 0;
}
