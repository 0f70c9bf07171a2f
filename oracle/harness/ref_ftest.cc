/* The reference's ftest runs (ftest.cc:52-415) with a chosen duration and
 * frame count, so that their output directories can be compared file by file
 * with the GPU driver's:
 *   ref_ftest <m> <duration> <frames> <output base path>
 *       simple-spin at m x m;
 *   ref_ftest <scenario> <arg> <duration> <frames> <output base path>
 *       circ-move, square, seven-star, fluid, flapper, flappers, full <m>;
 *       piston <G> (on m x 5m/2 with m from the environment variable
 *       REF_PISTON_M, default ftest's 320); multi-drop <m>,<type>;
 * each with ftest's objects, materials, domain, viscosity, fields and
 * padding, the reference's own classes, and the C library's rand() drawing
 * placements and tracers in ftest's order (a process of its own, so rand()
 * starts from its default state). Writes <output base path>.odr/.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle); never the product. */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <sys/types.h>
#include <vector>

#include "common.hh"
#include "fluid_2d.hh"
#include "object.hh"

extern "C" {
void* ref_sspin_create(int m,int ntrace,const char *base);
void ref_destroy(void *h);
void ref_solve(void *h,double duration,int frames);
}

int main(int argc,char **argv) {
    if(argc==5) {
        void *h=ref_sspin_create(atoi(argv[1]),512,argv[4]);
        ref_solve(h,atof(argv[2]),atoi(argv[3]));
        ref_destroy(h);
        return 0;
    }
    if(argc!=6) {
        fputs("Syntax: ref_ftest <m> <duration> <frames> <output base path>\n"
              "        ref_ftest <scenario> <arg> <duration> <frames> <output base path>\n",stderr);
        return 1;
    }
    const char *sc=argv[1],*arg=argv[2];
    const double T=atof(argv[3]);
    const int frames=atoi(argv[4]);
    std::string fa=argv[5];

    // ftest's defaults (ftest.cc:78-108)
    int m=200,n=200,ntrace=512;
    double tw=2.5,pinw=2.5,rhof=1,rhos=1,visc=1e-3,G=24,ev_mult=0.8,ev_trans_mult=1,dt_pad=0.4,dt_ev_pad=0.8;
    unsigned int fflags=8|16|64|128|256|512;
    bool set_velocity=true,solid_prd_bc=false;
    sim_type *sim_t=NULL;
    std::vector<object*> obj;
    if(!strcmp(sc,"circ-move")) {
        m=n=atoi(arg);rhos=4;visc=1e-3;
        obj.push_back(new obj_circle_track(-0.5,-0.5,0.25,2,4,24,strdup(fa.c_str())));
        sim_t=new sim_type(-1,1,-1,1,false,false);
    } else if(!strcmp(sc,"square")) {
        m=n=atoi(arg);rhos=3;
        obj.push_back(new obj_square(-0.02,0,0.5,0.01,0,2));
    } else if(!strcmp(sc,"seven-star")) {
        m=n=atoi(arg);rhos=3;
        obj.push_back(new obj_seven_point(0,0,0.62,0.16,M_PI,1));
    } else if(!strcmp(sc,"piston")) {
        G=atof(arg);
        const char *pm=getenv("REF_PISTON_M");
        m=pm?atoi(pm):320;n=m*5/2;rhos=2.;
        obj.push_back(new obj_piston(0.8,0.2,0.6,0.4,4.6,10,0.15,strdup(fa.c_str())));
        sim_t=new sim_type(-1,1,0,5,false,false);
    } else if(!strcmp(sc,"fluid")) {
        m=n=atoi(arg);visc=1e-3;ntrace=256;
        sim_t=new sim_velocity_pulses;
    } else if(!strcmp(sc,"full")) {
        m=n=atoi(arg);rhos=1;G=3;visc=1e-3;ntrace=0;set_velocity=false;solid_prd_bc=true;
        obj.push_back(new obj_full());
        sim_t=new sim_velocity_pulses;
    } else if(!strcmp(sc,"flapper")) {
        m=n=atoi(arg);rhos=4;G=10;visc=5e-4;
        obj.push_back(new obj_flapper(0,-0.8,0.026,0.25,0.021,0.14,0,2.2,8));
        sim_t=new sim_type(-1.5,1.5,-1.5,1.5,false,false);
    } else if(!strcmp(sc,"flappers")) {
        m=n=atoi(arg);rhos=4;G=10;visc=5e-4;
        const int cnum=28;
        double x,y,wx=0.25+0.026+0.01,wy=0.026+0.01,dx,dy;
        int i=0,j;bool good;
        while(i<cnum) {
            x=rnd(-1,1);y=rnd(-1,1);
            if(x+wx>0.98||x-wx<-0.98||y+wy>0.98||y-wy<-0.98) continue;
            good=true;
            for(j=0;j<i;j++) {
                obj_flapper *oc=reinterpret_cast<obj_flapper*>(obj[j]);
                dx=x-oc->cx;dy=y-oc->cy;
                if(fabs(dx)<2*wx&&fabs(dy)<2*wy) {good=false;break;}
            }
            if(good) {i++;obj.push_back(new obj_flapper(x,y,0.026,0.25,0.021,0.14,0,2.2,rnd(7,9)));}
        }
        sim_t=new sim_type(-1,1,-1,1,false,false);
    } else if(!strcmp(sc,"multi-drop")) {
        int type=0;
        if(sscanf(arg,"%d,%d",&m,&type)!=2) {fputs("multi-drop needs <m>,<type>\n",stderr);return 1;}
        n=m;rhos=3;G=2;visc=1e-3;
        const bool square=type==1;
        const int cnum=42;
        double x,y,r,dx,dy,dr;
        int i=0,j;bool good;
        while(i<cnum) {
            x=rnd(-1,1);y=rnd(-1,1);r=rnd(0.1,0.25);
            if(x+r>1||x-r<-1||y+r>1||y-r<-1) continue;
            good=true;
            for(j=0;j<i;j++) {
                obj_circle *oc=reinterpret_cast<obj_circle*>(obj[j]);
                dx=x-oc->cx;dy=y-oc->cy;dr=oc->cr+r;
                if(fabs(dx)<dr&&fabs(dy)<dr) {good=false;break;}
            }
            if(good) {
                i++;
                square?obj.push_back(new obj_square(x,y,r-0.05,0,0,rnd(-5,5)))
                      :obj.push_back(new obj_circle(x,y,r-0.05,0,0,rnd(-5,5)));
            }
        }
        sim_t=new sim_type(-1,1,-1,1,false,false);
    } else {
        fprintf(stderr,"Unknown scenario '%s'\n",sc);
        return 1;
    }
    std::string fout=fa+".odr";
    mkdir(fout.c_str(),S_IRWXU|S_IRWXG|S_IROTH|S_IXOTH);
    if(sim_t==NULL) sim_t=new sim_type();
    fluid_2d f2d(m,n,*sim_t,visc,rhof,tw,pinw,ntrace,fflags,fout.c_str());
    f2d.solid_prd_bc=solid_prd_bc;
    mat_const mc(G,rhos,ev_trans_mult,set_velocity);
    for(unsigned int k=0;k<obj.size();k++) f2d.add_object(obj[k],mc);
    f2d.initialize(ev_mult,dt_pad,dt_ev_pad);
    f2d.solve(T,frames);
    delete sim_t;
    for(unsigned int k=0;k<obj.size();k++) delete obj[k];
    return 0;
}
