/* C API over the reference's own classes, compiled from the unmodified
 * reference sources plus the clean-room TGMG shim (oracle/tgmg_shim).
 *
 * TEST INFRASTRUCTURE ONLY: the oracle. Only tests/, the smoke check and
 * bench.py's CPU-baseline / reference legs load the library built from this
 * file (oracle/_ref/libincrmt_ref.so); the product never does.
 *
 * The per-stage entry points call the private step functions of fluid_2d
 * (fluid_2d.cc:298-369) one at a time, so that every GPU kernel can be
 * compared with the reference function it replaces on the same state. The
 * access specifiers are opened for this translation unit only; the layout of
 * the classes is unchanged. */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <sys/stat.h>
#include <sys/types.h>
#include <vector>
#include <algorithm>
#include <limits>
#include <fstream>
#include <omp.h>

#define private public
#define protected public
#include "common.hh"
#include "object.hh"
#include "obj_field.hh"
#include "fluid_2d.hh"
#undef private
#undef protected

namespace {

/** The sediment workload's ellipse, which the reference lacks, written as
 * a harness-side subclass of the reference's obj_standard on the pattern of
 * obj_circle (object.hh:128-138, object.cc:22-34): translated reference map
 * (obj_standard::transform), at rest initially, and the circle's gravity
 * acceleration. Its level set is the same first-order distance the GPU's
 * ellipse uses: with r = |(X'/a, Y'/b)| in the body frame rotated by theta,
 * phi = (r - 1)/|grad r| = (r - 1) r / |(X'/a^2, Y'/b^2)|, zero exactly on the
 * boundary; the band rebuild turns the band values into distances. */
struct obj_ellipse : public obj_standard {
    const double ea, eb, cth, sth, grav;
    obj_ellipse(double cx_,double cy_,double a_,double b_,double theta,double grav_) :
        obj_standard(cx_,cy_,a_), ea(a_), eb(b_), cth(cos(theta)), sth(sin(theta)), grav(grav_) {}
    virtual double phi(double X,double Y) {
        const double xb=cth*X+sth*Y,yb=-sth*X+cth*Y,ia=1/ea,ib=1/eb;
        const double r=sqrt(xb*xb*ia*ia+yb*yb*ib*ib);
        const double gr=sqrt(xb*xb*ia*ia*ia*ia+yb*yb*ib*ib*ib*ib);
        if(gr==0) return -(ea<eb?ea:eb);
        return (r-1)*r/gr;
    }
    virtual void accel(double x,double y,double X,double Y,double phiv,double &accx,double &accy) {
        accy-=grav*op->trans_func_in(phiv);
    }
};

/** One reference simulation together with the objects it owns. */
struct ref_sim {
    sim_type *st;
    std::vector<object*> obj;
    fluid_2d *f;
    char *fout;
    char *fa;
};

/** fluid_2d::update_velocity copies nX,nY into X,Y at every grid point
 * (fluid_2d.cc:1368-1373, s_field::set_full_timestep), but nX,nY are only
 * ever computed inside the band (update_reference_map, extrapolate), and the
 * s_field arrays are never initialised (obj_field.cc). Outside the band X,Y
 * therefore take whatever the heap held, which depends on earlier
 * allocations in the process. The harness fills nX,nY with zeros once after
 * initialisation, the contents a fresh allocation has, so that the oracle is
 * deterministic; inside the band nothing changes. */
void zero_unset_refmap(fluid_2d &f) {
    const int mem=f.ml*f.nl;
    for(int k=0;k<f.n_obj;k++) {
        s_field *sp=f.olist[k]->sbase;
        for(int ij=0;ij<mem;ij++) sp[ij].nX=sp[ij].nY=0;
    }
}

/** Builds the ftest "simple-spin" scenario (ftest.cc:116-143, 383-400) at
 * an m x m grid, with the output directory <base>.odr. */
ref_sim* make_sspin(int m,int ntrace,const char *base) {
    ref_sim *r=new ref_sim;
    r->fa=new char[strlen(base)+1];
    strcpy(r->fa,base);
    r->fout=new char[strlen(base)+8];
    sprintf(r->fout,"%s.odr",base);
    mkdir(r->fout,S_IRWXU|S_IRWXG|S_IROTH|S_IXOTH);
    const double tw=2.5,pinw=2.5,rhof=1,rhos=3,visc=1e-2,G=48;
    const unsigned int fflags=8|16|64|128|256|512;
    obj_simple_spin *sp=new obj_simple_spin(0.8,0.5,0.125,0.2,M_PI,1,r->fa);
    // obj_simple_spin is built with one tracer, so its record buffer holds
    // 1+2*1=3 doubles (object.hh:318), but file_output writes four
    // (object.cc:213-217) and would overwrite the heap. Give it room for four.
    delete [] sp->buf;
    sp->buf=new double[4];
    r->obj.push_back(sp);
    r->st=new sim_type(-1,1,-1,1,false,false);
    r->f=new fluid_2d(m,m,*r->st,visc,rhof,tw,pinw,ntrace,fflags,r->fout);
    mat_const mc(G,rhos,1,true);
    for(unsigned int k=0;k<r->obj.size();k++) r->f->add_object(r->obj[k],mc);
    r->f->initialize(0.8,0.4,0.8);
    zero_unset_refmap(*r->f);
    return r;
}

/** A walled (or periodic) domain with any number of circles (type 1:
 * obj_circle(cx,cy,cr,uu,vv,omega,grav), object.hh:128-138), rounded rods
 * (type 2: obj_rounded_rod(cx,cy,cr,cl,grav), object.hh:229-230) and flags
 * (type 3: obj_flag(cx,cy,flag_l,flag_w,flag_a,perturb_v,ntrace),
 * object.hh:487-488), squares (5), seven-pointed stars (6), flappers (7),
 * pistons (8), circle trackers (9), triangles (11: obj_triangle(cx,cy,cr,
 * theta,grav)), lampreys (12: obj_lamprey(cx,cy,theta,le,dis,w1,w2,T,mlam))
 * hoops (13: obj_hoop(r_in,r_out,grav)) and the harness's ellipses (14:
 * obj_ellipse(cx,cy,a,b,theta,grav), above), each with its constructor's
 * arguments in order; mats holds G and rhos per object. flow_u > 0 selects
 * sim_horiz_flow(flow_u, geom) (sim_type.hh:125-126; y-periodic, inflow at the
 * left, zero pressure at the right) instead of sim_type(geom, x_prd, y_prd).
 * Output directory <base>.odr. */
ref_sim* make_multi(int m,int n,const double *geom,int x_prd,int y_prd,double visc,double rhof,
                    int ntrace,int nobj,const int *types,const double *params,const double *mats,
                    const char *base,double flow_u) {
    ref_sim *r=new ref_sim;
    r->fa=new char[strlen(base)+1];
    strcpy(r->fa,base);
    r->fout=new char[strlen(base)+8];
    sprintf(r->fout,"%s.odr",base);
    mkdir(r->fout,S_IRWXU|S_IRWXG|S_IROTH|S_IXOTH);
    const double tw=2.5,pinw=2.5;
    const unsigned int fflags=8|16|64|128|256|512;
    for(int k=0;k<nobj;k++) {
        const double *p=params+12*k;
        if(types[k]==1) r->obj.push_back(new obj_circle(p[0],p[1],p[2],p[3],p[4],p[5],p[6]));
        else if(types[k]==2) r->obj.push_back(new obj_rounded_rod(p[0],p[1],p[2],p[3],p[4]));
        else if(types[k]==5) r->obj.push_back(new obj_square(p[0],p[1],p[2],p[3],p[4],p[5],p[6]));
        else if(types[k]==6) r->obj.push_back(new obj_seven_point(p[0],p[1],p[2],p[3],p[4],p[5]));
        else if(types[k]==7) r->obj.push_back(new obj_flapper(p[0],p[1],p[2],p[3],p[4],p[5],p[6],p[7],p[8]));
        else if(types[k]==8) r->obj.push_back(new obj_piston(p[0],p[1],p[2],p[3],p[4],p[5],p[6],r->fa));
        else if(types[k]==9) r->obj.push_back(new obj_circle_track(p[0],p[1],p[2],p[3],p[4],p[5],r->fa));
        else if(types[k]==11) r->obj.push_back(new obj_triangle(p[0],p[1],p[2],p[3],p[4]));
        else if(types[k]==12) r->obj.push_back(new obj_lamprey(p[0],p[1],p[2],p[3],p[4],p[5],p[6],p[7],p[8]));
        else if(types[k]==13) r->obj.push_back(new obj_hoop(p[0],p[1],p[2]));
        else if(types[k]==14) r->obj.push_back(new obj_ellipse(p[0],p[1],p[2],p[3],p[4],p[5]));
        else r->obj.push_back(new obj_flag(p[0],p[1],p[2],p[3],p[4],p[5],static_cast<int>(p[6]),r->fa));
    }
    if(flow_u>0) r->st=new sim_horiz_flow(flow_u,geom[0],geom[1],geom[2],geom[3]);
    else r->st=new sim_type(geom[0],geom[1],geom[2],geom[3],x_prd!=0,y_prd!=0);
    r->f=new fluid_2d(m,n,*r->st,visc,rhof,tw,pinw,ntrace,fflags,r->fout);
    for(int k=0;k<nobj;k++) {
        mat_const mc(mats[2*k],mats[2*k+1],1,true);
        r->f->add_object(r->obj[k],mc);
    }
    r->f->initialize(0.8,0.4,0.8);
    zero_unset_refmap(*r->f);
    return r;
}

/** conv_test's scenario (conv_test.cc:52-125): sim_velocity_pulses on the
 * doubly periodic [-1,1]^2, circles (type 1), squares (type 5) of
 * (cx,cy,cr,uu,vv,omega,grav) or the full solid (type 10, obj_full) with
 * mat_const(G,rhos,1,false), initialised with the given extra-viscosity and
 * time-step padding factors; solid_prd sets fluid_2d::solid_prd_bc as
 * conv_test's type 2 does (conv_test.cc:120). */
ref_sim* make_pulses(int m,double visc,double rhof,int ntrace,int nobj,const int *types,const double *params,
                     const double *mats,double ev_mult,double dt_pad,double dt_ev_pad,const char *base,
                     int solid_prd) {
    ref_sim *r=new ref_sim;
    r->fa=new char[strlen(base)+1];
    strcpy(r->fa,base);
    r->fout=new char[strlen(base)+8];
    sprintf(r->fout,"%s.odr",base);
    mkdir(r->fout,S_IRWXU|S_IRWXG|S_IROTH|S_IXOTH);
    const double tw=2.5,pinw=2.5;
    const unsigned int fflags=8|2048;
    for(int k=0;k<nobj;k++) {
        const double *p=params+12*k;
        if(types[k]==5) r->obj.push_back(new obj_square(p[0],p[1],p[2],p[3],p[4],p[5],p[6]));
        else if(types[k]==10) r->obj.push_back(new obj_full());
        else r->obj.push_back(new obj_circle(p[0],p[1],p[2],p[3],p[4],p[5],p[6]));
    }
    r->st=new sim_velocity_pulses;
    r->f=new fluid_2d(m,m,*r->st,visc,rhof,tw,pinw,ntrace,fflags,r->fout);
    for(int k=0;k<nobj;k++) {
        mat_const mc(mats[2*k],mats[2*k+1],1,false);
        r->f->add_object(r->obj[k],mc);
    }
    r->f->solid_prd_bc=solid_prd!=0;
    r->f->initialize(ev_mult,dt_pad,dt_ev_pad);
    zero_unset_refmap(*r->f);
    return r;
}

/** Address of field number id (0..23, in the member order of struct field,
 * fields.hh:7-49) at grid index ij of the full (ghosted) array. */
inline double& fld(fluid_2d &f,int id,int ij) {
    return reinterpret_cast<double*>(f.fbase+ij)[id];
}

/** Address of solid field number id (0..19, member order of struct s_field,
 * fields.hh:51-79) of object k at full-array index ij. */
inline double& sfld(fluid_2d &f,int k,int id,int ij) {
    return reinterpret_cast<double*>(f.olist[k]->sbase+ij)[id];
}

}

extern "C" {

/** Creates the simple-spin simulation. \return an opaque handle. */
void* ref_sspin_create(int m,int ntrace,const char *base) {
    return make_sspin(m,ntrace,base);
}

void* ref_multi_create(int m,int n,const double *geom,int x_prd,int y_prd,double visc,double rhof,
                       int ntrace,int nobj,const int *types,const double *params,const double *mats,
                       const char *base,double flow_u) {
    return make_multi(m,n,geom,x_prd,y_prd,visc,rhof,ntrace,nobj,types,params,mats,base,flow_u);
}

void* ref_pulses_create(int m,double visc,double rhof,int ntrace,int nobj,const int *types,
                        const double *params,const double *mats,double ev_mult,double dt_pad,
                        double dt_ev_pad,const char *base,int solid_prd) {
    return make_pulses(m,visc,rhof,ntrace,nobj,types,params,mats,ev_mult,dt_pad,dt_ev_pad,base,solid_prd);
}

/** fluid_2d::l_comparison of the coarse simulation h against the fine one
 * (fluid_2d_io.cc:186-281): 32 doubles into err. */
void ref_l_comparison(void *h,void *fine,double *err) {
    static_cast<ref_sim*>(h)->f->l_comparison(*static_cast<ref_sim*>(fine)->f,err);
}

void ref_destroy(void *h) {
    ref_sim *r=static_cast<ref_sim*>(h);
    fluid_2d *f=r->f;
    delete f;
    for(unsigned int k=0;k<r->obj.size();k++) delete r->obj[k];
    delete r->st;
    delete [] r->fout;
    delete [] r->fa;
    delete r;
}

/** Grid facts: m, n, ml, nl, n_obj, m_fem, n_fem. */
void ref_dims(void *h,int *out) {
    fluid_2d &f=*static_cast<ref_sim*>(h)->f;
    out[0]=f.m;out[1]=f.n;out[2]=f.ml;out[3]=f.nl;out[4]=f.n_obj;
    out[5]=f.m_fem;out[6]=f.n_fem;
}

/** Scalars: dt_reg, time, dx, dy, eps, K_stiff of object 0 (if simple-spin). */
void ref_scalars(void *h,double *out) {
    fluid_2d &f=*static_cast<ref_sim*>(h)->f;
    out[0]=f.dt_reg;out[1]=f.time;out[2]=f.dx;out[3]=f.dy;out[4]=f.eps;
    out[5]=0;
    if(f.n_obj>0) {
        obj_simple_spin *o=dynamic_cast<obj_simple_spin*>(f.olist[0]->obj);
        if(o!=NULL) out[5]=o->K_stiff;
    }
}

void ref_set_time(void *h,double t) {static_cast<ref_sim*>(h)->f->time=t;}

/** Copies a full (ml x nl) array out of the simulation.
 * id 0..23: fluid field; 100..119: solid field (id-100) of object k;
 * 200: phi of object k; 201: level-set status of object k (as doubles). */
int ref_get(void *h,int id,int k,double *out) {
    fluid_2d &f=*static_cast<ref_sim*>(h)->f;
    const int mem=f.ml*f.nl;
    if(id>=0&&id<24) {for(int ij=0;ij<mem;ij++) out[ij]=fld(f,id,ij);return 0;}
    if(k<0||k>=f.n_obj) return -1;
    if(id>=100&&id<120) {for(int ij=0;ij<mem;ij++) out[ij]=sfld(f,k,id-100,ij);return 0;}
    if(id==200) {for(int ij=0;ij<mem;ij++) out[ij]=f.olist[k]->phi_base[ij];return 0;}
    if(id==201) {for(int ij=0;ij<mem;ij++) out[ij]=f.olist[k]->cbase[ij];return 0;}
    return -1;
}

/** Copies a full (ml x nl) array into the simulation (same ids as ref_get). */
int ref_set(void *h,int id,int k,const double *in) {
    fluid_2d &f=*static_cast<ref_sim*>(h)->f;
    const int mem=f.ml*f.nl;
    if(id>=0&&id<24) {for(int ij=0;ij<mem;ij++) fld(f,id,ij)=in[ij];return 0;}
    if(k<0||k>=f.n_obj) return -1;
    if(id>=100&&id<120) {for(int ij=0;ij<mem;ij++) sfld(f,k,id-100,ij)=in[ij];return 0;}
    if(id==200) {for(int ij=0;ij<mem;ij++) f.olist[k]->phi_base[ij]=in[ij];return 0;}
    if(id==201) {for(int ij=0;ij<mem;ij++) f.olist[k]->cbase[ij]=static_cast<int>(in[ij]);return 0;}
    return -1;
}

/** Narrow-band list of object k in traversal order (u_start..u_end, wrapping),
 * as full-array indices. \return the number of entries (at most cap). */
int ref_band(void *h,int k,int *out,int cap) {
    fluid_2d &f=*static_cast<ref_sim*>(h)->f;
    levelset &ls=f.olist[k]->ls;
    int c=0,l=ls.u_start;
    while(l!=ls.u_end&&c<cap) {
        out[c++]=ls.u[l];
        l=(l==ls.u_mem-1)?0:l+1;
    }
    return c;
}

/** Fluid tracers (ntrace x 4 doubles). */
void ref_get_tracers(void *h,double *out) {
    fluid_2d &f=*static_cast<ref_sim*>(h)->f;
    memcpy(out,f.tm,sizeof(double)*4*f.ntrace);
}

void ref_set_tracers(void *h,const double *in) {
    fluid_2d &f=*static_cast<ref_sim*>(h)->f;
    memcpy(f.tm,in,sizeof(double)*4*f.ntrace);
}

/** Special tracers of object k (6 doubles each: x, y, two stage values, X, Y).
 * \return the number of tracers, or -1. */
int ref_get_obj_tracers(void *h,int k,double *out) {
    fluid_2d &f=*static_cast<ref_sim*>(h)->f;
    obj_track *o=dynamic_cast<obj_track*>(f.olist[k]->obj);
    if(o==NULL) return -1;
    memcpy(out,o->tm,sizeof(double)*6*o->ntrace);
    return o->ntrace;
}

/** obj_track::count of object k (steps since its last record), or -1. */
int ref_obj_track_count(void *h,int k) {
    fluid_2d &f=*static_cast<ref_sim*>(h)->f;
    obj_track *o=dynamic_cast<obj_track*>(f.olist[k]->obj);
    return o==NULL?-1:o->count;
}

/** Multigrid solution arrays: which=0 MAC z (m*n), 1 FEM z (m_fem*n_fem),
 * 2 shared source array (m_fem*n_fem), 3 MAC edge 1/rho (2mn+m+n),
 * 4 FEM corner 1/rho (m_fem*n_fem). \return number of values. */
int ref_get_mg(void *h,int which,double *out) {
    fluid_2d &f=*static_cast<ref_sim*>(h)->f;
    int nv=0;const double *p=NULL;
    switch(which) {
        case 0: nv=f.mn;p=f.ms_mac->z;break;
        case 1: nv=f.m_fem*f.n_fem;p=f.ms_fem->z;break;
        case 2: nv=f.m_fem*f.n_fem;p=f.src;break;
        case 3: if(f.const_rho) return -1;
                nv=2*f.mn+f.m+f.n;p=static_cast<mgs_mac_varying_rho*>(f.ms_mac)->irho;break;
        case 4: if(f.const_rho) return -1;
                nv=f.m_fem*f.n_fem;p=static_cast<mgs_fem_varying_rho*>(f.ms_fem)->irho;break;
        default: return -1;
    }
    if(out!=NULL) memcpy(out,p,sizeof(double)*nv);
    return nv;
}

int ref_set_mg(void *h,int which,const double *in) {
    fluid_2d &f=*static_cast<ref_sim*>(h)->f;
    switch(which) {
        case 0: memcpy(f.ms_mac->z,in,sizeof(double)*f.mn);return 0;
        case 1: memcpy(f.ms_fem->z,in,sizeof(double)*f.m_fem*f.n_fem);return 0;
        case 2: memcpy(f.src,in,sizeof(double)*f.m_fem*f.n_fem);return 0;
    }
    return -1;
}

/** Total V-cycles of the MAC (which=0) or FEM (1) solver since the last reset;
 * reset clears the counters. */
int ref_vcycles(void *h,int which,int reset) {
    fluid_2d &f=*static_cast<ref_sim*>(h)->f;
    mgs_base *s=which==0?static_cast<mgs_base*>(f.ms_mac):static_cast<mgs_base*>(f.ms_fem);
    int v=s->tp.vcount_extra();
    if(reset) s->avg_v_cycles();
    return v;
}

/** Runs one reference step function on the current state.
 * stage: 0 update_tracers(1), 1 normal_derivatives_velocity,
 * 2 normal_derivatives_refmap, 3 godunov_upwinding_set<true>,
 * 4 edge_boundary_conditions, 5 compute_tangential_stability_derivatives,
 * 6 compute_half_time_edge_velocities, 7 compute_half_time_edge_reference_map,
 * 8 godunov_upwinding_set<false>, 9 mac_projection, 10 update_reference_map,
 * 11 pin, 12 set_boundaries, 13 compute_stress, 14 compute_ustar,
 * 15 finite_element_projection, 16 copy_pressure, 17 update_velocity,
 * 18 update_tracers(2), 19 set_rho, 20 step_forward, 21 build_band of every
 * object (without the pinning sweep), 22 extrapolate of every object. */
int ref_stage(void *h,int stage,double dt) {
    fluid_2d &f=*static_cast<ref_sim*>(h)->f;
    switch(stage) {
        case 0: f.update_tracers(1,dt);break;
        case 1: f.normal_derivatives_velocity(dt);break;
        case 2: f.normal_derivatives_refmap(dt);break;
        case 3: f.godunov_upwinding_set<true>();break;
        case 4: f.edge_boundary_conditions();break;
        case 5: f.compute_tangential_stability_derivatives();break;
        case 6: f.compute_half_time_edge_velocities(dt);break;
        case 7: f.compute_half_time_edge_reference_map(dt);break;
        case 8: f.godunov_upwinding_set<false>();break;
        case 9: f.mac_projection();break;
        case 10: f.update_reference_map(dt);break;
        case 11: f.pin();break;
        case 12: f.set_boundaries();break;
        case 13: f.compute_stress();break;
        case 14: f.compute_ustar(dt);break;
        case 15: f.finite_element_projection(dt);break;
        case 16: f.copy_pressure();break;
        case 17: f.update_velocity(dt);break;
        case 18: f.update_tracers(2,dt);break;
        case 19: f.set_rho();break;
        case 20: f.step_forward(dt);break;
        case 21: for(int k=0;k<f.n_obj;k++) f.olist[k]->ls.build_band();break;
        case 22: for(int k=0;k<f.n_obj;k++) f.olist[k]->extrapolate();break;
        default: return -1;
    }
    return 0;
}

/** Runs `steps` reference steps of size dt. */
void ref_steps(void *h,int steps,double dt) {
    fluid_2d &f=*static_cast<ref_sim*>(h)->f;
    for(int s=0;s<steps;s++) f.step_forward(dt);
}

/** fluid_2d::solve (fluid_2d.cc:254-295): frames of output written by the
 * reference's own writers into the simulation's output directory. */
void ref_solve(void *h,double duration,int frames) {
    static_cast<ref_sim*>(h)->f->solve(duration,frames);
}

/** Standalone variable-density solve of the reference's MAC (sys=0,
 * mgs_mac_varying_rho, mgs_mac.hh:64-102) or FEM (sys=1,
 * mgs_fem_varying_rho, mgs_fem.hh:86-136) system on an m x n cell grid over
 * [ax,bx]x[ay,by]. rho is the full (m+4)x(n+4) cell density array from which
 * the reference builds the coefficients (fluid_2d.cc:1140-1170); b is the
 * right-hand side (m*n for MAC, m_fem*n_fem for FEM; for FEM with zpr its
 * fixed column is zeroed as mgs_fem.cc:112 does); z is the initial guess on
 * input and the solution on output.
 * \param[out] stats vcycles, relative residual, wall seconds.
 * \return 0 on success, 1 if the solver did not converge. */
int ref_mg_solve(int sys,int m,int n,double ax,double bx,double ay,double by,
                 int xprd,int yprd,int zpr,const double *rho,double *b,double *z,
                 double *stats) {
    sim_type st(ax,bx,ay,by,xprd!=0,yprd!=0);
    fluid_2d f(m,n,st,1.,1.,2.5,2.5,0,0,".");
    f.zpr=zpr!=0;
    f.dt_reg=1.;
    f.ms_mac=NULL;f.ms_fem=NULL;
    for(int t=0;t<omp_get_max_threads();t++) f.coll[t]=NULL;
    const int mem=f.ml*f.nl;
    for(int ij=0;ij<mem;ij++) f.fbase[ij].rho=rho[ij];
    int ok;
    double t0=wtime();
    if(sys==0) {
        memcpy(f.src,b,sizeof(double)*f.mn);
        mgs_mac_varying_rho *ms=new mgs_mac_varying_rho(f);
        memcpy(ms->z,z,sizeof(double)*f.mn);
        t0=wtime();
        f.set_edge_irho(ms->irho);
        ms->mg.setup();
        ok=ms->mg.solve_v_cycle(ms->tp);
        stats[2]=wtime()-t0;
        memcpy(z,ms->z,sizeof(double)*f.mn);
        stats[0]=ms->mg.last_vcycles;stats[1]=ms->mg.last_rel_res;
        f.ms_mac=ms;
    } else {
        const int nf=f.m_fem*f.n_fem;
        memcpy(f.src,b,sizeof(double)*nf);
        mgs_fem_varying_rho *ms=new mgs_fem_varying_rho(f);
        memcpy(ms->z,z,sizeof(double)*nf);
        t0=wtime();
        f.set_corner_irho(ms->irho);
        ms->mg.setup();
        if(ms->zpr) for(int ij=ms->m-1;ij<ms->mn;ij+=ms->m) f.src[ij]=0;
        ok=ms->mg.solve_v_cycle(ms->tp);
        stats[2]=wtime()-t0;
        memcpy(z,ms->z,sizeof(double)*nf);
        memcpy(b,f.src,sizeof(double)*nf);
        stats[0]=ms->mg.last_vcycles;stats[1]=ms->mg.last_rel_res;
        f.ms_fem=ms;
    }
    return ok?0:1;
}

/** Applies the reference operator of sys (0 MAC, 1 FEM) built from rho to z:
 * out = A z, through the reference callbacks a_cc and mul_a. Grid and rho as
 * for ref_mg_solve. */
void ref_mg_apply(int sys,int m,int n,double ax,double bx,double ay,double by,
                  int xprd,int yprd,int zpr,const double *rho,const double *z,double *out) {
    sim_type st(ax,bx,ay,by,xprd!=0,yprd!=0);
    fluid_2d f(m,n,st,1.,1.,2.5,2.5,0,0,".");
    f.zpr=zpr!=0;
    f.dt_reg=1.;
    f.ms_mac=NULL;f.ms_fem=NULL;
    for(int t=0;t<omp_get_max_threads();t++) f.coll[t]=NULL;
    const int mem=f.ml*f.nl;
    for(int ij=0;ij<mem;ij++) f.fbase[ij].rho=rho[ij];
    if(sys==0) {
        mgs_mac_varying_rho *ms=new mgs_mac_varying_rho(f);
        f.set_edge_irho(ms->irho);
        memcpy(ms->z,z,sizeof(double)*f.mn);
        for(int ij=0;ij<f.mn;ij++) {int i=ij%m;out[ij]=ms->mul_a(i,ij)+ms->a_cc(i,ij)*ms->z[ij];}
        f.ms_mac=ms;
    } else {
        mgs_fem_varying_rho *ms=new mgs_fem_varying_rho(f);
        f.set_corner_irho(ms->irho);
        const int mf=ms->m,nf=ms->mn;
        memcpy(ms->z,z,sizeof(double)*nf);
        for(int ij=0;ij<nf;ij++) {int i=ij%mf;out[ij]=ms->mul_a(i,ij)+ms->a_cc(i,ij)*ms->z[ij];}
        f.ms_fem=ms;
    }
}

int ref_num_threads() {return omp_get_max_threads();}

}
