/* Clean-room TGMG-API shim: template definitions (test infrastructure, see
 * tgmg_config.hh for provenance and tgmg.hh for the method). The reference
 * includes this file from mgs_common.cc:73, mgs_mac.cc:74 and mgs_fem.cc:165
 * and instantiates it there, so it holds templates and inline functions only. */
#ifndef TGMG_CC
#define TGMG_CC

#include <cstring>
#include "tgmg.hh"

/** Wraps a grid index into [0,m) for a periodic direction, or flags it as
 * outside a non-periodic grid. */
inline int tgmg_wrap(int i,int m,bool p,bool &ok) {
    if(i<0) {if(p) i+=m;else ok=false;}
    else if(i>=m) {if(p) i-=m;else ok=false;}
    return i;
}

/** One-dimensional prolongation weight P(f,I) between fine index f and
 * coarse index I.
 * \param[in] (mf,mc) fine and coarse sizes.
 * \param[in] p whether the direction is periodic.
 * \param[in] k whether the direction is coarsened (else P is the identity). */
inline double tgmg_pw(int f,int I,int mf,int mc,bool p,bool k) {
    if(!k) return f==I?1.:0.;
    int d=f-2*I;
    if(p) {if(d>mf/2) d-=mf;else if(d<-mf/2) d+=mf;}
    if(d==0) return 1.;
    if(d==-1) return 0.5;
    if(d==1) return (p||I+1<mc)?0.5:1.;
    return 0.;
}

/** Fine indices carrying a nonzero weight for coarse index I: 2I-1,2I,2I+1
 * (wrapped or clipped) when coarsened, else I itself.
 * \return The number of indices written to f. */
inline int tgmg_support(int I,int mf,bool p,bool k,int *f) {
    if(!k) {*f=I;return 1;}
    int c=0;
    for(int d=-1;d<=1;d++) {
        bool ok=true;
        int g=tgmg_wrap(2*I+d,mf,p,ok);
        if(ok) f[c++]=g;
    }
    return c;
}

template<class V,class M>
tgmg_level<V,M>::tgmg_level(int m_,int n_,bool x_prd_,bool y_prd_)
    : m(m_), n(n_), mn(m_*n_), x_prd(x_prd_), y_prd(y_prd_), acc(0),
    st(new M[9*mn]), b(new V[mn]), z(new V[mn]), r(new V[mn]) {
    for(int ij=0;ij<9*mn;ij++) st[ij]=0;
    for(int ij=0;ij<mn;ij++) b[ij]=z[ij]=r[ij]=0;
}

template<class V,class M>
tgmg_level<V,M>::~tgmg_level() {
    delete [] r;delete [] z;delete [] b;delete [] st;
}

template<class V,class M>
double tgmg_level<V,M>::mul_a(int i,int ij) {
    const M *a=st+9*ij;
    const bool li=x_prd||i>0,ri=x_prd||i<m-1,dj=y_prd||ij>=m,uj=y_prd||ij<mn-m;
    const int l=li?il(i,ij):ij,r_=ri?ir(i,ij):ij;
    double t=0;
    if(dj) {
        int d=jd(ij),o=d-ij;
        if(li) t+=a[0]*z[l+o];
        t+=a[1]*z[d];
        if(ri) t+=a[2]*z[r_+o];
    }
    if(li) t+=a[3]*z[l];
    if(ri) t+=a[5]*z[r_];
    if(uj) {
        int u=ju(ij),o=u-ij;
        if(li) t+=a[6]*z[l+o];
        t+=a[7]*z[u];
        if(ri) t+=a[8]*z[r_+o];
    }
    return t;
}

template<class S,class V,class M>
tgmg_base<S,V,M>::tgmg_base(S &s_,V *b_,V *z_) : s(s_), m(s_.m), n(s_.n),
    mn(s_.mn), x_prd(s_.x_prd), y_prd(s_.y_prd), b(b_), z(z_) {}

/** One Gauss-Seidel sweep in four colours (0,0),(1,1),(1,0),(0,1). */
template<class S,class V,class M>
void tgmg_base<S,V,M>::gs_sweep() {
    static const int col[4][2]={{0,0},{1,1},{1,0},{0,1}};
    for(int c=0;c<4;c++) {
        const int pi=col[c][0],pj=col[c][1];
#pragma omp parallel for
        for(int j=pj;j<n;j+=2) for(int i=pi;i<m;i+=2) {
            int ij=i+m*j;
            z[ij]=s.inv_cc(i,ij,b[ij]-s.mul_a(i,ij));
        }
    }
}

template<class S,class V,class M>
void tgmg_base<S,V,M>::residual(V *r) {
#pragma omp parallel for
    for(int j=0;j<n;j++) for(int i=0;i<m;i++) {
        int ij=i+m*j;
        r[ij]=res(i,ij);
    }
}

template<class S,class V,class M>
double tgmg_base<S,V,M>::res_norm2() {
    double t=0;
#pragma omp parallel for reduction(+:t)
    for(int j=0;j<n;j++) for(int i=0;i<m;i++) {
        int ij=i+m*j;
        double q=res(i,ij);
        t+=q*q;
    }
    return t;
}

template<class S,class V,class M>
double tgmg_base<S,V,M>::rhs_norm2() {
    double t=0;
#pragma omp parallel for reduction(+:t)
    for(int ij=0;ij<mn;ij++) t+=b[ij]*b[ij];
    return t;
}

/** Writes an m x n field in the Gnuplot binary matrix format: a first row of
 * m and the x coordinates, then one row per y holding y and the values. */
template<class S,class V,class M>
void tgmg_base<S,V,M>::output(const char* filename,V *arr,double ax,double dx,double ay,double dy) {
    FILE *fp=fopen(filename,"wb");
    if(fp==NULL) {fprintf(stderr,"tgmg: can't open %s\n",filename);exit(1);}
    float *buf=new float[m+1];
    *buf=m;
    for(int i=0;i<m;i++) buf[i+1]=ax+i*dx;
    fwrite(buf,sizeof(float),m+1,fp);
    for(int j=0;j<n;j++) {
        *buf=ay+j*dy;
        for(int i=0;i<m;i++) buf[i+1]=arr[i+m*j];
        fwrite(buf,sizeof(float),m+1,fp);
    }
    delete [] buf;
    fclose(fp);
}

template<class S,class V,class M>
void tgmg_base<S,V,M>::clear_z() {
    for(int ij=0;ij<mn;ij++) z[ij]=0;
}

template<class S,class V,class M>
void tgmg_base<S,V,M>::output_res(const char* filename,double ax,double dx,double ay,double dy) {
    V *r=new V[mn];
    residual(r);
    output(filename,r,ax,dx,ay,dy);
    delete [] r;
}

/** Mean squared residual. */
template<class S,class V,class M>
double tgmg_base<S,V,M>::mds() {
    return res_norm2()/mn;
}

/** Whether a direction of size m can be halved: a periodic one needs an even
 * size whose half is at least 4, a non-periodic one at least 5 points. */
inline bool tgmg_can_coarsen(int m,bool p) {
    return p?(m%2==0&&m/2>=4):m>=5;
}

template<class S,class V,class M>
tgmg<S,V,M>::tgmg(S &s_,V *b_,V *z_) : tgmg_base<S,V,M>(s_,b_,z_),
    nlev(1), rf(new V[s_.mn]), last_vcycles(0), last_rel_res(0), ginv(NULL) {
    int m=this->m,n=this->n;
    bool xp=this->x_prd,yp=this->y_prd;
    while(nlev<tgmg_max_levels&&m*n>tgmg_coarsest_size) {
        bool kx=tgmg_can_coarsen(m,xp),ky=tgmg_can_coarsen(n,yp);
        if(!kx&&!ky) break;
        int mc=kx?(xp?m/2:(m+1)/2):m,nc=ky?(yp?n/2:(n+1)/2):n;
        cx[nlev-1]=kx;cy[nlev-1]=ky;
        lev[nlev]=new tgmg_level<V,M>(mc,nc,xp,yp);
        lb[nlev]=new tgmg_base<tgmg_level<V,M>,V,M>(*lev[nlev],lev[nlev]->b,lev[nlev]->z);
        nlev++;m=mc;n=nc;
    }
}

template<class S,class V,class M>
tgmg<S,V,M>::~tgmg() {
    for(int l=nlev-1;l>=1;l--) {delete lb[l];delete lev[l];}
    delete [] rf;
    if(ginv!=NULL) delete [] ginv;
}

/** Dense inverse of the coarsest operator by Gauss-Jordan elimination with
 * partial pivoting; the singular Neumann operator is regularised by
 * c e e^T first. */
template<class S,class V,class M>
void tgmg<S,V,M>::coarse_inverse() {
    tgmg_level<V,M> &c=*lev[nlev-1];
    const int N=c.mn,W=2*N;
    if(ginv==NULL) ginv=new double[N*N];
    double *a=new double[N*W];
    for(int k=0;k<N*W;k++) a[k]=0;
    double rsmax=0,dsum=0;
    for(int r=0;r<N;r++) {
        int i=r%c.m,j=r/c.m;
        double rs=0;
        for(int dj=-1;dj<=1;dj++) {
            bool oky=true;
            int jj=tgmg_wrap(j+dj,c.n,c.y_prd,oky);
            if(!oky) continue;
            for(int di=-1;di<=1;di++) {
                bool okx=true;
                int ii=tgmg_wrap(i+di,c.m,c.x_prd,okx);
                if(!okx) continue;
                double v=c.st[9*r+3*(dj+1)+di+1];
                a[r*W+ii+c.m*jj]+=v;
                rs+=v;
            }
        }
        if(fabs(rs)>rsmax) rsmax=fabs(rs);
        dsum+=fabs(c.st[9*r+4]);
        a[r*W+N+r]=1;
    }
    if(rsmax<=1e-10*dsum/N) {
        const double cc=dsum/N/N;
        for(int r=0;r<N;r++) for(int q=0;q<N;q++) a[r*W+q]+=cc;
    }
    for(int k=0;k<N;k++) {
        int p=k;
        for(int r=k+1;r<N;r++) if(fabs(a[r*W+k])>fabs(a[p*W+k])) p=r;
        if(p!=k) for(int q=0;q<W;q++) {double t=a[k*W+q];a[k*W+q]=a[p*W+q];a[p*W+q]=t;}
        const double iv=1.0/a[k*W+k];
        for(int q=0;q<W;q++) a[k*W+q]*=iv;
        for(int r=0;r<N;r++) {
            if(r==k) continue;
            const double f=a[r*W+k];
            if(f==0) continue;
            for(int q=0;q<W;q++) a[r*W+q]-=f*a[k*W+q];
        }
    }
    for(int r=0;r<N;r++) for(int q=0;q<N;q++) ginv[r*N+q]=a[r*W+N+q];
    delete [] a;
}

/** Rebuilds every coarse operator by the Galerkin product P^T A P. */
template<class S,class V,class M>
void tgmg<S,V,M>::setup() {
    for(int l=1;l<nlev;l++) {
        if(l==1) galerkin(this->s,this->m,this->n,this->x_prd,this->y_prd,*lev[1],cx[0],cy[0]);
        else {
            tgmg_level<V,M> &f=*lev[l-1];
            galerkin(f,f.m,f.n,f.x_prd,f.y_prd,*lev[l],cx[l-1],cy[l-1]);
        }
    }
    if(nlev>1&&lev[nlev-1]->mn<=tgmg_direct_max) coarse_inverse();
}

template<class S,class V,class M>
template<class T>
void tgmg<S,V,M>::galerkin(T &fs,int fm,int fn,bool fxp,bool fyp,tgmg_level<V,M> &c,bool kx,bool ky) {
    const int cm=c.m,cn=c.n;
#pragma omp parallel for
    for(int J=0;J<cn;J++) for(int I=0;I<cm;I++) {
        double q[9]={0,0,0,0,0,0,0,0,0};
        int fx[3],fy[3];
        int nfx=tgmg_support(I,fm,fxp,kx,fx),nfy=tgmg_support(J,fn,fyp,ky,fy);
        for(int b=0;b<nfy;b++) {
            double wy=tgmg_pw(fy[b],J,fn,cn,fyp,ky);
            for(int a=0;a<nfx;a++) {
                double w=wy*tgmg_pw(fx[a],I,fm,cm,fxp,kx);
                if(w==0) continue;
                int i=fx[a],ij=i+fm*fy[b];
                // Only entries whose neighbour lies inside the grid are
                // queried: the reference's FEM callbacks read their density
                // array before testing the boundary (mgs_fem.hh:121-128), so
                // an outward entry would read past its end.
                const bool l=fxp||i>0,r=fxp||i<fm-1,d=fyp||fy[b]>0,u=fyp||fy[b]<fn-1;
                double st[9]={d&&l?fs.a_dl(i,ij):0,d?fs.a_dc(i,ij):0,d&&r?fs.a_dr(i,ij):0,
                              l?fs.a_cl(i,ij):0,fs.a_cc(i,ij),r?fs.a_cr(i,ij):0,
                              u&&l?fs.a_ul(i,ij):0,u?fs.a_uc(i,ij):0,u&&r?fs.a_ur(i,ij):0};
                for(int dj=-1;dj<=1;dj++) {
                    bool oky=true;
                    int gy=tgmg_wrap(fy[b]+dj,fn,fyp,oky);
                    if(!oky) continue;
                    for(int di=-1;di<=1;di++) {
                        double av=st[3*(dj+1)+di+1];
                        if(av==0) continue;
                        bool okx=true;
                        int gx=tgmg_wrap(i+di,fm,fxp,okx);
                        if(!okx) continue;
                        for(int kj=-1;kj<=1;kj++) {
                            bool ok=true;
                            int Ky=tgmg_wrap(J+kj,cn,fyp,ok);
                            if(!ok) continue;
                            double vy=tgmg_pw(gy,Ky,fn,cn,fyp,ky);
                            if(vy==0) continue;
                            for(int ki=-1;ki<=1;ki++) {
                                bool ok2=true;
                                int Kx=tgmg_wrap(I+ki,cm,fxp,ok2);
                                if(!ok2) continue;
                                double vx=tgmg_pw(gx,Kx,fm,cm,fxp,kx);
                                if(vx==0) continue;
                                q[3*(kj+1)+ki+1]+=w*av*vx*vy;
                            }
                        }
                    }
                }
            }
        }
        M *o=c.st+9*(I+cm*J);
        for(int k=0;k<9;k++) o[k]=q[k];
    }
}

/** Coarse right-hand side b_c = P^T r. */
template<class S,class V,class M>
void tgmg<S,V,M>::restrict_to(V *r,int fm,int fn,bool fxp,bool fyp,tgmg_level<V,M> &c,bool kx,bool ky) {
    const int cm=c.m,cn=c.n;
#pragma omp parallel for
    for(int J=0;J<cn;J++) for(int I=0;I<cm;I++) {
        int fx[3],fy[3];
        int nfx=tgmg_support(I,fm,fxp,kx,fx),nfy=tgmg_support(J,fn,fyp,ky,fy);
        double t=0;
        for(int b=0;b<nfy;b++) {
            double wy=tgmg_pw(fy[b],J,fn,cn,fyp,ky);
            for(int a=0;a<nfx;a++)
                t+=wy*tgmg_pw(fx[a],I,fm,cm,fxp,kx)*r[fx[a]+fm*fy[b]];
        }
        c.b[I+cm*J]=t;
        c.z[I+cm*J]=0;
    }
}

/** Fine correction z_f += P z_c. */
template<class S,class V,class M>
void tgmg<S,V,M>::prolong_add(V *zf,int fm,int fn,bool fxp,bool fyp,tgmg_level<V,M> &c,bool kx,bool ky) {
    const int cm=c.m,cn=c.n;
#pragma omp parallel for
    for(int j=0;j<fn;j++) for(int i=0;i<fm;i++) {
        int Is[2],Js[2],ni=0,nj=0;
        if(!kx) Is[ni++]=i;
        else {
            int lo=(i%2==0)?i/2:(i-1)/2;
            Is[ni++]=lo;
            if(i%2==1) {
                bool ok=true;
                int hi=tgmg_wrap(lo+1,cm,fxp,ok);
                if(ok) Is[ni++]=hi;
            }
        }
        if(!ky) Js[nj++]=j;
        else {
            int lo=(j%2==0)?j/2:(j-1)/2;
            Js[nj++]=lo;
            if(j%2==1) {
                bool ok=true;
                int hi=tgmg_wrap(lo+1,cn,fyp,ok);
                if(ok) Js[nj++]=hi;
            }
        }
        double t=0;
        for(int b=0;b<nj;b++) {
            double wy=tgmg_pw(j,Js[b],fn,cn,fyp,ky);
            for(int a=0;a<ni;a++)
                t+=wy*tgmg_pw(i,Is[a],fm,cm,fxp,kx)*c.z[Is[a]+cm*Js[b]];
        }
        zf[i+fm*j]+=t;
    }
}

template<class S,class V,class M>
void tgmg<S,V,M>::cycle(int l) {
    if(l==nlev-1) {
        if(l==0) this->smooth(tgmg_coarse_sweeps);
        else if(ginv!=NULL) {
            tgmg_level<V,M> &c=*lev[l];
            const int N=c.mn;
            for(int r=0;r<N;r++) {
                double t=0;
                for(int q=0;q<N;q++) t+=ginv[r*N+q]*c.b[q];
                c.z[r]=t;
            }
        } else lb[l]->smooth(tgmg_coarse_sweeps);
        return;
    }
    tgmg_level<V,M> &c=*lev[l+1];
    if(l==0) {
        this->smooth(tgmg_nu1);
        this->residual(rf);
        restrict_to(rf,this->m,this->n,this->x_prd,this->y_prd,c,cx[0],cy[0]);
        cycle(1);
        prolong_add(this->z,this->m,this->n,this->x_prd,this->y_prd,c,cx[0],cy[0]);
        this->smooth(tgmg_nu2);
    } else {
        tgmg_level<V,M> &f=*lev[l];
        lb[l]->smooth(tgmg_nu1);
        lb[l]->residual(f.r);
        restrict_to(f.r,f.m,f.n,f.x_prd,f.y_prd,c,cx[l],cy[l]);
        cycle(l+1);
        prolong_add(f.z,f.m,f.n,f.x_prd,f.y_prd,c,cx[l],cy[l]);
        lb[l]->smooth(tgmg_nu2);
    }
}

template<class S,class V,class M>
void tgmg<S,V,M>::v_cycle() {
    cycle(0);
}

/** Runs V-cycles until ||b-Az||_2 <= max(rtol*||b||_2, acc), checking after
 * every cycle, and records the count in tp.
 * \return Whether the target was reached within tgmg_max_vcycles. */
template<class S,class V,class M>
bool tgmg<S,V,M>::solve_v_cycle(tgmg_predict &tp) {
    double nb=sqrt(this->rhs_norm2()),tol=tgmg_rel_tol()*nb;
    if(tol<this->s.acc) tol=this->s.acc;
    for(int k=1;k<=tgmg_max_vcycles;k++) {
        v_cycle();
        double rn=sqrt(this->res_norm2());
        last_rel_res=nb>0?rn/nb:rn;
        if(rn<=tol) {tp.record(k);last_vcycles=k;return true;}
        if(!std::isfinite(rn)) {tp.record(k);last_vcycles=k;return false;}
    }
    tp.record(tgmg_max_vcycles);
    last_vcycles=tgmg_max_vcycles;
    return false;
}

template<class S,class V,class M>
bool tgmg<S,V,M>::solve_v_cycle() {
    tgmg_predict tp;
    return solve_v_cycle(tp);
}

#endif
