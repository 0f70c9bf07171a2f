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

/** Floor of a/2 for any sign of a. */
inline int tgmg_half(int a) {return a>=0?a/2:-((1-a)/2);}

/** Coarse base index of fine index i along a direction (i/2 rounded down
 * when the direction is coarsened, else i itself). */
inline int tgmg_base_of(int i,bool k) {return k?tgmg_half(i):i;}

/** Coarse index of corner q (0 or 1) above base B along a direction of
 * coarse size mc, or -1 where it falls outside a non-periodic grid or the
 * direction is not coarsened (q=1). */
inline int tgmg_corner(int B,int q,int mc,bool p,bool k) {
    if(!k&&q) return -1;
    int c=B+q;
    if(c<0||c>=mc) {if(!p) return -1;c=(c%mc+mc)%mc;}
    return c;
}

/** The nine stencil entries of fs at fine point (i,j) in the order
 * dl,dc,dr,cl,cc,cr,ul,uc,ur, zero where the neighbour lies outside a
 * non-periodic grid (only in-grid entries are queried: the reference's FEM
 * callbacks read their density array before testing the boundary,
 * mgs_fem.hh:121-128). */
template<class T>
inline void tgmg_stencil(T &fs,int fm,int fn,bool fxp,bool fyp,int i,int j,double *a) {
    const int ij=i+fm*j;
    const bool l=fxp||i>0,r=fxp||i<fm-1,d=fyp||j>0,u=fyp||j<fn-1;
    a[0]=d&&l?fs.a_dl(i,ij):0;a[1]=d?fs.a_dc(i,ij):0;a[2]=d&&r?fs.a_dr(i,ij):0;
    a[3]=l?fs.a_cl(i,ij):0;a[4]=fs.a_cc(i,ij);a[5]=r?fs.a_cr(i,ij):0;
    a[6]=u&&l?fs.a_ul(i,ij):0;a[7]=u?fs.a_uc(i,ij):0;a[8]=u&&r?fs.a_ur(i,ij):0;
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
    nlev(1), rf(new V[s_.mn]), last_vcycles(0), last_rel_res(0), ginv(NULL), built(false) {
    for(int l=0;l<tgmg_max_levels;l++) pw[l]=NULL;
}

/** Builds the coarse grids on the first setup(), when the system's stencil
 * can be read. The ratio r of the operator's y coupling to its x coupling
 * is measured on the fine level, summed over the grid: |D|+|U| against
 * |L|+|R|, the stencil collapsed onto its rows and columns ((dx/dy)^2 for
 * either pressure system with uniform coefficients). While one direction's
 * coupling exceeds the other's by more than tgmg_semi_ratio, only that
 * direction is halved, which divides (or multiplies) r by 4. */
template<class S,class V,class M>
void tgmg<S,V,M>::build_levels() {
    built=true;
    int m=this->m,n=this->n;
    bool xp=this->x_prd,yp=this->y_prd;
    double sx=0,sy=0;
    for(int j=0;j<n;j++) for(int i=0;i<m;i++) {
        double a[9];
        tgmg_stencil(this->s,m,n,xp,yp,i,j,a);
        sx+=fabs(a[0]+a[3]+a[6])+fabs(a[2]+a[5]+a[8]);
        sy+=fabs(a[0]+a[1]+a[2])+fabs(a[6]+a[7]+a[8]);
    }
    double r=sx>0?sy/sx:1;
    while(nlev<tgmg_max_levels&&m*n>tgmg_coarsest_size) {
        bool kx=tgmg_can_coarsen(m,xp),ky=tgmg_can_coarsen(n,yp);
        if(kx&&ky) {
            if(r>tgmg_semi_ratio) kx=false;
            else if(r<1/tgmg_semi_ratio) ky=false;
        }
        if(!kx&&!ky) break;
        if(kx&&!ky) r*=4;
        else if(ky&&!kx) r/=4;
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
    for(int l=0;l<tgmg_max_levels;l++) if(pw[l]!=NULL) delete [] pw[l];
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

/** Rebuilds the prolongation of every level and every coarse operator by
 * the Galerkin product P^T A P. */
template<class S,class V,class M>
void tgmg<S,V,M>::setup() {
    if(!built) build_levels();
    for(int l=1;l<nlev;l++) {
        if(l==1) {
            build_p(this->s,0,this->m,this->n,this->x_prd,this->y_prd,*lev[1],cx[0],cy[0]);
            galerkin(this->s,0,this->m,this->n,this->x_prd,this->y_prd,*lev[1],cx[0],cy[0]);
        } else {
            tgmg_level<V,M> &f=*lev[l-1];
            build_p(f,l-1,f.m,f.n,f.x_prd,f.y_prd,*lev[l],cx[l-1],cy[l-1]);
            galerkin(f,l-1,f.m,f.n,f.x_prd,f.y_prd,*lev[l],cx[l-1],cy[l-1]);
        }
    }
    if(nlev>1&&lev[nlev-1]->mn<=tgmg_direct_max) coarse_inverse();
}

/** Operator-dependent prolongation of level l (black-box multigrid: Dendy,
 * J. Comput. Phys. 48 (1982) 366-386), four weights per fine point, one per
 * corner q = qx+2qy of the coarse cell above its base (tgmg_base_of):
 * a point on a coarse point takes it with weight 1; a point between two
 * coarse points along x takes L/(-C) and R/(-C), with L, C, R its stencil
 * summed over the columns left of, through and right of it (the operator
 * collapsed along y), and likewise along y with the rows; a point between
 * four coarse points takes -(sum of its stencil entries times the weights of
 * its eight neighbours)/(its diagonal). With constant coefficients these are
 * the bilinear weights 1, 1/2, 1/4; across density jumps they follow the
 * flux, and at a Dirichlet edge (the zero-pressure edge of the MAC system)
 * the last point's weight drops below 1. The weights stay in double
 * precision: rounded ones would no longer map constants onto constants, and
 * the coarse operators of a pure-Neumann problem would lose their exact
 * null space. */
template<class S,class V,class M>
template<class T>
void tgmg<S,V,M>::build_p(T &fs,int l,int fm,int fn,bool fxp,bool fyp,tgmg_level<V,M> &c,bool kx,bool ky) {
    const int cm=c.m,cn=c.n;
    if(pw[l]==NULL) pw[l]=new double[4*fm*fn];
    double *P=pw[l];
    for(int pass=0;pass<2;pass++) {
#pragma omp parallel for
        for(int j=0;j<fn;j++) for(int i=0;i<fm;i++) {
            const bool xo=kx&&(i&1),yo=ky&&(j&1);
            if((pass==1)!=(xo&&yo)) continue;
            double a[9],*q=P+4*(i+fm*j);
            tgmg_stencil(fs,fm,fn,fxp,fyp,i,j,a);
            q[0]=q[1]=q[2]=q[3]=0;
            const int bx=tgmg_base_of(i,kx),by=tgmg_base_of(j,ky);
            const bool v1=tgmg_corner(bx,1,cm,fxp,kx)>=0,v2=tgmg_corner(by,1,cn,fyp,ky)>=0;
            if(!xo&&!yo) q[0]=1;
            else if(xo&&!yo) {
                const double L=a[0]+a[3]+a[6],C=a[1]+a[4]+a[7],R=a[2]+a[5]+a[8];
                q[0]=L/(-C);
                if(v1) q[1]=R/(-C);
            } else if(!xo&&yo) {
                const double D=a[0]+a[1]+a[2],Mr=a[3]+a[4]+a[5],U=a[6]+a[7]+a[8];
                q[0]=D/(-Mr);
                if(v2) q[2]=U/(-Mr);
            } else {
                double acc[4]={0,0,0,0};
                for(int dj=-1;dj<=1;dj++) for(int di=-1;di<=1;di++) {
                    const double av=a[3*(dj+1)+di+1];
                    if((di==0&&dj==0)||av==0) continue;
                    bool okx=true,oky=true;
                    const int gi=tgmg_wrap(i+di,fm,fxp,okx),gj=tgmg_wrap(j+dj,fn,fyp,oky);
                    if(!okx||!oky) continue;
                    const double *g=P+4*(gi+fm*gj);
                    const int ox=tgmg_base_of(i+di,kx)-bx,oy=tgmg_base_of(j+dj,ky)-by;
                    for(int r=0;r<4;r++) {
                        const int cx_=ox+(r&1),cy_=oy+(r>>1);
                        if(g[r]!=0&&cx_<=1&&cy_<=1) acc[cx_+2*cy_]+=av*g[r];
                    }
                }
                for(int r=0;r<4;r++) {
                    const bool ok=((r&1)==0||v1)&&((r>>1)==0||v2);
                    if(ok) q[r]=-acc[r]/a[4];
                }
            }
        }
    }
}

/** Weight of fine point (fi,fj) (unwrapped indices, in the grid once
 * wrapped) for coarse point (I,J), 0 when (I,J) is not one of its corners. */
template<class S,class V,class M>
inline double tgmg<S,V,M>::pweight(int l,int fm,int fn,bool fxp,bool fyp,bool kx,bool ky,int fi,int fj,int I,int J) {
    const int qx=I-tgmg_base_of(fi,kx),qy=J-tgmg_base_of(fj,ky);
    if(qx<0||qx>1||qy<0||qy>1) return 0;
    bool okx=true,oky=true;
    const int i=tgmg_wrap(fi,fm,fxp,okx),j=tgmg_wrap(fj,fn,fyp,oky);
    if(!okx||!oky) return 0;
    return pw[l][4*(i+fm*j)+qx+2*qy];
}

/** Galerkin coarse operator A_c = P^T A P of level l+1 from level l's
 * operator fs and prolongation, entry by entry: A_c((I,J),(I,J)+k) sums,
 * over the fine points f of the coarse point's support and the stencil
 * neighbours g of f, P(f,(I,J)) A(f,g) P(g,(I,J)+k). */
template<class S,class V,class M>
template<class T>
void tgmg<S,V,M>::galerkin(T &fs,int l,int fm,int fn,bool fxp,bool fyp,tgmg_level<V,M> &c,bool kx,bool ky) {
    const int cm=c.m,cn=c.n;
#pragma omp parallel for
    for(int J=0;J<cn;J++) for(int I=0;I<cm;I++) {
        double q[9]={0,0,0,0,0,0,0,0,0};
        const int x0=kx?2*I-1:I,x1=kx?2*I+1:I,y0=ky?2*J-1:J,y1=ky?2*J+1:J;
        for(int fj=y0;fj<=y1;fj++) for(int fi=x0;fi<=x1;fi++) {
            const double w=pweight(l,fm,fn,fxp,fyp,kx,ky,fi,fj,I,J);
            if(w==0) continue;
            bool okx=true,oky=true;
            const int i=tgmg_wrap(fi,fm,fxp,okx),j=tgmg_wrap(fj,fn,fyp,oky);
            double a[9];
            tgmg_stencil(fs,fm,fn,fxp,fyp,i,j,a);
            for(int dj=-1;dj<=1;dj++) for(int di=-1;di<=1;di++) {
                const double av=a[3*(dj+1)+di+1];
                if(av==0) continue;
                for(int kj=-1;kj<=1;kj++) for(int ki=-1;ki<=1;ki++) {
                    const double v=pweight(l,fm,fn,fxp,fyp,kx,ky,fi+di,fj+dj,I+ki,J+kj);
                    if(v!=0) q[3*(kj+1)+ki+1]+=w*av*v;
                }
            }
        }
        M *o=c.st+9*(I+cm*J);
        for(int k=0;k<9;k++) o[k]=q[k];
    }
}

/** Coarse right-hand side b_c = P^T r. */
template<class S,class V,class M>
void tgmg<S,V,M>::restrict_to(V *r,int l,int fm,int fn,bool fxp,bool fyp,tgmg_level<V,M> &c,bool kx,bool ky) {
    const int cm=c.m,cn=c.n;
#pragma omp parallel for
    for(int J=0;J<cn;J++) for(int I=0;I<cm;I++) {
        const int x0=kx?2*I-1:I,x1=kx?2*I+1:I,y0=ky?2*J-1:J,y1=ky?2*J+1:J;
        double t=0;
        for(int fj=y0;fj<=y1;fj++) for(int fi=x0;fi<=x1;fi++) {
            const double w=pweight(l,fm,fn,fxp,fyp,kx,ky,fi,fj,I,J);
            if(w==0) continue;
            bool okx=true,oky=true;
            const int i=tgmg_wrap(fi,fm,fxp,okx),j=tgmg_wrap(fj,fn,fyp,oky);
            t+=w*r[i+fm*j];
        }
        c.b[I+cm*J]=t;
        c.z[I+cm*J]=0;
    }
}

/** Fine correction z_f += P z_c. */
template<class S,class V,class M>
void tgmg<S,V,M>::prolong_add(V *zf,int l,int fm,int fn,bool fxp,bool fyp,tgmg_level<V,M> &c,bool kx,bool ky) {
    const int cm=c.m,cn=c.n;
#pragma omp parallel for
    for(int j=0;j<fn;j++) for(int i=0;i<fm;i++) {
        const double *q=pw[l]+4*(i+fm*j);
        const int bx=tgmg_base_of(i,kx),by=tgmg_base_of(j,ky);
        double t=0;
        for(int r=0;r<4;r++) {
            if(q[r]==0) continue;
            const int I=tgmg_corner(bx,r&1,cm,fxp,kx),J=tgmg_corner(by,r>>1,cn,fyp,ky);
            t+=q[r]*c.z[I+cm*J];
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
        restrict_to(rf,0,this->m,this->n,this->x_prd,this->y_prd,c,cx[0],cy[0]);
        cycle(1);
        prolong_add(this->z,0,this->m,this->n,this->x_prd,this->y_prd,c,cx[0],cy[0]);
        this->smooth(tgmg_nu2);
    } else {
        tgmg_level<V,M> &f=*lev[l];
        lb[l]->smooth(tgmg_nu1);
        lb[l]->residual(f.r);
        restrict_to(f.r,l,f.m,f.n,f.x_prd,f.y_prd,c,cx[l],cy[l]);
        cycle(l+1);
        prolong_add(f.z,l,f.m,f.n,f.x_prd,f.y_prd,c,cx[l],cy[l]);
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
