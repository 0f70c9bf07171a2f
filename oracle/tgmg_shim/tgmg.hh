/* Clean-room TGMG-API shim: class declarations (test infrastructure, see
 * tgmg_config.hh for provenance and scope).
 *
 * API surface, as consumed by the reference:
 *  - tgmg<S,V,M>(S&, V* b, V* z), setup(), solve_v_cycle(tgmg_predict&),
 *    solve_v_cycle(), v_cycle(), output_b/output_z/output_res
 *    (mgs_mac.cc:10-71, mgs_fem.cc:29-120, mg_test.cc:21-43);
 *  - tgmg_base<S,V,M>::{output,clear_z,output_res,mds}, explicitly
 *    instantiated at mgs_mac.cc:76-84 and mgs_fem.cc:167-175;
 *  - tgmg_level<V,M>, explicitly instantiated as a system of its own at
 *    mgs_common.cc:74 (the coarse levels).
 * From the system S it reads m, n, mn, x_prd, y_prd, acc, z and the stencil
 * callbacks a_dl..a_ur, inv_cc, mul_a (mgs_mac.hh:38-98, mgs_fem.hh:65-132).
 *
 * Method. Unknowns form an m x n grid with a 9-point stencil. A coarse level
 * keeps every second point of each direction that is coarsened (vertex-style:
 * coarse I sits on fine 2I; mc=(m+1)/2, or m/2 when periodic); on anisotropic
 * grids only the strongly coupled direction is coarsened until the coupling
 * is within a factor tgmg_semi_ratio of isotropic (semi-coarsening), with an
 * operator-dependent prolongation P (black-box multigrid weights from the
 * collapsed stencil: the bilinear 1, 1/2, 1/4 for constant coefficients,
 * following the flux across density jumps and Dirichlet edges), restriction
 * R=P^T and the Galerkin
 * operator A_c=P^T A P, rebuilt on every setup(). The smoother is Gauss-Seidel
 * in four colours (i&1,j&1) visited in the order (0,0),(1,1),(1,0),(0,1),
 * which is red-black ordering for a 5-point stencil and race-free for a
 * 9-point one. A V-cycle does tgmg_nu1 sweeps, restricts the residual,
 * recurses with a zero coarse guess, prolongs the correction and does
 * tgmg_nu2 sweeps; the coarsest level is solved exactly with a dense inverse
 * built at setup: A^-1, or (A + c e e^T)^-1 with c the mean diagonal / N when
 * A is the singular pure-Neumann operator (zero row sums, null space the
 * constants), which yields the solution of zero mean. A solve
 * runs V-cycles until ||b-Az||_2 <= max(rtol*||b||_2, acc). */
#ifndef TGMG_HH
#define TGMG_HH

#include <cstdio>
#include <cstdlib>
#include <cmath>

#include "tgmg_config.hh"
#include "tgmg_predict.hh"

/** A coarse multigrid level: a grid of unknowns with an explicitly stored
 * 9-point stencil, offering the same callback interface as the reference's
 * systems so that the generic smoother and residual code serve both. */
template<class V,class M>
struct tgmg_level {
    const int m,n,mn;
    const bool x_prd,y_prd;
    /** Residual floor; coarse levels never test it. */
    double acc;
    /** Stencil, nine entries per unknown in the order dl,dc,dr,cl,cc,cr,ul,uc,ur. */
    M* const st;
    /** Right-hand side and iterate of this level. */
    V* const b;
    V* const z;
    /** Scratch for this level's residual. */
    V* const r;
    tgmg_level(int m_,int n_,bool x_prd_,bool y_prd_);
    ~tgmg_level();
    inline int il(int i,int ij) {return i>0?ij-1:ij+m-1;}
    inline int ir(int i,int ij) {return i<m-1?ij+1:ij+1-m;}
    inline int jd(int ij) {return ij>=m?ij-m:ij+mn-m;}
    inline int ju(int ij) {return ij<mn-m?ij+m:ij+m-mn;}
    inline double a_dl(int i,int ij) {return st[9*ij];}
    inline double a_dc(int i,int ij) {return st[9*ij+1];}
    inline double a_dr(int i,int ij) {return st[9*ij+2];}
    inline double a_cl(int i,int ij) {return st[9*ij+3];}
    inline double a_cc(int i,int ij) {return st[9*ij+4];}
    inline double a_cr(int i,int ij) {return st[9*ij+5];}
    inline double a_ul(int i,int ij) {return st[9*ij+6];}
    inline double a_uc(int i,int ij) {return st[9*ij+7];}
    inline double a_ur(int i,int ij) {return st[9*ij+8];}
    inline double inv_cc(int i,int ij,double v) {return v/st[9*ij+4];}
    /** Off-diagonal part of A z at one unknown. Entries that would leave a
     * non-periodic grid are zero by construction and are skipped. */
    double mul_a(int i,int ij);
};

/** Generic single-level operations over a system S with the callback
 * interface: smoothing, residuals and output. */
template<class S,class V,class M>
class tgmg_base {
    public:
        S &s;
        const int m,n,mn;
        const bool x_prd,y_prd;
        V* b;
        V* z;
        tgmg_base(S &s_,V *b_,V *z_);
        void gs_sweep();
        void smooth(int k) {for(int l=0;l<k;l++) gs_sweep();}
        /** Residual b-Az at one unknown. */
        inline double res(int i,int ij) {
            return b[ij]-s.mul_a(i,ij)-s.a_cc(i,ij)*z[ij];
        }
        void residual(V *r);
        double res_norm2();
        double rhs_norm2();
        void output(const char* filename,V *arr,double ax,double dx,double ay,double dy);
        void clear_z();
        void output_res(const char* filename,double ax,double dx,double ay,double dy);
        double mds();
};

/** The multigrid solver over a system S. */
template<class S,class V,class M>
class tgmg : public tgmg_base<S,V,M> {
    public:
        /** Number of levels, including the finest. */
        int nlev;
        /** Coarse levels 1..nlev-1 (index 0 unused). */
        tgmg_level<V,M>* lev[tgmg_max_levels];
        /** Generic operations on the coarse levels. */
        tgmg_base<tgmg_level<V,M>,V,M>* lb[tgmg_max_levels];
        /** Whether level l+1 halves the x and y directions of level l. */
        bool cx[tgmg_max_levels],cy[tgmg_max_levels];
        /** Prolongation of level l to l+1: four weights per fine point of
         * level l (build_p), set by setup(). */
        double* pw[tgmg_max_levels];
        /** Fine-level residual scratch. */
        V* const rf;
        /** V-cycles of the most recent solve_v_cycle call. */
        int last_vcycles;
        /** Residual norm ratio ||b-Az||/||b|| reached by the most recent solve. */
        double last_rel_res;
        /** Dense inverse of the coarsest operator (regularised when singular),
         * or NULL when the coarsest level is solved by sweeps. */
        double *ginv;
        /** Whether the coarse grids exist (they are built by the first setup). */
        bool built;
        tgmg(S &s_,V *b_,V *z_);
        ~tgmg();
        void setup();
        void v_cycle();
        bool solve_v_cycle(tgmg_predict &tp);
        bool solve_v_cycle();
        void output_b(const char* filename,double ax,double dx,double ay,double dy) {
            this->output(filename,this->b,ax,dx,ay,dy);
        }
        void output_z(const char* filename,double ax,double dx,double ay,double dy) {
            this->output(filename,this->z,ax,dx,ay,dy);
        }
    private:
        void cycle(int l);
        template<class T>
        void build_p(T &fs,int l,int fm,int fn,bool fxp,bool fyp,tgmg_level<V,M> &c,bool kx,bool ky);
        inline double pweight(int l,int fm,int fn,bool fxp,bool fyp,bool kx,bool ky,int fi,int fj,int I,int J);
        template<class T>
        void galerkin(T &fs,int l,int fm,int fn,bool fxp,bool fyp,tgmg_level<V,M> &c,bool kx,bool ky);
        void restrict_to(V *r,int l,int fm,int fn,bool fxp,bool fyp,tgmg_level<V,M> &c,bool kx,bool ky);
        void prolong_add(V *zf,int l,int fm,int fn,bool fxp,bool fyp,tgmg_level<V,M> &c,bool kx,bool ky);
        void coarse_inverse();
        void build_levels();
};

#endif
