// ORACLE TEST INFRASTRUCTURE — not part of the product.
//
// Clean-room CPU implementation of the TGMG solver interface that the
// reference's linear-system classes are written against. TGMG itself
// (github chr1shr/tgmg, no pinned version; vdropimpact README.md:55-57,
// Makefile:3) is not available, so this header provides the same API with
// an algorithm of its own:
//
//   * problem-class concept (mgs_mac.hh:25-50, mgs_fem.hh:42-57,
//     visco_impl.hh:28-53): m, n, mn, a_{dl,dc,dr,cl,cc,cr,ul,uc,ur}(i,ij),
//     inv_cc(i,ij,v), mul_a(i,ij) and a solution array z shared with the
//     solver;
//   * solver API used by the reference (mgs_mac.hh:57-63, mgs_fem.hh:64-70,
//     visco_impl.cc:29-34, mg_test.cc:21-38): tgmg<S,V,M>(S&,V* b,V* z),
//     setup(), clear_z(), solve_v_cycle(tgmg_predict&), v_cycle(),
//     output(), output_b(), output_z(), output_res();
//   * tgmg_accuracy(scale,fac) (mgs_mac.cc:11, mgs_fem.cc:14,
//     visco_impl.cc:12).
//
// Algorithm: vertex-style coarsening (coarse point I sits on fine point 2I),
// bilinear prolongation P, restriction P^T, Galerkin coarse operators P^T A P
// stored as assembled 9-point stencils, four-colour Gauss-Seidel smoothing
// (a true Gauss-Seidel ordering for 9-point stencils, and independent of the
// OpenMP thread count), and a dense LU solve on the coarsest level. A solve
// stops once ||b-Az||_2 <= rtol*||b||_2 (rtol from tgmg_config.hh).
#ifndef VDI_ORACLE_TGMG_HH
#define VDI_ORACLE_TGMG_HH

#include <cstdio>
#include <cmath>
#include <limits>
#include <vector>

#include "tgmg_config.hh"
#include "tgmg_predict.hh"

/** Absolute accuracy scale in the reference's calls. The shim stores the
 * value (scale*fac*machine epsilon) in the problem's acc member but ends
 * solves on the relative residual instead. */
inline double tgmg_accuracy(double scale,double fac) {
    return scale*fac*std::numeric_limits<double>::epsilon();
}

/** Process-wide counters that the oracle driver reports. */
struct tgmg_stats_t {
    long solves,vcycles;
    int last_vcycles;
    double last_rel_res;
    int failures;
};
inline tgmg_stats_t& tgmg_stats() {
    static tgmg_stats_t s={0,0,0,0.,0};
    return s;
}

/** A coarse level: an assembled 9-point stencil per point, stored as
 * [dl,dc,dr,cl,cc,cr,ul,uc,ur], plus its own solution and source arrays. */
template<class V,class M>
struct tgmg_level {
    int m,n,mn;
    static const bool x_prd=false;
    static const bool y_prd=false;
    static const char gs_mode=0;
    M* const s;
    V* const z;
    V* const b;
    tgmg_level(int m_,int n_) : m(m_), n(n_), mn(m_*n_), s(new M[9*mn]),
        z(new V[mn]), b(new V[mn]) {}
    ~tgmg_level() {delete [] b;delete [] z;delete [] s;}
    inline M a_dl(int i,int ij) {return s[9*ij];}
    inline M a_dc(int i,int ij) {return s[9*ij+1];}
    inline M a_dr(int i,int ij) {return s[9*ij+2];}
    inline M a_cl(int i,int ij) {return s[9*ij+3];}
    inline M a_cc(int i,int ij) {return s[9*ij+4];}
    inline M a_cr(int i,int ij) {return s[9*ij+5];}
    inline M a_ul(int i,int ij) {return s[9*ij+6];}
    inline M a_uc(int i,int ij) {return s[9*ij+7];}
    inline M a_ur(int i,int ij) {return s[9*ij+8];}
    inline V inv_cc(int i,int ij,V v) {return v/s[9*ij+4];}
    inline V mul_a(int i,int ij) {
        const M* c=s+9*ij;
        const V* w=z+ij;
        V r=0;
        if(ij>=m) {
            if(i>0) r+=c[0]*w[-m-1];
            r+=c[1]*w[-m];
            if(i<m-1) r+=c[2]*w[-m+1];
        }
        if(i>0) r+=c[3]*w[-1];
        if(i<m-1) r+=c[5]*w[1];
        if(ij<mn-m) {
            if(i>0) r+=c[6]*w[m-1];
            r+=c[7]*w[m];
            if(i<m-1) r+=c[8]*w[m+1];
        }
        return r;
    }
  private:
    tgmg_level(const tgmg_level&);
    tgmg_level& operator=(const tgmg_level&);
};

/** Operations shared by every level: smoothing, residuals and output. */
template<class S,class V,class M>
class tgmg_base {
    public:
        S& sys;
        V* const b;
        V* const z;
        const int m,n,mn;
        tgmg_base(S& sys_,V* b_,V* z_) : sys(sys_), b(b_), z(z_),
            m(sys_.m), n(sys_.n), mn(sys_.m*sys_.n) {}
        void clear_z();
        void smooth(int sweeps,bool reverse);
        double residual(V* r);
        double res_norm_sq();
        double b_norm_sq();
        void output(const char* filename,V* data,double ax,double dx,double ay,double dy);
        void output_res(const char* filename,double ax,double dx,double ay,double dy);
        inline void output_b(const char* filename,double ax,double dx,double ay,double dy) {
            output(filename,b,ax,dx,ay,dy);
        }
        inline void output_z(const char* filename,double ax,double dx,double ay,double dy) {
            output(filename,z,ax,dx,ay,dy);
        }
        /** Fetches the 9-point stencil of the system at (i,j) in the order
         * [dl,dc,dr,cl,cc,cr,ul,uc,ur], zeroing entries that leave the grid. */
        inline void stencil(int i,int j,M* c) {
            int ij=i+m*j;
            c[0]=sys.a_dl(i,ij);c[1]=sys.a_dc(i,ij);c[2]=sys.a_dr(i,ij);
            c[3]=sys.a_cl(i,ij);c[4]=sys.a_cc(i,ij);c[5]=sys.a_cr(i,ij);
            c[6]=sys.a_ul(i,ij);c[7]=sys.a_uc(i,ij);c[8]=sys.a_ur(i,ij);
            for(int k=0;k<9;k++) {
                int di=k%3-1,dj=k/3-1;
                if(i+di<0||i+di>=m||j+dj<0||j+dj>=n) c[k]=0;
            }
        }
};

/** The multigrid solver for a problem class S. */
template<class S,class V,class M>
class tgmg : public tgmg_base<S,V,M> {
    public:
        tgmg(S& sys_,V* b_,V* z_);
        ~tgmg();
        void setup();
        bool solve_v_cycle(tgmg_predict& tp);
        void v_cycle();
    private:
        typedef tgmg_level<V,M> level;
        typedef tgmg_base<level,V,M> lbase;
        std::vector<level*> lev;
        std::vector<lbase*> lb;
        std::vector<V*> rc;
        V* r;
        bool ready;
        /** Dense LU factors of the coarsest operator. */
        std::vector<double> lu;
        std::vector<int> piv;
        int ndense;
        void free_levels();
        template<class T> void galerkin(tgmg_base<T,V,M>& f,level& c);
        template<class T> void factor_dense(tgmg_base<T,V,M>& f);
        void solve_dense(V* bb,V* zz);
        void restrict_to(int fm,int fn,const V* rf,level& c);
        void prolong_add(const level& c,int fm,int fn,V* zf);
        void coarse_cycle(int l);
        tgmg(const tgmg&);
        tgmg& operator=(const tgmg&);
};

#endif
