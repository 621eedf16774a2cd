// ORACLE TEST INFRASTRUCTURE — not part of the product.
//
// Template definitions for the clean-room TGMG-API shim declared in tgmg.hh.
// The reference includes this file from mgs_common.cc:53, mgs_mac.cc:29,
// mgs_fem.cc:48 and visco_impl.cc:42 and instantiates it explicitly there.
#ifndef VDI_ORACLE_TGMG_CC
#define VDI_ORACLE_TGMG_CC

#include <cstdio>
#include <cstdlib>
#include <cmath>

#include "tgmg.hh"

/** One-dimensional bilinear prolongation weights. Fine point f on a line
 * whose coarse line has cm points takes its value from at most two coarse
 * points; the last odd point of an even-length line copies its one coarse
 * neighbour.
 * \return The number of (index, weight) pairs written. */
inline int tgmg_pw(int f,int cm,int* I,double* w) {
    if((f&1)==0) {I[0]=f>>1;w[0]=1;return 1;}
    int l=f>>1,r=l+1;
    if(r<cm) {I[0]=l;w[0]=0.5;I[1]=r;w[1]=0.5;return 2;}
    I[0]=l;w[0]=1;return 1;
}

/** The weight with which fine point f draws on coarse point I (0 if none). */
inline double tgmg_w(int f,int cm,int I) {
    int J[2];double w[2];
    int k=tgmg_pw(f,cm,J,w);
    for(int q=0;q<k;q++) if(J[q]==I) return w[q];
    return 0;
}

template<class S,class V,class M>
void tgmg_base<S,V,M>::clear_z() {
    for(int ij=0;ij<mn;ij++) z[ij]=0;
}

/** Four-colour Gauss-Seidel: points with equal (i mod 2, j mod 2) do not
 * couple through a 9-point stencil, so each colour updates in parallel. */
template<class S,class V,class M>
void tgmg_base<S,V,M>::smooth(int sweeps,bool reverse) {
    static const int cx[4]={0,1,0,1},cy[4]={0,0,1,1};
    for(int s=0;s<sweeps;s++) for(int q=0;q<4;q++) {
        int c=reverse?3-q:q;
#pragma omp parallel for
        for(int j=cy[c];j<n;j+=2) for(int i=cx[c];i<m;i+=2) {
            int ij=i+m*j;
            z[ij]=sys.inv_cc(i,ij,b[ij]-sys.mul_a(i,ij));
        }
    }
}

/** Computes r=b-Az and returns the sum of squares of r. */
template<class S,class V,class M>
double tgmg_base<S,V,M>::residual(V* r) {
    double s=0;
#pragma omp parallel for reduction(+:s)
    for(int j=0;j<n;j++) for(int i=0;i<m;i++) {
        int ij=i+m*j;
        V q=b[ij]-sys.a_cc(i,ij)*z[ij]-sys.mul_a(i,ij);
        r[ij]=q;
        s+=double(q)*double(q);
    }
    return s;
}

template<class S,class V,class M>
double tgmg_base<S,V,M>::res_norm_sq() {
    double s=0;
#pragma omp parallel for reduction(+:s)
    for(int j=0;j<n;j++) for(int i=0;i<m;i++) {
        int ij=i+m*j;
        double q=double(b[ij]-sys.a_cc(i,ij)*z[ij]-sys.mul_a(i,ij));
        s+=q*q;
    }
    return s;
}

template<class S,class V,class M>
double tgmg_base<S,V,M>::b_norm_sq() {
    double s=0;
#pragma omp parallel for reduction(+:s)
    for(int ij=0;ij<mn;ij++) s+=double(b[ij])*double(b[ij]);
    return s;
}

/** Writes a field in the Gnuplot binary matrix format: a header row of the
 * column count and x coordinates, then one row per j of y and the values. */
template<class S,class V,class M>
void tgmg_base<S,V,M>::output(const char* filename,V* data,double ax,double dx,double ay,double dy) {
    FILE* f=fopen(filename,"wb");
    if(f==NULL) {fprintf(stderr,"Error opening file \"%s\"\n",filename);exit(1);}
    std::vector<float> row(m+1);
    row[0]=float(m);
    for(int i=0;i<m;i++) row[i+1]=float(ax+i*dx);
    fwrite(&row[0],sizeof(float),m+1,f);
    for(int j=0;j<n;j++) {
        row[0]=float(ay+j*dy);
        for(int i=0;i<m;i++) row[i+1]=float(data[i+m*j]);
        fwrite(&row[0],sizeof(float),m+1,f);
    }
    fclose(f);
}

template<class S,class V,class M>
void tgmg_base<S,V,M>::output_res(const char* filename,double ax,double dx,double ay,double dy) {
    std::vector<V> r(mn);
    residual(&r[0]);
    output(filename,&r[0],ax,dx,ay,dy);
}

template<class S,class V,class M>
tgmg<S,V,M>::tgmg(S& sys_,V* b_,V* z_) : tgmg_base<S,V,M>(sys_,b_,z_),
    r(new V[sys_.m*sys_.n]), ready(false), ndense(0) {}

template<class S,class V,class M>
tgmg<S,V,M>::~tgmg() {
    free_levels();
    delete [] r;
}

template<class S,class V,class M>
void tgmg<S,V,M>::free_levels() {
    for(size_t l=0;l<lev.size();l++) {
        delete lb[l];
        delete [] rc[l];
        delete lev[l];
    }
    lev.clear();lb.clear();rc.clear();
    ready=false;
}

/** Builds the coarse level c=P^T A P from the level f, gathering over the
 * fine points that draw on each coarse point so rows can run in parallel. */
template<class S,class V,class M>
template<class T>
void tgmg<S,V,M>::galerkin(tgmg_base<T,V,M>& f,level& c) {
    const int fm=f.m,fn=f.n,cm=c.m,cn=c.n;
#pragma omp parallel for
    for(int J=0;J<cn;J++) for(int I=0;I<cm;I++) {
        double acc[9]={0,0,0,0,0,0,0,0,0};
        M a[9];
        for(int fy=2*J-1;fy<=2*J+1;fy++) {
            if(fy<0||fy>=fn) continue;
            double wy=tgmg_w(fy,cn,J);
            if(wy==0) continue;
            for(int fx=2*I-1;fx<=2*I+1;fx++) {
                if(fx<0||fx>=fm) continue;
                double wx=tgmg_w(fx,cm,I);
                if(wx==0) continue;
                f.stencil(fx,fy,a);
                for(int k=0;k<9;k++) {
                    if(a[k]==0) continue;
                    int gx=fx+k%3-1,gy=fy+k/3-1;
                    int Jx[2],Jy[2];double vx[2],vy[2];
                    int nx=tgmg_pw(gx,cm,Jx,vx),ny=tgmg_pw(gy,cn,Jy,vy);
                    for(int p=0;p<nx;p++) for(int q=0;q<ny;q++) {
                        int ox=Jx[p]-I,oy=Jy[q]-J;
                        acc[(oy+1)*3+ox+1]+=wx*wy*double(a[k])*vx[p]*vy[q];
                    }
                }
            }
        }
        M* s=c.s+9*(I+cm*J);
        for(int k=0;k<9;k++) s[k]=M(acc[k]);
    }
}

/** Assembles the level's operator densely and factors it with partial
 * pivoting. */
template<class S,class V,class M>
template<class T>
void tgmg<S,V,M>::factor_dense(tgmg_base<T,V,M>& f) {
    const int m=f.m,n=f.n,N=m*n;
    ndense=N;
    lu.assign(size_t(N)*N,0.);
    piv.assign(N,0);
    M a[9];
    for(int j=0;j<n;j++) for(int i=0;i<m;i++) {
        f.stencil(i,j,a);
        for(int k=0;k<9;k++) if(a[k]!=0) {
            int g=(i+k%3-1)+m*(j+k/3-1);
            lu[size_t(i+m*j)*N+g]+=double(a[k]);
        }
    }
    for(int k=0;k<N;k++) {
        int p=k;double pv=fabs(lu[size_t(k)*N+k]);
        for(int q=k+1;q<N;q++) if(fabs(lu[size_t(q)*N+k])>pv) {pv=fabs(lu[size_t(q)*N+k]);p=q;}
        piv[k]=p;
        if(p!=k) for(int q=0;q<N;q++) std::swap(lu[size_t(k)*N+q],lu[size_t(p)*N+q]);
        double d=lu[size_t(k)*N+k];
        if(d==0) continue;
        for(int q=k+1;q<N;q++) {
            double l=lu[size_t(q)*N+k]/d;
            lu[size_t(q)*N+k]=l;
            if(l!=0) for(int c=k+1;c<N;c++) lu[size_t(q)*N+c]-=l*lu[size_t(k)*N+c];
        }
    }
}

template<class S,class V,class M>
void tgmg<S,V,M>::solve_dense(V* bb,V* zz) {
    const int N=ndense;
    std::vector<double> x(bb,bb+N);
    for(int k=0;k<N;k++) if(piv[k]!=k) std::swap(x[k],x[piv[k]]);
    for(int k=0;k<N;k++) for(int q=k+1;q<N;q++) x[q]-=lu[size_t(q)*N+k]*x[k];
    for(int k=N-1;k>=0;k--) {
        for(int q=k+1;q<N;q++) x[k]-=lu[size_t(k)*N+q]*x[q];
        double d=lu[size_t(k)*N+k];
        x[k]=d!=0?x[k]/d:0;
    }
    for(int k=0;k<N;k++) zz[k]=V(x[k]);
}

/** Builds the coarse hierarchy with Galerkin operators. */
template<class S,class V,class M>
void tgmg<S,V,M>::setup() {
    free_levels();
    int m=this->m,n=this->n;
    if(m*n<=tgmg_coarse_max||m<3||n<3) {
        factor_dense(*this);
        ready=true;
        return;
    }
    while(true) {
        int cm=(m+1)/2,cn=(n+1)/2;
        level* c=new level(cm,cn);
        if(lev.empty()) galerkin(*this,*c);
        else galerkin(*lb.back(),*c);
        lev.push_back(c);
        lb.push_back(new lbase(*c,c->b,c->z));
        rc.push_back(new V[cm*cn]);
        m=cm;n=cn;
        if(m*n<=tgmg_coarse_max||m<3||n<3) break;
    }
    factor_dense(*lb.back());
    ready=true;
}

/** c.b = P^T rf, gathered per coarse point. */
template<class S,class V,class M>
void tgmg<S,V,M>::restrict_to(int fm,int fn,const V* rf,level& c) {
    const int cm=c.m,cn=c.n;
#pragma omp parallel for
    for(int J=0;J<cn;J++) for(int I=0;I<cm;I++) {
        double s=0;
        for(int fy=2*J-1;fy<=2*J+1;fy++) {
            if(fy<0||fy>=fn) continue;
            double wy=tgmg_w(fy,cn,J);
            if(wy==0) continue;
            for(int fx=2*I-1;fx<=2*I+1;fx++) {
                if(fx<0||fx>=fm) continue;
                double wx=tgmg_w(fx,cm,I);
                if(wx!=0) s+=wx*wy*double(rf[fx+fm*fy]);
            }
        }
        c.b[I+cm*J]=V(s);
    }
}

/** zf += P c.z. */
template<class S,class V,class M>
void tgmg<S,V,M>::prolong_add(const level& c,int fm,int fn,V* zf) {
    const int cm=c.m,cn=c.n;
#pragma omp parallel for
    for(int j=0;j<fn;j++) for(int i=0;i<fm;i++) {
        int Ix[2],Iy[2];double wx[2],wy[2];
        int nx=tgmg_pw(i,cm,Ix,wx),ny=tgmg_pw(j,cn,Iy,wy);
        double s=0;
        for(int p=0;p<nx;p++) for(int q=0;q<ny;q++) s+=wx[p]*wy[q]*double(c.z[Ix[p]+cm*Iy[q]]);
        zf[i+fm*j]+=V(s);
    }
}

template<class S,class V,class M>
void tgmg<S,V,M>::coarse_cycle(int l) {
    level& L=*lev[l];
    if(l+1==int(lev.size())) {solve_dense(L.b,L.z);return;}
    lbase& B=*lb[l];
    B.clear_z();
    B.smooth(tgmg_nu1,false);
    B.residual(rc[l]);
    restrict_to(L.m,L.n,rc[l],*lev[l+1]);
    coarse_cycle(l+1);
    prolong_add(*lev[l+1],L.m,L.n,L.z);
    B.smooth(tgmg_nu2,true);
}

template<class S,class V,class M>
void tgmg<S,V,M>::v_cycle() {
    if(!ready) setup();
    if(lev.empty()) {solve_dense(this->b,this->z);return;}
    this->smooth(tgmg_nu1,false);
    this->residual(r);
    restrict_to(this->m,this->n,r,*lev[0]);
    coarse_cycle(0);
    prolong_add(*lev[0],this->m,this->n,this->z);
    this->smooth(tgmg_nu2,true);
}

/** V-cycles until ||b-Az||_2 <= rtol*||b||_2. Returns false on a
 * non-finite residual or when tgmg_max_vcycles is reached. */
template<class S,class V,class M>
bool tgmg<S,V,M>::solve_v_cycle(tgmg_predict& tp) {
    if(!ready) setup();
    tgmg_stats_t& st=tgmg_stats();
    double bn=sqrt(this->b_norm_sq());
    if(bn==0) {
        this->clear_z();
        tp.record(0);
        st.solves++;st.last_vcycles=0;st.last_rel_res=0;
        return true;
    }
    double thr=tgmg_rtol_ref()*bn,rn=sqrt(this->res_norm_sq());
    int k=0;
    while(!(rn<=thr)) {
        if(k>=tgmg_max_vcycles||!std::isfinite(rn)) {
            tp.record(k);
            st.solves++;st.vcycles+=k;st.last_vcycles=k;st.last_rel_res=rn/bn;st.failures++;
            return false;
        }
        v_cycle();k++;
        rn=sqrt(this->res_norm_sq());
    }
    tp.record(k);
    st.solves++;st.vcycles+=k;st.last_vcycles=k;st.last_rel_res=rn/bn;
    return true;
}

#endif
