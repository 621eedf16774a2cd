// ORACLE TEST INFRASTRUCTURE — not part of the product.
//
// Command-line driver over the reference's own classes (compiled unmodified
// from the reference sources against the shims in this directory). Tests and
// the CPU baseline run it as a subprocess, so a reference fatal_error()
// (common.cc:44-47 calls exit) cannot take the test process down.
//
//   step  <cfg> <nsteps> <out> [<in>]   run nsteps of fluid_2d::step_forward
//                                       (fluid_2d.cc:93-405) with the frame
//                                       timestep of fluid_2d::solve
//                                       (fluid_2d.cc:42), from init_fields
//                                       (fluid_2d_sio.cc:14-35) or from the
//                                       state file <in>; writes the state
//   dump  <cfg> <nsteps> <every> <out>  like step, appending a state every
//                                       <every> steps
//   time  <cfg> <nsteps> [<warmup>]     time nsteps after warmup untimed steps;
//                                       prints one JSON line
//   mac|fem <m> <n> <dx> <dy> <b> <z>   one solve with the test constructor
//                                       (mgs_mac.cc:23-27, mgs_fem.cc:26-30)
//                                       as mg_test.cc:20-35 does
//   visc <cfg> <vfx> <vfy> <horiz> <b> <z>  visco_impl::setup_and_solve
//                                       (visco_impl.cc:21-39)
//   heights <cfg> <nsteps> <out>        from init_fields, nsteps steps; writes
//                                       for steps 0..nsteps the time and the
//                                       gas-layer height h[m], the per-step
//                                       input of the lift-off analysis
//                                       (tt_analysis.cc:97-164)
//   tracers <cfg> <nsteps> <out>        from init_fields (tracers placed with
//                                       rand(), fluid_2d.cc:495-502), nsteps
//                                       steps; writes for steps 0..nsteps the
//                                       time, Vframe and the 2*ntrace tracer
//                                       coordinates (fluid_2d.cc:507-526,
//                                       fluid_2d_sio.cc:228-253)
//   tri  <n> <abcd> <out> [thomas]      tri_solve::solve_lapack
//                                       (tri_solve.cc:24-33) or solve()
//                                       (tri_solve.cc:37-49)
//
// State file: int32 m,n; double time,Vframe; u,v,p over the ghosted
// (m+4)x(n+4) array (row-major, row j+2, column i+2); then the gas layer's
// p[m+1], tau[m+4], h[m], fbd[m], pg[m+1], ht[m].
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "fluid_2d.hh"
#include "gas_layer_solve.hh"
#include "mgs_mac.hh"
#include "mgs_fem.hh"
#include "visco_impl.hh"
#include "tri_solve.hh"

static std::vector<double> read_doubles(const char* fn,size_t n) {
    std::vector<double> v(n);
    FILE* f=fopen(fn,"rb");
    if(f==NULL||fread(&v[0],sizeof(double),n,f)!=n) {fprintf(stderr,"cannot read %s\n",fn);exit(2);}
    fclose(f);
    return v;
}

static void write_doubles(const char* fn,const double* p,size_t n) {
    FILE* f=fopen(fn,"wb");
    if(f==NULL) {fprintf(stderr,"cannot write %s\n",fn);exit(2);}
    fwrite(p,sizeof(double),n,f);
    fclose(f);
}

static gas_layer_solve* gls(fluid_2d& f) {
    gas_layer_solve* g=dynamic_cast<gas_layer_solve*>(f.gl);
    if(g==NULL) {fputs("gas_layer_model required\n",stderr);exit(2);}
    return g;
}

static void save_state(fluid_2d& f,FILE* o) {
    int m=f.m,n=f.n,ml=f.ml,tot=ml*(n+4);
    gas_layer_solve* g=gls(f);
    fwrite(&m,sizeof(int),1,o);fwrite(&n,sizeof(int),1,o);
    fwrite(&f.time,sizeof(double),1,o);fwrite(&g->Vframe,sizeof(double),1,o);
    std::vector<double> buf(tot);
    for(int k=0;k<tot;k++) buf[k]=f.fbase[k].u;
    fwrite(&buf[0],sizeof(double),tot,o);
    for(int k=0;k<tot;k++) buf[k]=f.fbase[k].v;
    fwrite(&buf[0],sizeof(double),tot,o);
    for(int k=0;k<tot;k++) buf[k]=f.fbase[k].p;
    fwrite(&buf[0],sizeof(double),tot,o);
    fwrite(g->p,sizeof(double),m+1,o);
    fwrite(g->tau,sizeof(double),m+4,o);
    fwrite(g->h,sizeof(double),m,o);
    fwrite(g->fbd,sizeof(double),m,o);
    fwrite(g->pg,sizeof(double),m+1,o);
    fwrite(g->ht,sizeof(double),m,o);
}

static void load_state(fluid_2d& f,const char* fn) {
    FILE* in=fopen(fn,"rb");
    if(in==NULL) {fprintf(stderr,"cannot read %s\n",fn);exit(2);}
    int m,n;
    gas_layer_solve* g=gls(f);
    bool ok=fread(&m,sizeof(int),1,in)==1&&fread(&n,sizeof(int),1,in)==1;
    if(!ok||m!=f.m||n!=f.n) {fputs("state size mismatch\n",stderr);exit(2);}
    ok=fread(&f.time,sizeof(double),1,in)==1&&fread(&g->Vframe,sizeof(double),1,in)==1;
    int tot=f.ml*(n+4);
    std::vector<double> buf(tot);
    ok=ok&&fread(&buf[0],sizeof(double),tot,in)==size_t(tot);
    for(int k=0;k<tot;k++) f.fbase[k].u=buf[k];
    ok=ok&&fread(&buf[0],sizeof(double),tot,in)==size_t(tot);
    for(int k=0;k<tot;k++) f.fbase[k].v=buf[k];
    ok=ok&&fread(&buf[0],sizeof(double),tot,in)==size_t(tot);
    for(int k=0;k<tot;k++) f.fbase[k].p=buf[k];
    ok=ok&&fread(g->p,sizeof(double),m+1,in)==size_t(m+1);
    ok=ok&&fread(g->tau,sizeof(double),m+4,in)==size_t(m+4);
    ok=ok&&fread(g->h,sizeof(double),m,in)==size_t(m);
    ok=ok&&fread(g->fbd,sizeof(double),m,in)==size_t(m);
    ok=ok&&fread(g->pg,sizeof(double),m+1,in)==size_t(m+1);
    ok=ok&&fread(g->ht,sizeof(double),m,in)==size_t(m);
    if(!ok) {fputs("short state file\n",stderr);exit(2);}
    fclose(in);
    // hx is derived from h (gas_layer_solve.cc:55-59); recompute it the same
    // way the reference's restart loader does (gas_layer_solve.cc:318).
    for(int i=1;i<m;i++) g->hx[i]=g->xsp*(g->h[i]-g->h[i-1]);
    g->hx[0]=g->x_sym?0:g->hx[1];
    g->hx[m]=g->hx[m-1];
}

static double frame_dt(fluid_2d& f) {
    const char* e=getenv("VDI_REF_DT");
    if(e) return atof(e);
    double adt;
    f.timestep_select(f.t_end/f.nframes,adt);
    return adt;
}

static int run_steps(int argc,char** argv,bool dump,bool timed) {
    fluid_2d f(argv[2]);
    int nsteps=atoi(argv[3]);
    int every=dump?atoi(argv[4]):0;
    const char* out=timed?NULL:argv[dump?5:4];
    const char* in=(!dump&&!timed&&argc>5)?argv[5]:NULL;
    if(in) load_state(f,in);
    else f.init_fields();
    double dt=frame_dt(f);
    if(timed&&argc>4) for(int k=atoi(argv[4]);k>0;k--) f.step_forward(dt);
    FILE* o=NULL;
    if(dump) {o=fopen(out,"wb");save_state(f,o);}
    tgmg_stats_t& st=tgmg_stats();
    long v0=st.vcycles,s0=st.solves;
    double t0=wtime();
    for(int k=1;k<=nsteps;k++) {
        f.step_forward(dt);
        if(dump&&k%every==0) save_state(f,o);
    }
    double t1=wtime();
    if(dump) fclose(o);
    else if(!timed) {o=fopen(out,"wb");save_state(f,o);fclose(o);}
    int threads=1;
#ifdef _OPENMP
    threads=omp_get_max_threads();
#endif
    printf("{\"steps\": %d, \"dt\": %.17g, \"seconds\": %.9g, \"steps_per_s\": %.9g, "
           "\"solves\": %ld, \"vcycles\": %ld, \"threads\": %d, \"mg_failures\": %d}\n",
           nsteps,dt,t1-t0,nsteps/(t1-t0),st.solves-s0,st.vcycles-v0,threads,st.failures);
    return 0;
}

static void height_row(fluid_2d& f,std::vector<double>& rows) {
    gas_layer_solve* g=gls(f);
    rows.push_back(f.time);
    rows.insert(rows.end(),g->h,g->h+f.m);
}

static int run_heights(char** argv) {
    fluid_2d f(argv[2]);
    int nsteps=atoi(argv[3]);
    f.init_fields();
    double dt=frame_dt(f);
    std::vector<double> rows;
    height_row(f,rows);
    for(int k=1;k<=nsteps;k++) {
        f.step_forward(dt);
        height_row(f,rows);
    }
    write_doubles(argv[4],&rows[0],rows.size());
    printf("{\"steps\": %d, \"dt\": %.17g}\n",nsteps,dt);
    return 0;
}

static void tracer_row(fluid_2d& f,std::vector<double>& rows) {
    rows.push_back(f.time);
    rows.push_back(gls(f)->Vframe);
    rows.insert(rows.end(),f.tm,f.tm+2*f.ntrace);
}

static int run_tracers(char** argv) {
    fluid_2d f(argv[2]);
    int nsteps=atoi(argv[3]);
    f.init_fields();
    double dt=frame_dt(f);
    std::vector<double> rows;
    tracer_row(f,rows);
    for(int k=1;k<=nsteps;k++) {
        f.step_forward(dt);
        tracer_row(f,rows);
    }
    write_doubles(argv[4],&rows[0],rows.size());
    printf("{\"steps\": %d, \"dt\": %.17g, \"ntrace\": %d}\n",nsteps,dt,f.ntrace);
    return 0;
}

template<class T>
static int solve_one(T& msu,const char* zfile) {
    msu.mg.setup();
    bool ok=msu.mg.solve_v_cycle(msu.tp);
    write_doubles(zfile,msu.z,msu.mn);
    tgmg_stats_t& st=tgmg_stats();
    printf("{\"ok\": %d, \"vcycles\": %d, \"rel_res\": %.6g}\n",ok?1:0,st.last_vcycles,st.last_rel_res);
    return ok?0:1;
}

int main(int argc,char** argv) {
    if(argc<2) {fputs("usage: see source header\n",stderr);return 2;}
    const char* cmd=argv[1];
    if(strcmp(cmd,"step")==0&&argc>=5) return run_steps(argc,argv,false,false);
    if(strcmp(cmd,"dump")==0&&argc>=6) return run_steps(argc,argv,true,false);
    if(strcmp(cmd,"time")==0&&argc>=4) return run_steps(argc,argv,false,true);
    if(strcmp(cmd,"heights")==0&&argc>=5) return run_heights(argv);
    if(strcmp(cmd,"tracers")==0&&argc>=5) return run_tracers(argv);
    if((strcmp(cmd,"mac")==0||strcmp(cmd,"fem")==0)&&argc>=8) {
        int m=atoi(argv[2]),n=atoi(argv[3]);
        double dx=atof(argv[4]),dy=atof(argv[5]);
        std::vector<double> b=read_doubles(argv[6],size_t(m)*n);
        if(cmd[0]=='m') {mgs_mac msu(m,n,dx,dy,&b[0]);return solve_one(msu,argv[7]);}
        mgs_fem msu(m,n,dx,dy,&b[0]);
        return solve_one(msu,argv[7]);
    }
    if(strcmp(cmd,"visc")==0&&argc>=8) {
        fluid_2d f(argv[2]);
        double vfx=atof(argv[3]),vfy=atof(argv[4]);
        bool horiz=atoi(argv[5])!=0;
        std::vector<double> b=read_doubles(argv[6],size_t(f.m)*f.n);
        visco_impl vi(f,horiz);
        memcpy(f.src,&b[0],sizeof(double)*f.m*f.n);
        vi.setup_and_solve(vfx,vfy,0.);
        write_doubles(argv[7],vi.z,vi.mn);
        tgmg_stats_t& st=tgmg_stats();
        printf("{\"ok\": 1, \"vcycles\": %d, \"rel_res\": %.6g}\n",st.last_vcycles,st.last_rel_res);
        return 0;
    }
    if(strcmp(cmd,"tri")==0&&argc>=5) {
        int n=atoi(argv[2]);
        std::vector<double> abcd=read_doubles(argv[3],size_t(4)*n);
        tri_solve t(n);
        memcpy(t.a,&abcd[0],sizeof(double)*4*n);
        if(argc>5&&strcmp(argv[5],"thomas")==0) t.solve();
        else t.solve_lapack();
        write_doubles(argv[4],t.d,n);
        return 0;
    }
    fputs("bad arguments\n",stderr);
    return 2;
}
