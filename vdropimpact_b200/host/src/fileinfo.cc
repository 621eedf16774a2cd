// fileinfo (fileinfo.cc:11-193) over the C-ABI parser: the .cfg text goes to
// vdi_params_from_cfg (physics, unit conversion, domain) and
// vdi_run_options_from_cfg (output flags, restart frequency, tracers,
// timing format). A parse error exits through fatal_error, as the
// reference's checks do.
#include "fileinfo.hh"

#include <cstring>
#include <string>

#include "common.hh"

fileinfo::fileinfo(const char* infile)
    : m(-1), fflags(0), ntrace(0), nframes(-1), restart_freq(0), nif_mode(0), implicit_visc(false), x_sym(false),
      mr_time_output(false), ay(0.), tmult(-1), filename(NULL), gl(NULL) {
    int l = strlen(infile);
    if (l < 4) fatal_error("Filename is too short", 1);
    const char* ip = infile + l - 4;
    if (*ip != '.' || ip[1] != 'c' || ip[2] != 'f' || ip[3] != 'g') fatal_error("Filename must end in '.cfg'", 1);
    filename = new char[l + 1];
    memcpy(filename, infile, l - 3);
    char* fp = filename + l - 3;
    fp[0] = 'o';
    fp[1] = 'd';
    fp[2] = 'r';
    fp[3] = 0;
    FILE* f = safe_fopen(infile, "r");
    std::string text;
    char chunk[4096];
    size_t k;
    while ((k = fread(chunk, 1, sizeof(chunk), f)) > 0) text.append(chunk, k);
    fclose(f);
    vdi_run_options ro;
    int st = vdi_params_from_cfg(text.c_str(), &params);
    if (st == VDI_OK) st = vdi_run_options_from_cfg(text.c_str(), &ro);
    if (st != VDI_OK) fatal_error(vdi_last_error(), 1);
    m = params.m;
    n = params.n;
    fflags = ro.fflags;
    ntrace = params.ntrace;
    nif_mode = params.nif_mode;
    anif = params.nif_a;
    bnif = params.nif_b;
    nframes = params.nframes;
    restart_freq = ro.restart_freq;
    implicit_visc = params.implicit_visc != 0;
    x_sym = params.x_sym != 0;
    mr_time_output = ro.mr_time_output != 0;
    ax = params.ax;
    bx = params.bx;
    by = params.by;
    dx = (bx - ax) / m;
    dy = (by - ay) / n;
    xsp = 1. / dx;
    ysp = 1. / dy;
    rho = params.rho;
    mu = params.mu;
    muinv = 1. / mu;
    rhoinv = 1. / rho;
    tmult = params.tmult;
    t_end = params.t_end;
    gl = new gas_layer_solve(m, ax, bx, params.R, params.V, params.h0);
}

fileinfo::~fileinfo() {
    delete gl;
    delete[] filename;
}
