// Step-level harness around the FLUXOS reference sources, compiled here from
// the reference tree by oracle/Makefile into oracle/_ref/.
//
// TEST INFRASTRUCTURE ONLY. It links the reference's own translation units
// (hydrodynamics_calc.cpp, solver_wetdomain.cpp, solver_drydomain.cpp,
// ADEsolver_calc.cpp, common.cpp, initiate.cpp, read_functions.cpp,
// write_results.cpp, WINTRAsolver_calc.cpp and main.cpp renamed to
// fluxos_ref_main) and exposes a plain C API so tests can drive the reference
// one time step at a time and read its GlobVar grids.
//
// The start-up sequence below repeats main.cpp:104-262 call for call, and
// fxr_step repeats one iteration of the step loop main.cpp:273-406 (without
// the OpenWQ branches, which the oracle never enables). The Courant scan of
// main.cpp:300-323 lives inline in main(), so it is restated here; the
// whole-program entry point fluxos_ref_main is used to check that restatement.
#include <armadillo>
#include <chrono>
#include <cmath>
#include <cstring>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "ADEsolver_calc.h"
#include "GlobVar.h"
#include "WINTRAsolver_calc.h"
#include "common.h"
#include "hydrodynamics_calc.h"
#include "initiate.h"
#include "read_functions.h"
#include "write_results.h"

// The OpenWQ coupler (src/openwq/OpenWQ_hydrolink.cpp) needs the absent
// OpenWQ library; these empty definitions satisfy the linker. They are only
// reachable when the OPENWQ module is on, which the oracle never enables.
void openwq_hydrolink::openwq_decl(OpenWQ_couplercalls&, OpenWQ_hostModelconfig&, OpenWQ_json&,
                                   OpenWQ_wqconfig&, OpenWQ_units&, OpenWQ_utils&, OpenWQ_readjson&,
                                   OpenWQ_vars&, OpenWQ_initiate&, OpenWQ_watertransp&, OpenWQ_chem&,
                                   OpenWQ_extwatflux_ss&, OpenWQ_output&, std::string, unsigned long,
                                   unsigned long) {}
void openwq_hydrolink::openwq_time_start(OpenWQ_couplercalls&, OpenWQ_hostModelconfig&, OpenWQ_json&,
                                         OpenWQ_wqconfig&, OpenWQ_units&, OpenWQ_utils&,
                                         OpenWQ_readjson&, OpenWQ_vars&, OpenWQ_initiate&,
                                         OpenWQ_watertransp&, OpenWQ_chem&, OpenWQ_extwatflux_ss&,
                                         OpenWQ_solver&, OpenWQ_output&, GlobVar&) {}
void openwq_hydrolink::run_space_in(GlobVar&, OpenWQ_couplercalls&, OpenWQ_hostModelconfig&,
                                    OpenWQ_json&, OpenWQ_wqconfig&, OpenWQ_units&, OpenWQ_utils&,
                                    OpenWQ_readjson&, OpenWQ_vars&, OpenWQ_initiate&,
                                    OpenWQ_watertransp&, OpenWQ_chem&, OpenWQ_extwatflux_ss&,
                                    OpenWQ_solver&, OpenWQ_output&, std::string, int, int, double) {}
void openwq_hydrolink::openwq_time_end(OpenWQ_couplercalls&, OpenWQ_hostModelconfig&, OpenWQ_json&,
                                       OpenWQ_wqconfig&, OpenWQ_units&, OpenWQ_utils&, OpenWQ_readjson&,
                                       OpenWQ_vars&, OpenWQ_initiate&, OpenWQ_watertransp&,
                                       OpenWQ_chem&, OpenWQ_extwatflux_ss&, OpenWQ_solver&,
                                       OpenWQ_output&, GlobVar&) {}

namespace {

// Coupler objects the reference's forcing functions take by reference.
struct Coupler {
  OpenWQ_couplercalls cc;
  OpenWQ_hostModelconfig hm;
  OpenWQ_json js;
  OpenWQ_wqconfig wq;
  OpenWQ_units un;
  OpenWQ_utils ut;
  OpenWQ_readjson rj;
  OpenWQ_vars vars{1, 2};
  OpenWQ_initiate in;
  OpenWQ_watertransp wt;
  OpenWQ_chem ch;
  OpenWQ_extwatflux_ss ss;
  OpenWQ_solver so;
  OpenWQ_output ou;
  openwq_hydrolink link;
};

struct RefRun {
  std::unique_ptr<GlobVar> ds;
  Coupler cp;
  std::ofstream log;
  unsigned int it = 0;
  unsigned int print_next = 0;
  int nchem = 1;
  std::vector<unsigned int> chem_mobile{0};
  double hpall = 0.0;
  std::chrono::time_point<std::chrono::system_clock> start;
};

std::string dir_of(const std::string& s) {
  size_t found = s.find_last_of("/\\");
  return s.substr(0, found);
}

}  // namespace

// main.cpp is compiled with -Dmain=fluxos_ref_main (C++ linkage).
int fluxos_ref_main(int argc, char* argv[]);

extern "C" {

// The whole reference program: fxr_main(modset_path) == `fluxos <modset>`.
int fxr_main(const char* modset_path) {
  std::string a0("fluxos"), a1(modset_path);
  char* argv[] = {&a0[0], &a1[0], nullptr};
  return fluxos_ref_main(2, argv);
}

// main.cpp:104-262 (start-up), with ds.tim set to 0 because GlobVar leaves
// it uninitialised (GlobVar.h:94) and the reference never assigns it before
// the loop at main.cpp:271.
void* fxr_open(const char* modset_path) {
  auto* r = new RefRun();
  std::string modset(modset_path);
  r->log.open(dir_of(modset) + "/fluxos_ref_harness.log");
  json master;
  std::ifstream i(modset);
  master = json::parse(i, nullptr, false, true);
  unsigned int nr = 0, nc = 0;
  if (get_domain_size(&nr, &nc, master, r->log)) {
    delete r;
    return nullptr;
  }
  r->ds.reset(new GlobVar(nr + 2, nc + 2));
  GlobVar& ds = *r->ds;
  ds.cfl = 1;
  ds.ntim = 0;
  ds.cvdef = 0.07;
  ds.nuem = 1.793e-6;
  ds.master_MODSET = master;
  double ks_input = 0.0;
  if (read_modset(ds, modset, &ks_input, r->log)) {
    delete r;
    return nullptr;
  }
  ds.NROWS = ds.MROWS - 2;
  ds.NCOLS = ds.MCOLS - 2;
  if (read_geo(ds, ks_input, r->log)) {
    delete r;
    return nullptr;
  }
  ds.arbase = ds.dxy * ds.dxy;
  int ntim_meteo = read_meteo(ds, r->log);
  int ntim_inflow = read_inflow(ds, r->log);
  ds.ntim = std::max(ntim_meteo, ntim_inflow);
  if (ds.ade_solver != true) {
    ds.wintra = false;
    ds.openwq = false;
  }
  r->nchem = 1;
  unsigned int timstart = initiation(ds, r->nchem, r->log);
  ds.hdry = (*ds.ks).at(1, 1);
  r->print_next = timstart + ds.print_step;
  if (ds.wintra == true) ds.SWEstd = ds.SWEstd / 100;
  ds.tim = 0.0;
  ds.dtfl = 0.0;
  r->start = std::chrono::system_clock::now();
  return r;
}

void fxr_close(void* h) { delete static_cast<RefRun*>(h); }

int fxr_running(void* h) {
  auto* r = static_cast<RefRun*>(h);
  return r->ds->tim <= r->ds->ntim;
}

// Courant scan, restated from main.cpp:300-323 (inline in main()).
void fxr_courant(void* h) {
  auto* r = static_cast<RefRun*>(h);
  GlobVar& ds = *r->ds;
  ds.dtfl = 9.e10;
  r->hpall = 0.0f;
  double c0, hp, u0, v0;
  for (unsigned int icol = 1; icol <= ds.NCOLS; icol++) {
    for (unsigned int irow = 1; irow <= ds.NROWS; irow++) {
      hp = (*ds.h).at(irow, icol);
      (*ds.h0)(irow, icol) = hp;
      (*ds.ldry_prev).at(irow, icol) = (*ds.ldry).at(irow, icol);
      if (hp > ds.hdry) {
        (*ds.ldry).at(irow, icol) = 0.0f;
        hp = std::fmax((*ds.h).at(irow, icol), ds.hdry);
        r->hpall = std::fmax(r->hpall, (*ds.h).at(irow, icol));
        c0 = sqrt(ds.gacc * (*ds.h).at(irow, icol));
        u0 = std::fmax(.000001, fabs((*ds.qx).at(irow, icol) / hp));
        v0 = std::fmax(.000001, fabs((*ds.qy).at(irow, icol) / hp));
        ds.dtfl = fmin(fmin(ds.cfl * ds.dxy / (u0 + c0), ds.cfl * ds.dxy / (v0 + c0)), ds.dtfl);
      } else {
        (*ds.ldry).at(irow, icol) = 1.0f;
      }
      ds.dtfl = fmin(r->print_next - ds.tim, ds.dtfl);
    }
  }
}

int fxr_add_meteo(void* h) {
  auto* r = static_cast<RefRun*>(h);
  Coupler& c = r->cp;
  return add_meteo(*r->ds, c.link, c.cc, c.hm, c.js, c.wq, c.un, c.ut, c.rj, c.vars, c.in, c.wt, c.ch,
                   c.ss, c.so, c.ou, r->nchem)
             ? 1
             : 0;
}

int fxr_add_inflow(void* h) {
  auto* r = static_cast<RefRun*>(h);
  Coupler& c = r->cp;
  return add_inflow(*r->ds, c.link, c.cc, c.hm, c.js, c.wq, c.un, c.ut, c.rj, c.vars, c.in, c.wt,
                    c.ch, c.ss, c.so, c.ou, r->nchem)
             ? 1
             : 0;
}

void fxr_hydrodynamics(void* h) { hydrodynamics_calc(*static_cast<RefRun*>(h)->ds); }

void fxr_adesolver(void* h, int it, int ichem) {
  adesolver_calc(*static_cast<RefRun*>(h)->ds, it, ichem);
}

// One iteration of the step loop (main.cpp:273-406), printing excluded.
// Returns 0 on success, 1 when a forcing routine reported an error.
int fxr_step(void* h) {
  auto* r = static_cast<RefRun*>(h);
  GlobVar& ds = *r->ds;
  fxr_courant(h);
  ds.tim = ds.tim + ds.dtfl;
  if (fxr_add_meteo(h)) return 1;
  if (fxr_add_inflow(h)) return 1;
  if (r->hpall != 0) {
    r->it++;
    hydrodynamics_calc(ds);
    if (ds.ade_solver == true)
      for (size_t ichem = 0; ichem < r->chem_mobile.size(); ichem++)
        adesolver_calc(ds, r->it, r->chem_mobile[ichem]);
    if (ds.wintra == true)
      for (size_t ichem = 0; ichem < r->chem_mobile.size(); ichem++)
        wintrasolver_calc(ds, r->chem_mobile[ichem]);
  }
  return 0;
}

// main.cpp:444-468: returns 1 when a Results file was written.
int fxr_maybe_print(void* h) {
  auto* r = static_cast<RefRun*>(h);
  GlobVar& ds = *r->ds;
  if (ds.tim >= r->print_next) {
    auto end = std::chrono::system_clock::now();
    std::chrono::duration<double> el = end - r->start;
    bool ok = write_results(ds, std::round(r->print_next), el);
    if (!ok) return -1;
    r->print_next = r->print_next + ds.print_step;
    r->start = std::chrono::system_clock::now();
    return 1;
  }
  return 0;
}

double* fxr_grid(void* h, const char* name) {
  GlobVar& ds = *static_cast<RefRun*>(h)->ds;
  std::string n(name);
  arma::mat* m = nullptr;
  if (n == "z") m = ds.z.get();
  else if (n == "zb") m = ds.zb.get();
  else if (n == "h") m = ds.h.get();
  else if (n == "ux") m = ds.ux.get();
  else if (n == "uy") m = ds.uy.get();
  else if (n == "qx") m = ds.qx.get();
  else if (n == "qy") m = ds.qy.get();
  else if (n == "qxf") m = ds.qxf.get();
  else if (n == "qyf") m = ds.qyf.get();
  else if (n == "us") m = ds.us.get();
  else if (n == "dh") m = ds.dh.get();
  else if (n == "dqx") m = ds.dqx.get();
  else if (n == "dqy") m = ds.dqy.get();
  else if (n == "ks") m = ds.ks.get();
  else if (n == "fe_1") m = ds.fe_1.get();
  else if (n == "fe_2") m = ds.fe_2.get();
  else if (n == "fe_3") m = ds.fe_3.get();
  else if (n == "fn_1") m = ds.fn_1.get();
  else if (n == "fn_2") m = ds.fn_2.get();
  else if (n == "fn_3") m = ds.fn_3.get();
  else if (n == "twet") m = ds.twetimetracer.get();
  else if (n == "h0") m = ds.h0.get();
  else if (n == "soil_mass") m = ds.soil_mass.get();
  else if (n == "conc") m = &(*ds.conc_SW)[0];
  return m ? m->mem.data() : nullptr;
}

float* fxr_fgrid(void* h, const char* name) {
  GlobVar& ds = *static_cast<RefRun*>(h)->ds;
  std::string n(name);
  arma::fmat* m = nullptr;
  if (n == "ldry") m = ds.ldry.get();
  else if (n == "ldry_prev") m = ds.ldry_prev.get();
  else if (n == "wall") m = ds.innerNeumannBCWeir.get();
  else if (n == "meteo") m = ds.meteo.get();
  else if (n == "inflow") m = ds.inflow.get();
  return m ? m->mem.data() : nullptr;
}

double fxr_scalar(void* h, const char* name) {
  auto* r = static_cast<RefRun*>(h);
  GlobVar& ds = *r->ds;
  std::string n(name);
  if (n == "tim") return ds.tim;
  if (n == "dtfl") return ds.dtfl;
  if (n == "hdry") return ds.hdry;
  if (n == "ntim") return double(ds.ntim);
  if (n == "nrows") return double(ds.NROWS);
  if (n == "ncols") return double(ds.NCOLS);
  if (n == "dxy") return double(ds.dxy);
  if (n == "arbase") return double(ds.arbase);
  if (n == "print_next") return double(r->print_next);
  if (n == "print_step") return double(ds.print_step);
  if (n == "it") return double(r->it);
  if (n == "hpall") return r->hpall;
  if (n == "nodata") return ds.NODATA_VALUE;
  if (n == "xll") return ds.XLLCORNER;
  if (n == "yll") return ds.YLLCORNER;
  if (n == "D_coef") return ds.D_coef;
  if (n == "ade") return ds.ade_solver ? 1.0 : 0.0;
  if (n == "h_min_print") return double(ds.h_min_print);
  if (n == "inflow_nrow") return double(ds.inflow_nrow);
  if (n == "inflow_ncol") return double(ds.inflow_ncol);
  if (n == "has_inflow") return ds.inflow_file.empty() ? 0.0 : 1.0;
  if (n == "has_meteo") return ds.meteo_file.empty() ? 0.0 : 1.0;
  return std::nan("");
}

void fxr_set_scalar(void* h, const char* name, double v) {
  auto* r = static_cast<RefRun*>(h);
  GlobVar& ds = *r->ds;
  std::string n(name);
  if (n == "tim") ds.tim = v;
  else if (n == "dtfl") ds.dtfl = v;
  else if (n == "print_next") r->print_next = (unsigned int)v;
  else if (n == "it") r->it = (unsigned int)v;
}

}  // extern "C"
