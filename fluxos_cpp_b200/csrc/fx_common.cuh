// Shared definitions of the B200 FLUXOS-OVERLAND step kernels.
//
// Grid layout in HBM (structure of arrays, one allocation per field):
//   a field holds the (nrows+2) x (ncols+2) grid of the reference's GlobVar
//   (ghost ring included), column-major with irow fastest. Every column is
//   padded to `ld` elements, a multiple of 32, and row irow is stored at
//   position irow + FX_ROFF. The 1-element offset puts tile halo starts
//   (irow0 - 2 for tiles of 32 rows starting at irow 1 + 32k) on 32-element,
//   and therefore 256-byte, boundaries.
//   Element (irow, icol) of field f is f[icol * ld + irow + FX_ROFF].
#pragma once
#include <cstdint>

#define FX_ROFF 1
#define FX_MAX_CHEM 8
#define FX_METEO_ROWS 2000

// Per-cell flag byte.
#define FX_F_LDRY 0x01       // ldry (1 = dry) at the end of the last step
#define FX_F_LDRY_PREV 0x02  // ldry_prev of the last step (ADE rescale)
#define FX_F_WALL 0x04       // innerNeumannBCWeir (NODATA or 0 DEM cell)

// Device error codes (fx_ctl::error).
#define FX_DEVERR_WAIT_TIMEOUT 1

// Step control block, resident in device memory. One thread of k_finalize
// advances the clock exactly as main.cpp:271-325 does; every other kernel of
// the step reads it.
struct fx_ctl {
  double tim;         // simulated clock [s] (GlobVar::tim)
  double dtfl;        // this step's dt (GlobVar::dtfl)
  double ntim;        // run length: loop while tim <= ntim (main.cpp:271)
  double print_next;  // next output time (main.cpp:260-261)
  double print_step;
  double hpall;       // max wet depth seen by this step's Courant scan
  double meteoi;      // uniform melt depth added this step [m]
  double meteo_rate;  // forcing rate of this step's row [mm/day]
  double mconc;       // forcing concentration of this step's row
  unsigned long long acc_dtmin;  // bits of the running min of cell dts
  unsigned long long acc_hmax;   // bits of the running max wet depth
  long long steps;       // steps executed so far
  long long stop_after;  // do not start a step once steps == stop_after
  int it;                // solver iterations (main.cpp:387)
  int live;              // 1 while the current step runs
  int active;            // hpall != 0 in the current step
  int print_pending;     // tim >= print_next after the last step
  int finished;          // the loop condition tim <= ntim failed
  int forcing_overrun;   // the forcing table had no row with t > tim
  int error;             // FX_DEVERR_* set by a kernel
  int pad_;
};

// Everything a kernel needs, passed by value.
struct fx_dev {
  int nr, nc, ld, nchem;
  unsigned dxy_u;     // integer cell size (GlobVar.h:76)
  double dxy;         // same, as double
  double arbase;      // dxy*dxy (main.cpp:176)
  double hdry;        // dry threshold = ks(1,1) (main.cpp:259)
  double ks;          // roughness height of interior cells (ghost ks is 0)
  double nodata;      // NODATA_VALUE
  double gaccl;       // (double)(float)9.80665 (GlobVar.h:78)
  double sqrt_gaccl;  // sqrt(gaccl)
  double nueml;       // (double)(float)1.793e-6 (main.cpp:135)
  double cvdefl;      // (double)(float)0.07 (main.cpp:134)
  double cfl_dxy;     // (double)((float)cfl * (float)dxy) (main.cpp:316)
  int volrat_mode;    // 0: edge flux = weir formula, 1: edge flux = 0
  int ade;            // ADE module on
  int store_all_fluxes;  // 1 when forcing can remove water (see k_hydro)
  int pad_;
  double dcoef[FX_MAX_CHEM];
  // state
  double *z, *zb, *h, *qx, *qy, *twet, *h0;
  double *fe1, *fe2, *fe3, *fn1, *fn2, *fn3;
  double* conc;       // nchem planes of ld*(nc+2)
  uint8_t* flags;
  // extensions (nullptr = off)
  const double* manning;
  const double* melt_mult;
  // forcing table: times, rates, concentrations (float, as GlobVar::meteo)
  const float* meteo_t;
  const float* meteo_r;
  const float* meteo_c;
  int has_meteo;
  int pad2_;
  fx_ctl* ctl;
  // ADE sweep scratch
  double* ade_bnd;                 // per solute, per strip: (ncols+2) x 3
  unsigned long long* ade_prog;    // per solute, per strip: epoch<<32 | steps done
  long long plane;                 // elements per field = ld * (nc + 2)
};

__host__ __device__ inline long long fx_ix(const fx_dev& d, int irow, int icol) {
  return (long long)icol * d.ld + irow + FX_ROFF;
}
