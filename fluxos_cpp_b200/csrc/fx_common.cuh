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
#define FX_MAX_SLOTS 64

// Per-cell flag byte.
#define FX_F_LDRY 0x01       // ldry (1 = dry) at the end of the last step
#define FX_F_LDRY_PREV 0x02  // ldry_prev of the last step (ADE rescale)
#define FX_F_WALL 0x04       // innerNeumannBCWeir (NODATA or 0 DEM cell)
#define FX_F_NODATA 0x08     // zb == NODATA_VALUE: add_meteo skips the cell (common.cpp:214)

// Device error codes (fx_ctl::error).
#define FX_DEVERR_WAIT_TIMEOUT 1

// What the ADE sweep of one step needs besides the grids: written by
// k_finalize when the step starts, read by the sweep of the same step, which
// may run several steps later (the hydrodynamics run ahead, see fx_ade.cu).
struct fx_steprec {
  double dtfl;        // dt of the step
  double meteoi;      // uniform melt depth of the step
  double meteo_rate;  // forcing rate of the step's row [mm/day]
  double mconc;       // forcing concentration of the step's row
  long long step;     // absolute step number (1 = first step)
  long long batch;    // value of fx_ctl::batch when the step ran
  int live;           // the step ran
  int active;         // hpall != 0: the hydrodynamic update and the sweep ran
  int it;             // solver iteration count after the step
  int pad_;
  double inflowi;     // point-inflow depth added this step (common.cpp:309)
  double iconc;       // its concentration
  double inflow_hm;   // depth of the inflow cell after the melt, before the inflow
                      // (written by the hydrodynamic kernel; the ADE's dilution)
};

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
  long long batch;       // counts launch batches; the ADE sweep takes this batch's steps
  // water budget since the last reset, FP64 [m^3]: water added by the
  // forcing (melt, and the point inflow with its cell's fill to the bed),
  // and water that left through the outflow faces (E face of irow = NROWS,
  // N face of icol = NCOLS)
  double budget_melt;
  double budget_out;
  double inflowi;     // point-inflow depth of the current step
  double iconc;       // and its concentration
  fx_steprec rec[FX_MAX_SLOTS];  // per-slot record of the last steps
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
  int dxy_pow2;       // 1 when dxy is a power of two (then x/dxy == x*inv_dxy exactly)
  double inv_dxy;     // 1/dxy, exact when dxy_pow2
  double inv_area;    // 1/arbase, exact when dxy_pow2
  int volrat_mode;    // 0: edge flux = weir formula, 1: edge flux = 0
  int ade;            // ADE module on
  int store_all_fluxes;  // 1 when forcing can remove water (see k_hydro)
  int tile_rows;         // hydrodynamic tile: 32 x tile_rows threads (4, 8 or 16)
  double dcoef[FX_MAX_CHEM];
  // state. h, h0, fe1, fn1 and flags hold `nslot` planes each: the state
  // after step n lives in plane n % nslot, so the ADE sweep of a step can run
  // after the hydrodynamics of the following steps (fx_ade.cu). z, qx, qy
  // (eta, eta_lo, qx_f, qy_f) hold two planes: the state after step n is in
  // plane n & 1 (fx_pp).
  int nslot;
  int wintra;         // WINTRA soil release after each step's ADE sweep (needs ade)
  double *z, *zb, *qx, *qy, *twet;
  // FP64 per-step fields of a context: one 48-byte record per cell and slot
  // plane, {h0, h, hp (the depth before the step's melt, max(z - zb, 0),
  // common.cpp:216), fe_1, fn_1, flag byte (as the double's bits)}, read by
  // the ADE sweep as three 16-byte copies (fx_rec64). The hydrodynamic step
  // writes the record of each interior cell; the ghost ring holds what was
  // uploaded.
  double* rec64;
  // The same fields as separate arrays: set (and rec64 left null) only by
  // fx_adesolver_noalloc, whose caller owns them.
  double *h, *h0, *fe1, *fn1;
  double *fe2, *fe3, *fn2, *fn3;
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
  int has_inflow;     // INFLOW_FILE: a point source at (inflow_irow, inflow_icol)
  // point-inflow table (float, as GlobVar::inflow; rows from 0) and cell
  const float* inflow_t;
  const float* inflow_r;
  const float* inflow_c;
  int inflow_irow, inflow_icol;
  long long inflow_gi;  // fx_ix of the cell, -1 without inflow
  fx_ctl* ctl;
  // Single-precision state (prec32 = 1, fx_hydro.cu hydro_tile32): the depth
  // above the bed eta = z - zb is stored, and the bed enters only through
  // its differences to the east and north neighbours (sx = zb(E) - zb(P),
  // sy = zb(N) - zb(P), exact in FP64 from the FP64 bed), so water-surface
  // differences are sx + (eta_E - eta_P) and thin films keep their digits. The depth is held compensated,
  // as the pair (eta, eta_lo) with eta + eta_lo exact and |eta_lo| at most
  // half an ulp of eta: flux arithmetic reads eta alone, updates add to the
  // pair without rounding loss, and the wet/dry threshold tests compare
  // eta + eta_lo in FP64. zb stays FP64 for output.
  int prec32;
  int ade_hold;  // failure-detection test: the ADE sweep's dependency waits are never satisfied
  float *eta, *eta_lo, *qx_f, *qy_f, *twet_f;
  float *fe2_f, *fe3_f, *fn2_f, *fn3_f;
  float* conc_f;                              // nchem planes
  // FP32 state: the per-step fields (h, h0, the pre-melt depth hp, fe_1,
  // fn_1) as one 32-byte record per cell and slot plane, {h0, h, hp, the
  // step's melt depth} then {fe_1, fn_1, flag byte (as the float's bits), 0}: the
  // ADE sweep fetches a cell's step inputs as one sector instead of one
  // sector per field (fx_ade.cu). The hydrodynamic step writes the record of
  // each interior cell; the ghost ring holds what was uploaded. Cell gi of
  // slot plane offset o is rec32[2 * (o + gi)], rec32[2 * (o + gi) + 1]
  // (fx_rec). The flag byte is kept in the flags planes as well.
  float4* rec32;
  const float* manning_f;
  const float* melt_mult_f;
  // ADE sweep scratch
  double* ade_bnd;                 // per slot, solute, strip: (ncols+2) x 3
  unsigned long long* ade_prog;    // per slot, solute, strip: step<<32 | warp steps done
  long long plane;                 // elements per field = ld * (nc + 2)
  // WINTRA (WINTRAsolver_calc.cpp:26-58): the soil mass, one copy per solute
  // in the state's precision. The reference releases into each solute in
  // turn from one soil grid; each solute's sweep replays that whole
  // sequence on its own copy, so the copies stay identical and no solute's
  // sweep waits on another's.
  double soil_rate;   // SOIL_RELEASE_RATE [1/hour]
  double* soil;       // nchem planes (FP64 state)
  float* soil_f;      // nchem planes (FP32 state)
};

// Work tables of a batch of domains (one domain is a batch of one).
// A hydrodynamic tile: block (bx, by) of domain dom.
struct fx_tile {
  int dom, bx, by, pad;
};
// An ADE unit: strip s of solute k at the jj-th step of the batch, domain dom.
struct fx_unit {
  int dom, jj, k, s;
};

// x / dxy and x / dxy^2. When dxy is a power of two the quotient is an
// exact scaling, so multiplying by the exact reciprocal gives the same bits as
// the division and saves a multi-instruction FP64 divide.
__host__ __device__ inline double fx_div_dxy(const fx_dev& d, double x) {
  return d.dxy_pow2 ? x * d.inv_dxy : x / d.dxy;
}
__host__ __device__ inline double fx_div_area(const fx_dev& d, double x) {
  return d.dxy_pow2 ? x * d.inv_area : x / d.arbase;
}

inline void fx_set_cell_size(fx_dev& d, int dxy) {
  d.dxy_u = (unsigned)dxy;
  d.dxy = (double)dxy;
  d.arbase = (double)((unsigned long)dxy * (unsigned long)dxy);
  d.dxy_pow2 = dxy > 0 && (dxy & (dxy - 1)) == 0 && dxy <= (1 << 20);
  d.inv_dxy = 1.0 / d.dxy;
  d.inv_area = 1.0 / d.arbase;
}

__host__ __device__ inline long long fx_ix(const fx_dev& d, int irow, int icol) {
  return (long long)icol * d.ld + irow + FX_ROFF;
}

// Offset of the slot plane that holds the state after step n.
__host__ __device__ inline long long fx_slot(const fx_dev& d, long long step) {
  return (step % d.nslot) * d.plane;
}

// Compensated FP32 depth: (hi, lo) += x with no rounding loss (Knuth's
// two-sum, exact in round-to-nearest without contraction), renormalised so
// that |lo| <= ulp(hi) / 2.
__host__ __device__ inline void fx_dd_add(float& hi, float& lo, float x) {
  const float s = hi + x;
  const float bb = s - hi;
  const float err = (hi - (s - bb)) + (x - bb);
  const float t = lo + err;
  hi = s + t;
  lo = t - (hi - s);
}
__host__ __device__ inline double fx_dd_val(float hi, float lo) { return (double)hi + (double)lo; }

// Components of the FP32 state's per-step record (fx_dev::rec32).
enum { FX_R_H0 = 0, FX_R_H = 1, FX_R_HP = 2, FX_R_MI = 3, FX_R_FE1 = 4, FX_R_FN1 = 5, FX_R_FL = 6 };
// The record of the cell at slot-plane element o (slot offset + fx_ix).
__host__ __device__ inline float* fx_rec(const fx_dev& d, long long o) {
  return reinterpret_cast<float*>(d.rec32 + 2 * o);
}
// Components of the FP64 per-step record (fx_dev::rec64), 6 doubles a cell.
enum { FX_R64_H0 = 0, FX_R64_H = 1, FX_R64_HP = 2, FX_R64_FE1 = 3, FX_R64_FN1 = 4, FX_R64_FL = 5, FX_R64_N = 6 };
__host__ __device__ inline double* fx_rec64(const fx_dev& d, long long o) { return d.rec64 + FX_R64_N * o; }

// Offset of the plane of z (eta), qx, qy that holds the state after step n:
// these fields have two planes, so a step reads one while it writes the
// other (a tile reads its neighbours' cells as they were before the step).
__host__ __device__ inline long long fx_pp(const fx_dev& d, long long step) {
  return (step & 1) * d.plane;
}

// Tensor maps of the TMA-staged hydrodynamic kernel (fx_hydro.cu
// k_hydro_tma): the stencil fields as 3-D tensors (irow with the column
// padding, icol, plane). Built on the host (fx_capi.cu fx_build_tmaps).
#define FX_TM_Z 0   // z (FP64) or eta (FP32), two planes
#define FX_TM_LO 1  // eta_lo (FP32), two planes
#define FX_TM_ZB 2  // zb, one plane
#define FX_TM_QX 3  // qx, two planes
#define FX_TM_QY 4  // qy, two planes
#define FX_TM_MM 5  // melt multiplier, one plane (when set)
#define FX_TM_FL 6  // flags, nslot planes
#define FX_TM_COUNT 7
struct alignas(64) fx_tmap {
  unsigned long long opaque[16];  // a CUtensorMap
};
struct fx_tmaps {
  fx_tmap m[FX_TM_COUNT];
};

