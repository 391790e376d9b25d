// FP64 advection-dispersion (ADE) step of FLUXOS-OVERLAND for sm_100a.
//
// ADEsolver_calc.cpp:27-291 re-scales every concentration to the new depth
// (:47-73) and then sweeps the grid once in Gauss-Seidel order (:93-290):
// cell (ix, iy) uses the already-updated concentration and limited fluxes of
// (ix-1, iy) and (ix, iy-1). Only a wavefront reproduces that order exactly.
//
// Mapping. A warp owns a strip of 30 rows; lane t (< 30) owns row
// ix0 + t and marches along iy with a skew of one column per lane, so at warp
// step tau lane t updates (ix0 + t, tau - t + 1) and every lane's west
// neighbour was updated by lane t-1 one step earlier:
//   * the west carries (updated c, limited flux pfe, re-scaled c, dry flag)
//     move lane t-1 -> t with one shuffle per step;
//   * the south carries (updated c, limited flux qfn) stay in registers;
//   * east / east-east / north / north-north inputs are prefetched by the
//     owning lane and shuffled down; lanes 30 and 31 only prefetch the first
//     two rows of the next strip. Prefetches are cp.async copies into a
//     per-lane shared-memory ring, so no register waits on a load.
// The re-scale of :47-73 is pointwise, so it is applied to each record as it
// is loaded; the bounds of :51-62 come from the pre-sweep value of the east
// and north cells and the re-scaled value of the west and south cells.
//
// Steps in flight. The hydrodynamics of a batch of consecutive steps run
// first (fx_hydro.cu writes each step's depth, fluxes and flags to its own
// slot plane), then one launch sweeps all of them: step j+1 of a strip
// follows step j a few diagonals behind, because its inputs are step j's
// outputs on the same and the next strip. The solute dilution of add_meteo
// (common.cpp:226-234), the only other writer of the concentration, is
// applied here, to each record as it is loaded, with the depths before and
// after the step's melt that the hydrodynamic kernel stored. A single launch therefore holds
// steps x solutes x strips independent chains and pays the wavefront's
// start-up once per batch instead of once per step.
//
// Strips of one step hand over through a small boundary buffer (per column:
// updated c, pfe, re-scaled c of the strip's last row); every dependency is a
// release/acquire progress counter tagged with the step number. Every wait
// is bounded and sets fx_ctl::error when it gives up.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "fx_common.cuh"

namespace fxade {

constexpr int ROWS = 30;      // rows per strip (lanes 0..29 compute)
constexpr int WARPS = 4;      // warps per block
constexpr int CHUNK = 4;      // steps between progress checks and publications (the lag between
                              // strips is 2 * CHUNK + ROWS - 1 warp steps)
constexpr int RING = 4;       // per-lane prefetch slots (a power of two); a deeper ring takes shared
                              // memory from L1, which the lanes' skewed reads depend on (measured:
                              // 8 slots made the FP64 sweep 2.5x slower)
constexpr int DIST = 2;       // prefetch distance in columns (< RING)
constexpr long long SPIN_LIMIT = 1LL << 20;  // polls (well under a second) before giving up
constexpr long long HOLD_SPIN_LIMIT = 1LL << 12;  // the same with fx_dev.ade_hold (a test of the timeout path)

// Per-lane ring of prefetched cells, filled by cp.async (asynchronous
// global -> shared copies).
// T is the state's precision (double for the reference path, float for the
// single-precision state).
template <class T>
struct Ring;
// The FP64 ring: the concentration group, the cell's six per-step values
// {h0, h, hp, fe_1, fn_1, flag bits} and the melt multiplier. A context's
// record (fx_dev::rec64) lands in r as three 16-byte copies; the separate
// arrays of fx_adesolver_noalloc land in the same places one by one (the
// flag as the 4-byte word holding it, in r[5]'s low half).
template <>
struct Ring<double> {
  static constexpr int CV = 2;
  // the 16-byte aligned group of concentrations holding this lane's cell: it
  // is written during the launch by other warps, so it is copied with
  // cp.async.cg (L2 only; L1 is not coherent across SMs), which moves 16 bytes
  double c[RING][32][CV];
  double r[RING][32][FX_R64_N];
  double mm[RING][32];  // melt-rate multiplier (1 without a melt field)
};

// The FP32 state's ring: the concentration group and the cell's per-step
// record (fx_dev::rec32), two 16-byte copies from one 32-byte sector.
template <>
struct Ring<float> {
  static constexpr int CV = 4;
  float c[RING][32][CV];
  float4 a[RING][32];  // h0, h, hp, the step's melt depth
  float4 b[RING][32];  // fe_1, fn_1, flag byte (as the float's bits), 0
};

template <class T>
struct Rec {
  T c;   // concentration before the sweep (after dilution, before re-scale)
  T b;   // re-scaled concentration (ADEsolver_calc.cpp:64-72)
  T h;   // depth after the hydrodynamic update
  T qx;  // fe_1 of the cell
  T qy;  // fn_1 of the cell
  int ld;     // ldry (1 = dry); ghost cells read 0
};

// The state fields of the sweep in precision T.
template <class T>
struct Fields;
template <>
struct Fields<double> {
  static __device__ __forceinline__ const double* h(const fx_dev& d) { return d.h; }
  static __device__ __forceinline__ const double* h0(const fx_dev& d) { return d.h0; }
  static __device__ __forceinline__ const double* fe1(const fx_dev& d) { return d.fe1; }
  static __device__ __forceinline__ const double* fn1(const fx_dev& d) { return d.fn1; }
  static __device__ __forceinline__ const double* mm(const fx_dev& d) { return d.melt_mult; }
  static __device__ __forceinline__ double* conc(const fx_dev& d) { return d.conc; }
  static __device__ __forceinline__ double* soil(const fx_dev& d) { return d.soil; }
};
template <>
struct Fields<float> {
  static __device__ __forceinline__ const float* mm(const fx_dev& d) { return d.melt_mult_f; }
  static __device__ __forceinline__ float* conc(const fx_dev& d) { return d.conc_f; }
  static __device__ __forceinline__ float* soil(const fx_dev& d) { return d.soil_f; }
};

// Division and square root: IEEE-rounded in FP64 (bit parity with the
// reference); in FP32 the approximate hardware reciprocal and square root
// (PTX rcp.approx / sqrt.approx) refined by one Newton step with fused
// multiply-adds, without the IEEE code paths.
__device__ __forceinline__ double tdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float tdiv(float a, float b) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(b));
  const float q = a * r;
  return fmaf(fmaf(-b, q, a), r, q);
}
__device__ __forceinline__ double tsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ float tsqrt(float a) {
  float s, r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(s) : "f"(a));
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(s));
  const float t = fmaf(fmaf(-s, s, a), 0.5f * r, s);
  return a > 0.0f ? t : s;
}

template <class T>
__device__ __forceinline__ T div_dxy(const fx_dev& d, T x) {
  return d.dxy_pow2 ? x * (T)d.inv_dxy : tdiv(x, (T)d.dxy);
}
template <class T>
__device__ __forceinline__ T div_area(const fx_dev& d, T x) {
  return d.dxy_pow2 ? x * (T)d.inv_area : tdiv(x, (T)d.arbase);
}

// The step a unit works on.
struct StepIn {
  long long cur;        // slot plane offset of the step
  double meteo_rate, meteoi, mconc, dt;
  long long inflow_gi;  // the point-inflow cell (-1: none)
  double inflowi, iconc, inflow_hm;
  bool sweep;           // the sweep runs (hpall != 0 and it > 1)
  bool dilute;          // add_meteo's dilution runs
  bool wintra;          // the soil release follows the sweep (hpall != 0)
};

__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Issue the copies of cell (ix, iy) into ring slot `slot` of this lane. The
// shared and global addresses are formed once per cell (a 32-bit shared
// address of the lane's entry, one offset into the slot plane); a cell
// outside the grid copies 0 source bytes, which zero-fills its entries.
__device__ __forceinline__ void cp_async_sz(unsigned dst, const void* gmem, int n, int bytes) {
  if (bytes == 16) asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(gmem), "r"(n));
  else if (bytes == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(gmem), "r"(n));
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(gmem), "r"(n));
}
template <class T>
__device__ __forceinline__ void prefetch(const fx_dev& d, const StepIn& S, const T* A, Ring<T>& R, int lane,
                                         int ix, int iy) {
  using F = Fields<T>;
  constexpr int B = sizeof(T);
  const int slot = iy & (RING - 1);
  const bool inr = ix >= 0 && ix <= d.nr + 1 && iy >= 0 && iy <= d.nc + 1;
  const long long gi = inr ? fx_ix(d, ix, iy) : 0;
  const long long o = S.cur + gi;
  // the concentration is written during the launch by other warps: through L2 only
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                   (unsigned)__cvta_generic_to_shared(&R.c[slot][lane][0])),
               "l"(A + (gi & ~(long long)(Ring<T>::CV - 1))), "r"(inr ? 16 : 0));
  if constexpr (B == 4) {
    const float4* rec = d.rec32 + 2 * o;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(
                     (unsigned)__cvta_generic_to_shared(&R.a[slot][lane])),
                 "l"(rec), "r"(inr ? 16 : 0));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(
                     (unsigned)__cvta_generic_to_shared(&R.b[slot][lane])),
                 "l"(rec + 1), "r"(inr ? 16 : 0));
  } else {
    double* re = &R.r[slot][lane][0];
    const unsigned e = (unsigned)__cvta_generic_to_shared(re);
    if (d.rec64) {  // a context: the cell's record, 48 bytes
      const double* rec = fx_rec64(d, o);
      for (int q = 0; q < 3; ++q) cp_async_sz(e + 16 * q, rec + 2 * q, inr ? 16 : 0, 16);
    } else {  // fx_adesolver_noalloc: the caller's arrays (no melt, no slots)
      const int nb = inr ? 8 : 0;
      cp_async_sz(e + 8 * FX_R64_H0, F::h0(d) + o, nb, 8);
      cp_async_sz(e + 8 * FX_R64_H, F::h(d) + o, nb, 8);
      cp_async_sz(e + 8 * FX_R64_FE1, F::fe1(d) + o, nb, 8);
      cp_async_sz(e + 8 * FX_R64_FN1, F::fn1(d) + o, nb, 8);
      // the 4-byte word holding the flag byte (planes are multiples of 32 bytes)
      cp_async_sz(e + 8 * FX_R64_FL, d.flags + (o & ~3LL), inr ? 4 : 0, 4);
    }
    const bool mm_ok = S.dilute && F::mm(d) != nullptr;
    cp_async_sz((unsigned)__cvta_generic_to_shared(&R.mm[slot][lane]),
                mm_ok ? (const void*)(F::mm(d) + gi) : (const void*)d.flags, mm_ok && inr ? 8 : 0, 8);
  }
}

// The same record with the tests as branches (the FP64 state: lanes skip the
// IEEE divisions their cell does not need, which in FP64 costs more than the
// divergence).
template <class T>
__device__ __forceinline__ Rec<T> make_rec_br(const fx_dev& d, const StepIn& S, const Ring<T>& R, int lane, int ix,
                                           int iy) {
  static_assert(sizeof(T) == 8, "the branch form reads the FP64 ring");
  Rec<T> r;
  r.c = T(0);
  r.b = T(0);
  r.h = T(0);
  r.qx = T(0);
  r.qy = T(0);
  r.ld = 0;
  if (ix < 0 || ix > d.nr + 1 || iy < 0 || iy > d.nc + 1) return r;
  const int slot = iy & (RING - 1);
  const double* v = R.r[slot][lane];
  r.h = v[FX_R64_H];
  if (ix >= 1 && ix <= d.nr && iy >= 1 && iy <= d.nc) {
    const long long gi = fx_ix(d, ix, iy);
    // a record holds the flag byte itself, a separate flags array the word holding it
    const unsigned word = (unsigned)__double_as_longlong(v[FX_R64_FL]);
    const unsigned fl = (d.rec64 ? word : word >> (8 * (unsigned)(gi & 3))) & 0xffu;
    r.ld = fl & FX_F_LDRY;
    const int ldp = (fl & FX_F_LDRY_PREV) ? 1 : 0;
    T c = R.c[slot][lane][gi & (Ring<T>::CV - 1)];
    const T h0 = v[FX_R64_H0];
    // the inflow cell holds h0 only after its inflow; the melt's dilution
    // divides by the depth after the melt (common.cpp:226-234, 313-325)
    const bool inflow_cell = gi == S.inflow_gi;
    const T hm = inflow_cell ? (T)S.inflow_hm : h0;
    if (S.dilute && !(fl & FX_F_NODATA)) {
      const T hp = v[FX_R64_HP];
      if (hp != T(0)) {
        // the melt depth the hydrodynamic step added (melt_depth in fx_hydro.cu)
        const T mi = Fields<T>::mm(d)
                         ? (T)((double)S.meteo_rate * R.mm[slot][lane] / (1000. * 3600. * 24.) * S.dt)
                         : (T)S.meteoi;
        c = tdiv(c * hp + (mi * (T)S.mconc), hm);
      }
    }
    if (inflow_cell && hm != T(0)) c = tdiv(c * hm + (T)(S.inflowi * S.iconc), h0);
    r.c = c;
    if (!S.sweep) r.b = c;
    else if (r.ld == 0 && ldp == 0) r.b = tdiv(c * h0, r.h);
    else if (r.ld == 1) r.b = T(0);
    else r.b = c;
    r.qx = v[FX_R64_FE1];
    r.qy = v[FX_R64_FN1];
  }
  return r;
}

// The record of cell (ix, iy) from its ring slot: add_meteo's dilution
// (common.cpp:214-234) when the step has one, then the re-scale of
// ADEsolver_calc.cpp:64-72 when the step sweeps. Ghost cells carry only their
// depth (their concentration is 0 and never changes). The slot is always a
// ring entry, so it is read for every (ix, iy) and the values are selected:
// per-cell tests become selects and the block has no divergent branch (the
// step's dilution and point inflow are the same for the whole warp). Used by
// the FP32 state, whose divisions are a few fused operations; its ring holds
// the cell's per-step record (fx_dev::rec32).
template <class T>
__device__ __forceinline__ Rec<T> make_rec(const fx_dev& d, const StepIn& S, const Ring<T>& R, int lane, int ix,
                                           int iy) {
  static_assert(sizeof(T) == 4, "the select form reads the FP32 ring");
  const bool inr = ix >= 0 && ix <= d.nr + 1 && iy >= 0 && iy <= d.nc + 1;
  const bool interior = ix >= 1 && ix <= d.nr && iy >= 1 && iy <= d.nc;
  const int slot = iy & (RING - 1);
  const long long gi = fx_ix(d, ix, iy);  // an index into the ring's groups only, outside the grid
  const float4 ra = R.a[slot][lane], rb = R.b[slot][lane];
  const unsigned fl = __float_as_uint(rb.z);
  const int ld = fl & FX_F_LDRY;
  const bool ldp = (fl & FX_F_LDRY_PREV) != 0;
  const T h = ra.y;
  const T h0 = ra.x;
  T c = R.c[slot][lane][gi & (Ring<T>::CV - 1)];
  // the inflow cell holds h0 only after its inflow; the melt's dilution
  // divides by the depth after the melt (common.cpp:226-234, 313-325)
  const bool inflow_cell = S.inflow_gi >= 0 && interior && gi == S.inflow_gi;
  const T hm = inflow_cell ? (T)S.inflow_hm : h0;
  if (S.dilute) {
    const T hp = ra.z;
    const T mi = ra.w;  // the melt depth the hydrodynamic step added (melt32 in fx_hydro.cu)
    const bool use = !(fl & FX_F_NODATA) && hp != T(0);  // then hm >= hp > 0
    const T cd = tdiv(c * hp + (mi * (T)S.mconc), use ? hm : T(1));
    c = use ? cd : c;
  }
  if (S.inflow_gi >= 0) {
    const bool use = inflow_cell && hm != T(0);
    const T ci = tdiv(c * hm + (T)(S.inflowi * S.iconc), use ? h0 : T(1));
    c = use ? ci : c;
  }
  T b = c;
  if (S.sweep) {
    const bool wet2 = ld == 0 && !ldp;  // wet before and after the step: h > hdry
    const T bw = tdiv(c * h0, wet2 ? h : T(1));
    b = wet2 ? bw : (ld == 1 ? T(0) : c);
  }
  Rec<T> r;
  r.h = inr ? h : T(0);
  r.c = interior ? c : T(0);
  r.b = interior ? b : T(0);
  r.qx = interior ? rb.x : T(0);
  r.qy = interior ? rb.y : T(0);
  r.ld = interior ? ld : 0;
  return r;
}

template <class V>
__device__ __forceinline__ V shfl_d(V v, int src) { return __shfl_sync(0xffffffffu, v, src); }
template <class V>
__device__ __forceinline__ V shdn(V v, int k) { return __shfl_down_sync(0xffffffffu, v, k); }
template <class V>
__device__ __forceinline__ V shup(V v, int k) { return __shfl_up_sync(0xffffffffu, v, k); }

__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// One cell of the sweep, ADEsolver_calc.cpp:126-288, for a wet cell.
// T = double is the reference's arithmetic; T = float the single-precision
// state's (same operations, same order).
template <class T>
__device__ __forceinline__ void ade_cell(const fx_dev& d, T D, T dt, bool last_row, bool last_col, T hp,
                                         T he, T hn, T qxl, T qyl, T fw, T fp, T fe, T fee, T fs, T fn,
                                         T fnn, T pfw, T qfs, int ldE, int ldW, int ldEE, int ldN, int ldS,
                                         int ldNN, T cmax, T cmin, T& con, T& pfe_out, T& qfn_out) {
  // The expressions of ADEsolver_calc.cpp:126-288 in the same order and
  // operand types; both sides of every test are evaluated and the result
  // selected, so the cell is one straight-line block (independent parts of
  // the E and N faces interleave). A quotient that is not selected divides by
  // 1 instead of a possibly zero denominator (an FP64 division by zero takes
  // the division's slow path); a selected one is unchanged.
  const T nt = 1;
  const T dx = (T)d.dxy, dy = (T)d.dxy;
  const T area = (T)d.arbase, areae = (T)d.arbase, arean = (T)d.arbase;
  const T ntp = nt;
  const bool wetE = ldE == 0, wetN = ldN == 0;
  // E face (:151-194)
  const T hnue_e = fmax(hp * nt * he * nt, T(.0001));
  const T hne = div_dxy<T>(d, tsqrt(hnue_e) * T(2)) * dy * D;  // sigc = 0.5: /sigc is *2 exactly
  const T pfde = wetE ? -hne * (fe - fp) : T(0);
  const T mid_e = T(.5) * fp + T(.5) * fe;
  const T up_e = ldW == 0 ? T(-.125) * fw + T(.75) * fp + T(.375) * fe : mid_e;
  const T dn_e = ldEE == 0 ? T(.375) * fp + T(.75) * fe - T(.125) * fee : mid_e;
  T fem = wetE ? (qxl > T(0) ? up_e : dn_e) : T(0);
  fem = fmax(T(0), fem);
  fem = last_row ? T(0) : fem;  // :176-178, ghost concentration c(NROWS+1, iy) = 0
  const T pfce = qxl * fem * dy;
  T pfe = pfce + pfde;
  const T cvolrate_e = tdiv(-(fe * he) * areae, dt);
  pfe = pfe < T(0) ? (wetE ? fmax(pfe, cvolrate_e) : T(0)) : pfe;
  // N face (:198-241)
  const T hnue_n = fmax(T(.0001), hp * ntp * hn * nt);
  const T hnn = div_dxy<T>(d, tsqrt(hnue_n) * T(2)) * dx * D;
  const T qfdn = wetN ? -hnn * (fn - fp) : T(0);
  const T mid_n = T(.5) * fp + T(.5) * fn;
  const T up_n = ldS == 0 ? T(-.125) * fs + T(.75) * fp + T(.375) * fn : mid_n;
  const T dn_n = ldNN == 0 ? T(.375) * fp + T(.75) * fn - T(.125) * fnn : mid_n;
  T fnm = wetN ? (qyl > T(0) ? up_n : dn_n) : T(0);
  fnm = fmax(T(0), fnm);
  fnm = last_col ? T(0) : fnm;  // :223-225, ghost concentration c(ix, NCOLS+1) = 0
  const T qfcn = qyl * fnm * dx;
  T qfn = qfcn + qfdn;
  const T cvolrate_n = tdiv(-(fn * hn) * arean, dt);
  qfn = qfn < T(0) ? (wetN ? fmax(qfn, cvolrate_n) : T(0)) : qfn;
  // outflow limiter (:243-278)
  const T cvolpot = (fp * hp) * area;
  const T cvolrat = tdiv(cvolpot, dt) + pfw + qfs;
  const T sum = pfe + qfn;
  const bool pos = cvolrat > T(0);
  const bool pp = pfe > T(0), qp = qfn > T(0);
  // cvolrat > 0
  const bool both = pp && qp;
  const bool split = both && sum > cvolrat;
  const T cf = tdiv(qfn, split ? sum : T(1));
  T pfe_a = split ? (T(1) - cf) * cvolrat : pfe;
  T qfn_a = split ? cf * cvolrat : qfn;
  pfe_a = (!both && pp) ? fmin(pfe, (cvolrat - qfn)) : pfe_a;
  qfn_a = (!both && !pp && qp) ? fmin(qfn, (cvolrat - pfe)) : qfn_a;
  // cvolrat <= 0
  const bool c1 = pfe >= T(0) && qfn < T(0);
  const bool c2 = !c1 && pfe < T(0) && qfn >= T(0);
  const bool c3 = !c1 && !c2 && pfe >= T(0) && qfn >= T(0);
  const T cb1 = cvolrat - qfn, cb2 = cvolrat - pfe;
  T pfe_b = c1 ? (cb1 > T(0) ? fmin(pfe, cb1) : T(0)) : pfe;
  T qfn_b = c2 ? (cb2 > T(0) ? fmin(qfn, cb2) : T(0)) : qfn;
  pfe_b = c3 ? T(0) : pfe_b;
  qfn_b = c3 ? T(0) : qfn_b;
  pfe = pos ? pfe_a : pfe_b;
  qfn = pos ? qfn_a : qfn_b;
  const T dc = div_area<T>(d, (pfw - pfe + qfs - qfn) * dt);  // :281-286
  T cn = fp + tdiv(dc, hp != T(0) ? hp : T(1));  // hp is 0 only in a dry cell, whose result is not kept
  cn = fmin(cmax, cn);
  cn = fmax(cmin, cn);
  con = cn;
  pfe_out = pfe;
  qfn_out = qfn;
}

// The same cell with the tests as branches (the FP64 state, for the reason
// given at make_rec_br).
template <class T>
__device__ __forceinline__ void ade_cell_br(const fx_dev& d, T D, T dt, bool last_row, bool last_col, T hp,
                                         T he, T hn, T qxl, T qyl, T fw, T fp, T fe, T fee, T fs, T fn,
                                         T fnn, T pfw, T qfs, int ldE, int ldW, int ldEE, int ldN, int ldS,
                                         int ldNN, T cmax, T cmin, T& con, T& pfe_out, T& qfn_out) {
  const T nt = 1;
  const T dx = (T)d.dxy, dy = (T)d.dxy;
  const T area = (T)d.arbase, areae = (T)d.arbase, arean = (T)d.arbase;
  const T ntp = nt;
  T fem, pfde, hnue, hne;
  if (ldE == 0) {  // :151-172
    hnue = fmax(hp * nt * he * nt, T(.0001));
    hne = div_dxy<T>(d, tsqrt(hnue) * T(2)) * dy * D;  // sigc = 0.5: /sigc is *2 exactly
    pfde = -hne * (fe - fp);
    if (qxl > T(0)) {
      if (ldW == 0) fem = T(-.125) * fw + T(.75) * fp + T(.375) * fe;
      else fem = T(.5) * fp + T(.5) * fe;
    } else {
      if (ldEE == 0) fem = T(.375) * fp + T(.75) * fe - T(.125) * fee;
      else fem = T(.5) * fp + T(.5) * fe;
    }
  } else {
    fem = T(0);
    pfde = T(0);
  }
  fem = fmax(T(0), fem);
  if (last_row) fem = T(0);  // :176-178, ghost concentration c(NROWS+1, iy) = 0
  const T pfce = qxl * fem * dy;
  T pfe = pfce + pfde;
  if (pfe < T(0)) {  // :187-194
    if (ldE == 0) {
      const T cvolrate = tdiv(-(fe * he) * areae, dt);
      pfe = fmax(pfe, cvolrate);
    } else {
      pfe = T(0);
    }
  }
  T fnm, qfdn, hnn;
  if (ldN == 0) {  // :198-218
    hnue = fmax(T(.0001), hp * ntp * hn * nt);
    hnn = div_dxy<T>(d, tsqrt(hnue) * T(2)) * dx * D;
    qfdn = -hnn * (fn - fp);
    if (qyl > T(0)) {
      if (ldS == 0) fnm = T(-.125) * fs + T(.75) * fp + T(.375) * fn;
      else fnm = T(.5) * fp + T(.5) * fn;
    } else {
      if (ldNN == 0) fnm = T(.375) * fp + T(.75) * fn - T(.125) * fnn;
      else fnm = T(.5) * fp + T(.5) * fn;
    }
  } else {
    fnm = T(0);
    qfdn = T(0);
  }
  fnm = fmax(T(0), fnm);
  if (last_col) fnm = T(0);  // :223-225, ghost concentration c(ix, NCOLS+1) = 0
  const T qfcn = qyl * fnm * dx;
  T qfn = qfcn + qfdn;
  if (qfn < T(0)) {  // :234-241
    if (ldN == 0) {
      const T cvolrate = tdiv(-(fn * hn) * arean, dt);
      qfn = fmax(qfn, cvolrate);
    } else {
      qfn = T(0);
    }
  }
  const T cvolpot = (fp * hp) * area;  // :243-278
  const T cvolrat = tdiv(cvolpot, dt) + pfw + qfs;
  if (cvolrat > T(0)) {
    if (pfe > T(0) && qfn > T(0)) {
      if (pfe + qfn > cvolrat) {
        const T cf = tdiv(qfn, pfe + qfn);
        pfe = (T(1) - cf) * cvolrat;
        qfn = cf * cvolrat;
      }
    } else if (pfe > T(0)) {
      pfe = fmin(pfe, (cvolrat - qfn));
    } else if (qfn > T(0)) {
      qfn = fmin(qfn, (cvolrat - pfe));
    }
  } else {
    if (pfe >= T(0) && qfn < T(0)) {
      const T cbilan = cvolrat - qfn;
      if (cbilan > T(0)) pfe = fmin(pfe, cbilan);
      else pfe = T(0);
    } else if (pfe < T(0) && qfn >= T(0)) {
      const T cbilan = cvolrat - pfe;
      if (cbilan > T(0)) qfn = fmin(qfn, cbilan);
      else qfn = T(0);
    } else if (pfe >= T(0) && qfn >= T(0)) {
      pfe = T(0);
      qfn = T(0);
    }
  }
  const T dc = div_area<T>(d, (pfw - pfe + qfs - qfn) * dt);  // :281-286
  T cn = fp + tdiv(dc, hp);
  cn = fmin(cmax, cn);
  cn = fmax(cmin, cn);
  con = cn;
  pfe_out = pfe;
  qfn_out = qfn;
}

// wintrasolver_calc (WINTRAsolver_calc.cpp:39-57) at one cell after the
// step's sweep, for solute k with concentration c: a wet cell whose bed is
// not NODATA_VALUE releases soil * rate / 3600 * dt of its soil mass into
// the concentration, c + deltam / (h * arbase). The reference calls it once
// per solute on one soil grid (main.cpp:400-404); this solute's copy of the
// soil mass replays every solute's release and keeps its own term. The soil
// mass is read through L2 (other SMs wrote it in earlier steps).
template <class T>
__device__ __forceinline__ T soil_release(const fx_dev& d, const StepIn& S, int k, long long gi, T h, T c) {
  if (!((double)h > d.hdry) || (d.flags[S.cur + gi] & FX_F_NODATA)) return c;
  T* p = Fields<T>::soil(d) + (long long)k * d.plane + gi;
  T soil = __ldcg(p);
  T mine = T(0);
  for (int j = 0; j < d.nchem; ++j) {
    const T dm = tdiv(soil * (T)d.soil_rate, T(3600)) * (T)S.dt;
    soil = soil - dm;
    if (j == k) mine = dm;
  }
  *p = soil;
  return c + tdiv(mine, h * (T)d.arbase);
}

// The three progress counters a unit depends on: the west strip of its step
// and, on the previous step of the batch, its own strip and the next one.
// The last values seen are kept, so a requirement the producer has already
// passed costs no memory access; otherwise all three are reloaded together
// (one round trip). A null counter is no dependency.
struct Deps {
  const unsigned long long *w, *p0, *p1;
  unsigned long long tag_w, tag_p;
  unsigned long long seen_w, seen_p0, seen_p1;
};

__device__ __forceinline__ bool dep_ok(const unsigned long long* p, unsigned long long seen,
                                       unsigned long long tag, int need) {
  return !p || seen >= ((tag << 32) | (unsigned)need);
}

// Wait until the counters reach the given warp-step counts; false if the wait
// gave up (the error flag is then set).
// With d.ade_hold set (fx_set_option "fail_ade_waits") a unit that has a
// dependency never sees it met, so its wait runs out after HOLD_SPIN_LIMIT
// polls: the timeout path, exercised without a fault.
__device__ __forceinline__ bool wait_deps(const fx_dev& d, Deps& D, int need_w, int need_p0, int need_p1) {
  long long it = 0;
  const bool hold = d.ade_hold != 0;
  const long long limit = hold ? HOLD_SPIN_LIMIT : SPIN_LIMIT;
  for (;;) {
    const bool ok = dep_ok(D.w, D.seen_w, D.tag_w, need_w) && dep_ok(D.p0, D.seen_p0, D.tag_p, need_p0) &&
                    dep_ok(D.p1, D.seen_p1, D.tag_p, need_p1) && (!hold || (!D.w && !D.p0 && !D.p1));
    if (__all_sync(0xffffffffu, ok)) {
      // the counts that sufficed were read by relaxed loads: one fence orders
      // this warp's later reads of the producers' data after them (with the
      // producers' release stores). Counts kept from an earlier wait were
      // followed by this fence then.
      if (it > 0) asm volatile("fence.acq_rel.gpu;" ::: "memory");
      return true;
    }
    const bool stop = (++it > limit) || ((it & 63) == 0 && *(volatile int*)&d.ctl->error != 0);
    if (__any_sync(0xffffffffu, stop)) {
      if ((threadIdx.x & 31) == 0) atomicCAS(&d.ctl->error, 0, FX_DEVERR_WAIT_TIMEOUT);
      return false;
    }
    if (it > 1) __nanosleep(it < 8 ? 64 : (it < 64 ? 256 : 1024));
    // the three counters in one round trip (relaxed loads in flight together)
    D.seen_w = D.w ? ld_relaxed(D.w) : 0ull;
    D.seen_p0 = D.p0 ? ld_relaxed(D.p0) : 0ull;
    D.seen_p1 = D.p1 ? ld_relaxed(D.p1) : 0ull;
  }
}

// Sweep of one unit: strip s of solute k at the jj-th live step of the batch.
// Returns false when a wait gave up.
template <class T>
__device__ __forceinline__ bool ade_unit(const fx_dev& d, Ring<T>& R, int jj, int k, int s, int lane) {
  {
    const fx_ctl& cc = *d.ctl;
    // this batch's live steps are consecutive: the jj-th is minstep + jj
    int m = 0;
    long long minstep = 0;
    for (int q = 0; q < d.nslot; ++q) {
      const fx_steprec& r = cc.rec[q];
      if (r.live && r.batch == cc.batch) {
        minstep = (m == 0 || r.step < minstep) ? r.step : minstep;
        ++m;
      }
    }
    if (jj >= m) return true;
    const long long step = minstep + jj;
    const int slot = (int)(step % d.nslot);
    const int nstrips = (d.nr + ROWS - 1) / ROWS;
    const int TW = d.nc + ROWS - 1;  // warp steps per strip
    const long long bnd_stride = (long long)(d.nc + 2) * 3;
    auto unit_index = [&](int sl, int kk, int ss) { return ((long long)sl * d.nchem + kk) * nstrips + ss; };
    const fx_steprec& rec = cc.rec[slot];
    const unsigned long long tag = (unsigned long long)rec.step;
    StepIn S;
    S.cur = fx_slot(d, rec.step);
    S.meteo_rate = rec.meteo_rate;
    S.meteoi = rec.meteoi;
    S.mconc = rec.mconc;
    S.dt = rec.dtfl;
    S.sweep = rec.active && rec.it > 1;  // :45,74-77
    S.dilute = d.has_meteo != 0;
    S.wintra = d.wintra && rec.active;  // main.cpp:385-405
    S.inflow_gi = d.has_inflow ? d.inflow_gi : -1;
    S.inflowi = rec.inflowi;
    S.iconc = rec.iconc;
    S.inflow_hm = rec.inflow_hm;
    T* A = Fields<T>::conc(d) + k * d.plane;
    const T D = (T)d.dcoef[k];
    const int ix0 = 1 + s * ROWS;
    const int ix = ix0 + lane;
    const bool compute_lane = lane < ROWS && ix <= d.nr;
    // dependencies: the west strip of this step, this strip and the next
    // strip of the previous step of the batch (earlier batches are complete)
    const unsigned long long* prog_w = (s > 0) ? d.ade_prog + unit_index(slot, k, s - 1) : nullptr;
    const int pslot = (int)((step - 1) % d.nslot);
    const unsigned long long* prog_p0 = jj > 0 ? d.ade_prog + unit_index(pslot, k, s) : nullptr;
    const unsigned long long* prog_p1 =
        (jj > 0 && s + 1 < nstrips) ? d.ade_prog + unit_index(pslot, k, s + 1) : nullptr;
    unsigned long long* prog_me = d.ade_prog + unit_index(slot, k, s);
    const double* bnd_in = d.ade_bnd + unit_index(slot, k, s) * bnd_stride;
    double* bnd_out = (s + 1 < nstrips) ? d.ade_bnd + unit_index(slot, k, s + 1) * bnd_stride : nullptr;
    bool bail = false;
    Deps dep;
    dep.w = prog_w;
    dep.p0 = prog_p0;
    dep.p1 = prog_p1;
    dep.tag_w = tag;
    dep.tag_p = tag - 1;
    dep.seen_w = dep.seen_p0 = dep.seen_p1 = 0ull;
    // the previous step must have written every cell prefetched before the
    // next check, and the west strip of this step the boundary columns read
    // in the chunk. When lane 0 prefetches up to column col, lane t (< ROWS)
    // prefetches its row up to column col - t, which lane t of the previous
    // step's sweep of this strip, on the same skew, updates at warp step
    // col - 1: a count of col suffices. Lanes ROWS and ROWS + 1 prefetch the
    // next strip's rows 0 and 1 up to columns col - ROWS and col - ROWS - 1,
    // which that strip's lanes 0 and 1 update by warp step col - ROWS - 1.
    // (Each step's strip also reads and writes its own cells only after the
    // previous step did, at the same warp step of the skew, which these counts
    // cover.)
    auto need_p0 = [&](int col) { return min(col, TW); };
    auto need_p1 = [&](int col) { return max(0, min(col - ROWS, TW)); };
    if (!wait_deps(d, dep, min(CHUNK - 1 + ROWS, TW), need_p0(DIST + 3), need_p1(DIST + 3))) bail = true;

    // prime: the first three columns of this lane's row become records, then
    // columns iy0 + 3 .. iy0 + DIST + 2 go in flight (the ring holds only the
    // DIST + 1 columns in flight, so RING >= DIST + 1)
    static_assert(RING >= DIST + 1, "ring too shallow for the prefetch distance");
    const int iy0 = 1 - lane;
    if (!bail) {
      for (int j = 0; j < 3; ++j) {
        prefetch<T>(d, S, A, R, lane, ix, iy0 + j);
        cp_commit();
      }
    }
    cp_wait<0>();
    auto rec_at = [&](int col) {
      if constexpr (sizeof(T) == 4) return make_rec<T>(d, S, R, lane, ix, col);
      else return make_rec_br<T>(d, S, R, lane, ix, col);
    };
    Rec<T> cur = rec_at(iy0);
    Rec<T> n1 = rec_at(iy0 + 1);
    Rec<T> n2 = rec_at(iy0 + 2);
    if (!bail) {
      for (int j = 3; j < DIST + 3; ++j) {
        prefetch<T>(d, S, A, R, lane, ix, iy0 + j);
        cp_commit();
      }
    }
    // carries: outputs of this lane's previous cell (its south cell for the
    // next step, its west cell for lane + 1)
    T o_c = T(0), o_pfe = T(0), o_b = T(0), o_qfn = T(0);
    int o_ld = 0;
    // west-boundary values of the current and the next chunk (lane j holds
    // column chunk_start + 1 + j); strip 0's west neighbour is the ghost row 0:
    // c = 0, pfe = the ghost convective flux c(0,iy)*fe_1(0,iy)*dy = 0 (:106-116)
    T bw_c = T(0), bw_pfe = T(0), bw_b = T(0), bn_c = T(0), bn_pfe = T(0), bn_b = T(0);
    int bw_ld = 0, bn_ld = 0;
    if (!bail && prog_w) {
      const int iyb = 1 + lane;
      if (lane < CHUNK && iyb <= d.nc) {
        const double* p = bnd_in + (long long)iyb * 3;
        bn_c = (T)__ldcg(p);
        bn_pfe = (T)__ldcg(p + 1);
        bn_b = (T)__ldcg(p + 2);
        bn_ld = d.flags[S.cur + fx_ix(d, ix0 - 1, iyb)] & FX_F_LDRY;
      }
    }

    for (int tau = 0; tau < TW && !bail; ++tau) {
      if ((tau % CHUNK) == 0) {
        bw_c = bn_c;
        bw_pfe = bn_pfe;
        bw_b = bn_b;
        bw_ld = bn_ld;
        // columns lane 0 prefetches during this chunk, and the next chunk's
        // boundary (loaded now, used in CHUNK steps)
        const int col = tau + CHUNK + DIST + 3;
        if (!wait_deps(d, dep, min(tau + 2 * CHUNK - 1 + ROWS, TW), need_p0(col), need_p1(col))) {
          bail = true;
          break;
        }
        if (prog_w && tau + CHUNK < TW) {
          const int iyb = tau + CHUNK + 1 + lane;
          bn_c = bn_pfe = bn_b = T(0);
          bn_ld = 0;
          if (lane < CHUNK && iyb <= d.nc) {
            const double* p = bnd_in + (long long)iyb * 3;
            bn_c = (T)__ldcg(p);
            bn_pfe = (T)__ldcg(p + 1);
            bn_b = (T)__ldcg(p + 2);
            bn_ld = d.flags[S.cur + fx_ix(d, ix0 - 1, iyb)] & FX_F_LDRY;
          }
        }
      }
      const int iy = tau - lane + 1;
      // keep DIST columns in flight: column iy + DIST + 3 now; column iy + 3,
      // copied DIST steps ago, has landed after cp_wait and becomes the record
      // of the next step, made here so that its arithmetic and this step's
      // cell interleave
      prefetch<T>(d, S, A, R, lane, ix, iy + DIST + 3);
      cp_commit();
      cp_wait<DIST>();
      Rec<T> n3;
      if constexpr (sizeof(T) == 4) n3 = make_rec<T>(d, S, R, lane, ix, iy + 3);
      else n3 = make_rec_br<T>(d, S, R, lane, ix, iy + 3);
      // east (lane+1's next column), east-east (lane+2's column after next)
      const T E_c = shdn(n1.c, 1), E_b = shdn(n1.b, 1), E_h = shdn(n1.h, 1);
      const int E_ld = __shfl_down_sync(0xffffffffu, n1.ld, 1);
      T EE_b = shdn(n2.b, 2);
      int EE_ld = __shfl_down_sync(0xffffffffu, n2.ld, 2);
      // west: lane-1's outputs of the previous step, or the boundary
      T W_c = shup(o_c, 1), W_pfe = shup(o_pfe, 1), W_b = shup(o_b, 1);
      int W_ld = __shfl_up_sync(0xffffffffu, o_ld, 1);
      {
        const int j = tau % CHUNK;
        const T t_c = shfl_d(bw_c, j), t_pfe = shfl_d(bw_pfe, j), t_b = shfl_d(bw_b, j);
        const int t_ld = __shfl_sync(0xffffffffu, bw_ld, j);
        if (lane == 0) {
          W_c = t_c;
          W_pfe = t_pfe;
          W_b = t_b;
          W_ld = t_ld;
        }
      }
      if (compute_lane && iy >= 1 && iy <= d.nc) {
        const long long gi = fx_ix(d, ix, iy);
        const bool last_row = ix == d.nr, last_col = iy == d.nc;
        T out_c, pfe = T(0), qfn = T(0);
        if (last_row) {  // iee = min(ix+2, NROWS+1) = ie
          EE_b = E_b;
          EE_ld = E_ld;
        }
        const T NN_b = last_col ? n1.b : n2.b;  // inn = min(iy+2, NCOLS+1)
        const int NN_ld = last_col ? n1.ld : n2.ld;
        if constexpr (sizeof(T) == 4) {
          // the cell is computed for every lane and kept only for a wet cell
          // the sweep reaches: a dry cell gets 0 and no fluxes (:119-124), a
          // step without a sweep and the cell the sweep stops short of (:93)
          // keep the re-scaled value
          const T cmax = fmax(W_b, fmax(E_c, fmax(o_b, n1.c)));
          const T cmin = fmin(W_b, fmin(E_c, fmin(o_b, n1.c)));
          T cell_c, cell_pfe, cell_qfn;
          ade_cell<T>(d, D, (T)S.dt, last_row, last_col, cur.h, E_h, n1.h, cur.qx, cur.qy, W_c, cur.b, E_b,
                   EE_b, o_c, n1.b, NN_b, W_pfe, o_qfn, E_ld, W_ld, EE_ld, n1.ld, o_ld, NN_ld, cmax,
                   cmin, cell_c, cell_pfe, cell_qfn);
          const bool keep = !S.sweep || (last_row && last_col);
          const bool swept = !keep && cur.ld != 1;
          out_c = keep ? cur.b : (swept ? cell_c : T(0));
          pfe = swept ? cell_pfe : T(0);
          qfn = swept ? cell_qfn : T(0);
        } else if (!S.sweep || (last_row && last_col)) {
          out_c = cur.b;  // no sweep this step, or the cell the sweep stops short of (:93)
        } else if (cur.ld == 1) {
          out_c = T(0);  // :119-124
        } else {
          const T cmax = fmax(W_b, fmax(E_c, fmax(o_b, n1.c)));
          const T cmin = fmin(W_b, fmin(E_c, fmin(o_b, n1.c)));
          ade_cell_br<T>(d, D, (T)S.dt, last_row, last_col, cur.h, E_h, n1.h, cur.qx, cur.qy, W_c, cur.b, E_b,
                      EE_b, o_c, n1.b, NN_b, W_pfe, o_qfn, E_ld, W_ld, EE_ld, n1.ld, o_ld, NN_ld, cmax,
                      cmin, out_c, pfe, qfn);
        }
        // the sweep's neighbours and the next strip read the value before the
        // soil release, which follows the whole sweep in the reference
        A[gi] = S.wintra ? soil_release<T>(d, S, k, gi, cur.h, out_c) : out_c;
        if (lane == ROWS - 1 && bnd_out) {
          double* p = bnd_out + (long long)iy * 3;
          p[0] = (double)out_c;
          p[1] = (double)pfe;
          p[2] = (double)cur.b;
        }
        o_c = out_c;
        o_pfe = pfe;
        o_b = cur.b;
        o_ld = cur.ld;
        o_qfn = qfn;
      } else if (iy < 1) {
        // not started: the south neighbour of column 1 is the ghost column
        o_c = T(0);
        o_pfe = T(0);
        o_b = T(0);
        o_ld = 0;
        o_qfn = T(0);
      }
      // publish progress: every lane's writes of this chunk, then the count.
      // The warp barrier orders the other lanes' writes before lane 0's
      // release store, which makes them visible with the count to a warp
      // that reads it and then fences. The next strip of this step overwrites
      // its first two rows only after this count passes the column by ROWS
      // steps; lanes 30 and 31 copied those rows DIST + 3 columns ahead, and
      // cp_wait retires a copy DIST steps after it was issued, so the copies
      // have landed by then.
      if (((tau + 1) % CHUNK) == 0 || tau + 1 == TW) {
        __syncwarp();
        if (lane == 0) st_release(prog_me, (tag << 32) | (unsigned)(tau + 1));
      }
      cur = n1;
      n1 = n2;
      n2 = n3;
    }
    cp_wait<0>();
    return !bail;
  }
}

// One domain: the descriptor is a kernel parameter. Unit u is strip
// u % nstrips of solute (u / nstrips) % nchem at step u / (nstrips * nchem).
// Resident blocks per SM the sweep kernels are compiled for (3: 168
// registers in FP64, 152 in FP32). More resident warps do not pay: their
// rings take shared memory from L1, which serves the lanes' skewed reads
// (FP32 at 4096 x 4096: 1.17 ms per step with 3 blocks, 1.45 with 4 at 128
// registers, 1.41 with 5).
#ifndef FX_ADE_F32_BLOCKS
#define FX_ADE_F32_BLOCKS 3
#endif
template <class T>
struct AdeBlocks {
  static constexpr int value = 3;
};
template <>
struct AdeBlocks<float> {
  static constexpr int value = FX_ADE_F32_BLOCKS;
};

template <class T>
__global__ void __launch_bounds__(WARPS * 32, AdeBlocks<T>::value) k_ade_one(const __grid_constant__ fx_dev d,
                                                                           int nunits) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  Ring<T>& R = reinterpret_cast<Ring<T>*>(smem_raw)[wib];
  const int nwarps = gridDim.x * WARPS;
  if (!d.ade) return;
  const int nstrips = (d.nr + ROWS - 1) / ROWS;
  for (int u = blockIdx.x * WARPS + wib; u < nunits; u += nwarps) {
    const int s = u % nstrips, k = (u / nstrips) % d.nchem, jj = u / (nstrips * d.nchem);
    if (!ade_unit<T>(d, R, jj, k, s, lane)) return;
  }
}

// A batch of domains: units come from the unit table; each warp copies its
// unit's descriptor to its own shared-memory slot.
template <class T>
__global__ void __launch_bounds__(WARPS * 32, AdeBlocks<T>::value) k_ade_batch(const fx_dev* __restrict__ devs,
                                                         const fx_unit* __restrict__ units, int nunits) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ fx_dev wdev[WARPS];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  Ring<T>& R = reinterpret_cast<Ring<T>*>(smem_raw)[wib];
  const int nwarps = gridDim.x * WARPS;
  int have = -1;
  for (int u = blockIdx.x * WARPS + wib; u < nunits; u += nwarps) {
    const fx_unit un = units[u];
    if (un.dom != have) {
      __syncwarp();
      const unsigned long long* src = reinterpret_cast<const unsigned long long*>(devs + un.dom);
      unsigned long long* dst = reinterpret_cast<unsigned long long*>(&wdev[wib]);
      for (int i = lane; i < (int)(sizeof(fx_dev) / 8); i += 32) dst[i] = src[i];
      __syncwarp();
      have = un.dom;
    }
    const fx_dev& d = wdev[wib];
    if (!d.ade) continue;
    if (!ade_unit<T>(d, R, un.jj, un.k, un.s, lane)) return;
  }
}

}  // namespace fxade

int fx_ade_rows_per_strip() { return fxade::ROWS; }
int fx_ade_threads_per_block() { return fxade::WARPS * 32; }
static size_t ade_smem(bool prec32) {
  return (prec32 ? sizeof(fxade::Ring<float>) : sizeof(fxade::Ring<double>)) * fxade::WARPS;
}

void fx_launch_ade(const fx_dev* devs, const fx_unit* units, int nunits, int nblocks, bool prec32, cudaStream_t s) {
  if (prec32) fxade::k_ade_batch<float><<<nblocks, fxade::WARPS * 32, ade_smem(true), s>>>(devs, units, nunits);
  else fxade::k_ade_batch<double><<<nblocks, fxade::WARPS * 32, ade_smem(false), s>>>(devs, units, nunits);
}
void fx_launch_ade_one(const fx_dev& d, int nunits, int nblocks, cudaStream_t s) {
  if (d.prec32) fxade::k_ade_one<float><<<nblocks, fxade::WARPS * 32, ade_smem(true), s>>>(d, nunits);
  else fxade::k_ade_one<double><<<nblocks, fxade::WARPS * 32, ade_smem(false), s>>>(d, nunits);
}

// Appends the ADE units of domain `dom` for a batch of `steps` steps, in the
// order their dependencies require (step, then solute, then strip).
void fx_units_of(int dom, int nr, int nchem, int steps, std::vector<fx_unit>& out) {
  const int nstrips = (nr + fxade::ROWS - 1) / fxade::ROWS;
  for (int jj = 0; jj < steps; ++jj)
    for (int k = 0; k < nchem; ++k)
      for (int s = 0; s < nstrips; ++s) out.push_back(fx_unit{dom, jj, k, s});
}

// Resident blocks per SM of a sweep kernel. The kernel then asks for the
// smallest shared-memory carveout that still holds that many blocks: the
// rest of the SM's on-chip memory is L1, which serves the lanes' skewed
// reads. The count is queried again under the carveout, and the carveout
// is dropped if it would hold fewer blocks.
template <class K>
static int max_blocks_of(K kernel, size_t smem, int nsm, int* out) {
  int per = 0;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return -1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, fxade::WARPS * 32, smem) != cudaSuccess)
    return -1;
  int dev = 0, sm_max = 0, reserved = 0;
  cudaFuncAttributes fa;
  if (per > 0 && cudaGetDevice(&dev) == cudaSuccess &&
      cudaDeviceGetAttribute(&sm_max, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) == cudaSuccess &&
      cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) == cudaSuccess &&
      cudaFuncGetAttributes(&fa, kernel) == cudaSuccess && sm_max > 0) {
    const long long need = (long long)per * ((long long)smem + (long long)fa.sharedSizeBytes + reserved);
    const int pct = (int)std::min<long long>(100, (need * 100 + sm_max - 1) / sm_max);
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, pct) == cudaSuccess) {
      int per2 = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, kernel, fxade::WARPS * 32, smem) != cudaSuccess)
        return -1;
      if (per2 < per &&
          cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, -1) != cudaSuccess)
        return -1;
    }
  }
  cudaGetLastError();  // a refused hint leaves no error behind
  *out = per * nsm;
  return 0;
}

// Resident blocks of the sweep kernels of one precision on this device (the
// smaller of the one-domain and batch forms), after raising their dynamic
// shared memory limit.
int fx_ade_max_blocks_for(bool prec32, int* out) {
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
  int a = 0, b = 0;
  if (prec32) {
    if (max_blocks_of(fxade::k_ade_one<float>, ade_smem(true), nsm, &a) ||
        max_blocks_of(fxade::k_ade_batch<float>, ade_smem(true), nsm, &b))
      return -1;
  } else {
    if (max_blocks_of(fxade::k_ade_one<double>, ade_smem(false), nsm, &a) ||
        max_blocks_of(fxade::k_ade_batch<double>, ade_smem(false), nsm, &b))
      return -1;
  }
  *out = std::min(a, b);
  return 0;
}

// Resident blocks of the sweep kernels on this device (the smallest of the
// four variants), after raising their dynamic shared memory limit.
int fx_ade_max_blocks(int* out) {
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
  int a = 0, b = 0, c = 0, e = 0;
  if (max_blocks_of(fxade::k_ade_one<double>, ade_smem(false), nsm, &a) ||
      max_blocks_of(fxade::k_ade_one<float>, ade_smem(true), nsm, &b) ||
      max_blocks_of(fxade::k_ade_batch<double>, ade_smem(false), nsm, &c) ||
      max_blocks_of(fxade::k_ade_batch<float>, ade_smem(true), nsm, &e))
    return -1;
  *out = std::min(std::min(a, b), std::min(c, e));
  return 0;
}
