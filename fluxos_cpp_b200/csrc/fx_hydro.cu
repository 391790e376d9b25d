// FP64 hydrodynamic step of FLUXOS-OVERLAND for sm_100a.
//
// One launch of k_hydro performs, for a 32 x 8 tile of cells:
//   * the snowmelt forcing of common.cpp:210-262 (add_meteo), including the
//     solute dilution, applied on the fly to every cell the tile reads;
//   * Loop 1 of hydrodynamics_calc.cpp:53-73 (depth, wet flag, wet time);
//   * Loop 2 (:76-90): the east and north face fluxes of solver_wet
//     (solver_wetdomain.cpp:27-342) and solver_dry (solver_drydomain.cpp:27-194)
//     for the tile and its west/south halo, each face once, held in shared
//     memory and used by both cells that share it;
//   * Loop 3 (:93-120) and Loop 4 (:123-154): divergence and update;
//   * the optional Manning friction extension;
//   * the per-cell part of the NEXT step's Courant scan (main.cpp:300-323),
//     reduced with warp shuffles and one atomic per block.
// k_finalize then turns the reduction into the next dt and advances the
// clock on the device, so a run of steps needs no host round trip.
//
// Every expression keeps the reference's operand types and evaluation order
// (the library is built with --fmad=false), so results match the CPU
// reference bit for bit except where noted at fx_pow15.
#include <cuda_runtime.h>

#include <vector>

#include "fx_common.cuh"

namespace fx {

// A block of 32 x BY threads owns a tile of 31 rows (irow) x BY-1 columns
// (icol): with its west row and south column of halo faces the tile has
// exactly 32 x BY face-flux cells, one per thread, so the flux phase runs in
// a single wave and no warp waits at the barrier for a second round. BY (the
// tile rows along icol: 4, 8 or 16) is chosen per domain or batch, by the
// autotuner (fx_autotune) or fx_set_option("tile_rows").
constexpr int BX = 32;          // threads along irow: one warp
constexpr int TX = 31;          // owned rows
constexpr int SX = TX + 3;      // stencil rows irow0-2..irow0+TX
constexpr int FXN = TX + 1;     // flux rows irow0-1..irow0+TX-1
template <int BY>
struct Tile {
  static constexpr int TY = BY - 1;            // owned columns
  static constexpr int SY = TY + 3;            // stencil columns icol0-2..icol0+TY
  static constexpr int FYN = TY + 1;           // flux columns icol0-1..icol0+TY-1
  static constexpr int NSTEN = SX * SY, NFLUX = FXN * FYN, NTHREADS = BX * BY;
  static_assert(NFLUX == NTHREADS, "one face-flux cell per thread");
};

// stencil cell classes
constexpr unsigned char C_DRY = 1;   // Loop-1 ldry == 1 (interior cells only)
constexpr unsigned char C_WALL = 2;  // innerNeumannBCWeir == 1
constexpr unsigned char C_INT = 4;   // interior cell (1..NROWS, 1..NCOLS)

template <int BY>
struct HydroSmem {
  static constexpr int NSTEN = Tile<BY>::NSTEN, NFLUX = Tile<BY>::NFLUX, NW = Tile<BY>::NTHREADS / 32;
  double budget[2 * NW];
  double z[NSTEN], zb[NSTEN], qx[NSTEN], qy[NSTEN];
  // cell velocities q / max(h, hdry, ks) of the stencil, formed once per
  // cell for the wet solver's shear terms (the same expression and operands
  // the solver divides for each face, so the same values); kept for tiles
  // up to 8 rows, the largest tile's state stays within 48 KB
  static constexpr bool VEL = BY <= 8;
  double u[VEL ? NSTEN : 1], v[VEL ? NSTEN : 1];
  double f[6][NFLUX];
  unsigned char cls[NSTEN];
  short wet_list[NFLUX], dry_list[NFLUX], stale_list[NFLUX];
  int nwet, ndry, nstale;
  double red_dt[NW], red_h[NW];
};

// sqrt(h)^3 = pow(h, 1.5) for h >= 0, correctly rounded: s = sqrt(h) is
// refined to a double-double with its exact residual (fma(-s, s, h)), and the
// product h * (s + s_lo) is formed with an exact fma error term (Dekker/Knuth
// error-free transformations; Muller et al., Handbook of Floating-Point
// Arithmetic, ch. 4-5). glibc's pow differs from the correctly rounded value
// in about 1e-3 of arguments, so the edge weir flux may differ from the CPU
// reference by one unit in the last place there.
__device__ __forceinline__ double fx_pow15(double h) {
  if (h == 0.0) return 0.0;
  double s = sqrt(h);
  double e = fma(-s, s, h);
  double slo = e / (2.0 * s);
  double p = h * s;
  double pe = fma(h, s, -p);
  return p + (pe + h * slo);
}

// Cube root of x >= 0 by Newton iteration on the mantissa, using only
// frexp/ldexp and IEEE +,-,*,/, so the oracle's C (ox_cbrt) computes the
// same bits. Used by the Manning extension only.
__device__ __forceinline__ double fx_cbrt(double x) {
  if (!(x > 0.0) || isinf(x)) return x;
  int e;
  double m = frexp(x, &e);
  int r = e % 3;
  if (r < 0) r += 3;
  m = ldexp(m, r);
  e -= r;
  double y = 0.5 + 0.35 * m;
#pragma unroll 1
  for (int i = 0; i < 7; ++i) y = y - (y * y * y - m) / (3.0 * y * y);
  return ldexp(y, e / 3);
}

__device__ __forceinline__ int sidx(int sr, int sc) { return sc * SX + sr; }

// solver_wetdomain.cpp:27-342 for the flux cell at stencil (sr, sc).
template <class SM>
__device__ void solver_wet(const fx_dev& d, const SM& S, int sr, int sc, int irow, int icol,
                           double dtl, double out[6]) {
  const double hdryl = d.hdry, gaccl = d.gaccl;
  const int P = sidx(sr, sc), W = sidx(sr - 1, sc), E = sidx(sr + 1, sc);
  const int Sx = sidx(sr, sc - 1), N = sidx(sr, sc + 1);
  const int ES = sidx(sr + 1, sc - 1), EN = sidx(sr + 1, sc + 1), WN = sidx(sr - 1, sc + 1);
  auto ksat = [&](int k) { return (S.cls[k] & C_INT) ? d.ks : 0.0; };
  auto hat = [&](int k) { return fmax(0.0, S.z[k] - S.zb[k]); };
  const double kspl = ksat(P);
  const double nueml = d.nueml, cvdefl = d.cvdefl;
  const unsigned dx = d.dxy_u, dy = d.dxy_u;
  bool lroe = true;
  double volrat = d.volrat_mode == 0 ? __longlong_as_double(0x7ff0000000000000LL) : 0.0;

  const bool ldp_dry = S.cls[P] & C_DRY;
  const bool lde_dry = S.cls[E] & C_DRY;
  const bool ldn_dry = S.cls[N] & C_DRY;

  const double zbw = S.zb[W], zbp = S.zb[P], zbe = S.zb[E], zbs = S.zb[Sx], zbn = S.zb[N];
  const double zw = S.z[W], zp = S.z[P], ze = S.z[E], zs = S.z[Sx], zn = S.z[N];
  double qp = S.qx[P], qe = S.qx[E], qn = S.qx[N];
  double rw = S.qy[W], rp = S.qy[P], re = S.qy[E], rn = S.qy[N];

  const double zbpe = .5 * (zbe + zbp);
  const double zbpn = .5 * (zbn + zbp);
  const double hp = fmax(0.0, zp - zbp);
  const double hp0 = fmax(fmax(hdryl, hp), kspl);
  const double hw = fmax(0.0, zw - zbw);
  double he = fmax(0.0, ze - zbe);
  const double hs = fmax(0.0, zs - zbs);
  double hn = fmax(0.0, zn - zbn);

  double hme = .5 * (hp + he);
  double qme = .5 * (qp + qe);
  double rme = .5 * (rp + re);
  double hmn = .5 * (hp + hn);
  double qmn = .5 * (qp + qn);
  double rmn = .5 * (rp + rn);

  double dze = ze - zp;
  const double dqe = qe - qp;
  const double dre = re - rp;
  double dzn = zn - zp;
  const double drn = rn - rp;
  const double dqn = qn - qp;

  if (lde_dry) {  // :121-147
    hme = fmax(0.0, zp - zbpe);
    he = 0.0;
    qe = 0.0;
    re = 0.0;
    if (hme > hdryl) {
      if (ze >= zp) {
        qme = 0.0;
        rme = 0.0;
      } else {
        dze = fmin(fabs(dze), hme);
        qme = 0.296 * dze * sqrt(gaccl * dze);
        volrat = 0.5 * dx * hp / dtl;
        qme = fmin(qme, volrat);
        rme = 0.0;
      }
    } else {
      qme = 0.0;
      rme = 0.0;
      hme = 0.0;
    }
    lroe = false;
  }
  if (ldn_dry) {  // :148-175
    hmn = fmax(0.0, zp - zbpn);
    hn = 0.0;
    qn = 0.0;
    rn = 0.0;
    if (hmn > hdryl) {
      if (zn >= zp) {
        qmn = 0.0;
        rmn = 0.0;
      } else {
        dzn = fmin(fabs(dzn), hmn);
        rmn = 0.296 * dzn * sqrt(gaccl * dzn);
        qmn = 0.0;
        volrat = 0.5 * dy * hp / dtl;
        rmn = fmin(rmn, volrat);
      }
    } else {
      qmn = 0.0;
      rmn = 0.0;
      hmn = 0.0;
    }
    lroe = false;
  }

  // :177-203 turbulent stress; the shear velocity us is identically 0 in
  // the reference (set to 0 by initiate.cpp:176 and both update loops).
  const double cme = sqrt(gaccl * hme);
  const double cmn = sqrt(gaccl * hmn);
  const double ume = qme / fmax(hme, hdryl);
  const double vme = rme / fmax(hme, hdryl);
  const double umn = qmn / fmax(hmn, hdryl);
  const double vmn = rmn / fmax(hmn, hdryl);
  const double cnp = cvdefl * 0.0 * hp + nueml;
  const double cne = cvdefl * 0.0 * he + nueml;
  const double cnn = cvdefl * 0.0 * hn + nueml;
  const double hne = .5 * (cnp + cne) * sqrt(hp * he);
  const double hnn = .5 * (cnp + cnn) * sqrt(hp * hn);

  const double up = qp / hp0;
  // neighbour velocities from the stencil (solver_wetdomain.cpp: each is
  // q / max(max(h, hdry), ks) of its cell; a dry neighbour's discharge is 0,
  // so its velocity is 0 whatever depth the division uses)
  double un, us0, use0, une, ve, vw, vwn, ven;
  if constexpr (SM::VEL) {
    un = S.u[N];
    us0 = S.u[Sx];
    use0 = S.u[ES];
    une = S.u[EN];
    ve = S.v[E];
    vw = S.v[W];
    vwn = S.v[WN];
    ven = S.v[EN];
  } else {
    un = qn / fmax(fmax(hn, hdryl), ksat(N));
    us0 = S.qx[Sx] / fmax(fmax(hs, hdryl), ksat(Sx));
    use0 = S.qx[ES] / fmax(fmax(hat(ES), hdryl), ksat(ES));
    une = S.qx[EN] / fmax(fmax(hat(EN), hdryl), ksat(EN));
    ve = re / fmax(fmax(he, hdryl), ksat(E));
    vw = rw / fmax(fmax(hw, hdryl), ksat(W));
    vwn = S.qy[WN] / fmax(fmax(hat(WN), hdryl), ksat(WN));
    ven = S.qy[EN] / fmax(fmax(hat(EN), hdryl), ksat(EN));
  }
  const double vp = rp / hp0;


  const double txye = hne * (fx_div_dxy(d, ve - vp) + fx_div_dxy(d, .25 * (un + une - us0 - use0)));
  const double txyn = hnn * (fx_div_dxy(d, un - up) + fx_div_dxy(d, .25 * (ve + ven - vw - vwn)));

  const double fe1c = qme;
  const double fe2c = qme * ume;
  const double fe3c = qme * vme - txye;
  const double fn1c = rmn;
  const double fn2c = rmn * umn - txyn;
  const double fn3c = rmn * vmn;

  double fe1r, fe2r, fe3r, fn1r, fn2r, fn3r;
  if (lroe) {  // :213-285
    double cc;
    if (hme > d.hdry) {
      double dzea = fabs(dze);
      if (dzea > 0.5 * hme) {
        double dhea = fabs(he - hp);
        dzea = fmin(dzea, dhea);
        dze = copysign(dzea, dze);
      }
      cc = .25 / cme;
    } else {
      cc = 0.0;
    }
    double c1 = ume, c2 = ume + cme, c3 = ume - cme;
    double c1a = fabs(c1), c2a = fabs(c2), c3a = fabs(c3);
    double a11 = c2 * c3a - c2a * c3;
    double a12 = c2a - c3a;
    double a21 = c2 * c3 * (c3a - c2a);
    double a22 = c2a * c2 - c3a * c3;
    double a31 = vme * (c2 * c3a - 2. * cme * c1a - c2a * c3);
    double a32 = vme * (c2a - c3a);
    double a33 = 2. * cme * c1a;
    fe1r = -(a11 * dze + a12 * dqe) * cc;
    fe2r = -(a21 * dze + a22 * dqe) * cc;
    fe3r = -(a31 * dze + a32 * dqe + a33 * dre) * cc;

    if (!ldp_dry && hmn > d.hdry) {
      double dzna = fabs(dzn);
      double dhna = fabs(hn - hp);
      dzna = fmin(dzna, dhna);
      dzn = copysign(dzna, dzn);
      cc = .25 / cmn;
    } else {
      cc = 0.0;
    }
    c1 = vmn;
    c2 = vmn + cmn;
    c3 = vmn - cmn;
    c1a = fabs(c1);
    c2a = fabs(c2);
    c3a = fabs(c3);
    a11 = c2 * c3a - c2a * c3;
    double a13 = c2a - c3a;
    a21 = umn * (c2 * c3a - 2. * cmn * c1a - c2a * c3);
    a22 = 2. * cmn * c1a;
    double a23 = umn * (c2a - c3a);
    a31 = c2 * c3 * (c3a - c2a);
    a33 = c2a * c2 - c3a * c3;
    fn1r = -(a11 * dzn + a13 * drn) * cc;
    fn2r = -(a21 * dzn + a22 * dqn + a23 * drn) * cc;
    fn3r = -(a31 * dzn + a33 * drn) * cc;
  } else {
    fe1r = fe2r = fe3r = fn1r = fn2r = fn3r = 0.0;
  }

  const double fe2p = .5 * gaccl * (hme * hme);
  const double fn3p = .5 * gaccl * (hmn * hmn);
  double fe1 = fe1c + fe1r;
  const double fe2 = fe2c + fe2r + fe2p;
  const double fe3 = fe3c + fe3r;
  double fn1 = fn1c + fn1r;
  const double fn2 = fn2c + fn2r;
  const double fn3 = fn3c + fn3r + fn3p;

  if (icol == 1 || icol == d.nc) fn1 = fmin(volrat, d.sqrt_gaccl * fx_pow15(fmax(hp, 0.0)));
  if (irow == 1 || irow == d.nr) fe1 = fmin(volrat, d.sqrt_gaccl * fx_pow15(fmax(hp, 0.0)));

  const double volpot = d.arbase * hp;
  volrat = volpot / dtl;
  if (volrat > 0.0) {  // :309-332
    if (fe1 > 0.0 && fn1 > 0.0) {
      if (fe1 * dy + fn1 * dx > volrat) {
        double cf = fn1 * dx / (fe1 * dy + fn1 * dx);
        fe1 = fx_div_dxy(d, (1. - cf) * volrat);
        fn1 = fx_div_dxy(d, cf * volrat);
      }
    } else if (fe1 > 0.0) {
      fe1 = fx_div_dxy(d, fmin(fe1 * dy, volrat));
    } else if (fn1 > 0.0) {
      fn1 = fx_div_dxy(d, fmin(fn1 * dx, volrat));
    }
  } else {
    fe1 = 0.0;
    fn1 = 0.0;
  }
  out[0] = fe1;
  out[1] = fe2;
  out[2] = fe3;
  out[3] = fn1;
  out[4] = fn2;
  out[5] = fn3;
}

// solver_drydomain.cpp:78-194 (the cell is dry and has a wet neighbour).
template <class SM>
__device__ void solver_dry(const fx_dev& d, const SM& S, int sr, int sc, int irow, int icol,
                           double dtl, double out[6]) {
  const int P = sidx(sr, sc), E = sidx(sr + 1, sc), N = sidx(sr, sc + 1);
  const double gaccl = d.gaccl;
  double volrat = d.volrat_mode == 0 ? __longlong_as_double(0x7ff0000000000000LL) : 0.0;
  const bool lde_dry = S.cls[E] & C_DRY, ldn_dry = S.cls[N] & C_DRY;
  const double zbp = S.zb[P], zbe = S.zb[E], zbn = S.zb[N];
  const double zp = S.z[P], ze = S.z[E], zn = S.z[N];
  const double hp = fmax(0.0, zp - zp);  // :85 reads z - z
  const double he = fmax(0.0, ze - zbe);
  const double hn = fmax(0.0, zn - zbn);
  const double zbpe = .5 * (zbe + zbp);
  const double zbpn = .5 * (zbn + zbp);
  double dze = ze - zp, dzn = zn - zp;
  double fe1 = 0.0, fe2 = 0.0, fe3 = 0.0, fn1 = 0.0, fn2 = 0.0, fn3 = 0.0;
  if (!lde_dry) {  // :115-145
    double hme = fmax(0.0, ze - zbpe);
    if (hme > d.hdry) {
      if (ze <= zp) {
        double fe2p = .5 * gaccl * hme * hme;
        fe1 = 0.0;
        fe2 = fe2p;
        fe3 = 0.0;
      } else {
        dze = fmin(fabs(dze), hme);
        double qme = 0.296 * dze * sqrt(gaccl * dze);
        hme = 0.444 * dze;
        volrat = d.dxy * he / dtl;
        qme = -fmin(qme, volrat);
        double ume = qme / hme;
        fe1 = qme;
        fe2 = qme * ume + .5 * gaccl * hme * hme;
        fe3 = 0.0;
      }
    }
  }
  if (!ldn_dry) {  // :146-175
    double hmn = fmax(0.0, zn - zbpn);
    if (hmn > d.hdry) {
      if (zn <= zp) {
        double fn3p = .5 * gaccl * hmn * hmn;
        fn1 = 0.0;
        fn2 = 0.0;
        fn3 = fn3p;
      } else {
        dzn = fmin(fabs(dzn), hmn);
        double rmn = 0.296 * dzn * sqrt(gaccl * dzn);
        hmn = 0.444 * dzn;
        volrat = d.dxy * hn / dtl;
        rmn = -fmin(rmn, volrat);
        double vmn = rmn / hmn;
        fn1 = rmn;
        fn2 = 0.0;
        fn3 = rmn * vmn + .5 * gaccl * hmn * hmn;
      }
    }
  }
  if (icol == 1 || icol == d.nc) fn1 = fmin(volrat, d.sqrt_gaccl * fx_pow15(fmax(hp, 0.0)));
  if (irow == 1 || irow == d.nr) fe1 = fmin(volrat, d.sqrt_gaccl * fx_pow15(fmax(hp, 0.0)));
  out[0] = fe1;
  out[1] = fe2;
  out[2] = fe3;
  out[3] = fn1;
  out[4] = fn2;
  out[5] = fn3;
}

// The Courant candidate of one cell (main.cpp:308-316), or +inf if dry.
__device__ __forceinline__ void courant_cell(const fx_dev& d, double h, double qx, double qy,
                                             double& dtc, double& hm) {
  dtc = __longlong_as_double(0x7ff0000000000000LL);
  hm = 0.0;
  if (h > d.hdry) {
    double hp = fmax(h, d.hdry);
    double c0 = sqrt(d.gaccl * h);
    double u0 = fmax(.000001, fabs(qx / hp));
    double v0 = fmax(.000001, fabs(qy / hp));
    // min(a / (u0 + c0), a / (v0 + c0)) with a > 0 is a / (max(u0, v0) + c0)
    // bit for bit: rounded addition and division are monotone
    double c = d.cfl_dxy / (fmax(u0, v0) + c0);
    if (c == c) dtc = c;
    hm = h;
  }
}

// Block-wide min/max followed by one atomic each on the control block.
template <class SM>
__device__ void reduce_courant(const fx_dev& d, SM& S, double dtc, double hm) {
  for (int o = 16; o > 0; o >>= 1) {
    dtc = fmin(dtc, __shfl_xor_sync(0xffffffffu, dtc, o));
    hm = fmax(hm, __shfl_xor_sync(0xffffffffu, hm, o));
  }
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nw = (blockDim.x * blockDim.y) / 32;
  if ((tid & 31) == 0) {
    S.red_dt[tid >> 5] = dtc;
    S.red_h[tid >> 5] = hm;
  }
  __syncthreads();
  if (tid == 0) {
    double a = S.red_dt[0], b = S.red_h[0];
    for (int w = 1; w < nw; ++w) {
      a = fmin(a, S.red_dt[w]);
      b = fmax(b, S.red_h[w]);
    }
    if (a < __longlong_as_double(0x7ff0000000000000LL))
      atomicMin(&d.ctl->acc_dtmin, (unsigned long long)__double_as_longlong(a));
    if (b > 0.0) atomicMax(&d.ctl->acc_hmax, (unsigned long long)__double_as_longlong(b));
  }
}

// Shared-memory staging of a tile's stencil by TMA (k_hydro_tma). Each field
// of the stencil (rows irow0-2..irow0+TX, columns icol0-2..icol0+TY) arrives
// as one box of W elements x (BY+2) columns. A TMA box must start on a
// 16-byte boundary along irow, so the box starts at the stencil's first row
// rounded down to 4 (4-byte elements), 2 (8-byte) or 16 (1-byte) elements,
// and the stencil sits `xo` elements into it. Rows and columns outside the
// field read 0 (TMA out-of-bounds fill; the field padding is 0 as well), as
// the per-thread loads of the unstaged path do.
constexpr int STG_W4 = 40, STG_W8 = 36, STG_W1 = 64;  // box widths: 34 + largest offset, 16-byte multiples
__host__ __device__ constexpr int stg_round(int b) { return (b + 127) / 128 * 128; }
template <bool P32, int BY>
struct StageLayout {
  static constexpr int SY = BY + 2;
  static constexpr int B4 = stg_round(STG_W4 * SY * 4), B8 = stg_round(STG_W8 * SY * 8), B1 = stg_round(STG_W1 * SY);
  // FP64 stage: z, zb, qx, qy, melt multiplier (8-byte boxes), flags (1-byte)
  // FP32 stage: eta, eta_lo, qx, qy, melt multiplier (4-byte boxes), zb (8-byte), flags
  static constexpr int O_Z = 0;                                   // z | eta
  static constexpr int O_LO = P32 ? B4 : 0;                       // - | eta_lo
  static constexpr int O_ZB = P32 ? 2 * B4 : B8;                  // zb
  static constexpr int O_QX = P32 ? 2 * B4 + B8 : 2 * B8;         // qx
  static constexpr int O_QY = P32 ? 3 * B4 + B8 : 3 * B8;         // qy
  static constexpr int O_MM = P32 ? 4 * B4 + B8 : 4 * B8;         // melt multiplier
  static constexpr int O_FL = P32 ? 5 * B4 + B8 : 5 * B8;         // flags
  static constexpr int BYTES = O_FL + B1;
};

// x offsets of the stencil in the staged boxes of tile column bx.
struct StageOff {
  int o4, o8, o1;
};
__device__ __forceinline__ StageOff stage_off(int bx) {
  const int x = TX * bx;  // element index of stencil row 0: irow0 - 2 + FX_ROFF
  return StageOff{x & 3, x & 1, x & 15};
}

// A thread's share of a launch's reductions, kept across the tiles it works
// on and reduced once per block (reduce_part): the smallest Courant dt and
// the largest wet depth (exact in any order) and the FP64 water budget.
struct TilePart {
  double dtc, hm, melt, out;
  __device__ __forceinline__ void add(double dt, double h, double m, double o) {
    dtc = fmin(dtc, dt);
    hm = fmax(hm, h);
    melt += m;
    out += o;
  }
};
__device__ __forceinline__ TilePart tile_part() {
  TilePart p;
  p.dtc = __longlong_as_double(0x7ff0000000000000LL);
  p.hm = p.melt = p.out = 0.0;
  return p;
}

// The fields of the control block a step kernel reads.
struct StepCtl {
  double dtfl, meteoi, meteo_rate, mconc, inflowi;
  double twet_inc;  // dtfl / 3600, the wet-time increment (hydrodynamics_calc.cpp:69-70), once per tile
  long long steps;
  int live, active;
};

// Block sum of the step's water budget terms, one double atomic each.
__device__ void reduce_budget(const fx_dev& d, double* red, double melt, double out) {
  for (int o = 16; o > 0; o >>= 1) {
    melt += __shfl_xor_sync(0xffffffffu, melt, o);
    out += __shfl_xor_sync(0xffffffffu, out, o);
  }
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nw = (blockDim.x * blockDim.y) / 32;
  __syncthreads();
  if ((tid & 31) == 0) {
    red[2 * (tid >> 5)] = melt;
    red[2 * (tid >> 5) + 1] = out;
  }
  __syncthreads();
  if (tid == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < nw; ++w) {
      a += red[2 * w];
      b += red[2 * w + 1];
    }
    if (a != 0.0) atomicAdd(&d.ctl->budget_melt, a);
    if (b != 0.0) atomicAdd(&d.ctl->budget_out, b);
  }
}

// The block's reductions of a launch: Courant dt and wet depth, then the
// budget (every thread of the block calls it).
template <class SM>
__device__ __forceinline__ void reduce_part(const fx_dev& d, SM& S, const TilePart& acc) {
  reduce_courant(d, S, acc.dtc, acc.hm);
  reduce_budget(d, S.budget, acc.melt, acc.out);
}

__device__ __forceinline__ double melt_depth(const fx_dev& d, const StepCtl& c, long long gi) {
  if (d.melt_mult) return (double)c.meteo_rate * d.melt_mult[gi] / (1000. * 3600. * 24.) * c.dtfl;
  if (d.melt_mult_f) return (double)c.meteo_rate * (double)d.melt_mult_f[gi] / (1000. * 3600. * 24.) * c.dtfl;
  return c.meteoi;
}

// The point inflow of common.cpp:300-309 on its cell's water level (after
// the melt): a level below the bed is first raised to the bed, then the
// step's inflow depth is added.
__device__ __forceinline__ double inflow_z(double z, double zb, double inflowi) {
  if (z <= zb) z = zb;
  return z + inflowi;
}
// The same on the FP32 state's compensated depth.
__device__ __forceinline__ void inflow_eta(float& eta, float& lo, double inflowi) {
  if (fx_dd_val(eta, lo) <= 0.0) {
    eta = 0.0f;
    lo = 0.0f;
  }
  fx_dd_add(eta, lo, (float)inflowi);
}
__device__ __forceinline__ bool is_inflow(const fx_dev& d, int r, int q) {
  return d.has_inflow && r == d.inflow_irow && q == d.inflow_icol;
}
// The depth the inflow cell had after the melt, for the ADE's dilution.
__device__ __forceinline__ void record_inflow_hm(const fx_dev& d, const StepCtl& c, double hm) {
  d.ctl->rec[c.steps % d.nslot].inflow_hm = hm;
}


// ===================== single-precision step (prec32) =======================
// The same step as the FP64 body, on the depth eta = z - zb and the bed
// differences sx = zb(E) - zb(P), sy = zb(N) - zb(P), formed exactly in FP64
// from the stencil's bed values: every water-surface difference of the
// reference is rewritten without the bed elevation itself,
//   ze - zp = sx(P) + (eta_E - eta_P),  zp - zbpe = eta_P - sx(P)/2,
//   ze - zbpe = eta_E + sx(P)/2,        h = max(0, eta),
// and likewise to the north with sy. Flux, update and friction arithmetic is
// FP32 on the high part of the compensated depth; the branch tests on
// near-zero depths (wet/dry, the face-depth thresholds of both solvers) and
// the signs of near-zero surface differences are decided in FP64 on the
// compensated depth; the Courant candidates and the water budget are FP64.

template <int BY>
struct HydroSmem32 {
  static constexpr int NSTEN = Tile<BY>::NSTEN, NFLUX = Tile<BY>::NFLUX, NW = Tile<BY>::NTHREADS / 32;
  double budget[2 * NW];
  double red_dt[NW], red_h[NW];
  double zb[NSTEN];
  float eta[NSTEN], eta_lo[NSTEN], qx[NSTEN], qy[NSTEN];
  // cell velocities q / max(h, hdry, ks) of the stencil, formed once per
  // cell for the wet solver's shear terms (each face reads eight of them)
  static constexpr bool VEL = true;
  float u[NSTEN], v[NSTEN];
  float f[6][NFLUX];
  unsigned char cls[NSTEN];
};

// FP32 arithmetic divides and takes square roots by the approximate hardware
// reciprocal and square root (PTX rcp.approx / sqrt.approx) refined by one
// Newton step with fused multiply-adds: close to correctly rounded for the
// finite, normal operands of this scheme, without the IEEE code paths; the
// FP64 path keeps IEEE-rounded operations for bit parity with the reference.
__device__ __forceinline__ float frcp(float a) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
  return fmaf(fmaf(-a, r, 1.0f), r, r);
}
__device__ __forceinline__ float fdiv(float a, float b) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(b));
  const float q = a * r;
  return fmaf(fmaf(-b, q, a), r, q);
}
__device__ __forceinline__ float fsqrt(float a) {
  float s, r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(s) : "f"(a));
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(s));
  const float t = fmaf(fmaf(-s, s, a), 0.5f * r, s);
  return a > 0.0f ? t : s;
}
// Cube root of h > 0 as 2^(log2(h) / 3) (the friction term only).
__device__ __forceinline__ float fcbrt(float h) {
  float l, r;
  asm("lg2.approx.f32 %0, %1;" : "=f"(l) : "f"(h));
  l = l * (1.0f / 3.0f);
  asm("ex2.approx.f32 %0, %1;" : "=f"(r) : "f"(l));
  return r;
}

// The melt depth the FP32 state adds to a cell this step: the step's
// uniform depth c.meteoi (rate / (1000*3600*24) * dt, computed once in
// k_finalize) times the cell's melt multiplier, rounded once to float. The
// budget counts this float value, the water actually added.
__device__ __forceinline__ float melt32(const fx_dev& d, const StepCtl& c, float mm) {
  return d.melt_mult_f ? (float)(c.meteoi * (double)mm) : (float)c.meteoi;
}

// The Courant candidate of main.cpp:300-323 for the FP32 state. It stays
// FP64, so the FP32 state's dt sequence follows the reference's formula to
// the last bits, but with two divisions instead of four: depth > hdry, so
// the reference's max(h, hdry) is h; u0 and v0 share one reciprocal; and
// min(cfl dxy / (u0 + c0), cfl dxy / (v0 + c0)) = cfl dxy / (max(u0, v0) + c0).
__device__ __forceinline__ void courant_cell32(const fx_dev& d, double depth, float qx, float qy, double& dtc,
                                               double& hm) {
  dtc = __longlong_as_double(0x7ff0000000000000LL);
  hm = 0.0;
  if (depth > d.hdry) {
    const double rh = 1.0 / depth;
    const double c0 = sqrt(d.gaccl * depth);
    const double u0 = fmax(.000001, fabs((double)qx * rh)), v0 = fmax(.000001, fabs((double)qy * rh));
    const double cc = d.cfl_dxy / (fmax(u0, v0) + c0);
    if (cc == cc) dtc = cc;
    hm = depth;
  }
}

__device__ __forceinline__ float div_dxy_f(const fx_dev& d, float x) {
  return d.dxy_pow2 ? x * (float)d.inv_dxy : fdiv(x, (float)d.dxy);
}

// The Roe face-depth test of the FP32 state, `.5 * (max(0, dP) + max(0, dQ))
// > hdry` on the two cells' compensated FP64 depths, decided from its FP32
// value x = .5f * (max(0, eta_P) + max(0, eta_Q)) where that is safe: each
// eta differs from its compensated depth by at most half an ulp and the sum
// rounds once, so |x - exact| <= x * 2^-23, and outside the band
// [hdry (1 - 2^-19), hdry (1 + 2^-19)] (bounds rounded to float) x and the
// exact value lie on the same side of hdry. Inside the band the FP64 test
// (`exact`) decides. The outcome is the FP64 test's in every case.
template <class F>
__device__ __forceinline__ bool above_hdry(float x, float lo, float hi, F exact) {
  if (x > hi) return true;
  if (x < lo) return false;
  return exact();
}

template <class SM>
__device__ void solver_wet32(const fx_dev& d, const SM& S, int sr, int sc, int irow, int icol,
                             float dtl, float out[6]) {
  const double hdry = d.hdry;
  const float hdryl = (float)d.hdry, gaccl = (float)d.gaccl;
  const float hdry_lo = (float)(hdry * (1.0 - 0x1p-19)), hdry_hi = (float)(hdry * (1.0 + 0x1p-19));
  const int P = sidx(sr, sc), W = sidx(sr - 1, sc), E = sidx(sr + 1, sc);
  const int Sx = sidx(sr, sc - 1), N = sidx(sr, sc + 1);
  const int ES = sidx(sr + 1, sc - 1), EN = sidx(sr + 1, sc + 1), WN = sidx(sr - 1, sc + 1);
  auto ksat = [&](int k) { return (S.cls[k] & C_INT) ? (float)d.ks : 0.0f; };
  const float kspl = ksat(P);
  const float nueml = (float)d.nueml;
  const float dx = (float)d.dxy, dy = dx;
  bool lroe = true;
  float volrat = d.volrat_mode == 0 ? __int_as_float(0x7f800000) : 0.0f;
  const bool ldp_dry = S.cls[P] & C_DRY, lde_dry = S.cls[E] & C_DRY, ldn_dry = S.cls[N] & C_DRY;
  // bed differences: exact in FP64 for the branch tests, rounded for the flux arithmetic
  const double sx_d = S.zb[E] - S.zb[P], sy_d = S.zb[N] - S.zb[P];
  const float etap = S.eta[P], sxp = (float)sx_d, syp = (float)sy_d;
  // compensated depths for the branch tests (FP64, as the FP64 path decides
  // them), formed where a test needs them
  auto dd = [&](int k) { return fx_dd_val(S.eta[k], S.eta_lo[k]); };
  float qp = S.qx[P], qe = S.qx[E], qn = S.qx[N];
  float rw = S.qy[W], rp = S.qy[P], re = S.qy[E], rn = S.qy[N];
  const float hp = fmaxf(0.0f, etap);
  const float hp0 = fmaxf(fmaxf(hdryl, hp), kspl);
  const float hw = fmaxf(0.0f, S.eta[W]);
  float he = fmaxf(0.0f, S.eta[E]);
  const float hs = fmaxf(0.0f, S.eta[Sx]);
  float hn = fmaxf(0.0f, S.eta[N]);
  float hme = .5f * (hp + he), qme = .5f * (qp + qe), rme = .5f * (rp + re);
  float hmn = .5f * (hp + hn), qmn = .5f * (qp + qn), rmn = .5f * (rp + rn);
  float dze = sxp + (S.eta[E] - etap);
  const float dqe = qe - qp, dre = re - rp;
  float dzn = syp + (S.eta[N] - etap);
  const float drn = rn - rp, dqn = qn - qp;
  if (lde_dry) {
    hme = fmaxf(0.0f, etap - .5f * sxp);
    he = qe = re = 0.0f;
    const double dP = dd(P), dE = dd(E);
    const double dze_d = sx_d + (dE - dP);
    if (fmax(0.0, dP - .5 * sx_d) > hdry) {
      if (dze_d >= 0.0) {
        qme = rme = 0.0f;
      } else {
        dze = fminf((float)fabs(dze_d), hme);
        qme = 0.296f * dze * fsqrt(gaccl * dze);
        volrat = fdiv(0.5f * dx * hp, dtl);
        qme = fminf(qme, volrat);
        rme = 0.0f;
      }
    } else {
      qme = rme = hme = 0.0f;
    }
    lroe = false;
  }
  if (ldn_dry) {
    hmn = fmaxf(0.0f, etap - .5f * syp);
    hn = qn = rn = 0.0f;
    const double dP = dd(P), dN = dd(N);
    const double dzn_d = sy_d + (dN - dP);
    if (fmax(0.0, dP - .5 * sy_d) > hdry) {
      if (dzn_d >= 0.0) {
        qmn = rmn = 0.0f;
      } else {
        dzn = fminf((float)fabs(dzn_d), hmn);
        rmn = 0.296f * dzn * fsqrt(gaccl * dzn);
        qmn = 0.0f;
        volrat = fdiv(0.5f * dy * hp, dtl);
        rmn = fminf(rmn, volrat);
      }
    } else {
      qmn = rmn = hmn = 0.0f;
    }
    lroe = false;
  }
  const float cme = fsqrt(gaccl * hme), cmn = fsqrt(gaccl * hmn);
  const float rhme = frcp(fmaxf(hme, hdryl)), rhmn = frcp(fmaxf(hmn, hdryl));
  const float ume = qme * rhme, vme = rme * rhme;
  const float umn = qmn * rhmn, vmn = rmn * rhmn;
  const float hne = nueml * fsqrt(hp * he);  // (cvdef*us*h + nuem), us = 0
  const float hnn = nueml * fsqrt(hp * hn);
  const float rhp0 = frcp(hp0);
  const float up = qp * rhp0;
  // neighbour velocities from the stencil (a dry neighbour's discharge is 0,
  // so its velocity is 0 whatever depth the division uses)
  const float un = S.u[N];
  const float us0 = S.u[Sx];
  const float use0 = S.u[ES];
  const float une = S.u[EN];
  const float vp = rp * rhp0;
  const float ve = S.v[E];
  const float vw = S.v[W];
  const float vwn = S.v[WN];
  const float ven = S.v[EN];
  const float txye = hne * (div_dxy_f(d, ve - vp) + div_dxy_f(d, .25f * (un + une - us0 - use0)));
  const float txyn = hnn * (div_dxy_f(d, un - up) + div_dxy_f(d, .25f * (ve + ven - vw - vwn)));
  const float fe1c = qme, fe2c = qme * ume, fe3c = qme * vme - txye;
  const float fn1c = rmn, fn2c = rmn * umn - txyn, fn3c = rmn * vmn;
  float fe1r = 0.f, fe2r = 0.f, fe3r = 0.f, fn1r = 0.f, fn2r = 0.f, fn3r = 0.f;
  if (lroe) {
    float cc;
    if (above_hdry(hme, hdry_lo, hdry_hi, [&] { return .5 * (fmax(0.0, dd(P)) + fmax(0.0, dd(E))) > hdry; })) {
      float dzea = fabsf(dze);
      if (dzea > 0.5f * hme) {
        dzea = fminf(dzea, fabsf(he - hp));
        dze = copysignf(dzea, dze);
      }
      cc = fdiv(.25f, cme);
    } else {
      cc = 0.0f;
    }
    float c1 = ume, c2 = ume + cme, c3 = ume - cme;
    float c1a = fabsf(c1), c2a = fabsf(c2), c3a = fabsf(c3);
    fe1r = -((c2 * c3a - c2a * c3) * dze + (c2a - c3a) * dqe) * cc;
    fe2r = -(c2 * c3 * (c3a - c2a) * dze + (c2a * c2 - c3a * c3) * dqe) * cc;
    fe3r = -(vme * (c2 * c3a - 2.f * cme * c1a - c2a * c3) * dze + vme * (c2a - c3a) * dqe + 2.f * cme * c1a * dre) * cc;
    if (!ldp_dry &&
        above_hdry(hmn, hdry_lo, hdry_hi, [&] { return .5 * (fmax(0.0, dd(P)) + fmax(0.0, dd(N))) > hdry; })) {
      float dzna = fminf(fabsf(dzn), fabsf(hn - hp));
      dzn = copysignf(dzna, dzn);
      cc = fdiv(.25f, cmn);
    } else {
      cc = 0.0f;
    }
    c1 = vmn;
    c2 = vmn + cmn;
    c3 = vmn - cmn;
    c1a = fabsf(c1);
    c2a = fabsf(c2);
    c3a = fabsf(c3);
    fn1r = -((c2 * c3a - c2a * c3) * dzn + (c2a - c3a) * drn) * cc;
    fn2r = -(umn * (c2 * c3a - 2.f * cmn * c1a - c2a * c3) * dzn + 2.f * cmn * c1a * dqn + umn * (c2a - c3a) * drn) * cc;
    fn3r = -(c2 * c3 * (c3a - c2a) * dzn + (c2a * c2 - c3a * c3) * drn) * cc;
  }
  float fe1 = fe1c + fe1r;
  const float fe2 = fe2c + fe2r + .5f * gaccl * (hme * hme);
  const float fe3 = fe3c + fe3r;
  float fn1 = fn1c + fn1r;
  const float fn2 = fn2c + fn2r;
  const float fn3 = fn3c + fn3r + .5f * gaccl * (hmn * hmn);
  if (icol == 1 || icol == d.nc || irow == 1 || irow == d.nr) {  // the edge weir, on edge cells only
    const float weir = fsqrt(gaccl) * hp * fsqrt(hp);
    if (icol == 1 || icol == d.nc) fn1 = fminf(volrat, weir);
    if (irow == 1 || irow == d.nr) fe1 = fminf(volrat, weir);
  }
  volrat = fdiv((float)d.arbase * hp, dtl);
  {  // solver_wetdomain.cpp:309-332 as selects: one straight-line block, the
     // quotient of the split kept only when the split applies
    const float sdy = fe1 * dy, sdx = fn1 * dx, sum = sdy + sdx;
    const bool pos = volrat > 0.0f, pe = fe1 > 0.0f, pn = fn1 > 0.0f;
    const bool split = pos && pe && pn && sum > volrat;
    const float cf = fdiv(sdx, split ? sum : 1.0f);
    const float e = div_dxy_f(d, split ? (1.f - cf) * volrat : fminf(sdy, volrat));
    const float n = div_dxy_f(d, split ? cf * volrat : fminf(sdx, volrat));
    fe1 = !pos ? 0.0f : ((split || (pe && !pn)) ? e : fe1);
    fn1 = !pos ? 0.0f : ((split || (pn && !pe)) ? n : fn1);
  }
  out[0] = fe1;
  out[1] = fe2;
  out[2] = fe3;
  out[3] = fn1;
  out[4] = fn2;
  out[5] = fn3;
}

template <class SM>
__device__ void solver_dry32(const fx_dev& d, const SM& S, int sr, int sc, int irow, int icol,
                             float dtl, float out[6]) {
  const int P = sidx(sr, sc), E = sidx(sr + 1, sc), N = sidx(sr, sc + 1);
  const float gaccl = (float)d.gaccl;
  float volrat = d.volrat_mode == 0 ? __int_as_float(0x7f800000) : 0.0f;
  const bool lde_dry = S.cls[E] & C_DRY, ldn_dry = S.cls[N] & C_DRY;
  const double sx_d = S.zb[E] - S.zb[P], sy_d = S.zb[N] - S.zb[P];
  const float etap = S.eta[P], etae = S.eta[E], etan = S.eta[N], sxp = (float)sx_d, syp = (float)sy_d;
  const double dP = fx_dd_val(etap, S.eta_lo[P]), dE = fx_dd_val(etae, S.eta_lo[E]);
  const double dN = fx_dd_val(etan, S.eta_lo[N]);
  const float he = fmaxf(0.0f, etae), hn = fmaxf(0.0f, etan);
  float dze = sxp + (etae - etap), dzn = syp + (etan - etap);
  float fe1 = 0.f, fe2 = 0.f, fe3 = 0.f, fn1 = 0.f, fn2 = 0.f, fn3 = 0.f;
  if (!lde_dry) {
    float hme = fmaxf(0.0f, etae + .5f * sxp);
    const double dze_d = sx_d + (dE - dP);
    if (fmax(0.0, dE + .5 * sx_d) > d.hdry) {
      if (dze_d <= 0.0) {
        fe2 = .5f * gaccl * hme * hme;
      } else {
        // the surface difference is positive (decided in FP64); its FP32
        // value can round to 0, where the inflow and its momentum are 0
        dze = fminf((float)dze_d, hme);
        volrat = fdiv((float)d.dxy * he, dtl);
        if (dze > 0.0f) {
          float qme = 0.296f * dze * fsqrt(gaccl * dze);
          hme = 0.444f * dze;
          qme = -fminf(qme, volrat);
          fe1 = qme;
          fe2 = qme * fdiv(qme, hme) + .5f * gaccl * hme * hme;
        }
      }
    }
  }
  if (!ldn_dry) {
    float hmn = fmaxf(0.0f, etan + .5f * syp);
    const double dzn_d = sy_d + (dN - dP);
    if (fmax(0.0, dN + .5 * sy_d) > d.hdry) {
      if (dzn_d <= 0.0) {
        fn3 = .5f * gaccl * hmn * hmn;
      } else {
        dzn = fminf((float)dzn_d, hmn);
        volrat = fdiv((float)d.dxy * hn, dtl);
        if (dzn > 0.0f) {
          float rmn = 0.296f * dzn * fsqrt(gaccl * dzn);
          hmn = 0.444f * dzn;
          rmn = -fminf(rmn, volrat);
          fn1 = rmn;
          fn3 = rmn * fdiv(rmn, hmn) + .5f * gaccl * hmn * hmn;
        }
      }
    }
  }
  // the dry cell's own depth is taken as 0 (solver_drydomain.cpp:85): the weir is 0
  if (icol == 1 || icol == d.nc) fn1 = fminf(volrat, 0.0f);
  if (irow == 1 || irow == d.nr) fe1 = fminf(volrat, 0.0f);
  out[0] = fe1;
  out[1] = fe2;
  out[2] = fe3;
  out[3] = fn1;
  out[4] = fn2;
  out[5] = fn3;
}

// The FP64 per-step record of an owned cell in the step's slot
// (fx_dev::rec64), as three 16-byte stores.
__device__ __forceinline__ void put_rec64(const fx_dev& d, long long o, double h0, double h, double hp, double fe1,
                                          double fn1, uint8_t fl) {
  double2* r = reinterpret_cast<double2*>(fx_rec64(d, o));
  r[0] = make_double2(h0, h);
  r[1] = make_double2(hp, fe1);
  r[2] = make_double2(fn1, __longlong_as_double((long long)fl));
}

// The per-step record of an owned cell in the step's slot (fx_dev::rec32).
__device__ __forceinline__ void put_rec32(const fx_dev& d, long long o, float h0, float h, float hp, float mi,
                                          float fe1, float fn1, uint8_t fl) {
  float4* r = d.rec32 + 2 * o;
  r[0] = make_float4(h0, h, hp, mi);
  r[1] = make_float4(fe1, fn1, __uint_as_float((unsigned)fl), 0.0f);
}

template <int BY>
__device__ __forceinline__ bool hydro_tile32(const fx_dev& d, const StepCtl& c, const fx_tile& tile,
                                             HydroSmem32<BY>& S, TilePart& acc, const unsigned char* stg = nullptr,
                                             int bad = 0) {
  using L = StageLayout<true, BY>;
  const StageOff so = stage_off(tile.bx);
  constexpr int TY = Tile<BY>::TY, NSTEN = Tile<BY>::NSTEN, NFLUX = Tile<BY>::NFLUX;
  constexpr int NTHREADS = Tile<BY>::NTHREADS;
  const int lx = threadIdx.x, ly = threadIdx.y;
  const int tid = ly * BX + lx;
  const int irow0 = 1 + tile.bx * TX, icol0 = 1 + tile.by * TY;
  const int irow = irow0 + lx, icol = icol0 + ly;
  const bool own = lx < TX && ly < TY && irow <= d.nr && icol <= d.nc;
  const float dtl = (float)c.dtfl;
  const bool melt_on = d.has_meteo != 0;
  const long long sprev = fx_slot(d, c.steps - 1), scur = fx_slot(d, c.steps);
  const long long pprev = fx_pp(d, c.steps - 1), pcur = fx_pp(d, c.steps);
  double dtc = __longlong_as_double(0x7ff0000000000000LL), hm = 0.0, bmelt = 0.0, bout = 0.0;

  if (!c.active) {
    if (own) {
      const long long gi = fx_ix(d, irow, icol);
      const float etapre = d.eta[pprev + gi];
      float eta1 = etapre, lo1 = d.eta_lo[pprev + gi];
      const uint8_t fl = d.flags[sprev + gi];
      const float hpre = fmaxf(0.0f, etapre);
      uint8_t ld = fx_dd_val(etapre, lo1) > d.hdry ? 0 : 1;
      float h1 = hpre;
      double depth = fx_dd_val(etapre, lo1);
      float mir = 0.0f;  // the record's melt depth
      if (melt_on && !(fl & FX_F_NODATA)) {
        const float mi = melt32(d, c, d.melt_mult_f ? d.melt_mult_f[gi] : 1.0f);
        mir = mi;
        bmelt = (double)mi * d.arbase;
        fx_dd_add(eta1, lo1, mi);
        h1 = fmaxf(eta1, 0.0f);
        depth = fx_dd_val(eta1, lo1);
        if (depth <= d.hdry) ld = 0;
      }
      if (is_inflow(d, irow, icol)) {  // common.cpp:300-315
        const double dm = fx_dd_val(eta1, lo1);
        record_inflow_hm(d, c, fmax(dm, 0.0));
        inflow_eta(eta1, lo1, c.inflowi);
        depth = fx_dd_val(eta1, lo1);
        bmelt += (depth - dm) * d.arbase;
        h1 = fmaxf(eta1, 0.0f);
        ld = depth <= d.hdry ? 1 : 0;
      }
      const float qx = d.qx_f[pprev + gi], qy = d.qy_f[pprev + gi];
      d.eta[pcur + gi] = eta1;
      d.eta_lo[pcur + gi] = lo1;
      d.qx_f[pcur + gi] = qx;
      d.qy_f[pcur + gi] = qy;
      const uint8_t fl1 = (fl & (FX_F_WALL | FX_F_NODATA)) | ((fl & FX_F_LDRY) ? FX_F_LDRY_PREV : 0) | ld;
      d.flags[scur + gi] = fl1;
      // fluxes are unchanged by a step without solver
      const float* rp = fx_rec(d, sprev + gi);
      const bool melted = melt_on && !(fl & FX_F_NODATA);
      put_rec32(d, scur + gi, h1, h1, melted ? hpre : 0.0f, mir,
                rp[FX_R_FE1], rp[FX_R_FN1], fl1);
      courant_cell32(d, fmax(0.0, depth), qx, qy, dtc, hm);
    }
    acc.add(dtc, hm, bmelt, 0.0);
    return true;
  }

  if (stg) {
    // staged by TMA: the same values, read from shared memory
    const float* g_eta = reinterpret_cast<const float*>(stg + L::O_Z);
    const float* g_lo = reinterpret_cast<const float*>(stg + L::O_LO);
    const double* g_zb = reinterpret_cast<const double*>(stg + L::O_ZB);
    const float* g_qx = reinterpret_cast<const float*>(stg + L::O_QX);
    const float* g_qy = reinterpret_cast<const float*>(stg + L::O_QY);
    const float* g_mm = reinterpret_cast<const float*>(stg + L::O_MM);
    const uint8_t* g_fl = stg + L::O_FL;
    for (int k = tid; k < NSTEN; k += NTHREADS) {
      const int sr = k % SX, scc = k / SX;
      const int r = irow0 - 2 + sr, q = icol0 - 2 + scc;
      const int i4 = scc * STG_W4 + sr + so.o4;
      float eta = g_eta[i4], lo = g_lo[i4], qx = g_qx[i4], qy = g_qy[i4];
      const double zb = g_zb[scc * STG_W8 + sr + so.o8];
      unsigned char cl = 0;
      if (r >= 1 && r <= d.nr && q >= 1 && q <= d.nc) {
        cl = C_INT;
        const uint8_t fl = g_fl[scc * STG_W1 + sr + so.o1];
        if (fl & FX_F_WALL) cl |= C_WALL;
        if (melt_on && !(fl & FX_F_NODATA)) fx_dd_add(eta, lo, melt32(d, c, g_mm[i4]));
        if (is_inflow(d, r, q)) inflow_eta(eta, lo, c.inflowi);
        if (fx_dd_val(eta, lo) <= d.hdry) {
          qx = 0.f;
          qy = 0.f;
          cl |= C_DRY;
        }
      }
      S.eta[k] = eta;
      S.eta_lo[k] = lo;
      S.zb[k] = zb;
      S.qx[k] = qx;
      S.qy[k] = qy;
      S.cls[k] = cl;
      {
        const float den = fmaxf(fmaxf(fmaxf(0.0f, eta), (float)d.hdry), (cl & C_INT) ? (float)d.ks : 0.0f);
        S.u[k] = fdiv(qx, den);
        S.v[k] = fdiv(qy, den);
      }
    }
  } else
  for (int k = tid; k < NSTEN; k += NTHREADS) {
    const int sr = k % SX, scc = k / SX;
    const int r = irow0 - 2 + sr, q = icol0 - 2 + scc;
    float eta = 0.f, lo = 0.f, qx = 0.f, qy = 0.f;
    double zb = 0.0;
    unsigned char cl = 0;
    if (r >= 0 && r <= d.nr + 1 && q >= 0 && q <= d.nc + 1) {
      const long long gi = fx_ix(d, r, q);
      eta = d.eta[pprev + gi];
      lo = d.eta_lo[pprev + gi];
      zb = d.zb[gi];
      qx = d.qx_f[pprev + gi];
      qy = d.qy_f[pprev + gi];
      if (r >= 1 && r <= d.nr && q >= 1 && q <= d.nc) {
        cl = C_INT;
        const uint8_t fl = d.flags[sprev + gi];
        if (fl & FX_F_WALL) cl |= C_WALL;
        if (melt_on && !(fl & FX_F_NODATA)) fx_dd_add(eta, lo, melt32(d, c, d.melt_mult_f ? d.melt_mult_f[gi] : 1.0f));
        if (is_inflow(d, r, q)) inflow_eta(eta, lo, c.inflowi);
        if (fx_dd_val(eta, lo) <= d.hdry) {
          qx = 0.f;
          qy = 0.f;
          cl |= C_DRY;
        }
      }
    }
    S.eta[k] = eta;
    S.eta_lo[k] = lo;
    S.zb[k] = zb;
    S.qx[k] = qx;
    S.qy[k] = qy;
    S.cls[k] = cl;
      {
        const float den = fmaxf(fmaxf(fmaxf(0.0f, eta), (float)d.hdry), (cl & C_INT) ? (float)d.ks : 0.0f);
        S.u[k] = fdiv(qx, den);
        S.v[k] = fdiv(qy, den);
      }
  }
  // the stencil is complete; a thread whose stage wait gave up (bad) stops
  // the whole block here, before anything is written to global memory
  if (__syncthreads_or(bad)) return false;
  {
    // Each thread computes its own face-flux cell (NFLUX == NTHREADS), wet,
    // dry or kept, without the FP64 path's work lists: in FP32 the lists'
    // gathering cost more than the divergence they avoid (4096^2 wet start
    // 1.4 % and the 64-scenario batch 6 % faster without them).
    const int k = tid;
    const int fr = k % FXN, fc = k / FXN;
    const int sr = fr + 1, scc = fc + 1;
    const unsigned char cl = S.cls[sidx(sr, scc)];
    float o[6];
    if (!(cl & C_INT) || (cl & C_WALL)) {
      for (int j = 0; j < 6; ++j) S.f[j][k] = 0.0f;
    } else if (cl & C_DRY) {
      const bool alldry = (S.cls[sidx(sr - 1, scc)] & C_DRY) && (S.cls[sidx(sr + 1, scc)] & C_DRY) &&
                          (S.cls[sidx(sr, scc - 1)] & C_DRY) && (S.cls[sidx(sr, scc + 1)] & C_DRY);
      if (alldry) {  // all five cells dry: the last computed fluxes stay (solver_drydomain.cpp:60-76)
        const long long gi = fx_ix(d, irow0 - 1 + fr, icol0 - 1 + fc);
        const float* rp = fx_rec(d, sprev + gi);
        S.f[0][k] = rp[FX_R_FE1];
        S.f[1][k] = d.fe2_f[gi];
        S.f[2][k] = d.fe3_f[gi];
        S.f[3][k] = rp[FX_R_FN1];
        S.f[4][k] = d.fn2_f[gi];
        S.f[5][k] = d.fn3_f[gi];
      } else {
        solver_dry32(d, S, sr, scc, irow0 - 1 + fr, icol0 - 1 + fc, dtl, o);
        for (int j = 0; j < 6; ++j) S.f[j][k] = o[j];
      }
    } else {
      solver_wet32(d, S, sr, scc, irow0 - 1 + fr, icol0 - 1 + fc, dtl, o);
      for (int j = 0; j < 6; ++j) S.f[j][k] = o[j];
    }
  }
  __syncthreads();
  if (own) {
    const long long gi = fx_ix(d, irow, icol);
    const int sP = sidx(lx + 2, ly + 2);
    const int fP = (ly + 1) * FXN + (lx + 1), fW = (ly + 1) * FXN + lx, fS = ly * FXN + (lx + 1);
    const unsigned char cl = S.cls[sP];
    const bool wall = cl & C_WALL;
    const int i4 = (ly + 2) * STG_W4 + lx + 2 + so.o4;
    const uint8_t fl = stg ? stg[L::O_FL + (ly + 2) * STG_W1 + lx + 2 + so.o1] : d.flags[sprev + gi];
    const float eta1 = S.eta[sP];
    const float etapre = stg ? reinterpret_cast<const float*>(stg + L::O_Z)[i4] : d.eta[pprev + gi];
    float h0v = fmaxf(0.0f, etapre);
    double mi = 0.0;
    float hpv = 0.0f, miv = 0.0f;  // the record's pre-melt depth and melt depth
    if (melt_on && !(fl & FX_F_NODATA)) {
      h0v = fmaxf(eta1, 0.0f);
      hpv = fmaxf(etapre, 0.0f);
      const float mm = !d.melt_mult_f ? 1.0f
                       : (stg ? reinterpret_cast<const float*>(stg + L::O_MM)[i4] : d.melt_mult_f[gi]);
      miv = melt32(d, c, mm);
      mi = (double)miv;
      bmelt = mi * d.arbase;
    }
    if (is_inflow(d, irow, icol)) {  // common.cpp:300-315 (h0 = the depth after the inflow)
      float em = etapre, lm = stg ? reinterpret_cast<const float*>(stg + L::O_LO)[i4] : d.eta_lo[pprev + gi];
      if (melt_on && !(fl & FX_F_NODATA)) fx_dd_add(em, lm, (float)mi);
      const double dm = fx_dd_val(em, lm);
      record_inflow_hm(d, c, fmax(dm, 0.0));
      bmelt += (fx_dd_val(eta1, S.eta_lo[sP]) - dm) * d.arbase;
      h0v = fmaxf(eta1, 0.0f);
    }
    if (!(cl & C_DRY)) d.twet_f[gi] += (float)c.twet_inc;
    float dh = 0.f, dqx = 0.f, dqy = 0.f, qxfP = 0.f, qyfP = 0.f;
    if (!wall) {
      dh = (div_dxy_f(d, S.f[0][fW] - S.f[0][fP]) + div_dxy_f(d, S.f[3][fS] - S.f[3][fP])) * dtl;
      dqx = (div_dxy_f(d, S.f[1][fW] - S.f[1][fP]) + div_dxy_f(d, S.f[4][fS] - S.f[4][fP])) * dtl;
      dqy = (div_dxy_f(d, S.f[2][fW] - S.f[2][fP]) + div_dxy_f(d, S.f[5][fS] - S.f[5][fP])) * dtl;
      qxfP = S.f[0][fP] * dtl;
      qyfP = S.f[3][fP] * dtl;
      const unsigned char clE = S.cls[sidx(lx + 3, ly + 2)], clN = S.cls[sidx(lx + 2, ly + 3)];
      if (irow == d.nr || (clE & C_WALL)) bout += (double)S.f[0][fP] * d.dxy * c.dtfl;
      if (icol == d.nc || (clN & C_WALL)) bout += (double)S.f[3][fP] * d.dxy * c.dtfl;
    }
    const unsigned char clW = S.cls[sidx(lx + 1, ly + 2)], clS = S.cls[sidx(lx + 2, ly + 1)];
    const float qxfW = ((clW & C_INT) && !(clW & C_WALL)) ? S.f[0][fW] * dtl : 0.0f;
    const float qyfS = ((clS & C_INT) && !(clS & C_WALL)) ? S.f[3][fS] * dtl : 0.0f;
    float eta = eta1, lo = S.eta_lo[sP];
    fx_dd_add(eta, lo, dh);
    const float h = fmaxf(0.0f, eta);
    const double depth = fx_dd_val(eta, lo);
    float qx, qy;
    uint8_t ld;
    if (depth < d.hdry || wall) {
      qx = qy = 0.0f;
      ld = 1;
    } else {
      qx = S.qx[sP] + dqx;
      qy = S.qy[sP] + dqy;
      qx = .1f * qxfW + .8f * qx + .1f * qxfP;
      qy = .1f * qyfS + .8f * qy + .1f * qyfP;
      ld = 0;
    }
    if (d.manning_f && ld == 0 && !wall) {
      const float n = d.manning_f[gi];
      if (n != 0.0f) {
        const float qm = fsqrt(qx * qx + qy * qy);
        const float den = 1.0f + fdiv(dtl * (float)d.gaccl * n * n * qm, h * h * fcbrt(h));
        const float rden = frcp(den);
        qx = qx * rden;
        qy = qy * rden;
      }
    }
    d.eta[pcur + gi] = eta;
    d.eta_lo[pcur + gi] = lo;
    d.qx_f[pcur + gi] = qx;
    d.qy_f[pcur + gi] = qy;
    const uint8_t fl1 = (fl & (FX_F_WALL | FX_F_NODATA)) | ((fl & FX_F_LDRY) ? FX_F_LDRY_PREV : 0) | ld;
    d.flags[scur + gi] = fl1;
    float fe1v = 0.0f, fn1v = 0.0f;
    if ((cl & C_INT) && !wall) {
      const bool computed =
          !(cl & C_DRY) || !((S.cls[sidx(lx + 1, ly + 2)] & C_DRY) && (S.cls[sidx(lx + 3, ly + 2)] & C_DRY) &&
                             (S.cls[sidx(lx + 2, ly + 1)] & C_DRY) && (S.cls[sidx(lx + 2, ly + 3)] & C_DRY));
      fe1v = S.f[0][fP];
      fn1v = S.f[3][fP];
      if (computed && (d.store_all_fluxes || !(depth > d.hdry))) {
        d.fe2_f[gi] = S.f[1][fP];
        d.fe3_f[gi] = S.f[2][fP];
        d.fn2_f[gi] = S.f[4][fP];
        d.fn3_f[gi] = S.f[5][fP];
      }
    }
    put_rec32(d, scur + gi, h0v, h, hpv, miv, fe1v, fn1v, fl1);
    courant_cell32(d, fmax(0.0, depth), qx, qy, dtc, hm);
  }
  acc.add(dtc, hm, bmelt, bout);
  return true;
}

// The FP64 step of one tile (the reference's arithmetic, bit for bit).
template <int BY>
__device__ __forceinline__ bool hydro_tile64(const fx_dev& d, const StepCtl& c, const fx_tile& tile,
                                             HydroSmem<BY>& S, TilePart& acc, const unsigned char* stg = nullptr,
                                             int bad = 0) {
  using L = StageLayout<false, BY>;
  const StageOff so = stage_off(tile.bx);
  constexpr int TY = Tile<BY>::TY, NSTEN = Tile<BY>::NSTEN, NFLUX = Tile<BY>::NFLUX;
  constexpr int NTHREADS = Tile<BY>::NTHREADS;
  const int lx = threadIdx.x, ly = threadIdx.y;
  const int tid = ly * BX + lx;
  const int irow0 = 1 + tile.bx * TX, icol0 = 1 + tile.by * TY;
  const int irow = irow0 + lx, icol = icol0 + ly;
  const bool own = lx < TX && ly < TY && irow <= d.nr && icol <= d.nc;
  const double dtl = c.dtfl;
  const bool melt_on = d.has_meteo != 0;

  // Slot planes: the state after the previous step, and the one this step
  // writes (h, h0, fe_1, fn_1, flags), and the two planes of z, qx, qy (see
  // fx_common.cuh): every block reads the previous step's plane, halo
  // included, and writes the other.
  const long long sprev = fx_slot(d, c.steps - 1), scur = fx_slot(d, c.steps);
  const long long pprev = fx_pp(d, c.steps - 1), pcur = fx_pp(d, c.steps);

  if (!c.active) {
    // No wet cell: the step is the Courant scan plus add_meteo only
    // (main.cpp:300-370, the solver block at :385 is skipped). The solute
    // dilution of add_meteo is applied by the ADE sweep (fx_ade.cu).
    double dtc = __longlong_as_double(0x7ff0000000000000LL), hm = 0.0, bmelt = 0.0;
    if (own) {
      const long long gi = fx_ix(d, irow, icol);
      const double zb = d.zb[gi], zpre = d.z[pprev + gi];
      const uint8_t fl = d.flags[sprev + gi];
      const double hpre = fmax(0.0, zpre - zb);
      uint8_t ld = hpre > d.hdry ? 0 : 1;  // Courant scan (:308-320)
      double z1 = zpre, h1 = hpre, hpv = 0.0;
      if (melt_on && zb != d.nodata) {
        const double mi = melt_depth(d, c, gi);
        bmelt = mi * d.arbase;
        hpv = fmax(zpre - zb, 0.0);  // the dilution's hp (common.cpp:216)
        z1 = zpre + mi;
        h1 = fmax(z1 - zb, 0.0);
        if (h1 <= d.hdry) ld = 0;  // common.cpp:219-222
      }
      if (is_inflow(d, irow, icol)) {  // common.cpp:300-315
        const double zm = z1;
        record_inflow_hm(d, c, fmax(zm - zb, 0.0));
        z1 = inflow_z(z1, zb, c.inflowi);
        h1 = fmax(z1 - zb, 0.0);
        ld = h1 <= d.hdry ? 1 : 0;
        bmelt += (z1 - zm) * d.arbase;
      }
      const double qx = d.qx[pprev + gi], qy = d.qy[pprev + gi];
      d.z[pcur + gi] = z1;
      d.qx[pcur + gi] = qx;
      d.qy[pcur + gi] = qy;
      const uint8_t fl1 = (fl & (FX_F_WALL | FX_F_NODATA)) | ((fl & FX_F_LDRY) ? FX_F_LDRY_PREV : 0) | ld;
      d.flags[scur + gi] = fl1;
      const double* rp = fx_rec64(d, sprev + gi);  // fluxes are unchanged by a step without solver
      put_rec64(d, scur + gi, h1, h1, hpv, rp[FX_R64_FE1], rp[FX_R64_FN1], fl1);
      courant_cell(d, h1, qx, qy, dtc, hm);
    }
    acc.add(dtc, hm, bmelt, 0.0);
    return true;
  }

  // ---- phase A: stencil load, melt, Loop 1 ---------------------------------
  if (tid == 0) {
    S.nwet = 0;
    S.ndry = 0;
    S.nstale = 0;
  }
  if (stg) {
    // staged by TMA: the same values, read from shared memory
    const double* g_z = reinterpret_cast<const double*>(stg + L::O_Z);
    const double* g_zb = reinterpret_cast<const double*>(stg + L::O_ZB);
    const double* g_qx = reinterpret_cast<const double*>(stg + L::O_QX);
    const double* g_qy = reinterpret_cast<const double*>(stg + L::O_QY);
    const double* g_mm = reinterpret_cast<const double*>(stg + L::O_MM);
    const uint8_t* g_fl = stg + L::O_FL;
    for (int k = tid; k < NSTEN; k += NTHREADS) {
      const int sr = k % SX, sc = k / SX;
      const int r = irow0 - 2 + sr, q = icol0 - 2 + sc;
      const int i8 = sc * STG_W8 + sr + so.o8;
      double z = g_z[i8], qx = g_qx[i8], qy = g_qy[i8];
      const double zb = g_zb[i8];
      unsigned char cl = 0;
      if (r >= 1 && r <= d.nr && q >= 1 && q <= d.nc) {
        cl = C_INT;
        if (g_fl[sc * STG_W1 + sr + so.o1] & FX_F_WALL) cl |= C_WALL;
        if (melt_on && zb != d.nodata)
          z = z + (d.melt_mult ? (double)c.meteo_rate * g_mm[i8] / (1000. * 3600. * 24.) * c.dtfl : c.meteoi);
        if (is_inflow(d, r, q)) z = inflow_z(z, zb, c.inflowi);
        const double h1 = fmax(0.0, z - zb);
        if (h1 <= d.hdry) {
          qx = 0.0;
          qy = 0.0;
          cl |= C_DRY;
        }
      }
      S.z[k] = z;
      S.zb[k] = zb;
      S.qx[k] = qx;
      S.qy[k] = qy;
      S.cls[k] = cl;
      if constexpr (HydroSmem<BY>::VEL) {
        const double den = fmax(fmax(fmax(0.0, z - zb), d.hdry), (cl & C_INT) ? d.ks : 0.0);
        S.u[k] = qx / den;
        S.v[k] = qy / den;
      }
    }
  } else
  for (int k = tid; k < NSTEN; k += NTHREADS) {
    const int sr = k % SX, sc = k / SX;
    const int r = irow0 - 2 + sr, q = icol0 - 2 + sc;
    double z = 0.0, zb = 0.0, qx = 0.0, qy = 0.0;
    unsigned char cl = 0;
    if (r >= 0 && r <= d.nr + 1 && q >= 0 && q <= d.nc + 1) {
      const long long gi = fx_ix(d, r, q);
      z = d.z[pprev + gi];
      zb = d.zb[gi];
      qx = d.qx[pprev + gi];
      qy = d.qy[pprev + gi];
      if (r >= 1 && r <= d.nr && q >= 1 && q <= d.nc) {
        cl = C_INT;
        if (d.flags[sprev + gi] & FX_F_WALL) cl |= C_WALL;
        if (melt_on && zb != d.nodata) z = z + melt_depth(d, c, gi);
        if (is_inflow(d, r, q)) z = inflow_z(z, zb, c.inflowi);
        const double h1 = fmax(0.0, z - zb);
        if (h1 <= d.hdry) {
          qx = 0.0;
          qy = 0.0;
          cl |= C_DRY;
        }
      }
    }
    S.z[k] = z;
    S.zb[k] = zb;
    S.qx[k] = qx;
    S.qy[k] = qy;
    S.cls[k] = cl;
    if constexpr (HydroSmem<BY>::VEL) {
      const double den = fmax(fmax(fmax(0.0, z - zb), d.hdry), (cl & C_INT) ? d.ks : 0.0);
      S.u[k] = qx / den;
      S.v[k] = qy / den;
    }
  }
  // the stencil is complete; a thread whose stage wait gave up (bad) stops
  // the whole block here, before anything is written to global memory
  if (__syncthreads_or(bad)) return false;

  // ---- phase B: classify flux cells into warp-uniform work lists ----------
  for (int k = tid; k < NFLUX; k += NTHREADS) {
    const int fr = k % FXN, fc = k / FXN;
    const int sr = fr + 1, sc = fc + 1;
    const unsigned char cl = S.cls[sidx(sr, sc)];
    if (!(cl & C_INT) || (cl & C_WALL)) {
      for (int j = 0; j < 6; ++j) S.f[j][k] = 0.0;  // never written in the reference
      continue;
    }
    if (cl & C_DRY) {
      const bool alldry = (S.cls[sidx(sr - 1, sc)] & C_DRY) && (S.cls[sidx(sr + 1, sc)] & C_DRY) &&
                          (S.cls[sidx(sr, sc - 1)] & C_DRY) && (S.cls[sidx(sr, sc + 1)] & C_DRY);
      if (alldry) S.stale_list[atomicAdd(&S.nstale, 1)] = (short)k;
      else S.dry_list[atomicAdd(&S.ndry, 1)] = (short)k;
    } else {
      S.wet_list[atomicAdd(&S.nwet, 1)] = (short)k;
    }
  }
  __syncthreads();

  // ---- phase C: face fluxes (each face once) -------------------------------
  {
    const int nwet = S.nwet, ndry = S.ndry, nstale = S.nstale;
    double o[6];
    for (int i = tid; i < nwet; i += NTHREADS) {
      const int k = S.wet_list[i];
      const int fr = k % FXN, fc = k / FXN;
      solver_wet(d, S, fr + 1, fc + 1, irow0 - 1 + fr, icol0 - 1 + fc, dtl, o);
      for (int j = 0; j < 6; ++j) S.f[j][k] = o[j];
    }
    for (int i = tid; i < ndry; i += NTHREADS) {
      const int k = S.dry_list[i];
      const int fr = k % FXN, fc = k / FXN;
      solver_dry(d, S, fr + 1, fc + 1, irow0 - 1 + fr, icol0 - 1 + fc, dtl, o);
      for (int j = 0; j < 6; ++j) S.f[j][k] = o[j];
    }
    // All five cells dry: the reference returns before storing
    // (solver_drydomain.cpp:60-76), so the fluxes of the last step that
    // computed them stay in effect.
    for (int i = tid; i < nstale; i += NTHREADS) {
      const int k = S.stale_list[i];
      const int fr = k % FXN, fc = k / FXN;
      const long long gi = fx_ix(d, irow0 - 1 + fr, icol0 - 1 + fc);
      const double* rp = fx_rec64(d, sprev + gi);
      S.f[0][k] = rp[FX_R64_FE1];
      S.f[1][k] = d.fe2[gi];
      S.f[2][k] = d.fe3[gi];
      S.f[3][k] = rp[FX_R64_FN1];
      S.f[4][k] = d.fn2[gi];
      S.f[5][k] = d.fn3[gi];
    }
  }
  __syncthreads();

  // ---- phase D: Loop 3, Loop 4, friction, store, next Courant --------------
  double dtc = __longlong_as_double(0x7ff0000000000000LL), hm = 0.0, bmelt = 0.0, bout = 0.0;
  if (own) {
    const long long gi = fx_ix(d, irow, icol);
    const int sP = sidx(lx + 2, ly + 2);
    const int fP = (ly + 1) * FXN + (lx + 1), fW = (ly + 1) * FXN + lx, fS = ly * FXN + (lx + 1);
    const unsigned char cl = S.cls[sP];
    const bool wall = cl & C_WALL;
    const int i8 = (ly + 2) * STG_W8 + lx + 2 + so.o8;
    const uint8_t fl = stg ? stg[L::O_FL + (ly + 2) * STG_W1 + lx + 2 + so.o1] : d.flags[sprev + gi];
    const double zb = S.zb[sP];
    const double z1 = S.z[sP];
    const double zpre = stg ? reinterpret_cast<const double*>(stg + L::O_Z)[i8] : d.z[pprev + gi];

    // add_meteo's h0 (common.cpp:223): the depth after the melt, or the
    // Courant scan's copy of h (main.cpp:305) for cells it skips. Its solute
    // dilution (:226-234) is applied by the ADE sweep (fx_ade.cu).
    double h0v = fmax(0.0, zpre - zb);
    double mi = 0.0, hpv = 0.0;
    if (melt_on && zb != d.nodata) {
      h0v = fmax(z1 - zb, 0.0);
      hpv = fmax(zpre - zb, 0.0);  // the dilution's hp (common.cpp:216)
      mi = (stg && d.melt_mult) ? (double)c.meteo_rate * reinterpret_cast<const double*>(stg + L::O_MM)[i8] /
                                      (1000. * 3600. * 24.) * c.dtfl
                                : melt_depth(d, c, gi);
      bmelt = mi * d.arbase;
    }
    if (is_inflow(d, irow, icol)) {  // common.cpp:300-315 (h0 = the depth after the inflow)
      const double zm = (melt_on && zb != d.nodata) ? zpre + mi : zpre;
      record_inflow_hm(d, c, fmax(zm - zb, 0.0));
      bmelt += (z1 - zm) * d.arbase;
      h0v = fmax(z1 - zb, 0.0);
    }
    // Loop 1 wet time (:69-70)
    if (!(cl & C_DRY)) d.twet[gi] += c.twet_inc;  // dtl / 3600

    // Loop 3 (:93-120)
    double dh = 0.0, dqx = 0.0, dqy = 0.0, qxfP = 0.0, qyfP = 0.0;
    if (!wall) {
      dh = (fx_div_dxy(d, S.f[0][fW] - S.f[0][fP]) + fx_div_dxy(d, S.f[3][fS] - S.f[3][fP])) * dtl;
      dqx = (fx_div_dxy(d, S.f[1][fW] - S.f[1][fP]) + fx_div_dxy(d, S.f[4][fS] - S.f[4][fP])) * dtl;
      dqy = (fx_div_dxy(d, S.f[2][fW] - S.f[2][fP]) + fx_div_dxy(d, S.f[5][fS] - S.f[5][fP])) * dtl;
      qxfP = S.f[0][fP] * dtl;
      qyfP = S.f[3][fP] * dtl;
    }
    const unsigned char clW = S.cls[sidx(lx + 1, ly + 2)], clS = S.cls[sidx(lx + 2, ly + 1)];
    if (!wall) {
      // water leaving the domain this step: through the outflow faces, and
      // into wall cells (which never take it up, hydrodynamics_calc.cpp:111-117)
      const unsigned char clE = S.cls[sidx(lx + 3, ly + 2)], clN = S.cls[sidx(lx + 2, ly + 3)];
      if (irow == d.nr || (clE & C_WALL)) bout += S.f[0][fP] * d.dxy * dtl;
      if (icol == d.nc || (clN & C_WALL)) bout += S.f[3][fP] * d.dxy * dtl;
    }
    const double qxfW = ((clW & C_INT) && !(clW & C_WALL)) ? S.f[0][fW] * dtl : 0.0;
    const double qyfS = ((clS & C_INT) && !(clS & C_WALL)) ? S.f[3][fS] * dtl : 0.0;

    // Loop 4 (:123-154)
    const double z = z1 + dh;
    const double h = fmax(0.0, z - zb);
    double qx, qy;
    uint8_t ld;
    if (h < d.hdry || wall) {
      qx = 0.0;
      qy = 0.0;
      ld = 1;
    } else {
      qx = S.qx[sP] + dqx;
      qy = S.qy[sP] + dqy;
      qx = .1 * qxfW + .8 * qx + .1 * qxfP;
      qy = .1 * qyfS + .8 * qy + .1 * qyfP;
      ld = 0;
    }
    // Extension: semi-implicit Manning friction (n = 0 leaves q unchanged).
    if (d.manning && ld == 0 && !wall) {
      const double n = d.manning[gi];
      if (n != 0.0) {
        const double qm = sqrt(qx * qx + qy * qy);
        const double h73 = h * h * fx_cbrt(h);
        const double den = 1.0 + dtl * d.gaccl * n * n * qm / h73;
        qx = qx / den;
        qy = qy / den;
      }
    }
    d.z[pcur + gi] = z;
    d.qx[pcur + gi] = qx;
    d.qy[pcur + gi] = qy;
    const uint8_t fl1 = (fl & (FX_F_WALL | FX_F_NODATA)) | ((fl & FX_F_LDRY) ? FX_F_LDRY_PREV : 0) | ld;
    d.flags[scur + gi] = fl1;
    // Fluxes computed this step become the grid values (stale ones are
    // already there). fe_2/fe_3/fn_2/fn_3 are read back only when this cell
    // is dry with four dry neighbours at a later solver step; a cell that
    // ends the step wet (h > hdry) is wet again at the next solver step as
    // long as forcing adds water, so those three-quarters of the flux
    // traffic are skipped for it.
    const unsigned char clP = cl;
    double fe1v = 0.0, fn1v = 0.0;
    if ((clP & C_INT) && !(clP & C_WALL)) {
      const bool computed =
          !(clP & C_DRY) || !((S.cls[sidx(lx + 1, ly + 2)] & C_DRY) && (S.cls[sidx(lx + 3, ly + 2)] & C_DRY) &&
                              (S.cls[sidx(lx + 2, ly + 1)] & C_DRY) && (S.cls[sidx(lx + 2, ly + 3)] & C_DRY));
      // fe_1/fn_1 of every cell go to this step's slot: computed ones, or the
      // stale ones carried over (already in S.f for stale cells).
      fe1v = S.f[0][fP];
      fn1v = S.f[3][fP];
      if (computed && (d.store_all_fluxes || !(h > d.hdry))) {
        d.fe2[gi] = S.f[1][fP];
        d.fe3[gi] = S.f[2][fP];
        d.fn2[gi] = S.f[4][fP];
        d.fn3[gi] = S.f[5][fP];
      }
    }  // walls: fe_1 = fn_1 = 0, never written in the reference
    put_rec64(d, scur + gi, h0v, h, hpv, fe1v, fn1v, fl1);
    courant_cell(d, h, qx, qy, dtc, hm);
  }
  acc.add(dtc, hm, bmelt, bout);
  return true;
}

// Reads the step's fields of the control block (written by k_finalize) into
// shared memory, then runs the tile in the domain's precision.
template <bool P32, int BY>
__device__ __forceinline__ void hydro_block(const fx_dev& d, const fx_tile& tile, HydroSmem<BY>& S,
                                            StepCtl& sc) {
  static_assert(sizeof(HydroSmem32<BY>) <= sizeof(HydroSmem<BY>), "FP32 tile state reuses the FP64 one");
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    const fx_ctl& g = *d.ctl;
    sc.dtfl = g.dtfl;
    sc.meteoi = g.meteoi;
    sc.meteo_rate = g.meteo_rate;
    sc.mconc = g.mconc;
    sc.inflowi = g.inflowi;
    sc.twet_inc = g.dtfl / 3600;
    sc.steps = g.steps;
    sc.live = g.live;
    sc.active = g.active;
  }
  __syncthreads();
  const StepCtl c = sc;
  if (!c.live) return;
  TilePart acc = tile_part();
  if constexpr (P32) hydro_tile32<BY>(d, c, tile, *reinterpret_cast<HydroSmem32<BY>*>(&S), acc);
  else hydro_tile64<BY>(d, c, tile, S, acc);
  reduce_part(d, S, acc);
}

// Blocks per SM the launch bounds ask for: 768 threads for FP64 (at most 85
// registers each), 1024 for FP32 (at most 64). The kernel is bound by
// instruction latency and tile barriers, so resident warps pay for the
// spills this costs: at 4096 x 4096 cells the FP32 kernel took 1.50 ms per
// step at 64 registers against 1.73 ms at 80 (3 blocks), the FP64 one 4.01
// ms at 85 against 4.39 ms at 128 (2 blocks).
template <bool P32, int BY>
constexpr int min_blocks() { return (P32 ? 32 : 24) / BY > 0 ? (P32 ? 32 : 24) / BY : 1; }

// One domain: the descriptor is a kernel parameter (constant bank), so its
// fields are instruction operands. Block (x, y) is tile (x, y).
template <bool P32, int BY>
__global__ void __launch_bounds__(BX * BY, min_blocks<P32, BY>()) k_hydro_one(const __grid_constant__ fx_dev d) {
  __shared__ HydroSmem<BY> S;
  __shared__ StepCtl sc;
  const fx_tile tile{0, (int)blockIdx.x, (int)blockIdx.y, 0};
  hydro_block<P32, BY>(d, tile, S, sc);
}

// A batch of domains: one block per entry of the tile table; the block copies
// its domain's descriptor to shared memory.
template <bool P32, int BY>
__global__ void __launch_bounds__(BX * BY, min_blocks<P32, BY>()) k_hydro_batch(const fx_dev* __restrict__ devs,
                                                                        const fx_tile* __restrict__ tiles) {
  __shared__ HydroSmem<BY> S;
  __shared__ fx_dev sd;
  __shared__ StepCtl sc;
  const fx_tile tile = tiles[blockIdx.x];
  {
    const int tid = threadIdx.y * BX + threadIdx.x;
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(devs + tile.dom);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sd);
    for (int i = tid; i < (int)(sizeof(fx_dev) / 8); i += BX * BY) dst[i] = src[i];
  }
  __syncthreads();
  hydro_block<P32, BY>(sd, tile, S, sc);
}
static_assert(sizeof(fx_dev) % 8 == 0, "descriptor copied as 8-byte words");

// ---- TMA-staged persistent form -------------------------------------------
// One block per SM slot loops over the domain's tiles. Thread 0 loads the
// stencil of the block's next tile into the other of two shared-memory
// stages with TMA (cp.async.bulk.tensor, completion counted on an mbarrier)
// while the block computes the current one, so the halo reads of a tile
// overlap the arithmetic of the previous tile.

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const void* map, int x, int y, int z,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Issue the loads of tile t's stencil into stage `stg` (thread 0).
template <bool P32, int BY>
__device__ __forceinline__ void stage_issue(const fx_dev& d, const fx_tmaps& tm, int t, int ntx, long long step_prev,
                                            unsigned char* stg, unsigned long long* bar) {
  using L = StageLayout<P32, BY>;
  const int bx = t % ntx, by = t / ntx;
  const int x = TX * bx, y = (BY - 1) * by - 1;  // stencil origin (irow0 - 2 + FX_ROFF, icol0 - 2)
  const int x4 = x & ~3, x8 = x & ~1, x1 = x & ~15;
  const int pp = (int)(step_prev & 1), sl = (int)(step_prev % d.nslot);
  const bool mm = P32 ? d.melt_mult_f != nullptr : d.melt_mult != nullptr;
  const unsigned bytes = (unsigned)((P32 ? 4 * STG_W4 * L::SY * 4 + STG_W8 * L::SY * 8
                                         : 4 * STG_W8 * L::SY * 8) +
                                    (mm ? (P32 ? STG_W4 * L::SY * 4 : STG_W8 * L::SY * 8) : 0) + STG_W1 * L::SY);
  mbar_expect_tx(bar, bytes);
  if (P32) {
    tma_load_3d(stg + L::O_Z, &tm.m[FX_TM_Z], x4, y, pp, bar);
    tma_load_3d(stg + L::O_LO, &tm.m[FX_TM_LO], x4, y, pp, bar);
    tma_load_3d(stg + L::O_ZB, &tm.m[FX_TM_ZB], x8, y, 0, bar);
    tma_load_3d(stg + L::O_QX, &tm.m[FX_TM_QX], x4, y, pp, bar);
    tma_load_3d(stg + L::O_QY, &tm.m[FX_TM_QY], x4, y, pp, bar);
    if (mm) tma_load_3d(stg + L::O_MM, &tm.m[FX_TM_MM], x4, y, 0, bar);
  } else {
    tma_load_3d(stg + L::O_Z, &tm.m[FX_TM_Z], x8, y, pp, bar);
    tma_load_3d(stg + L::O_ZB, &tm.m[FX_TM_ZB], x8, y, 0, bar);
    tma_load_3d(stg + L::O_QX, &tm.m[FX_TM_QX], x8, y, pp, bar);
    tma_load_3d(stg + L::O_QY, &tm.m[FX_TM_QY], x8, y, pp, bar);
    if (mm) tma_load_3d(stg + L::O_MM, &tm.m[FX_TM_MM], x8, y, 0, bar);
  }
  tma_load_3d(stg + L::O_FL, &tm.m[FX_TM_FL], x1, y, sl, bar);
}

constexpr long long STAGE_SPIN_LIMIT = 1LL << 22;  // polls of a stage's mbarrier before giving up

template <bool P32, int BY>
__global__ void __launch_bounds__(BX * BY, min_blocks<P32, BY>())
    k_hydro_tma(const __grid_constant__ fx_dev d, const __grid_constant__ fx_tmaps tm, int ntx, int nty) {
  using L = StageLayout<P32, BY>;
  __shared__ HydroSmem<BY> S;
  __shared__ StepCtl sc;
  __shared__ __align__(8) unsigned long long bar[2];
  extern __shared__ __align__(128) unsigned char dyn[];
  unsigned char* stage0 = dyn + ((128 - (smem_u32(dyn) & 127)) & 127);
  const int tid = threadIdx.y * BX + threadIdx.x;
  const int ntiles = ntx * nty;
  if (tid == 0) {
    const fx_ctl& g = *d.ctl;
    sc.dtfl = g.dtfl;
    sc.meteoi = g.meteoi;
    sc.meteo_rate = g.meteo_rate;
    sc.mconc = g.mconc;
    sc.inflowi = g.inflowi;
    sc.twet_inc = g.dtfl / 3600;
    sc.steps = g.steps;
    sc.live = g.live;
    sc.active = g.active;
  }
  __syncthreads();
  const StepCtl c = sc;
  if (!c.live) return;
  TilePart acc = tile_part();
  if (!c.active) {  // no solver this step: cell-local work only, nothing to stage
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      const fx_tile tile{0, t % ntx, t / ntx, 0};
      if constexpr (P32) hydro_tile32<BY>(d, c, tile, *reinterpret_cast<HydroSmem32<BY>*>(&S), acc);
      else hydro_tile64<BY>(d, c, tile, S, acc);
      __syncthreads();
    }
    reduce_part(d, S, acc);
    return;
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (blockIdx.x < ntiles) stage_issue<P32, BY>(d, tm, blockIdx.x, ntx, c.steps - 1, stage0, &bar[0]);
  }
  __syncthreads();
  unsigned parity = 0u;  // bit q: phase of stage q's barrier
  int st = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int tn = t + gridDim.x;
    if (tid == 0 && tn < ntiles)
      stage_issue<P32, BY>(d, tm, tn, ntx, c.steps - 1, stage0 + (st ^ 1) * L::BYTES, &bar[st ^ 1]);
    // wait for this tile's stencil, bounded; each thread waits for itself,
    // and the tile's first barrier (after the stencil is read) tells the
    // whole block whether any wait gave up
    long long it = 0;
    int bad = 0;
    while (!mbar_try_wait(&bar[st], (parity >> st) & 1u)) {
      if (++it > STAGE_SPIN_LIMIT) {
        bad = 1;
        break;
      }
    }
    parity ^= 1u << st;
    const fx_tile tile{0, t % ntx, t / ntx, 0};
    bool done;
    if constexpr (P32)
      done = hydro_tile32<BY>(d, c, tile, *reinterpret_cast<HydroSmem32<BY>*>(&S), acc, stage0 + st * L::BYTES, bad);
    else done = hydro_tile64<BY>(d, c, tile, S, acc, stage0 + st * L::BYTES, bad);
    if (!done) {  // every thread of the block takes this branch
      if (tid == 0) {
        atomicCAS(&d.ctl->error, 0, FX_DEVERR_WAIT_TIMEOUT);
        // let the copy of the next tile, if one was issued, land before the block exits
        long long w = 0;
        if (tn < ntiles)
          while (!mbar_try_wait(&bar[st ^ 1], (parity >> (st ^ 1)) & 1u) && ++w < STAGE_SPIN_LIMIT) {
          }
      }
      return;
    }
    __syncthreads();  // the stage is free for the load issued two tiles later
    st ^= 1;
  }
  reduce_part(d, S, acc);
}

// ---- TMA-staged persistent form for a batch --------------------------------
// Each block walks a contiguous range of the packed tile table of all the
// batch's domains (so it crosses few domain boundaries). Thread 0 stages the
// stencil of the block's next tile with that domain's own tensor maps (a
// device array, one set per domain) while the block computes the current
// tile; a domain without a solver step this launch (stopped, or no wet cell)
// gets no stage. The domain's descriptor and step fields sit in shared
// memory while the block works on its tiles, and the block's Courant and
// budget partials go to a domain when the block leaves it.

// Thread 0: stage tile t of the table into `stg` if its domain runs the
// solver this step; returns whether a copy was issued.
template <bool P32, int BY>
__device__ __forceinline__ bool batch_stage(const fx_dev* __restrict__ devs, const fx_tmaps* __restrict__ tms,
                                            const fx_tile* __restrict__ tiles, int t, unsigned char* stg,
                                            unsigned long long* bar, int& fenced) {
  const fx_tile tl = tiles[t];
  const fx_dev& dm = devs[tl.dom];
  const fx_ctl& g = *dm.ctl;
  if (!g.live || !g.active) return false;
  const fx_tmaps& tm = tms[tl.dom];
  if (fenced != tl.dom) {
    // the maps were written by a host copy before the launch; order the
    // tensor-map proxy's reads of a domain's maps after it, once per domain
    for (int f = 0; f < FX_TM_COUNT; ++f)
      asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&tm.m[f]) : "memory");
    fenced = tl.dom;
  }
  const int ntx = (dm.nr + TX - 1) / TX;
  stage_issue<P32, BY>(dm, tm, tl.by * ntx + tl.bx, ntx, g.steps - 1, stg, bar);
  return true;
}

template <bool P32, int BY>
__global__ void __launch_bounds__(BX * BY, min_blocks<P32, BY>())
    k_hydro_batch_tma(const fx_dev* __restrict__ devs, const fx_tmaps* __restrict__ tms,
                      const fx_tile* __restrict__ tiles, int ntiles) {
  using L = StageLayout<P32, BY>;
  __shared__ HydroSmem<BY> S;
  __shared__ fx_dev sd;
  __shared__ StepCtl sc;
  __shared__ __align__(8) unsigned long long bar[2];
  __shared__ int staged[2];  // the tile each stage holds (-1: none)
  __shared__ int abort_flag;
  extern __shared__ __align__(128) unsigned char dyn[];
  unsigned char* stage0 = dyn + ((128 - (smem_u32(dyn) & 127)) & 127);
  const int tid = threadIdx.y * BX + threadIdx.x;
  const int t0 = (int)((long long)ntiles * blockIdx.x / gridDim.x);
  const int t1 = (int)((long long)ntiles * (blockIdx.x + 1) / gridDim.x);
  if (t0 >= t1) return;
  int fenced = -1;  // thread 0: the domain whose maps it last fenced
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
    staged[0] = batch_stage<P32, BY>(devs, tms, tiles, t0, stage0, &bar[0], fenced) ? t0 : -1;
    staged[1] = -1;
  }
  __syncthreads();
  unsigned parity = 0u;  // bit q: phase of stage q's barrier
  int st = 0, dom = -1;
  TilePart acc = tile_part();
  for (int t = t0; t < t1; ++t) {
    const fx_tile tl = tiles[t];
    if (tl.dom != dom) {
      if (dom >= 0) reduce_part(sd, S, acc);  // the partials of the domain the block leaves
      acc = tile_part();
      __syncthreads();
      const unsigned long long* src = reinterpret_cast<const unsigned long long*>(devs + tl.dom);
      unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sd);
      for (int i = tid; i < (int)(sizeof(fx_dev) / 8); i += BX * BY) dst[i] = src[i];
      __syncthreads();
      if (tid == 0) {
        const fx_ctl& g = *sd.ctl;
        sc.dtfl = g.dtfl;
        sc.meteoi = g.meteoi;
        sc.meteo_rate = g.meteo_rate;
        sc.mconc = g.mconc;
        sc.inflowi = g.inflowi;
        sc.twet_inc = g.dtfl / 3600;
        sc.steps = g.steps;
        sc.live = g.live;
        sc.active = g.active;
      }
      __syncthreads();
      dom = tl.dom;
    }
    if (tid == 0)
      staged[st ^ 1] = (t + 1 < t1 && batch_stage<P32, BY>(devs, tms, tiles, t + 1, stage0 + (st ^ 1) * L::BYTES,
                                                           &bar[st ^ 1], fenced))
                           ? t + 1 : -1;
    const bool mine = staged[st] == t;  // this tile's stencil is (being) staged
    if (mine) {
      long long it = 0;
      while (!mbar_try_wait(&bar[st], (parity >> st) & 1u)) {
        if (++it > STAGE_SPIN_LIMIT) {
          abort_flag = 1;
          break;
        }
      }
      parity ^= 1u << st;
    }
    __syncthreads();
    if (abort_flag) {
      if (tid == 0) {
        atomicCAS(&sd.ctl->error, 0, FX_DEVERR_WAIT_TIMEOUT);
        long long w = 0;  // let a copy already issued for the next tile land before the block exits
        if (staged[st ^ 1] >= 0)
          while (!mbar_try_wait(&bar[st ^ 1], (parity >> (st ^ 1)) & 1u) && ++w < STAGE_SPIN_LIMIT) {
          }
      }
      return;
    }
    const StepCtl c = sc;
    if (c.live) {
      const fx_tile tile{0, tl.bx, tl.by, 0};
      const unsigned char* stg = mine ? stage0 + st * L::BYTES : nullptr;
      if constexpr (P32) hydro_tile32<BY>(sd, c, tile, *reinterpret_cast<HydroSmem32<BY>*>(&S), acc, stg);
      else hydro_tile64<BY>(sd, c, tile, S, acc, stg);
    }
    __syncthreads();  // the stage is free for the copy issued next iteration
    st ^= 1;
  }
  if (dom >= 0) reduce_part(sd, S, acc);
}

// Courant scan of the state as uploaded (the scan at the top of the first
// step). Also used after a host edit of the state.
template <int BY>
__global__ void __launch_bounds__(BX * BY) k_courant_scan(const fx_dev* __restrict__ devs,
                                                         const fx_tile* __restrict__ tiles) {
  constexpr int TY = Tile<BY>::TY;
  __shared__ HydroSmem<BY> S;
  __shared__ fx_dev sd;
  const fx_tile tile = tiles[blockIdx.x];
  if (threadIdx.x == 0 && threadIdx.y == 0) sd = devs[tile.dom];
  __syncthreads();
  const fx_dev& d = sd;
  const int irow = 1 + tile.bx * TX + threadIdx.x, icol = 1 + tile.by * TY + threadIdx.y;
  double dtc = __longlong_as_double(0x7ff0000000000000LL), hm = 0.0;
  if (threadIdx.x < TX && threadIdx.y < TY && irow <= d.nr && icol <= d.nc) {
    const long long gi = fx_ix(d, irow, icol);
    const long long sl = fx_slot(d, d.ctl->steps), pl = fx_pp(d, d.ctl->steps);
    if (d.prec32)
      courant_cell32(d, fmax(0.0, fx_dd_val(d.eta[pl + gi], d.eta_lo[pl + gi])), d.qx_f[pl + gi],
                     d.qy_f[pl + gi], dtc, hm);
    else
      courant_cell(d, fx_rec64(d, sl + gi)[FX_R64_H], d.qx[pl + gi], d.qy[pl + gi], dtc, hm);
  }
  reduce_courant(d, S, dtc, hm);
}

// First row a (0-based) of the forcing table with t[a] > tim
// (common.cpp:195-200). Returns -1 when no row qualifies.
__device__ int forcing_row(const float* t, double tim) {
  for (int a = 0; a < FX_METEO_ROWS; ++a)
    if (t[a] > tim) return a;
  return -1;
}

// The clock update of one step, one thread per domain (main.cpp:271-325 and
// common.cpp:195-208).
__global__ void k_finalize(const fx_dev* __restrict__ devs, int ndom) {
  const int dom = blockIdx.x * blockDim.x + threadIdx.x;
  if (dom >= ndom) return;
  const fx_dev& d = devs[dom];
  fx_ctl& c = *d.ctl;
  c.live = 0;
  if (c.error || c.print_pending || c.finished || c.steps >= c.stop_after) return;
  if (!(c.tim <= c.ntim)) {
    c.finished = 1;
    return;
  }
  const double dtmin = __longlong_as_double((long long)c.acc_dtmin);
  const double hpall = __longlong_as_double((long long)c.acc_hmax);
  double dt = fmin(9.e10, dtmin);
  dt = fmin(c.print_next - c.tim, dt);
  c.dtfl = dt;
  c.hpall = hpall;
  c.tim = c.tim + dt;
  if (d.has_meteo) {
    int row = forcing_row(d.meteo_t, c.tim);
    if (row < 0) {
      c.forcing_overrun = 1;
      row = FX_METEO_ROWS - 1;
    }
    c.meteo_rate = (double)d.meteo_r[row];
    c.meteoi = (double)d.meteo_r[row] / (1000. * 3600. * 24.) * dt;
    c.mconc = (double)d.meteo_c[row];
  } else {
    c.meteo_rate = 0.0;
    c.meteoi = 0.0;
    c.mconc = 0.0;
  }
  if (d.has_inflow) {  // common.cpp:300-311; table rows from 0 (read_functions.cpp:311)
    int row = forcing_row(d.inflow_t, c.tim);
    if (row < 0) {
      c.forcing_overrun = 1;
      row = FX_METEO_ROWS - 1;
    }
    c.inflowi = (double)d.inflow_r[row] * dt / d.arbase;  // / pow(dxy, 2), exact
    c.iconc = (double)d.inflow_c[row];
  } else {
    c.inflowi = 0.0;
    c.iconc = 0.0;
  }
  c.active = hpall != 0.0;
  if (c.active) c.it = c.it + 1;
  c.print_pending = c.tim >= c.print_next;
  c.steps = c.steps + 1;
  fx_steprec& r = c.rec[c.steps % d.nslot];
  r.dtfl = c.dtfl;
  r.meteoi = c.meteoi;
  r.meteo_rate = c.meteo_rate;
  r.mconc = c.mconc;
  r.inflowi = c.inflowi;
  r.iconc = c.iconc;
  r.inflow_hm = 0.0;
  r.step = c.steps;
  r.batch = c.batch;
  r.live = 1;
  r.active = c.active;
  r.it = c.it;
  c.acc_dtmin = (unsigned long long)__double_as_longlong(__longlong_as_double(0x7ff0000000000000LL));
  c.acc_hmax = 0ull;
  c.live = 1;
}

// Opens a batch of steps whose ADE sweeps run together (fx_ade.cu).
__global__ void k_batch_begin(const fx_dev* __restrict__ devs, int ndom) {
  const int dom = blockIdx.x * blockDim.x + threadIdx.x;
  if (dom < ndom) devs[dom].ctl->batch = devs[dom].ctl->batch + 1;
}

// Sets the bed flags that never change (NODATA bed) in every slot plane.
// One thread per 4 cells of a column (ld is a multiple of 32, so the 4 share
// the column): the four flags bytes of a slot move as one 32-bit word.
__global__ void k_mark_static(const fx_dev* __restrict__ devs, int dom) {
  const fx_dev& d = devs[dom];
  const long long i = 4 * (blockIdx.x * (long long)blockDim.x + threadIdx.x);
  if (i >= d.plane) return;
  const int icol = (int)(i / d.ld), irow0 = (int)(i - (long long)icol * d.ld) - FX_ROFF;
  if (icol < 1 || icol > d.nc) return;
  const double2 z01 = *reinterpret_cast<const double2*>(d.zb + i);
  const double2 z23 = *reinterpret_cast<const double2*>(d.zb + i + 2);
  const double zb[4] = {z01.x, z01.y, z23.x, z23.y};
  unsigned keep = 0xffffffffu, set = 0u;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int irow = irow0 + j;
    if (irow < 1 || irow > d.nr) continue;
    keep &= ~((unsigned)FX_F_NODATA << (8 * j));
    if (zb[j] == d.nodata) set |= (unsigned)FX_F_NODATA << (8 * j);
  }
  if (keep == 0xffffffffu) return;
  unsigned* f = reinterpret_cast<unsigned*>(d.flags + i);
  const long long step = d.plane / 4;
  for (int k = 0; k < d.nslot; ++k) f[k * step] = (f[k * step] & keep) | set;
}

// FP32 state: the compensated depth (eta, eta_lo) = z - zb over the whole
// grid (ghost ring included), from a staged FP64 z in the field layout, into
// both planes.
__global__ void k_eta_from_z(const __grid_constant__ fx_dev d, const double* __restrict__ z) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < d.plane;
       i += (long long)gridDim.x * blockDim.x) {
    const double depth = z[i] - d.zb[i];
    const float hi = (float)depth;
    d.eta[i] = d.eta[d.plane + i] = hi;
    d.eta_lo[i] = d.eta_lo[d.plane + i] = (float)(depth - (double)hi);
  }
}

// Stored water sum(z - zb) * dxy^2 over the interior cells that are not
// walls (the quantity the update conserves: a cell overdrawn by its
// neighbours' outflow holds a small negative depth until it refills, where h
// reads 0) and solute mass sum(c * h) * dxy^2, FP64 block sums added into
// out[0] and out[1 + k].
__global__ void __launch_bounds__(256) k_mass(const __grid_constant__ fx_dev d, double* __restrict__ out) {
  __shared__ double red[8][1 + FX_MAX_CHEM];
  const long long sl = fx_slot(d, d.ctl->steps), pl = fx_pp(d, d.ctl->steps);
  double acc[1 + FX_MAX_CHEM];
  for (int k = 0; k <= FX_MAX_CHEM; ++k) acc[k] = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < d.plane;
       i += (long long)gridDim.x * blockDim.x) {
    const int icol = (int)(i / d.ld), irow = (int)(i % d.ld) - FX_ROFF;
    if (irow < 1 || irow > d.nr || icol < 1 || icol > d.nc) continue;
    if (d.flags[sl + i] & FX_F_WALL) continue;
    const double h = d.prec32 ? (double)fx_rec(d, sl + i)[FX_R_H] : fx_rec64(d, sl + i)[FX_R64_H];
    acc[0] += d.prec32 ? fx_dd_val(d.eta[pl + i], d.eta_lo[pl + i]) : d.z[pl + i] - d.zb[i];
    for (int k = 0; k < d.nchem; ++k)
      acc[1 + k] += h * (d.prec32 ? (double)d.conc_f[k * d.plane + i] : d.conc[k * d.plane + i]);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int k = 0; k <= d.nchem; ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[w][k] = v;
  }
  __syncthreads();
  if (threadIdx.x <= d.nchem) {
    double v = 0.0;
    for (int j = 0; j < 8; ++j) v += red[j][threadIdx.x];
    atomicAdd(&out[threadIdx.x], v * d.arbase);
  }
}

}  // namespace fx

// Launch helpers used by fx_capi.cu and fx_batch.cu. `devs` is a device
// array of ndom domain descriptors; tile tables are built by fx_tiles_of.
void fx_launch_finalize(const fx_dev* devs, int ndom, cudaStream_t s) {
  fx::k_finalize<<<(ndom + 127) / 128, 128, 0, s>>>(devs, ndom);
}
void fx_launch_batch_begin(const fx_dev* devs, int ndom, cudaStream_t s) {
  fx::k_batch_begin<<<(ndom + 127) / 128, 128, 0, s>>>(devs, ndom);
}
void fx_launch_mark_static(const fx_dev* devs, int dom, long long plane, cudaStream_t s) {
  fx::k_mark_static<<<(unsigned)((plane / 4 + 255) / 256), 256, 0, s>>>(devs, dom);
}
namespace {
template <int BY>
void launch_hydro_batch(const fx_dev* devs, const fx_tile* tiles, int ntiles, bool prec32, cudaStream_t s) {
  if (prec32) fx::k_hydro_batch<true, BY><<<ntiles, dim3(fx::BX, BY), 0, s>>>(devs, tiles);
  else fx::k_hydro_batch<false, BY><<<ntiles, dim3(fx::BX, BY), 0, s>>>(devs, tiles);
}
template <int BY>
void launch_hydro_one(const fx_dev& d, cudaStream_t s) {
  const dim3 grid((d.nr + fx::TX - 1) / fx::TX, (d.nc + fx::Tile<BY>::TY - 1) / fx::Tile<BY>::TY);
  if (d.prec32) fx::k_hydro_one<true, BY><<<grid, dim3(fx::BX, BY), 0, s>>>(d);
  else fx::k_hydro_one<false, BY><<<grid, dim3(fx::BX, BY), 0, s>>>(d);
}
}  // namespace

bool fx_tile_rows_ok(int r) { return r == 4 || r == 8 || r == 16; }

void fx_launch_hydro(const fx_dev* devs, const fx_tile* tiles, int ntiles, bool prec32, int tile_rows,
                     cudaStream_t s) {
  if (tile_rows == 4) launch_hydro_batch<4>(devs, tiles, ntiles, prec32, s);
  else if (tile_rows == 16) launch_hydro_batch<16>(devs, tiles, ntiles, prec32, s);
  else launch_hydro_batch<8>(devs, tiles, ntiles, prec32, s);
}
void fx_launch_hydro_one(const fx_dev& d, cudaStream_t s) {
  if (d.tile_rows == 4) launch_hydro_one<4>(d, s);
  else if (d.tile_rows == 16) launch_hydro_one<16>(d, s);
  else launch_hydro_one<8>(d, s);
}
namespace {
template <int BY>
void launch_hydro_tma(const fx_dev& d, const fx_tmaps& tm, int nblocks, cudaStream_t s) {
  const int ntx = (d.nr + fx::TX - 1) / fx::TX, nty = (d.nc + fx::Tile<BY>::TY - 1) / fx::Tile<BY>::TY;
  const size_t dyn = (size_t)2 * (d.prec32 ? fx::StageLayout<true, BY>::BYTES : fx::StageLayout<false, BY>::BYTES) + 128;
  if (d.prec32) fx::k_hydro_tma<true, BY><<<nblocks, dim3(fx::BX, BY), dyn, s>>>(d, tm, ntx, nty);
  else fx::k_hydro_tma<false, BY><<<nblocks, dim3(fx::BX, BY), dyn, s>>>(d, tm, ntx, nty);
}
template <bool P32, int BY>
int tma_blocks(int* out) {
  const size_t dyn = (size_t)2 * fx::StageLayout<P32, BY>::BYTES + 128;
  if (cudaFuncSetAttribute(fx::k_hydro_tma<P32, BY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn) !=
      cudaSuccess)
    return -1;
  int dev = 0, nsm = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fx::k_hydro_tma<P32, BY>, fx::BX * BY, dyn) !=
      cudaSuccess)
    return -1;
  *out = per * nsm;
  return 0;
}
}  // namespace

namespace {
template <bool P32, int BY>
size_t batch_tma_dyn() { return (size_t)2 * fx::StageLayout<P32, BY>::BYTES + 128; }
template <int BY>
void launch_hydro_batch_tma(const fx_dev* devs, const fx_tmaps* tms, const fx_tile* tiles, int ntiles, int nblocks,
                            bool prec32, cudaStream_t s) {
  if (prec32)
    fx::k_hydro_batch_tma<true, BY><<<nblocks, dim3(fx::BX, BY), batch_tma_dyn<true, BY>(), s>>>(devs, tms, tiles,
                                                                                              ntiles);
  else
    fx::k_hydro_batch_tma<false, BY><<<nblocks, dim3(fx::BX, BY), batch_tma_dyn<false, BY>(), s>>>(devs, tms, tiles,
                                                                                                ntiles);
}
template <bool P32, int BY>
int batch_tma_blocks(int* out) {
  const size_t dyn = batch_tma_dyn<P32, BY>();
  if (cudaFuncSetAttribute(fx::k_hydro_batch_tma<P32, BY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn) !=
      cudaSuccess)
    return -1;
  int dev = 0, nsm = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fx::k_hydro_batch_tma<P32, BY>, fx::BX * BY, dyn) !=
      cudaSuccess)
    return -1;
  *out = per * nsm;
  return 0;
}
}  // namespace

// The TMA-staged persistent hydrodynamic launch of a batch: `tms` holds one
// set of tensor maps per domain, built for `tile_rows`.
void fx_launch_hydro_batch_tma(const fx_dev* devs, const fx_tmaps* tms, const fx_tile* tiles, int ntiles,
                               int nblocks, bool prec32, int tile_rows, cudaStream_t s) {
  if (tile_rows == 4) launch_hydro_batch_tma<4>(devs, tms, tiles, ntiles, nblocks, prec32, s);
  else if (tile_rows == 16) launch_hydro_batch_tma<16>(devs, tms, tiles, ntiles, nblocks, prec32, s);
  else launch_hydro_batch_tma<8>(devs, tms, tiles, ntiles, nblocks, prec32, s);
}
int fx_hydro_batch_tma_blocks(bool prec32, int tile_rows, int* out) {
  if (tile_rows == 4) return prec32 ? batch_tma_blocks<true, 4>(out) : batch_tma_blocks<false, 4>(out);
  if (tile_rows == 16) return prec32 ? batch_tma_blocks<true, 16>(out) : batch_tma_blocks<false, 16>(out);
  return prec32 ? batch_tma_blocks<true, 8>(out) : batch_tma_blocks<false, 8>(out);
}

void fx_launch_hydro_tma(const fx_dev& d, const fx_tmaps& tm, int nblocks, cudaStream_t s) {
  if (d.tile_rows == 4) launch_hydro_tma<4>(d, tm, nblocks, s);
  else if (d.tile_rows == 16) launch_hydro_tma<16>(d, tm, nblocks, s);
  else launch_hydro_tma<8>(d, tm, nblocks, s);
}

// Resident blocks of the TMA-staged hydrodynamic kernel (after raising its
// dynamic shared memory limit); the persistent grid is at most this.
int fx_hydro_tma_blocks(bool prec32, int tile_rows, int* out) {
  if (tile_rows == 4) return prec32 ? tma_blocks<true, 4>(out) : tma_blocks<false, 4>(out);
  if (tile_rows == 16) return prec32 ? tma_blocks<true, 16>(out) : tma_blocks<false, 16>(out);
  return prec32 ? tma_blocks<true, 8>(out) : tma_blocks<false, 8>(out);
}

void fx_launch_courant_scan(const fx_dev* devs, const fx_tile* tiles, int ntiles, int tile_rows, cudaStream_t s) {
  if (tile_rows == 4) fx::k_courant_scan<4><<<ntiles, dim3(fx::BX, 4), 0, s>>>(devs, tiles);
  else if (tile_rows == 16) fx::k_courant_scan<16><<<ntiles, dim3(fx::BX, 16), 0, s>>>(devs, tiles);
  else fx::k_courant_scan<8><<<ntiles, dim3(fx::BX, 8), 0, s>>>(devs, tiles);
}
void fx_launch_eta_from_z(const fx_dev& d, const double* z, cudaStream_t s) {
  fx::k_eta_from_z<<<592, 256, 0, s>>>(d, z);
}
void fx_launch_mass(const fx_dev& d, double* out, cudaStream_t s) { fx::k_mass<<<296, 256, 0, s>>>(d, out); }
// Appends the tiles of domain `dom` (nr x nc interior cells) to a table.
void fx_tiles_of(int dom, int nr, int nc, int tile_rows, std::vector<fx_tile>& out) {
  const int ty = tile_rows - 1;
  const int gx = (nr + fx::TX - 1) / fx::TX, gy = (nc + ty - 1) / ty;
  for (int by = 0; by < gy; ++by)
    for (int bx = 0; bx < gx; ++bx) out.push_back(fx_tile{dom, bx, by, 0});
}
