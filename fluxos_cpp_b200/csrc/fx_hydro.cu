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

#include "fx_common.cuh"

namespace fx {

// A block of 32 x 8 threads owns a tile of 31 rows (irow) x 7 columns (icol):
// with its west row and south column of halo faces the tile has exactly
// 32 x 8 = 256 face-flux cells, one per thread, so the flux phase runs in a
// single wave and no warp waits at the barrier for a second round.
constexpr int BX = 32, BY = 8;                  // threads
constexpr int TX = 31, TY = 7;                  // owned cells
constexpr int SX = TX + 3, SY = TY + 3;        // stencil: rows irow0-2..irow0+TX, cols icol0-2..icol0+TY
constexpr int FXN = TX + 1, FYN = TY + 1;      // fluxes: rows irow0-1..irow0+TX-1, cols icol0-1..icol0+TY-1
constexpr int NSTEN = SX * SY, NFLUX = FXN * FYN;
constexpr int NTHREADS = BX * BY;
static_assert(NFLUX == NTHREADS, "one face-flux cell per thread");

// stencil cell classes
constexpr unsigned char C_DRY = 1;   // Loop-1 ldry == 1 (interior cells only)
constexpr unsigned char C_WALL = 2;  // innerNeumannBCWeir == 1
constexpr unsigned char C_INT = 4;   // interior cell (1..NROWS, 1..NCOLS)

struct HydroSmem {
  double z[NSTEN], zb[NSTEN], qx[NSTEN], qy[NSTEN];
  double f[6][NFLUX];
  unsigned char cls[NSTEN];
  short wet_list[NFLUX], dry_list[NFLUX], stale_list[NFLUX];
  int nwet, ndry, nstale;
  double red_dt[NTHREADS / 32], red_h[NTHREADS / 32];
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
__device__ void solver_wet(const fx_dev& d, const HydroSmem& S, int sr, int sc, int irow, int icol,
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
  const double un = qn / fmax(fmax(hn, hdryl), ksat(N));
  const double us0 = S.qx[Sx] / fmax(fmax(hs, hdryl), ksat(Sx));
  const double use0 = S.qx[ES] / fmax(fmax(hat(ES), hdryl), ksat(ES));
  const double une = S.qx[EN] / fmax(fmax(hat(EN), hdryl), ksat(EN));
  const double vp = rp / hp0;
  const double ve = re / fmax(fmax(he, hdryl), ksat(E));
  const double vw = rw / fmax(fmax(hw, hdryl), ksat(W));
  const double vwn = S.qy[WN] / fmax(fmax(hat(WN), hdryl), ksat(WN));
  const double ven = S.qy[EN] / fmax(fmax(hat(EN), hdryl), ksat(EN));

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
__device__ void solver_dry(const fx_dev& d, const HydroSmem& S, int sr, int sc, int irow, int icol,
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
    double c = fmin(d.cfl_dxy / (u0 + c0), d.cfl_dxy / (v0 + c0));
    if (c == c) dtc = c;
    hm = h;
  }
}

// Block-wide min/max followed by one atomic each on the control block.
__device__ void reduce_courant(const fx_dev& d, HydroSmem& S, double dtc, double hm) {
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

__device__ __forceinline__ double melt_depth(const fx_dev& d, const fx_ctl& c, long long gi) {
  if (d.melt_mult) return (double)c.meteo_rate * d.melt_mult[gi] / (1000. * 3600. * 24.) * c.dtfl;
  return c.meteoi;
}

__global__ void __launch_bounds__(NTHREADS) k_hydro(fx_dev d) {
  __shared__ HydroSmem S;
  const fx_ctl c = *d.ctl;
  if (!c.live) return;
  const int lx = threadIdx.x, ly = threadIdx.y;
  const int tid = ly * BX + lx;
  const int irow0 = 1 + blockIdx.x * TX, icol0 = 1 + blockIdx.y * TY;
  const int irow = irow0 + lx, icol = icol0 + ly;
  const bool own = lx < TX && ly < TY && irow <= d.nr && icol <= d.nc;
  const double dtl = c.dtfl;
  const bool melt_on = d.has_meteo != 0;

  // Slot planes: the state after the previous step, and the one this step
  // writes (h, h0, fe_1, fn_1, flags; see fx_common.cuh).
  const long long sprev = fx_slot(d, c.steps - 1), scur = fx_slot(d, c.steps);

  if (!c.active) {
    // No wet cell: the step is the Courant scan plus add_meteo only
    // (main.cpp:300-370, the solver block at :385 is skipped). The solute
    // dilution of add_meteo is applied by the ADE sweep (fx_ade.cu).
    double dtc = __longlong_as_double(0x7ff0000000000000LL), hm = 0.0;
    if (own) {
      const long long gi = fx_ix(d, irow, icol);
      const double zb = d.zb[gi], zpre = d.z[gi];
      const uint8_t fl = d.flags[sprev + gi];
      const double hpre = fmax(0.0, zpre - zb);
      uint8_t ld = hpre > d.hdry ? 0 : 1;  // Courant scan (:308-320)
      double z1 = zpre, h1 = hpre;
      if (melt_on && zb != d.nodata) {
        const double mi = melt_depth(d, c, gi);
        if (d.ade) d.hpm[scur + gi] = fmax(zpre - zb, 0.0);  // the dilution's hp (common.cpp:216)
        z1 = zpre + mi;
        h1 = fmax(z1 - zb, 0.0);
        if (h1 <= d.hdry) ld = 0;  // common.cpp:219-222
        d.z[gi] = z1;
      }
      d.h[scur + gi] = h1;
      d.h0[scur + gi] = h1;
      d.flags[scur + gi] = (fl & (FX_F_WALL | FX_F_NODATA)) | ((fl & FX_F_LDRY) ? FX_F_LDRY_PREV : 0) | ld;
      if (scur != sprev) {  // fluxes are unchanged by a step without solver
        d.fe1[scur + gi] = d.fe1[sprev + gi];
        d.fn1[scur + gi] = d.fn1[sprev + gi];
      }
      courant_cell(d, h1, d.qx[gi], d.qy[gi], dtc, hm);
    }
    reduce_courant(d, S, dtc, hm);
    return;
  }

  // ---- phase A: stencil load, melt, Loop 1 ---------------------------------
  if (tid == 0) {
    S.nwet = 0;
    S.ndry = 0;
    S.nstale = 0;
  }
  for (int k = tid; k < NSTEN; k += NTHREADS) {
    const int sr = k % SX, sc = k / SX;
    const int r = irow0 - 2 + sr, q = icol0 - 2 + sc;
    double z = 0.0, zb = 0.0, qx = 0.0, qy = 0.0;
    unsigned char cl = 0;
    if (r >= 0 && r <= d.nr + 1 && q >= 0 && q <= d.nc + 1) {
      const long long gi = fx_ix(d, r, q);
      z = d.z[gi];
      zb = d.zb[gi];
      qx = d.qx[gi];
      qy = d.qy[gi];
      if (r >= 1 && r <= d.nr && q >= 1 && q <= d.nc) {
        cl = C_INT;
        if (d.flags[sprev + gi] & FX_F_WALL) cl |= C_WALL;
        if (melt_on && zb != d.nodata) z = z + melt_depth(d, c, gi);
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
  }
  __syncthreads();

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
      S.f[0][k] = d.fe1[sprev + gi];
      S.f[1][k] = d.fe2[gi];
      S.f[2][k] = d.fe3[gi];
      S.f[3][k] = d.fn1[sprev + gi];
      S.f[4][k] = d.fn2[gi];
      S.f[5][k] = d.fn3[gi];
    }
  }
  __syncthreads();

  // ---- phase D: Loop 3, Loop 4, friction, store, next Courant --------------
  double dtc = __longlong_as_double(0x7ff0000000000000LL), hm = 0.0;
  if (own) {
    const long long gi = fx_ix(d, irow, icol);
    const int sP = sidx(lx + 2, ly + 2);
    const int fP = (ly + 1) * FXN + (lx + 1), fW = (ly + 1) * FXN + lx, fS = ly * FXN + (lx + 1);
    const unsigned char cl = S.cls[sP];
    const bool wall = cl & C_WALL;
    const uint8_t fl = d.flags[sprev + gi];
    const double zb = S.zb[sP];
    const double z1 = S.z[sP];
    const double zpre = d.z[gi];

    // add_meteo's h0 (common.cpp:223): the depth after the melt, or the
    // Courant scan's copy of h (main.cpp:305) for cells it skips. Its solute
    // dilution (:226-234) is applied by the ADE sweep (fx_ade.cu).
    double h0v = fmax(0.0, zpre - zb);
    if (melt_on && zb != d.nodata) {
      h0v = fmax(z1 - zb, 0.0);
      if (d.ade) d.hpm[scur + gi] = fmax(zpre - zb, 0.0);  // the dilution's hp (common.cpp:216)
    }
    // Loop 1 wet time (:69-70)
    if (!(cl & C_DRY)) d.twet[gi] += dtl / 3600;

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
    d.z[gi] = z;
    d.h[scur + gi] = h;
    d.qx[gi] = qx;
    d.qy[gi] = qy;
    d.h0[scur + gi] = h0v;
    d.flags[scur + gi] = (fl & (FX_F_WALL | FX_F_NODATA)) | ((fl & FX_F_LDRY) ? FX_F_LDRY_PREV : 0) | ld;
    // Fluxes computed this step become the grid values (stale ones are
    // already there). fe_2/fe_3/fn_2/fn_3 are read back only when this cell
    // is dry with four dry neighbours at a later solver step; a cell that
    // ends the step wet (h > hdry) is wet again at the next solver step as
    // long as forcing adds water, so those three-quarters of the flux
    // traffic are skipped for it.
    const unsigned char clP = cl;
    if ((clP & C_INT) && !(clP & C_WALL)) {
      const bool computed =
          !(clP & C_DRY) || !((S.cls[sidx(lx + 1, ly + 2)] & C_DRY) && (S.cls[sidx(lx + 3, ly + 2)] & C_DRY) &&
                              (S.cls[sidx(lx + 2, ly + 1)] & C_DRY) && (S.cls[sidx(lx + 2, ly + 3)] & C_DRY));
      // fe_1/fn_1 of every cell go to this step's slot: computed ones, or the
      // stale ones carried over (already in S.f for stale cells).
      d.fe1[scur + gi] = S.f[0][fP];
      d.fn1[scur + gi] = S.f[3][fP];
      if (computed && (d.store_all_fluxes || !(h > d.hdry))) {
        d.fe2[gi] = S.f[1][fP];
        d.fe3[gi] = S.f[2][fP];
        d.fn2[gi] = S.f[4][fP];
        d.fn3[gi] = S.f[5][fP];
      }
    } else if (scur != sprev) {
      d.fe1[scur + gi] = 0.0;  // walls: never written in the reference
      d.fn1[scur + gi] = 0.0;
    }
    courant_cell(d, h, qx, qy, dtc, hm);
  }
  reduce_courant(d, S, dtc, hm);
}

// Courant scan of the state as uploaded (the scan at the top of the first
// step). Also used after a host edit of the state.
__global__ void __launch_bounds__(NTHREADS) k_courant_scan(fx_dev d) {
  const int irow = 1 + blockIdx.x * BX + threadIdx.x, icol = 1 + blockIdx.y * BY + threadIdx.y;
  __shared__ HydroSmem S;
  double dtc = __longlong_as_double(0x7ff0000000000000LL), hm = 0.0;
  if (irow <= d.nr && icol <= d.nc) {
    const long long gi = fx_ix(d, irow, icol);
    courant_cell(d, d.h[fx_slot(d, d.ctl->steps) + gi], d.qx[gi], d.qy[gi], dtc, hm);
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

// The clock update of one step, single thread (main.cpp:271-325 and
// common.cpp:195-208).
__global__ void k_finalize(fx_dev d) {
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
  c.active = hpall != 0.0;
  if (c.active) c.it = c.it + 1;
  c.print_pending = c.tim >= c.print_next;
  c.steps = c.steps + 1;
  fx_steprec& r = c.rec[c.steps % d.nslot];
  r.dtfl = c.dtfl;
  r.meteoi = c.meteoi;
  r.meteo_rate = c.meteo_rate;
  r.mconc = c.mconc;
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
__global__ void k_batch_begin(fx_dev d) { d.ctl->batch = d.ctl->batch + 1; }

// Sets the bed flags that never change (NODATA bed) in every slot plane.
__global__ void k_mark_static(fx_dev d) {
  const long long n = d.plane;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int icol = (int)(i / d.ld), irow = (int)(i % d.ld) - FX_ROFF;
    if (irow < 1 || irow > d.nr || icol < 1 || icol > d.nc) continue;
    const bool nod = d.zb[i] == d.nodata;
    for (int k = 0; k < d.nslot; ++k) {
      uint8_t& f = d.flags[k * d.plane + i];
      f = (uint8_t)((f & ~FX_F_NODATA) | (nod ? FX_F_NODATA : 0));
    }
  }
}

}  // namespace fx

// Launch helpers used by fx_capi.cu.
void fx_launch_finalize(const fx_dev& d, cudaStream_t s) { fx::k_finalize<<<1, 1, 0, s>>>(d); }
void fx_launch_batch_begin(const fx_dev& d, cudaStream_t s) { fx::k_batch_begin<<<1, 1, 0, s>>>(d); }
void fx_launch_mark_static(const fx_dev& d, cudaStream_t s) { fx::k_mark_static<<<592, 256, 0, s>>>(d); }

void fx_launch_hydro(const fx_dev& d, cudaStream_t s) {
  dim3 b(fx::BX, fx::BY), g((d.nr + fx::TX - 1) / fx::TX, (d.nc + fx::TY - 1) / fx::TY);
  fx::k_hydro<<<g, b, 0, s>>>(d);
}

void fx_launch_courant_scan(const fx_dev& d, cudaStream_t s) {
  dim3 b(fx::BX, fx::BY), g((d.nr + fx::BX - 1) / fx::BX, (d.nc + fx::BY - 1) / fx::BY);
  fx::k_courant_scan<<<g, b, 0, s>>>(d);
}
