/* CPU restatement of the FLUXOS-OVERLAND explicit time step (FP64).
 *
 * TEST INFRASTRUCTURE ONLY: the checker the CUDA path is compared with. It is
 * loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg,
 * never by the product.
 *
 * Every function restates one reference function, expression by expression,
 * keeping the reference's operand types (float-typed constants such as gacc,
 * integer cell size) and its evaluation order so the results agree bit for
 * bit with the reference built in oracle/_ref. Citations are file:line within
 * src/fluxos/ of DiogoCostaPT/FLUXOS_cpp.
 */
#include "fluxos_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define OX_METEO_ROWS 2000 /* GlobVar.h:72-73: fmat(2000,3) */

struct ox_state {
  int nrows, ncols, mrows, mcols, nchem;
  size_t ncell;
  /* GlobVar.h:76-80 */
  unsigned long dxy, arbase, ntim;
  float gacc, cfl, cvdef, nuem;
  /* GlobVar.h:93-104 */
  double hdry, dtfl, tim, nodata;
  double* dcoef; /* one D per solute; the reference has one global D_coef */
  unsigned long print_step;
  unsigned int print_next, it;
  double hpall;
  int ade, has_meteo, has_inflow, volrat_mode;
  unsigned long inflow_nrow, inflow_ncol;
  int wintra;               /* EXTERNAL_MODULES.WINTRA.STATUS (main.cpp:209-213: off without ADE) */
  double soil_release_rate; /* SOIL_RELEASE_RATE [1/hour] (GlobVar.h:95) */
  /* grids */
  double *z, *zb, *h, *ux, *uy, *qx, *qy, *qxf, *qyf, *us, *dh, *dqx, *dqy, *ks;
  double *fe_1, *fe_2, *fe_3, *fn_1, *fn_2, *fn_3, *twet, *h0, *soil_mass;
  double* conc; /* nchem planes */
  float *ldry, *ldry_prev, *wall, *meteo, *inflow;
  /* extensions */
  const double* manning;
  const double* melt_mult;
};

#define IX(s, r, c) ((size_t)(c) * (size_t)(s)->mrows + (size_t)(r))
#define AT(s, a, r, c) ((s)->a[IX(s, r, c)])

static double* dgrid(size_t n) { return (double*)calloc(n, sizeof(double)); }
static float* fgrid(size_t n) { return (float*)calloc(n, sizeof(float)); }

ox_state* ox_create(int nrows, int ncols, int nchem) {
  ox_state* s = (ox_state*)calloc(1, sizeof(ox_state));
  s->nrows = nrows;
  s->ncols = ncols;
  s->mrows = nrows + 2;
  s->mcols = ncols + 2;
  s->nchem = nchem < 1 ? 1 : nchem;
  s->ncell = (size_t)s->mrows * (size_t)s->mcols;
  size_t n = s->ncell;
  /* main.cpp:132-135 and GlobVar.h:78: float-typed constants */
  s->gacc = 9.80665f;
  s->cfl = 1.0f;
  s->cvdef = 0.07f;
  s->nuem = 1.793e-6f;
  s->dxy = 1;
  s->arbase = 1;
  s->nodata = -9999.0;
  s->ade = 1;
  s->dcoef = dgrid((size_t)s->nchem);
  double** dg[] = {&s->z,    &s->zb,   &s->h,    &s->ux,   &s->uy,   &s->qx,        &s->qy,
                   &s->qxf,  &s->qyf,  &s->us,   &s->dh,   &s->dqx,  &s->dqy,       &s->ks,
                   &s->fe_1, &s->fe_2, &s->fe_3, &s->fn_1, &s->fn_2, &s->fn_3,      &s->twet,
                   &s->h0,   &s->soil_mass};
  for (size_t i = 0; i < sizeof(dg) / sizeof(dg[0]); ++i) *dg[i] = dgrid(n);
  s->conc = dgrid(n * (size_t)s->nchem);
  s->ldry = fgrid(n);
  s->ldry_prev = fgrid(n);
  s->wall = fgrid(n);
  s->meteo = fgrid(OX_METEO_ROWS * 3 + 1);
  s->inflow = fgrid(OX_METEO_ROWS * 3 + 1);
  return s;
}

void ox_destroy(ox_state* s) {
  if (!s) return;
  double* dg[] = {s->z,    s->zb,   s->h,    s->ux,   s->uy,   s->qx,   s->qy,   s->qxf,
                  s->qyf,  s->us,   s->dh,   s->dqx,  s->dqy,  s->ks,   s->fe_1, s->fe_2,
                  s->fe_3, s->fn_1, s->fn_2, s->fn_3, s->twet, s->h0,   s->soil_mass,
                  s->conc, s->dcoef};
  for (size_t i = 0; i < sizeof(dg) / sizeof(dg[0]); ++i) free(dg[i]);
  free(s->ldry);
  free(s->ldry_prev);
  free(s->wall);
  free(s->meteo);
  free(s->inflow);
  free(s);
}

double* ox_grid(ox_state* s, const char* n) {
  if (!strcmp(n, "z")) return s->z;
  if (!strcmp(n, "zb")) return s->zb;
  if (!strcmp(n, "h")) return s->h;
  if (!strcmp(n, "ux")) return s->ux;
  if (!strcmp(n, "uy")) return s->uy;
  if (!strcmp(n, "qx")) return s->qx;
  if (!strcmp(n, "qy")) return s->qy;
  if (!strcmp(n, "qxf")) return s->qxf;
  if (!strcmp(n, "qyf")) return s->qyf;
  if (!strcmp(n, "us")) return s->us;
  if (!strcmp(n, "dh")) return s->dh;
  if (!strcmp(n, "dqx")) return s->dqx;
  if (!strcmp(n, "dqy")) return s->dqy;
  if (!strcmp(n, "ks")) return s->ks;
  if (!strcmp(n, "fe_1")) return s->fe_1;
  if (!strcmp(n, "fe_2")) return s->fe_2;
  if (!strcmp(n, "fe_3")) return s->fe_3;
  if (!strcmp(n, "fn_1")) return s->fn_1;
  if (!strcmp(n, "fn_2")) return s->fn_2;
  if (!strcmp(n, "fn_3")) return s->fn_3;
  if (!strcmp(n, "twet")) return s->twet;
  if (!strcmp(n, "h0")) return s->h0;
  if (!strcmp(n, "soil_mass")) return s->soil_mass;
  if (!strncmp(n, "conc", 4)) {
    int k = n[4] ? atoi(n + 4) : 0;
    if (k < 0 || k >= s->nchem) return NULL;
    return s->conc + (size_t)k * s->ncell;
  }
  return NULL;
}

float* ox_fgrid(ox_state* s, const char* n) {
  if (!strcmp(n, "ldry")) return s->ldry;
  if (!strcmp(n, "ldry_prev")) return s->ldry_prev;
  if (!strcmp(n, "wall")) return s->wall;
  if (!strcmp(n, "meteo")) return s->meteo;
  if (!strcmp(n, "inflow")) return s->inflow;
  return NULL;
}

double ox_scalar(ox_state* s, const char* n) {
  if (!strcmp(n, "tim")) return s->tim;
  if (!strcmp(n, "dtfl")) return s->dtfl;
  if (!strcmp(n, "hdry")) return s->hdry;
  if (!strcmp(n, "ntim")) return (double)s->ntim;
  if (!strcmp(n, "nrows")) return s->nrows;
  if (!strcmp(n, "ncols")) return s->ncols;
  if (!strcmp(n, "nchem")) return s->nchem;
  if (!strcmp(n, "dxy")) return (double)s->dxy;
  if (!strcmp(n, "arbase")) return (double)s->arbase;
  if (!strcmp(n, "print_next")) return s->print_next;
  if (!strcmp(n, "print_step")) return (double)s->print_step;
  if (!strcmp(n, "it")) return s->it;
  if (!strcmp(n, "hpall")) return s->hpall;
  if (!strcmp(n, "nodata")) return s->nodata;
  if (!strcmp(n, "D_coef")) return s->dcoef[0];
  if (!strncmp(n, "D_coef", 6) && n[6]) {
    int k = atoi(n + 6);
    return (k >= 0 && k < s->nchem) ? s->dcoef[k] : NAN;
  }
  if (!strcmp(n, "ade")) return s->ade;
  if (!strcmp(n, "has_meteo")) return s->has_meteo;
  if (!strcmp(n, "has_inflow")) return s->has_inflow;
  if (!strcmp(n, "volrat_mode")) return s->volrat_mode;
  if (!strcmp(n, "inflow_nrow")) return (double)s->inflow_nrow;
  if (!strcmp(n, "inflow_ncol")) return (double)s->inflow_ncol;
  if (!strcmp(n, "wintra")) return s->wintra;
  if (!strcmp(n, "soil_release_rate")) return s->soil_release_rate;
  return NAN;
}

void ox_set_scalar(ox_state* s, const char* n, double v) {
  if (!strcmp(n, "tim")) s->tim = v;
  else if (!strcmp(n, "dtfl")) s->dtfl = v;
  else if (!strcmp(n, "hdry")) s->hdry = v;
  else if (!strcmp(n, "ntim")) s->ntim = (unsigned long)v;
  else if (!strcmp(n, "dxy")) {
    s->dxy = (unsigned long)v;
    s->arbase = s->dxy * s->dxy; /* main.cpp:176 */
  } else if (!strcmp(n, "print_next")) s->print_next = (unsigned int)v;
  else if (!strcmp(n, "print_step")) s->print_step = (unsigned long)v;
  else if (!strcmp(n, "it")) s->it = (unsigned int)v;
  else if (!strcmp(n, "nodata")) s->nodata = v;
  else if (!strcmp(n, "D_coef")) {
    for (int k = 0; k < s->nchem; ++k) s->dcoef[k] = v;
  } else if (!strncmp(n, "D_coef", 6) && n[6]) {
    int k = atoi(n + 6);
    if (k >= 0 && k < s->nchem) s->dcoef[k] = v;
  } else if (!strcmp(n, "ade")) s->ade = (int)v;
  else if (!strcmp(n, "has_meteo")) s->has_meteo = (int)v;
  else if (!strcmp(n, "has_inflow")) s->has_inflow = (int)v;
  else if (!strcmp(n, "volrat_mode")) s->volrat_mode = (int)v;
  else if (!strcmp(n, "inflow_nrow")) s->inflow_nrow = (unsigned long)v;
  else if (!strcmp(n, "inflow_ncol")) s->inflow_ncol = (unsigned long)v;
  else if (!strcmp(n, "wintra")) s->wintra = (int)v;
  else if (!strcmp(n, "soil_release_rate")) s->soil_release_rate = v;
}

void ox_set_manning(ox_state* s, const double* n_field) { s->manning = n_field; }
void ox_set_melt_field(ox_state* s, const double* mult) { s->melt_mult = mult; }

/* ------------------------------------------------------------------------ */
/* Host-side set-up                                                          */
/* ------------------------------------------------------------------------ */

/* read_functions.cpp:175-225. zb_raw holds the DEM values as read (already
 * rounded to float, read_functions.cpp:118,155) on the full (nrows+2) x
 * (ncols+2) grid with a zero ghost ring. Cells equal to NODATA or to exactly
 * 0 become walls whose bed is the float mean of their valid neighbours. */
void ox_geo_prepare(ox_state* s, const double* zb_raw, double ks_input) {
  const float nodata = (float)s->nodata;
  for (int icol = 1; icol <= s->ncols; icol++) {
    for (int irow = 1; irow <= s->nrows; irow++) {
      float zbp = (float)zb_raw[IX(s, irow, icol)];
      float zbp_corr;
      if (zbp == s->nodata || zbp == 0.0f) {
        float zbn = (float)zb_raw[IX(s, irow + 1, icol)];
        float zbs = (float)zb_raw[IX(s, irow - 1, icol)];
        float zbe = (float)zb_raw[IX(s, irow, icol + 1)];
        float zbw = (float)zb_raw[IX(s, irow, icol - 1)];
        int n = 0;
        zbp_corr = 0.0f;
        AT(s, wall, irow, icol) = 1.0f;
        if (zbn != s->nodata && zbn != 0.0f && irow < s->nrows) {
          zbp_corr += zbn;
          n++;
        }
        if (zbs != s->nodata && zbs != 0.0f && irow > 1) {
          zbp_corr += zbs;
          n++;
        }
        if (zbe != s->nodata && zbe != 0.0f && icol < s->ncols) {
          zbp_corr += zbe;
          n++;
        }
        if (zbw != s->nodata && zbw != 0.0f && icol > 1) {
          zbp_corr += zbw;
          n++;
        }
        if (zbp_corr == 0.0f) {
          zbp_corr = zbp;
        } else {
          zbp_corr /= n;
        }
      } else {
        AT(s, wall, irow, icol) = 0.0f;
        zbp_corr = fabsf(zbp);
      }
      AT(s, zb, irow, icol) = zbp_corr;
      AT(s, ks, irow, icol) = ks_input;
    }
  }
  (void)nodata;
}

/* initiate.cpp:43-90 (bed at cell centres), :159-188 (zero initial state),
 * :192-228 (ghost ring). main.cpp:259 sets hdry = ks(1,1). */
void ox_initiation_zero(ox_state* s) {
  const int NR = s->nrows, NC = s->ncols, NR1 = NR + 1, NC1 = NC + 1;
  double* zbs1 = (double*)calloc((size_t)s->mrows, sizeof(double));
  for (int irow = 0; irow <= NR1; irow++) {
    zbs1[irow] = AT(s, zb, irow, 1);
    AT(s, zb, irow, 0) = AT(s, zb, irow, 1);
    AT(s, zb, irow, NC1) = AT(s, zb, irow, NC);
  }
  for (int icol = 0; icol <= NC1; icol++) {
    AT(s, zb, 0, icol) = AT(s, zb, 1, icol);
    AT(s, zb, NR1, icol) = AT(s, zb, NR, icol);
  }
  AT(s, zb, 0, NC1) = AT(s, zb, 1, NC);
  AT(s, zb, NR1, NC1) = AT(s, zb, NR, NC);
  for (int icol = 1; icol <= NC; icol++) {
    double zbsw = zbs1[1];
    int icol1 = icol + 1;
    double zbnw = AT(s, zb, 1, icol1);
    zbs1[1] = zbnw;
    for (int irow = 1; irow <= NR; irow++) {
      int irow1 = irow + 1;
      double zbse = zbs1[irow1];
      double zbne = AT(s, zb, irow1, icol1);
      unsigned a = 0;
      double zbsum = 0;
      if (fabs(zbsw) != 99999) {
        zbsum = zbsum + zbsw;
        a = a + 1;
      }
      if (fabs(zbse) != 99999) {
        zbsum = zbsum + zbse;
        a = a + 1;
      }
      if (fabs(zbnw) != 99999) {
        zbsum = zbsum + zbnw;
        a = a + 1;
      }
      if (fabs(zbne) != 99999) {
        zbsum = zbsum + zbne;
        a = a + 1;
      }
      AT(s, zb, irow, icol) = (zbsum) / a;
      zbs1[irow1] = zbne;
      zbsw = zbse;
      zbnw = zbne;
    }
  }
  free(zbs1);
  /* :93-107 then :166-187 (no restart): the latter overwrites the former. */
  for (int icol = 1; icol <= NC; icol++) {
    for (int irow = 1; irow <= NR; irow++) {
      AT(s, h, irow, icol) = 0.0;
      AT(s, z, irow, icol) = AT(s, zb, irow, icol);
      AT(s, ux, irow, icol) = 0.0;
      AT(s, uy, irow, icol) = 0.0;
      AT(s, qx, irow, icol) = 0.0;
      AT(s, qy, irow, icol) = 0.0;
      AT(s, us, irow, icol) = 0.0;
      AT(s, soil_mass, irow, icol) = 0.0;
      AT(s, twet, irow, icol) = 0.0;
      AT(s, ldry, irow, icol) = 1.0f;
      for (int k = 0; k < s->nchem; ++k)
        s->conc[(size_t)k * s->ncell + IX(s, irow, icol)] = s->ade ? 0.0 : -1.0;
    }
  }
  /* :192-228 */
  for (int icol = 0; icol <= NC1; icol++) {
    AT(s, zb, 0, icol) = 1.5 * AT(s, zb, 1, icol) - .5 * AT(s, zb, 2, icol);
    AT(s, zb, NR1, icol) = 1.5 * AT(s, zb, NR, icol) - .5 * AT(s, zb, NR - 1, icol);
    AT(s, z, 0, icol) = 1.5 * AT(s, z, 1, icol) - .5 * AT(s, z, 2, icol);
    AT(s, z, NR1, icol) = 1.5 * AT(s, z, NR, icol) - .5 * AT(s, z, NR - 1, icol);
    AT(s, h, 0, icol) = fmax(0.0, AT(s, z, 0, icol) - AT(s, zb, 0, icol));
    AT(s, h, NR1, icol) = fmax(0.0, AT(s, z, NR1, icol) - AT(s, zb, NR1, icol));
    AT(s, qx, 0, icol) = 0.0;
    AT(s, qy, NR1, icol) = 0.0;
    AT(s, qxf, 0, icol) = 0.0;
  }
  for (int irow = 0; irow <= NR1; irow++) {
    AT(s, zb, irow, 0) = 1.5 * AT(s, zb, irow, 1) - .5 * AT(s, zb, irow, 2);
    AT(s, zb, irow, NC1) = 1.5 * AT(s, zb, irow, NC) - .5 * AT(s, zb, irow, NC - 1);
    AT(s, z, irow, 0) = 1.5 * AT(s, z, irow, 1) - .5 * AT(s, z, irow, 2);
    AT(s, z, irow, NC1) = 1.5 * AT(s, z, irow, NC) - .5 * AT(s, z, irow, NC - 1);
    AT(s, h, irow, 0) = fmax(0.0, AT(s, z, irow, 0) - AT(s, zb, irow, 0));
    AT(s, h, irow, NC1) = fmax(0.0, AT(s, z, irow, NC1) - AT(s, zb, irow, NC1));
    AT(s, qx, irow, 0) = 0.0;
    AT(s, qy, irow, NC1) = 0.0;
    AT(s, qyf, irow, 0) = 0.0;
  }
  s->hdry = AT(s, ks, 1, 1); /* main.cpp:259 */
  s->tim = 0.0;
  s->it = 0;
}

/* ------------------------------------------------------------------------ */
/* Step seams                                                                */
/* ------------------------------------------------------------------------ */

/* main.cpp:273-275 and :300-323. */
void ox_courant(ox_state* s) {
  s->dtfl = 9.e10;
  s->hpall = 0.0f;
  const float cfl_dxy = s->cfl * (float)s->dxy; /* float * size_t -> float */
  for (int icol = 1; icol <= s->ncols; icol++) {
    for (int irow = 1; irow <= s->nrows; irow++) {
      double hp = AT(s, h, irow, icol);
      AT(s, h0, irow, icol) = hp;
      AT(s, ldry_prev, irow, icol) = AT(s, ldry, irow, icol);
      if (hp > s->hdry) {
        AT(s, ldry, irow, icol) = 0.0f;
        hp = fmax(AT(s, h, irow, icol), s->hdry);
        s->hpall = fmax(s->hpall, AT(s, h, irow, icol));
        double c0 = sqrt((double)s->gacc * AT(s, h, irow, icol));
        double u0 = fmax(.000001, fabs(AT(s, qx, irow, icol) / hp));
        double v0 = fmax(.000001, fabs(AT(s, qy, irow, icol) / hp));
        s->dtfl = fmin(fmin((double)cfl_dxy / (u0 + c0), (double)cfl_dxy / (v0 + c0)), s->dtfl);
      } else {
        AT(s, ldry, irow, icol) = 1.0f;
      }
      s->dtfl = fmin((double)s->print_next - s->tim, s->dtfl);
    }
  }
}

/* Forcing-row search of common.cpp:195-200 / :307-312: the first row whose
 * time exceeds tim. Rows past the table read as time 0, so a table whose
 * last time is <= tim runs off the end in the reference; the oracle stops at
 * the last row and reports it. */
static int forcing_row(const float* tab, double tim, int* overran) {
  int a;
  for (a = 0; a < OX_METEO_ROWS; a++)
    if (tab[a] > tim) return a;
  *overran = 1;
  return OX_METEO_ROWS - 1;
}

/* common.cpp:164-273 (OpenWQ branch excluded). Returns 1 if the forcing
 * table was exhausted (undefined behaviour in the reference). */
int ox_add_meteo(ox_state* s) {
  if (!s->has_meteo) return 0;
  int overran = 0;
  int row = forcing_row(s->meteo, s->tim, &overran);
  double meteoi = (double)s->meteo[OX_METEO_ROWS + row] / (1000. * 3600. * 24.) * s->dtfl;
  double mconc = (double)s->meteo[2 * OX_METEO_ROWS + row];
  for (int icol = 1; icol <= s->ncols; icol++) {
    for (int irow = 1; irow <= s->nrows; irow++) {
      size_t i = IX(s, irow, icol);
      if (s->zb[i] != s->nodata) {
        double mi = meteoi;
        if (s->melt_mult) mi = (double)s->meteo[OX_METEO_ROWS + row] * s->melt_mult[i] /
                               (1000. * 3600. * 24.) * s->dtfl;
        double hp = fmax(s->z[i] - s->zb[i], 0.0);
        s->z[i] = s->z[i] + mi;
        s->h[i] = fmax(s->z[i] - s->zb[i], 0.0);
        if (s->h[i] <= s->hdry) s->ldry[i] = 0.0f;
        s->h0[i] = s->h[i];
        if (s->ade && hp != 0.0) {
          for (int k = 0; k < s->nchem; ++k) {
            double* c = s->conc + (size_t)k * s->ncell;
            c[i] = (c[i] * hp + (mi * mconc)) / (s->h[i]);
          }
        }
      }
    }
  }
  return overran;
}

/* common.cpp:277-390 (OpenWQ branch excluded): a point source at
 * (inflow_nrow, inflow_ncol). Inflow rows start at table row 0
 * (read_functions.cpp:311). Returns 1 on error. */
int ox_add_inflow(ox_state* s) {
  if (!s->has_inflow) return 0;
  int overran = 0;
  int row = forcing_row(s->inflow, s->tim, &overran);
  size_t irow = s->inflow_nrow, icol = s->inflow_ncol;
  double dxy = (double)s->dxy;
  double inflowi = (double)s->inflow[OX_METEO_ROWS + row] * s->dtfl / (pow(dxy, 2));
  double iconc = (double)s->inflow[2 * OX_METEO_ROWS + row];
  if (irow > (size_t)s->nrows + 1 || icol > (size_t)s->ncols + 1) return 1;
  size_t i = IX(s, irow, icol);
  if (s->zb[i] != s->nodata) {
    if (s->z[i] <= s->zb[i]) s->z[i] = s->zb[i];
    double hp = fmax(s->z[i] - s->zb[i], 0.0);
    s->z[i] = s->z[i] + inflowi;
    s->h[i] = fmax(s->z[i] - s->zb[i], 0.0);
    s->ldry[i] = (s->h[i] <= s->hdry) ? 1.0f : 0.0f;
    s->h0[i] = s->h[i];
    if (s->ade && hp != 0.0) {
      for (int k = 0; k < s->nchem; ++k) {
        double* c = s->conc + (size_t)k * s->ncell;
        c[i] = (c[i] * hp + (inflowi * iconc)) / (s->h[i]);
      }
    }
    return overran;
  }
  return 1;
}

/* read_functions.cpp:130-165: the DEM body after six header lines, parsed
 * token by token as float (stringstream >> float, i.e. strtof), first data
 * line into irow = nrows, counting down. zb_raw is the full grid, ghost ring
 * left at 0. Returns 0 on success. */
int ox_read_dem(const char* path, int nrows, int ncols, double* zb_raw) {
  FILE* f = fopen(path, "r");
  if (!f) return 1;
  size_t cap = 1 << 16, len = 0;
  char* line = (char*)malloc(cap);
  int c, hdr = 0, irow = nrows;
  for (;;) {
    len = 0;
    while ((c = fgetc(f)) != EOF && c != '\n') {
      if (len + 1 >= cap) line = (char*)realloc(line, cap *= 2);
      line[len++] = (char)c;
    }
    line[len] = 0;
    if (c == EOF && len == 0) break;
    if (hdr < 6) {
      hdr++;
      continue;
    }
    int icol = 1;
    char* p = line;
    for (;;) {
      while (*p == ' ' || *p == '\t' || *p == '\r') p++;
      if (!*p) break;
      char* end;
      float v = strtof(p, &end);
      char* tok_end = p;
      while (*tok_end && *tok_end != ' ' && *tok_end != '\t' && *tok_end != '\r') tok_end++;
      if (end != p && irow >= 0 && irow <= nrows + 1 && icol <= ncols + 1)
        zb_raw[(size_t)icol * (size_t)(nrows + 2) + (size_t)irow] = v;
      icol++;
      p = tok_end;
    }
    irow--;
    if (c == EOF) break;
  }
  free(line);
  fclose(f);
  return 0;
}

double ox_weir_term(double gacc, double hp) { return sqrt(gacc) * pow(fmax(hp, 0.0), 1.5); }

/* solver_wetdomain.cpp:27-342: E and N face fluxes of a wet cell. */
static void solver_wet(ox_state* s, int irow, int icol) {
  const unsigned NROWSl = (unsigned)s->nrows, NCOLSl = (unsigned)s->ncols;
  const double hdryl = s->hdry, gaccl = (double)s->gacc;
  const double kspl = AT(s, ks, irow, icol);
  const double nueml = (double)s->nuem, cvdefl = (double)s->cvdef;
  const unsigned is = icol - 1, in = icol + 1;
  const unsigned inn = (unsigned)fmin(icol + 2, NCOLSl + 1);
  const unsigned iw = irow - 1, ie = irow + 1;
  const unsigned dx = (unsigned)s->dxy, dy = (unsigned)s->dxy;
  int lroe = 1;
  double volrat = s->volrat_mode == 0 ? HUGE_VAL : 0.0; /* uninitialised in the reference */

  const float ldp = AT(s, ldry, irow, icol), lde = AT(s, ldry, ie, icol), ldn = AT(s, ldry, irow, in);

  const double zbw = AT(s, zb, iw, icol), zbp = AT(s, zb, irow, icol), zbe = AT(s, zb, ie, icol);
  const double zbs = AT(s, zb, irow, is), zbn = AT(s, zb, irow, in);
  const double zw = AT(s, z, iw, icol), zp = AT(s, z, irow, icol), ze = AT(s, z, ie, icol);
  const double zs = AT(s, z, irow, is), zn = AT(s, z, irow, in);
  double qp = AT(s, qx, irow, icol), qe = AT(s, qx, ie, icol), qn = AT(s, qx, irow, in);
  double rw = AT(s, qy, iw, icol), rp = AT(s, qy, irow, icol), re = AT(s, qy, ie, icol);
  double rn = AT(s, qy, irow, in);
  (void)inn; /* znn/zbnn/hnn of :75,81,100 are overwritten before use (:189) */

  const double zbpe = .5 * (zbe + zbp);
  const double zbpn = .5 * (zbn + zbp);
  const double hp = fmax(0.0, AT(s, z, irow, icol) - zbp);
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

  const double dtl = s->dtfl;

  if (lde == 1.0f) { /* :121-147 */
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
    lroe = 0;
  }
  if (ldn == 1.0f) { /* :148-175 */
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
    lroe = 0;
  }

  /* :177-203 turbulent stress */
  const double cme = sqrt(gaccl * hme);
  const double cmn = sqrt(gaccl * hmn);
  const double ume = qme / fmax(hme, hdryl);
  const double vme = rme / fmax(hme, hdryl);
  const double umn = qmn / fmax(hmn, hdryl);
  const double vmn = rmn / fmax(hmn, hdryl);

  const double cnp = cvdefl * AT(s, us, irow, icol) * hp + nueml;
  const double cne = cvdefl * AT(s, us, ie, icol) * he + nueml;
  const double cnn = cvdefl * AT(s, us, irow, in) * hn + nueml;
  const double hne = .5 * (cnp + cne) * sqrt(hp * he);
  const double hnn = .5 * (cnp + cnn) * sqrt(hp * hn);

  const double up = qp / hp0;
  const double un = qn / fmax(fmax(hn, hdryl), AT(s, ks, irow, in));
  const double us0 = AT(s, qx, irow, is) / fmax(fmax(hs, hdryl), AT(s, ks, irow, is));
  const double use0 = AT(s, qx, ie, is) / fmax(fmax(AT(s, h, ie, is), hdryl), AT(s, ks, ie, is));
  const double une = AT(s, qx, ie, in) / fmax(fmax(AT(s, h, ie, in), hdryl), AT(s, ks, ie, in));
  const double vp = rp / hp0;
  const double ve = re / fmax(fmax(he, hdryl), AT(s, ks, ie, icol));
  const double vw = rw / fmax(fmax(hw, hdryl), AT(s, ks, iw, icol));
  const double vwn = AT(s, qy, iw, in) / fmax(fmax(AT(s, h, iw, in), hdryl), AT(s, ks, iw, in));
  const double ven = AT(s, qy, ie, in) / fmax(fmax(AT(s, h, ie, in), hdryl), AT(s, ks, ie, in));

  const double txye = hne * ((ve - vp) / fabs((double)dx) + .25 * (un + une - us0 - use0) / dy);
  const double txyn = hnn * ((un - up) / fabs((double)dy) + .25 * (ve + ven - vw - vwn) / dx);

  /* :205-211 convection */
  const double fe1c = qme;
  const double fe2c = qme * ume;
  const double fe3c = qme * vme - txye;
  const double fn1c = rmn;
  const double fn2c = rmn * umn - txyn;
  const double fn3c = rmn * vmn;

  /* :213-285 Roe dissipation */
  double fe1r, fe2r, fe3r, fn1r, fn2r, fn3r;
  if (lroe) {
    double cc;
    if (hme > s->hdry) {
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

    if (ldp == 0.0f && hmn > s->hdry) {
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

  /* :287-297 */
  const double fe2p = .5 * gaccl * (hme * hme);
  const double fn3p = .5 * gaccl * (hmn * hmn);
  double fe1 = fe1c + fe1r;
  const double fe2 = fe2c + fe2r + fe2p;
  const double fe3 = fe3c + fe3r;
  double fn1 = fn1c + fn1r;
  const double fn2 = fn2c + fn2r;
  const double fn3 = fn3c + fn3r + fn3p;

  /* :299-307 edge weir */
  if ((unsigned)icol == 1 || (unsigned)icol == NCOLSl) fn1 = fmin(volrat, sqrt(gaccl) * pow(fmax(hp, 0.0), 1.5));
  if ((unsigned)irow == 1 || (unsigned)irow == NROWSl) fe1 = fmin(volrat, sqrt(gaccl) * pow(fmax(hp, 0.0), 1.5));

  /* :309-332 outflow limited to the water in the cell */
  const double volpot = (double)s->arbase * hp;
  volrat = volpot / dtl;
  if (volrat > 0.0) {
    if (fe1 > 0.0 && fn1 > 0.0) {
      if (fe1 * dy + fn1 * dx > volrat) {
        double cf = fn1 * dx / (fe1 * dy + fn1 * dx);
        fe1 = (1. - cf) * volrat / dy;
        fn1 = cf * volrat / dx;
      }
    } else if (fe1 > 0.0) {
      fe1 = fmin(fe1 * dy, volrat) / dy;
    } else if (fn1 > 0.0) {
      fn1 = fmin(fn1 * dx, volrat) / dx;
    }
  } else {
    fe1 = 0.0;
    fn1 = 0.0;
  }

  AT(s, fn_1, irow, icol) = fn1;
  AT(s, fn_2, irow, icol) = fn2;
  AT(s, fn_3, irow, icol) = fn3;
  AT(s, fe_1, irow, icol) = fe1;
  AT(s, fe_2, irow, icol) = fe2;
  AT(s, fe_3, irow, icol) = fe3;
}

/* solver_drydomain.cpp:27-194: E and N face fluxes of a dry cell. */
static void solver_dry(ox_state* s, int irow, int icol) {
  const unsigned is = icol - 1, in = icol + 1, iw = irow - 1, ie = irow + 1;
  const float ldw = AT(s, ldry, iw, icol), ldp = AT(s, ldry, irow, icol);
  const float lde = AT(s, ldry, ie, icol), lds = AT(s, ldry, irow, is), ldn = AT(s, ldry, irow, in);
  const double gaccl = (double)s->gacc;
  const unsigned NCOLSl = (unsigned)s->ncols, NROWSl = (unsigned)s->nrows;
  double volrat = s->volrat_mode == 0 ? HUGE_VAL : 0.0; /* uninitialised in the reference */
  double fe1, fe2, fe3, fn1, fn2, fn3;

  if (ldw == 1 && ldp == 1 && lde == 1 && lds == 1 && ldn == 1) { /* :60-76 */
    /* The reference zeroes only its local fe1..fn3 and returns before the
     * stores at :188-193, so the six flux grids keep the values of the last
     * step that computed them. Loop 3 then reuses those stale fluxes. */
    AT(s, dh, irow, icol) = 0.0;
    AT(s, dqx, irow, icol) = 0.0;
    AT(s, dqy, irow, icol) = 0.0;
    AT(s, qxf, irow, icol) = 0.0;
    AT(s, qyf, irow, icol) = 0.0;
    AT(s, qx, irow, icol) = 0.0;
    AT(s, qy, irow, icol) = 0.0;
    return;
  }
  const double zbp = AT(s, zb, irow, icol), zbe = AT(s, zb, ie, icol), zbn = AT(s, zb, irow, in);
  const double zp = AT(s, z, irow, icol), ze = AT(s, z, ie, icol), zn = AT(s, z, irow, in);
  const double hp = fmax(0.0, AT(s, z, irow, icol) - AT(s, z, irow, icol)); /* :85 */
  const double he = fmax(0.0, ze - zbe);
  const double hn = fmax(0.0, zn - zbn);
  const double zbpe = .5 * (zbe + zbp);
  const double zbpn = .5 * (zbn + zbp);
  double hme, qme, hmn, rmn, dze = ze - zp, dzn = zn - zp;
  const double dtl = s->dtfl;

  fe1 = fe2 = fe3 = fn1 = fn2 = fn3 = 0.0;
  if (lde == 0.0f) { /* :115-145 */
    hme = fmax(0.0, ze - zbpe);
    if (hme > s->hdry) {
      if (ze <= zp) {
        double fe2p = .5 * gaccl * hme * hme;
        fe1 = 0.0;
        fe2 = fe2p;
        fe3 = 0.0;
      } else {
        dze = fmin(fabs(dze), hme);
        qme = 0.296 * dze * sqrt(gaccl * dze);
        hme = 0.444 * dze;
        volrat = (double)s->dxy * he / dtl;
        qme = -fmin(qme, volrat);
        double ume = qme / hme;
        fe1 = qme;
        fe2 = qme * ume + .5 * gaccl * hme * hme;
        fe3 = 0.0;
      }
    } else {
      fe1 = fe2 = fe3 = 0.0;
    }
  }
  if (ldn == 0.0f) { /* :146-175 */
    hmn = fmax(0.0, zn - zbpn);
    if (hmn > s->hdry) {
      if (zn <= zp) {
        double fn3p = .5 * gaccl * hmn * hmn;
        fn1 = 0.0;
        fn2 = 0.0;
        fn3 = fn3p;
      } else {
        dzn = fmin(fabs(dzn), hmn);
        rmn = 0.296 * dzn * sqrt(gaccl * dzn);
        hmn = 0.444 * dzn;
        volrat = (double)s->dxy * hn / dtl;
        rmn = -fmin(rmn, volrat);
        double vmn = rmn / hmn;
        fn1 = rmn;
        fn2 = 0.0;
        fn3 = rmn * vmn + .5 * gaccl * hmn * hmn;
      }
    } else {
      fn1 = fn2 = fn3 = 0.0;
    }
  }
  /* :177-185 edge weir (hp is 0 here, :85) */
  if ((unsigned)icol == 1 || (unsigned)icol == NCOLSl) fn1 = fmin(volrat, sqrt(gaccl) * pow(fmax(hp, 0.0), 1.5));
  if ((unsigned)irow == 1 || (unsigned)irow == NROWSl) fe1 = fmin(volrat, sqrt(gaccl) * pow(fmax(hp, 0.0), 1.5));

  AT(s, fn_1, irow, icol) = fn1;
  AT(s, fn_2, irow, icol) = fn2;
  AT(s, fn_3, irow, icol) = fn3;
  AT(s, fe_1, irow, icol) = fe1;
  AT(s, fe_2, irow, icol) = fe2;
  AT(s, fe_3, irow, icol) = fe3;
}

/* hydrodynamics_calc.cpp:27-157 (the four OpenMP loops, run serially; they
 * carry no cross-cell reduction so the order does not change results). */
void ox_hydrodynamics(ox_state* s) {
  const double dtl = s->dtfl;
  const int NR = s->nrows, NC = s->ncols;
  const double dxy = (double)s->dxy;
  for (int icol = 1; icol <= NC; icol++) { /* :53-73 */
    for (int irow = 1; irow <= NR; irow++) {
      size_t i = IX(s, irow, icol);
      double hp = fmax(0.0, s->z[i] - s->zb[i]);
      s->h[i] = hp;
      if (hp <= s->hdry) {
        s->qx[i] = 0.0;
        s->qy[i] = 0.0;
        s->us[i] = 0.0;
        s->ldry[i] = 1.0f;
      } else {
        s->ldry[i] = 0.0f;
        s->twet[i] += dtl / 3600;
      }
    }
  }
  for (int icol = 1; icol <= NC; icol++) { /* :76-90 */
    for (int irow = 1; irow <= NR; irow++) {
      size_t i = IX(s, irow, icol);
      float cell_neumann = s->wall[i];
      if (s->ldry[i] == 1.0f && cell_neumann == 0.0f) solver_dry(s, irow, icol);
      else if (cell_neumann == 0.0f) solver_wet(s, irow, icol);
    }
  }
  for (int icol = 1; icol <= NC; icol++) { /* :93-120 */
    for (int irow = 1; irow <= NR; irow++) {
      size_t i = IX(s, irow, icol);
      if (s->wall[i] == 0.0f) {
        s->dh[i] = ((AT(s, fe_1, irow - 1, icol) - s->fe_1[i]) / dxy +
                    (AT(s, fn_1, irow, icol - 1) - s->fn_1[i]) / dxy) *
                   dtl;
        s->dqx[i] = ((AT(s, fe_2, irow - 1, icol) - s->fe_2[i]) / dxy +
                     (AT(s, fn_2, irow, icol - 1) - s->fn_2[i]) / dxy) *
                    dtl;
        s->dqy[i] = ((AT(s, fe_3, irow - 1, icol) - s->fe_3[i]) / dxy +
                     (AT(s, fn_3, irow, icol - 1) - s->fn_3[i]) / dxy) *
                    dtl;
        s->qxf[i] = s->fe_1[i] * dtl;
        s->qyf[i] = s->fn_1[i] * dtl;
      } else {
        s->dh[i] = s->dqx[i] = s->dqy[i] = s->qxf[i] = s->qyf[i] = 0.0;
      }
    }
  }
  for (int icol = 1; icol <= NC; icol++) { /* :123-154 */
    for (int irow = 1; irow <= NR; irow++) {
      size_t i = IX(s, irow, icol);
      s->z[i] = s->z[i] + s->dh[i];
      double hp = fmax(0.0, s->z[i] - s->zb[i]);
      s->h[i] = hp;
      if (hp < s->hdry || s->wall[i] == 1.0f) {
        s->qx[i] = 0.0;
        s->qy[i] = 0.0;
        s->us[i] = 0.0;
        s->ldry[i] = 1.0f;
      } else {
        s->qx[i] = s->qx[i] + s->dqx[i];
        s->qy[i] = s->qy[i] + s->dqy[i];
        s->qx[i] = .1 * AT(s, qxf, irow - 1, icol) + .8 * s->qx[i] + .1 * s->qxf[i];
        s->qy[i] = .1 * AT(s, qyf, irow, icol - 1) + .8 * s->qy[i] + .1 * s->qyf[i];
        s->ldry[i] = 0.0f;
      }
    }
  }
}

/* Cube root of x >= 0 by Newton iteration on the mantissa, using only
 * frexp/ldexp and IEEE +,-,*,/ (no libm approximation), so the CUDA path
 * (fx_hydro.cu, fx_cbrt) computes the same bits. */
static double ox_cbrt(double x) {
  if (!(x > 0.0) || isinf(x)) return x;
  int e;
  double m = frexp(x, &e);
  int r = e % 3;
  if (r < 0) r += 3;
  m = ldexp(m, r);
  e -= r;
  double y = 0.5 + 0.35 * m;
  for (int i = 0; i < 7; ++i) y = y - (y * y * y - m) / (3.0 * y * y);
  return ldexp(y, e / 3);
}

/* Extension (no reference counterpart): semi-implicit Manning friction on
 * wet, non-wall cells after the hydrodynamic update,
 *   q <- q / (1 + dt g n^2 |q| / h^(7/3)).
 * n = 0 leaves q bit-for-bit unchanged. */
void ox_manning(ox_state* s) {
  if (!s->manning) return;
  const double g = (double)s->gacc, dt = s->dtfl;
  for (int icol = 1; icol <= s->ncols; icol++) {
    for (int irow = 1; irow <= s->nrows; irow++) {
      size_t i = IX(s, irow, icol);
      double n = s->manning[i];
      if (s->ldry[i] != 0.0f || s->wall[i] != 0.0f || n == 0.0) continue;
      double hp = s->h[i];
      double qm = sqrt(s->qx[i] * s->qx[i] + s->qy[i] * s->qy[i]);
      double h73 = hp * hp * ox_cbrt(hp);
      double den = 1.0 + dt * g * n * n * qm / h73;
      s->qx[i] = s->qx[i] / den;
      s->qy[i] = s->qy[i] / den;
    }
  }
}

/* ADEsolver_calc.cpp:27-291: one Gauss-Seidel sweep for solute ichem. */
void ox_adesolver(ox_state* s, int it, int ichem) {
  if (ichem < 0 || ichem >= s->nchem) return;
  double* c = s->conc + (size_t)ichem * s->ncell;
  const unsigned long NR = (unsigned long)s->nrows, NC = (unsigned long)s->ncols;
  const double nt = 1, sigc = 0.5;
  const double D = s->dcoef[ichem];
  if (!(it > 1)) return; /* :45,74-77 */
  double* qfcds = dgrid((size_t)s->mrows * (size_t)s->mcols);
  double* cmaxr = dgrid(s->ncell);
  double* cminr = dgrid(s->ncell);
#define C(r, q) c[IX(s, r, q)]
  for (unsigned long a = 1; a <= NC * NR; a++) { /* :47-73 */
    unsigned long iy = ((a - 1) / NR) + 1;
    unsigned long ix = a - NR * (iy - 1);
    size_t i = IX(s, ix, iy);
    cmaxr[i] = fmax(C(ix - 1, iy), fmax(C(ix + 1, iy), fmax(C(ix, iy - 1), C(ix, iy + 1))));
    cminr[i] = fmin(C(ix - 1, iy), fmin(C(ix + 1, iy), fmin(C(ix, iy - 1), C(ix, iy + 1))));
    double hnew = s->h[i];
    if (s->ldry[i] == 0 && s->ldry_prev[i] == 0) {
      c[i] = c[i] * s->h0[i] / hnew;
    } else if (s->ldry[i] == 1) {
      c[i] = 0.0;
    }
  }
  const double dx = (double)s->dxy, dy = (double)s->dxy;
  const double arb = (double)s->arbase;
  double pfe = 0, pfce, pfde, hne, hnn, hp, he, hn, fp, fe;
  for (unsigned long a = 1; a < NC * NR; a++) { /* :93-290 */
    unsigned long iy = ((a - 1) / NR) + 1;
    unsigned long ix = a - NR * (iy - 1);
    unsigned long is = iy - 1, in = iy + 1;
    unsigned long inn = (unsigned long)fmin(iy + 2, NC + 1);
    unsigned long iw = ix - 1, ie = ix + 1;
    unsigned long iee = (unsigned long)fmin(ix + 2, NR + 1);
    size_t i = IX(s, ix, iy);

    if (ix == 1) { /* :106-116 */
      pfce = C(0, iy) * AT(s, fe_1, 0, iy) * dy;
      hp = fmax(AT(s, h, 1, iy), s->hdry);
      he = fmax(AT(s, h, 2, iy), s->hdry);
      fp = C(0, iy);
      fe = C(1, iy);
      hne = sqrt(hp * nt * he * nt) / sigc / fabs(dx) * dy * D;
      pfde = 0.;
      pfe = pfce;
    }
    if (s->ldry[i] == 1) { /* :119-124 */
      pfe = 0.;
      qfcds[ix] = 0.;
      c[i] = 0.;
      continue;
    }
    const double area = arb, areae = arb, arean = arb;
    const double ntp = nt;
    hp = s->h[i];
    he = AT(s, h, ie, iy);
    hn = AT(s, h, ix, in);
    const double qxl = s->fe_1[i];
    const double qyl = s->fn_1[i];
    const double fw = C(iw, iy);
    fp = C(ix, iy);
    fe = C(ie, iy);
    const double fee = C(iee, iy);
    const double fs = C(ix, is);
    const double fn = C(ix, in);
    const double fnn = C(ix, inn);
    const double pfw = pfe;
    const double qfs = qfcds[ix];

    double fem, fnm, qfdn, qfn, hnue;
    if (AT(s, ldry, ie, iy) == 0) { /* :151-172 */
      hnue = fmax(hp * nt * he * nt, .0001);
      hne = sqrt(hnue) / sigc / dx * dy * D;
      pfde = -hne * (fe - fp);
      if (qxl > 0.0) {
        if (AT(s, ldry, iw, iy) == 0) fem = -.125 * fw + .75 * fp + .375 * fe;
        else fem = 0.5 * fp + 0.5 * fe;
      } else {
        if (AT(s, ldry, iee, iy) == 0) fem = .375 * fp + .75 * fe - .125 * fee;
        else fem = 0.5 * fp + 0.5 * fe;
      }
    } else {
      fem = 0.;
      pfde = 0.;
    }
    fem = fmax(0., fem);
    if (ix == NR) fem = C(NR + 1, iy);
    pfce = qxl * fem * dy;
    pfe = pfce + pfde;
    if (pfe < 0) { /* :187-194 */
      if (AT(s, ldry, ie, iy) == 0) {
        double cvolrate = -(fe * he) * areae / s->dtfl;
        pfe = fmax(pfe, cvolrate);
      } else {
        pfe = 0.;
      }
    }
    if (AT(s, ldry, ix, in) == 0) { /* :198-218 */
      hnue = fmax(.0001, hp * ntp * hn * nt);
      hnn = sqrt(hnue) / sigc / dy * dx * D;
      qfdn = -hnn * (fn - fp);
      if (qyl > 0.0) {
        if (AT(s, ldry, ix, is) == 0) fnm = -.125 * fs + .75 * fp + .375 * fn;
        else fnm = 0.5 * fp + .5 * fn;
      } else {
        if (AT(s, ldry, ix, inn) == 0) fnm = .375 * fp + .75 * fn - .125 * fnn;
        else fnm = .5 * fp + .5 * fn;
      }
    } else {
      fnm = 0.;
      qfdn = 0.;
    }
    fnm = fmax(0., fnm);
    if (iy == NC) fnm = C(ix, NC + 1);
    const double qfcn = qyl * fnm * dx;
    qfn = qfcn + qfdn;
    if (qfn < 0) { /* :234-241 */
      if (AT(s, ldry, ix, in) == 0) {
        double cvolrate = -(fn * hn) * arean / s->dtfl;
        qfn = fmax(qfn, cvolrate);
      } else {
        qfn = 0.;
      }
    }
    /* :243-278 */
    const double cvolpot = (fp * hp) * area;
    const double cvolrat = cvolpot / s->dtfl + pfw + qfs;
    if (cvolrat > 0.0) {
      if (pfe > 0. && qfn > 0.) {
        if (pfe + qfn > cvolrat) {
          double cf = qfn / (pfe + qfn);
          pfe = (1. - cf) * cvolrat;
          qfn = cf * cvolrat;
        }
      } else if (pfe > 0.) {
        pfe = fmin(pfe, (cvolrat - qfn));
      } else if (qfn > 0.) {
        qfn = fmin(qfn, (cvolrat - pfe));
      }
    } else {
      if (pfe >= 0. && qfn < 0.) {
        double cbilan = cvolrat - qfn;
        if (cbilan > 0.) pfe = fmin(pfe, cbilan);
        else pfe = 0.;
      } else if (pfe < 0. && qfn >= 0.) {
        double cbilan = cvolrat - pfe;
        if (cbilan > 0.) qfn = fmin(qfn, cbilan);
        else qfn = 0.;
      } else if (pfe >= 0. && qfn >= 0.) {
        pfe = 0.0;
        qfn = 0.0;
      }
    }
    /* :281-288 */
    const double dc = (pfw - pfe + qfs - qfn) * s->dtfl / area;
    double con = c[i] + dc / hp;
    con = fmin(cmaxr[i], con);
    con = fmax(cminr[i], con);
    c[i] = con;
    qfcds[ix] = qfn;
  }
#undef C
  free(qfcds);
  free(cmaxr);
  free(cminr);
}

/* One iteration of main.cpp:273-406 (printing excluded; WINTRA and OpenWQ
 * are outside this path). Returns 1 if a forcing table ran out. */
/* wintrasolver_calc (WINTRAsolver_calc.cpp:26-58) for solute ichem: every
 * wet cell whose bed is not NODATA_VALUE releases the first-order fraction
 * soil_release_rate/3600*dtfl of its soil mass into its concentration. The
 * reference also computes a tanh melt factor (:33-36) that nothing reads;
 * it is not restated. */
void ox_wintra(ox_state* s, int ichem) {
  double* c = s->conc + (size_t)ichem * s->ncell;
  for (int icol = 1; icol <= s->ncols; icol++) {
    for (int irow = 1; irow <= s->nrows; irow++) {
      const size_t i = IX(s, irow, icol);
      const double hp = s->h[i];
      const double zbp = s->zb[i];
      if (hp > s->hdry && zbp != s->nodata) {
        const double deltam = s->soil_mass[i] * s->soil_release_rate / 3600 * s->dtfl;
        s->soil_mass[i] = s->soil_mass[i] - deltam;
        c[i] = c[i] + deltam / (hp * (double)s->arbase);
      }
    }
  }
}

int ox_step(ox_state* s) {
  int err = 0;
  ox_courant(s);
  s->tim = s->tim + s->dtfl;
  err |= ox_add_meteo(s);
  err |= ox_add_inflow(s);
  if (s->hpall != 0) {
    s->it++;
    ox_hydrodynamics(s);
    ox_manning(s);
    if (s->ade)
      for (int k = 0; k < s->nchem; ++k) ox_adesolver(s, (int)s->it, k);
    if (s->ade && s->wintra)  /* main.cpp:399-404 */
      for (int k = 0; k < s->nchem; ++k) ox_wintra(s, k);
  }
  return err;
}

int ox_running(ox_state* s) { return s->tim <= (double)s->ntim; }
int ox_print_due(ox_state* s) { return s->tim >= (double)s->print_next; }
void ox_print_done(ox_state* s) { s->print_next = s->print_next + (unsigned int)s->print_step; }
