/* CPU restatement of the FLUXOS-OVERLAND explicit time step (FP64).
 *
 * TEST INFRASTRUCTURE ONLY: the correctness checker for the CUDA path. Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * The state mirrors the reference's GlobVar (src/fluxos/GlobVar.h:25-117):
 * every grid is (nrows+2) x (ncols+2) doubles (flags: floats), column-major
 * with irow fastest, ghost ring included, zero-initialised.
 *
 * Parity is pinned against the reference sources compiled here
 * (oracle/_ref/libfluxos_ref.so, same function-level API with the prefix
 * fxr_) and against the fixtures in tests/golden/.
 */
#ifndef FLUXOS_ORACLE_H
#define FLUXOS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ox_state ox_state;

/* volrat_mode: how the uninitialised `volrat` of solver_wetdomain.cpp:37 /
 * solver_drydomain.cpp:36 reads at domain-edge cells. 0 = +inf ("weir": the
 * edge flux is the weir formula), 1 = 0 ("closed"). */
ox_state* ox_create(int nrows, int ncols, int nchem);
void ox_destroy(ox_state* s);

double* ox_grid(ox_state* s, const char* name);  /* z zb h qx qy us ks fe_1.. conc conc1 .. */
float* ox_fgrid(ox_state* s, const char* name);  /* ldry ldry_prev wall meteo */
double ox_scalar(ox_state* s, const char* name);
void ox_set_scalar(ox_state* s, const char* name, double v);

/* Extensions with no reference counterpart (NULL = off, the parity mode). */
void ox_set_manning(ox_state* s, const double* n_field);   /* per-cell Manning n */
void ox_set_melt_field(ox_state* s, const double* mult);   /* per-cell melt multiplier */

/* Host-side set-up: read_functions.cpp:175-225 then initiate.cpp:43-90,159-228. */
int ox_read_dem(const char* path, int nrows, int ncols, double* zb_raw);
void ox_geo_prepare(ox_state* s, const double* zb_raw, double ks_input);
void ox_initiation_zero(ox_state* s);

/* The step seams. */
void ox_courant(ox_state* s);                   /* main.cpp:300-323 */
int ox_add_meteo(ox_state* s);                  /* common.cpp:164-273 */
int ox_add_inflow(ox_state* s);                 /* common.cpp:277-390 */
void ox_hydrodynamics(ox_state* s);             /* hydrodynamics_calc.cpp:27-157 */
void ox_adesolver(ox_state* s, int it, int ichem); /* ADEsolver_calc.cpp:27-291 */
void ox_manning(ox_state* s);                   /* extension, after the hydro update */
void ox_wintra(ox_state* s, int ichem);         /* WINTRAsolver_calc.cpp:26-58 */
int ox_step(ox_state* s);                       /* main.cpp:273-406 without printing */
int ox_running(ox_state* s);                    /* main.cpp:271 loop condition */
int ox_print_due(ox_state* s);                  /* main.cpp:444 */
void ox_print_done(ox_state* s);                /* main.cpp:458 */

/* The weir term sqrt(g)*pow(h,1.5) exactly as the reference evaluates it
 * (exported so tests can compare the CUDA evaluation with libm). */
double ox_weir_term(double gacc, double hp);

#ifdef __cplusplus
}
#endif
#endif
