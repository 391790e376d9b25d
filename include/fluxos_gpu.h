/* fluxos_gpu.h: C ABI of libfluxos_gpu.so, the B200 (sm_100a) implementation
 * of the FLUXOS-OVERLAND explicit time step.
 *
 * Plain C types only: sizes are ints, grids are host pointers to the
 * reference's GlobVar layout, i.e. (NROWS+2) x (NCOLS+2) values, column-major
 * with irow fastest, ghost ring included (src/fluxos/GlobVar.h:31-74). Every
 * call returns FX_OK (0) or a negative FX_ERR_* code and never throws; the
 * message of the last failure is fx_last_error(). A context owns its device
 * memory and one CUDA stream; use one host thread per context. Contexts are
 * independent of each other.
 *
 * Reference interfaces replaced (DiogoCostaPT/FLUXOS_cpp, src/fluxos/):
 *   fx_step / fx_run_to_print : one or more iterations of the step loop
 *       main.cpp:271-470, i.e. the Courant scan main.cpp:300-325,
 *       add_meteo (common.cpp:164, common.h:50-67),
 *       hydrodynamics_calc (hydrodynamics_calc.h:24) and
 *       adesolver_calc (ADEsolver_calc.h:25)
 *   fx_open_modset : the start-up main.cpp:87-262 with read_modset,
 *       read_geo, read_meteo (read_functions.h:25-43) and initiation
 *       (initiate.h)
 *   fx_write_results : write_results (write_results.cpp:30)
 *   fx_run : the whole program `fluxos <modset.json>` (main.cpp:70)
 */
#ifndef FLUXOS_GPU_H
#define FLUXOS_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define FX_OK 0
#define FX_ERR_ARG -1    /* bad argument or size */
#define FX_ERR_CUDA -2   /* a CUDA runtime call failed (message has the call) */
#define FX_ERR_IO -3     /* an input file could not be read or an output written */
#define FX_ERR_STATE -4  /* call out of order (e.g. stepping a finished run) */
#define FX_ERR_DEVICE -5 /* a kernel raised its error flag (a bounded wait gave up) */
#define FX_ERR_NOMEM -6  /* device allocation failed */

#define FX_MAX_CHEM 8

typedef struct fx_ctx fx_ctx;

/* Domain (GlobVar.h:75-76,104; read_functions.cpp:130-139). */
typedef struct fx_grid {
  int nrows;     /* NROWS: interior cells along irow */
  int ncols;     /* NCOLS: interior cells along icol */
  int dxy;       /* cell size [m], an integer as in the reference */
  int nchem;     /* solutes, 1..FX_MAX_CHEM (the reference has 1) */
  double nodata; /* NODATA_VALUE */
  double xll;    /* XLLCORNER */
  double yll;    /* YLLCORNER */
} fx_grid;

/* Physics and run control. */
typedef struct fx_params {
  double hdry;       /* dry threshold; the reference sets it to ks(1,1) (main.cpp:259) */
  double ks;         /* ROUGNESS_HEIGHT of interior cells */
  double ntim;       /* run while tim <= ntim (main.cpp:192,271) */
  double print_step; /* PRINT_STEP [s] */
  double print_next; /* first output time (main.cpp:260-261) */
  double tim;        /* starting clock (0 in the reference) */
  double h_min_print;/* H_MIN_TO_PRINT as the reference stores it (an integer) */
  int ade;           /* EXTERNAL_MODULES.ADE_TRANSPORT.STATUS */
  int volrat_mode;   /* domain-edge weir: 0 = weir formula (default), 1 = closed */
  double d_coef[FX_MAX_CHEM]; /* dispersion coefficient per solute */
  int steps_in_flight; /* steps whose ADE sweeps run in one launch, 1..63; 0 = as many as
                          * the per-step planes allow within 1 GiB, from 8 to 63 */
  int precision;       /* 0 = FP64, the reference's arithmetic (default);
                          1 = FP32 state: the depth above the bed eta = z - zb and
                          the bed's differences to the east and north neighbours
                          are stored instead of z, flux/update/ADE arithmetic is
                          FP32; the clock, the wet/dry threshold tests and the
                          water budget stay FP64. Not bit-compatible with the
                          reference: see tests/test_gpu_fp32.py for its error. */
  int wintra;          /* EXTERNAL_MODULES.WINTRA.STATUS: the soil release of
                          wintrasolver_calc (WINTRAsolver_calc.cpp:26-58) after
                          each step's ADE sweep; off unless ade is on
                          (main.cpp:209-213) */
  double soil_release_rate; /* SOIL_RELEASE_RATE [1/hour] */
} fx_params;

/* Clock and status read back from the device. */
typedef struct fx_status {
  double tim;           /* simulated clock [s] */
  double dtfl;          /* last dt [s] */
  double print_next;    /* next output time [s] */
  double hpall;         /* max wet depth of the last Courant scan */
  long long steps;      /* steps executed since creation */
  int it;               /* solver iterations (main.cpp:387) */
  int print_pending;    /* tim >= print_next: write results, then fx_print_done */
  int finished;         /* tim > ntim: the run is over */
  int device_error;     /* nonzero when a kernel gave up a bounded wait */
  int forcing_overrun;  /* the forcing table had no row later than tim */
  double budget_melt;   /* water added by the forcing (melt, point inflow) since creation [m^3], FP64 */
  double budget_out;    /* water that left through the outflow faces (E face of
                           irow = NROWS, N face of icol = NCOLS) or into wall
                           cells since creation [m^3], FP64 */
} fx_status;

/* --- context ------------------------------------------------------------ */
int fx_create(const fx_grid* g, const fx_params* p, fx_ctx** out);
void fx_destroy(fx_ctx* ctx);
const char* fx_last_error(const fx_ctx* ctx); /* ctx may be NULL: last global error */
int fx_device_bytes(const fx_ctx* ctx, long long* bytes); /* device memory held */
/* Device memory fx_create would take for this grid and these parameters,
 * plus `extension_grids` per-cell extension grids (fx_set_manning,
 * fx_set_melt_field): the figure an admission policy sizes against. */
int fx_footprint(const fx_grid* g, const fx_params* p, int extension_grids, long long* bytes);

/* --- state ---------------------------------------------------------------
 * Field names: "z" "zb" "h" "qx" "qy" "twet" "h0" "fe_1" "fe_2" "fe_3"
 * "fn_1" "fn_2" "fn_3" "conc" (solute 0) "conc1".."conc7" "soil_mass" (the
 * soil mass WINTRA releases [g]; 0 until uploaded, as the reference's
 * initiation leaves it without a restart file).
 * Uploads take the full (nrows+2) x (ncols+2) grid; fx_upload_flags takes the
 * float flag grids ldry and innerNeumannBCWeir (wall) of GlobVar. After the
 * state is complete call fx_prepare once (it runs the first Courant scan). */
int fx_upload(fx_ctx* ctx, const char* field, const double* host_grid);
int fx_download(fx_ctx* ctx, const char* field, double* host_grid);
int fx_upload_flags(fx_ctx* ctx, const float* ldry, const float* wall);
int fx_download_flags(fx_ctx* ctx, float* ldry, float* ldry_prev, float* wall);
/* Forcing table of GlobVar::meteo: 2000 rows x 3 columns (time [s], rate
 * [mm/day], concentration), column-major float as arma::fmat(2000,3).
 * has_meteo = 0 means no METEO_FILE (add_meteo returns at common.cpp:190). */
int fx_set_forcing(fx_ctx* ctx, const float* table_2000x3, int has_meteo);
/* Point inflow of INFLOW_FILE (add_inflow, common.cpp:277-390): the table of
 * GlobVar::inflow, 2000 rows x 3 columns (time [s], discharge [m^3/s],
 * concentration) column-major float with data from row 0, and the interior
 * cell (irow, icol) it enters (read_functions.cpp:228-231). NULL switches it
 * off. FX_ERR_ARG if the cell is outside the interior or a NODATA cell. With
 * more than one solute every solute takes the table's one concentration
 * column (the reference's table has one). The discharged volume is counted
 * in fx_status.budget_melt. */
int fx_set_inflow(fx_ctx* ctx, const float* table_2000x3, int irow, int icol);
/* Extensions without a reference counterpart (NULL switches them off):
 * per-cell Manning n (semi-implicit friction after the update) and a
 * per-cell multiplier of the melt rate. Full grids as for fx_upload. */
int fx_set_manning(fx_ctx* ctx, const double* n_grid);
int fx_set_melt_field(fx_ctx* ctx, const double* mult_grid);
/* Options: "store_all_fluxes" (1 keeps fe_2/fe_3/fn_2/fn_3 current on the
 * device every step; 0, the default, skips those stores for cells that end a
 * step wet, whose values are never read back by a later step);
 * "tile_rows" (4, 8 or 16: hydrodynamic tiles of 31 x (tile_rows - 1) cells,
 * 32 x tile_rows threads; default 8); "tma" (1, the default: a persistent
 * hydrodynamic kernel whose blocks stage each tile's stencil into shared
 * memory by TMA while computing the previous tile; 0: one block per tile
 * loading its stencil itself). Results depend on neither.
 * "fail_ade_waits" (1: for testing failure detection, the ADE sweep's
 * dependency waits are never satisfied, so they give up after a few
 * thousand polls, the kernels return, and the step returns FX_ERR_DEVICE
 * with fx_status.device_error set; the context then refuses further steps
 * and stays destroyable, the device stays usable). */
int fx_set_option(fx_ctx* ctx, const char* name, long long value);
int fx_prepare(fx_ctx* ctx);

/* --- stepping ------------------------------------------------------------ */
/* Run up to nsteps steps; stops early when an output is due or the run ends. */
int fx_step(fx_ctx* ctx, int nsteps, fx_status* st);
/* Run until an output is due or the run ends. */
int fx_run_to_print(fx_ctx* ctx, fx_status* st);
/* Acknowledge a due output: print_next += print_step (main.cpp:458). */
int fx_print_done(fx_ctx* ctx);
int fx_get_status(fx_ctx* ctx, fx_status* st);
/* The context's CUDA stream (a cudaStream_t), for callers that time it. */
void* fx_stream(fx_ctx* ctx);
/* Device time of n steps in milliseconds, measured with CUDA events on the
 * context's stream, plus the summed time of the hydro and ADE kernels
 * measured launch by launch (for roofline accounting). */
int fx_time_steps(fx_ctx* ctx, int nsteps, double* ms_total, double* ms_hydro, double* ms_ade);
/* Stored water sum(h) * dxy^2 over the interior cells [m^3] and, when
 * solute_mass is not NULL, the stored mass sum(conc * h) * dxy^2 of each of
 * the nchem solutes, summed on the device in FP64. With the budget of
 * fx_status, water(t) - water(0) = budget_melt - budget_out up to rounding. */
int fx_mass(fx_ctx* ctx, double* water, double* solute_mass);
/* Autotuner: runs trial_steps real steps with each tile shape (tile_rows 4,
 * 8, 16), twice (in that order, then in the reverse order, so a state that
 * grows dearer as the trials advance it favours no shape), keeps the one
 * whose hydrodynamic kernel took least time per step over both runs and
 * returns it in *tile_rows (may be NULL). */
int fx_autotune(fx_ctx* ctx, int trial_steps, int* tile_rows);

/* --- batches --------------------------------------------------------------
 * No counterpart in the reference (it runs one domain per process). A batch
 * steps several contexts together: one CUDA graph per batch of steps holds
 * the clock updates of all members, one hydrodynamic launch over all their
 * tiles per step and one ADE launch over all their solute strips, so small
 * and large domains share the GPU. Every member keeps its own clock, dt,
 * forcing and outputs, and stops on its own (output due, run over, step
 * budget spent). Members are added or removed between fx_batch_step calls;
 * while in a batch, a context is stepped only through it (its upload,
 * download and output calls stay valid between batch steps). */
typedef struct fx_batch fx_batch;
int fx_batch_create(fx_batch** out);
void fx_batch_destroy(fx_batch* b);
const char* fx_batch_last_error(const fx_batch* b);
int fx_batch_add(fx_batch* b, fx_ctx* ctx);
int fx_batch_remove(fx_batch* b, fx_ctx* ctx);
int fx_batch_size(const fx_batch* b);
/* Up to nsteps steps of every member; st (may be NULL) receives the members'
 * status in the order they were added. */
int fx_batch_step(fx_batch* b, int nsteps, fx_status* st);
void* fx_batch_stream(fx_batch* b);
/* Options of the batch's launches: "tile_rows" (4, 8, 16, as for
 * fx_set_option), "steps_in_flight" (upper bound on the steps per graph,
 * 1..63; the members' own steps_in_flight bound it too) and "tma" (1, the
 * default: the persistent TMA-staged hydrodynamic kernel when every member
 * allows it; 0: one block per tile; results are identical). */
int fx_batch_set_option(fx_batch* b, const char* name, long long value);
/* Autotuner of the batch: tries each tile shape, then each steps-in-flight
 * bound (2, 4, 8, 16, 31, 63, up to the members' own), for trial_steps real
 * steps of all members (at least 2 x the bound), each twice (in that order,
 * then in the reverse order), keeps the fastest over both runs (time per
 * cell-step) and returns the choice (pointers may be NULL). */
int fx_batch_autotune(fx_batch* b, int trial_steps, int* tile_rows, int* steps_in_flight);

/* --- allocation-free ADE sweep -------------------------------------------
 * No counterpart in the reference. For callers that cannot call cudaMalloc
 * (their device memory comes from their own pool or arena, or they run
 * inside a fixed memory budget): one ADE step, ADEsolver_calc for one solute
 * with it > 1, applied in place to `conc` on device arrays the caller owns.
 * Arrays hold (nrows+2) x (ncols+2) cells; cell (irow, icol) is element
 * icol*ld + irow + 1 (ld >= nrows+3, ld*(ncols+2) a multiple of 4; conc
 * 16-byte aligned, the other grids 8-byte, flags 4-byte); `flags`
 * holds one byte per cell: bit 0 ldry, bit 1 ldry_prev, bit 2 wall. h, h0,
 * fe_1, fn_1 are the depth after and before the hydrodynamic update and the
 * face fluxes of that update; dtfl is its time step. The call allocates
 * nothing: its scratch is one static 8 MiB device array per GPU. A grid fits
 * when ceil(nrows/30) * (ncols+2) * 24 bytes plus a fixed part of a few KiB
 * is at most 8 MiB (square grids up to about 3,200 x 3,200 cells); larger
 * grids return FX_ERR_ARG. The first call on a device (and the first after
 * its CUDA context is replaced, e.g. by cudaDeviceReset) looks up that
 * array's device address; make the first call before any stream capture.
 * All calls share the array and calls that overlap on the GPU race. stream
 * NULL = the default stream; the call synchronises the stream and returns
 * when the sweep has finished. */
int fx_adesolver_noalloc(double* conc, const double* h, const double* h0, const unsigned char* flags,
                         const double* fe_1, const double* fn_1, int nrows, int ncols, int ld, int dxy,
                         double dtfl, double d_coef, void* stream);

/* --- the reference's file surface (host C++) ---------------------------- */
/* read_geo's wall/roughness step (read_functions.cpp:175-225) and the zero
 * initial state of initiation (initiate.cpp:43-107,159-228) from the DEM
 * values as read (float-rounded, GlobVar layout, ghost ring 0); uploads the
 * state and runs fx_prepare. */
int fx_initiate(fx_ctx* ctx, const double* zb_raw);
/* Host-only part of the start-up below (no GPU needed): parse the modset,
 * DEM and forcing files and build the initial state exactly as main.cpp:
 * 104-262 does. Call once with all array pointers NULL to fill g and p (the
 * sizes), then with arrays of (nrows+2)*(ncols+2) elements and a 3*2000
 * forcing table. */
int fx_load_modset(const char* modset_path, fx_grid* g, fx_params* p, double* zb, double* z,
                   double* h, double* qx, double* qy, double* twet, double* conc, double* soil_mass,
                   float* ldry, float* wall, float* table_2000x3, int* has_meteo);
/* Start-up of main.cpp:87-262 from a modset file: reads the master file
 * (with comments), the ESRI ASCII DEM, the forcing CSV, applies initiation
 * (bed averaging, zero or restart initial state, ghost ring), uploads. */
int fx_open_modset(const char* modset_path, fx_ctx** out);
/* write_results (write_results.cpp:30-101): Results/<t>.txt of the current
 * state; path NULL means <OUTPUT_FOLDER>/<print_next>.txt. */
int fx_write_results(fx_ctx* ctx, const char* path);
/* The same file written while the context keeps stepping: the selected
 * rows are compacted on the device (cells with zb != 0 and h >
 * H_MIN_TO_PRINT, in the file's order) on the context's stream, copied to
 * pinned memory on a second stream, and formatted and written by a host
 * thread. Returns once the rows are placed; the state may then be stepped.
 * fx_results_wait waits for every file started and returns the first error
 * (FX_ERR_IO when a file could not be written); fx_destroy waits too. The
 * row buffer (80 bytes per printed cell) is held on the device until
 * fx_destroy and is counted by fx_device_bytes, not by fx_footprint. */
int fx_write_results_async(fx_ctx* ctx, const char* path);
int fx_results_wait(fx_ctx* ctx);
/* The writer itself on host grids (no GPU needed); soil_mass may be NULL
 * (a column of zeros). */
int fx_write_results_host(const char* path, int nrows, int ncols, int dxy, double xll, double yll,
                          double h_min_print, const double* z, const double* zb, const double* h,
                          const double* qx, const double* qy, const double* conc,
                          const double* soil_mass, const double* fe_1, const double* fn_1,
                          const double* twet);
/* The whole program: open, step, write every output, close. */
int fx_run(const char* modset_path);

#ifdef __cplusplus
}
#endif
#endif
