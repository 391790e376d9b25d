// Host-side definition of fx_ctx, shared by the C ABI (fx_capi.cu) and the
// file surface (host/fluxos_io.cpp). Not part of the public header.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "fluxos_gpu.h"
#include "fx_common.cuh"

struct fx_ctx {
  fx_grid g{};
  fx_params p{};
  fx_dev d{};
  cudaStream_t stream = nullptr;
  fx_ctl* ctl_host = nullptr;  // pinned mirror of the device control block
  long long stop_host = 0;     // pinned-free staging for the stop field
  std::string err;
  std::vector<void*> allocs;
  long long bytes = 0;
  int ade_strips = 0;
  int ade_blocks = 0;
  int batch_steps = 1;         // steps per batch (ADE sweeps in flight)
  fx_dev* d_dev = nullptr;     // device copy of d (a batch of one domain)
  fx_tile* d_tiles = nullptr;  // this domain's hydrodynamic tiles
  int ntiles = 0, nunits = 0;  // hydrodynamic tiles; ADE units of a full batch
  bool dev_dirty = true;       // d changed since it was copied to d_dev
  long long dev_version = 0;   // counts changes of d (batches compare it)
  bool prepared = false;
  bool graph_dirty = true;
  bool store_all_opt = false;
  bool negative_forcing = false;
  cudaGraphExec_t graph_exec = nullptr;
  // FP32 state: host grids (FP64) cross to and from the device through
  // `stage`, one FP64 plane in the field layout, and are converted there by
  // kernels; z is held as eta = z - zb, so an uploaded z (or the z of the
  // state when zb is replaced) waits in `zstage` until fx_prepare converts
  // it with the bed then current (`z_pending`).
  double* stage = nullptr;
  double* zstage = nullptr;
  bool z_pending = false;
  double* d_mass = nullptr;    // fx_mass result: water, then one mass per solute
  // TMA-staged hydrodynamic kernel (one domain): tensor maps of the stencil
  // fields, rebuilt with the descriptor; its persistent grid size
  fx_tmaps tmaps{};
  bool use_tma = true;
  int tma_blocks = 0;
  // file surface (filled by fx_open_modset)
  double h_min_print = 0.0;
  std::string output_folder;
  // Results writer state (fluxos_io.cpp): device scratch of the row
  // compaction, pinned buffers and the writer threads; released by
  // fx_results_release
  struct fx_results_state* res = nullptr;
};

int fx_fail(fx_ctx* ctx, int code, const char* fmt, ...);
void fx_results_release(fx_ctx* ctx);  // waits for pending Results files, frees the writer's buffers
int fx_sync_dev(fx_ctx* ctx);
void fx_fill_status(const fx_ctl& k, fx_status* st);

// Launch helpers (fx_hydro.cu, fx_ade.cu). `devs` is a device array of
// domain descriptors; the *_one forms take one domain's descriptor by value.
void fx_launch_finalize(const fx_dev* devs, int ndom, cudaStream_t s);
void fx_launch_batch_begin(const fx_dev* devs, int ndom, cudaStream_t s);
// plane: the domain's elements per field (fx_dev::plane)
void fx_launch_mark_static(const fx_dev* devs, int dom, long long plane, cudaStream_t s);
void fx_launch_hydro(const fx_dev* devs, const fx_tile* tiles, int ntiles, bool prec32, int tile_rows,
                     cudaStream_t s);
void fx_launch_hydro_one(const fx_dev& d, cudaStream_t s);
void fx_launch_hydro_tma(const fx_dev& d, const fx_tmaps& tm, int nblocks, cudaStream_t s);
int fx_hydro_tma_blocks(bool prec32, int tile_rows, int* out);
void fx_launch_hydro_batch_tma(const fx_dev* devs, const fx_tmaps* tms, const fx_tile* tiles, int ntiles,
                               int nblocks, bool prec32, int tile_rows, cudaStream_t s);
int fx_hydro_batch_tma_blocks(bool prec32, int tile_rows, int* out);
// Tensor maps of a context's stencil fields for a tile shape (fx_capi.cu).
int fx_build_tmaps_for(fx_ctx* c, int tile_rows, fx_tmaps* out);
bool fx_tma_fits(const fx_ctx* c, int tile_rows);
void fx_launch_courant_scan(const fx_dev* devs, const fx_tile* tiles, int ntiles, int tile_rows, cudaStream_t s);
void fx_launch_ade(const fx_dev* devs, const fx_unit* units, int nunits, int nblocks, bool prec32, cudaStream_t s);
void fx_launch_ade_one(const fx_dev& d, int nunits, int nblocks, cudaStream_t s);
void fx_launch_eta_from_z(const fx_dev& d, const double* z, cudaStream_t s);
void fx_launch_mass(const fx_dev& d, double* out, cudaStream_t s);
void fx_tiles_of(int dom, int nr, int nc, int tile_rows, std::vector<fx_tile>& out);
// Results rows on the device (fx_results.cu): per-column counts (nc
// unsigned) and their exclusive scan (nc + 1 long long, the total last);
// then the rows as column arrays in `buf`: irow, icol (int32) and
// FX_RES_NVAL FP64 columns, `total` entries each.
#define FX_RES_NVAL 9
void fx_launch_results_count(const fx_dev& d, double h_min_print, unsigned* counts, long long* offs,
                             cudaStream_t s);
void fx_launch_results_write(const fx_dev& d, double h_min_print, const long long* offs, void* buf,
                             long long total, cudaStream_t s);
bool fx_tile_rows_ok(int tile_rows);
void fx_units_of(int dom, int nr, int nchem, int steps, std::vector<fx_unit>& out);
int fx_ade_rows_per_strip();
int fx_ade_threads_per_block();
int fx_ade_max_blocks(int* out);
int fx_ade_max_blocks_for(bool prec32, int* out);
