// C ABI of libfluxos_gpu.so: context, device state, stepping (see
// include/fluxos_gpu.h for the contract and the reference interfaces each
// entry point replaces).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "fluxos_gpu.h"
#include "fx_common.cuh"
#include "fx_internal.h"

static thread_local std::string g_last_error;

static const unsigned long long kInfBits = 0x7ff0000000000000ull;

int fx_fail(fx_ctx* ctx, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = buf;
  g_last_error = buf;
  return code;
}

#define FX_CK(ctx, call)                                                                   \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return fx_fail(ctx, e_ == cudaErrorMemoryAllocation ? FX_ERR_NOMEM : FX_ERR_CUDA,    \
                     "%s failed: %s", #call, cudaGetErrorString(e_));                      \
  } while (0)

// A state field on the device: its planes (one per slot for the fields the
// ADE sweep reads after later steps, see fx_common.cuh), its element type.
struct FieldRef {
  void* ptr = nullptr;
  bool f32 = false;   // float (FP32 state) instead of double
  bool slot = false;  // one plane per slot
  bool pair = false;  // two planes, the current one is fx_pp(steps)
  int copies = 1;     // identical planes (the soil mass: one per solute)
  int rec = -1;       // per-step field: its component of the slot records (FX_R64_* or FX_R_*)
};

static FieldRef field_ref(fx_ctx* c, const char* name) {
  fx_dev& d = c->d;
  FieldRef r;
  const bool p32 = d.prec32 != 0;
  auto pick = [&](void* p64, void* p32v, bool slot, bool pair = false) {
    r.ptr = p32 ? p32v : p64;
    r.f32 = p32;
    r.slot = slot;
    r.pair = pair;
  };
  // a per-step field: a component of the slot records (FP64 rec64, FP32 rec32)
  auto pick_rec = [&](int comp64, int comp32) {
    pick(d.rec64, d.rec32, true);
    r.rec = p32 ? comp32 : comp64;
  };
  if (!strcmp(name, "zb")) r.ptr = d.zb;  // FP64 in both forms
  else if (!strcmp(name, "z")) {
    if (!p32) pick(d.z, nullptr, false, true);  // FP32: held as eta, see fx_upload / fx_download
  } else if (!strcmp(name, "h")) pick_rec(FX_R64_H, FX_R_H);
  else if (!strcmp(name, "qx")) pick(d.qx, d.qx_f, false, true);
  else if (!strcmp(name, "qy")) pick(d.qy, d.qy_f, false, true);
  else if (!strcmp(name, "twet")) pick(d.twet, d.twet_f, false);
  else if (!strcmp(name, "h0")) pick_rec(FX_R64_H0, FX_R_H0);
  else if (!strcmp(name, "fe_1")) pick_rec(FX_R64_FE1, FX_R_FE1);
  else if (!strcmp(name, "fe_2")) pick(d.fe2, d.fe2_f, false);
  else if (!strcmp(name, "fe_3")) pick(d.fe3, d.fe3_f, false);
  else if (!strcmp(name, "fn_1")) pick_rec(FX_R64_FN1, FX_R_FN1);
  else if (!strcmp(name, "fn_2")) pick(d.fn2, d.fn2_f, false);
  else if (!strcmp(name, "fn_3")) pick(d.fn3, d.fn3_f, false);
  else if (!strncmp(name, "conc", 4)) {
    int k = name[4] ? atoi(name + 4) : 0;
    if (k >= 0 && k < d.nchem)
      pick(d.conc ? d.conc + (long long)k * d.plane : nullptr,
           d.conc_f ? d.conc_f + (long long)k * d.plane : nullptr, false);
  } else if (!strcmp(name, "soil_mass")) {
    pick(d.soil, d.soil_f, false);
    r.copies = d.nchem;
  }
  return r;
}

// "soil_mass" is allocated with the WINTRA module or by its first upload;
// until then it reads as zeros.
static bool known_field(fx_ctx* c, const char* name) {
  return !strcmp(name, "z") || !strcmp(name, "soil_mass") || field_ref(c, name).ptr != nullptr;
}

static int dev_alloc(fx_ctx* c, void** p, size_t bytes);

static int alloc_soil(fx_ctx* c) {
  fx_dev& d = c->d;
  if (d.soil || d.soil_f) return FX_OK;
  const size_t bytes = (size_t)d.plane * d.nchem * (d.prec32 ? sizeof(float) : sizeof(double));
  int rc = d.prec32 ? dev_alloc(c, (void**)&d.soil_f, bytes) : dev_alloc(c, (void**)&d.soil, bytes);
  if (rc) return rc;
  c->graph_dirty = true;
  c->dev_dirty = true;
  c->dev_version++;
  return FX_OK;
}

static int dev_alloc(fx_ctx* c, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return fx_fail(c, FX_ERR_NOMEM, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
  }
  c->allocs.push_back(*p);
  c->bytes += (long long)bytes;
  e = cudaMemsetAsync(*p, 0, bytes, c->stream);
  if (e != cudaSuccess) return fx_fail(c, FX_ERR_CUDA, "cudaMemsetAsync failed: %s", cudaGetErrorString(e));
  return FX_OK;
}

static int read_ctl(fx_ctx* c) {
  FX_CK(c, cudaMemcpyAsync(c->ctl_host, c->d.ctl, sizeof(fx_ctl), cudaMemcpyDeviceToHost, c->stream));
  FX_CK(c, cudaStreamSynchronize(c->stream));
  return FX_OK;
}

void fx_fill_status(const fx_ctl& k, fx_status* st) {
  if (!st) return;
  st->tim = k.tim;
  st->dtfl = k.dtfl;
  st->print_next = k.print_next;
  st->hpall = k.hpall;
  st->steps = k.steps;
  st->it = k.it;
  st->print_pending = k.print_pending;
  st->finished = k.finished;
  st->device_error = k.error;
  st->forcing_overrun = k.forcing_overrun;
  st->budget_melt = k.budget_melt;  // melt and point inflow
  st->budget_out = k.budget_out;
}

// cuTensorMapEncodeTiled from the driver (the runtime links statically; the
// entry point is looked up once).
static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// One stencil field as a 3-D tensor (irow incl. the column padding, icol,
// plane) with a box of `box_x` x (tile_rows + 2) x 1 elements.
static int encode_field(fx_ctx* c, fx_tmap* out, const void* base, CUtensorMapDataType type, int esz,
                        int planes, int box_x, int tile_rows) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
  if (!enc) return fx_fail(c, FX_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  const fx_dev& d = c->d;
  cuuint64_t dims[3] = {(cuuint64_t)d.ld, (cuuint64_t)(d.nc + 2), (cuuint64_t)planes};
  cuuint64_t strides[2] = {(cuuint64_t)d.ld * esz, (cuuint64_t)d.plane * esz};
  cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)(tile_rows + 2), 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(reinterpret_cast<CUtensorMap*>(out), type, 3, const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fx_fail(c, FX_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return FX_OK;
}

// Tensor maps of the TMA-staged hydrodynamic kernels for the current fields
// and a tile shape (box widths: 40 4-byte, 36 8-byte, 64 1-byte elements).
int fx_build_tmaps_for(fx_ctx* c, int tile_rows, fx_tmaps* out) {
  const fx_dev& d = c->d;
  fx_tmap* m = out->m;
  const int r = tile_rows;
  int rc;
  const CUtensorMapDataType F32 = CU_TENSOR_MAP_DATA_TYPE_FLOAT32, F64 = CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  if (d.prec32) {
    if ((rc = encode_field(c, &m[FX_TM_Z], d.eta, F32, 4, 2, 40, r)) ||
        (rc = encode_field(c, &m[FX_TM_LO], d.eta_lo, F32, 4, 2, 40, r)) ||
        (rc = encode_field(c, &m[FX_TM_QX], d.qx_f, F32, 4, 2, 40, r)) ||
        (rc = encode_field(c, &m[FX_TM_QY], d.qy_f, F32, 4, 2, 40, r)) ||
        (rc = encode_field(c, &m[FX_TM_MM], d.melt_mult_f ? (const void*)d.melt_mult_f : (const void*)d.eta, F32, 4,
                           1, 40, r)))
      return rc;
  } else {
    if ((rc = encode_field(c, &m[FX_TM_Z], d.z, F64, 8, 2, 36, r)) ||
        (rc = encode_field(c, &m[FX_TM_LO], d.z, F64, 8, 2, 36, r)) ||
        (rc = encode_field(c, &m[FX_TM_QX], d.qx, F64, 8, 2, 36, r)) ||
        (rc = encode_field(c, &m[FX_TM_QY], d.qy, F64, 8, 2, 36, r)) ||
        (rc = encode_field(c, &m[FX_TM_MM], d.melt_mult ? (const void*)d.melt_mult : (const void*)d.z, F64, 8, 1,
                           36, r)))
      return rc;
  }
  if ((rc = encode_field(c, &m[FX_TM_ZB], d.zb, F64, 8, 1, 36, r)) ||
      (rc = encode_field(c, &m[FX_TM_FL], d.flags, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, d.nslot, 64, r)))
    return rc;
  return FX_OK;
}

// The context's own maps (its tile shape) and the resident blocks of its
// persistent launch.
static int build_tmaps(fx_ctx* c) {
  int rc = fx_build_tmaps_for(c, c->d.tile_rows, &c->tmaps);
  if (rc) return rc;
  if (fx_hydro_tma_blocks(c->d.prec32 != 0, c->d.tile_rows, &c->tma_blocks) != 0 || c->tma_blocks < 1)
    return fx_fail(c, FX_ERR_CUDA, "occupancy query for the TMA-staged hydrodynamic kernel failed");
  return FX_OK;
}

static bool tma_fits(const fx_ctx* c);

// Copies the host descriptor of the domain to its device copy when it
// changed, and rebuilds the tensor maps that point into its fields.
int fx_sync_dev(fx_ctx* c) {
  if (!c->dev_dirty) return FX_OK;
  FX_CK(c, cudaMemcpyAsync(c->d_dev, &c->d, sizeof(fx_dev), cudaMemcpyHostToDevice, c->stream));
  FX_CK(c, cudaStreamSynchronize(c->stream));
  if (c->use_tma && tma_fits(c)) {
    int rc = build_tmaps(c);
    if (rc) return rc;
  }
  c->dev_dirty = false;
  return FX_OK;
}

// Hydrodynamic tiles of 32 x r threads: the tile table and the descriptor.
static int set_tile_rows(fx_ctx* c, int r) {
  if (!fx_tile_rows_ok(r)) return fx_fail(c, FX_ERR_ARG, "tile_rows must be 4, 8 or 16 (got %d)", r);
  std::vector<fx_tile> tiles;
  fx_tiles_of(0, c->d.nr, c->d.nc, r, tiles);
  FX_CK(c, cudaMemcpyAsync(c->d_tiles, tiles.data(), sizeof(fx_tile) * tiles.size(), cudaMemcpyHostToDevice,
                           c->stream));
  FX_CK(c, cudaStreamSynchronize(c->stream));
  c->ntiles = (int)tiles.size();
  c->d.tile_rows = r;
  c->graph_dirty = true;
  c->dev_dirty = true;
  c->dev_version++;
  return FX_OK;
}

extern "C" {

const char* fx_last_error(const fx_ctx* ctx) { return ctx ? ctx->err.c_str() : g_last_error.c_str(); }

// Steps in flight when the caller leaves it to the library: as many as the
// per-step planes of h, h0, the pre-melt depth, fe_1, fn_1 and flags allow
// within 1 GiB, at least 8 and at most 63. A launch of the ADE sweep pays the
// wavefront's start-up (the strips and columns of the grid, once), so small
// grids, whose sweeps are short, run far faster with many steps per launch;
// large grids keep 8 (and the memory).
static int default_steps_in_flight(long long plane, bool prec32) {
  // per slot: a 32-byte (FP32) or 48-byte (FP64) record per cell, and a flag byte
  const long long per_step = plane * ((prec32 ? 32LL : 48LL) + 1);
  const long long k = per_step > 0 ? (1LL << 30) / per_step : FX_MAX_SLOTS - 1;
  return (int)std::max(8LL, std::min<long long>(FX_MAX_SLOTS - 1, k));
}

int fx_create(const fx_grid* g, const fx_params* p, fx_ctx** out) {
  if (!g || !p || !out) return fx_fail(nullptr, FX_ERR_ARG, "fx_create: null argument");
  *out = nullptr;
  if (g->nrows < 2 || g->ncols < 2)
    return fx_fail(nullptr, FX_ERR_ARG, "fx_create: need nrows, ncols >= 2 (got %d x %d)", g->nrows,
                   g->ncols);
  if (g->nchem < 1 || g->nchem > FX_MAX_CHEM)
    return fx_fail(nullptr, FX_ERR_ARG, "fx_create: nchem must be 1..%d", FX_MAX_CHEM);
  if (g->dxy < 1) return fx_fail(nullptr, FX_ERR_ARG, "fx_create: dxy must be a positive integer");
  if ((long long)g->nrows * g->ncols > (1LL << 31))
    return fx_fail(nullptr, FX_ERR_ARG, "fx_create: grid larger than 2^31 cells");
  fx_ctx* c = new fx_ctx();
  c->g = *g;
  c->p = *p;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    fx_fail(nullptr, FX_ERR_CUDA, "cudaStreamCreate failed: %s", cudaGetErrorString(e));
    delete c;
    return FX_ERR_CUDA;
  }
  fx_dev& d = c->d;
  memset(&d, 0, sizeof(d));
  d.inflow_gi = -1;
  d.nr = g->nrows;
  d.nc = g->ncols;
  d.nchem = g->nchem;
  d.ld = ((g->nrows + 2 + FX_ROFF + 31) / 32) * 32;
  d.plane = (long long)d.ld * (g->ncols + 2);
  fx_set_cell_size(d, g->dxy);
  d.hdry = p->hdry;
  d.ks = p->ks;
  d.nodata = g->nodata;
  const float gacc = 9.80665f, cfl = 1.0f, cvdef = 0.07f, nuem = 1.793e-6f;  // main.cpp:132-135
  d.gaccl = (double)gacc;
  d.sqrt_gaccl = std::sqrt(d.gaccl);
  d.nueml = (double)nuem;
  d.cvdefl = (double)cvdef;
  d.cfl_dxy = (double)(cfl * (float)g->dxy);
  d.volrat_mode = p->volrat_mode;
  d.ade = p->ade;
  d.wintra = (p->wintra && p->ade) ? 1 : 0;  // main.cpp:209-213
  d.soil_rate = p->soil_release_rate;
  for (int k = 0; k < FX_MAX_CHEM; ++k) d.dcoef[k] = p->d_coef[k];
  {
    int k = p->steps_in_flight > 0 ? p->steps_in_flight : default_steps_in_flight(d.plane, p->precision == 1);
    if (k > FX_MAX_SLOTS - 1) k = FX_MAX_SLOTS - 1;
    d.nslot = k + 1;  // a batch of k steps plus the state before it
    c->batch_steps = k;
  }
  int rc = FX_OK;
  if (p->precision != 0 && p->precision != 1) {
    rc = fx_fail(c, FX_ERR_ARG, "fx_create: precision must be 0 (FP64) or 1 (FP32)");
    goto fail;
  }
  d.prec32 = p->precision;
  if (!d.prec32) {
    const size_t pb = (size_t)d.plane * sizeof(double);
    double** fields[] = {&d.zb, &d.twet, &d.fe2, &d.fe3, &d.fn2, &d.fn3};
    double** pair_fields[] = {&d.z, &d.qx, &d.qy};
    for (double** f : fields)
      if ((rc = dev_alloc(c, (void**)f, pb)) != FX_OK) goto fail;
    for (double** f : pair_fields)
      if ((rc = dev_alloc(c, (void**)f, 2 * pb)) != FX_OK) goto fail;
    if ((rc = dev_alloc(c, (void**)&d.rec64, pb * FX_R64_N * d.nslot)) != FX_OK) goto fail;
    // staging plane of the per-step fields' uploads and downloads
    if ((rc = dev_alloc(c, (void**)&c->stage, pb)) != FX_OK) goto fail;
    if ((rc = dev_alloc(c, (void**)&d.conc, pb * g->nchem)) != FX_OK) goto fail;
  } else {
    const size_t pf = (size_t)d.plane * sizeof(float);
    float** fields[] = {&d.twet_f, &d.fe2_f, &d.fe3_f, &d.fn2_f, &d.fn3_f};
    float** pair_fields[] = {&d.eta, &d.eta_lo, &d.qx_f, &d.qy_f};
    if ((rc = dev_alloc(c, (void**)&d.zb, (size_t)d.plane * sizeof(double))) != FX_OK) goto fail;
    for (float** f : fields)
      if ((rc = dev_alloc(c, (void**)f, pf)) != FX_OK) goto fail;
    for (float** f : pair_fields)
      if ((rc = dev_alloc(c, (void**)f, 2 * pf)) != FX_OK) goto fail;
    if ((rc = dev_alloc(c, (void**)&d.rec32, (size_t)d.plane * d.nslot * 2 * sizeof(float4))) != FX_OK) goto fail;
    if ((rc = dev_alloc(c, (void**)&d.conc_f, pf * g->nchem)) != FX_OK) goto fail;
    if ((rc = dev_alloc(c, (void**)&c->stage, (size_t)d.plane * sizeof(double))) != FX_OK) goto fail;
    if ((rc = dev_alloc(c, (void**)&c->zstage, (size_t)d.plane * sizeof(double))) != FX_OK) goto fail;
  }
  if (d.wintra && (rc = alloc_soil(c)) != FX_OK) goto fail;
  if ((rc = dev_alloc(c, (void**)&c->d_mass, sizeof(double) * (1 + FX_MAX_CHEM))) != FX_OK) goto fail;
  if ((rc = dev_alloc(c, (void**)&d.flags, (size_t)d.plane * d.nslot)) != FX_OK) goto fail;
  if ((rc = dev_alloc(c, (void**)&d.ctl, sizeof(fx_ctl))) != FX_OK) goto fail;
  {
    float* tab = nullptr;
    if ((rc = dev_alloc(c, (void**)&tab, sizeof(float) * 3 * FX_METEO_ROWS)) != FX_OK) goto fail;
    d.meteo_t = tab;
    d.meteo_r = tab + FX_METEO_ROWS;
    d.meteo_c = tab + 2 * FX_METEO_ROWS;
  }
  c->ade_strips = (g->nrows + fx_ade_rows_per_strip() - 1) / fx_ade_rows_per_strip();
  if ((rc = dev_alloc(c, (void**)&d.ade_bnd,
                      sizeof(double) * (size_t)d.nslot * g->nchem * c->ade_strips * (g->ncols + 2) * 3)) != FX_OK)
    goto fail;
  if ((rc = dev_alloc(c, (void**)&d.ade_prog,
                      sizeof(unsigned long long) * (size_t)d.nslot * g->nchem * c->ade_strips)) != FX_OK)
    goto fail;
  {
    int maxb = 0;
    if (fx_ade_max_blocks_for(d.prec32 != 0, &maxb) != 0 || maxb < 1) {
      rc = fx_fail(c, FX_ERR_CUDA, "occupancy query for the ADE sweep failed");
      goto fail;
    }
    const int units = c->batch_steps * g->nchem * c->ade_strips;
    const int per_block = fx_ade_threads_per_block() / 32;
    int want = (units + per_block - 1) / per_block;
    c->ade_blocks = want < maxb ? want : maxb;
  }
  {
    // this domain's tile table (domain 0 of a batch of one), sized for the
    // smallest tiles (most entries)
    std::vector<fx_tile> tiles;
    fx_tiles_of(0, g->nrows, g->ncols, 4, tiles);
    c->nunits = c->batch_steps * g->nchem * c->ade_strips;
    if ((rc = dev_alloc(c, (void**)&c->d_tiles, sizeof(fx_tile) * tiles.size())) != FX_OK) goto fail;
    if ((rc = dev_alloc(c, (void**)&c->d_dev, sizeof(fx_dev))) != FX_OK) goto fail;
    if ((rc = set_tile_rows(c, 8)) != FX_OK) goto fail;
  }
  e = cudaMallocHost((void**)&c->ctl_host, sizeof(fx_ctl));
  if (e != cudaSuccess) {
    rc = fx_fail(c, FX_ERR_CUDA, "cudaMallocHost failed: %s", cudaGetErrorString(e));
    goto fail;
  }
  memset(c->ctl_host, 0, sizeof(fx_ctl));
  c->ctl_host->tim = p->tim;
  c->ctl_host->ntim = p->ntim;
  c->ctl_host->print_next = p->print_next;
  c->ctl_host->print_step = p->print_step;
  c->ctl_host->acc_dtmin = kInfBits;
  c->ctl_host->stop_after = 0;
  e = cudaMemcpyAsync(d.ctl, c->ctl_host, sizeof(fx_ctl), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    rc = fx_fail(c, FX_ERR_CUDA, "control block upload failed: %s", cudaGetErrorString(e));
    goto fail;
  }
  c->h_min_print = p->h_min_print;
  if ((rc = fx_sync_dev(c)) != FX_OK) goto fail;
  *out = c;
  return FX_OK;
fail:
  g_last_error = c->err;
  fx_destroy(c);
  return rc;
}

void fx_destroy(fx_ctx* c) {
  if (!c) return;
  fx_results_release(c);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  for (void* p : c->allocs) cudaFree(p);
  if (c->ctl_host) cudaFreeHost(c->ctl_host);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int fx_device_bytes(const fx_ctx* c, long long* bytes) {
  if (!c || !bytes) return FX_ERR_ARG;
  *bytes = c->bytes;
  return FX_OK;
}

int fx_footprint(const fx_grid* g, const fx_params* p, int extension_grids, long long* bytes) {
  if (!g || !p || !bytes || g->nrows < 2 || g->ncols < 2 || g->nchem < 1 || g->nchem > FX_MAX_CHEM)
    return fx_fail(nullptr, FX_ERR_ARG, "fx_footprint: bad argument");
  // the allocations of fx_create, field by field, plus the extension grids
  const long long ld = ((g->nrows + 2 + FX_ROFF + 31) / 32) * 32;
  const long long plane = ld * (g->ncols + 2);
  long long k = p->steps_in_flight > 0 ? p->steps_in_flight : default_steps_in_flight(plane, p->precision == 1);
  if (k > FX_MAX_SLOTS - 1) k = FX_MAX_SLOTS - 1;
  const long long nslot = k + 1;
  const long long strips = (g->nrows + fx_ade_rows_per_strip() - 1) / fx_ade_rows_per_strip();
  const long long gx = (g->nrows + 30) / 31, gy = (g->ncols + 6) / 7;
  long long b = 0;
  if (p->precision == 1)  // zb, twet and the flux fields, pairs, slot records, solutes, extensions, 2 staging planes
    b += plane * (8 + 5 * 4 + 4 * 2 * 4 + 32 * nslot + 4LL * g->nchem + 4LL * extension_grids + 16);
  else
    b += plane * (6 * 8 + 3 * 2 * 8 + 48 * nslot + 8LL * g->nchem + 8LL * extension_grids + 8);  // + staging
  if (p->wintra && p->ade) b += plane * g->nchem * (p->precision == 1 ? 4 : 8);  // soil mass
  b += plane * nslot;                                   // flags
  b += (long long)sizeof(fx_ctl) + 3 * FX_METEO_ROWS * 4 + (long long)sizeof(fx_dev);
  b += 8LL * nslot * g->nchem * strips * (g->ncols + 2) * 3 + 8LL * nslot * g->nchem * strips;
  b += (long long)sizeof(fx_tile) * gx * gy + (long long)sizeof(fx_unit) * k * g->nchem * strips;
  b += 8LL * (1 + FX_MAX_CHEM);
  *bytes = b;
  return FX_OK;
}

// Copies a host grid (double, GlobVar layout) into `planes` consecutive
// planes of a device field, converting to float for FP32 fields.
// Elementwise conversions over whole planes in the field layout (the
// padding rows are 0 on both sides and stay 0).
__global__ void k_f64_to_f32(const double* __restrict__ src, float* __restrict__ dst, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = (float)src[i];
}
__global__ void k_f32_to_f64(const float* __restrict__ src, double* __restrict__ dst, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}
// Per-step field `comp` of the slot records (R = float: rec32, 8 floats a
// cell; R = double: rec64, 6 doubles a cell) from an FP64 plane: the current
// slot's, and the ghost ring's in every slot. Nothing reads another slot's
// interior before a step has written it (a step writes its slot's interior
// records; the ADE sweep reads the slots of the steps it sweeps), while the
// ghost ring is never written by a step.
extern "C++" {
template <class R, int N>
__global__ void k_rec_put(const __grid_constant__ fx_dev d, R* __restrict__ rec, const double* __restrict__ src,
                          int comp, int cur) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < d.plane;
       i += (long long)gridDim.x * blockDim.x) {
    const R v = (R)src[i];
    rec[N * ((long long)cur * d.plane + i) + comp] = v;
    const int icol = (int)(i / d.ld), irow = (int)(i - (long long)icol * d.ld) - FX_ROFF;
    if (irow < 0 || irow > d.nr + 1) continue;  // padding
    if (irow == 0 || irow == d.nr + 1 || icol == 0 || icol == d.nc + 1)
      for (int k = 0; k < d.nslot; ++k)
        if (k != cur) rec[N * ((long long)k * d.plane + i) + comp] = v;
  }
}
template <class R, int N>
__global__ void k_rec_get(const R* __restrict__ rec, int comp, double* __restrict__ dst, long long plane) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane; i += (long long)gridDim.x * blockDim.x)
    dst[i] = (double)rec[N * i + comp];
}
}  // extern "C++"
// z = zb + (eta + eta_lo) of the FP32 state (the order of get_z32's host sum before).
__global__ void k_z_of_eta(const double* __restrict__ zb, const float* __restrict__ eta,
                           const float* __restrict__ lo, double* __restrict__ z, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    z[i] = zb[i] + ((double)eta[i] + (double)lo[i]);
}
static int plane_grid(long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 16); }

// Host grid (FP64, GlobVar layout) -> device plane in the field layout: one
// pitched copy, straight into an FP64 field, or into the staging plane and
// converted on the device for an FP32 field.
static int copy_in(fx_ctx* c, double* dst64, const double* host) {
  const int mr = c->d.nr + 2, mc = c->d.nc + 2;
  FX_CK(c, cudaMemcpy2DAsync(dst64 + FX_ROFF, (size_t)c->d.ld * sizeof(double), host, (size_t)mr * sizeof(double),
                             (size_t)mr * sizeof(double), (size_t)mc, cudaMemcpyHostToDevice, c->stream));
  return FX_OK;
}
static int copy_out(fx_ctx* c, double* host, const double* src64) {
  const int mr = c->d.nr + 2, mc = c->d.nc + 2;
  FX_CK(c, cudaMemcpy2DAsync(host, (size_t)mr * sizeof(double), src64 + FX_ROFF, (size_t)c->d.ld * sizeof(double),
                             (size_t)mr * sizeof(double), (size_t)mc, cudaMemcpyDeviceToHost, c->stream));
  return FX_OK;
}

static int put_grid(fx_ctx* c, void* dst, bool f32, int planes, const double* host) {
  int rc;
  if (!f32) {
    for (int k = 0; k < planes; ++k)
      if ((rc = copy_in(c, (double*)dst + k * c->d.plane, host))) return rc;
  } else {
    if ((rc = copy_in(c, c->stage, host))) return rc;
    for (int k = 0; k < planes; ++k)
      k_f64_to_f32<<<plane_grid(c->d.plane), 256, 0, c->stream>>>(c->stage, (float*)dst + k * c->d.plane,
                                                                   c->d.plane);
    FX_CK(c, cudaGetLastError());
  }
  FX_CK(c, cudaStreamSynchronize(c->stream));
  return FX_OK;
}

// Copies one plane of a device field into a host grid (double).
static int get_grid(fx_ctx* c, const void* src, bool f32, double* host) {
  int rc;
  if (!f32) {
    rc = copy_out(c, host, (const double*)src);
  } else {
    k_f32_to_f64<<<plane_grid(c->d.plane), 256, 0, c->stream>>>((const float*)src, c->stage, c->d.plane);
    FX_CK(c, cudaGetLastError());
    rc = copy_out(c, host, c->stage);
  }
  if (rc) return rc;
  FX_CK(c, cudaStreamSynchronize(c->stream));
  return FX_OK;
}

// FP32 state: the current z = zb + (eta + eta_lo) into the device plane `z`
// (field layout).
static int z32_into(fx_ctx* c, double* z) {
  int rc = read_ctl(c);
  if (rc) return rc;
  const long long pp = fx_pp(c->d, c->ctl_host->steps);
  k_z_of_eta<<<plane_grid(c->d.plane), 256, 0, c->stream>>>(c->d.zb, c->d.eta + pp, c->d.eta_lo + pp, z,
                                                            c->d.plane);
  FX_CK(c, cudaGetLastError());
  return FX_OK;
}

// FP32 state: z on the host (the z still waiting for fx_prepare, if any).
static int get_z32(fx_ctx* c, double* host) {
  int rc;
  if (!c->z_pending && (rc = z32_into(c, c->stage))) return rc;
  if ((rc = copy_out(c, host, c->z_pending ? c->zstage : c->stage))) return rc;
  FX_CK(c, cudaStreamSynchronize(c->stream));
  return FX_OK;
}

int fx_upload(fx_ctx* c, const char* field, const double* host) {
  if (!c || !field || !host) return fx_fail(c, FX_ERR_ARG, "fx_upload: null argument");
  if (!known_field(c, field)) return fx_fail(c, FX_ERR_ARG, "fx_upload: unknown field '%s'", field);
  int rc;
  if (c->d.prec32 && !strcmp(field, "z")) {
    // converted by fx_prepare with the bed then current
    if ((rc = copy_in(c, c->zstage, host))) return rc;
    FX_CK(c, cudaStreamSynchronize(c->stream));
    c->z_pending = true;
  } else if (c->d.prec32 && !strcmp(field, "zb")) {
    // z stays what it was (as for FP64 state): keep it until fx_prepare
    if (!c->z_pending) {
      if ((rc = z32_into(c, c->zstage))) return rc;
      c->z_pending = true;
    }
    if ((rc = put_grid(c, c->d.zb, false, 1, host))) return rc;
  } else {
    if (!strcmp(field, "soil_mass") && (rc = alloc_soil(c))) return rc;
    const FieldRef f = field_ref(c, field);
    if (f.rec >= 0) {  // FP32 per-step field: one component of every slot's records
      if ((rc = read_ctl(c))) return rc;
      if ((rc = copy_in(c, c->stage, host))) return rc;
      const int cur = (int)(c->ctl_host->steps % c->d.nslot);
      if (c->d.prec32)
        k_rec_put<float, 8><<<plane_grid(c->d.plane), 256, 0, c->stream>>>(
            c->d, reinterpret_cast<float*>(c->d.rec32), c->stage, f.rec, cur);
      else
        k_rec_put<double, FX_R64_N><<<plane_grid(c->d.plane), 256, 0, c->stream>>>(c->d, c->d.rec64, c->stage,
                                                                                   f.rec, cur);
      FX_CK(c, cudaGetLastError());
      FX_CK(c, cudaStreamSynchronize(c->stream));
      c->prepared = false;
      return FX_OK;
    }
    // Every plane of a slot or pair field holds the uploaded grid: the steps
    // overwrite the interior cells only, and the ghost ring they read stays
    // as uploaded. The host grid crosses PCIe once, into the current plane;
    // the other planes are device-to-device copies of it.
    const size_t esz = f.f32 ? sizeof(float) : sizeof(double);
    const int planes = f.slot ? c->d.nslot : (f.pair ? 2 : f.copies);
    long long cur = 0;
    if (planes > 1) {
      if ((rc = read_ctl(c))) return rc;
      cur = f.slot ? c->ctl_host->steps % c->d.nslot : (c->ctl_host->steps & 1);
    }
    char* base = (char*)f.ptr;
    const size_t pbytes = (size_t)c->d.plane * esz;
    if ((rc = put_grid(c, base + cur * pbytes, f.f32, 1, host))) return rc;
    for (int k = 0; k < planes; ++k)
      if (k != cur)
        FX_CK(c, cudaMemcpyAsync(base + k * pbytes, base + cur * pbytes, pbytes, cudaMemcpyDeviceToDevice,
                                 c->stream));
    FX_CK(c, cudaStreamSynchronize(c->stream));
  }
  c->prepared = false;
  return FX_OK;
}

int fx_download(fx_ctx* c, const char* field, double* host) {
  if (!c || !field || !host) return fx_fail(c, FX_ERR_ARG, "fx_download: null argument");
  if (!known_field(c, field)) return fx_fail(c, FX_ERR_ARG, "fx_download: unknown field '%s'", field);
  if (c->d.prec32 && !strcmp(field, "z")) return get_z32(c, host);
  const FieldRef f = field_ref(c, field);
  if (!f.ptr) {  // soil_mass never set
    std::fill(host, host + ((size_t)c->d.nr + 2) * ((size_t)c->d.nc + 2), 0.0);
    return FX_OK;
  }
  if (f.rec >= 0) {  // FP32 per-step field: one component of the current slot's records
    int rc = read_ctl(c);
    if (rc) return rc;
    const long long o = fx_slot(c->d, c->ctl_host->steps);
    if (c->d.prec32)
      k_rec_get<float, 8><<<plane_grid(c->d.plane), 256, 0, c->stream>>>(fx_rec(c->d, o), f.rec, c->stage,
                                                                        c->d.plane);
    else
      k_rec_get<double, FX_R64_N><<<plane_grid(c->d.plane), 256, 0, c->stream>>>(fx_rec64(c->d, o), f.rec,
                                                                                c->stage, c->d.plane);
    FX_CK(c, cudaGetLastError());
    if ((rc = copy_out(c, host, c->stage))) return rc;
    FX_CK(c, cudaStreamSynchronize(c->stream));
    return FX_OK;
  }
  const size_t esz = f.f32 ? sizeof(float) : sizeof(double);
  const char* src = (const char*)f.ptr;
  if (f.slot || f.pair) {
    int rc = read_ctl(c);
    if (rc) return rc;
    src += (f.slot ? fx_slot(c->d, c->ctl_host->steps) : fx_pp(c->d, c->ctl_host->steps)) * esz;
  }
  return get_grid(c, src, f.f32, host);
}

// The flag byte of each grid cell from the two uploaded float planes (1.0 =
// set), into plane 0 of the flags; padding rows are left as they are.
__global__ void k_flags_of(const float* __restrict__ ldry, const float* __restrict__ wall, uint8_t* __restrict__ fl,
                           int ld, int mr, long long plane) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane; i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i % ld) - FX_ROFF;
    if (r < 0 || r >= mr) continue;
    fl[i] = (uint8_t)((ldry[i] == 1.0f ? FX_F_LDRY : 0) | (wall[i] == 1.0f ? FX_F_WALL : 0));
  }
}

int fx_upload_flags(fx_ctx* c, const float* ldry, const float* wall) {
  if (!c || !ldry || !wall) return fx_fail(c, FX_ERR_ARG, "fx_upload_flags: null argument");
  const int mr = c->d.nr + 2, mc = c->d.nc + 2;
  if (c->d.nslot >= 9) {
    // The two float planes cross the bus as they are, into the last 8 slot
    // planes of the flags (4 bytes per cell each), are combined on the device
    // into plane 0, which is then copied over the others.
    const size_t pl = (size_t)c->d.plane;
    float* sl = reinterpret_cast<float*>(c->d.flags + pl * (c->d.nslot - 8));
    float* sw = reinterpret_cast<float*>(c->d.flags + pl * (c->d.nslot - 4));
    for (int q = 0; q < 2; ++q)
      FX_CK(c, cudaMemcpy2DAsync((q ? sw : sl) + FX_ROFF, (size_t)c->d.ld * sizeof(float), q ? wall : ldry,
                                 (size_t)mr * sizeof(float), (size_t)mr * sizeof(float), (size_t)mc,
                                 cudaMemcpyHostToDevice, c->stream));
    k_flags_of<<<plane_grid(c->d.plane), 256, 0, c->stream>>>(sl, sw, c->d.flags, c->d.ld, mr, c->d.plane);
    FX_CK(c, cudaGetLastError());
    for (int k = 1; k < c->d.nslot; ++k)
      FX_CK(c, cudaMemcpyAsync(c->d.flags + k * pl, c->d.flags, pl, cudaMemcpyDeviceToDevice, c->stream));
    FX_CK(c, cudaStreamSynchronize(c->stream));
    c->prepared = false;
    return FX_OK;
  }
  std::vector<uint8_t> fl((size_t)mr * mc);
  for (size_t i = 0; i < fl.size(); ++i)
    fl[i] = (uint8_t)((ldry[i] == 1.0f ? FX_F_LDRY : 0) | (wall[i] == 1.0f ? FX_F_WALL : 0));
  // one copy from the host, then device-to-device into the other slot planes
  FX_CK(c, cudaMemcpy2DAsync(c->d.flags + FX_ROFF, (size_t)c->d.ld, fl.data(), (size_t)mr, (size_t)mr, (size_t)mc,
                             cudaMemcpyHostToDevice, c->stream));
  for (int k = 1; k < c->d.nslot; ++k)
    FX_CK(c, cudaMemcpyAsync(c->d.flags + k * c->d.plane, c->d.flags, (size_t)c->d.plane, cudaMemcpyDeviceToDevice,
                             c->stream));
  FX_CK(c, cudaStreamSynchronize(c->stream));
  c->prepared = false;
  return FX_OK;
}

int fx_download_flags(fx_ctx* c, float* ldry, float* ldry_prev, float* wall) {
  if (!c) return FX_ERR_ARG;
  const int mr = c->d.nr + 2, mc = c->d.nc + 2;
  std::vector<uint8_t> fl((size_t)mr * mc);
  int rc = read_ctl(c);
  if (rc) return rc;
  FX_CK(c, cudaMemcpy2DAsync(fl.data(), (size_t)mr, c->d.flags + fx_slot(c->d, c->ctl_host->steps) + FX_ROFF,
                             (size_t)c->d.ld, (size_t)mr, (size_t)mc, cudaMemcpyDeviceToHost, c->stream));
  FX_CK(c, cudaStreamSynchronize(c->stream));
  for (size_t i = 0; i < fl.size(); ++i) {
    if (ldry) ldry[i] = (fl[i] & FX_F_LDRY) ? 1.0f : 0.0f;
    if (ldry_prev) ldry_prev[i] = (fl[i] & FX_F_LDRY_PREV) ? 1.0f : 0.0f;
    if (wall) wall[i] = (fl[i] & FX_F_WALL) ? 1.0f : 0.0f;
  }
  return FX_OK;
}

int fx_set_forcing(fx_ctx* c, const float* tab, int has_meteo) {
  if (!c) return FX_ERR_ARG;
  c->d.has_meteo = has_meteo ? 1 : 0;
  if (has_meteo) {
    if (!tab) return fx_fail(c, FX_ERR_ARG, "fx_set_forcing: null table");
    FX_CK(c, cudaMemcpyAsync((void*)c->d.meteo_t, tab, sizeof(float) * 3 * FX_METEO_ROWS, cudaMemcpyHostToDevice,
                             c->stream));
    FX_CK(c, cudaStreamSynchronize(c->stream));
    // A negative rate can dry a wet cell within a step; keep every flux then.
    bool neg = false;
    for (int a = 0; a < FX_METEO_ROWS; ++a) neg |= tab[FX_METEO_ROWS + a] < 0.0f;
    c->negative_forcing = neg;
  }
  c->d.store_all_fluxes = (c->store_all_opt || c->negative_forcing) ? 1 : 0;
  c->graph_dirty = true;
  c->dev_dirty = true;
  c->dev_version++;
  return FX_OK;
}

// The discharge table and cell of add_inflow (common.cpp:277-390). The cell
// check of common.cpp:324,380-383 (zb equal to NODATA_VALUE) runs once here
// instead of every step.
int fx_set_inflow(fx_ctx* c, const float* tab, int irow, int icol) {
  if (!c) return FX_ERR_ARG;
  fx_dev& d = c->d;
  if (!tab) {
    d.has_inflow = 0;
    d.inflow_gi = -1;
  } else {
    if (irow < 1 || irow > d.nr || icol < 1 || icol > d.nc)
      return fx_fail(c, FX_ERR_ARG, "fx_set_inflow: cell (%d, %d) is not an interior cell", irow, icol);
    double zb = 0.0;
    FX_CK(c, cudaMemcpyAsync(&zb, d.zb + fx_ix(d, irow, icol), sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    FX_CK(c, cudaStreamSynchronize(c->stream));
    if (zb == d.nodata)  // common.cpp:380-383
      return fx_fail(c, FX_ERR_ARG, "fx_set_inflow: inflow ix,iy in NODATA_VALUE cell");
    if (!d.inflow_t) {
      float* t = nullptr;
      int rc = dev_alloc(c, (void**)&t, sizeof(float) * 3 * FX_METEO_ROWS);
      if (rc) return rc;
      d.inflow_t = t;
      d.inflow_r = t + FX_METEO_ROWS;
      d.inflow_c = t + 2 * FX_METEO_ROWS;
    }
    FX_CK(c, cudaMemcpyAsync((void*)d.inflow_t, tab, sizeof(float) * 3 * FX_METEO_ROWS, cudaMemcpyHostToDevice,
                             c->stream));
    FX_CK(c, cudaStreamSynchronize(c->stream));
    d.has_inflow = 1;
    d.inflow_irow = irow;
    d.inflow_icol = icol;
    d.inflow_gi = fx_ix(d, irow, icol);
  }
  c->graph_dirty = true;
  c->dev_dirty = true;
  c->dev_version++;
  return FX_OK;
}

// A per-cell extension grid: FP64 copy for FP64 state, FP32 copy for FP32.
static int set_optional_field(fx_ctx* c, const double* host, const double** slot64, const float** slot32) {
  const bool f32 = c->d.prec32 != 0;
  c->graph_dirty = true;
  c->dev_dirty = true;
  c->dev_version++;
  if (!host) {
    *slot64 = nullptr;
    *slot32 = nullptr;
    return FX_OK;
  }
  void* p = f32 ? (void*)*slot32 : (void*)*slot64;
  if (!p) {
    int rc = dev_alloc(c, &p, (size_t)c->d.plane * (f32 ? sizeof(float) : sizeof(double)));
    if (rc != FX_OK) return rc;
  }
  int rc = put_grid(c, p, f32, 1, host);
  if (rc) return rc;
  if (f32) *slot32 = (const float*)p;
  else *slot64 = (const double*)p;
  return FX_OK;
}

int fx_set_manning(fx_ctx* c, const double* n) {
  if (!c) return FX_ERR_ARG;
  return set_optional_field(c, n, &c->d.manning, &c->d.manning_f);
}

int fx_set_melt_field(fx_ctx* c, const double* m) {
  if (!c) return FX_ERR_ARG;
  return set_optional_field(c, m, &c->d.melt_mult, &c->d.melt_mult_f);
}

int fx_set_option(fx_ctx* c, const char* name, long long v) {
  if (!c || !name) return FX_ERR_ARG;
  if (!strcmp(name, "store_all_fluxes")) {
    c->store_all_opt = v != 0;
    c->d.store_all_fluxes = (c->store_all_opt || c->negative_forcing) ? 1 : 0;
    c->graph_dirty = true;
    c->dev_dirty = true;
    c->dev_version++;
    return FX_OK;
  }
  if (!strcmp(name, "tile_rows")) return set_tile_rows(c, (int)v);
  if (!strcmp(name, "fail_ade_waits")) {
    c->d.ade_hold = v != 0 ? 1 : 0;
    c->graph_dirty = true;
    c->dev_dirty = true;
    c->dev_version++;
    return FX_OK;
  }
  if (!strcmp(name, "tma")) {
    c->use_tma = v != 0;
    c->graph_dirty = true;
    c->dev_dirty = true;
    c->dev_version++;
    return FX_OK;
  }
  return fx_fail(c, FX_ERR_ARG, "fx_set_option: unknown option '%s'", name);
}

int fx_prepare(fx_ctx* c) {
  if (!c) return FX_ERR_ARG;
  int rc = read_ctl(c);
  if (rc) return rc;
  c->ctl_host->acc_dtmin = kInfBits;
  c->ctl_host->acc_hmax = 0ull;
  FX_CK(c, cudaMemcpyAsync(c->d.ctl, c->ctl_host, sizeof(fx_ctl), cudaMemcpyHostToDevice, c->stream));
  if ((rc = fx_sync_dev(c))) return rc;
  if (c->d.prec32) {
    if (c->z_pending) {
      // the pending z (field layout) with the current bed
      fx_launch_eta_from_z(c->d, c->zstage, c->stream);
      FX_CK(c, cudaGetLastError());
      FX_CK(c, cudaStreamSynchronize(c->stream));
      c->z_pending = false;
    }
  }
  fx_launch_mark_static(c->d_dev, 0, c->d.plane, c->stream);
  fx_launch_courant_scan(c->d_dev, c->d_tiles, c->ntiles, c->d.tile_rows, c->stream);
  FX_CK(c, cudaGetLastError());
  FX_CK(c, cudaStreamSynchronize(c->stream));
  c->prepared = true;
  return FX_OK;
}

}  // extern "C"

// One batch of m steps: the clock and the hydrodynamics step by step, then
// the ADE sweeps of all m steps in one launch (fx_ade.cu).
// The staged kernel's boxes (64 rows of flags, tile_rows + 2 columns) must
// fit in the field; smaller grids use the per-tile kernel.
// A grid at least as large as a staged box (64 rows incl. the padding, the
// tile's columns and their halo) for a tile shape.
bool fx_tma_fits(const fx_ctx* c, int tile_rows) { return c->d.ld >= 64 && c->d.nc + 2 >= tile_rows + 2; }
static bool tma_fits(const fx_ctx* c) { return fx_tma_fits(c, c->d.tile_rows); }

static void launch_hydro(fx_ctx* c) {
  if (c->use_tma && tma_fits(c)) fx_launch_hydro_tma(c->d, c->tmaps, c->tma_blocks, c->stream);
  else fx_launch_hydro_one(c->d, c->stream);
}

static void launch_batch(fx_ctx* c, int m) {
  fx_launch_batch_begin(c->d_dev, 1, c->stream);
  for (int i = 0; i < m; ++i) {
    fx_launch_finalize(c->d_dev, 1, c->stream);
    launch_hydro(c);
  }
  fx_launch_ade_one(c->d, c->nunits, c->ade_blocks, c->stream);
}

static int ensure_graph(fx_ctx* c) {
  int rc = fx_sync_dev(c);
  if (rc) return rc;
  if (c->graph_exec && !c->graph_dirty) return FX_OK;
  if (c->graph_exec) {
    cudaGraphExecDestroy(c->graph_exec);
    c->graph_exec = nullptr;
  }
  cudaGraph_t graph = nullptr;
  FX_CK(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  launch_batch(c, c->batch_steps);
  FX_CK(c, cudaStreamEndCapture(c->stream, &graph));
  cudaError_t e = cudaGraphInstantiate(&c->graph_exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return fx_fail(c, FX_ERR_CUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(e));
  c->graph_dirty = false;
  return FX_OK;
}

static int set_stop(fx_ctx* c, long long stop_after) {
  c->stop_host = stop_after;
  FX_CK(c, cudaMemcpyAsync(&c->d.ctl->stop_after, &c->stop_host, sizeof(long long), cudaMemcpyHostToDevice,
                           c->stream));
  return FX_OK;
}

static int status_rc(fx_ctx* c) {
  if (c->ctl_host->error)
    return fx_fail(c, FX_ERR_DEVICE, "device error %d: a bounded wait in the ADE sweep gave up",
                   c->ctl_host->error);
  return FX_OK;
}

extern "C" {

int fx_step(fx_ctx* c, int nsteps, fx_status* st) {
  if (!c || nsteps < 0) return FX_ERR_ARG;
  if (!c->prepared) {
    int rc = fx_prepare(c);
    if (rc) return rc;
  }
  int rc = read_ctl(c);
  if (rc) return rc;
  if (c->ctl_host->error) {  // a kernel gave up a wait: the state is not stepped further
    fx_fill_status(*c->ctl_host, st);
    return status_rc(c);
  }
  if ((rc = set_stop(c, c->ctl_host->steps + nsteps))) return rc;
  if ((rc = ensure_graph(c))) return rc;
  int left = nsteps;
  while (left >= c->batch_steps) {
    FX_CK(c, cudaGraphLaunch(c->graph_exec, c->stream));
    left -= c->batch_steps;
  }
  if (left > 0) launch_batch(c, left);
  FX_CK(c, cudaGetLastError());
  if ((rc = read_ctl(c))) return rc;
  fx_fill_status(*c->ctl_host, st);
  return status_rc(c);
}

int fx_run_to_print(fx_ctx* c, fx_status* st) {
  if (!c) return FX_ERR_ARG;
  for (;;) {
    int rc = read_ctl(c);
    if (rc) return rc;
    const fx_ctl& k = *c->ctl_host;
    if (k.print_pending || k.finished || k.error) break;
    // Enough steps to reach the next output at the current dt, within limits.
    double est = (k.dtfl > 0 && std::isfinite(k.dtfl)) ? (k.print_next - k.tim) / k.dtfl : 16.0;
    long long n = (long long)std::ceil(est) + 2;
    if (n < c->batch_steps) n = c->batch_steps;
    if (n > 4096) n = 4096;
    rc = fx_step(c, (int)n, nullptr);
    if (rc) return rc;
  }
  fx_fill_status(*c->ctl_host, st);
  return status_rc(c);
}

int fx_print_done(fx_ctx* c) {
  if (!c) return FX_ERR_ARG;
  int rc = read_ctl(c);
  if (rc) return rc;
  c->ctl_host->print_next = c->ctl_host->print_next + c->ctl_host->print_step;
  c->ctl_host->print_pending = 0;
  FX_CK(c, cudaMemcpyAsync(c->d.ctl, c->ctl_host, sizeof(fx_ctl), cudaMemcpyHostToDevice, c->stream));
  FX_CK(c, cudaStreamSynchronize(c->stream));
  return FX_OK;
}

int fx_get_status(fx_ctx* c, fx_status* st) {
  if (!c || !st) return FX_ERR_ARG;
  int rc = read_ctl(c);
  if (rc) return rc;
  fx_fill_status(*c->ctl_host, st);
  return FX_OK;
}

void* fx_stream(fx_ctx* c) { return c ? (void*)c->stream : nullptr; }

int fx_mass(fx_ctx* c, double* water, double* solute_mass) {
  if (!c || !water) return fx_fail(c, FX_ERR_ARG, "fx_mass: null argument");
  if (!c->prepared) {
    int rc = fx_prepare(c);
    if (rc) return rc;
  }
  double out[1 + FX_MAX_CHEM];
  FX_CK(c, cudaMemsetAsync(c->d_mass, 0, sizeof(out), c->stream));
  fx_launch_mass(c->d, c->d_mass, c->stream);
  FX_CK(c, cudaGetLastError());
  FX_CK(c, cudaMemcpyAsync(out, c->d_mass, sizeof(out), cudaMemcpyDeviceToHost, c->stream));
  FX_CK(c, cudaStreamSynchronize(c->stream));
  *water = out[0];
  if (solute_mass)
    for (int k = 0; k < c->d.nchem; ++k) solute_mass[k] = out[1 + k];
  return FX_OK;
}

int fx_time_steps(fx_ctx* c, int n, double* ms_total, double* ms_hydro, double* ms_ade) {
  if (!c || n < 1) return FX_ERR_ARG;
  if (!c->prepared) {
    int rc = fx_prepare(c);
    if (rc) return rc;
  }
  int rc = fx_sync_dev(c);
  if (rc) return rc;
  rc = read_ctl(c);
  if (rc) return rc;
  if ((rc = set_stop(c, c->ctl_host->steps + n))) return rc;
  // events: the start, then per step: after its clock update and after its
  // hydro launch, and per batch: after the sweep
  std::vector<cudaEvent_t> ev;
  ev.reserve(4 + 4 * (size_t)n);
  auto record = [&](size_t* idx) -> int {
    cudaEvent_t e = nullptr;
    FX_CK(c, cudaEventCreate(&e));
    ev.push_back(e);
    FX_CK(c, cudaEventRecord(e, c->stream));
    *idx = ev.size() - 1;
    return FX_OK;
  };
  size_t e_start = 0, a = 0, b = 0;
  std::vector<std::pair<size_t, size_t>> hyd, ade;
  int erc = record(&e_start);
  const int K = c->batch_steps;
  for (int left = n; left > 0 && !erc;) {
    const int m = left < K ? left : K;
    left -= m;
    fx_launch_batch_begin(c->d_dev, 1, c->stream);
    for (int i = 0; i < m && !erc; ++i) {
      fx_launch_finalize(c->d_dev, 1, c->stream);
      if ((erc = record(&a))) break;
      launch_hydro(c);
      if ((erc = record(&b))) break;
      hyd.push_back({a, b});
    }
    if (erc) break;
    a = b;
    fx_launch_ade_one(c->d, c->nunits, c->ade_blocks, c->stream);
    if ((erc = record(&b))) break;
    ade.push_back({a, b});
  }
  if (erc) {
    for (auto& e : ev) cudaEventDestroy(e);
    return erc;
  }
  FX_CK(c, cudaGetLastError());
  FX_CK(c, cudaStreamSynchronize(c->stream));
  double th = 0, ta = 0;
  float ms = 0;
  for (auto& pr : hyd) {
    FX_CK(c, cudaEventElapsedTime(&ms, ev[pr.first], ev[pr.second]));
    th += ms;
  }
  for (auto& pr : ade) {
    FX_CK(c, cudaEventElapsedTime(&ms, ev[pr.first], ev[pr.second]));
    ta += ms;
  }
  FX_CK(c, cudaEventElapsedTime(&ms, ev[e_start], ev.back()));
  for (auto& e : ev) cudaEventDestroy(e);
  if (ms_total) *ms_total = ms;
  if (ms_hydro) *ms_hydro = th;
  if (ms_ade) *ms_ade = ta;
  if ((rc = read_ctl(c))) return rc;
  return status_rc(c);
}

int fx_autotune(fx_ctx* c, int trial_steps, int* tile_rows) {
  if (!c || trial_steps < 1) return fx_fail(c, FX_ERR_ARG, "fx_autotune: bad argument");
  // Each candidate runs trial_steps real steps (results do not depend on the
  // tile shape); the hydrodynamic kernel time per step decides. The state
  // changes as the run advances (a spreading wet front makes later steps
  // dearer), so the candidates run twice, in one order and then in the
  // reverse order, and each is scored by the sum of its two times per step:
  // a drift that is linear in the step count adds the same to every score.
  const int cand[3] = {4, 8, 16};
  double ms[3] = {0.0, 0.0, 0.0};
  bool ok[3] = {true, true, true};
  for (int pass = 0; pass < 2; ++pass) {
    for (int q = 0; q < 3; ++q) {
      const int j = pass == 0 ? q : 2 - q;
      int rc = set_tile_rows(c, cand[j]);
      if (rc) return rc;
      rc = read_ctl(c);
      if (rc) return rc;
      const long long s0 = c->ctl_host->steps;
      double tot = 0, hyd = 0, ade = 0;
      rc = fx_time_steps(c, trial_steps, &tot, &hyd, &ade);
      if (rc) return rc;
      const long long ran = c->ctl_host->steps - s0;
      if (ran < 1) {  // the run stopped (output due or over): nothing measured
        ok[j] = false;
        continue;
      }
      ms[j] += hyd / (double)ran;
    }
  }
  double best_ms = 0.0;
  int best = c->d.tile_rows;
  for (int j = 0; j < 3; ++j) {
    if (!ok[j]) continue;
    if (best_ms == 0.0 || ms[j] < best_ms) {
      best_ms = ms[j];
      best = cand[j];
    }
  }
  int rc = set_tile_rows(c, best);
  if (rc) return rc;
  if (tile_rows) *tile_rows = best;
  return FX_OK;
}

}  // extern "C"
