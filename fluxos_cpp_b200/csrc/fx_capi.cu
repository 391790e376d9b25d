// C ABI of libfluxos_gpu.so: context, device state, stepping (see
// include/fluxos_gpu.h for the contract and the reference interfaces each
// entry point replaces).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "fluxos_gpu.h"
#include "fx_common.cuh"
#include "fx_internal.h"

void fx_launch_finalize(const fx_dev& d, cudaStream_t s);
void fx_launch_batch_begin(const fx_dev& d, cudaStream_t s);
void fx_launch_mark_static(const fx_dev& d, cudaStream_t s);
void fx_launch_hydro(const fx_dev& d, cudaStream_t s);
void fx_launch_courant_scan(const fx_dev& d, cudaStream_t s);
void fx_launch_ade(const fx_dev& d, int nstrips, int nblocks, cudaStream_t s);
int fx_ade_rows_per_strip();
int fx_ade_threads_per_block();
int fx_ade_max_blocks(int* out);

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

// Fields with one plane per slot (the state after step n lives in plane
// n % nslot); the others have a single plane.
static bool slot_field(const char* name) {
  return !strcmp(name, "h") || !strcmp(name, "h0") || !strcmp(name, "fe_1") || !strcmp(name, "fn_1");
}

static double* field_ptr(fx_ctx* c, const char* name) {
  fx_dev& d = c->d;
  if (!strcmp(name, "z")) return d.z;
  if (!strcmp(name, "zb")) return d.zb;
  if (!strcmp(name, "h")) return d.h;
  if (!strcmp(name, "qx")) return d.qx;
  if (!strcmp(name, "qy")) return d.qy;
  if (!strcmp(name, "twet")) return d.twet;
  if (!strcmp(name, "h0")) return d.h0;
  if (!strcmp(name, "fe_1")) return d.fe1;
  if (!strcmp(name, "fe_2")) return d.fe2;
  if (!strcmp(name, "fe_3")) return d.fe3;
  if (!strcmp(name, "fn_1")) return d.fn1;
  if (!strcmp(name, "fn_2")) return d.fn2;
  if (!strcmp(name, "fn_3")) return d.fn3;
  if (!strncmp(name, "conc", 4)) {
    int k = name[4] ? atoi(name + 4) : 0;
    if (k < 0 || k >= d.nchem) return nullptr;
    return d.conc + (long long)k * d.plane;
  }
  return nullptr;
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

static void fill_status(const fx_ctl& k, fx_status* st) {
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
}

extern "C" {

const char* fx_last_error(const fx_ctx* ctx) { return ctx ? ctx->err.c_str() : g_last_error.c_str(); }

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
  for (int k = 0; k < FX_MAX_CHEM; ++k) d.dcoef[k] = p->d_coef[k];
  {
    int k = p->steps_in_flight > 0 ? p->steps_in_flight : 8;
    if (k > FX_MAX_SLOTS - 1) k = FX_MAX_SLOTS - 1;
    d.nslot = k + 1;  // a batch of k steps plus the state before it
    c->batch_steps = k;
  }
  const size_t pb = (size_t)d.plane * sizeof(double);
  int rc = FX_OK;
  double** fields[] = {&d.z, &d.zb, &d.qx, &d.qy, &d.twet, &d.fe2, &d.fe3, &d.fn2, &d.fn3};
  double** slot_fields[] = {&d.h, &d.h0, &d.hpm, &d.fe1, &d.fn1};
  for (double** f : fields)
    if ((rc = dev_alloc(c, (void**)f, pb)) != FX_OK) goto fail;
  for (double** f : slot_fields)
    if ((rc = dev_alloc(c, (void**)f, pb * d.nslot)) != FX_OK) goto fail;
  if ((rc = dev_alloc(c, (void**)&d.conc, pb * g->nchem)) != FX_OK) goto fail;
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
    if (fx_ade_max_blocks(&maxb) != 0 || maxb < 1) {
      rc = fx_fail(c, FX_ERR_CUDA, "occupancy query for the ADE sweep failed");
      goto fail;
    }
    const int units = c->batch_steps * g->nchem * c->ade_strips;
    const int per_block = fx_ade_threads_per_block() / 32;
    int want = (units + per_block - 1) / per_block;
    c->ade_blocks = want < maxb ? want : maxb;
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
  *out = c;
  return FX_OK;
fail:
  g_last_error = c->err;
  fx_destroy(c);
  return rc;
}

void fx_destroy(fx_ctx* c) {
  if (!c) return;
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

int fx_upload(fx_ctx* c, const char* field, const double* host) {
  if (!c || !field || !host) return fx_fail(c, FX_ERR_ARG, "fx_upload: null argument");
  double* dst = field_ptr(c, field);
  if (!dst) return fx_fail(c, FX_ERR_ARG, "fx_upload: unknown field '%s'", field);
  const int mr = c->d.nr + 2, mc = c->d.nc + 2;
  const int planes = slot_field(field) ? c->d.nslot : 1;  // every slot holds the uploaded state
  for (int k = 0; k < planes; ++k)
    FX_CK(c, cudaMemcpy2DAsync(dst + k * c->d.plane + FX_ROFF, (size_t)c->d.ld * sizeof(double), host,
                               (size_t)mr * sizeof(double), (size_t)mr * sizeof(double), (size_t)mc,
                               cudaMemcpyHostToDevice, c->stream));
  FX_CK(c, cudaStreamSynchronize(c->stream));
  c->prepared = false;
  return FX_OK;
}

int fx_download(fx_ctx* c, const char* field, double* host) {
  if (!c || !field || !host) return fx_fail(c, FX_ERR_ARG, "fx_download: null argument");
  double* src = field_ptr(c, field);
  if (!src) return fx_fail(c, FX_ERR_ARG, "fx_download: unknown field '%s'", field);
  if (slot_field(field)) {
    int rc = read_ctl(c);
    if (rc) return rc;
    src += fx_slot(c->d, c->ctl_host->steps);
  }
  const int mr = c->d.nr + 2, mc = c->d.nc + 2;
  FX_CK(c, cudaMemcpy2DAsync(host, (size_t)mr * sizeof(double), src + FX_ROFF, (size_t)c->d.ld * sizeof(double),
                             (size_t)mr * sizeof(double), (size_t)mc, cudaMemcpyDeviceToHost, c->stream));
  FX_CK(c, cudaStreamSynchronize(c->stream));
  return FX_OK;
}

int fx_upload_flags(fx_ctx* c, const float* ldry, const float* wall) {
  if (!c || !ldry || !wall) return fx_fail(c, FX_ERR_ARG, "fx_upload_flags: null argument");
  const int mr = c->d.nr + 2, mc = c->d.nc + 2;
  std::vector<uint8_t> fl((size_t)mr * mc);
  for (size_t i = 0; i < fl.size(); ++i)
    fl[i] = (uint8_t)((ldry[i] == 1.0f ? FX_F_LDRY : 0) | (wall[i] == 1.0f ? FX_F_WALL : 0));
  for (int k = 0; k < c->d.nslot; ++k)
    FX_CK(c, cudaMemcpy2DAsync(c->d.flags + k * c->d.plane + FX_ROFF, (size_t)c->d.ld, fl.data(), (size_t)mr,
                               (size_t)mr, (size_t)mc, cudaMemcpyHostToDevice, c->stream));
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
  return FX_OK;
}

static int set_optional_field(fx_ctx* c, const double* host, const double** slot, const char* what) {
  if (!host) {
    *slot = nullptr;
    c->graph_dirty = true;
    return FX_OK;
  }
  double* p = const_cast<double*>(*slot);
  if (!p) {
    int rc = dev_alloc(c, (void**)&p, (size_t)c->d.plane * sizeof(double));
    if (rc != FX_OK) return rc;
  }
  const int mr = c->d.nr + 2, mc = c->d.nc + 2;
  FX_CK(c, cudaMemcpy2DAsync(p + FX_ROFF, (size_t)c->d.ld * sizeof(double), host, (size_t)mr * sizeof(double),
                             (size_t)mr * sizeof(double), (size_t)mc, cudaMemcpyHostToDevice, c->stream));
  FX_CK(c, cudaStreamSynchronize(c->stream));
  (void)what;
  *slot = p;
  c->graph_dirty = true;
  return FX_OK;
}

int fx_set_manning(fx_ctx* c, const double* n) {
  if (!c) return FX_ERR_ARG;
  return set_optional_field(c, n, &c->d.manning, "manning");
}

int fx_set_melt_field(fx_ctx* c, const double* m) {
  if (!c) return FX_ERR_ARG;
  return set_optional_field(c, m, &c->d.melt_mult, "melt");
}

int fx_set_option(fx_ctx* c, const char* name, long long v) {
  if (!c || !name) return FX_ERR_ARG;
  if (!strcmp(name, "store_all_fluxes")) {
    c->store_all_opt = v != 0;
    c->d.store_all_fluxes = (c->store_all_opt || c->negative_forcing) ? 1 : 0;
    c->graph_dirty = true;
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
  fx_launch_mark_static(c->d, c->stream);
  fx_launch_courant_scan(c->d, c->stream);
  FX_CK(c, cudaGetLastError());
  FX_CK(c, cudaStreamSynchronize(c->stream));
  c->prepared = true;
  return FX_OK;
}

}  // extern "C"

// One batch of m steps: the clock and the hydrodynamics step by step, then
// the ADE sweeps of all m steps in one launch (fx_ade.cu).
static void launch_batch(fx_ctx* c, int m) {
  fx_launch_batch_begin(c->d, c->stream);
  for (int i = 0; i < m; ++i) {
    fx_launch_finalize(c->d, c->stream);
    fx_launch_hydro(c->d, c->stream);
  }
  fx_launch_ade(c->d, c->ade_strips, c->ade_blocks, c->stream);
}

static int ensure_graph(fx_ctx* c) {
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
  fill_status(*c->ctl_host, st);
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
  fill_status(*c->ctl_host, st);
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
  fill_status(*c->ctl_host, st);
  return FX_OK;
}

void* fx_stream(fx_ctx* c) { return c ? (void*)c->stream : nullptr; }

int fx_time_steps(fx_ctx* c, int n, double* ms_total, double* ms_hydro, double* ms_ade) {
  if (!c || n < 1) return FX_ERR_ARG;
  if (!c->prepared) {
    int rc = fx_prepare(c);
    if (rc) return rc;
  }
  int rc = read_ctl(c);
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
    fx_launch_batch_begin(c->d, c->stream);
    for (int i = 0; i < m && !erc; ++i) {
      fx_launch_finalize(c->d, c->stream);
      if ((erc = record(&a))) break;
      fx_launch_hydro(c->d, c->stream);
      if ((erc = record(&b))) break;
      hyd.push_back({a, b});
    }
    if (erc) break;
    a = b;
    fx_launch_ade(c->d, c->ade_strips, c->ade_blocks, c->stream);
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

}  // extern "C"
