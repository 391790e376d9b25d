// Batches: several domains (contexts) advanced together by the same
// launches, each with its own clock, dt, forcing and outputs.
//
// A batch of K steps is one CUDA graph: open the batch in every domain, then
// K times (clock update of every domain, one hydrodynamic launch over the
// concatenated tile table of all domains), then one ADE launch over the
// interleaved unit table of all domains (fx_ade.cu). The hydrodynamic launch
// is the persistent TMA-staged batch kernel (each domain's stencil fields
// staged through its own tensor maps, kept in a device array) when every
// member's grid is large enough for a staged box; otherwise one block per
// tile loads its own stencil. Domains that stop (an
// output is due, the run ended, or their step budget is spent) skip their
// tiles and units until the host releases them, while the others go on.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "fluxos_gpu.h"
#include "fx_common.cuh"
#include "fx_internal.h"


struct fx_batch {
  std::vector<fx_ctx*> doms;
  cudaStream_t stream = nullptr;
  fx_dev* d_devs = nullptr;
  fx_tile* d_tiles = nullptr;
  fx_unit* d_units = nullptr;
  fx_tmaps* d_tmaps = nullptr;  // one set of tensor maps per member (batch tile shape)
  size_t cap_devs = 0, cap_tiles = 0, cap_units = 0, cap_tmaps = 0;
  int ntiles = 0, nunits = 0, K = 1, ade_blocks = 1;
  bool use_tma = true;   // option "tma": the TMA-staged batch kernel where the members allow it
  bool hydro_tma = false;  // the current graph uses it
  int tma_blocks = 0;
  int tile_rows = 8;              // hydrodynamic tile shape of the batch's launches
  int k_limit = FX_MAX_SLOTS;     // upper bound on steps per graph (ADE sweeps in flight)
  bool dirty = true;  // membership or a descriptor changed: rebuild tables and graph
  cudaGraphExec_t graph = nullptr;
  std::vector<long long> stop_host;
  std::vector<long long> versions;  // members' descriptor versions in the tables
  std::string err;
};

#define FXB_CK(b, call)                                                                         \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) {                                                                    \
      int rc_ = fx_fail(nullptr, FX_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
      (b)->err = fx_last_error(nullptr);                                                        \
      return rc_;                                                                               \
    }                                                                                           \
  } while (0)

static int grow(fx_batch* b, void** p, size_t* cap, size_t need) {
  if (need <= *cap) return FX_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  size_t n = std::max(need, *cap * 2);
  FXB_CK(b, cudaMalloc(p, n));
  *cap = n;
  return FX_OK;
}

// Tables and graph for the current members.
static int rebuild(fx_batch* b) {
  if (b->versions.size() != b->doms.size()) b->dirty = true;
  for (size_t i = 0; i < b->doms.size() && !b->dirty; ++i)
    if (b->doms[i]->dev_version != b->versions[i]) b->dirty = true;
  if (!b->dirty) return FX_OK;
  const int n = (int)b->doms.size();
  b->K = b->k_limit;
  for (fx_ctx* c : b->doms) b->K = std::min(b->K, c->batch_steps);
  if (n == 0) b->K = 1;
  std::vector<fx_dev> devs(n);
  std::vector<fx_tile> tiles;
  std::vector<std::vector<fx_unit>> per(n);
  size_t total_units = 0;
  for (int i = 0; i < n; ++i) {
    fx_ctx* c = b->doms[i];
    devs[i] = c->d;
    fx_tiles_of(i, c->g.nrows, c->g.ncols, b->tile_rows, tiles);
    fx_units_of(i, c->g.nrows, c->g.nchem, b->K, per[i]);
    total_units += per[i].size();
  }
  // interleave domains, keeping each domain's own order (its dependencies)
  std::vector<fx_unit> units;
  units.reserve(total_units);
  std::vector<size_t> pos(n, 0);
  for (bool any = true; any;) {
    any = false;
    for (int i = 0; i < n; ++i)
      if (pos[i] < per[i].size()) {
        units.push_back(per[i][pos[i]++]);
        any = true;
      }
  }
  int rc;
  if ((rc = grow(b, (void**)&b->d_devs, &b->cap_devs, sizeof(fx_dev) * std::max(n, 1)))) return rc;
  if ((rc = grow(b, (void**)&b->d_tiles, &b->cap_tiles, sizeof(fx_tile) * std::max<size_t>(tiles.size(), 1))))
    return rc;
  if ((rc = grow(b, (void**)&b->d_units, &b->cap_units, sizeof(fx_unit) * std::max<size_t>(units.size(), 1))))
    return rc;
  if (n) FXB_CK(b, cudaMemcpyAsync(b->d_devs, devs.data(), sizeof(fx_dev) * n, cudaMemcpyHostToDevice, b->stream));
  if (!tiles.empty())
    FXB_CK(b, cudaMemcpyAsync(b->d_tiles, tiles.data(), sizeof(fx_tile) * tiles.size(), cudaMemcpyHostToDevice,
                              b->stream));
  if (!units.empty())
    FXB_CK(b, cudaMemcpyAsync(b->d_units, units.data(), sizeof(fx_unit) * units.size(), cudaMemcpyHostToDevice,
                              b->stream));
  // tensor maps of every member for the batch's tile shape
  b->hydro_tma = b->use_tma && n > 0;
  for (int i = 0; i < n && b->hydro_tma; ++i)
    if (!b->doms[i]->use_tma || !fx_tma_fits(b->doms[i], b->tile_rows)) b->hydro_tma = false;
  if (b->hydro_tma) {
    std::vector<fx_tmaps> tm(n);
    for (int i = 0; i < n; ++i)
      if ((rc = fx_build_tmaps_for(b->doms[i], b->tile_rows, &tm[i]))) {
        b->err = fx_last_error(nullptr);
        return rc;
      }
    if ((rc = grow(b, (void**)&b->d_tmaps, &b->cap_tmaps, sizeof(fx_tmaps) * n))) return rc;
    FXB_CK(b, cudaMemcpyAsync(b->d_tmaps, tm.data(), sizeof(fx_tmaps) * n, cudaMemcpyHostToDevice, b->stream));
    if (fx_hydro_batch_tma_blocks(b->doms[0]->d.prec32 != 0, b->tile_rows, &b->tma_blocks) != 0 ||
        b->tma_blocks < 1) {
      int r = fx_fail(nullptr, FX_ERR_CUDA, "occupancy query for the TMA-staged batch kernel failed");
      b->err = fx_last_error(nullptr);
      return r;
    }
  }
  FXB_CK(b, cudaStreamSynchronize(b->stream));
  b->ntiles = (int)tiles.size();
  b->nunits = (int)units.size();
  int maxb = 0;
  if (fx_ade_max_blocks_for(n > 0 && b->doms[0]->d.prec32 != 0, &maxb) != 0 || maxb < 1) {
    int r = fx_fail(nullptr, FX_ERR_CUDA, "occupancy query for the ADE sweep failed");
    b->err = fx_last_error(nullptr);
    return r;
  }
  const int per_block = fx_ade_threads_per_block() / 32;
  b->ade_blocks = std::max(1, std::min((b->nunits + per_block - 1) / per_block, maxb));
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  if (n) {
    const bool prec32 = b->doms[0]->d.prec32 != 0;  // members share it (fx_batch_add)
    cudaGraph_t g = nullptr;
    FXB_CK(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    fx_launch_batch_begin(b->d_devs, n, b->stream);
    for (int i = 0; i < b->K; ++i) {
      fx_launch_finalize(b->d_devs, n, b->stream);
      if (b->hydro_tma)
        fx_launch_hydro_batch_tma(b->d_devs, b->d_tmaps, b->d_tiles, b->ntiles,
                                  std::min(b->ntiles, b->tma_blocks), prec32, b->tile_rows, b->stream);
      else
        fx_launch_hydro(b->d_devs, b->d_tiles, b->ntiles, prec32, b->tile_rows, b->stream);
    }
    fx_launch_ade(b->d_devs, b->d_units, b->nunits, b->ade_blocks, prec32, b->stream);
    FXB_CK(b, cudaStreamEndCapture(b->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      int r = fx_fail(nullptr, FX_ERR_CUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(e));
      b->err = fx_last_error(nullptr);
      return r;
    }
  }
  b->versions.resize(n);
  for (int i = 0; i < n; ++i) b->versions[i] = b->doms[i]->dev_version;
  b->dirty = false;
  return FX_OK;
}

extern "C" {

int fx_batch_create(fx_batch** out) {
  if (!out) return fx_fail(nullptr, FX_ERR_ARG, "fx_batch_create: null argument");
  fx_batch* b = new fx_batch();
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete b;
    return fx_fail(nullptr, FX_ERR_CUDA, "cudaStreamCreate failed: %s", cudaGetErrorString(e));
  }
  *out = b;
  return FX_OK;
}

void fx_batch_destroy(fx_batch* b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->d_devs) cudaFree(b->d_devs);
  if (b->d_tiles) cudaFree(b->d_tiles);
  if (b->d_units) cudaFree(b->d_units);
  if (b->d_tmaps) cudaFree(b->d_tmaps);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

const char* fx_batch_last_error(const fx_batch* b) { return b ? b->err.c_str() : ""; }

int fx_batch_add(fx_batch* b, fx_ctx* c) {
  if (!b || !c) return fx_fail(nullptr, FX_ERR_ARG, "fx_batch_add: null argument");
  if (std::find(b->doms.begin(), b->doms.end(), c) != b->doms.end())
    return fx_fail(nullptr, FX_ERR_ARG, "fx_batch_add: context already in the batch");
  if (!b->doms.empty() && b->doms[0]->d.prec32 != c->d.prec32)
    return fx_fail(nullptr, FX_ERR_ARG, "fx_batch_add: members of a batch share one precision");
  if (!c->prepared) {
    int rc = fx_prepare(c);
    if (rc) return rc;
  }
  b->doms.push_back(c);
  b->dirty = true;
  return FX_OK;
}

int fx_batch_remove(fx_batch* b, fx_ctx* c) {
  if (!b || !c) return fx_fail(nullptr, FX_ERR_ARG, "fx_batch_remove: null argument");
  auto it = std::find(b->doms.begin(), b->doms.end(), c);
  if (it == b->doms.end()) return fx_fail(nullptr, FX_ERR_ARG, "fx_batch_remove: context not in the batch");
  cudaStreamSynchronize(b->stream);
  b->doms.erase(it);
  b->dirty = true;
  return FX_OK;
}

int fx_batch_size(const fx_batch* b) { return b ? (int)b->doms.size() : 0; }

// Up to nsteps steps of every member (each stops early at its own outputs or
// end); then the members' clocks are read back into st[0..n-1] (may be NULL).
int fx_batch_step(fx_batch* b, int nsteps, fx_status* st) {
  if (!b || nsteps < 0) return fx_fail(nullptr, FX_ERR_ARG, "fx_batch_step: bad argument");
  const int n = (int)b->doms.size();
  if (n == 0) return FX_OK;
  for (fx_ctx* c : b->doms)
    if (!c->prepared) {  // state was edited since the member joined
      int r = fx_prepare(c);
      if (r) return r;
    }
  int rc = rebuild(b);
  if (rc) return rc;
  // every member's step budget: its steps so far + nsteps
  for (fx_ctx* c : b->doms) {
    FXB_CK(b, cudaMemcpyAsync(c->ctl_host, c->d.ctl, sizeof(fx_ctl), cudaMemcpyDeviceToHost, b->stream));
  }
  FXB_CK(b, cudaStreamSynchronize(b->stream));
  b->stop_host.resize(n);
  for (int i = 0; i < n; ++i) {
    fx_ctx* c = b->doms[i];
    b->stop_host[i] = c->ctl_host->steps + nsteps;
    FXB_CK(b, cudaMemcpyAsync(&c->d.ctl->stop_after, &b->stop_host[i], sizeof(long long), cudaMemcpyHostToDevice,
                              b->stream));
  }
  for (int left = nsteps; left > 0; left -= b->K) FXB_CK(b, cudaGraphLaunch(b->graph, b->stream));
  for (fx_ctx* c : b->doms)
    FXB_CK(b, cudaMemcpyAsync(c->ctl_host, c->d.ctl, sizeof(fx_ctl), cudaMemcpyDeviceToHost, b->stream));
  FXB_CK(b, cudaStreamSynchronize(b->stream));
  int derr = 0;
  for (int i = 0; i < n; ++i) {
    const fx_ctl& k = *b->doms[i]->ctl_host;
    if (k.error) derr = k.error;
    if (st) fx_fill_status(k, &st[i]);
  }
  if (derr) {
    int r = fx_fail(nullptr, FX_ERR_DEVICE, "device error %d in a batch member: a bounded wait gave up", derr);
    b->err = fx_last_error(nullptr);
    return r;
  }
  return FX_OK;
}

void* fx_batch_stream(fx_batch* b) { return b ? (void*)b->stream : nullptr; }

int fx_batch_set_option(fx_batch* b, const char* name, long long v) {
  if (!b || !name) return fx_fail(nullptr, FX_ERR_ARG, "fx_batch_set_option: null argument");
  if (!strcmp(name, "tile_rows")) {
    if (!fx_tile_rows_ok((int)v)) return fx_fail(nullptr, FX_ERR_ARG, "tile_rows must be 4, 8 or 16");
    b->tile_rows = (int)v;
  } else if (!strcmp(name, "steps_in_flight")) {
    if (v < 1 || v > FX_MAX_SLOTS - 1) return fx_fail(nullptr, FX_ERR_ARG, "steps_in_flight must be 1..63");
    b->k_limit = (int)v;
  } else if (!strcmp(name, "tma")) {
    b->use_tma = v != 0;
  } else {
    return fx_fail(nullptr, FX_ERR_ARG, "fx_batch_set_option: unknown option '%s'", name);
  }
  b->dirty = true;
  return FX_OK;
}

// Cell-steps per second of `steps` batch steps (wall clock around
// fx_batch_step, which ends with a stream synchronisation).
static int trial(fx_batch* b, int steps, double* rate) {
  const int n = (int)b->doms.size();
  std::vector<fx_status> st0(n), st1(n);
  int rc = fx_batch_step(b, 0, st0.data());
  if (rc) return rc;
  const auto t0 = std::chrono::steady_clock::now();
  rc = fx_batch_step(b, steps, st1.data());
  if (rc) return rc;
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  double cells = 0;
  for (int i = 0; i < n; ++i)
    cells += (double)(st1[i].steps - st0[i].steps) * b->doms[i]->g.nrows * (double)b->doms[i]->g.ncols;
  *rate = secs > 0 ? cells / secs : 0.0;
  return FX_OK;
}

int fx_batch_autotune(fx_batch* b, int trial_steps, int* tile_rows, int* steps_in_flight) {
  if (!b || trial_steps < 1) return fx_fail(nullptr, FX_ERR_ARG, "fx_batch_autotune: bad argument");
  if (b->doms.empty()) return FX_OK;
  int kmax = FX_MAX_SLOTS - 1;
  for (fx_ctx* c : b->doms) kmax = std::min(kmax, c->batch_steps);
  // warm-up of the current configuration (first graph, caches)
  double rate = 0;
  int rc = trial(b, trial_steps, &rate);
  if (rc) return rc;
  // Each choice is tried twice, in one order and then in the reverse order,
  // and scored by the sum of its two times per cell-step: the members' state
  // changes as the trials advance it, and a drift linear in the step count
  // adds the same to every score.
  auto sweep = [&](const int* vals, int nv, auto apply, auto steps_for, int* best_val) -> int {
    double score[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool ok[8] = {false, false, false, false, false, false, false, false};
    for (int pass = 0; pass < 2; ++pass) {
      for (int q = 0; q < nv; ++q) {
        const int j = pass == 0 ? q : nv - 1 - q;
        apply(vals[j]);
        int rc2 = trial(b, 1, &rate);  // rebuilds the tables and the graph
        if (rc2) return rc2;
        if ((rc2 = trial(b, steps_for(vals[j]), &rate))) return rc2;
        if (rate > 0) {
          score[j] += 1.0 / rate;
          ok[j] = pass == 0 ? true : ok[j];
        } else {
          ok[j] = false;
        }
      }
    }
    double lo = -1;
    for (int j = 0; j < nv; ++j)
      if (ok[j] && (lo < 0 || score[j] < lo)) {
        lo = score[j];
        *best_val = vals[j];
      }
    return FX_OK;
  };
  int best_rows = b->tile_rows;
  const int rows[3] = {4, 8, 16};
  rc = sweep(rows, 3, [&](int r) { b->tile_rows = r; b->dirty = true; }, [&](int) { return trial_steps; },
             &best_rows);
  if (rc) return rc;
  b->tile_rows = best_rows;
  b->dirty = true;
  int best_k = std::min(b->k_limit, kmax);
  int ks[6], nk = 0;
  for (int k : {2, 4, 8, 16, 31, 63})
    if (k <= kmax) ks[nk++] = k;
  rc = sweep(ks, nk, [&](int k) { b->k_limit = k; b->dirty = true; },
             [&](int k) { return std::max(trial_steps, 2 * k); }, &best_k);
  if (rc) return rc;
  b->k_limit = best_k;
  b->dirty = true;
  if (tile_rows) *tile_rows = best_rows;
  if (steps_in_flight) *steps_in_flight = best_k;
  return FX_OK;
}

}  // extern "C"
