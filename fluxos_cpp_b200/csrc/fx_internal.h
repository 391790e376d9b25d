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
  bool prepared = false;
  bool graph_dirty = true;
  bool store_all_opt = false;
  bool negative_forcing = false;
  cudaGraphExec_t graph_exec = nullptr;
  // file surface (filled by fx_open_modset)
  double h_min_print = 0.0;
  std::string output_folder;
};

int fx_fail(fx_ctx* ctx, int code, const char* fmt, ...);
