// fx_adesolver_noalloc: one ADE sweep on caller-owned device arrays that
// allocates no memory at all.
//
// Who needs it: callers that are not allowed to call cudaMalloc while they
// run. A host model that hands out all of its device memory from its own pool
// or arena must stay inside that budget, and a job under a hard memory cap may
// not grow; coupling layers (the role OpenWQ plays next to FLUXOS) own the
// solute arrays and only want the transport step applied to them. Such
// callers pass device pointers they already hold; this entry point then
// creates no context, stream or buffer of its own.
//
// The sweep needs scratch memory: per strip of 30 rows, the hand-over values
// of the strip's last row (3 doubles per column) and a progress counter, plus
// the domain descriptor, the strip table and a control block. Here that
// scratch is the file-scope device array g_noalloc_scratch of
// FX_NOALLOC_SCRATCH_BYTES (8 MiB), which every GPU that loads the library
// holds until the process exits. A grid fits when
// ceil(nrows / 30) * (ncols + 2) * 24 bytes plus the fixed part (a few KiB)
// is at most 8 MiB (square grids up to about 3,200 x 3,200 cells); larger
// grids are rejected with FX_ERR_ARG and a message giving the bytes needed.
//
// Set-up: the first call on a device, with that device current, looks up the
// device address of the array (cudaGetSymbolAddress; the array's name in host
// code is only a host-side stand-in) and the sweep kernel's launch limits, and
// keeps them for that device's CUDA context. A later call repeats the set-up
// only if the device's context has changed (after cudaDeviceReset the module,
// and with it the array, is loaded anew). Make the first call on each device
// before any stream capture.
//
// Every call shares the one array: calls that overlap on the GPU (other
// streams, other host threads) race on it and must be serialised by the
// caller. The array keeps the last call's contents; each call clears the
// progress counters and rewrites the descriptor, strip table and control
// block, the only scratch that must start from a known value (the hand-over
// values are written before they are read). The call reads the sweep's error
// flag back and synchronises its stream before it returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "fluxos_gpu.h"
#include "fx_common.cuh"

void fx_launch_ade(const fx_dev* devs, const fx_unit* units, int nunits, int nblocks, bool prec32, cudaStream_t s);
int fx_ade_rows_per_strip();
int fx_ade_threads_per_block();
int fx_ade_max_blocks(int* out);
int fx_fail(fx_ctx* ctx, int code, const char* fmt, ...);

#define FX_NOALLOC_SCRATCH_BYTES (8u << 20)

static __device__ __align__(256) unsigned char g_noalloc_scratch[FX_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
constexpr size_t kCtlBytes = (sizeof(fx_ctl) + 255) & ~(size_t)255;  // fx_ctl, rounded up
constexpr size_t kDevBytes = (sizeof(fx_dev) + 255) & ~(size_t)255;  // fx_dev, rounded up

struct DeviceSetup {
  bool ready = false;
  unsigned long long ctx_id = 0;     // the CUDA context the set-up belongs to
  unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch
  int max_blocks = 0;
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;

// The unique id of the calling thread's current CUDA context (0: none, or the
// driver cannot tell). Context ids are never reused within a process, so a
// changed id means the module and its static array were loaded anew. The two
// driver calls are reached through the runtime, so libcuda is not linked.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool resolved = false;
  if (!resolved) {
    void* a = nullptr;
    void* b = nullptr;
    cudaDriverEntryPointQueryResult qa, qb;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) == cudaSuccess &&
        qa == cudaDriverEntryPointSuccess &&
        cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) == cudaSuccess &&
        qb == cudaDriverEntryPointSuccess) {
      get_current = reinterpret_cast<CtxGetCurrentFn>(a);
      get_id = reinterpret_cast<CtxGetIdFn>(b);
    }
    cudaGetLastError();
    resolved = true;
  }
  if (!get_current || !get_id) return 0;
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Writes the scratch's control block, domain descriptor and work table: one
// sweep with it > 1 (the ADE is skipped on the first solver iteration,
// ADEsolver_calc.cpp:45), one solute, every strip.
__global__ void k_noalloc_setup(fx_dev d, fx_dev* dst, fx_unit* units, int nstrips, double dtfl) {
  for (int s = threadIdx.x; s < nstrips; s += blockDim.x) units[s] = fx_unit{0, 0, 0, s};
  if (threadIdx.x != 0) return;
  *dst = d;
  fx_ctl* ctl = d.ctl;
  fx_ctl c = {};
  c.dtfl = dtfl;
  c.live = 1;
  c.active = 1;
  c.it = 2;
  c.steps = 1;
  c.stop_after = 1;
  c.batch = 1;
  c.rec[0].dtfl = dtfl;
  c.rec[0].step = 1;
  c.rec[0].batch = 1;
  c.rec[0].live = 1;
  c.rec[0].active = 1;
  c.rec[0].it = 2;
  *ctl = c;
}

size_t round256(size_t n) { return (n + 255) & ~(size_t)255; }

}  // namespace

extern "C" int fx_adesolver_noalloc(double* conc, const double* h, const double* h0, const unsigned char* flags,
                                    const double* fe_1, const double* fn_1, int nrows, int ncols, int ld, int dxy,
                                    double dtfl, double d_coef, void* stream) {
  if (!conc || !h || !h0 || !flags || !fe_1 || !fn_1)
    return fx_fail(nullptr, FX_ERR_ARG, "fx_adesolver_noalloc: null array");
  if (nrows < 2 || ncols < 2 || dxy < 1)
    return fx_fail(nullptr, FX_ERR_ARG, "fx_adesolver_noalloc: need nrows, ncols >= 2 and dxy >= 1");
  if (ld < nrows + 2 + FX_ROFF || (((long long)ld * (ncols + 2)) & 3) != 0)
    return fx_fail(nullptr, FX_ERR_ARG,
                   "fx_adesolver_noalloc: ld must be >= nrows + 3 and ld * (ncols + 2) a multiple of 4");
  if (((size_t)flags & 3) != 0 || ((size_t)conc & 15) != 0 || ((size_t)h & 7) != 0 || ((size_t)h0 & 7) != 0 ||
      ((size_t)fe_1 & 7) != 0 || ((size_t)fn_1 & 7) != 0)
    return fx_fail(nullptr, FX_ERR_ARG, "fx_adesolver_noalloc: misaligned array");
  if (!(dtfl > 0.0)) return fx_fail(nullptr, FX_ERR_ARG, "fx_adesolver_noalloc: dtfl must be > 0");

  const int rows = fx_ade_rows_per_strip();
  const int nstrips = (nrows + rows - 1) / rows;
  const size_t unit_bytes = round256((size_t)nstrips * sizeof(fx_unit));
  const size_t prog_bytes = round256((size_t)nstrips * sizeof(unsigned long long));
  const size_t bnd_bytes = (size_t)nstrips * (size_t)(ncols + 2) * 3 * sizeof(double);
  const size_t need = kCtlBytes + kDevBytes + unit_bytes + prog_bytes + bnd_bytes;
  if (need > FX_NOALLOC_SCRATCH_BYTES)
    return fx_fail(nullptr, FX_ERR_ARG,
                   "fx_adesolver_noalloc: a %d x %d grid needs %zu bytes of scratch, more than the %u-byte "
                   "static array (use fx_step on a context instead)",
                   nrows, ncols, need, (unsigned)FX_NOALLOC_SCRATCH_BYTES);

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fx_fail(nullptr, FX_ERR_CUDA, "cudaGetDevice failed: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fx_fail(nullptr, FX_ERR_ARG, "device index %d out of range", dev);
  DeviceSetup s;
  {
    // set-up once per device and context, with the device current: the
    // device address of the static array (its host-side name is not one)
    // and the sweep kernel's resident blocks
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup& g = g_setup[dev];
    const unsigned long long ctx = current_context_id();
    if (!g.ready || ctx == 0 || ctx != g.ctx_id) {
      g.ready = false;
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return fx_fail(nullptr, FX_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch) failed: %s",
                       cudaGetErrorString(e));
      int mb = 0;
      if (fx_ade_max_blocks(&mb) != 0 || mb < 1)
        return fx_fail(nullptr, FX_ERR_CUDA, "occupancy query for the ADE sweep failed");
      g.scratch = (unsigned char*)p;
      g.max_blocks = mb;
      g.ctx_id = current_context_id();  // the look-up made the device's context current
      g.ready = true;
    }
    s = g;
  }
  cudaStream_t st = (cudaStream_t)stream;

  fx_dev d;
  memset(&d, 0, sizeof(d));
  d.nr = nrows;
  d.nc = ncols;
  d.ld = ld;
  d.nchem = 1;
  d.nslot = 1;
  d.plane = (long long)ld * (ncols + 2);
  fx_set_cell_size(d, dxy);
  d.ade = 1;
  d.dcoef[0] = d_coef;
  d.conc = conc;
  d.h = const_cast<double*>(h);
  d.h0 = const_cast<double*>(h0);
  d.flags = const_cast<uint8_t*>(flags);
  d.fe1 = const_cast<double*>(fe_1);
  d.fn1 = const_cast<double*>(fn_1);
  unsigned char* p = s.scratch;
  d.ctl = reinterpret_cast<fx_ctl*>(p);
  fx_dev* d_dev = reinterpret_cast<fx_dev*>(p + kCtlBytes);
  fx_unit* d_units = reinterpret_cast<fx_unit*>(p + kCtlBytes + kDevBytes);
  d.ade_prog = reinterpret_cast<unsigned long long*>(p + kCtlBytes + kDevBytes + unit_bytes);
  d.ade_bnd = reinterpret_cast<double*>(p + kCtlBytes + kDevBytes + unit_bytes + prog_bytes);

  k_noalloc_setup<<<1, 128, 0, st>>>(d, d_dev, d_units, nstrips, dtfl);
  e = cudaMemsetAsync(d.ade_prog, 0, prog_bytes, st);
  if (e != cudaSuccess) return fx_fail(nullptr, FX_ERR_CUDA, "cudaMemsetAsync failed: %s", cudaGetErrorString(e));
  const int per_block = fx_ade_threads_per_block() / 32;
  int nblocks = (nstrips + per_block - 1) / per_block;
  if (nblocks > s.max_blocks) nblocks = s.max_blocks;
  fx_launch_ade(d_dev, d_units, nstrips, nblocks, false, st);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fx_fail(nullptr, FX_ERR_CUDA, "ADE sweep launch failed: %s", cudaGetErrorString(e));
  int err = 0;
  e = cudaMemcpyAsync(&err, &d.ctl->error, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fx_fail(nullptr, FX_ERR_CUDA, "ADE sweep failed: %s", cudaGetErrorString(e));
  if (err) return fx_fail(nullptr, FX_ERR_DEVICE, "device error %d: a bounded wait in the ADE sweep gave up", err);
  return FX_OK;
}
