// The rows of a Results file selected and packed on the device.
//
// write_results (write_results.cpp:30-101) prints one row per interior cell
// with zb != 0 and h > H_MIN_TO_PRINT, columns irow, icol, X, Y, z, z - zb,
// ux, uy, qx * dxy, qy * dxy, us, conc, soil_mass, fe_1, fn_1, twet, cells in
// column-major order (icol outer, irow inner). Here the selection is a
// stream compaction in that order: a count per column (one warp per column,
// warp ballots), an exclusive scan of the counts, then each warp writes its
// column's selected cells at the column's offset. The rows go out as column
// arrays in one buffer, so one device-to-host copy moves them; the host
// formats the text (fluxos_io.cpp). Values are the ones fx_download returns
// for the same state (FP32 state: z = zb + (eta + eta_lo) in FP64), so the
// text matches the host writer's on downloaded grids.
#include "fx_common.cuh"
#include "fx_internal.h"

namespace fxres {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ double cell_h(const fx_dev& d, long long sl, long long gi) {
  return d.prec32 ? (double)fx_rec(d, sl + gi)[FX_R_H] : fx_rec64(d, sl + gi)[FX_R64_H];
}

__device__ __forceinline__ bool selected(const fx_dev& d, long long sl, long long gi, double hmin) {
  return d.zb[gi] != 0.0 && cell_h(d, sl, gi) > hmin;  // write_results.cpp:44-47
}

// Selected cells per column; counts[icol - 1].
__global__ void k_count(const __grid_constant__ fx_dev d, double hmin, unsigned* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  const long long sl = fx_slot(d, d.ctl->steps);
  for (int icol = 1 + warp; icol <= d.nc; icol += nwarps) {
    unsigned n = 0;
    for (int r0 = 1; r0 <= d.nr; r0 += 32) {
      const int irow = r0 + lane;
      const bool p = irow <= d.nr && selected(d, sl, fx_ix(d, irow, icol), hmin);
      n += __popc(__ballot_sync(kFull, p));
    }
    if (lane == 0) counts[icol - 1] = n;
  }
}

// Exclusive scan of n counts by one block of 1024 threads; offs[n] = total.
__global__ void __launch_bounds__(1024) k_scan(const unsigned* __restrict__ counts, int n,
                                               long long* __restrict__ offs) {
  __shared__ long long wsum[32];
  __shared__ long long carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const long long v = i < n ? (long long)counts[i] : 0;
    long long x = v;  // inclusive scan within the warp
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(kFull, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      long long w = wsum[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(kFull, w, o);
        if (lane >= o) w += y;
      }
      wsum[lane] = w;
    }
    __syncthreads();
    const long long excl = carry + (warp > 0 ? wsum[warp - 1] : 0) + (x - v);
    if (i < n) offs[i] = excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) offs[n] = carry;
}

// The packed rows: irow and icol (int32), then nine FP64 columns z, z - zb,
// qx * dxy, qy * dxy, conc, soil_mass, fe_1, fn_1, twet; each array holds
// `total` entries, back to back.
struct Out {
  int* irow;
  int* icol;
  double* v[FX_RES_NVAL];
};

__global__ void k_write(const __grid_constant__ fx_dev d, double hmin, const long long* __restrict__ offs,
                        long long total, Out o) {
  const int lane = threadIdx.x & 31;
  const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  const long long steps = d.ctl->steps;
  const long long sl = fx_slot(d, steps), pp = fx_pp(d, steps);
  const double dx = d.dxy;
  for (int icol = 1 + warp; icol <= d.nc; icol += nwarps) {
    long long pos = offs[icol - 1];
    for (int r0 = 1; r0 <= d.nr; r0 += 32) {
      const int irow = r0 + lane;
      const long long gi = irow <= d.nr ? fx_ix(d, irow, icol) : 0;
      const bool p = irow <= d.nr && selected(d, sl, gi, hmin);
      const unsigned b = __ballot_sync(kFull, p);
      const long long k = pos + __popc(b & ((1u << lane) - 1u));
      if (p && k < total) {
        const double zb = d.zb[gi];
        double z, qx, qy, conc, soil, fe1, fn1, twet;
        if (d.prec32) {
          z = zb + ((double)d.eta[pp + gi] + (double)d.eta_lo[pp + gi]);
          qx = (double)d.qx_f[pp + gi];
          qy = (double)d.qy_f[pp + gi];
          conc = (double)d.conc_f[gi];
          soil = d.soil_f ? (double)d.soil_f[gi] : 0.0;
          fe1 = (double)fx_rec(d, sl + gi)[FX_R_FE1];
          fn1 = (double)fx_rec(d, sl + gi)[FX_R_FN1];
          twet = (double)d.twet_f[gi];
        } else {
          z = d.z[pp + gi];
          qx = d.qx[pp + gi];
          qy = d.qy[pp + gi];
          conc = d.conc[gi];
          soil = d.soil ? d.soil[gi] : 0.0;
          fe1 = fx_rec64(d, sl + gi)[FX_R64_FE1];
          fn1 = fx_rec64(d, sl + gi)[FX_R64_FN1];
          twet = d.twet[gi];
        }
        o.irow[k] = irow;
        o.icol[k] = icol;
        o.v[0][k] = z;
        o.v[1][k] = z - zb;
        o.v[2][k] = qx * dx;
        o.v[3][k] = qy * dx;
        o.v[4][k] = conc;
        o.v[5][k] = soil;
        o.v[6][k] = fe1;
        o.v[7][k] = fn1;
        o.v[8][k] = twet;
      }
      pos += __popc(b);
    }
  }
}

int grid_for(const fx_dev& d) {
  const int warps = d.nc < 148 * 16 ? d.nc : 148 * 16;
  return (warps * 32 + 255) / 256;
}

}  // namespace fxres

void fx_launch_results_count(const fx_dev& d, double h_min_print, unsigned* counts, long long* offs,
                             cudaStream_t s) {
  fxres::k_count<<<fxres::grid_for(d), 256, 0, s>>>(d, h_min_print, counts);
  fxres::k_scan<<<1, 1024, 0, s>>>(counts, d.nc, offs);
}

void fx_launch_results_write(const fx_dev& d, double h_min_print, const long long* offs, void* buf,
                             long long total, cudaStream_t s) {
  fxres::Out o;
  char* p = (char*)buf;
  o.irow = (int*)p;
  o.icol = (int*)(p + 4 * total);
  for (int k = 0; k < FX_RES_NVAL; ++k) o.v[k] = (double*)(p + 8 * total + 8 * total * k);
  fxres::k_write<<<fxres::grid_for(d), 256, 0, s>>>(d, h_min_print, offs, total, o);
}
