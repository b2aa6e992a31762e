// swe_noalloc.cu -- maxDt() for callers that cannot allocate device memory.
//
// Some callers of this library may not call cudaMalloc at all: a host
// runtime that owns every byte of device memory through its own arena (a
// Node worker or game loop handed a fixed device pool), a process running
// under a hard device-memory cap, or code inside a region where the
// surrounding framework forbids allocation.  swe_max_dt() reduces through
// per-simulation buffers the library allocated at swe_create(); this entry
// point computes the same CFL step from device arrays the caller already
// owns, and keeps its reduction scratch in one fixed array compiled into the
// library instead of allocating any.
//
// The scratch array (SWE_NOALLOC_MAX_ROWS + 1 doubles, 128 KB) lives on
// every GPU that loads the library until the process exits.  Slot 0 holds
// the last-block ticket, slots 1..ny the per-row maxima.  Every call shares
// it, so two calls whose kernels overlap on the GPU race and give undefined
// results: serialise them (one stream, or events between streams).
#include "../../include/swe_b200.h"
#include "swe_math.cuh"

#include <cuda_runtime.h>
#include <cmath>
#include <mutex>
#include <string>

namespace {

constexpr int MAX_ROWS = SWE_NOALLOC_MAX_ROWS;
constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) double g_noalloc_scratch[MAX_ROWS + 1];

// Device address of g_noalloc_scratch on each device.  In host code the
// symbol is only a host-side stand-in, so the address is looked up on the
// first call on each device, with that device current, and passed to the
// kernel.  Only a successful lookup is kept: a failed one is tried again on
// the next call.  The address belongs to the device's context, so it goes
// stale after cudaDeviceReset(); the entry point is not for use after one.
double* g_addr[MAX_DEVICES] = {};
std::mutex g_addr_mu;

// Each block reduces one interior row; the last block to finish reduces the
// row maxima and writes dt = cfl / max (Infinity when no cell is wet),
// src/swe.mjs:632-647.
__global__ void k_cfl_rows_noalloc(int nx, int ny, const double* h, const double* hu, const double* hv,
                                   const double* dxRow, const double* dyCFL, double minDepth, double eps4,
                                   double cfl, double* scratch, double* out) {
  __shared__ double s_max[8];
  __shared__ bool s_last;
  const int W = nx + 4;
  const int j = blockIdx.x + 2;
  double m = 0;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) {
    const int k = j * W + (i + 2);
    const double hk = h[k];
    if (hk <= minDepth) continue;
    const double c = sqrt(SWE_G * hk);
    const double den = swe::vel_den(hk, eps4);
    const double u = fabs(swe::vel_num(hu[k], hk) / den), v = fabs(swe::vel_num(hv[k], hk) / den);
    const double s = (u + c) / dxRow[j] + (v + c) / dyCFL[j];
    if (s > m) m = s;
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = s_max[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) mm = fmax(mm, s_max[w]);
    scratch[1 + blockIdx.x] = mm;
    __threadfence();
    unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch);
    s_last = atomicAdd(ticket, 1u) == (unsigned int)(ny - 1);
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    __threadfence();
    double mm = 0;
    for (int q = 0; q < ny; q++) mm = fmax(mm, ((volatile double*)scratch)[1 + q]);
    *out = mm > 0 ? cfl / mm : INFINITY;
    *reinterpret_cast<unsigned int*>(scratch) = 0;
  }
}

}  // namespace

namespace swe_host { void set_error(const std::string& msg); }   // swe_api.cu: swe_last_error()

extern "C" int swe_max_dt_noalloc(int nx, int ny, const double* h, const double* hu, const double* hv,
                                  const double* dx_row, const double* dy_cfl, double min_depth,
                                  double cfl, double* dt_out, void* stream) {
  if (nx < 1 || ny < 1 || !h || !hu || !hv || !dx_row || !dy_cfl || !dt_out) {
    swe_host::set_error("swe_max_dt_noalloc: nx, ny must be >= 1 and every pointer non-null");
    return SWE_EINVAL;
  }
  if (ny > MAX_ROWS) {
    swe_host::set_error("swe_max_dt_noalloc: ny = " + std::to_string(ny) + " exceeds the fixed scratch of " +
            std::to_string(MAX_ROWS) + " rows; use swe_max_dt on a handle for larger grids");
    return SWE_EINVAL;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) {
    swe_host::set_error(std::string("swe_max_dt_noalloc: no usable current device: ") + cudaGetErrorString(e));
    return SWE_ECUDA;
  }
  // Set-up on the first call on this device (before any stream capture).
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_addr_mu);
    if (!g_addr[dev]) {
      void* p = nullptr;
      const cudaError_t le = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (le != cudaSuccess || !p) {
        swe_host::set_error(std::string("swe_max_dt_noalloc: cudaGetSymbolAddress failed: ") +
                            cudaGetErrorString(le));
        return SWE_ECUDA;
      }
      g_addr[dev] = static_cast<double*>(p);
    }
    scratch = g_addr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // The ticket must start at zero; clear it rather than trust the last call.
  e = cudaMemsetAsync(scratch, 0, sizeof(double), st);
  if (e == cudaSuccess) {
    const double eps4 = std::pow(swe::jmax(min_depth, 1e-12), 4.0);
    k_cfl_rows_noalloc<<<ny, 256, 0, st>>>(nx, ny, h, hu, hv, dx_row, dy_cfl, min_depth, eps4, cfl,
                                           scratch, dt_out);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    swe_host::set_error(std::string("swe_max_dt_noalloc: ") + cudaGetErrorString(e));
    return SWE_ECUDA;
  }
  return SWE_OK;
}
