// swe_batch.cu -- many independent basins of uneven sizes advanced together.
//
// Each basin is a complete ShallowWater (its own grid, bed, metric, Manning
// n, boundaries and Flather tide) with its own dt = maxDt() every step.  One
// ensemble step is five launches whatever the number of basins:
//   k_batch_prepare     dt and Flather values of every basin (one thread each)
//   k_batch_bc(A)       ghost rings of every basin (grid y = basin)
//   k_batch_stage<1>    every tile of every basin, from one tile list
//   k_batch_bc(B)
//   k_batch_stage<2>    ... the last tile of each basin closes that basin's step
// and a run of steps is captured as a CUDA graph.  The stage kernel is the
// same tile function as the single-grid kernel, so each basin's result is
// bit-identical to advancing it alone.  The tile list's row height, the
// number of CTAs (one per tile, or a persistent grid looping over the list)
// and the order of the tiles form the schedule, which swe_batch_autotune
// chooses by timing candidates on the ensemble itself.
#include "../../include/swe_b200.h"
#include "swe_kernels.cuh"
#include "swe_split.cuh"

#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

namespace swe_host { void set_error(const std::string& msg); }

namespace {

using swe::BCArgs;
using swe::Control;
using swe::PrepArgs;
using swe::StageArgs;

struct BatchBasin {
  StageArgs s1, s2;       // stage 1 (A -> B) and stage 2 (B -> A) arguments
  BCArgs bcA, bcB;
  Control* ctl;
  PrepArgs prep;
  swe::SplitBufs sp;      // faces and source terms of the tiled stage kernels
};

struct BatchTile { int basin, strip, y0, y1, part; };

__global__ void k_batch_prepare(BatchBasin* basins, int nb) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < nb) swe::prepare_one(basins[q].ctl, basins[q].prep);
}

__global__ void k_batch_bc(BatchBasin* basins, int which) {
  const BatchBasin& B = basins[blockIdx.y];
  if (B.ctl->stop) return;
  swe::apply_bc_range(which == 0 ? B.bcA : B.bcB, B.ctl, blockIdx.x * blockDim.x + threadIdx.x,
                      gridDim.x * blockDim.x);
}

template <int MODE>
__global__ void __launch_bounds__(swe::BX, SWE_STAGE_MIN_BLOCKS)
k_batch_stage(BatchBasin* basins, const BatchTile* tiles, int ntiles) {
  extern __shared__ double smem[];
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BatchTile tile = tiles[t];
    const BatchBasin& B = basins[tile.basin];
    swe::stage_tile<MODE>(MODE == 1 ? B.s1 : B.s2, B.ctl, tile.strip, tile.y0, tile.y1, tile.part, smem);
    __syncthreads();          // the next tile reuses the shared rings
  }
}

// The tiled stage pair over the tile list: a tile is (basin, tile column,
// tile row) of that basin's 32 x 8 tiling; its partial slot closes the
// basin's step exactly as in the single-grid kernels.
template <int MODE>
__global__ void __launch_bounds__(swe::SP_THREADS, SWE_SPLIT_FACES_MIN_BLOCKS)
k_batch_split_faces(BatchBasin* basins, const BatchTile* tiles, int ntiles) {
  __shared__ swe::FacesSmem sm;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BatchTile tile = tiles[t];
    const BatchBasin& B = basins[tile.basin];
    if (!B.ctl->stop) swe::split_faces_tile(MODE == 1 ? B.s1 : B.s2, B.sp, tile.strip, tile.y0, sm);
  }
}

template <int MODE>
__global__ void __launch_bounds__(swe::SP_THREADS, SWE_SPLIT_CELLS_MIN_BLOCKS)
k_batch_split_cells(BatchBasin* basins, const BatchTile* tiles, int ntiles) {
  __shared__ swe::CellsSmem sm;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BatchTile tile = tiles[t];
    const BatchBasin& B = basins[tile.basin];
    const StageArgs& a = MODE == 1 ? B.s1 : B.s2;
    if (!B.ctl->stop) swe::split_cells_tile<MODE>(a, B.sp, B.ctl, tile.strip, tile.y0, tile.part, a.nblocks, sm, true);
    __syncthreads();          // the next tile reuses the shared limiter tile
  }
}

// ---- one persistent launch per ensemble step --------------------------------
// A device work queue holds every piece of one ensemble step, phase-major:
//   phase 0  prepare          one item per basin   (dt, Flather values)
//   phase 1  ghost fill of A  one item per basin
//   phase 2  faces of A       one item per tile    (the tile list's order)
//   phase 3  cells, stage 1   one item per tile    (the basin's last tile closes stage 1)
//   phase 4  ghost fill of B  one item per basin
//   phase 5  faces of B       one item per tile
//   phase 6  cells, stage 2   one item per tile    (the basin's last tile closes the step)
// Each CTA takes the next item from a queue head (one atomic) and, before it
// touches memory, waits until the previous phase of the item's basin is
// complete (a per-basin count: 1 or the basin's tile count).  Items are taken
// in queue order, so every item a CTA waits on was taken earlier by a CTA
// that is running; the waits therefore end, whatever the grid size.  Each
// wait still carries a time limit: past it the CTA records a timeout, every
// CTA drops the rest of the step, and the host reads SWE_ETIMEOUT.  The
// completion count is released after a __threadfence and read back with one,
// so a phase's writes are visible to the next phase's CTAs, as at a kernel
// boundary.  The tile functions are the single-grid ones: each basin's result
// is bit-identical to advancing it alone.
constexpr int QPHASES = 7;

struct QueueCtl {
  int* head;                  // next item; reset before every launch
  int* done;                  // [basin * QPHASES + phase]; reset before every launch
  int* err;                   // 1: a wait ran out of time (sticky until the host reads it)
  long long limit_ns;         // the time limit of one wait
  int hold;                   // debug: a basin whose prepare is never marked done (-1: none)
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Thread 0: until done[slot] >= need, bounded by the time limit.
__device__ bool queue_wait(const QueueCtl& q, int slot, int need) {
  volatile int* d = q.done;
  volatile int* e = q.err;
  if (d[slot] >= need) return true;
  const unsigned long long t0 = global_ns();
  while (d[slot] < need) {
    if (*e) return false;
    if ((long long)(global_ns() - t0) > q.limit_ns) {
      atomicExch(q.err, 1);
      return false;
    }
    __nanosleep(256);
  }
  return true;
}

union QueueSmem {
  swe::FacesSmem f;
  swe::CellsSmem c;
};

#ifndef SWE_QUEUE_MIN_BLOCKS
#define SWE_QUEUE_MIN_BLOCKS 3
#endif
__global__ void __launch_bounds__(swe::SP_THREADS, SWE_QUEUE_MIN_BLOCKS)
k_batch_queue_step(BatchBasin* basins, const BatchTile* tiles, int nb, int ntiles, QueueCtl q) {
  __shared__ QueueSmem sm;
  __shared__ int s_item, s_go;
  const int total = 3 * nb + 4 * ntiles;
  for (;;) {
    if (threadIdx.x == 0) s_item = *(volatile int*)q.err ? total : atomicAdd(q.head, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= total) return;                       // uniform
    // the item's phase, basin and (tile phases) tile
    int phase, j = it;
    const int len[QPHASES] = {nb, nb, ntiles, ntiles, nb, ntiles, ntiles};
    for (phase = 0; phase < QPHASES - 1 && j >= len[phase]; phase++) j -= len[phase];
    const bool per_tile = phase == 2 || phase == 3 || phase == 5 || phase == 6;
    const BatchTile tile = per_tile ? tiles[j] : BatchTile{j, 0, 0, 0, 0};
    const int b = tile.basin;
    const BatchBasin& B = basins[b];
    if (threadIdx.x == 0) {
      bool ok = true;
      if (phase > 0) {
        const int prev = phase - 1;
        const int need = (prev == 2 || prev == 3 || prev == 5) ? B.s1.nblocks : 1;
        ok = queue_wait(q, b * QPHASES + prev, need);
      }
      __threadfence();
      s_go = ok ? 1 : 0;
    }
    __syncthreads();
    if (!s_go) return;                             // timed out: drop the rest of the step
    const bool stop = phase > 0 && B.ctl->stop != 0;  // set by this step's prepare
    switch (phase) {
      case 0: if (threadIdx.x == 0) swe::prepare_one(B.ctl, B.prep); break;
      case 1: if (!stop) swe::apply_bc_range(B.bcA, B.ctl, threadIdx.x, blockDim.x); break;
      case 2: if (!stop) swe::split_faces_tile(B.s1, B.sp, tile.strip, tile.y0, sm.f); break;
      case 3: if (!stop) swe::split_cells_tile<1>(B.s1, B.sp, B.ctl, tile.strip, tile.y0, tile.part, B.s1.nblocks,
                                                  sm.c, true);
              break;
      case 4: if (!stop) swe::apply_bc_range(B.bcB, B.ctl, threadIdx.x, blockDim.x); break;
      case 5: if (!stop) swe::split_faces_tile(B.s2, B.sp, tile.strip, tile.y0, sm.f); break;
      default: if (!stop) swe::split_cells_tile<2>(B.s2, B.sp, B.ctl, tile.strip, tile.y0, tile.part,
                                                   B.s2.nblocks, sm.c, true);
               break;
    }
    __syncthreads();                               // the item's writes, then its completion
    if (threadIdx.x == 0 && !(phase == 0 && b == q.hold)) {
      __threadfence();
      atomicAdd(q.done + b * QPHASES + phase, 1);
    }
  }
}

int fail(int code, const std::string& m) { swe_host::set_error(m); return code; }

#define CU(call)                                                                   \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) return fail(SWE_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

}  // namespace

struct swe_batch {
  int nb = 0;
  std::vector<swe_options> opts;
  std::vector<int> W, H;
  std::vector<size_t> off;          // per-basin offset (doubles) of its block in the pool
  std::vector<BatchBasin> host;     // descriptors (device pointers inside)
  cudaStream_t st = nullptr;
  double* pool = nullptr;           // all basins' fields, metric rows and partial slots
  Control* ctls = nullptr;
  BatchBasin* d_basins = nullptr;
  BatchTile* d_tiles = nullptr;
  int ntiles = 0, tile_cap = 0;
  int rows = 32, ctas = 0, order = 0;   // the schedule
  int impl = 1;                         // stage kernels: 0 fused tiles, 1 the tiled pair
  int grid = 0;
  double* save = nullptr;           // autotune snapshot of every basin's A and control
  size_t save_doubles = 0;
  cudaGraphExec_t gexec = nullptr;
  int g_steps = 0;
  unsigned long long version = 1, g_version = 0;
  // one persistent launch per step over a work queue (tiled pair only)
  int queue = 0;
  int* d_queue = nullptr;           // head, done[nb * QPHASES], err
  long long wait_ns = 2000000000LL; // a wait gives up after 2 s
  int hold = -1;
};

namespace {

size_t round_up(size_t n) { return (n + 31) & ~size_t(31); }   // 256-byte multiples

// Tiles of a basin in the tiled pair's 32 x 8 tiling.
size_t split_tiles(int W, int H) {
  return (size_t)((W + swe::SPX - 1) / swe::SPX) * ((H + swe::SPY - 1) / swe::SPY);
}

// Partial slots a basin needs: one per tile at the finest tiling either
// stage implementation uses (4-row fused tiles, or 32 x 8 tiles).
size_t part_slots(int W, int H) {
  const size_t fused = (size_t)((W + swe::SX - 1) / swe::SX) * ((H + 3) / 4);
  const size_t split = (size_t)((W + swe::SPX - 1) / swe::SPX) * ((H + swe::SPY - 1) / swe::SPY);
  return std::max(fused, split);
}

// Fill the tile list for the current schedule and upload it.
int build_tiles(swe_batch* s) {
  std::vector<std::vector<BatchTile>> per(s->nb);
  for (int b = 0; b < s->nb; b++) {
    if (s->impl == 1) {
      const int gx = (s->W[b] + swe::SPX - 1) / swe::SPX, gy = (s->H[b] + swe::SPY - 1) / swe::SPY;
      int part = 0;
      for (int y = 0; y < gy; y++)
        for (int x = 0; x < gx; x++) per[b].push_back({b, x, y, 0, part++});
      continue;
    }
    const int gx = (s->W[b] + swe::SX - 1) / swe::SX;
    const int gy = (s->H[b] + s->rows - 1) / s->rows;
    const int ry = (s->H[b] + gy - 1) / gy;
    int part = 0;
    for (int y = 0; y < gy; y++)
      for (int x = 0; x < gx; x++) {
        const int y0 = y * ry;
        per[b].push_back({b, x, y0, std::min(y0 + ry, s->H[b]), part++});
      }
  }
  std::vector<int> basin_order(s->nb);
  std::iota(basin_order.begin(), basin_order.end(), 0);
  if (s->order == 1)                // largest basins first
    std::stable_sort(basin_order.begin(), basin_order.end(),
                     [&](int a, int b) { return (long)s->W[a] * s->H[a] > (long)s->W[b] * s->H[b]; });
  std::vector<BatchTile> tiles;
  if (s->order == 2) {              // round robin over basins
    size_t most = 0;
    for (auto& v : per) most = std::max(most, v.size());
    for (size_t k = 0; k < most; k++)
      for (int b : basin_order)
        if (k < per[b].size()) tiles.push_back(per[b][k]);
  } else {
    for (int b : basin_order) tiles.insert(tiles.end(), per[b].begin(), per[b].end());
  }
  s->ntiles = (int)tiles.size();
  if (s->ntiles > s->tile_cap) {
    if (s->d_tiles) { cudaStreamSynchronize(s->st); cudaFree(s->d_tiles); s->d_tiles = nullptr; }
    CU(cudaMalloc(&s->d_tiles, sizeof(BatchTile) * s->ntiles));
    s->tile_cap = s->ntiles;
  }
  CU(cudaMemcpyAsync(s->d_tiles, tiles.data(), sizeof(BatchTile) * s->ntiles, cudaMemcpyHostToDevice, s->st));
  // partial-slot counts per basin follow the tile count
  for (int b = 0; b < s->nb; b++) {
    s->host[b].s1.nblocks = (int)per[b].size();
    s->host[b].s2.nblocks = (int)per[b].size();
  }
  CU(cudaMemcpyAsync(s->d_basins, s->host.data(), sizeof(BatchBasin) * s->nb, cudaMemcpyHostToDevice, s->st));
  s->grid = s->ctas > 0 ? s->ctas : s->ntiles;
  CU(cudaStreamSynchronize(s->st));
  s->version++;
  return SWE_OK;
}

int queue_grid(const swe_batch* s) {
  if (s->ctas > 0) return s->ctas;
  int dev = 0, sms = 148, occ = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch_queue_step, swe::SP_THREADS, 0);
  return sms * std::max(occ, 1);                 // one CTA per resident slot
}

int enqueue_queue_step(swe_batch* s) {
  const size_t nint = 1 + (size_t)QPHASES * s->nb;   // head and the completion counts (not err)
  CU(cudaMemsetAsync(s->d_queue, 0, sizeof(int) * nint, s->st));
  QueueCtl q;
  q.head = s->d_queue;
  q.done = s->d_queue + 1;
  q.err = s->d_queue + nint;
  q.limit_ns = s->wait_ns;
  q.hold = s->hold;
  k_batch_queue_step<<<queue_grid(s), swe::SP_THREADS, 0, s->st>>>(s->d_basins, s->d_tiles, s->nb, s->ntiles, q);
  CU(cudaGetLastError());
  return SWE_OK;
}

int enqueue_batch_step(swe_batch* s) {
  if (s->queue && s->impl == 1) return enqueue_queue_step(s);
  k_batch_prepare<<<(s->nb + 63) / 64, 64, 0, s->st>>>(s->d_basins, s->nb);
  CU(cudaGetLastError());
  int most = 0;
  for (int b = 0; b < s->nb; b++) most = std::max(most, 4 * s->opts[b].ny + 4 * (s->opts[b].nx + 4));
  const dim3 bcg((most + 255) / 256, s->nb);
  k_batch_bc<<<bcg, 256, 0, s->st>>>(s->d_basins, 0);
  CU(cudaGetLastError());
  if (s->impl == 1) {
    k_batch_split_faces<1><<<s->grid, swe::SP_THREADS, 0, s->st>>>(s->d_basins, s->d_tiles, s->ntiles);
    k_batch_split_cells<1><<<s->grid, swe::SP_THREADS, 0, s->st>>>(s->d_basins, s->d_tiles, s->ntiles);
  } else {
    k_batch_stage<1><<<s->grid, swe::BX, swe::STAGE_SMEM_BYTES, s->st>>>(s->d_basins, s->d_tiles, s->ntiles);
  }
  CU(cudaGetLastError());
  k_batch_bc<<<bcg, 256, 0, s->st>>>(s->d_basins, 1);
  CU(cudaGetLastError());
  if (s->impl == 1) {
    k_batch_split_faces<2><<<s->grid, swe::SP_THREADS, 0, s->st>>>(s->d_basins, s->d_tiles, s->ntiles);
    k_batch_split_cells<2><<<s->grid, swe::SP_THREADS, 0, s->st>>>(s->d_basins, s->d_tiles, s->ntiles);
  } else {
    k_batch_stage<2><<<s->grid, swe::BX, swe::STAGE_SMEM_BYTES, s->st>>>(s->d_basins, s->d_tiles, s->ntiles);
  }
  CU(cudaGetLastError());
  return SWE_OK;
}

int run_steps(swe_batch* s, int steps) {
  const int chunk = 16;
  if (steps >= chunk && (!s->gexec || s->g_version != s->version || s->g_steps != chunk)) {
    if (s->gexec) { cudaGraphExecDestroy(s->gexec); s->gexec = nullptr; }
    cudaGraph_t graph;
    CU(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
    for (int q = 0; q < chunk; q++) {
      const int rc = enqueue_batch_step(s);
      if (rc) { cudaStreamEndCapture(s->st, &graph); return rc; }
    }
    CU(cudaStreamEndCapture(s->st, &graph));
    const cudaError_t e = cudaGraphInstantiate(&s->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(SWE_ECUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    s->g_steps = chunk;
    s->g_version = s->version;
  }
  int left = steps;
  while (left >= chunk) { CU(cudaGraphLaunch(s->gexec, s->st)); left -= chunk; }
  for (int q = 0; q < left; q++) { const int rc = enqueue_batch_step(s); if (rc) return rc; }
  return SWE_OK;
}

// CFL rate of every basin's current state (the step's epilogue keeps it
// current afterwards).
__global__ void k_batch_cfl(BatchBasin* basins) {
  const BatchBasin& B = basins[blockIdx.x];
  const StageArgs& a = B.s1;
  __shared__ double sm[32];
  double m = 0;
  for (int q = threadIdx.x; q < a.nx * a.ny; q += blockDim.x) {
    const int j = q / a.nx + 2, i = q % a.nx + 2, k = j * a.W + i;
    const double hk = a.h[k];
    if (hk <= a.minDepth) continue;
    const double cc = sqrt(SWE_G * hk);
    const double den = swe::vel_den(hk, a.eps4);
    const double u = fabs(swe::qdiv(swe::vel_num(a.hu[k], hk), den)), v = fabs(swe::qdiv(swe::vel_num(a.hv[k], hk), den));
    const double sr = (u + cc) / a.m.dxRow[j] + (v + cc) / a.m.dyCFL[j];
    if (sr > m) m = sr;
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) mm = fmax(mm, sm[w]);
    B.ctl->next_max = mm;
  }
}

void free_batch(swe_batch* s) {
  if (s->gexec) cudaGraphExecDestroy(s->gexec);
  if (s->pool) cudaFree(s->pool);
  if (s->ctls) cudaFree(s->ctls);
  if (s->d_basins) cudaFree(s->d_basins);
  if (s->d_tiles) cudaFree(s->d_tiles);
  if (s->d_queue) cudaFree(s->d_queue);
  if (s->save) cudaFree(s->save);
  if (s->st) cudaStreamDestroy(s->st);
}

}  // namespace

extern "C" {

int swe_batch_create(int n, const swe_options* opts, const double* const* b, const double* const* h,
                     swe_batch** out) {
  if (!out) return fail(SWE_EINVAL, "null output handle");
  *out = nullptr;
  if (n < 1 || !opts || !b || !h) return fail(SWE_EINVAL, "swe_batch_create: n >= 1 basins with options, b and h");
  swe_batch* s = new swe_batch();
  auto bail = [&](int rc) { free_batch(s); delete s; return rc; };
  s->nb = n;
  s->opts.assign(opts, opts + n);
  std::vector<std::vector<double>> geom(n);
  std::vector<double> scal(6);
  size_t total = 0;
  for (int q = 0; q < n; q++) {
    const swe_options& o = opts[q];
    if (o.nx < 1 || o.ny < 1) return bail(fail(SWE_EINVAL, "basin " + std::to_string(q) + ": nx and ny must be >= 1"));
    if (o.limiter < 0 || o.limiter > 2) return bail(fail(SWE_EINVAL, "unknown limiter; have minmod,mc,central"));
    s->W.push_back(o.nx + 4);
    s->H.push_back(o.ny + 4);
    geom[q].assign((size_t)(SWE_GEOM_NROWS + 3) * s->H[q], 0.0);
    int rc = swe_compute_geometry(&o, geom[q].data(), scal.data());
    if (rc) return bail(rc);
    for (int r = 0; r < 3; r++) {            // reciprocal rows after the 13 metric rows
      const int src = r == 0 ? SWE_GEOM_DXROW : r == 1 ? SWE_GEOM_DYROWN : SWE_GEOM_DYROWS;
      for (int j = 0; j < s->H[q]; j++)
        geom[q][(size_t)(SWE_GEOM_NROWS + r) * s->H[q] + j] = 1.0 / geom[q][(size_t)src * s->H[q] + j];
    }
    const size_t N = (size_t)s->W[q] * s->H[q];
    s->off.push_back(total);
    // b, A (3), B (3), the tiled pair's fields, metric rows, partial slots
    // (3 x one per tile, for the most tiles either kernel uses)
    total += round_up(N) * (7 + swe::SPLIT_FIELDS) + round_up((size_t)(SWE_GEOM_NROWS + 3) * s->H[q]) +
             round_up(3 * part_slots(s->W[q], s->H[q])) + round_up((split_tiles(s->W[q], s->H[q]) + 1) / 2);
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
    return bail(fail(SWE_ECUDA, "no CUDA device is available; this library has no CPU path"));
  if (cudaFuncSetAttribute(k_batch_stage<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, swe::STAGE_SMEM_BYTES) ||
      cudaFuncSetAttribute(k_batch_stage<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, swe::STAGE_SMEM_BYTES) ||
      cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) ||
      cudaMalloc(&s->pool, sizeof(double) * total) ||
      cudaMalloc(&s->ctls, sizeof(Control) * n) ||
      cudaMalloc(&s->d_basins, sizeof(BatchBasin) * n) ||
      cudaMalloc(&s->d_queue, sizeof(int) * (2 + (size_t)QPHASES * n)) ||
      cudaMemsetAsync(s->d_queue, 0, sizeof(int) * (2 + (size_t)QPHASES * n), s->st))
    return bail(fail(SWE_ECUDA, std::string("swe_batch_create: ") + cudaGetErrorString(cudaGetLastError())));
  cudaMemsetAsync(s->ctls, 0, sizeof(Control) * n, s->st);
  cudaMemsetAsync(s->pool, 0, sizeof(double) * total, s->st);
  s->host.resize(n);
  for (int q = 0; q < n; q++) {
    const swe_options& o = opts[q];
    const size_t N = (size_t)s->W[q] * s->H[q], rN = round_up(N);
    double* base = s->pool + s->off[q];
    double* fb = base;
    double* A[3] = {base + rN, base + 2 * rN, base + 3 * rN};
    double* Bf[3] = {base + 4 * rN, base + 5 * rN, base + 6 * rN};
    double* spl = base + 7 * rN;                // the tiled pair's fields
    double* g = base + (7 + swe::SPLIT_FIELDS) * rN;
    const int Hq = s->H[q];
    double* parts = g + round_up((size_t)(SWE_GEOM_NROWS + 3) * Hq);
    const size_t pcap = part_slots(s->W[q], Hq);
    cudaMemcpyAsync(fb, b[q], sizeof(double) * N, cudaMemcpyHostToDevice, s->st);
    cudaMemcpyAsync(A[0], h[q], sizeof(double) * N, cudaMemcpyHostToDevice, s->st);
    cudaMemcpyAsync(g, geom[q].data(), sizeof(double) * geom[q].size(), cudaMemcpyHostToDevice, s->st);
    BatchBasin& B = s->host[q];
    std::memset(&B, 0, sizeof B);
    StageArgs a;
    std::memset(&a, 0, sizeof a);
    a.W = s->W[q]; a.H = Hq; a.nx = o.nx; a.ny = o.ny; a.b = fb;
    a.m.dxRow = g + SWE_GEOM_DXROW * Hq; a.m.dyRowN = g + SWE_GEOM_DYROWN * Hq;
    a.m.dyRowS = g + SWE_GEOM_DYROWS * Hq; a.m.dyCFL = g + SWE_GEOM_DYCFL * Hq;
    a.m.bedPhi = g + SWE_GEOM_BEDPHI * Hq; a.m.geoCoef = g + SWE_GEOM_GEOCOEF * Hq;
    a.m.fRow = g + SWE_GEOM_FROW * Hq; a.m.tanPhi = g + SWE_GEOM_TANPHI * Hq;
    a.m.rdxRow = g + (SWE_GEOM_NROWS + 0) * Hq; a.m.rdyRowN = g + (SWE_GEOM_NROWS + 1) * Hq;
    a.m.rdyRowS = g + (SWE_GEOM_NROWS + 2) * Hq;
    a.dryfold = swe::dry_fold_ok(geom[q].data() + (size_t)SWE_GEOM_NROWS * Hq, (size_t)3 * Hq);
    double Rv = 0;
    {
      std::vector<double> sc(6);
      std::vector<double> tmp((size_t)SWE_GEOM_NROWS * Hq);
      swe_compute_geometry(&o, tmp.data(), sc.data());
      Rv = sc[SWE_SCALAR_R];
    }
    a.m.R = Rv;
    a.minDepth = o.min_depth; a.eps4 = std::pow(swe::jmax(o.min_depth, 1e-12), 4.0);
    a.coriolis = o.coriolis; a.sph = o.sphere; a.order = o.order; a.lim = o.limiter;
    a.manning = o.manning;
    a.part_max = parts; a.part_fl1 = parts + pcap; a.part_fl2 = parts + 2 * pcap;
    B.s1 = a; B.s1.h = A[0]; B.s1.hu = A[1]; B.s1.hv = A[2]; B.s1.oh = Bf[0]; B.s1.ohu = Bf[1]; B.s1.ohv = Bf[2];
    B.s2 = a; B.s2.h = Bf[0]; B.s2.hu = Bf[1]; B.s2.hv = Bf[2]; B.s2.oh = A[0]; B.s2.ohu = A[1]; B.s2.ohv = A[2];
    BCArgs bc;
    bc.nx = o.nx; bc.ny = o.ny; bc.W = s->W[q]; bc.H = Hq;
    for (int side = 0; side < 4; side++) bc.kind[side] = (o.sphere && side < 2) ? SWE_BC_PERIODIC : SWE_BC_REFLECT;
    bc.minDepth = o.min_depth; bc.eps4 = a.eps4; bc.b = fb;
    B.bcA = bc; B.bcA.h = A[0]; B.bcA.hu = A[1]; B.bcA.hv = A[2];
    B.bcB = bc; B.bcB.h = Bf[0]; B.bcB.hu = Bf[1]; B.bcB.hv = Bf[2];
    B.ctl = s->ctls + q;
    B.sp = swe::split_bufs_at(spl, rN);
    B.sp.dry = reinterpret_cast<int*>(parts + round_up(3 * pcap));   // one flag per 32 x 8 tile
    B.sp.ntx = (s->W[q] + swe::SPX - 1) / swe::SPX;
    B.sp.nty = (Hq + swe::SPY - 1) / swe::SPY;
    B.prep.mode = 1; B.prep.dt_host = 0; B.prep.cfl = o.cfl; B.prep.t_end = INFINITY;
  }
  int rc = build_tiles(s);
  if (rc) return bail(rc);
  k_batch_cfl<<<n, 256, 0, s->st>>>(s->d_basins);
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s->st) != cudaSuccess)
    return bail(fail(SWE_ECUDA, "swe_batch_create: initial CFL rate failed"));
  *out = s;
  return SWE_OK;
}

int swe_batch_destroy(swe_batch* s) {
  if (!s) return SWE_OK;
  if (s->st) cudaStreamSynchronize(s->st);
  free_batch(s);
  delete s;
  return SWE_OK;
}

int swe_batch_set_boundary(swe_batch* s, int basin, int side, int kind) {
  if (!s || basin < 0 || basin >= s->nb || side < 0 || side > 3 || kind < 0 || kind > 3)
    return fail(SWE_EINVAL, "swe_batch_set_boundary: bad basin, side or kind");
  s->host[basin].bcA.kind[side] = kind;
  s->host[basin].bcB.kind[side] = kind;
  if (kind != SWE_BC_FLATHER) s->host[basin].prep.fl_kind[side] = 0;
  CU(cudaMemcpyAsync(s->d_basins + basin, &s->host[basin], sizeof(BatchBasin), cudaMemcpyHostToDevice, s->st));
  CU(cudaStreamSynchronize(s->st));
  return SWE_OK;
}

int swe_batch_set_flather_tide(swe_batch* s, int basin, int side, double msl, int n, const double* amp,
                               const double* omega, const double* phase_deg, double u_coef) {
  if (!s || basin < 0 || basin >= s->nb || side < 0 || side > 3 || n < 0 || n > swe::MAX_TIDE ||
      (n > 0 && (!amp || !omega || !phase_deg)))
    return fail(SWE_EINVAL, "swe_batch_set_flather_tide: bad basin, side or table (at most 16 constituents)");
  Control c;
  CU(cudaMemcpyAsync(&c, s->ctls + basin, sizeof c, cudaMemcpyDeviceToHost, s->st));
  CU(cudaStreamSynchronize(s->st));
  c.tide_n[side] = n; c.tide_msl[side] = msl; c.tide_ucoef[side] = u_coef;
  for (int q = 0; q < n; q++) {
    c.tide_amp[side][q] = amp[q]; c.tide_omega[side][q] = omega[q]; c.tide_phase[side][q] = phase_deg[q];
  }
  CU(cudaMemcpyAsync(s->ctls + basin, &c, sizeof c, cudaMemcpyHostToDevice, s->st));
  s->host[basin].bcA.kind[side] = SWE_BC_FLATHER;
  s->host[basin].bcB.kind[side] = SWE_BC_FLATHER;
  s->host[basin].prep.fl_kind[side] = 1;
  CU(cudaMemcpyAsync(s->d_basins + basin, &s->host[basin], sizeof(BatchBasin), cudaMemcpyHostToDevice, s->st));
  CU(cudaStreamSynchronize(s->st));
  return SWE_OK;
}

int swe_batch_set_schedule(swe_batch* s, int rows_per_tile, int ctas, int order) {
  if (!s || !(rows_per_tile == 0 || (rows_per_tile >= 4 && rows_per_tile <= swe::RY_MAX)) || ctas < 0 ||
      order < 0 || order > 2)
    return fail(SWE_EINVAL, "swe_batch_set_schedule: rows 0 (tiled pair) or in [4, 64], ctas >= 0, order 0..2");
  s->impl = rows_per_tile == 0 ? 1 : 0;
  if (rows_per_tile) s->rows = rows_per_tile;
  s->ctas = ctas; s->order = order;
  return build_tiles(s);
}

int swe_batch_get_schedule(swe_batch* s, int* out4) {
  if (!s || !out4) return fail(SWE_EINVAL, "null argument");
  out4[0] = s->impl == 1 ? 0 : s->rows; out4[1] = s->ctas; out4[2] = s->order; out4[3] = s->ntiles;
  return SWE_OK;
}

int swe_batch_run(swe_batch* s, int steps) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  if (steps <= 0) return SWE_OK;
  return run_steps(s, steps);
}

int swe_batch_synchronize(swe_batch* s) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  CU(cudaStreamSynchronize(s->st));
  int* err = s->d_queue + 1 + (size_t)QPHASES * s->nb;
  int e = 0;
  CU(cudaMemcpy(&e, err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    CU(cudaMemset(err, 0, sizeof(int)));
    return fail(SWE_ETIMEOUT, "swe_batch: a work-queue wait ran past its time limit; the steps in flight "
                              "were dropped and the basins' state is not a completed step");
  }
  return SWE_OK;
}

int swe_batch_set_launch(swe_batch* s, int queue) {
  if (!s || (queue != 0 && queue != 1)) return fail(SWE_EINVAL, "swe_batch_set_launch: 0 (a launch per phase) or 1");
  if (queue && s->impl != 1)
    return fail(SWE_EINVAL, "swe_batch_set_launch: the work queue runs the tiled stage pair (schedule rows 0)");
  s->queue = queue;
  s->version++;
  return SWE_OK;
}

int swe_batch_get_launch(swe_batch* s, int* queue) {
  if (!s || !queue) return fail(SWE_EINVAL, "null argument");
  *queue = s->queue && s->impl == 1 ? 1 : 0;
  return SWE_OK;
}

int swe_batch_set_wait_limit(swe_batch* s, double seconds) {
  if (!s || !(seconds > 0) || !(seconds <= 60)) return fail(SWE_EINVAL, "swe_batch_set_wait_limit: 0 < seconds <= 60");
  s->wait_ns = (long long)(seconds * 1e9);
  s->version++;
  return SWE_OK;
}

int swe_batch_debug_hold(swe_batch* s, int basin) {
  if (!s || basin < -1 || basin >= s->nb) return fail(SWE_EINVAL, "swe_batch_debug_hold: a basin or -1");
  s->hold = basin;
  s->version++;
  return SWE_OK;
}

int swe_batch_get_stream(swe_batch* s, void** stream) {
  if (!s || !stream) return fail(SWE_EINVAL, "null argument");
  *stream = (void*)s->st;
  return SWE_OK;
}

int swe_batch_get_field(swe_batch* s, int basin, int field, double* out) {
  if (!s || !out || basin < 0 || basin >= s->nb) return fail(SWE_EINVAL, "swe_batch_get_field: bad basin");
  const BatchBasin& B = s->host[basin];
  const double* p = field == SWE_FIELD_B ? B.s1.b : field == SWE_FIELD_H ? B.s1.h :
                    field == SWE_FIELD_HU ? B.s1.hu : field == SWE_FIELD_HV ? B.s1.hv : nullptr;
  if (!p) return fail(SWE_EINVAL, "swe_batch_get_field: b, h, hu or hv");
  CU(cudaMemcpyAsync(out, p, sizeof(double) * s->W[basin] * s->H[basin], cudaMemcpyDeviceToHost, s->st));
  CU(cudaStreamSynchronize(s->st));
  return SWE_OK;
}

int swe_batch_get_scalar(swe_batch* s, int basin, int which, double* out) {
  if (!s || !out || basin < 0 || basin >= s->nb) return fail(SWE_EINVAL, "swe_batch_get_scalar: bad basin");
  Control c;
  CU(cudaMemcpyAsync(&c, s->ctls + basin, sizeof c, cudaMemcpyDeviceToHost, s->st));
  CU(cudaStreamSynchronize(s->st));
  if (which == SWE_SCALAR_T) *out = c.t;
  else if (which == SWE_SCALAR_STEPS) *out = c.steps;
  else if (which == SWE_SCALAR_MASS_FLOORED) *out = c.mass_floored;
  else return fail(SWE_EINVAL, "swe_batch_get_scalar: t, steps or massFloored");
  return SWE_OK;
}

int swe_batch_autotune(swe_batch* s, int trial_steps, int* best4, double* best_ms) {
  if (!s || trial_steps < 1) return fail(SWE_EINVAL, "swe_batch_autotune: trial_steps >= 1");
  // snapshot every basin's state and control, restored after each trial
  size_t n = 0;
  for (int b = 0; b < s->nb; b++) n += 3 * (size_t)s->W[b] * s->H[b];
  if (!s->save) {
    CU(cudaMalloc(&s->save, sizeof(double) * n + sizeof(Control) * s->nb));
    s->save_doubles = n;
  }
  auto snapshot = [&](bool restore) -> int {
    size_t o = 0;
    for (int b = 0; b < s->nb; b++) {
      const size_t N = (size_t)s->W[b] * s->H[b];
      double* f[3] = {s->host[b].s2.oh, s->host[b].s2.ohu, s->host[b].s2.ohv};   // A = (h, hu, hv)
      for (int q = 0; q < 3; q++) {
        if (restore) CU(cudaMemcpyAsync(f[q], s->save + o, sizeof(double) * N, cudaMemcpyDeviceToDevice, s->st));
        else CU(cudaMemcpyAsync(s->save + o, f[q], sizeof(double) * N, cudaMemcpyDeviceToDevice, s->st));
        o += N;
      }
    }
    Control* cs = reinterpret_cast<Control*>(s->save + s->save_doubles);
    if (restore) CU(cudaMemcpyAsync(s->ctls, cs, sizeof(Control) * s->nb, cudaMemcpyDeviceToDevice, s->st));
    else CU(cudaMemcpyAsync(cs, s->ctls, sizeof(Control) * s->nb, cudaMemcpyDeviceToDevice, s->st));
    return SWE_OK;
  };
  int rc = snapshot(false);
  if (rc) return rc;
  int dev = 0, sms = 148, occ = 3, occ_split = 3;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch_stage<2>, swe::BX, swe::STAGE_SMEM_BYTES);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_split, k_batch_split_faces<2>, swe::SP_THREADS, 0);
  const int rows_c[] = {0, 16, 24, 32, 48, 64};          // 0: the tiled pair
  double best = INFINITY;
  int bi = s->impl, br = s->rows, bc = s->ctas, bo = s->order, bq = s->queue;
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  // candidates: (rows, ctas index, order) with a launch per phase, then the
  // tiled pair as one queue launch per step over a resident or a
  // one-per-SM grid
  for (int r : rows_c)
    for (int ci = 0; ci < 5; ci++)
      for (int o = 0; o < 3; o++) {
        const bool queue = ci >= 3;
        if (queue && r != 0) continue;
        const int per_sm = std::max(r == 0 ? occ_split : occ, 1);
        const int c = queue ? (ci == 3 ? 0 : sms) : (ci == 0 ? 0 : ci * sms * per_sm);
        s->impl = r == 0 ? 1 : 0;
        if (r) s->rows = r;
        s->ctas = c; s->order = o; s->queue = queue ? 1 : 0;
        rc = build_tiles(s);
        if (rc) return rc;
        rc = run_steps(s, 1);                    // warm
        if (rc) return rc;
        CU(cudaEventRecord(e0, s->st));
        rc = run_steps(s, trial_steps);
        if (rc) return rc;
        CU(cudaEventRecord(e1, s->st));
        CU(cudaEventSynchronize(e1));
        float ms = 0;
        CU(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) { best = ms; bi = s->impl; br = s->rows; bc = c; bo = o; bq = s->queue; }
        rc = snapshot(true);
        if (rc) return rc;
        rc = swe_batch_synchronize(s);           // a timed-out trial reports here
        if (rc) return rc;
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  s->impl = bi; s->rows = br; s->ctas = bc; s->order = bo; s->queue = bq;
  rc = build_tiles(s);
  if (rc) return rc;
  CU(cudaStreamSynchronize(s->st));
  if (best4) { best4[0] = bi == 1 ? 0 : br; best4[1] = bc; best4[2] = bo; best4[3] = s->ntiles; }
  if (best_ms) *best_ms = best / trial_steps;
  return SWE_OK;
}

}  // extern "C"
