// swe_split.cuh -- one SSP-RK2 stage as two tiled kernels.
//
// The same arithmetic as stage_tile<MODE> (swe_kernels.cuh), operation for
// operation and in the same accumulation order, organised for occupancy
// instead of on-chip reuse:
//
//   k_split_faces   a 32 x 8 tile of cells per CTA: the state of the tile
//                   and a one-cell halo into shared memory with its
//                   velocities, the MUSCL slopes of the tile (plus the east
//                   column and north row the faces need), then per cell its
//                   east x face and north y face (HLLC, src/swe.mjs:415-475)
//                   and its bed / geometric source terms (src/swe.mjs:570-598),
//                   written to face and term arrays.  This holds the FP64
//                   work (two HLLC solves per cell) at 256 threads per CTA.
//   k_split_cells   per cell: the positivity limiter of the cell and its
//                   neighbours from the faces (src/swe.mjs:511-529), the
//                   four faces gathered west, east, south, north
//                   (src/swe.mjs:530-555), the source terms, Coriolis, and
//                   the stage update with its epilogue (dryClean, friction,
//                   sponge, CFL rate; src/swe.mjs:659-813).  The last block
//                   to finish closes the step as the fused kernel does.
//
// Both are written as tile functions (split_faces_tile, split_cells_tile)
// that a single-grid kernel calls once and the batched ensemble calls for
// every tile of its tile list.  Face arrays are indexed by their left /
// lower cell and are zero where no face exists, so the limiter reads them
// unconditionally.
//
// Dry tiles.  When every cell of a tile and its one-cell halo has h exactly
// 0, every face the tile owns is exactly +0 (both sides dry, so HLLC and
// both pressure corrections vanish), every slope is 0, and its source terms
// are +-0.  The face kernel then writes only the tile's dry flag; the cell
// kernel reads a face or source term of a flagged tile as +0 without
// loading it, and skips the limiter of a tile whose 3 x 3 neighbourhood is
// all flagged (theta is 1 when the faces are zero).  Sums of +-0 terms
// round to the same doubles either way, so the results are unchanged bit
// for bit; only the memory traffic of dry land goes.
#pragma once

#include <cuda.h>                 // CUtensorMap

#include "swe_kernels.cuh"

namespace swe {
namespace {

constexpr int SPX = 32, SPY = 8;                 // tile of owned cells
constexpr int SP_THREADS = SPX * SPY;
constexpr int SSX = SPX + 3, SSY = SPY + 3;     // state tile: cols i0-1 .. i0+SPX+1, rows j0-1 .. j0+SPY+1

// A face is kept as the four values the gather reads: the mass flux M, the
// transverse flux T, and the normal-momentum flux plus each side's pressure
// correction, N + pL for the left / lower cell and N + pR for the right /
// upper one (the same sums the gather forms, so no rounding changes).
enum { F_M = 0, F_T = 1, F_NPL = 2, F_NPR = 3, SPLIT_FACE_FIELDS = 4 };
constexpr int SPLIT_FIELDS = 2 * SPLIT_FACE_FIELDS + 4;   // faces, 3 source terms, u

struct SplitBufs {
  double* fx[SPLIT_FACE_FIELDS];   // x face (k|k+1)
  double* fy[SPLIT_FACE_FIELDS];   // y face (k|k+W)
  double* tb[3];                   // bed term x, bed term y, geometric source
  double* U;                       // cell velocity u (spherical Coriolis)
  // optional, for the adjoint's tape: every cell's slopes (x: eta, b, u, v;
  // then y) and velocity v; with them set, u is written for every cell too
  // (and no tile is skipped as dry)
  double* sl[8];
  double* V;
  int* dry;                        // per tile: 1 when its faces were not written (dry), or null
  int ntx, nty;                    // tiles per row and column of the grid
  // optional, per tile of the stage's input / output state: 1 when every
  // cell of the tile has h exactly 0 and none is a ghost cell (so nothing
  // but a stage or the host writes it), 2 when moreover the cell kernel
  // settled the tile to h = hu = hv = +0 without computing it (below).
  // The cell kernel writes odry_out with the state; the face kernel reads
  // odry_in.  Whoever else writes the state clears them.
  const int* odry_in;
  int* odry_out;
};

// The SPLIT_FIELDS fields of one grid, `stride` doubles apart from `base`.
__host__ __forceinline__ SplitBufs split_bufs_at(double* base, size_t stride) {
  SplitBufs b;
  for (int q = 0; q < SPLIT_FACE_FIELDS; q++) {
    b.fx[q] = base + q * stride;
    b.fy[q] = base + (SPLIT_FACE_FIELDS + q) * stride;
  }
  for (int q = 0; q < 3; q++) b.tb[q] = base + (2 * SPLIT_FACE_FIELDS + q) * stride;
  b.U = base + (2 * SPLIT_FACE_FIELDS + 3) * stride;
  for (int q = 0; q < 8; q++) b.sl[q] = nullptr;
  b.V = nullptr;
  b.dry = nullptr;
  b.ntx = b.nty = 0;
  b.odry_in = nullptr;
  b.odry_out = nullptr;
  return b;
}

// Whether `n` reciprocal metric values are all finite (StageArgs::dryfold).
__host__ inline int dry_fold_ok(const double* recip, size_t n) {
  for (size_t q = 0; q < n; q++)
    if (!(recip[q] - recip[q] == 0)) return 0;      // inf - inf and NaN - NaN are NaN
  return 1;
}

// 8-byte global -> shared copy that runs asynchronously (cp.async, sm_80+):
// a thread issues all of its copies, then waits once, so their latencies
// overlap instead of adding up.  Only the issuing thread reads the copied
// value, after cp_async_wait_all.
__device__ __forceinline__ void cp_async8(void* sdst, const void* gsrc) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// The state tile is stored SSXT = SSX + 1 columns wide starting one column
// further west (gi = i0 - 2 at column 0, so column TCOL + lx holds gi =
// i0 - 1 + lx): that is the box a tensor-map copy can fetch, whose first
// column must sit on a 16-byte boundary of the row (an even column index).
// Each array starts on a 128-byte boundary for the same copy.
constexpr int TCOL = 1, SSXT = SSX + TCOL;
struct FacesSmem {
  alignas(128) double b[SSY][SSXT];
  alignas(128) double h[SSY][SSXT];
  alignas(128) double U[SSY][SSXT];
  alignas(128) double V[SSY][SSXT];
  double xs[4][SPY][SPX + 1];                   // x slopes of cols i0 .. i0+SPX, rows j0 .. j0+SPY-1
  double ys[4][SPY + 1][SPX];                   // y slopes of cols i0 .. i0+SPX-1, rows j0 .. j0+SPY
};

// One cell of a faces tile: its source terms, its east x face and north y face.
__device__ __forceinline__ void split_faces_cell(const StageArgs& a, const SplitBufs& s, const FacesSmem& sm,
                                                 int lx, int ly, int gi, int gj, bool sph, bool bedOn) {
  const int W = a.W, H = a.H;
  const double dry = a.minDepth;
  const int k = gj * W + gi;
  const int cx = lx + 1 + TCOL, cy = ly + 1;
  const double bk = sm.b[cy][cx], hk = sm.h[cy][cx], Uk = sm.U[cy][cx], Vk = sm.V[cy][cx];
  const double xsE = sm.xs[0][ly][lx], xsB = sm.xs[1][ly][lx];
  const double nsE = sm.ys[0][ly][lx], nsB = sm.ys[1][ly][lx];

  // bed term and geometric source of the cell (src/swe.mjs:570-598)
  double tb0 = 0, tb1 = 0, tg = 0;
  if (bedOn && gj >= 2 && gj < H - 2 && gi >= 2 && gi < W - 2) {
    const double eC = bk + hk;
    {
      const double hP = jmax0(eC + 0.5 * xsE - (bk + 0.5 * xsB));
      const double hM = jmax0(eC - 0.5 * xsE - (bk - 0.5 * xsB));
      tb0 = div_unless_zero(-SWE_G * 0.5 * (hP + hM) * xsB, xsB, a.m.dxRow[gj]);
    }
    {
      const double hP = jmax0(eC + 0.5 * nsE - (bk + 0.5 * nsB));
      const double hM = jmax0(eC - 0.5 * nsE - (bk - 0.5 * nsB));
      tb1 = div_unless_zero(-SWE_G * 0.5 * (hP + hM) * nsB, nsB, a.m.bedPhi[gj]);
      if (sph) tg = a.m.geoCoef[gj] * SWE_G * (hP * hP + hM * hM);
    }
  }
  s.tb[0][k] = tb0; s.tb[1][k] = tb1; s.tb[2][k] = tg;
  if (s.sl[0]) {
    for (int q = 0; q < 4; q++) { s.sl[q][k] = sm.xs[q][ly][lx]; s.sl[4 + q][k] = sm.ys[q][ly][lx]; }
    s.U[k] = Uk;
    s.V[k] = Vk;
  } else if (sph) {
    s.U[k] = Uk;
  }

  // The east x face (k|k+1), then the north y face (k|k+W; v normal, u
  // transverse), through one copy of the face solve: a loop of two passes
  // that is not unrolled, so that the solve, the bulk of the kernel's code,
  // sits in the instruction cache once.
  constexpr int XS = SPY * (SPX + 1), YS = (SPY + 1) * SPX;   // strides of xs[q], ys[q]
#pragma unroll 1
  for (int d = 0; d < 2; d++) {
    const bool on = d == 0 ? (gj >= 2 && gj < H - 2 && gi >= 1 && gi < W - 2)
                           : (gj >= 1 && gj < H - 2 && gi >= 2 && gi < W - 2);
    const double* sp = d == 0 ? &sm.xs[0][ly][lx] : &sm.ys[0][ly][lx];
    const int fs = d == 0 ? XS : YS, no = d == 0 ? 1 : SPX;       // field stride, the neighbour's offset
    const int qn = d == 0 ? 2 : 3, qt = 5 - qn;                  // normal and transverse velocity slopes
    const int ry = d == 0 ? cy : cy + 1, rx = d == 0 ? cx + 1 : cx;
    Face f = {0, 0, 0, 0, 0};
    if (on) {
      f = face_flux(bk, hk, d == 0 ? Uk : Vk, d == 0 ? Vk : Uk, sp[0], sp[fs], sp[qn * fs], sp[qt * fs],
                    sm.b[ry][rx], sm.h[ry][rx], d == 0 ? sm.U[ry][rx] : sm.V[ry][rx],
                    d == 0 ? sm.V[ry][rx] : sm.U[ry][rx],
                    sp[no], sp[fs + no], sp[qn * fs + no], sp[qt * fs + no], dry);
    }
    double* const* o = d == 0 ? s.fx : s.fy;
    o[F_M][k] = f.M; o[F_T][k] = f.T; o[F_NPL][k] = f.N + f.pL; o[F_NPR][k] = f.N + f.pR;
  }
}

__device__ __forceinline__ void split_faces_finish(const StageArgs& a, const SplitBufs& s, int tx, int ty,
                                                   FacesSmem& sm, int t);

// A tile whose 3 x 3 neighbourhood of tiles holds only h == 0 (outside the
// grid counts as zero state) is dry with its halo: nothing to load.  Marks
// it dry and returns true (uniform across the CTA).
__device__ __forceinline__ bool split_faces_settled(const SplitBufs& s, int tx, int ty, int t) {
  if (!(s.odry_in && s.dry && !s.sl[0])) return false;
  int f = 1;
  if (t < 9) {
    const int r = t / 3, c = t - 3 * r, txn = tx - 1 + c, tyn = ty - 1 + r;
    if (txn >= 0 && txn < s.ntx && tyn >= 0 && tyn < s.nty) f = s.odry_in[tyn * s.ntx + txn];
  }
  if (__syncthreads_and(f)) {
    if (t == 0) s.dry[ty * s.ntx + tx] = 1;
    return true;
  }
  return false;
}

// Faces and source terms of the tile (tx, ty).  Every thread of the CTA
// calls it; it returns with the shared memory free for the next tile.
__device__ __forceinline__ void split_faces_tile(const StageArgs& a, const SplitBufs& s, int tx, int ty,
                                                 FacesSmem& sm) {
  const int W = a.W, H = a.H;
  const int i0 = tx * SPX, j0 = ty * SPY;
  const int t = threadIdx.x;
  if (split_faces_settled(s, tx, ty, t)) return;

  // state of the tile and its halo (zero outside the grid): b, h, hu, hv
  // copied into b, h, U, V with every copy of the thread in flight at once;
  // once the tile is known to be wet, each thread turns the hu, hv it
  // copied into velocities in place
  for (int q = t; q < SSX * SSY; q += SP_THREADS) {
    const int ly = q / SSX, lx = q - ly * SSX;
    const int gi = i0 - 1 + lx, gj = j0 - 1 + ly;
    if (gi >= 0 && gi < W && gj >= 0 && gj < H) {
      const int k = gj * W + gi;
      cp_async8(&sm.b[ly][lx + TCOL], a.b + k);
      cp_async8(&sm.h[ly][lx + TCOL], a.h + k);
      cp_async8(&sm.U[ly][lx + TCOL], a.hu + k);
      cp_async8(&sm.V[ly][lx + TCOL], a.hv + k);
    } else {
      sm.b[ly][lx + TCOL] = 0; sm.h[ly][lx + TCOL] = 0; sm.U[ly][lx + TCOL] = 0; sm.V[ly][lx + TCOL] = 0;
    }
  }
  if (t < SSY) {                                // column 0 (i0 - 2) is in the box but not needed
    sm.b[t][0] = 0; sm.h[t][0] = 0; sm.U[t][0] = 0; sm.V[t][0] = 0;
  }
  cp_async_wait_all();
  split_faces_finish(a, s, tx, ty, sm, t);
}

// Limited slopes of eta, b, u, v at the state-tile cell (cy, cx) along x
// (DX = 1) or y (DX = 0), src/swe.mjs:364-411: all four are 0 unless `on`
// and the cell and both neighbours along the direction are wet.  LIM 0 is
// the MC limiter inline; LIM -1 the options' limiter chosen at run time.
// out[q * stride]: the slopes of eta, b, u, v in turn (each stored as soon
// as it is formed).
template <int DX, int LIM>
__device__ __forceinline__ void tile_slopes(const FacesSmem& sm, int lim, double dry, bool on, int cy, int cx,
                                            double* out, int stride) {
  constexpr int DY = 1 - DX;
  const int l = LIM < 0 ? lim : LIM;
  double sE = 0, sB = 0, sU = 0, sV = 0;
  if (on) {
    const double hk = sm.h[cy][cx], hp = sm.h[cy + DY][cx + DX], hm = sm.h[cy - DY][cx - DX];
    if (!(hk <= dry || hp <= dry || hm <= dry)) {
      const double bk = sm.b[cy][cx], bp = sm.b[cy + DY][cx + DX], bm = sm.b[cy - DY][cx - DX];
      sE = limiter(l, (bk + hk) - (bm + hm), (bp + hp) - (bk + hk));
      sB = limiter(l, bk - bm, bp - bk);
      const double uk = sm.U[cy][cx];
      sU = limiter(l, uk - sm.U[cy - DY][cx - DX], sm.U[cy + DY][cx + DX] - uk);
      const double vk = sm.V[cy][cx];
      sV = limiter(l, vk - sm.V[cy - DY][cx - DX], sm.V[cy + DY][cx + DX] - vk);
    }
  }
  out[0] = sE; out[stride] = sB; out[2 * stride] = sU; out[3 * stride] = sV;
}

// The rest of a faces tile once its state tile is in shared memory: the
// dry test, velocities, slopes and faces.  Every thread of the CTA calls it.
template <int LIM>
__device__ __forceinline__ void split_faces_finish_l(const StageArgs& a, const SplitBufs& s, int tx, int ty,
                                                     FacesSmem& sm, int t) {
  const int W = a.W, H = a.H;
  const int i0 = tx * SPX, j0 = ty * SPY;
  const double dry = a.minDepth, eps4 = a.eps4;
  const bool order2 = a.order >= 2;
  const bool sph = a.sph != 0;
  const bool bedOn = order2 || sph;
  int dryHere = 1;
  for (int q = t; q < SSX * SSY; q += SP_THREADS) {
    const int ly = q / SSX, lx = q - ly * SSX;
    if (!(sm.h[ly][lx + TCOL] == 0)) dryHere = 0;     // zero outside the grid
  }
  const bool allDry = __syncthreads_and(dryHere) && s.dry && !s.sl[0];
  if (s.dry && t == 0) s.dry[ty * s.ntx + tx] = allDry ? 1 : 0;
  if (allDry) return;                           // uniform across the CTA
  // velocities over the whole box; a cell outside the grid has h = hu =
  // hv = 0 there and gets u = v = +0, as it would have kept
  // The box has more cells than the CTA has threads: the second pass goes
  // to the last threads, since the first two warps take the extra slopes.
  constexpr int VREM = SSXT * SSY - SP_THREADS;
  static_assert(VREM > 0 && VREM <= SP_THREADS, "one or two box cells per thread");
  for (int pass = 0; pass < 2; pass++) {
    if (pass == 1 && t < SP_THREADS - VREM) break;
    const int q = pass == 0 ? t : t + VREM;
    const int ly = q / SSXT, c = q - ly * SSXT;
    const double h = sm.h[ly][c], hu = sm.U[ly][c], hv = sm.V[ly][c];
    double U, V;
    if (h == 0) {                  // +-0 / den == +-0 and NaN / den == NaN: no division needed
      U = vel_num(hu, h); V = vel_num(hv, h);
    } else {
      const double den = vel_den(h, eps4);
      U = qdiv(vel_num(hu, h), den); V = qdiv(vel_num(hv, h), den);
    }
    sm.U[ly][c] = U; sm.V[ly][c] = V;
  }
  __syncthreads();

  // slopes (src/swe.mjs:364-411): each thread its own cell in x and y; the
  // east column's x slopes (the first SPY threads) and the north row's y
  // slopes (the second warp) besides
  const int lx = t % SPX, ly = t / SPX;
  const int gi = i0 + lx, gj = j0 + ly;
  constexpr int XS = SPY * (SPX + 1), YS = (SPY + 1) * SPX;   // strides of xs[q], ys[q]
  {
    const bool on = order2 && gj >= 1 && gj < H - 1 && gi >= 1 && gi < W - 1;
    const int cy = ly + 1, cx = lx + 1 + TCOL;
    tile_slopes<1, LIM>(sm, a.lim, dry, on, cy, cx, &sm.xs[0][ly][lx], XS);
    tile_slopes<0, LIM>(sm, a.lim, dry, on, cy, cx, &sm.ys[0][ly][lx], YS);
  }
  if (t < SPY) {                                // x slopes of column i0 + SPX, row j0 + t
    const int ei = i0 + SPX, ej = j0 + t;
    const bool on = order2 && ej >= 1 && ej < H - 1 && ei >= 1 && ei < W - 1;
    tile_slopes<1, LIM>(sm, a.lim, dry, on, t + 1, SPX + 1 + TCOL, &sm.xs[0][t][SPX], XS);
  } else if (t >= 32 && t < 32 + SPX) {         // y slopes of row j0 + SPY, column i0 + t - 32
    const int c = t - 32, ni = i0 + c, nj = j0 + SPY;
    const bool on = order2 && nj >= 1 && nj < H - 1 && ni >= 1 && ni < W - 1;
    tile_slopes<0, LIM>(sm, a.lim, dry, on, SPY + 1, c + 1 + TCOL, &sm.ys[0][SPY][c], YS);
  }
  __syncthreads();

  if (gi < W && gj < H) split_faces_cell(a, s, sm, lx, ly, gi, gj, sph, bedOn);
  __syncthreads();
}

__device__ __forceinline__ void split_faces_finish(const StageArgs& a, const SplitBufs& s, int tx, int ty,
                                                   FacesSmem& sm, int t) {
  if (a.lim == 0) split_faces_finish_l<0>(a, s, tx, ty, sm, t);    // mc, the default
  else split_faces_finish_l<-1>(a, s, tx, ty, sm, t);
}

// ---- the state tile by tensor-map copies (TMA) --------------------------------
// One thread issues four 2-D bulk tensor copies (b, h, hu, hv of the stage
// input) of the box SSXT x SSY at column i0 - 2 (even, so its first element
// sits on a 16-byte boundary of the row) and row j0 - 1; the copies fill
// cells outside the grid with zeros, which is what the tile needs there, and
// complete on an mbarrier the whole CTA waits on.  That replaces the 1540
// per-element copies and their address arithmetic.  The maps cover this
// simulation's own device buffers only (no multicast).  Grids whose padded
// width is odd (a row stride that is not a multiple of 16 bytes) take the
// per-element path; both give the same bits.
struct TileMaps { CUtensorMap m[4]; };
constexpr unsigned TILE_TX_BYTES = 4u * SSY * SSXT * sizeof(double);

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
               "selp.u32 %0, 1, 0, p;\n}\n"
               : "=r"(ok)
               : "r"(smem_addr(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load_tile(void* dst, const CUtensorMap* map, int x, int y,
                                              unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
      ::"r"(smem_addr(dst)), "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}
// Every thread: until the phase `parity` of bar completes, at most `tries`
// polls (each of which may suspend the thread for a while).
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, int tries) {
  for (int it = 0; it < tries; it++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
constexpr int TMA_WAIT_TRIES = 1 << 22;

// split_faces_tile with the state tile fetched by tensor-map copies.  bar
// is an initialised mbarrier in shared memory and parity its phase, flipped
// here for the next tile.  A copy that does not complete within the bound
// sets bit 4 of Control::status and leaves the tile's faces unwritten.
__device__ __forceinline__ void split_faces_tile_tma(const StageArgs& a, const SplitBufs& s, int tx, int ty,
                                                     FacesSmem& sm, const TileMaps& maps,
                                                     unsigned long long* bar, unsigned& parity, Control* ctl,
                                                     bool check_settled = true) {
  const int t = threadIdx.x;
  if (check_settled && split_faces_settled(s, tx, ty, t)) return;
  if (t == 0) {
    // the generic-proxy accesses of a previous tile come before the copy's writes
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    mbar_expect_tx(bar, TILE_TX_BYTES);
    const int x = tx * SPX - 2, y = ty * SPY - 1;
    tma_load_tile(&sm.b[0][0], &maps.m[0], x, y, bar);
    tma_load_tile(&sm.h[0][0], &maps.m[1], x, y, bar);
    tma_load_tile(&sm.U[0][0], &maps.m[2], x, y, bar);
    tma_load_tile(&sm.V[0][0], &maps.m[3], x, y, bar);
  }
  const bool ok = mbar_wait_bounded(bar, parity, TMA_WAIT_TRIES);
  parity ^= 1u;
  if (!__syncthreads_and(ok)) {                     // uniform: give up on the tile
    if (t == 0) atomicOr(&ctl->status, 4);
    mbar_wait_bounded(bar, parity ^ 1u, TMA_WAIT_TRIES);   // let a late copy land first
    __syncthreads();
    return;
  }
  split_faces_finish(a, s, tx, ty, sm, t);
}

// CTAs per SM of the face kernels.  The tensor-map kernel of the stepping
// loop at 5 (48 registers, 168 / 216 bytes of spills) measured +1.8% on the
// beach over 4 (64 registers) and the same all-wet; 6 (40 registers) +1.2%.
// The per-element kernel, which the adjoint's passes use (they also write
// the slopes and velocities to the tape), stays at 4: at 5 its gradient cost
// 2% more against an unchanged forward.
#ifndef SWE_SPLIT_FACES_MIN_BLOCKS
#define SWE_SPLIT_FACES_MIN_BLOCKS 5
#endif
#ifndef SWE_SPLIT_FACES_PLAIN_MIN_BLOCKS
#define SWE_SPLIT_FACES_PLAIN_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(SP_THREADS, SWE_SPLIT_FACES_PLAIN_MIN_BLOCKS)
k_split_faces(StageArgs a, SplitBufs s, Control* ctl) {
  pdl_enter();
  if (ctl->stop) return;
  __shared__ FacesSmem sm;
  split_faces_tile(a, s, blockIdx.x, blockIdx.y, sm);
}

// The face kernel with its state tile fetched by tensor-map copies.
__global__ void __launch_bounds__(SP_THREADS, SWE_SPLIT_FACES_MIN_BLOCKS)
k_split_faces_tma(StageArgs a, SplitBufs s, Control* ctl, const __grid_constant__ TileMaps maps) {
  __shared__ FacesSmem sm;
  __shared__ alignas(8) unsigned long long bar;
  if (threadIdx.x == 0) mbar_init(&bar, 1);        // before the wait: touches no global memory
  pdl_enter();
  if (ctl->stop) return;
  __syncthreads();
  unsigned parity = 0;
  split_faces_tile_tma(a, s, blockIdx.x, blockIdx.y, sm, maps, &bar, parity, ctl);
}

// ---- the face kernel over a list of the tiles it must compute ----------------
// On wet/dry grids most tiles settle: their 3 x 3 neighbourhood is recorded
// dry, and the face kernel only writes their dry flag.  A CTA per tile then
// spends much of the launch on CTAs that read nine flags and exit.
// k_face_list does that test for every tile (one thread each), writes the
// dry flag of the settled ones itself, and appends the others to a list
// that the face kernel's first CTAs take.  The list's order depends on
// timing, the results do not: every tile writes
// only its own faces, terms and flag.  count is this stage's counter (the
// list kernel of the other stage zeroes it again, after its face kernel
// has run).
//
// The same kernel lists the tiles the cell kernel must run when some may be
// left out (cell_skip: the settling cell kernel is in use and nothing it
// takes rules settling out; otherwise the cell kernel runs every tile).
// The cell kernel settles a ghost-free tile whose 3 x 3 dry flags are set
// (its faces are all +0), and writes nothing but +0 and 0 partials when the
// tile's output record already says (+0, +0, +0): record 2.  Those partial
// slots hold +0 and 0 since that record was written, so the tile can be
// left out altogether when every tile of its 3 x 3 neighbourhood settles in
// the face kernel (their dry flags are then set here) and its own output
// record is 2.  The count of settled tiles (one in 16) that the cell kernel
// keeps is kept here for the tiles left out.
// The warp-aggregated append of `on` lanes to list (a block base from one
// atomic on count); every thread of the block calls it.
__device__ __forceinline__ void block_append(bool on, int value, int* list, int* count, int cap, int* wbase,
                                             int* base) {
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  const unsigned m = __ballot_sync(0xffffffffu, on);
  if (lane == 0) wbase[w] = __popc(m);
  __syncthreads();
  if (t == 0) {
    int n = 0;
    for (int q = 0; q < (int)blockDim.x / 32; q++) { const int c = wbase[q]; wbase[q] = n; n += c; }
    *base = n ? atomicAdd(count, n) : 0;
  }
  __syncthreads();
  if (on) {
    const int at = *base + wbase[w] + __popc(m & ((1u << lane) - 1));
    if (at < cap) list[at] = value;              // always, while each stage's counter is reset in turn
  }
  __syncthreads();
}
// One CTA per 32 x 8 region of tiles: the records of the region and two
// tiles around it go to shared memory in one coalesced pass, the settled
// test of the region and one tile around it is made there, and each thread
// then decides for its own tile.
constexpr int LX = 32, LY = 8;                     // tiles per list CTA
struct TileLists {
  int* list; int* count; int* other_count;         // the face kernel's
  int cell_skip;
  int* clist; int* ccount; int* other_ccount;      // the cell kernel's
  int W, H;
};
// The lists of the region (rx, ry) of tiles; every thread of the CTA calls it.
__device__ __forceinline__ void face_list_region(const SplitBufs& s, Control* ctl, const TileLists& L, int rx,
                                                 int ry) {
  __shared__ unsigned char rec[LY + 4][LX + 4];      // record dry (or outside the grid)
  __shared__ unsigned char fs[LY + 2][LX + 2];       // settles in the face kernel
  __shared__ int wbase[LX * LY / 32], base;
  int* const list = L.list; int* const count = L.count; int* const clist = L.clist; int* const ccount = L.ccount;
  const int cell_skip = L.cell_skip, W = L.W, H = L.H;
  const int t = threadIdx.x, ntx = s.ntx, nty = s.nty, ntiles = ntx * nty;
  const int bx = rx * LX, by = ry * LY;
  for (int q = t; q < (LY + 4) * (LX + 4); q += LX * LY) {
    const int ly = q / (LX + 4), lx = q - ly * (LX + 4), gx = bx - 2 + lx, gy = by - 2 + ly;
    rec[ly][lx] = (gx < 0 || gx >= ntx || gy < 0 || gy >= nty || s.odry_in[gy * ntx + gx] != 0) ? 1 : 0;
  }
  __syncthreads();
  for (int q = t; q < (LY + 2) * (LX + 2); q += LX * LY) {
    const int fy = q / (LX + 2), fx = q - fy * (LX + 2);
    unsigned char d = 1;
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) d &= rec[fy + r][fx + c];
    fs[fy][fx] = d;
  }
  __syncthreads();
  const int lx = t % LX, ly = t / LX, tx = bx + lx, ty = by + ly;
  bool faces = false, cells = false;
  if (tx < ntx && ty < nty) {
    const int tile = ty * ntx + tx;
    const bool settled = fs[ly + 1][lx + 1] != 0;
    if (settled) s.dry[tile] = 1;
    faces = !settled;
    cells = true;
    const double dt = ctl->dt;
    const int i0 = tx * SPX, j0 = ty * SPY;
    if (cell_skip && settled && dt > 0 && dt < INFINITY && i0 >= 2 && i0 + SPX <= W - 2 && j0 >= 2 &&
        j0 + SPY <= H - 2 && s.odry_out[tile] == 2) {
      unsigned char all = 1;
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) all &= fs[ly + r][lx + c];
      if (all) {
        cells = false;
        if ((tile & 15) == 0) atomicAdd(&ctl->settled_next, 1);
      }
    }
  }
  if (rx == 0 && ry == 0 && t == 0) { *L.other_count = 0; *L.other_ccount = 0; }
  const int tile = ty * ntx + tx;
  block_append(faces, tile, list, count, ntiles, wbase, &base);
  if (cell_skip) block_append(cells, tile, clist, ccount, ntiles, wbase, &base);   // uniform
}
__global__ void __launch_bounds__(LX * LY) k_face_list(SplitBufs s, Control* ctl, TileLists L) {
  pdl_enter();
  face_list_region(s, ctl, L, blockIdx.x, blockIdx.y);
}
// The ghost fill of the stage's input (its first nbc blocks, as k_apply_bc)
// and the stage's lists (the other blocks, one per region of nrx columns of
// regions) in one launch: the lists read only the records, the fill only
// the state.
__global__ void __launch_bounds__(LX * LY) k_bc_face_list(BCArgs b, int respect_stop, int nbc, SplitBufs s,
                                                          Control* ctl, TileLists L, int nrx) {
  pdl_enter();
  if ((int)blockIdx.x < nbc) {                     // uniform per block
    if (respect_stop && ctl->stop) return;
    apply_bc_range(b, ctl, blockIdx.x * blockDim.x + threadIdx.x, nbc * blockDim.x);
    return;
  }
  const int r = blockIdx.x - nbc;
  face_list_region(s, ctl, L, r % nrx, r / nrx);
}

// The face kernel over the list: CTA b computes the list's entry b, and the
// CTAs past the list's length exit after reading it.
__global__ void __launch_bounds__(SP_THREADS, SWE_SPLIT_FACES_MIN_BLOCKS)
k_split_faces_tma_list(StageArgs a, SplitBufs s, Control* ctl, const __grid_constant__ TileMaps maps,
                       const int* list, const int* count) {
  __shared__ FacesSmem sm;
  __shared__ alignas(8) unsigned long long bar;
  pdl_enter();
  if ((int)blockIdx.x >= min(*count, s.ntx * s.nty) || ctl->stop) return;
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  const int tile = list[blockIdx.x];
  unsigned parity = 0;
  split_faces_tile_tma(a, s, tile % s.ntx, tile / s.ntx, sm, maps, &bar, parity, ctl, false);
}

struct CellsSmem {
  double st[6][SP_THREADS];       // each thread's own cell: h, hu, hv, then U0 (stage 2)
  double th[SPY + 2][SPX + 2];
  double red[2][SP_THREADS / 32];
  int dry[3][3];                  // dry flags of the tile's 3 x 3 neighbourhood
  int prev;                       // the output tile's record as this kernel left it last time
  bool last;
};

// The cell kernel's inputs from the face kernel, staged by tensor-map copies
// for the tile at (i0, j0) (TMA variant): the mass fluxes of every face the
// limiter ring and the gather touch, the other face values of the gather and
// the depths of the ring, and the tile's source terms.  x = i0 - 2 (even)
// for every box but yt's and tb's (x = i0); cells outside the grid read as
// zeros, which the dry flags replace in any case.
struct CellFaceTiles {
  alignas(128) double xm[SPY + 2][SPX + 4];      // fx M, rows j0-1.., columns i0-2..
  alignas(128) double ym[SPY + 3][SPX + 4];      // fy M, rows j0-2.., columns i0-2..
  alignas(128) double hr[SPY + 2][SPX + 4];      // h of the stage input, rows j0-1.., columns i0-2..
  alignas(128) double xt[3][SPY][SPX + 2];       // fx T, N + pL, N + pR, rows j0.., columns i0-2..
  alignas(128) double yt[3][SPY + 1][SPX];       // fy T, N + pL, N + pR, rows j0-1.., columns i0..
  alignas(128) double tb[3][SPY][SPX];           // the tile's bed terms x, y and geometric source
};
enum { CM_XM, CM_YM, CM_H, CM_XT, CM_YT = CM_XT + 3, CM_TB = CM_YT + 3, CM_COUNT = CM_TB + 3 };
struct CellMaps { CUtensorMap m[CM_COUNT]; };
constexpr unsigned CELL_TX_BYTES = sizeof(double) * (unsigned)((SPY + 2) * (SPX + 4) + (SPY + 3) * (SPX + 4) +
                                                               (SPY + 2) * (SPX + 4) + 3 * SPY * (SPX + 2) +
                                                               3 * (SPY + 1) * SPX + 3 * SPY * SPX);

// A face / source-term value owned by cell (gi, gj) of the 3 x 3 tile
// neighbourhood of the tile at (i0, j0): +0 when its tile was dry.
__device__ __forceinline__ double split_load(const CellsSmem& sm, int i0, int j0, int gi, int gj,
                                             const double* arr, int k) {
  const int c = gi < i0 ? 0 : (gi >= i0 + SPX ? 2 : 1);
  const int r = gj < j0 ? 0 : (gj >= j0 + SPY ? 2 : 1);
  return sm.dry[r][c] ? 0.0 : arr[k];
}

// Positivity limiter of cell (gi, gj) from its four faces' mass fluxes
// (src/swe.mjs:511-529), with the same conservative pre-test as stage_tile.
__device__ __forceinline__ double split_theta(const StageArgs& a, const SplitBufs& s, const CellsSmem& sm,
                                              int i0, int j0, double dt, int gi, int gj) {
  const int W = a.W, H = a.H;
  if (!(dt > 0 && gj >= 1 && gj < H - 1 && gi >= 1 && gi < W - 1)) return 1;
  const int k = gj * W + gi;
  const double fxE = split_load(sm, i0, j0, gi, gj, s.fx[F_M], k);
  const double fxW = split_load(sm, i0, j0, gi - 1, gj, s.fx[F_M], k - 1);
  const double fyN = split_load(sm, i0, j0, gi, gj, s.fy[F_M], k);
  const double fyS = split_load(sm, i0, j0, gi, gj - 1, s.fy[F_M], k - W);
  const double avail = a.h[k];
  const double est = ((fxE > 0 ? fxE : 0) - (fxW < 0 ? fxW : 0)) * a.m.rdxRow[gj]
                   + (fyN > 0 ? fyN : 0) * a.m.rdyRowN[gj] - (fyS < 0 ? fyS : 0) * a.m.rdyRowS[gj];
  double th = 1;
  if (!(est * dt * (1 + 1e-12) < avail)) {
    double out = 0;
    if (fxE > 0) out += fxE / a.m.dxRow[gj];
    if (fxW < 0) out -= fxW / a.m.dxRow[gj];
    if (fyN > 0) out += fyN / a.m.dyRowN[gj];
    if (fyS < 0) out -= fyS / a.m.dyRowS[gj];
    if (out * dt > avail) th = avail > 0 ? avail / (out * dt) : 0;
  }
  return th;
}

// split_theta from the staged tiles: the same values, read from shared
// memory (+0 where split_load gives +0).
__device__ __forceinline__ bool split_dry_at(const CellsSmem& sm, int i0, int j0, int gi, int gj) {
  const int c = gi < i0 ? 0 : (gi >= i0 + SPX ? 2 : 1);
  const int r = gj < j0 ? 0 : (gj >= j0 + SPY ? 2 : 1);
  return sm.dry[r][c] != 0;
}
__device__ __forceinline__ double split_theta_st(const StageArgs& a, const CellFaceTiles& ft, const CellsSmem& sm,
                                                 int i0, int j0, double dt, int gi, int gj) {
  const int W = a.W, H = a.H;
  if (!(dt > 0 && gj >= 1 && gj < H - 1 && gi >= 1 && gi < W - 1)) return 1;
  const int cx = gi - i0 + 2, rx = gj - j0 + 1, ry = gj - j0 + 2;
  const double fxE = split_dry_at(sm, i0, j0, gi, gj) ? 0.0 : ft.xm[rx][cx];
  const double fxW = split_dry_at(sm, i0, j0, gi - 1, gj) ? 0.0 : ft.xm[rx][cx - 1];
  const double fyN = split_dry_at(sm, i0, j0, gi, gj) ? 0.0 : ft.ym[ry][cx];
  const double fyS = split_dry_at(sm, i0, j0, gi, gj - 1) ? 0.0 : ft.ym[ry - 1][cx];
  const double avail = ft.hr[rx][cx];
  const double est = ((fxE > 0 ? fxE : 0) - (fxW < 0 ? fxW : 0)) * a.m.rdxRow[gj]
                   + (fyN > 0 ? fyN : 0) * a.m.rdyRowN[gj] - (fyS < 0 ? fyS : 0) * a.m.rdyRowS[gj];
  double th = 1;
  if (!(est * dt * (1 + 1e-12) < avail)) {
    double out = 0;
    if (fxE > 0) out += fxE / a.m.dxRow[gj];
    if (fxW < 0) out -= fxW / a.m.dxRow[gj];
    if (fyN > 0) out += fyN / a.m.dyRowN[gj];
    if (fyS < 0) out -= fyS / a.m.dyRowS[gj];
    if (out * dt > avail) th = avail > 0 ? avail / (out * dt) : 0;
  }
  return th;
}

// The close of a stage by one block: the partials of its `nparts` tiles
// reduced in a fixed order (strided per thread, then a fixed tree), so the
// sums are the same in every run.
template <int MODE>
__device__ __forceinline__ void split_close_block(const StageArgs& a, Control* ctl, int nparts, CellsSmem& sm) {
  const int t = threadIdx.x;
  const double dt = ctl->dt;
  double m = 0, f = 0;
  // The partials are read at L2 (__ldcg: another CTA of the same launch may
  // have written them, and L1 is not coherent), CLOSE_BATCH loads in flight
  // per thread; each thread still adds its slots q = t, t + 256, ... in
  // increasing order.
  constexpr int CLOSE_BATCH = 8;
  const double* pf = MODE == 1 ? a.part_fl1 : a.part_fl2;
  int q = t;
  for (; q + (CLOSE_BATCH - 1) * SP_THREADS < nparts; q += CLOSE_BATCH * SP_THREADS) {
    double vf[CLOSE_BATCH], vm[CLOSE_BATCH];
#pragma unroll
    for (int u = 0; u < CLOSE_BATCH; u++) {
      vf[u] = __ldcg(pf + q + u * SP_THREADS);
      if (MODE == 2) vm[u] = __ldcg(a.part_max + q + u * SP_THREADS);
    }
#pragma unroll
    for (int u = 0; u < CLOSE_BATCH; u++) {
      if (MODE == 2) m = fmax(m, vm[u]);
      f += vf[u];
    }
  }
  for (; q < nparts; q += SP_THREADS) {
    if (MODE == 2) m = fmax(m, __ldcg(a.part_max + q));
    f += __ldcg(pf + q);
  }
  for (int o = 16; o > 0; o >>= 1) {
    m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    f += __shfl_down_sync(0xffffffffu, f, o);
  }
  __syncthreads();
  if ((t & 31) == 0) { sm.red[0][t >> 5] = m; sm.red[1][t >> 5] = f; }
  __syncthreads();
  if (t == 0) {
    m = sm.red[0][0]; f = sm.red[1][0];
    for (int w = 1; w < SP_THREADS / 32; w++) { m = fmax(m, sm.red[0][w]); f += sm.red[1][w]; }
    if (MODE == 1) {
      ctl->floored1 = f;
    } else {
      ctl->next_max = m;
      ctl->mass_floored = ctl->floored1 + f;
      ctl->t = ctl->t + dt;
      ctl->steps = ctl->steps + 1;
    }
    ctl->counter = 0;
  }
}

// One cell's gather, source terms, update and epilogue, adding to the
// tile's partials.  DRY: the tile's 3 x 3 neighbourhood is flagged dry, so
// every face the cell reads is +0 and theta is 1.  With finite reciprocal
// metrics (StageArgs::dryfold) each face term is then +0 * (finite) = +-0
// added to or taken from a +0 sum, and the bed terms are +0, so the sums
// are +0 with or without them: DRY leaves them out and gives the same bits.
// ST: the face values come from the staged tiles ft.
template <int MODE, bool DRY, bool ST = false>
__device__ __forceinline__ void split_cell(const StageArgs& a, const SplitBufs& s, const CellsSmem& sm, int t,
                                           int lx, int ly, int gi, int gj, double dt, double& locMax,
                                           double& locFl, double& hout, const CellFaceTiles* ft = nullptr) {
  const int W = a.W, H = a.H;
  const double dry = a.minDepth, eps4 = a.eps4;
  const bool sph = a.sph != 0;
  const bool bedOn = a.order >= 2 || sph;
  const bool corOn = sph || (a.coriolis != 0 && a.coriolis == a.coriolis);
  const int k = gj * W + gi;
  // every load of the cell first, so they are in flight together
  const bool rowX = gj >= 2 && gj < H - 2, colY = gi >= 2 && gi < W - 2;
  const bool hasW = rowX && gi - 1 >= 1 && gi - 1 < W - 2, hasE = rowX && gi >= 1 && gi < W - 2;
  const bool hasS = colY && gj - 1 >= 1 && gj - 1 < H - 2, hasN = colY && gj >= 1 && gj < H - 2;
  const bool interior = colY && rowX;
  double wM = 0, wT = 0, wN = 0, eM = 0, eT = 0, eN = 0, sM = 0, sT = 0, sN = 0, nM = 0, nT = 0, nN = 0;
  const bool dW = sm.dry[1][lx == 0 ? 0 : 1], dS = sm.dry[ly == 0 ? 0 : 1][1], dC = sm.dry[1][1];
  if (ST) {
    if (!DRY && hasW && !dW) { wM = ft->xm[ly + 1][lx + 1]; wT = ft->xt[0][ly][lx + 1]; wN = ft->xt[2][ly][lx + 1]; }
    if (!DRY && hasE && !dC) { eM = ft->xm[ly + 1][lx + 2]; eT = ft->xt[0][ly][lx + 2]; eN = ft->xt[1][ly][lx + 2]; }
    if (!DRY && hasS && !dS) { sM = ft->ym[ly + 1][lx + 2]; sT = ft->yt[0][ly][lx]; sN = ft->yt[2][ly][lx]; }
    if (!DRY && hasN && !dC) { nM = ft->ym[ly + 2][lx + 2]; nT = ft->yt[0][ly + 1][lx]; nN = ft->yt[1][ly + 1][lx]; }
  } else {
    if (!DRY && hasW && !dW) { wM = s.fx[F_M][k - 1]; wT = s.fx[F_T][k - 1]; wN = s.fx[F_NPR][k - 1]; }
    if (!DRY && hasE && !dC) { eM = s.fx[F_M][k]; eT = s.fx[F_T][k]; eN = s.fx[F_NPL][k]; }
    if (!DRY && hasS && !dS) { sM = s.fy[F_M][k - W]; sT = s.fy[F_T][k - W]; sN = s.fy[F_NPR][k - W]; }
    if (!DRY && hasN && !dC) { nM = s.fy[F_M][k]; nT = s.fy[F_T][k]; nN = s.fy[F_NPL][k]; }
  }
  cp_async_wait_all();
  const double hin = sm.st[0][t], huin = sm.st[1][t], hvin = sm.st[2][t];
  double tb0 = 0, tb1 = 0, tg = 0, Uk = 0;
  if (!DRY && interior && bedOn && !dC) {
    if (ST) { tb0 = ft->tb[0][ly][lx]; tb1 = ft->tb[1][ly][lx]; if (sph) tg = ft->tb[2][ly][lx]; }
    else { tb0 = s.tb[0][k]; tb1 = s.tb[1][k]; if (sph) tg = s.tb[2][k]; }
  }
  if (interior && sph) {
    if (!DRY && !dC) Uk = s.U[k];
    else Uk = vel_num(huin, hin);               // h is 0 here: the face kernel's u
  }
  double U0h = 0, U0hu = 0, U0hv = 0;
  if (MODE == 2) { U0h = sm.st[3][t]; U0hu = sm.st[4][t]; U0hv = sm.st[5][t]; }
  const double thC = DRY ? 1.0 : sm.th[ly + 1][lx + 1];
  const double rdx = a.m.rdxRow[gj], dxr = a.m.dxRow[gj];
  double ah = 0, ahu = 0, ahv = 0;
  if (!DRY && hasW) {                                       // west face, cell is its right side
    const double thf = wM >= 0 ? sm.th[ly + 1][lx] : thC;
    const double inv = thf == 1 ? rdx : thf / dxr;
    ah += wM * inv; ahu += wN * inv; ahv += wT * inv;
  }
  if (!DRY && hasE) {                                       // east face, cell is its left side
    const double thf = eM >= 0 ? thC : sm.th[ly + 1][lx + 2];
    const double inv = thf == 1 ? rdx : thf / dxr;
    ah -= eM * inv; ahu -= eN * inv; ahv -= eT * inv;
  }
  if (!DRY && hasS) {                                       // south face, cell is its upper side
    const double thf = sM >= 0 ? sm.th[ly][lx + 1] : thC;
    const double invR = thf == 1 ? a.m.rdyRowS[gj] : thf / a.m.dyRowS[gj];
    ah += sM * invR; ahv += sN * invR; ahu += sT * invR;
  }
  if (!DRY && hasN) {                                       // north face, cell is its lower side
    const double thf = nM >= 0 ? thC : sm.th[ly + 2][lx + 1];
    const double invL = thf == 1 ? a.m.rdyRowN[gj] : thf / a.m.dyRowN[gj];
    ah -= nM * invL; ahv -= nN * invL; ahu -= nT * invL;
  }
  if (interior) {
    if (!DRY && bedOn) {
      ahu += tb0;
      ahv += tb1;
      if (sph) ahv += tg;
    }
    if (sph) {
      const double fe = a.m.fRow[gj] + Uk * (a.m.tanPhi[gj] / a.m.R);
      ahu += fe * hvin;
      ahv -= fe * huin;
    } else if (corOn) {
      ahu += a.coriolis * hvin;
      ahv -= a.coriolis * huin;
    }
  }
  if (a.tape_th) a.tape_th[k] = thC;
  if (MODE == 1) {
    double nh = hin + dt * ah, nhu = huin + dt * ahu, nhv = hvin + dt * ahv;
    if (a.tape_hpre) a.tape_hpre[k] = nh;
    if (interior) {                                 // dryClean, src/swe.mjs:734-745
      if (nh < 0) { locFl -= nh; nh = 0; }
      if (nh <= dry) { nhu = 0; nhv = 0; }
    }
    hout = nh;
    a.oh[k] = nh; a.ohu[k] = nhu; a.ohv[k] = nhv;
  } else {
    const double h0 = U0h, hu0 = U0hu, hv0 = U0hv;   // U0 (in place)
    if (a.h0c) { a.h0c[k] = h0; a.hu0c[k] = hu0; a.hv0c[k] = hv0; }
    double nh = 0.5 * (h0 + hin + dt * ah);
    double nhu = 0.5 * (hu0 + huin + dt * ahu);
    double nhv = 0.5 * (hv0 + hvin + dt * ahv);
    if (a.tape_hpre) a.tape_hpre[k] = nh;
    if (interior) {
      if (nh < 0) { locFl -= nh; nh = 0; }
      if (nh <= dry) { nhu = 0; nhv = 0; }
      if (a.tape_pre[0]) { a.tape_pre[0][k] = nh; a.tape_pre[1][k] = nhu; a.tape_pre[2][k] = nhv; }
      // friction, src/swe.mjs:659-704
      const double n = a.nfield ? a.nfield[k] : a.manning;
      const bool fricOn = a.nfield ? true : (n != 0 && n == n);
      if (fricOn) {
        if (nh <= dry) { nhu = 0; nhv = 0; }
        else if (n != 0 && n == n) {
          const double den = vel_den(nh, eps4);
          const double u = qdiv(vel_num(nhu, nh), den), v = qdiv(vel_num(nhv, nh), den);
          const double speed = hypot(u, v);
          if (!(speed < 1e-14)) {
            const double denom = 1 + dt * SWE_G * n * n * speed / pow43(nh);
            nhu = qdiv(nhu, denom);
            nhv = qdiv(nhv, denom);
          }
        }
      }
      // sponge, src/swe.mjs:1188-1197
      if (a.sponge_width > 0) {
        const int ii = gi - 2, jj = gj - 2;
        int d;
        if (a.sponge_side == 1) d = a.nx - 1 - ii; else if (a.sponge_side == 0) d = ii;
        else if (a.sponge_side == 3) d = a.ny - 1 - jj; else d = jj;
        if (d < a.sponge_width) {
          const double f = jmin(1, a.sponge_str[d] * dt * 60);
          const double target = jmax0(a.sponge_ref - __ldg(a.b + k));
          nh = nh + (target - nh) * f;
          nhu = nhu - nhu * f;
          nhv = nhv - nhv * f;
        }
      }
      // CFL rate of the final state, src/swe.mjs:632-647
      if (!(nh <= dry)) {
        const double cc = sqrt(SWE_G * nh);
        const double den = vel_den(nh, eps4);
        const double u = fabs(qdiv(vel_num(nhu, nh), den)), v = fabs(qdiv(vel_num(nhv, nh), den));
        const double sr5 = (u + cc) / dxr + (v + cc) / a.m.dyCFL[gj];
        if (sr5 > locMax) locMax = sr5;
      }
    }
    hout = nh;
    a.oh[k] = nh; a.ohu[k] = nhu; a.ohv[k] = nhv;
  }
}

// Limiter, gather, update and epilogue of the tile (tx, ty), which holds
// partial slot `part` of the `nparts` of its grid.  With `ticket`, the last
// tile of the grid to finish closes the step; without, the step is closed
// by k_split_close after the launch.  Every thread of the CTA calls it.
// SETTLE: tiles may settle (below); without it the function is the plain
// tile update, which grids with little dry land run faster.
// TMA: the limiter ring's and the gather's inputs are staged into ft by
// tensor-map copies (maps, completing on bar) once the tile is known to be
// computed; a copy that does not complete within the bound sets bit 4 of
// Control::status and leaves the tile's output unwritten.
template <int MODE, bool SETTLE = false, bool TMA = false>
__device__ __forceinline__ void split_cells_tile(const StageArgs& a, const SplitBufs& s, Control* ctl, int tx,
                                                 int ty, int part, int nparts, CellsSmem& sm, bool ticket,
                                                 CellFaceTiles* ft = nullptr, const CellMaps* maps = nullptr,
                                                 unsigned long long* bar = nullptr) {
  static_assert(MODE == 1 || MODE == 2, "stages only");
  const int W = a.W, H = a.H;
  const int i0 = tx * SPX, j0 = ty * SPY;
  const int t = threadIdx.x;
  const double dt = ctl->dt;
  const int lx = t % SPX, ly = t / SPX;
  const int gi = i0 + lx, gj = j0 + ly;

  // Whether the tile could settle (below), from what is known without a
  // load.  When a quarter or more of the tiles settled in each stage of the
  // last step (Control::settled counts one in 16, both stages), such a tile
  // copies its state only once the flags say that it must be computed, so
  // a settled tile reads nothing; otherwise every tile copies its state at
  // once, in flight with the flags.
  const bool canSettle = SETTLE && !ticket && s.odry_out && s.dry && a.dryfold && a.minDepth >= 0 && a.sponge_width <= 0 &&
                         !a.h0c && !a.tape_th && !a.tape_hpre && !a.tape_pre[0] &&
                         i0 >= 2 && i0 + SPX <= W - 2 && j0 >= 2 && j0 + SPY <= H - 2;
  const bool defer = canSettle && 32 * ctl->settled >= nparts;   // uniform across the grid
  if (!defer && gi < W && gj < H) {
    const int k = gj * W + gi;
    cp_async8(&sm.st[0][t], a.h + k);
    cp_async8(&sm.st[1][t], a.hu + k);
    cp_async8(&sm.st[2][t], a.hv + k);
    if (MODE == 2) {
      cp_async8(&sm.st[3][t], a.oh + k);
      cp_async8(&sm.st[4][t], a.ohu + k);
      cp_async8(&sm.st[5][t], a.ohv + k);
    }
  }
  if (t < 9) {
    const int r = t / 3, c = t - 3 * r, txn = tx - 1 + c, tyn = ty - 1 + r;
    int f = 0;                                    // no flags: nothing is skipped
    if (s.dry) {
      f = 1;                                      // outside the grid: no faces there
      if (txn >= 0 && txn < s.ntx && tyn >= 0 && tyn < s.nty) f = s.dry[tyn * s.ntx + txn];
    }
    sm.dry[r][c] = f;
  }
  __syncthreads();
  const bool allDry = sm.dry[0][0] & sm.dry[0][1] & sm.dry[0][2] & sm.dry[1][0] & sm.dry[1][1] &
                      sm.dry[1][2] & sm.dry[2][0] & sm.dry[2][1] & sm.dry[2][2];
  const bool fold = allDry && a.dryfold;          // uniform across the CTA
  // A folded tile settles without its state.  Its input has h = +-0 on the
  // tile (the flags), and so does U0 in stage 2 (the output record, which
  // describes U0 as this kernel wrote it in the previous step).  Every face
  // and source term is +0 (the fold), so stage 1 gives h = +-0 + dt * (+0)
  // and stage 2 h = 0.5 ((+-0 + +-0) + dt * (+0)): both +0 for dt > 0.
  // dryClean then sets hu = hv = +0 (h <= minDepth when minDepth >= 0), as
  // does friction; with no sponge nothing else writes the cell, the CFL
  // rate and the floored mass get nothing, and h = +0 never floors.  All
  // cells are interior (ghost-free tile).  So the tile's output is exactly
  // (+0, +0, +0), and when the record says the tile already holds that (2)
  // nothing is written at all.  The tape and the U0 copy need the values:
  // not with them.
  if (canSettle && fold && dt > 0 && dt < INFINITY) {   // uniform; only folded tiles read the record
    if (t == 0) sm.prev = s.odry_out[ty * s.ntx + tx];
    __syncthreads();
    if (MODE == 1 || sm.prev >= 1) {
      if (!defer) cp_async_wait_all();            // the copies of U0 read what is written next
      if (sm.prev != 2 && gi < W && gj < H) {
        const int k = gj * W + gi;
        a.oh[k] = 0.0; a.ohu[k] = 0.0; a.ohv[k] = 0.0;
      }
      if (t == 0) {                               // no cell contributes: +0 and 0 (the reduction's result)
        s.odry_out[ty * s.ntx + tx] = 2;
        if (MODE == 1) a.part_fl1[part] = 0;
        else { a.part_max[part] = 0; a.part_fl2[part] = 0; }
        if ((part & 15) == 0) atomicAdd(&ctl->settled_next, 1);
      }
      return;                                     // canSettle excludes the ticket
    }
  }
  // the cell's own state, in flight while the limiter is worked out
  if (defer && gi < W && gj < H) {
    const int k = gj * W + gi;
    cp_async8(&sm.st[0][t], a.h + k);
    cp_async8(&sm.st[1][t], a.hu + k);
    cp_async8(&sm.st[2][t], a.hv + k);
    if (MODE == 2) {
      cp_async8(&sm.st[3][t], a.oh + k);
      cp_async8(&sm.st[4][t], a.ohu + k);
      cp_async8(&sm.st[5][t], a.ohv + k);
    }
  }
  if (TMA && !fold) {
    if (t == 0) {
      // the generic-proxy accesses of the shared memory come before the copies' writes
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      mbar_expect_tx(bar, CELL_TX_BYTES);
      const int x = i0 - 2;
      tma_load_tile(&ft->xm[0][0], &maps->m[CM_XM], x, j0 - 1, bar);
      tma_load_tile(&ft->ym[0][0], &maps->m[CM_YM], x, j0 - 2, bar);
      tma_load_tile(&ft->hr[0][0], &maps->m[CM_H], x, j0 - 1, bar);
      for (int q = 0; q < 3; q++) {
        tma_load_tile(&ft->xt[q][0][0], &maps->m[CM_XT + q], x, j0, bar);
        tma_load_tile(&ft->yt[q][0][0], &maps->m[CM_YT + q], i0, j0 - 1, bar);
        tma_load_tile(&ft->tb[q][0][0], &maps->m[CM_TB + q], i0, j0, bar);
      }
    }
    const bool ok = mbar_wait_bounded(bar, 0, TMA_WAIT_TRIES);
    if (!__syncthreads_and(ok)) {                   // uniform: give up on the tile
      if (t == 0) atomicOr(&ctl->status, 4);
      mbar_wait_bounded(bar, 0, TMA_WAIT_TRIES);    // let a late copy land first
      cp_async_wait_all();
      __syncthreads();
      return;
    }
  }
  if (!fold) {
    // the ring's second pass on the last threads, as the velocities'
    constexpr int TREM = (SPX + 2) * (SPY + 2) - SP_THREADS;
    static_assert(TREM > 0 && TREM <= SP_THREADS, "one or two ring cells per thread");
    for (int pass = 0; pass < 2; pass++) {
      if (pass == 1 && t < SP_THREADS - TREM) break;
      const int q = pass == 0 ? t : t + TREM;
      const int ly = q / (SPX + 2), lx = q - ly * (SPX + 2);
      if (TMA) sm.th[ly][lx] = allDry ? 1.0 : split_theta_st(a, *ft, sm, i0, j0, dt, i0 - 1 + lx, j0 - 1 + ly);
      else sm.th[ly][lx] = allDry ? 1.0 : split_theta(a, s, sm, i0, j0, dt, i0 - 1 + lx, j0 - 1 + ly);
    }
    __syncthreads();
  }

  double locMax = 0, locFl = 0, hout = 0;
  if (gi < W && gj < H) {
    if (fold) split_cell<MODE, true>(a, s, sm, t, lx, ly, gi, gj, dt, locMax, locFl, hout);
    else split_cell<MODE, false, TMA>(a, s, sm, t, lx, ly, gi, gj, dt, locMax, locFl, hout, ft);
  }
  if (s.odry_out) {                               // the written tile's flag
    const bool ghostFree = i0 >= 2 && i0 + SPX <= W - 2 && j0 >= 2 && j0 + SPY <= H - 2;
    const bool own = __syncthreads_and(hout == 0) && ghostFree;
    if (t == 0) s.odry_out[ty * s.ntx + tx] = own ? 1 : 0;
  }

  // per-block partials, then the last block of the grid closes the step.
  // When no cell contributed (both start at +0 and only change to nonzero
  // values), the reduction would give +0 and 0: those are written directly.
  const bool any = __syncthreads_or(locMax != 0 || locFl != 0);   // uniform
  if (any) {
    for (int o = 16; o > 0; o >>= 1) {
      locMax = fmax(locMax, __shfl_down_sync(0xffffffffu, locMax, o));
      locFl += __shfl_down_sync(0xffffffffu, locFl, o);
    }
    if ((t & 31) == 0) { sm.red[0][t >> 5] = locMax; sm.red[1][t >> 5] = locFl; }
    __syncthreads();
  }
  if (t == 0) {
    double m = 0, f = 0;
    if (any) {
      m = sm.red[0][0]; f = sm.red[1][0];
      for (int w = 1; w < SP_THREADS / 32; w++) { m = fmax(m, sm.red[0][w]); f += sm.red[1][w]; }
    }
    if (MODE == 1) a.part_fl1[part] = f;
    else { a.part_max[part] = m; a.part_fl2[part] = f; }
    if (ticket) {
      __threadfence();
      const unsigned int tk = atomicAdd(&ctl->counter, 1u);
      sm.last = (tk == (unsigned int)(nparts - 1));
    }
  }
  if (!ticket) return;
  __syncthreads();
  if (!sm.last) return;                         // uniform across the CTA
  __threadfence();
  split_close_block<MODE>(a, ctl, nparts, sm);
}

#ifndef SWE_SPLIT_CELLS_MIN_BLOCKS
#define SWE_SPLIT_CELLS_MIN_BLOCKS 4
#endif
template <int MODE, bool SETTLE = false>
__global__ void __launch_bounds__(SP_THREADS, SWE_SPLIT_CELLS_MIN_BLOCKS)
k_split_cells(StageArgs a, SplitBufs s, Control* ctl) {
  pdl_enter();
  if (ctl->stop) return;
  __shared__ CellsSmem sm;
  split_cells_tile<MODE, SETTLE>(a, s, ctl, blockIdx.x, blockIdx.y, blockIdx.y * gridDim.x + blockIdx.x,
                         gridDim.x * gridDim.y, sm, false);
}

// The close of a stage over CLOSE_BLOCKS blocks: block b reduces its run of
// the tiles' partial slots (strided per thread, then a fixed tree) into
// scratch, and the last block to finish (a ticket among the CLOSE_BLOCKS)
// combines the blocks' results in block order (a fixed tree in one warp)
// and closes the stage as split_close_block does.  The maximum is the same
// in any order; the floored mass is summed in this fixed order.  One block
// reading 16 705 slots spent most of its time in dependent rounds of L2
// loads.  MODE 2 closes the whole step: stage 1's floored mass is needed
// only there, so it is summed here too (the same order as MODE 1 sums it)
// and stage 1 needs no close of its own.  scratch holds 3 * CLOSE_BLOCKS
// doubles.
constexpr int CLOSE_BLOCKS = 32;
template <int MODE>
__global__ void __launch_bounds__(SP_THREADS) k_split_close_multi(StageArgs a, Control* ctl, int nparts,
                                                                    double* scratch) {
  pdl_enter();
  if (ctl->stop) return;
  __shared__ double red[3][SP_THREADS / 32];
  __shared__ int last;
  const int t = threadIdx.x, b = blockIdx.x;
  const int chunk = (nparts + CLOSE_BLOCKS - 1) / CLOSE_BLOCKS;
  const int q0 = b * chunk, q1 = min(nparts, q0 + chunk);
  const double* pf = MODE == 1 ? a.part_fl1 : a.part_fl2;
  double m = 0, f = 0, f1 = 0;
  for (int q = q0 + t; q < q1; q += SP_THREADS) {
    if (MODE == 2) {
      m = fmax(m, __ldcg(a.part_max + q));
      f1 += __ldcg(a.part_fl1 + q);
    }
    f += __ldcg(pf + q);
  }
  for (int o = 16; o > 0; o >>= 1) {
    m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    f += __shfl_down_sync(0xffffffffu, f, o);
    f1 += __shfl_down_sync(0xffffffffu, f1, o);
  }
  if ((t & 31) == 0) { red[0][t >> 5] = m; red[1][t >> 5] = f; red[2][t >> 5] = f1; }
  __syncthreads();
  if (t == 0) {
    m = red[0][0]; f = red[1][0]; f1 = red[2][0];
    for (int w = 1; w < SP_THREADS / 32; w++) { m = fmax(m, red[0][w]); f += red[1][w]; f1 += red[2][w]; }
    scratch[b] = m;
    scratch[CLOSE_BLOCKS + b] = f;
    scratch[2 * CLOSE_BLOCKS + b] = f1;
    __threadfence();
    last = atomicAdd(&ctl->counter, 1u) == (unsigned int)(CLOSE_BLOCKS - 1);
  }
  __syncthreads();
  if (!last || t >= 32) return;                   // uniform per block; warp 0 of the last block goes on
  __threadfence();
  static_assert(CLOSE_BLOCKS == 32, "one block result per lane");
  m = __ldcg(scratch + t);
  f = __ldcg(scratch + CLOSE_BLOCKS + t);
  f1 = __ldcg(scratch + 2 * CLOSE_BLOCKS + t);
  for (int o = 16; o > 0; o >>= 1) {
    m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    f += __shfl_down_sync(0xffffffffu, f, o);
    f1 += __shfl_down_sync(0xffffffffu, f1, o);
  }
  if (t == 0) {
    const double dt = ctl->dt;
    if (MODE == 1) {
      ctl->floored1 = f;
    } else {
      ctl->floored1 = f1;
      ctl->next_max = m;
      ctl->mass_floored = f1 + f;
      ctl->t = ctl->t + dt;
      ctl->steps = ctl->steps + 1;
    }
    ctl->counter = 0;
  }
}

// The cell kernel with its face and depth inputs staged by tensor-map copies
// (maps over this simulation's own buffers only, no multicast).
template <int MODE, bool SETTLE = false>
__global__ void __launch_bounds__(SP_THREADS, SWE_SPLIT_CELLS_MIN_BLOCKS)
k_split_cells_tma(StageArgs a, SplitBufs s, Control* ctl, const __grid_constant__ CellMaps maps) {
  __shared__ CellsSmem sm;
  __shared__ CellFaceTiles ft;
  __shared__ alignas(8) unsigned long long bar;
  if (threadIdx.x == 0) mbar_init(&bar, 1);        // before the wait: touches no global memory
  pdl_enter();
  if (ctl->stop) return;
  split_cells_tile<MODE, SETTLE, true>(a, s, ctl, blockIdx.x, blockIdx.y, blockIdx.y * gridDim.x + blockIdx.x,
                                       gridDim.x * gridDim.y, sm, false, &ft, &maps, &bar);
}

// The cell kernel over its list: CTA b runs the list's entry b; the CTAs
// past the list's length exit after reading it.
template <int MODE, bool SETTLE = false>
__global__ void __launch_bounds__(SP_THREADS, SWE_SPLIT_CELLS_MIN_BLOCKS)
k_split_cells_tma_list(StageArgs a, SplitBufs s, Control* ctl, const __grid_constant__ CellMaps maps,
                       const int* list, const int* count) {
  __shared__ CellsSmem sm;
  __shared__ CellFaceTiles ft;
  __shared__ alignas(8) unsigned long long bar;
  pdl_enter();
  const int ntiles = s.ntx * s.nty;
  if ((int)blockIdx.x >= min(*count, ntiles) || ctl->stop) return;
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  const int tile = list[blockIdx.x];
  split_cells_tile<MODE, SETTLE, true>(a, s, ctl, tile % s.ntx, tile / s.ntx, tile, ntiles, sm, false, &ft, &maps,
                                       &bar);
}

// Closes the stage k_split_cells left open: one block, no atomics (a
// ticket shared by every tile of a large grid serialises in L2).
template <int MODE>
__global__ void __launch_bounds__(SP_THREADS) k_split_close(StageArgs a, Control* ctl, int nparts) {
  pdl_enter();
  if (ctl->stop) return;
  __shared__ CellsSmem sm;
  split_close_block<MODE>(a, ctl, nparts, sm);
}

}  // namespace
}  // namespace swe
