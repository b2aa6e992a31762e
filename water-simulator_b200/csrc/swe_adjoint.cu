// swe_adjoint.cu -- discrete adjoint of the SSP-RK2 step: gradients of a
// gauge misfit with respect to the bed and the Manning-n field.
//
//   J = sum over steps s, gauges g of (b_g + h_g(s) - obs(s, g))^2
//
// Forward: the bit-exact step kernels of the library, dt = maxDt() each step
// (the dt sequence is recorded and then held fixed), the state stored every
// `checkpoint_every` steps.  Backward: for each segment, newest first, the
// segment is stepped forward again from its checkpoint (same kernels and
// arithmetic, so every branch is the branch the forward pass took), and
// each step's tape is kept as the tiled stage kernels write it: both stage
// inputs with their ghosts, their velocities, slopes and face fluxes, both
// positivity-limiter fields, the depths before each dryClean and friction's
// input.  Then each step is reversed from its tape: the hand-written reverse
// kernels run friction, dryClean, the stage combination, the residual and
// the ghost-cell maps backwards.  The initial depth h = max(0, eta0 - b) is
// part of the map from b to J.
//
// Scope: Cartesian grids; per side reflect (the default), outflow, periodic
// or Flather with a constant exterior state or a tide; any order and
// limiter, Coriolis, scalar or per-cell Manning n.  No sponge.
#include "../../include/swe_b200.h"
#include "swe_kernels.cuh"
#include "swe_split.cuh"
#include "swe_adjoint_math.cuh"

#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

namespace swe_host { void set_error(const std::string& msg); }

namespace {

using swe::BCArgs;
using swe::Control;
using swe::adj::FaceIn;
using swe::StageArgs;
using swe::pdl_enter;

int fail(int code, const std::string& m) { swe_host::set_error(m); return code; }

// Per step, what the step's prepare left in the control block: t at the
// start of the step, then the Flather sides' exterior eta[4] and u[4]
// (constants, or a tide at t).  The forward records it; the tape pass
// starts each segment from its t, and the reverse of the ghost fill reads
// the exterior state of the step it reverses.
constexpr int STEP_REC = 9;

#define CU(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) return fail(SWE_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// ---- forward intermediates of one residual evaluation ----------------------
struct Inter {
  double *U, *V;
  double *s[8];          // sE0 sB0 sU0 sV0 (x), sE1 sB1 sU1 sV1 (y)
  double *fx[swe::SPLIT_FACE_FIELDS], *fy[swe::SPLIT_FACE_FIELDS];   // M, T, N + pL, N + pR of the
                         // x face (k|k+1) and the y face (k|k+W), as the tiled face kernel writes them
};
using swe::F_M;
using swe::F_T;
using swe::F_NPL;
using swe::F_NPR;

struct Geo { int W, H, nx, ny; double minDepth, eps4, coriolis; int order, lim;
             const double *dxRow, *dyRowN, *dyRowS, *bedPhi; };

__device__ __forceinline__ bool xface_on(const Geo& g, int i, int j) { return j >= 2 && j < g.H - 2 && i >= 1 && i < g.W - 2; }
__device__ __forceinline__ bool yface_on(const Geo& g, int i, int j) { return j >= 1 && j < g.H - 2 && i >= 2 && i < g.W - 2; }

__device__ __forceinline__ FaceIn xface_in(const Geo& g, const double* b, const double* h, const Inter& it, int k) {
  const int r = k + 1;
  return {b[k], h[k], it.U[k], it.V[k], it.s[0][k], it.s[1][k], it.s[2][k], it.s[3][k],
          b[r], h[r], it.U[r], it.V[r], it.s[0][r], it.s[1][r], it.s[2][r], it.s[3][r]};
}
__device__ __forceinline__ FaceIn yface_in(const Geo& g, const double* b, const double* h, const Inter& it, int k) {
  const int r = k + g.W;        // v normal, u transverse
  return {b[k], h[k], it.V[k], it.U[k], it.s[4][k], it.s[5][k], it.s[7][k], it.s[6][k],
          b[r], h[r], it.V[r], it.U[r], it.s[4][r], it.s[5][r], it.s[7][r], it.s[6][r]};
}

// ---- adjoint of the residual -------------------------------------------------
struct AdjBuf {
  double *lR[3];          // adjoints of rh, rhu, rhv (input)
};

// Face accumulation (src/swe.mjs:530-555) backwards, one face at a time:
// the adjoints of the face's outputs (M, N, T, pL, pR) and the part of the
// positivity limiter's adjoint it sends to its upwind cell.
struct FaceAdj { double lM, lN, lT, lpL, lpR, lth; };

__device__ __forceinline__ FaceAdj xface_adj(const Geo& g, const Inter& it, const double* theta, const AdjBuf& a,
                                             int k, int i, int j) {
  FaceAdj f = {0, 0, 0, 0, 0, 0};
  if (!xface_on(g, i, j)) return f;
  const int kL = k, kR = k + 1;
  const double M = it.fx[F_M][k], T = it.fx[F_T][k], NpL = it.fx[F_NPL][k], NpR = it.fx[F_NPR][k];
  const double th = M >= 0 ? theta[kL] : theta[kR];
  const double inv = th / g.dxRow[j];
  f.lM = inv * (a.lR[0][kR] - a.lR[0][kL]);
  f.lN = inv * (a.lR[1][kR] - a.lR[1][kL]);
  f.lT = inv * (a.lR[2][kR] - a.lR[2][kL]);
  f.lpL = -inv * a.lR[1][kL];
  f.lpR = inv * a.lR[1][kR];
  const double linv = M * (a.lR[0][kR] - a.lR[0][kL]) + NpR * a.lR[1][kR] - NpL * a.lR[1][kL] +
                      T * (a.lR[2][kR] - a.lR[2][kL]);
  f.lth = swe::qdiv(linv, g.dxRow[j]);          // adjoints are often +-0 (qdiv)
  return f;
}

__device__ __forceinline__ FaceAdj yface_adj(const Geo& g, const Inter& it, const double* theta, const AdjBuf& a,
                                             int k, int i, int j) {
  FaceAdj f = {0, 0, 0, 0, 0, 0};
  if (!yface_on(g, i, j)) return f;
  const int kL = k, kR = k + g.W;
  const double M = it.fy[F_M][k], T = it.fy[F_T][k], NpL = it.fy[F_NPL][k], NpR = it.fy[F_NPR][k];
  const double th = M >= 0 ? theta[kL] : theta[kR];
  const double invL = th / g.dyRowN[j], invR = th / g.dyRowS[j + 1];
  // rh[kL] -= M invL; rhv[kL] -= (N + pL) invL; rhu[kL] -= T invL; rh[kR] += M invR; ...
  f.lM = invR * a.lR[0][kR] - invL * a.lR[0][kL];
  f.lN = invR * a.lR[2][kR] - invL * a.lR[2][kL];
  f.lT = invR * a.lR[1][kR] - invL * a.lR[1][kL];
  f.lpL = -invL * a.lR[2][kL];
  f.lpR = invR * a.lR[2][kR];
  const double linvL = -(M * a.lR[0][kL] + NpL * a.lR[2][kL] + T * a.lR[1][kL]);
  const double linvR = M * a.lR[0][kR] + NpR * a.lR[2][kR] + T * a.lR[1][kR];
  f.lth = swe::qdiv(linvL, g.dyRowN[j]) + swe::qdiv(linvR, g.dyRowS[j + 1]);
  return f;
}

// Positivity limiter (src/swe.mjs:511-529) backwards for cell k: the
// adjoint of its outgoing flux budget and of its depth.  Both are zero
// unless the limiter fired (theta < 1), so callers only come here then.
__device__ __forceinline__ void theta_adj(const Geo& g, const Inter& it, const double* theta, const double* h,
                                          double dt, const AdjBuf& a, int k, double& lout, double& lh) {
  lout = 0; lh = 0;
  const int i = k % g.W, j = k / g.W;
  if (!(dt > 0 && i >= 1 && i < g.W - 1 && j >= 1 && j < g.H - 1)) return;
  double lth = 0;
  if (it.fx[F_M][k] >= 0) lth += xface_adj(g, it, theta, a, k, i, j).lth;              // east face, upwind = k
  if (it.fx[F_M][k - 1] < 0) lth += xface_adj(g, it, theta, a, k - 1, i - 1, j).lth;   // west face
  if (it.fy[F_M][k] >= 0) lth += yface_adj(g, it, theta, a, k, i, j).lth;              // north face
  if (it.fy[F_M][k - g.W] < 0) lth += yface_adj(g, it, theta, a, k - g.W, i, j - 1).lth;   // south face
  double out = 0;
  if (it.fx[F_M][k] > 0) out += it.fx[F_M][k] / g.dxRow[j];
  if (it.fx[F_M][k - 1] < 0) out -= it.fx[F_M][k - 1] / g.dxRow[j];
  if (it.fy[F_M][k] > 0) out += it.fy[F_M][k] / g.dyRowN[j];
  if (it.fy[F_M][k - g.W] < 0) out -= it.fy[F_M][k - g.W] / g.dyRowS[j];
  const double avail = h[k];
  if (out * dt > avail && avail > 0) {                 // theta = avail / (out dt)
    lh = lth / (out * dt);
    lout = -lth * avail / (out * out * dt);
  }
}

__device__ __forceinline__ double lout_of(const Geo& g, const Inter& it, const double* theta, const double* h,
                                          double dt, const AdjBuf& a, int k) {
  double lo = 0, lh = 0;
  if (theta[k] < 1) theta_adj(g, it, theta, h, dt, a, k, lo, lh);
  return lo;
}

// ---- the residual backwards on 32-column tiles ---------------------------------
// The face kernels hand each cell the sum of its two faces' adjoints in one
// direction (8 values) instead of each face's 16, and the cell kernel runs
// the cell gather and the slopes' neighbour gather in one pass over a tile
// with a one-cell ring, so neither the per-face halves nor the slope
// derivatives go through device memory.
//
// x faces: a warp is 32 consecutive cells of a row (tile column bx).  Lane
// t's face is (i | i+1); its right half belongs to lane t+1 (a shuffle),
// lane 31's to lane 0 of tile bx+1 (the edge buffer ex, indexed (j, bx)).
// y faces: a 32 x 8 tile; row ty's upper half goes to row ty+1 through
// shared memory, row 7's to row 0 of tile row by+1 (ey, indexed (by, i)).
// Per-cell sums are in FaceIn's left-side order: b, h, normal, transverse,
// sE, sB, s(normal), s(transverse).
constexpr int AT_X = 32;           // tile width (one warp)
constexpr int AT_XROWS = 4;        // rows per x-face block (128 threads)
constexpr int AT_Y = 8;            // rows per y-face / cell tile (256 threads)
// The face kernels are latency bound: capped at 64 registers (32 warps per
// SM; a few hundred bytes of spills) they measured faster than at 80
// (24 warps) or at their natural 112 (16 warps).
#ifndef SWE_ADJ_FACE_WARPS
#define SWE_ADJ_FACE_WARPS 32
#endif
// The cell kernel waits on memory, but it keeps its natural 80 registers
// (three blocks, 24 warps per SM): capped at 64 (four blocks) or 48 (five)
// it spills and measured slower.
#ifndef SWE_ADJ_CELL_BLOCKS
#define SWE_ADJ_CELL_BLOCKS 3
#endif

struct FaceSums {
  double *sx[8], *sy[8];           // per cell: its east + west x faces, its north + south y faces
  double *ex[8], *ey[8];           // halves that cross a tile edge
  int ntx;                         // tiles per row (ceil(W / 32))
};

__global__ void __launch_bounds__(AT_X * AT_XROWS, SWE_ADJ_FACE_WARPS / AT_XROWS)
k_adj_xfaces(Geo g, const double* b, const double* h, Inter it, const double* theta, double dt, AdjBuf a,
             FaceSums S) {
  pdl_enter();
  const int tx = threadIdx.x, bx = blockIdx.x;
  const int i = bx * AT_X + tx, j = blockIdx.y * AT_XROWS + threadIdx.y;
  const bool valid = i < g.W && j < g.H;
  const int k = j * g.W + i;
  FaceIn gx = {};
  if (valid && xface_on(g, i, j)) {
    const FaceAdj f = xface_adj(g, it, theta, a, k, i, j);
    double lM = f.lM;
    const double M = it.fx[F_M][k];
    if (M > 0) lM += swe::qdiv(lout_of(g, it, theta, h, dt, a, k), g.dxRow[j]);
    if (M < 0) lM -= swe::qdiv(lout_of(g, it, theta, h, dt, a, k + 1), g.dxRow[j]);
    gx = swe::adj::face_rev(xface_in(g, b, h, it, k), g.minDepth, lM, f.lN, f.lT, f.lpL, f.lpR);
  }
  const double* p = &gx.bL;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const double r = __shfl_up_sync(0xffffffffu, p[8 + q], 1);
    if (valid) S.sx[q][k] = tx > 0 ? p[q] + r : p[q];
  }
  if (tx == AT_X - 1 && j < g.H) {
#pragma unroll
    for (int q = 0; q < 8; q++) S.ex[q][(size_t)j * S.ntx + bx] = p[8 + q];
  }
}

__global__ void __launch_bounds__(AT_X * AT_Y, SWE_ADJ_FACE_WARPS / AT_Y)
k_adj_yfaces(Geo g, const double* b, const double* h, Inter it, const double* theta, double dt, AdjBuf a,
             FaceSums S) {
  pdl_enter();
  __shared__ double up[AT_Y][8][AT_X];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = blockIdx.x * AT_X + tx, j = blockIdx.y * AT_Y + ty;
  const bool valid = i < g.W && j < g.H;
  const int k = j * g.W + i;
  FaceIn gy = {};
  if (valid && yface_on(g, i, j)) {
    const FaceAdj f = yface_adj(g, it, theta, a, k, i, j);
    double lM = f.lM;
    const double M = it.fy[F_M][k];
    if (M > 0) lM += swe::qdiv(lout_of(g, it, theta, h, dt, a, k), g.dyRowN[j]);
    if (M < 0) lM -= swe::qdiv(lout_of(g, it, theta, h, dt, a, k + g.W), g.dyRowS[j + 1]);
    gy = swe::adj::face_rev(yface_in(g, b, h, it, k), g.minDepth, lM, f.lN, f.lT, f.lpL, f.lpR);
  }
  const double* p = &gy.bL;
#pragma unroll
  for (int q = 0; q < 8; q++) up[ty][q][tx] = p[8 + q];
  __syncthreads();
  if (valid) {
#pragma unroll
    for (int q = 0; q < 8; q++) S.sy[q][k] = ty > 0 ? p[q] + up[ty - 1][q][tx] : p[q];
  }
  if (ty == AT_Y - 1 && i < g.W) {
#pragma unroll
    for (int q = 0; q < 8; q++) S.ey[q][(size_t)blockIdx.y * g.W + i] = p[8 + q];
  }
}

// The face sums of cell (i, j) in direction d (0: x, 1: y), with the half
// that crossed a tile edge: b, h, U, V and the four slope adjoints of that
// direction (sE, sB, sU, sV).
__device__ __forceinline__ void face_sums(const Geo& g, const FaceSums& S, int d, int i, int j, int k,
                                          double& db, double& dh, double& dU, double& dV, double ls[4]) {
  double v[8];
  if (d == 0) {
#pragma unroll
    for (int q = 0; q < 8; q++) v[q] = S.sx[q][k];
    if ((i & (AT_X - 1)) == 0 && i >= AT_X) {
      const size_t e = (size_t)j * S.ntx + (i / AT_X - 1);
#pragma unroll
      for (int q = 0; q < 8; q++) v[q] += S.ex[q][e];
    }
    db = v[0]; dh = v[1]; dU = v[2]; dV = v[3];
    ls[0] = v[4]; ls[1] = v[5]; ls[2] = v[6]; ls[3] = v[7];
  } else {
#pragma unroll
    for (int q = 0; q < 8; q++) v[q] = S.sy[q][k];
    if ((j % AT_Y) == 0 && j >= AT_Y) {
      const size_t e = (size_t)(j / AT_Y - 1) * g.W + i;
#pragma unroll
      for (int q = 0; q < 8; q++) v[q] += S.ey[q][e];
    }
    // y faces: normal = V, transverse = U; slopes sE1 sB1 sV1 sU1
    db = v[0]; dh = v[1]; dV = v[2]; dU = v[3];
    ls[0] = v[4]; ls[1] = v[5]; ls[3] = v[6]; ls[2] = v[7];
  }
}

// The bed term of direction d backwards (src/swe.mjs:570-598, Cartesian),
// into the slope adjoints of that direction and the cell's b, h adjoints.
__device__ __forceinline__ void bed_term_adj(const Geo& g, const double* b, const double* h, const Inter& it,
                                             const AdjBuf& a, int d, int j, int k, double ls[4], double& db,
                                             double& dh) {
  const double bk = b[k], eC = bk + h[k];
  const double sE = it.s[4 * d][k], sB = it.s[4 * d + 1][k];
  const double aP = eC + 0.5 * sE - (bk + 0.5 * sB), aM = eC - 0.5 * sE - (bk - 0.5 * sB);
  const double hP = swe::jmax0(aP), hM = swe::jmax0(aM);
  const double div = d == 0 ? g.dxRow[j] : g.bedPhi[j];
  const double lterm = a.lR[1 + d][k];
  const double lhPM = lterm * swe::qdiv(-SWE_G * 0.5 * sB, div);
  const double ldb = swe::qdiv(lterm * (-SWE_G * 0.5 * (hP + hM)), div);
  double leC = 0;
  if (aP > 0) { leC += lhPM; ls[0] += 0.5 * lhPM; db -= lhPM; ls[1] -= 0.5 * lhPM; }
  if (aM > 0) { leC += lhPM; ls[0] -= 0.5 * lhPM; db -= lhPM; ls[1] += 0.5 * lhPM; }
  ls[1] += ldb;
  db += leC; dh += leC;
}

// The limiter's derivatives for the four slopes of direction d at cell
// (i, j): ga (with respect to X[k] - X[km]) and gc (X[kp] - X[k]), each
// times the slope's adjoint.
__device__ __forceinline__ void limiter_adj(const Geo& g, const double* b, const double* h, const Inter& it, int d,
                                            int i, int j, int k, const double ls[4], double ga[4], double gc[4]) {
#pragma unroll
  for (int q = 0; q < 4; q++) { ga[q] = 0; gc[q] = 0; }
  if (!(g.order >= 2 && i >= 1 && i < g.W - 1 && j >= 1 && j < g.H - 1)) return;
  const int kp = d == 0 ? k + 1 : k + g.W, km = d == 0 ? k - 1 : k - g.W;
  if (h[k] <= g.minDepth || h[kp] <= g.minDepth || h[km] <= g.minDepth) return;
  const double eC = b[k] + h[k], eP = b[kp] + h[kp], eM = b[km] + h[km];
  const double X0[4] = {eC - eM, b[k] - b[km], it.U[k] - it.U[km], it.V[k] - it.V[km]};
  const double X1[4] = {eP - eC, b[kp] - b[k], it.U[kp] - it.U[k], it.V[kp] - it.V[k]};
#pragma unroll
  for (int q = 0; q < 4; q++) {
    double da, dc;
    swe::adj::limiter_grad(g.lim, X0[q], X1[q], da, dc);
    ga[q] = ls[q] * da;
    gc[q] = ls[q] * dc;
  }
}

// The slope adjoints of direction d at a cell, as its own tile computes
// them: face sums, plus the bed term on interior cells.
__device__ __forceinline__ void dir_slopes(const Geo& g, const double* b, const double* h, const Inter& it,
                                           const AdjBuf& a, const FaceSums& S, int d, int i, int j, int k,
                                           double ls[4], double& db, double& dh, double& dU, double& dV) {
  face_sums(g, S, d, i, j, k, db, dh, dU, dV, ls);
  const bool interior = i >= 2 && i < g.W - 2 && j >= 2 && j < g.H - 2;
  if (interior && g.order >= 2) bed_term_adj(g, b, h, it, a, d, j, k, ls, db, dh);
}

// Per cell of a 32 x 8 tile: gather the face sums, the bed term and
// Coriolis backwards, the positivity limiter's depth adjoint, the limiter
// derivatives of the slopes; then each cell collects the slope derivatives
// that land on it from itself and its four neighbours (the ring cells'
// derivatives are formed by this block too), and the velocities' reverse.
__global__ void __launch_bounds__(AT_X * AT_Y, SWE_ADJ_CELL_BLOCKS)
k_adj_cells_tiled(Geo g, const double* b, const double* h, const double* hu, const double* hv, Inter it,
                  const double* theta, double dt, AdjBuf a, FaceSums S, double* lb, double* lh, double* lhu,
                  double* lhv) {
  pdl_enter();
  // slope derivatives: [d][q] of ga / gc, on the tile plus a ring (rows 0..9, cols 0..33)
  __shared__ double sga[2][4][AT_Y + 2][AT_X + 2];
  __shared__ double sgc[2][4][AT_Y + 2][AT_X + 2];
  const int tx = threadIdx.x, ty = threadIdx.y, t = ty * AT_X + tx;
  const int i0 = blockIdx.x * AT_X, j0 = blockIdx.y * AT_Y;
  const int i = i0 + tx, j = j0 + ty;
  const bool valid = i < g.W && j < g.H;
  const int k = j * g.W + i;
  double db = 0, dh = 0, dU = 0, dV = 0, dhu = 0, dhv = 0;
  if (valid) {
    double ls[2][4];
    double xb, xh, xU, xV, yb, yh, yU, yV;
    face_sums(g, S, 0, i, j, k, xb, xh, xU, xV, ls[0]);
    face_sums(g, S, 1, i, j, k, yb, yh, yU, yV, ls[1]);
    db = xb + yb; dh = xh + yh; dU = xU + yU; dV = xV + yV;
    {
      double lo = 0, lhq = 0;
      if (theta[k] < 1) theta_adj(g, it, theta, h, dt, a, k, lo, lhq);
      dh += lhq;
    }
    const bool interior = i >= 2 && i < g.W - 2 && j >= 2 && j < g.H - 2;
    if (interior && g.order >= 2) {
      bed_term_adj(g, b, h, it, a, 0, j, k, ls[0], db, dh);
      bed_term_adj(g, b, h, it, a, 1, j, k, ls[1], db, dh);
    }
    if (interior && g.coriolis != 0 && g.coriolis == g.coriolis) {   // rhu += f hv; rhv -= f hu
      dhv += g.coriolis * a.lR[1][k];
      dhu -= g.coriolis * a.lR[2][k];
    }
#pragma unroll
    for (int d = 0; d < 2; d++) {
      double ga[4], gc[4];
      limiter_adj(g, b, h, it, d, i, j, k, ls[d], ga, gc);
#pragma unroll
      for (int q = 0; q < 4; q++) { sga[d][q][ty + 1][tx + 1] = ga[q]; sgc[d][q][ty + 1][tx + 1] = gc[q]; }
    }
  }
  // The ring: what a neighbour outside the tile sends in.  Left column: its
  // x-slope gc; right column: its x-slope ga; bottom row: its y-slope gc;
  // top row: its y-slope ga.  Threads 0..79 take one ring cell each.
  if (t < 2 * AT_Y + 2 * AT_X) {
    int ri, rj, d, sx, sy;
    bool want_c;
    if (t < AT_Y) { ri = i0 - 1; rj = j0 + t; d = 0; want_c = true; sx = 0; sy = t + 1; }
    else if (t < 2 * AT_Y) { ri = i0 + AT_X; rj = j0 + t - AT_Y; d = 0; want_c = false; sx = AT_X + 1; sy = t - AT_Y + 1; }
    else if (t < 2 * AT_Y + AT_X) { ri = i0 + t - 2 * AT_Y; rj = j0 - 1; d = 1; want_c = true; sx = ri - i0 + 1; sy = 0; }
    else { ri = i0 + t - 2 * AT_Y - AT_X; rj = j0 + AT_Y; d = 1; want_c = false; sx = ri - i0 + 1; sy = AT_Y + 1; }
    if (ri >= 0 && ri < g.W && rj >= 0 && rj < g.H) {
      const int rk = rj * g.W + ri;
      double ls[4], rb, rh, rU, rV;
      dir_slopes(g, b, h, it, a, S, d, ri, rj, rk, ls, rb, rh, rU, rV);
      double ga[4], gc[4];
      limiter_adj(g, b, h, it, d, ri, rj, rk, ls, ga, gc);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        if (want_c) sgc[d][q][sy][sx] = gc[q]; else sga[d][q][sy][sx] = ga[q];
      }
    }
  }
  __syncthreads();
  if (!valid) return;
  double lX[4] = {0, 0, 0, 0};                       // eta, b, U, V
#pragma unroll
  for (int d = 0; d < 2; d++) {
    const bool hasM = d == 0 ? i >= 1 : j >= 1;
    const bool hasP = d == 0 ? i + 1 < g.W : j + 1 < g.H;
    const int mx = d == 0 ? tx : tx + 1, my = d == 0 ? ty + 1 : ty;
    const int px = d == 0 ? tx + 2 : tx + 1, py = d == 0 ? ty + 1 : ty + 2;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      double v = sga[d][q][ty + 1][tx + 1] - sgc[d][q][ty + 1][tx + 1];
      if (hasM) v += sgc[d][q][my][mx];
      if (hasP) v -= sga[d][q][py][px];
      lX[q] += v;
    }
  }
  const double lU = lX[2] + dU, lV = lX[3] + dV;
  double dqU, dhU, dqV, dhV;
  swe::adj::vel_grad(hu[k], h[k], g.eps4, dqU, dhU);
  swe::adj::vel_grad(hv[k], h[k], g.eps4, dqV, dhV);
  lb[k] += lX[0] + lX[1] + db;
  lh[k] += lX[0] + dh + lU * dhU + lV * dhV;
  lhu[k] = (lhu[k] + dhu) + lU * dqU;
  lhv[k] = (lhv[k] + dhv) + lV * dqV;
}

// ---- the rest of the step backwards ----------------------------------------
// The ghost fill backwards.  Every final ghost value is one interior source
// cell under one map (swe::ghost_source: a copy, a copy with hu or hv
// negated, or the Flather state of a side, src/swe.mjs:1026-1126), so each
// ghost's adjoint moves to its source.  The host lists the ghosts of every
// source in the order of the forward fill; one thread per source adds its
// ghosts' adjoints in that order and zeroes them, so the sums are the same
// in every run.  The forward state of the source (the stage input, whose
// interior the fill left as it was) gives the Flather map's Jacobian.

// The Flather ghost backwards (the map of swe::flather_cell): L* is the
// ghost's adjoint, a* the source's, accumulated.
__device__ __forceinline__ void flather_rev(int side, double e0, double u0, double minDepth, double eps4, double b,
                                            double h, double hu, double hv, double Lb, double Lh, double Lhu,
                                            double Lhv, double& ab, double& ah, double& ahu, double& ahv) {
  const bool we = side < 2;
  const double Ln = we ? Lhu : Lhv;                 // the ghost's normal momentum
  ab += Lb;                                         // g.b = b
  if (h <= minDepth) {                              // g.h = max(0, e0 - b), momenta 0
    if (e0 - b > 0) ab -= Lh;
    return;
  }
  if (we) ahv += Lhv; else ahu += Lhu;              // the transverse momentum is copied
  const double qn = we ? hu : hv;
  const double etaInt = b + h;
  const double r = sqrt(SWE_G / h);
  const double sgn = (side == 0 || side == 2) ? 1 : -1;
  const double uInt = swe::vel(qn, h, eps4);
  const double Rin = u0 + sgn * e0 * r;
  const double Rout = uInt - sgn * etaInt * r;
  const double un = 0.5 * (Rin + Rout);
  const double en = sgn * (Rin - Rout) / (2 * r);
  const double gh = swe::jmax0(en - b);
  // g.h = max(0, en - b), g.qn = g.h un
  const double Lgh = Lh + Ln * un;
  const double Lun = Ln * gh;
  const double Len = en - b > 0 ? Lgh : 0;
  ab -= Len;
  // un = (Rin + Rout) / 2, en = sgn (Rin - Rout) / (2 r)
  const double LRin = 0.5 * Lun + Len * sgn / (2 * r);
  const double LRout = 0.5 * Lun - Len * sgn / (2 * r);
  double Lr = -Len * en / r;
  // Rout = uInt - sgn etaInt r, Rin = u0 + sgn e0 r
  Lr += -sgn * etaInt * LRout + sgn * e0 * LRin;
  const double LetaInt = -sgn * r * LRout;
  ab += LetaInt;
  ah += LetaInt;
  double dq, dh;
  swe::adj::vel_grad(qn, h, eps4, dq, dh);
  if (we) ahu += LRout * dq; else ahv += LRout * dq;
  ah += LRout * dh;
  ah += Lr * (-0.5 * r / h);                        // r = sqrt(G / h)
}

// map: sources[nsrc], offsets[nsrc + 1], ghosts[n], transforms[n] (padded
// cell indices; swe::GT_*).  X: the stage input the fill was applied to.
__global__ void k_adj_bc(int nsrc, const int* map, const double* b, const double* h, const double* hu,
                         const double* hv, const double* fl, double minDepth, double eps4, double* lb, double* lh,
                         double* lhu, double* lhv) {
  pdl_enter();
  const int* src = map;
  const int* off = map + nsrc;
  const int* gcell = off + nsrc + 1;
  const int* gtr = gcell + off[nsrc];
  for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < nsrc; u += gridDim.x * blockDim.x) {
    const int sk = src[u];
    double ab = lb[sk], ah = lh[sk], ahu = lhu[sk], ahv = lhv[sk];
    for (int m = off[u]; m < off[u + 1]; m++) {
      const int gk = gcell[m], tr = gtr[m];
      const double Lb = lb[gk], Lh = lh[gk], Lhu = lhu[gk], Lhv = lhv[gk];
      lb[gk] = 0; lh[gk] = 0; lhu[gk] = 0; lhv[gk] = 0;
      if (tr >= swe::GT_FLATHER) {
        const int side = tr - swe::GT_FLATHER;
        flather_rev(side, fl[side], fl[4 + side], minDepth, eps4, b[sk], h[sk], hu[sk], hv[sk], Lb, Lh, Lhu,
                    Lhv, ab, ah, ahu, ahv);
      } else {
        ab += Lb;
        ah += Lh;
        ahu += tr == swe::GT_FLIPU ? -Lhu : Lhu;
        ahv += tr == swe::GT_FLIPV ? -Lhv : Lhv;
      }
    }
    lb[sk] = ab; lh[sk] = ah; lhu[sk] = ahu; lhv[sk] = ahv;
  }
}

// The end of the step backwards, one pass per cell: friction (as
// k_adj_friction), dryClean from the stage-2 pre-clean depth (as
// k_adj_dryclean), then A = 0.5 (W1 + B + dt R2), which sends
// lB = 0.5 lA, lR = 0.5 dt lA and leaves lA <- 0.5 lA (= lW1).
__device__ __forceinline__ void friction_rev(double minDepth, double eps4, double n, double dt, double hk,
                                             double qu, double qv, double& a0, double& a1, double& a2,
                                             double* ln, int k) {
  if (!(n != 0 && n == n)) return;                  // identity (scalar n == 0 skips entirely)
  if (hk <= minDepth) { a1 = 0; a2 = 0; return; }
  const double den = swe::vel_den(hk, eps4);
  const double u = swe::qdiv(swe::vel_num(qu, hk), den), v = swe::qdiv(swe::vel_num(qv, hk), den);
  const double speed = hypot(u, v);
  if (speed < 1e-14) return;
  const double P = swe::pow43(hk);                // the forward's own value
  const double K = dt * SWE_G * n * n;
  const double denom = 1 + K * speed / P;
  const double ghu = a1, ghv = a2;
  const double lden = swe::qdiv(-(ghu * qu + ghv * qv), denom * denom);
  double gh = 0, gq = swe::qdiv(ghu, denom), gr = swe::qdiv(ghv, denom);
  const double lspeed = lden * K / P;
  const double lP = -lden * K * speed / (P * P);
  if (ln) ln[k] += lden * dt * SWE_G * 2 * n * speed / P;
  gh += lP * (4.0 / 3.0) * P / hk;
  const double lu = lspeed * u / speed, lv = lspeed * v / speed;
  double dqU, dhU, dqV, dhV;
  swe::adj::vel_grad(qu, hk, eps4, dqU, dhU);
  swe::adj::vel_grad(qv, hk, eps4, dqV, dhV);
  gq += lu * dqU; gr += lv * dqV; gh += lu * dhU + lv * dhV;
  a0 += gh; a1 = gq; a2 = gr;
}

__global__ void k_adj_tail2(int W, int H, double minDepth, double eps4, double manning, const double* nfield,
                            double dt, const double* fh, const double* fhu, const double* fhv, const double* hA,
                            double* lA0, double* lA1, double* lA2, double* ln, double* lB0, double* lB1,
                            double* lB2, double* lR0, double* lR1, double* lR2) {
  pdl_enter();
  const double hdt = 0.5 * dt;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < W * H; k += gridDim.x * blockDim.x) {
    const int i = k % W, j = k / W;
    double a0 = lA0[k], a1 = lA1[k], a2 = lA2[k];
    if (i >= 2 && i < W - 2 && j >= 2 && j < H - 2) {
      friction_rev(minDepth, eps4, nfield ? nfield[k] : manning, dt, fh[k], fhu[k], fhv[k], a0, a1, a2, ln, k);
      const double hp = hA[k];
      const double hc = hp < 0 ? 0 : hp;
      if (hp < 0) a0 = 0;
      if (hc <= minDepth) { a1 = 0; a2 = 0; }
    }
    lB0[k] = 0.5 * a0; lB1[k] = 0.5 * a1; lB2[k] = 0.5 * a2;
    lR0[k] = hdt * a0; lR1[k] = hdt * a1; lR2[k] = hdt * a2;
    lA0[k] = 0.5 * a0; lA1[k] = 0.5 * a1; lA2[k] = 0.5 * a2;
  }
}

// Stage 1 backwards after its ghost map: dryClean from the stage-1
// pre-clean depth, then B = W1 + dt R1: lW1 += lB, lR = dt lB (lB is dead
// afterwards, so the cleaned values are not stored).
__global__ void k_adj_tail1(int W, int H, double minDepth, double dt, const double* hB, const double* lB0,
                            const double* lB1, const double* lB2, double* lA0, double* lA1, double* lA2,
                            double* lR0, double* lR1, double* lR2) {
  pdl_enter();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < W * H; k += gridDim.x * blockDim.x) {
    const int i = k % W, j = k / W;
    double b0 = lB0[k], b1 = lB1[k], b2 = lB2[k];
    if (i >= 2 && i < W - 2 && j >= 2 && j < H - 2) {
      const double hp = hB[k];
      const double hc = hp < 0 ? 0 : hp;
      if (hp < 0) b0 = 0;
      if (hc <= minDepth) { b1 = 0; b2 = 0; }
    }
    lA0[k] += 1.0 * b0; lA1[k] += 1.0 * b1; lA2[k] += 1.0 * b2;
    lR0[k] = dt * b0; lR1[k] = dt * b1; lR2[k] = dt * b2;
  }
}

// J += sum_g (b + h - obs)^2 (one thread, fixed order); and its adjoint.
// J += sum over gauges, in gauge order, of (b + h - obs)^2; eta at the gauges.
// The loads run in parallel; one thread adds the squares in order.
constexpr int MISFIT_THREADS = 256;
__global__ void k_misfit(const double* b, const double* h, const int* gk, const double* obs, int ng,
                         double* J, double* eta_out) {
  pdl_enter();
  __shared__ double r2[MISFIT_THREADS];
  double s = 0;
  if (threadIdx.x == 0) s = *J;
  for (int base = 0; base < ng; base += MISFIT_THREADS) {
    const int q = base + threadIdx.x;
    if (q < ng) {
      const double e = b[gk[q]] + h[gk[q]];
      if (eta_out) eta_out[q] = e;
      if (obs) { const double r = e - obs[q]; r2[threadIdx.x] = r * r; }
    }
    __syncthreads();
    if (threadIdx.x == 0 && obs)
      for (int t = 0; t < MISFIT_THREADS && base + t < ng; t++) s += r2[t];
    __syncthreads();
  }
  if (threadIdx.x == 0) *J = s;
}
// The misfit backwards: lh, lb += 2 (b + h - obs) at every gauge.  Gauges
// that share a cell form a group, added in gauge order by one thread, so the
// sums are those of a sequential pass over the gauges; groups run in parallel.
__global__ void k_adj_misfit(const double* b, const double* h, const int* gcell, const int* goff, const int* gidx,
                             int ngroups, const double* obs, double* lb, double* lh) {
  pdl_enter();
  for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < ngroups; u += gridDim.x * blockDim.x) {
    const int k = gcell[u];
    const double e = b[k] + h[k];
    double ah = lh[k], ab = lb[k];
    for (int m = goff[u]; m < goff[u + 1]; m++) {
      const double r = e - obs[gidx[m]];
      ah += 2 * r;
      ab += 2 * r;
    }
    lh[k] = ah;
    lb[k] = ab;
  }
}
// After a step's prepare: t and the Flather exterior state into rec (STEP_REC doubles).
__global__ void k_record_step(const Control* ctl, double* rec) {
  pdl_enter();
  if (threadIdx.x == 0) {
    rec[0] = ctl->t;
    for (int q = 0; q < 4; q++) { rec[1 + q] = ctl->fl_eta[q]; rec[5 + q] = ctl->fl_u[q]; }
  }
}
// The time of the step a segment's tape pass starts with.
__global__ void k_set_t(Control* ctl, const double* rec) {
  pdl_enter();
  if (threadIdx.x == 0) ctl->t = rec[0];
}
__global__ void k_record_dt(const Control* ctl, double* dts, int s) {
  pdl_enter();
  if (threadIdx.x == 0) dts[s] = ctl->dt;
}
// dst[q] = src[q] for q < nf (checkpoints and the segment tape's copies of
// the state, as a kernel so that the stepping chain stays one of kernels).
__global__ void k_copy(size_t n, int nf, double* d0, double* d1, double* d2, const double* s0, const double* s1,
                       const double* s2) {
  pdl_enter();
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    d0[k] = s0[k];
    if (nf > 1) { d1[k] = s1[k]; d2[k] = s2[k]; }
  }
}
// h0 = max(0, eta0 - b): d h0 / d b = -1 where eta0 - b > 0 (interior).
__global__ void k_adj_initial(int W, int H, const double* b, const double* eta0, const double* lh, double* lb) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < W * H; k += gridDim.x * blockDim.x) {
    const int i = k % W, j = k / W;
    if (!(i >= 2 && i < W - 2 && j >= 2 && j < H - 2)) continue;
    if (eta0[k] - b[k] > 0) lb[k] -= lh[k];
  }
}
// h0 = max(0, eta0 - b) over the padded grid, as the constructor samples it.
__global__ void k_init_state(int N, const double* b, const double* eta0, double* h, double* hu, double* hv) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    h[k] = swe::jmax0(eta0[k] - b[k]); hu[k] = 0; hv[k] = 0;
  }
}
}  // namespace

struct swe_adjoint {
  swe_options o;
  int W, H, N, steps, every, nseg, ng;
  double eps4;
  cudaStream_t st = nullptr;
  std::vector<double*> allocs;
  double *b, *eta0, *nfield = nullptr, *geom;
  double *A[3], *Bf[3], *X[3];                            // state, stage-1 output, segment state
  double *ckpt, *tape;                                    // checkpoints, one segment's tapes
  double *dts, *obs = nullptr, *J, *eta_series = nullptr;
  int* gk;
  int* gmeta = nullptr;          // gauge groups by cell: cells, offsets, gauge indices
  int ngroups = 0;
  double *lA[3], *lB[3], *lb, *ln;
  AdjBuf ab;
  FaceSums fs;                     // per-cell face sums of the tiled reverse kernels
  double *part;
  Control* ctl;
  int nblocks;
  dim3 grid;
  swe::SplitBufs sb;               // the tiled stage kernels' fields
  dim3 sgrid;
  int pcap = 0;                    // partial slots per kind (the most tiles either kernel uses)
  bool forward_done = false;
  bool pdl = true;                 // programmatic dependent launch between the stepping kernels
  bool fixed_dt = false;         // forward uses the given dt sequence instead of maxDt()
  int kind[4] = {SWE_BC_REFLECT, SWE_BC_REFLECT, SWE_BC_REFLECT, SWE_BC_REFLECT};   // W, E, S, N
  double fl_eta[4] = {0, 0, 0, 0}, fl_u[4] = {0, 0, 0, 0};   // constant exterior state of the Flather sides
  int fl_kind[4] = {0, 0, 0, 0};  // 1: the side's exterior state is the tide of ctl_init
  Control ctl_init = {};          // the control block each forward starts from (tide tables, zeros)
  double* rec = nullptr;          // STEP_REC doubles per step
  int* gmap = nullptr;           // the ghost fill by source (k_adj_bc)
  int nsrc = 0;
  std::vector<double> dts_host;  // the dt sequence, read once per backward pass
};

namespace {

Geo geo_of(const swe_adjoint* s) {
  Geo g;
  g.W = s->W; g.H = s->H; g.nx = s->o.nx; g.ny = s->o.ny;
  g.minDepth = s->o.min_depth; g.eps4 = s->eps4; g.coriolis = s->o.coriolis;
  g.order = s->o.order; g.lim = s->o.limiter;
  g.dxRow = s->geom + SWE_GEOM_DXROW * s->H; g.dyRowN = s->geom + SWE_GEOM_DYROWN * s->H;
  g.dyRowS = s->geom + SWE_GEOM_DYROWS * s->H; g.bedPhi = s->geom + SWE_GEOM_BEDPHI * s->H;
  return g;
}

StageArgs stage_args(const swe_adjoint* s, double* const* in, double* const* out) {
  StageArgs a;
  std::memset(&a, 0, sizeof a);
  a.W = s->W; a.H = s->H; a.nx = s->o.nx; a.ny = s->o.ny; a.b = s->b;
  a.h = in[0]; a.hu = in[1]; a.hv = in[2];
  if (out) { a.oh = out[0]; a.ohu = out[1]; a.ohv = out[2]; }
  const double* g = s->geom;
  const int H = s->H;
  a.m.dxRow = g + SWE_GEOM_DXROW * H; a.m.dyRowN = g + SWE_GEOM_DYROWN * H; a.m.dyRowS = g + SWE_GEOM_DYROWS * H;
  a.m.dyCFL = g + SWE_GEOM_DYCFL * H; a.m.bedPhi = g + SWE_GEOM_BEDPHI * H; a.m.geoCoef = g + SWE_GEOM_GEOCOEF * H;
  a.m.fRow = g + SWE_GEOM_FROW * H; a.m.tanPhi = g + SWE_GEOM_TANPHI * H;
  a.m.rdxRow = g + (SWE_GEOM_NROWS + 0) * H; a.m.rdyRowN = g + (SWE_GEOM_NROWS + 1) * H;
  a.m.rdyRowS = g + (SWE_GEOM_NROWS + 2) * H; a.m.R = INFINITY;
  a.minDepth = s->o.min_depth; a.eps4 = s->eps4; a.coriolis = s->o.coriolis;
  a.sph = 0; a.order = s->o.order; a.lim = s->o.limiter;
  a.manning = s->o.manning; a.nfield = s->nfield;
  a.part_max = s->part; a.part_fl1 = s->part + s->pcap; a.part_fl2 = s->part + 2 * s->pcap;
  a.nblocks = s->nblocks;
  return a;
}

BCArgs bc_args(const swe_adjoint* s, double* const* f) {
  BCArgs a;
  a.nx = s->o.nx; a.ny = s->o.ny; a.W = s->W; a.H = s->H;
  for (int q = 0; q < 4; q++) a.kind[q] = s->kind[q];
  a.minDepth = s->o.min_depth; a.eps4 = s->eps4;
  a.b = s->b; a.h = f[0]; a.hu = f[1]; a.hv = f[2];
  return a;
}

int G1(const swe_adjoint* s) { return std::min(4096, (s->N + 255) / 256); }
int bcb(const swe_adjoint* s) { return (4 * s->o.ny + 4 * (s->o.nx + 4) + 255) / 256; }
int adjbc_blocks(const swe_adjoint* s) { return std::max(1, (s->nsrc + 255) / 256); }

// A launch on the handle's stream that, with `pdl`, may be scheduled while
// the previous kernel drains (every kernel here waits for its predecessors
// in pdl_enter before touching memory).  The first kernel after a memset or
// a copy is launched without it.
template <typename... KArgs, typename... Args>
cudaError_t launch(const swe_adjoint* s, bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s->st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = (pdl && s->pdl) ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}
#define LAUNCH(...) CU(launch(s, true, __VA_ARGS__))

int copy3(swe_adjoint* s, double* const* dst, double* const* src, bool pdl = true) {
  CU(launch(s, pdl, k_copy, dim3(G1(s)), dim3(256), (size_t)s->N, 3, dst[0], dst[1], dst[2],
            (const double*)src[0], (const double*)src[1], (const double*)src[2]));
  return SWE_OK;
}

// The step's prepare: dt = maxDt() from the CFL rate (auto_dt) or the
// recorded dt of step k, and the Flather exterior state at the control
// block's t.
swe::PrepArgs prep_of(const swe_adjoint* s, bool auto_dt, int k) {
  swe::PrepArgs p;
  std::memset(&p, 0, sizeof p);
  p.mode = auto_dt ? 1 : 4;
  p.cfl = s->o.cfl;
  p.t_end = INFINITY;
  p.dt_dev = s->dts + k;
  for (int q = 0; q < 4; q++) { p.fl_kind[q] = s->fl_kind[q]; p.fl_eta[q] = s->fl_eta[q]; p.fl_u[q] = s->fl_u[q]; }
  return p;
}

// One forward step of state X in place.
int fwd_step(swe_adjoint* s, double* const* X, bool auto_dt, int step_index) {
  LAUNCH(swe::k_prepare, dim3(1), dim3(32), s->ctl, prep_of(s, auto_dt, step_index));
  LAUNCH(k_record_step, dim3(1), dim3(32), (const Control*)s->ctl, s->rec + (size_t)STEP_REC * step_index);
  const dim3 spb(swe::SP_THREADS);
  const int nparts = (int)(s->sgrid.x * s->sgrid.y);
  LAUNCH(swe::k_apply_bc, dim3(bcb(s)), dim3(256), bc_args(s, X), (const Control*)s->ctl, 0);
  const StageArgs a1 = stage_args(s, X, s->Bf);
  LAUNCH(swe::k_split_faces, s->sgrid, spb, a1, s->sb, s->ctl);
  LAUNCH(swe::k_split_cells<1>, s->sgrid, spb, a1, s->sb, s->ctl);
  LAUNCH(swe::k_split_close<1>, dim3(1), spb, a1, s->ctl, nparts);
  LAUNCH(swe::k_apply_bc, dim3(bcb(s)), dim3(256), bc_args(s, s->Bf), (const Control*)s->ctl, 0);
  const StageArgs a2 = stage_args(s, s->Bf, X);
  LAUNCH(swe::k_split_faces, s->sgrid, spb, a2, s->sb, s->ctl);
  LAUNCH(swe::k_split_cells<2>, s->sgrid, spb, a2, s->sb, s->ctl);
  LAUNCH(swe::k_split_close<2>, dim3(1), spb, a2, s->ctl, nparts);
  if (auto_dt) LAUNCH(k_record_dt, dim3(1), dim3(32), (const Control*)s->ctl, s->dts, step_index);
  return SWE_OK;
}


// R^T: given ab.lR (adjoint of rh, rhu, rhv over all cells) at state X (ghosts
// filled), add into lX (h, hu, hv) and lb.
// `it` holds the velocities, slopes and faces of X, as the tape recorded them.
int residual_adjoint(swe_adjoint* s, double* const* X, const Inter& it, const double* theta, double dt,
                     double* const* lX) {
  const Geo g = geo_of(s);
  const int ntx = (s->W + AT_X - 1) / AT_X;
  const double* b = s->b;
  const double* h = X[0];
  LAUNCH(k_adj_xfaces, dim3(ntx, (s->H + AT_XROWS - 1) / AT_XROWS), dim3(AT_X, AT_XROWS), g, b, h, it, theta, dt,
         s->ab, s->fs);
  LAUNCH(k_adj_yfaces, dim3(ntx, (s->H + AT_Y - 1) / AT_Y), dim3(AT_X, AT_Y), g, b, h, it, theta, dt, s->ab, s->fs);
  LAUNCH(k_adj_cells_tiled, dim3(ntx, (s->H + AT_Y - 1) / AT_Y), dim3(AT_X, AT_Y), g, b, h, (const double*)X[1],
         (const double*)X[2], it, theta, dt, s->ab, s->fs, s->lb, lX[0], lX[1], lX[2]);
  return SWE_OK;
}

// One step's tape: what the reverse of the step reads.  The segment pass
// writes it while stepping forward from the segment's checkpoint with the
// same tiled stage kernels and the recorded dt, so the states are the
// forward pass's own.
struct Tape {
  double* W1[3];   // stage-1 input with ghosts filled
  double* th1;     // positivity limiter of stage 1
  double* hB;      // stage-1 depth before dryClean
  double* Bp[3];   // stage-2 input with ghosts filled
  double* th2;     // positivity limiter of stage 2
  double* hA;      // stage-2 depth before dryClean
  double* Bf[3];   // friction's input
  double* hX;      // the step's output depth (the misfit reads it)
  Inter it1, it2;  // velocities, slopes and faces of the two stage inputs
};
constexpr int INTER_FIELDS = 2 + 8 + 2 * swe::SPLIT_FACE_FIELDS;
constexpr int TAPE_FIELDS = 14 + 2 * INTER_FIELDS;

Inter inter_at(double* p, size_t N) {
  Inter it;
  it.U = p; it.V = p + N;
  for (int q = 0; q < 8; q++) it.s[q] = p + (2 + q) * N;
  for (int q = 0; q < swe::SPLIT_FACE_FIELDS; q++) {
    it.fx[q] = p + (10 + q) * N;
    it.fy[q] = p + (10 + swe::SPLIT_FACE_FIELDS + q) * N;
  }
  return it;
}

Tape tape_at(const swe_adjoint* s, int t) {
  double* p = s->tape + (size_t)t * TAPE_FIELDS * s->N;
  const size_t N = s->N;
  Tape T;
  for (int q = 0; q < 3; q++) { T.W1[q] = p + q * N; T.Bp[q] = p + (5 + q) * N; T.Bf[q] = p + (10 + q) * N; }
  T.th1 = p + 3 * N; T.hB = p + 4 * N; T.th2 = p + 8 * N; T.hA = p + 9 * N; T.hX = p + 13 * N;
  T.it1 = inter_at(p + 14 * N, N);
  T.it2 = inter_at(p + (14 + INTER_FIELDS) * N, N);
  return T;
}

// The tiled kernels' buffers for a stage whose faces, slopes and velocities
// go to the tape (the source terms stay in the handle's scratch).
swe::SplitBufs tape_bufs(const swe_adjoint* s, const Inter& it) {
  swe::SplitBufs b = s->sb;
  for (int q = 0; q < swe::SPLIT_FACE_FIELDS; q++) { b.fx[q] = it.fx[q]; b.fy[q] = it.fy[q]; }
  for (int q = 0; q < 8; q++) b.sl[q] = it.s[q];
  b.U = it.U;
  b.V = it.V;
  return b;
}

// Step k forward from X (in place) and record its tape: the tiled stage
// kernels write the limiter, the depth before dryClean and friction's input
// as they go.
int tape_step(swe_adjoint* s, double* const* X, int k, const Tape& T) {
  const dim3 spb(swe::SP_THREADS);
  const int nparts = (int)(s->sgrid.x * s->sgrid.y);
  if (k % s->every == 0) LAUNCH(k_set_t, dim3(1), dim3(32), s->ctl, (const double*)(s->rec + (size_t)STEP_REC * k));
  LAUNCH(swe::k_prepare, dim3(1), dim3(32), s->ctl, prep_of(s, false, k));
  // the step input with its ghosts, in X (U0 of the in-place stage 2) and on the tape
  LAUNCH(swe::k_apply_bc, dim3(bcb(s)), dim3(256), bc_args(s, X), (const Control*)s->ctl, 0);
  if (int rc = copy3(s, T.W1, X)) return rc;
  StageArgs a1 = stage_args(s, T.W1, T.Bp);
  a1.tape_th = T.th1; a1.tape_hpre = T.hB;
  const swe::SplitBufs b1 = tape_bufs(s, T.it1);
  LAUNCH(swe::k_split_faces, s->sgrid, spb, a1, b1, s->ctl);
  LAUNCH(swe::k_split_cells<1>, s->sgrid, spb, a1, b1, s->ctl);
  LAUNCH(swe::k_split_close<1>, dim3(1), spb, a1, s->ctl, nparts);
  LAUNCH(swe::k_apply_bc, dim3(bcb(s)), dim3(256), bc_args(s, T.Bp), (const Control*)s->ctl, 0);
  StageArgs a2 = stage_args(s, T.Bp, X);
  a2.tape_th = T.th2; a2.tape_hpre = T.hA;
  for (int q = 0; q < 3; q++) a2.tape_pre[q] = T.Bf[q];
  const swe::SplitBufs b2 = tape_bufs(s, T.it2);
  LAUNCH(swe::k_split_faces, s->sgrid, spb, a2, b2, s->ctl);
  LAUNCH(swe::k_split_cells<2>, s->sgrid, spb, a2, b2, s->ctl);
  LAUNCH(swe::k_split_close<2>, dim3(1), spb, a2, s->ctl, nparts);
  LAUNCH(k_copy, dim3(G1(s)), dim3(256), (size_t)s->N, 1, T.hX, (double*)nullptr, (double*)nullptr,
         (const double*)X[0], (const double*)nullptr, (const double*)nullptr);
  return SWE_OK;
}

// Reverse step k: on entry lA holds the adjoint of the step's output
// (interior), on exit the adjoint of its input (interior); lb and ln
// accumulate.
int reverse_step(swe_adjoint* s, int k, const Tape& T) {
  const int gb = G1(s);
  const double dt = s->dts_host[k];
  double* lA[3] = {s->lA[0], s->lA[1], s->lA[2]};
  double* lB[3] = {s->lB[0], s->lB[1], s->lB[2]};
  // friction, dryClean, A = 0.5 (W1 + Bp + dt R2) backwards in one pass
  LAUNCH(k_adj_tail2, dim3(gb), dim3(256), s->W, s->H, s->o.min_depth, s->eps4, s->o.manning,
         (const double*)s->nfield, dt, (const double*)T.Bf[0], (const double*)T.Bf[1], (const double*)T.Bf[2],
         (const double*)T.hA, lA[0], lA[1], lA[2], s->ln, lB[0], lB[1], lB[2], s->ab.lR[0], s->ab.lR[1],
         s->ab.lR[2]);
  int rc = residual_adjoint(s, T.Bp, T.it2, T.th2, dt, lB);
  if (rc) return rc;
  LAUNCH(k_adj_bc, dim3(adjbc_blocks(s)), dim3(256), s->nsrc, (const int*)s->gmap, (const double*)s->b,
         (const double*)T.Bp[0], (const double*)T.Bp[1], (const double*)T.Bp[2],
         (const double*)(s->rec + (size_t)STEP_REC * k + 1), s->o.min_depth, s->eps4,
         s->lb, lB[0], lB[1], lB[2]);
  // dryClean and B = W1 + dt R1 backwards: lW1 += lB, lR1 = dt lB
  LAUNCH(k_adj_tail1, dim3(gb), dim3(256), s->W, s->H, s->o.min_depth, dt, (const double*)T.hB,
         (const double*)lB[0], (const double*)lB[1], (const double*)lB[2], lA[0], lA[1], lA[2], s->ab.lR[0],
         s->ab.lR[1], s->ab.lR[2]);
  rc = residual_adjoint(s, T.W1, T.it1, T.th1, dt, lA);
  if (rc) return rc;
  LAUNCH(k_adj_bc, dim3(adjbc_blocks(s)), dim3(256), s->nsrc, (const int*)s->gmap, (const double*)s->b,
         (const double*)T.W1[0], (const double*)T.W1[1], (const double*)T.W1[2],
         (const double*)(s->rec + (size_t)STEP_REC * k + 1), s->o.min_depth, s->eps4,
         s->lb, lA[0], lA[1], lA[2]);
  CU(cudaGetLastError());
  return SWE_OK;
}

// The ghost fill by source, for k_adj_bc: every ghost in the order of the
// forward fill (swe::apply_bc_range: the W/E rings row by row, then the S/N
// rings column by column), grouped by source in order of first appearance.
int build_ghost_map(swe_adjoint* s) {
  const int nx = s->o.nx, ny = s->o.ny, W = s->W;
  const int nwe = 4 * ny, nsn = 4 * (nx + 4);
  std::vector<int> src;
  std::vector<std::vector<std::pair<int, int>>> members;
  std::unordered_map<int, int> group;
  for (int q = 0; q < nwe + nsn; q++) {
    int i, j;
    if (q < nwe) {
      j = q / 4;
      const int r = q % 4;
      i = r < 2 ? -1 - r : nx + (r - 2);
    } else {
      const int p = q - nwe;
      i = p / 4 - 2;
      const int r = p % 4;
      j = r < 2 ? -1 - r : ny + (r - 2);
    }
    int si, sj;
    const int tr = swe::ghost_source(s->kind, nx, ny, i, j, si, sj);
    const int gk = (j + 2) * W + (i + 2), sk = (sj + 2) * W + (si + 2);
    auto it = group.find(sk);
    int u;
    if (it == group.end()) {
      u = (int)src.size();
      group.emplace(sk, u);
      src.push_back(sk);
      members.emplace_back();
    } else {
      u = it->second;
    }
    members[u].push_back({gk, tr});
  }
  std::vector<int> map(src);
  map.push_back(0);
  for (auto& m : members) map.push_back(map.back() + (int)m.size());
  for (auto& m : members)
    for (auto& e : m) map.push_back(e.first);
  for (auto& m : members)
    for (auto& e : m) map.push_back(e.second);
  CU(cudaStreamSynchronize(s->st));
  if (s->gmap) cudaFree(s->gmap);
  s->gmap = nullptr;
  s->nsrc = 0;
  CU(cudaMalloc(&s->gmap, sizeof(int) * map.size()));
  CU(cudaMemcpyAsync(s->gmap, map.data(), sizeof(int) * map.size(), cudaMemcpyHostToDevice, s->st));
  CU(cudaStreamSynchronize(s->st));
  s->nsrc = (int)src.size();
  return SWE_OK;
}

void free_adj(swe_adjoint* s) {
  for (double* p : s->allocs) cudaFree(p);
  if (s->gk) cudaFree(s->gk);
  if (s->gmeta) cudaFree(s->gmeta);
  if (s->gmap) cudaFree(s->gmap);
  if (s->ctl) cudaFree(s->ctl);
  if (s->st) cudaStreamDestroy(s->st);
}

}  // namespace

extern "C" {

int swe_adjoint_create(const swe_options* o, const double* b, const double* eta0, const double* manning_field,
                       int n_gauges, const int* gauge_cells, int steps, int checkpoint_every, swe_adjoint** out) {
  if (!out) return fail(SWE_EINVAL, "null output handle");
  *out = nullptr;
  if (!o || !b || !eta0 || steps < 1 || checkpoint_every < 1 || n_gauges < 1 || !gauge_cells)
    return fail(SWE_EINVAL, "swe_adjoint_create: options, b, eta0, gauges, steps >= 1, checkpoint_every >= 1");
  if (o->sphere) return fail(SWE_EINVAL, "swe_adjoint_create: the adjoint covers Cartesian grids");
  if (o->nx < 1 || o->ny < 1 || o->limiter < 0 || o->limiter > 2)
    return fail(SWE_EINVAL, "swe_adjoint_create: bad grid size or limiter");
  swe_adjoint* s = new swe_adjoint();
  auto bail = [&](int rc) { free_adj(s); delete s; return rc; };
  s->o = *o;
  s->W = o->nx + 4; s->H = o->ny + 4; s->N = s->W * s->H;
  s->steps = steps; s->every = checkpoint_every; s->nseg = (steps + checkpoint_every - 1) / checkpoint_every;
  s->ng = n_gauges;
  s->eps4 = std::pow(swe::jmax(o->min_depth, 1e-12), 4.0);
  for (int q = 0; q < n_gauges; q++)
    if (gauge_cells[q] < 0 || gauge_cells[q] >= s->N) return bail(fail(SWE_EINVAL, "gauge cell out of range"));
  const size_t N = s->N;
  if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(SWE_ECUDA, "swe_adjoint_create: stream"));
  auto alloc = [&](size_t n) -> double* {
    double* p = nullptr;
    if (cudaMalloc(&p, sizeof(double) * std::max<size_t>(n, 1)) != cudaSuccess) return nullptr;
    cudaMemsetAsync(p, 0, sizeof(double) * std::max<size_t>(n, 1), s->st);
    s->allocs.push_back(p);
    return p;
  };
  bool ok = true;
  auto A = [&](size_t n) { double* p = alloc(n); ok = ok && p; return p; };
  s->b = A(N); s->eta0 = A(N); s->geom = A((SWE_GEOM_NROWS + 3) * (size_t)s->H);
  if (manning_field) s->nfield = A(N);
  for (int q = 0; q < 3; q++) {
    s->A[q] = A(N); s->Bf[q] = A(N); s->X[q] = A(N);
    s->lA[q] = A(N); s->lB[q] = A(N);
  }
  s->ckpt = A(3 * N * (size_t)s->nseg);
  s->tape = nullptr;               // allocated by the first backward pass
  s->dts = A(steps);
  s->rec = A((size_t)STEP_REC * steps);
  s->obs = A((size_t)steps * n_gauges);
  s->eta_series = A((size_t)steps * n_gauges);
  s->J = A(1);
  s->lb = A(N); s->ln = A(N);
  for (int q = 0; q < 3; q++) s->ab.lR[q] = A(N);
  {
    const int ntx = (s->W + AT_X - 1) / AT_X, nty = (s->H + AT_Y - 1) / AT_Y;
    s->fs.ntx = ntx;
    for (int q = 0; q < 8; q++) {
      s->fs.sx[q] = A(N); s->fs.sy[q] = A(N);
      s->fs.ex[q] = A((size_t)ntx * s->H); s->fs.ey[q] = A((size_t)nty * s->W);
    }
  }
  const int gx = (s->W + swe::SX - 1) / swe::SX, gy = (s->H + 31) / 32;
  s->grid = dim3(gx, gy);
  s->nblocks = gx * gy;
  s->sgrid = dim3((s->W + swe::SPX - 1) / swe::SPX, (s->H + swe::SPY - 1) / swe::SPY);
  s->pcap = std::max(std::max(s->nblocks, (int)(s->sgrid.x * s->sgrid.y)), 1024);
  s->part = A(3 * (size_t)s->pcap);
  {
    double* spl = A((size_t)swe::SPLIT_FIELDS * N);
    if (spl) s->sb = swe::split_bufs_at(spl, N);
  }
  if (!ok || cudaMalloc(&s->ctl, sizeof(Control)) != cudaSuccess || cudaMalloc(&s->gk, sizeof(int) * n_gauges) != cudaSuccess)
    return bail(fail(SWE_ECUDA, "swe_adjoint_create: device allocation failed"));
  cudaMemsetAsync(s->ctl, 0, sizeof(Control), s->st);
  {
    const char* pe = std::getenv("SWE_B200_PDL");
    s->pdl = !(pe && std::strcmp(pe, "0") == 0);
  }
  std::vector<double> geom((size_t)(SWE_GEOM_NROWS + 3) * s->H), sc(6);
  int rc = swe_compute_geometry(o, geom.data(), sc.data());
  if (rc) return bail(rc);
  for (int r = 0; r < 3; r++) {
    const int src = r == 0 ? SWE_GEOM_DXROW : r == 1 ? SWE_GEOM_DYROWN : SWE_GEOM_DYROWS;
    for (int j = 0; j < s->H; j++)
      geom[(size_t)(SWE_GEOM_NROWS + r) * s->H + j] = 1.0 / geom[(size_t)src * s->H + j];
  }
  cudaMemcpyAsync(s->geom, geom.data(), sizeof(double) * geom.size(), cudaMemcpyHostToDevice, s->st);
  cudaMemcpyAsync(s->b, b, sizeof(double) * N, cudaMemcpyHostToDevice, s->st);
  cudaMemcpyAsync(s->eta0, eta0, sizeof(double) * N, cudaMemcpyHostToDevice, s->st);
  if (manning_field) cudaMemcpyAsync(s->nfield, manning_field, sizeof(double) * N, cudaMemcpyHostToDevice, s->st);
  cudaMemcpyAsync(s->gk, gauge_cells, sizeof(int) * n_gauges, cudaMemcpyHostToDevice, s->st);
  {
    // group the gauges by cell, groups in order of first appearance
    std::vector<int> cells;
    std::vector<std::vector<int>> members;
    std::unordered_map<int, int> group_of;
    for (int q = 0; q < n_gauges; q++) {
      auto it = group_of.find(gauge_cells[q]);
      int u;
      if (it == group_of.end()) {
        u = (int)cells.size();
        group_of.emplace(gauge_cells[q], u);
        cells.push_back(gauge_cells[q]);
        members.emplace_back();
      } else {
        u = it->second;
      }
      members[u].push_back(q);
    }
    s->ngroups = (int)cells.size();
    std::vector<int> meta(cells);
    meta.push_back(0);
    for (auto& m : members) meta.push_back(meta.back() + (int)m.size());
    for (auto& m : members) meta.insert(meta.end(), m.begin(), m.end());
    if (cudaMalloc(&s->gmeta, sizeof(int) * meta.size()) != cudaSuccess)
      return bail(fail(SWE_ECUDA, "swe_adjoint_create: out of device memory"));
    cudaMemcpyAsync(s->gmeta, meta.data(), sizeof(int) * meta.size(), cudaMemcpyHostToDevice, s->st);
    if (cudaStreamSynchronize(s->st) != cudaSuccess) return bail(fail(SWE_ECUDA, "swe_adjoint_create: upload"));
  }
  if (cudaStreamSynchronize(s->st) != cudaSuccess) return bail(fail(SWE_ECUDA, "swe_adjoint_create: upload"));
  if (int rc = build_ghost_map(s)) return bail(rc);
  *out = s;
  return SWE_OK;
}

int swe_adjoint_destroy(swe_adjoint* s) {
  if (!s) return SWE_OK;
  if (s->st) cudaStreamSynchronize(s->st);
  free_adj(s);
  delete s;
  return SWE_OK;
}

int swe_adjoint_set_observations(swe_adjoint* s, const double* obs) {
  if (!s || !obs) return fail(SWE_EINVAL, "null argument");
  CU(cudaMemcpyAsync(s->obs, obs, sizeof(double) * s->steps * s->ng, cudaMemcpyHostToDevice, s->st));
  CU(cudaStreamSynchronize(s->st));
  return SWE_OK;
}

int swe_adjoint_forward(swe_adjoint* s, double* J, double* gauge_eta) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  const int gb = G1(s);
  k_init_state<<<gb, 256, 0, s->st>>>(s->N, s->b, s->eta0, s->A[0], s->A[1], s->A[2]);
  CU(cudaMemcpyAsync(s->ctl, &s->ctl_init, sizeof(Control), cudaMemcpyHostToDevice, s->st));   // t = 0, tide tables
  CU(cudaMemsetAsync(s->J, 0, sizeof(double), s->st));
  {
    StageArgs a = stage_args(s, s->A, nullptr);
    swe::k_cfl_rate<<<std::min(1024, std::max(1, (s->o.nx * s->o.ny + 255) / 256)), swe::BX, 0, s->st>>>(a, s->ctl, s->part);
  }
  for (int k = 0; k < s->steps; k++) {
    if (k % s->every == 0) {
      double* dst[3] = {s->ckpt + (size_t)(k / s->every) * 3 * s->N, s->ckpt + ((size_t)(k / s->every) * 3 + 1) * s->N,
                        s->ckpt + ((size_t)(k / s->every) * 3 + 2) * s->N};
      if (int rc = copy3(s, dst, s->A)) return rc;
    }
    int rc = fwd_step(s, s->A, !s->fixed_dt, k);
    if (rc) return rc;
    LAUNCH(k_misfit, dim3(1), dim3(MISFIT_THREADS), (const double*)s->b, (const double*)s->A[0],
           (const int*)s->gk, (const double*)(s->obs + (size_t)k * s->ng), s->ng, s->J,
           s->eta_series + (size_t)k * s->ng);
  }
  CU(cudaGetLastError());
  if (J) CU(cudaMemcpyAsync(J, s->J, sizeof(double), cudaMemcpyDeviceToHost, s->st));
  if (gauge_eta)
    CU(cudaMemcpyAsync(gauge_eta, s->eta_series, sizeof(double) * s->steps * s->ng, cudaMemcpyDeviceToHost, s->st));
  CU(cudaStreamSynchronize(s->st));
  s->forward_done = true;
  return SWE_OK;
}

int swe_adjoint_backward(swe_adjoint* s, double* grad_b, double* grad_n) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  if (!s->forward_done) return fail(SWE_EINVAL, "swe_adjoint_backward: run swe_adjoint_forward first");
  const size_t N = s->N;
  for (int q = 0; q < 3; q++) CU(cudaMemsetAsync(s->lA[q], 0, sizeof(double) * N, s->st));
  CU(cudaMemsetAsync(s->lb, 0, sizeof(double) * N, s->st));
  CU(cudaMemsetAsync(s->ln, 0, sizeof(double) * N, s->st));
  if (!s->tape) {
    const size_t bytes = sizeof(double) * TAPE_FIELDS * N * (size_t)std::min(s->every, s->steps);
    if (cudaMalloc(&s->tape, bytes) != cudaSuccess) {
      cudaGetLastError();
      s->tape = nullptr;
      char buf[200];
      std::snprintf(buf, sizeof buf, "swe_adjoint_backward: the tape of one segment (%.2f GB) does not fit on "
                    "the device; use a smaller checkpoint_every", bytes / 1e9);
      return fail(SWE_ECUDA, buf);
    }
    s->allocs.push_back(s->tape);
  }
  s->dts_host.assign(s->steps, 0.0);
  CU(cudaMemcpyAsync(s->dts_host.data(), s->dts, sizeof(double) * s->steps, cudaMemcpyDeviceToHost, s->st));
  CU(cudaStreamSynchronize(s->st));
  for (int sg = s->nseg - 1; sg >= 0; sg--) {
    const int k0 = sg * s->every, k1 = std::min(s->steps, k0 + s->every);
    // the segment forward from its checkpoint, recording each step's tape
    double* src[3] = {s->ckpt + (size_t)sg * 3 * N, s->ckpt + ((size_t)sg * 3 + 1) * N, s->ckpt + ((size_t)sg * 3 + 2) * N};
    // the first kernel after the memsets and the tape allocation waits for them in stream order
    if (int rc = copy3(s, s->X, src, sg != s->nseg - 1)) return rc;
    for (int k = k0; k < k1; k++) {
      int rc = tape_step(s, s->X, k, tape_at(s, k - k0));
      if (rc) return rc;
    }
    for (int k = k1 - 1; k >= k0; k--) {
      const Tape T = tape_at(s, k - k0);
      LAUNCH(k_adj_misfit, dim3((s->ngroups + 127) / 128), dim3(128), (const double*)s->b, (const double*)T.hX,
             (const int*)s->gmeta, (const int*)(s->gmeta + s->ngroups), (const int*)(s->gmeta + 2 * s->ngroups + 1),
             s->ngroups, (const double*)(s->obs + (size_t)k * s->ng), s->lb, s->lA[0]);
      int rc = reverse_step(s, k, T);
      if (rc) return rc;
    }
  }
  k_adj_initial<<<G1(s), 256, 0, s->st>>>(s->W, s->H, s->b, s->eta0, s->lA[0], s->lb);
  CU(cudaGetLastError());
  if (grad_b) CU(cudaMemcpyAsync(grad_b, s->lb, sizeof(double) * N, cudaMemcpyDeviceToHost, s->st));
  if (grad_n) CU(cudaMemcpyAsync(grad_n, s->ln, sizeof(double) * N, cudaMemcpyDeviceToHost, s->st));
  CU(cudaStreamSynchronize(s->st));
  return SWE_OK;
}

int swe_adjoint_dt_sequence(swe_adjoint* s, double* dts_out, const double* dts_in) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  if (dts_in) {
    CU(cudaMemcpyAsync(s->dts, dts_in, sizeof(double) * s->steps, cudaMemcpyHostToDevice, s->st));
    s->fixed_dt = true;
  }
  if (dts_out) CU(cudaMemcpyAsync(dts_out, s->dts, sizeof(double) * s->steps, cudaMemcpyDeviceToHost, s->st));
  CU(cudaStreamSynchronize(s->st));
  return SWE_OK;
}

int swe_adjoint_set_boundary(swe_adjoint* s, int side, int kind) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  if (side < 0 || side > 3 || kind < SWE_BC_REFLECT || kind > SWE_BC_FLATHER)
    return fail(SWE_EINVAL, "swe_adjoint_set_boundary: side 0..3 (W, E, S, N), kind reflect/outflow/periodic/flather");
  s->kind[side] = kind;
  if (kind != SWE_BC_FLATHER) s->fl_kind[side] = 0;
  s->forward_done = false;
  return build_ghost_map(s);
}

int swe_adjoint_set_flather_values(swe_adjoint* s, int side, double eta_ext, double u_ext) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  if (side < 0 || side > 3) return fail(SWE_EINVAL, "swe_adjoint_set_flather_values: side 0..3 (W, E, S, N)");
  s->fl_eta[side] = eta_ext;
  s->fl_u[side] = u_ext;
  s->fl_kind[side] = 0;
  s->kind[side] = SWE_BC_FLATHER;
  s->forward_done = false;
  return build_ghost_map(s);
}

int swe_adjoint_set_flather_tide(swe_adjoint* s, int side, double msl, int n, const double* amp, const double* omega,
                                 const double* phase_deg, double u_coef) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  if (side < 0 || side > 3) return fail(SWE_EINVAL, "swe_adjoint_set_flather_tide: side 0..3 (W, E, S, N)");
  if (n < 0 || n > swe::MAX_TIDE) return fail(SWE_EINVAL, "tide tables hold at most 16 constituents");
  if (n > 0 && (!amp || !omega || !phase_deg)) return fail(SWE_EINVAL, "null tide table");
  Control& c = s->ctl_init;
  c.tide_n[side] = n; c.tide_msl[side] = msl; c.tide_ucoef[side] = u_coef;
  for (int q = 0; q < n; q++) {
    c.tide_amp[side][q] = amp[q]; c.tide_omega[side][q] = omega[q]; c.tide_phase[side][q] = phase_deg[q];
  }
  s->fl_kind[side] = 1;
  s->kind[side] = SWE_BC_FLATHER;
  s->forward_done = false;
  return build_ghost_map(s);
}

int swe_adjoint_get_stream(swe_adjoint* s, void** stream) {
  if (!s || !stream) return fail(SWE_EINVAL, "null argument");
  *stream = (void*)s->st;
  return SWE_OK;
}

}  // extern "C"
