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
// Scope: Cartesian grids, walls (reflect) on every side, any order and
// limiter, Coriolis, scalar or per-cell Manning n.  No sponge or Flather.
#include "../../include/swe_b200.h"
#include "swe_kernels.cuh"
#include "swe_split.cuh"
#include "swe_adjoint_math.cuh"

#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
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

int fail(int code, const std::string& m) { swe_host::set_error(m); return code; }

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
  double *gx[16], *gy[16];// face-input adjoints (FaceIn order)
  double *gs[16];         // per cell: (dslope/da, dslope/dc) x adjoint, 8 slopes
  double *dir[4];         // per cell: direct adjoints of b, h, U, V
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
  f.lth = linv / g.dxRow[j];
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
  f.lth = linvL / g.dyRowN[j] + linvR / g.dyRowS[j + 1];
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

// The faces backwards: limiter terms into the flux adjoint, then
// face_flux's reverse.
// 128 registers at most: 16 warps per SM instead of the 8 that 140 leave.
constexpr int FACES_CORE_THREADS = 128;
#ifndef SWE_FACES_CORE_MIN_BLOCKS
#define SWE_FACES_CORE_MIN_BLOCKS 4
#endif
// One launch for the x faces and one for the y faces: one face per thread
// fits 128 registers without spilling (16 warps per SM) and measured
// faster than both faces per thread at 128 or 168 registers.
#ifndef SWE_FACES_CORE_SPLIT
#define SWE_FACES_CORE_SPLIT 1
#endif
// WHICH: 0 the x face of each cell, 1 its y face, 2 both.
template <int WHICH>
__global__ void __launch_bounds__(FACES_CORE_THREADS, SWE_FACES_CORE_MIN_BLOCKS)
k_adj_faces_core(Geo g, const double* b, const double* h, Inter it, const double* theta, double dt, AdjBuf a) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < g.W * g.H; k += gridDim.x * blockDim.x) {
    const int i = k % g.W, j = k / g.W;
    if (WHICH != 1) {
      FaceIn gx = {};
      if (xface_on(g, i, j)) {
        const FaceAdj f = xface_adj(g, it, theta, a, k, i, j);
        double lM = f.lM;
        const double M = it.fx[F_M][k];
        if (M > 0) lM += lout_of(g, it, theta, h, dt, a, k) / g.dxRow[j];
        if (M < 0) lM -= lout_of(g, it, theta, h, dt, a, k + 1) / g.dxRow[j];
        gx = swe::adj::face_rev(xface_in(g, b, h, it, k), g.minDepth, lM, f.lN, f.lT, f.lpL, f.lpR);
      }
      const double* px = &gx.bL;
      for (int q = 0; q < 16; q++) a.gx[q][k] = px[q];
    }
    if (WHICH != 0) {
      FaceIn gy = {};
      if (yface_on(g, i, j)) {
        const FaceAdj f = yface_adj(g, it, theta, a, k, i, j);
        double lM = f.lM;
        const double M = it.fy[F_M][k];
        if (M > 0) lM += lout_of(g, it, theta, h, dt, a, k) / g.dyRowN[j];
        if (M < 0) lM -= lout_of(g, it, theta, h, dt, a, k + g.W) / g.dyRowS[j + 1];
        gy = swe::adj::face_rev(yface_in(g, b, h, it, k), g.minDepth, lM, f.lN, f.lT, f.lpL, f.lpR);
      }
      const double* py = &gy.bL;
      for (int q = 0; q < 16; q++) a.gy[q][k] = py[q];
    }
  }
}

enum { F_BL, F_HL, F_NL, F_TL, F_SEL, F_SBL, F_SNL, F_STL, F_BR, F_HR, F_NR, F_TR, F_SER, F_SBR, F_SNR, F_STR };

// Per cell: gather the faces' adjoints, add the bed term and Coriolis
// backwards, then the limiter derivatives of each slope.
__global__ void k_adj_cells(Geo g, const double* b, const double* h, const double* hu, const double* hv,
                            Inter it, const double* theta, double dt, AdjBuf a, double* lhu, double* lhv) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < g.W * g.H; k += gridDim.x * blockDim.x) {
    const int i = k % g.W, j = k / g.W;
    double db = 0, dh = 0, dU = 0, dV = 0;
    double ls[8] = {0, 0, 0, 0, 0, 0, 0, 0};         // sE0 sB0 sU0 sV0 sE1 sB1 sU1 sV1
    if (i + 1 < g.W && xface_on(g, i, j)) {          // east x face, cell is its left side
      db += a.gx[F_BL][k]; dh += a.gx[F_HL][k]; dU += a.gx[F_NL][k]; dV += a.gx[F_TL][k];
      ls[0] += a.gx[F_SEL][k]; ls[1] += a.gx[F_SBL][k]; ls[2] += a.gx[F_SNL][k]; ls[3] += a.gx[F_STL][k];
    }
    if (i >= 1 && xface_on(g, i - 1, j)) {           // west x face, cell is its right side
      const int f = k - 1;
      db += a.gx[F_BR][f]; dh += a.gx[F_HR][f]; dU += a.gx[F_NR][f]; dV += a.gx[F_TR][f];
      ls[0] += a.gx[F_SER][f]; ls[1] += a.gx[F_SBR][f]; ls[2] += a.gx[F_SNR][f]; ls[3] += a.gx[F_STR][f];
    }
    if (yface_on(g, i, j)) {                         // north y face, cell is its lower side (v normal)
      db += a.gy[F_BL][k]; dh += a.gy[F_HL][k]; dV += a.gy[F_NL][k]; dU += a.gy[F_TL][k];
      ls[4] += a.gy[F_SEL][k]; ls[5] += a.gy[F_SBL][k]; ls[7] += a.gy[F_SNL][k]; ls[6] += a.gy[F_STL][k];
    }
    if (j >= 1 && yface_on(g, i, j - 1)) {           // south y face, cell is its upper side
      const int f = k - g.W;
      db += a.gy[F_BR][f]; dh += a.gy[F_HR][f]; dV += a.gy[F_NR][f]; dU += a.gy[F_TR][f];
      ls[4] += a.gy[F_SER][f]; ls[5] += a.gy[F_SBR][f]; ls[7] += a.gy[F_SNR][f]; ls[6] += a.gy[F_STR][f];
    }
    {
      double lo = 0, lh = 0;
      if (theta[k] < 1) theta_adj(g, it, theta, h, dt, a, k, lo, lh);
      dh += lh;
    }
    double dhu = 0, dhv = 0;
    const bool interior = i >= 2 && i < g.W - 2 && j >= 2 && j < g.H - 2;
    if (interior && g.order >= 2) {                  // bed term, src/swe.mjs:570-598 (Cartesian)
      const double bk = b[k], eC = bk + h[k];
      for (int d = 0; d < 2; d++) {
        const double sE = it.s[4 * d][k], sB = it.s[4 * d + 1][k];
        const double aP = eC + 0.5 * sE - (bk + 0.5 * sB), aM = eC - 0.5 * sE - (bk - 0.5 * sB);
        const double hP = swe::jmax0(aP), hM = swe::jmax0(aM);
        const double div = d == 0 ? g.dxRow[j] : g.bedPhi[j];
        const double lterm = a.lR[1 + d][k];
        const double lhPM = lterm * (-SWE_G * 0.5 * sB / div);
        const double ldb = lterm * (-SWE_G * 0.5 * (hP + hM)) / div;
        double leC = 0;
        if (aP > 0) { leC += lhPM; ls[4 * d] += 0.5 * lhPM; db -= lhPM; ls[4 * d + 1] -= 0.5 * lhPM; }
        if (aM > 0) { leC += lhPM; ls[4 * d] -= 0.5 * lhPM; db -= lhPM; ls[4 * d + 1] += 0.5 * lhPM; }
        ls[4 * d + 1] += ldb;
        db += leC; dh += leC;
      }
    }
    if (interior && g.coriolis != 0 && g.coriolis == g.coriolis) {   // rhu += f hv; rhv -= f hu
      dhv += g.coriolis * a.lR[1][k];
      dhu -= g.coriolis * a.lR[2][k];
    }
    a.dir[0][k] = db; a.dir[1][k] = dh; a.dir[2][k] = dU; a.dir[3][k] = dV;
    lhu[k] += dhu; lhv[k] += dhv;
    // slopes: s = lim(X[k] - X[km], X[kp] - X[k]) for X = eta, b, U, V
    for (int d = 0; d < 2; d++) {
      double ga[4] = {0, 0, 0, 0}, gc[4] = {0, 0, 0, 0};
      if (g.order >= 2 && i >= 1 && i < g.W - 1 && j >= 1 && j < g.H - 1) {
        const int kp = d == 0 ? k + 1 : k + g.W, km = d == 0 ? k - 1 : k - g.W;
        if (!(h[k] <= g.minDepth || h[kp] <= g.minDepth || h[km] <= g.minDepth)) {
          const double eC = b[k] + h[k], eP = b[kp] + h[kp], eM = b[km] + h[km];
          const double X0[4] = {eC - eM, b[k] - b[km], it.U[k] - it.U[km], it.V[k] - it.V[km]};
          const double X1[4] = {eP - eC, b[kp] - b[k], it.U[kp] - it.U[k], it.V[kp] - it.V[k]};
          for (int q = 0; q < 4; q++) {
            double da, dc;
            swe::adj::limiter_grad(g.lim, X0[q], X1[q], da, dc);
            ga[q] = ls[4 * d + q] * da;
            gc[q] = ls[4 * d + q] * dc;
          }
        }
      }
      for (int q = 0; q < 4; q++) { a.gs[8 * d + 2 * q][k] = ga[q]; a.gs[8 * d + 2 * q + 1][k] = gc[q]; }
    }
  }
}

// Per cell: the slopes' derivatives land on the cell and its neighbours;
// eta = b + h, and the velocities' reverse.
__global__ void k_adj_cells_final(Geo g, const double* h, const double* hu, const double* hv, Inter it, AdjBuf a,
                                  double* lb, double* lh, double* lhu, double* lhv) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < g.W * g.H; k += gridDim.x * blockDim.x) {
    const int i = k % g.W, j = k / g.W;
    double lX[4] = {0, 0, 0, 0};                     // eta, b, U, V
    for (int d = 0; d < 2; d++) {
      const int st = d == 0 ? 1 : g.W;
      const bool hasM = d == 0 ? i >= 1 : j >= 1;
      const bool hasP = d == 0 ? i + 1 < g.W : j + 1 < g.H;
      for (int q = 0; q < 4; q++) {
        const double* GA = a.gs[8 * d + 2 * q];
        const double* GC = a.gs[8 * d + 2 * q + 1];
        double v = GA[k] - GC[k];                    // own slope: a = X[k] - X[km], c = X[kp] - X[k]
        if (hasM) v += GC[k - st];                   // slope of km: its c = X[k] - X[km]
        if (hasP) v -= GA[k + st];                   // slope of kp: its a = X[kp] - X[k]
        lX[q] += v;
      }
    }
    const double lU = lX[2] + a.dir[2][k], lV = lX[3] + a.dir[3][k];
    double dqU, dhU, dqV, dhV;
    swe::adj::vel_grad(hu[k], h[k], g.eps4, dqU, dhU);
    swe::adj::vel_grad(hv[k], h[k], g.eps4, dqV, dhV);
    lb[k] += lX[0] + lX[1] + a.dir[0][k];
    lh[k] += lX[0] + a.dir[1][k] + lU * dhU + lV * dhV;
    lhu[k] += lU * dqU;
    lhv[k] += lV * dqV;
  }
}

// ---- the rest of the step backwards ----------------------------------------
// Reflect walls: a ghost takes the clamped mirror source and flips the normal
// momentum (src/swe.mjs:1026-1039; corners from the S/N pass).  Backwards,
// each ghost's adjoint moves to its source cell.  Every ghost has exactly one
// source, and every source is an interior cell, so the map is a gather: one
// thread per interior cell of the two-cell band along the edges adds the
// ghosts that map to it, in the order of the forward fill (S/N pass by
// column then ghost row, south before north; then the W/E pass), and zeroes
// them.  The sums are therefore the same in every run.
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ void adj_bc_move(int W, int gi, int gj, int sk, double shu, double shv, double* lb,
                                            double* lh, double* lhu, double* lhv, double& ab, double& ah,
                                            double& ahu, double& ahv) {
  const int gk = (gj + 2) * W + (gi + 2);
  if (lb) { ab += lb[gk]; lb[gk] = 0; }
  if (lh) {
    ah += lh[gk]; lh[gk] = 0;
    ahu += shu * lhu[gk]; lhu[gk] = 0;
    ahv += shv * lhv[gk]; lhv[gk] = 0;
  }
  (void)sk;
}

__global__ void k_adj_bc(int nx, int ny, double* lb, double* lh, double* lhu, double* lhv) {
  const int W = nx + 4;
  const int rows[4] = {0, 1, ny - 2, ny - 1};
  const int cols[4] = {0, 1, nx - 2, nx - 1};
  const int total = 4 * nx + 4 * ny;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    int si, sj;
    if (t < 4 * nx) {                              // the two rows along each of S and N
      const int r = t / nx;
      si = t - r * nx;
      sj = rows[r];
      if (sj < 0 || sj > ny - 1) continue;
      bool dup = false;
      for (int q = 0; q < r; q++) dup |= rows[q] == sj;
      if (dup) continue;
    } else {                                       // the two columns along W and E, other rows
      const int u = t - 4 * nx;
      sj = u / 4;
      const int c = u - 4 * sj;
      si = cols[c];
      if (si < 0 || si > nx - 1) continue;
      bool dup = false;
      for (int q = 0; q < c; q++) dup |= cols[q] == si;
      for (int q = 0; q < 4; q++) dup |= rows[q] == sj;
      if (dup) continue;
    }
    const int sk = (sj + 2) * W + (si + 2);
    double ab = lb ? lb[sk] : 0, ah = 0, ahu = 0, ahv = 0;
    if (lh) { ah = lh[sk]; ahu = lhu[sk]; ahv = lhv[sk]; }
    // S/N pass: columns i that clamp to si, in increasing order
    int ilist[5], ni = 0;
    if (si == 0) { ilist[ni++] = -2; ilist[ni++] = -1; }
    ilist[ni++] = si;
    if (si == nx - 1) { ilist[ni++] = nx; ilist[ni++] = nx + 1; }
    for (int q = 0; q < ni; q++) {
      const int i = ilist[q];
      for (int gg = 0; gg < 2; gg++) {
        if (clampi(gg, 0, ny - 1) == sj)                       // south ghost row -1-gg
          adj_bc_move(W, i, -1 - gg, sk, 1, -1, lb, lh, lhu, lhv, ab, ah, ahu, ahv);
        if (clampi(ny - 1 - gg, 0, ny - 1) == sj)              // north ghost row ny+gg
          adj_bc_move(W, i, ny + gg, sk, 1, -1, lb, lh, lhu, lhv, ab, ah, ahu, ahv);
      }
    }
    // W/E pass of row sj
    for (int gg = 0; gg < 2; gg++) {
      if (clampi(gg, 0, nx - 1) == si) adj_bc_move(W, -1 - gg, sj, sk, -1, 1, lb, lh, lhu, lhv, ab, ah, ahu, ahv);
      if (clampi(nx - 1 - gg, 0, nx - 1) == si) adj_bc_move(W, nx + gg, sj, sk, -1, 1, lb, lh, lhu, lhv, ab, ah, ahu, ahv);
    }
    if (lb) lb[sk] = ab;
    if (lh) { lh[sk] = ah; lhu[sk] = ahu; lhv[sk] = ahv; }
  }
}

// dryClean (src/swe.mjs:734-745) backwards, from the pre-clean depth:
// a floored depth and zeroed momenta pass no adjoint.  Ghost outputs are
// dead (the next ghost fill overwrites them), so their adjoints are cleared.
__global__ void k_adj_dryclean(int W, int H, double minDepth, const double* hpre, double* lh, double* lhu, double* lhv) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < W * H; k += gridDim.x * blockDim.x) {
    const int i = k % W, j = k / W;
    if (!(i >= 2 && i < W - 2 && j >= 2 && j < H - 2)) continue;
    const double hp = hpre[k];
    const double hc = hp < 0 ? 0 : hp;
    if (hp < 0) lh[k] = 0;
    if (hc <= minDepth) { lhu[k] = 0; lhv[k] = 0; }
  }
}

// applyFriction (src/swe.mjs:659-704) backwards, from the post-dryClean state.
__global__ void k_adj_friction(int W, int H, double minDepth, double eps4, double manning, const double* nfield,
                               double dt, const double* h, const double* hu, const double* hv,
                               double* lh, double* lhu, double* lhv, double* ln) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < W * H; k += gridDim.x * blockDim.x) {
    const int i = k % W, j = k / W;
    if (!(i >= 2 && i < W - 2 && j >= 2 && j < H - 2)) continue;
    const double n = nfield ? nfield[k] : manning;
    if (!(n != 0 && n == n)) continue;               // identity (scalar n == 0 skips entirely)
    const double hk = h[k];
    if (hk <= minDepth) { lhu[k] = 0; lhv[k] = 0; continue; }
    const double den = swe::vel_den(hk, eps4);
    const double u = swe::vel_num(hu[k], hk) / den, v = swe::vel_num(hv[k], hk) / den;
    const double speed = hypot(u, v);
    if (speed < 1e-14) continue;
    const double P = pow(hk, 4.0 / 3.0);
    const double K = dt * SWE_G * n * n;
    const double denom = 1 + K * speed / P;
    const double ghu = lhu[k], ghv = lhv[k];
    const double lden = -(ghu * hu[k] + ghv * hv[k]) / (denom * denom);
    double gh = 0, gq = ghu / denom, gr = ghv / denom;
    const double lspeed = lden * K / P;
    const double lP = -lden * K * speed / (P * P);
    if (ln) ln[k] += lden * dt * SWE_G * 2 * n * speed / P;
    gh += lP * (4.0 / 3.0) * P / hk;
    const double lu = lspeed * u / speed, lv = lspeed * v / speed;
    double dqU, dhU, dqV, dhV;
    swe::adj::vel_grad(hu[k], hk, eps4, dqU, dhU);
    swe::adj::vel_grad(hv[k], hk, eps4, dqV, dhV);
    gq += lu * dqU; gr += lv * dqV; gh += lu * dhU + lv * dhV;
    lh[k] += gh; lhu[k] = gq; lhv[k] = gr;
  }
}

// J += sum_g (b + h - obs)^2 (one thread, fixed order); and its adjoint.
// J += sum over gauges, in gauge order, of (b + h - obs)^2; eta at the gauges.
// The loads run in parallel; one thread adds the squares in order.
constexpr int MISFIT_THREADS = 256;
__global__ void k_misfit(const double* b, const double* h, const int* gk, const double* obs, int ng,
                         double* J, double* eta_out) {
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
__global__ void k_set_dt(Control* ctl, const double* dts, int s) {
  if (threadIdx.x == 0) { ctl->dt = dts[s]; ctl->stop = 0; }
}
__global__ void k_record_dt(const Control* ctl, double* dts, int s) {
  if (threadIdx.x == 0) dts[s] = ctl->dt;
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
// dryClean's result (src/swe.mjs:734-745) on the interior, copying ghosts as they are.
// The stage combinations backwards, three fields at once.
// A = 0.5 (W1 + B + dt R2):  lB = 0.5 lA, lR = 0.5 dt lA, lA <- 0.5 lA (= lW1).
__global__ void k_split_stage2(int N, double dt, double* lA0, double* lA1, double* lA2, double* lB0, double* lB1,
                               double* lB2, double* lR0, double* lR1, double* lR2) {
  const double hdt = 0.5 * dt;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const double a0 = lA0[k], a1 = lA1[k], a2 = lA2[k];
    lB0[k] = 0.5 * a0; lB1[k] = 0.5 * a1; lB2[k] = 0.5 * a2;
    lR0[k] = hdt * a0; lR1[k] = hdt * a1; lR2[k] = hdt * a2;
    lA0[k] = 0.5 * a0; lA1[k] = 0.5 * a1; lA2[k] = 0.5 * a2;
  }
}
// B = W1 + dt R1:  lW1 += lB, lR = dt lB.
__global__ void k_split_stage1(int N, double dt, const double* lB0, const double* lB1, const double* lB2,
                               double* lA0, double* lA1, double* lA2, double* lR0, double* lR1, double* lR2) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const double b0 = lB0[k], b1 = lB1[k], b2 = lB2[k];
    lA0[k] += 1.0 * b0; lA1[k] += 1.0 * b1; lA2[k] += 1.0 * b2;
    lR0[k] = dt * b0; lR1[k] = dt * b1; lR2[k] = dt * b2;
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
  double *part;
  Control* ctl;
  int nblocks;
  dim3 grid;
  swe::SplitBufs sb;               // the tiled stage kernels' fields
  dim3 sgrid;
  int pcap = 0;                    // partial slots per kind (the most tiles either kernel uses)
  bool forward_done = false;
  bool fixed_dt = false;         // forward uses the given dt sequence instead of maxDt()
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
  for (int q = 0; q < 4; q++) a.kind[q] = SWE_BC_REFLECT;
  a.minDepth = s->o.min_depth; a.eps4 = s->eps4;
  a.b = s->b; a.h = f[0]; a.hu = f[1]; a.hv = f[2];
  return a;
}

int G1(const swe_adjoint* s) { return std::min(4096, (s->N + 255) / 256); }
int bcb(const swe_adjoint* s) { return (4 * s->o.ny + 4 * (s->o.nx + 4) + 255) / 256; }
int adjbc_blocks(const swe_adjoint* s) { return (4 * s->o.nx + 4 * s->o.ny + 255) / 256; }

// One forward step of state X in place, dt from the device control block
// (set by k_set_dt or, when auto_dt, from the CFL rate).
int fwd_step(swe_adjoint* s, double* const* X, bool auto_dt, int step_index) {
  if (auto_dt) {
    swe::PrepArgs p;
    std::memset(&p, 0, sizeof p);
    p.mode = 1; p.cfl = s->o.cfl; p.t_end = INFINITY;
    swe::k_prepare<<<1, 32, 0, s->st>>>(s->ctl, p);
  } else {
    k_set_dt<<<1, 32, 0, s->st>>>(s->ctl, s->dts, step_index);
  }
  swe::k_apply_bc<<<bcb(s), 256, 0, s->st>>>(bc_args(s, X), s->ctl, 0);
  const StageArgs a1 = stage_args(s, X, s->Bf);
  swe::k_split_faces<<<s->sgrid, swe::SP_THREADS, 0, s->st>>>(a1, s->sb, s->ctl);
  swe::k_split_cells<1><<<s->sgrid, swe::SP_THREADS, 0, s->st>>>(a1, s->sb, s->ctl);
  swe::k_split_close<1><<<1, swe::SP_THREADS, 0, s->st>>>(a1, s->ctl, (int)(s->sgrid.x * s->sgrid.y));
  swe::k_apply_bc<<<bcb(s), 256, 0, s->st>>>(bc_args(s, s->Bf), s->ctl, 0);
  const StageArgs a2 = stage_args(s, s->Bf, X);
  swe::k_split_faces<<<s->sgrid, swe::SP_THREADS, 0, s->st>>>(a2, s->sb, s->ctl);
  swe::k_split_cells<2><<<s->sgrid, swe::SP_THREADS, 0, s->st>>>(a2, s->sb, s->ctl);
  swe::k_split_close<2><<<1, swe::SP_THREADS, 0, s->st>>>(a2, s->ctl, (int)(s->sgrid.x * s->sgrid.y));
  CU(cudaGetLastError());
  if (auto_dt) k_record_dt<<<1, 32, 0, s->st>>>(s->ctl, s->dts, step_index);
  return SWE_OK;
}

void copy3(swe_adjoint* s, double* const* dst, double* const* src) {
  for (int q = 0; q < 3; q++)
    cudaMemcpyAsync(dst[q], src[q], sizeof(double) * s->N, cudaMemcpyDeviceToDevice, s->st);
}

// R^T: given ab.lR (adjoint of rh, rhu, rhv over all cells) at state X (ghosts
// filled), add into lX (h, hu, hv) and lb.
// `it` holds the velocities, slopes and faces of X, as the tape recorded them.
int residual_adjoint(swe_adjoint* s, double* const* X, const Inter& it, const double* theta, double dt,
                     double* const* lX) {
  const Geo g = geo_of(s);
  const int gb = G1(s);
  const int fcb = std::min(148 * 4 * 4, (s->N + FACES_CORE_THREADS - 1) / FACES_CORE_THREADS);
  if (SWE_FACES_CORE_SPLIT) {
    k_adj_faces_core<0><<<fcb, FACES_CORE_THREADS, 0, s->st>>>(g, s->b, X[0], it, theta, dt, s->ab);
    k_adj_faces_core<1><<<fcb, FACES_CORE_THREADS, 0, s->st>>>(g, s->b, X[0], it, theta, dt, s->ab);
  } else {
    k_adj_faces_core<2><<<fcb, FACES_CORE_THREADS, 0, s->st>>>(g, s->b, X[0], it, theta, dt, s->ab);
  }
  k_adj_cells<<<gb, 256, 0, s->st>>>(g, s->b, X[0], X[1], X[2], it, theta, dt, s->ab, lX[1], lX[2]);
  k_adj_cells_final<<<gb, 256, 0, s->st>>>(g, X[0], X[1], X[2], it, s->ab, s->lb, lX[0], lX[1], lX[2]);
  CU(cudaGetLastError());
  return SWE_OK;
}

// One step's tape: what the reverse of the step reads.  The segment pass
// writes it while stepping forward from the segment's checkpoint; the step
// is the same arithmetic as the fused kernels (their updates are these
// elementwise expressions, their residual is k_stage<0>), so the states are
// the forward pass's own.
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
  const int N = s->N;
  k_set_dt<<<1, 32, 0, s->st>>>(s->ctl, s->dts, k);
  copy3(s, T.W1, X);
  swe::k_apply_bc<<<bcb(s), 256, 0, s->st>>>(bc_args(s, T.W1), s->ctl, 0);
  StageArgs a1 = stage_args(s, T.W1, T.Bp);
  a1.tape_th = T.th1; a1.tape_hpre = T.hB;
  const swe::SplitBufs b1 = tape_bufs(s, T.it1);
  swe::k_split_faces<<<s->sgrid, swe::SP_THREADS, 0, s->st>>>(a1, b1, s->ctl);
  swe::k_split_cells<1><<<s->sgrid, swe::SP_THREADS, 0, s->st>>>(a1, b1, s->ctl);
  swe::k_split_close<1><<<1, swe::SP_THREADS, 0, s->st>>>(a1, s->ctl, (int)(s->sgrid.x * s->sgrid.y));
  swe::k_apply_bc<<<bcb(s), 256, 0, s->st>>>(bc_args(s, T.Bp), s->ctl, 0);
  copy3(s, X, T.W1);                               // U0 of the in-place stage 2
  StageArgs a2 = stage_args(s, T.Bp, X);
  a2.tape_th = T.th2; a2.tape_hpre = T.hA;
  for (int q = 0; q < 3; q++) a2.tape_pre[q] = T.Bf[q];
  const swe::SplitBufs b2 = tape_bufs(s, T.it2);
  swe::k_split_faces<<<s->sgrid, swe::SP_THREADS, 0, s->st>>>(a2, b2, s->ctl);
  swe::k_split_cells<2><<<s->sgrid, swe::SP_THREADS, 0, s->st>>>(a2, b2, s->ctl);
  swe::k_split_close<2><<<1, swe::SP_THREADS, 0, s->st>>>(a2, s->ctl, (int)(s->sgrid.x * s->sgrid.y));
  cudaMemcpyAsync(T.hX, X[0], sizeof(double) * N, cudaMemcpyDeviceToDevice, s->st);
  CU(cudaGetLastError());
  return SWE_OK;
}

// Reverse step k: on entry lA holds the adjoint of the step's output
// (interior), on exit the adjoint of its input (interior); lb and ln
// accumulate.
int reverse_step(swe_adjoint* s, int k, const Tape& T) {
  const int N = s->N, gb = G1(s);
  const double dt = s->dts_host[k];
  double* lA[3] = {s->lA[0], s->lA[1], s->lA[2]};
  double* lB[3] = {s->lB[0], s->lB[1], s->lB[2]};
  k_adj_friction<<<gb, 256, 0, s->st>>>(s->W, s->H, s->o.min_depth, s->eps4, s->o.manning, s->nfield, dt,
                                        T.Bf[0], T.Bf[1], T.Bf[2], lA[0], lA[1], lA[2], s->ln);
  k_adj_dryclean<<<gb, 256, 0, s->st>>>(s->W, s->H, s->o.min_depth, T.hA, lA[0], lA[1], lA[2]);
  // A = 0.5 (W1 + Bp + dt R2): lB = 0.5 lA, lR2 = 0.5 dt lA, lW1 = 0.5 lA
  k_split_stage2<<<gb, 256, 0, s->st>>>(N, dt, lA[0], lA[1], lA[2], lB[0], lB[1], lB[2], s->ab.lR[0],
                                        s->ab.lR[1], s->ab.lR[2]);
  int rc = residual_adjoint(s, T.Bp, T.it2, T.th2, dt, lB);
  if (rc) return rc;
  k_adj_bc<<<adjbc_blocks(s), 256, 0, s->st>>>(s->o.nx, s->o.ny, s->lb, lB[0], lB[1], lB[2]);
  k_adj_dryclean<<<gb, 256, 0, s->st>>>(s->W, s->H, s->o.min_depth, T.hB, lB[0], lB[1], lB[2]);
  // B = W1 + dt R1 (all cells): lW1 += lB, lR1 = dt lB
  k_split_stage1<<<gb, 256, 0, s->st>>>(N, dt, lB[0], lB[1], lB[2], lA[0], lA[1], lA[2], s->ab.lR[0],
                                        s->ab.lR[1], s->ab.lR[2]);
  rc = residual_adjoint(s, T.W1, T.it1, T.th1, dt, lA);
  if (rc) return rc;
  k_adj_bc<<<adjbc_blocks(s), 256, 0, s->st>>>(s->o.nx, s->o.ny, s->lb, lA[0], lA[1], lA[2]);
  CU(cudaGetLastError());
  return SWE_OK;
}

void free_adj(swe_adjoint* s) {
  for (double* p : s->allocs) cudaFree(p);
  if (s->gk) cudaFree(s->gk);
  if (s->gmeta) cudaFree(s->gmeta);
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
  s->obs = A((size_t)steps * n_gauges);
  s->eta_series = A((size_t)steps * n_gauges);
  s->J = A(1);
  s->lb = A(N); s->ln = A(N);
  for (int q = 0; q < 3; q++) s->ab.lR[q] = A(N);
  for (int q = 0; q < 16; q++) { s->ab.gx[q] = A(N); s->ab.gy[q] = A(N); s->ab.gs[q] = A(N); }
  for (int q = 0; q < 4; q++) s->ab.dir[q] = A(N);
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
  cudaFuncSetAttribute(swe::k_stage<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, swe::STAGE_SMEM_BYTES);
  cudaFuncSetAttribute(swe::k_stage<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, swe::STAGE_SMEM_BYTES);
  cudaFuncSetAttribute(swe::k_stage<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, swe::STAGE_SMEM_BYTES);
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
  CU(cudaMemsetAsync(s->ctl, 0, sizeof(Control), s->st));
  CU(cudaMemsetAsync(s->J, 0, sizeof(double), s->st));
  {
    StageArgs a = stage_args(s, s->A, nullptr);
    swe::k_cfl_rate<<<std::min(1024, std::max(1, (s->o.nx * s->o.ny + 255) / 256)), swe::BX, 0, s->st>>>(a, s->ctl, s->part);
  }
  for (int k = 0; k < s->steps; k++) {
    if (k % s->every == 0) {
      double* dst[3] = {s->ckpt + (size_t)(k / s->every) * 3 * s->N, s->ckpt + ((size_t)(k / s->every) * 3 + 1) * s->N,
                        s->ckpt + ((size_t)(k / s->every) * 3 + 2) * s->N};
      copy3(s, dst, s->A);
    }
    int rc = fwd_step(s, s->A, !s->fixed_dt, k);
    if (rc) return rc;
    k_misfit<<<1, MISFIT_THREADS, 0, s->st>>>(s->b, s->A[0], s->gk, s->obs + (size_t)k * s->ng, s->ng, s->J,
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
    copy3(s, s->X, src);
    for (int k = k0; k < k1; k++) {
      int rc = tape_step(s, s->X, k, tape_at(s, k - k0));
      if (rc) return rc;
    }
    for (int k = k1 - 1; k >= k0; k--) {
      const Tape T = tape_at(s, k - k0);
      k_adj_misfit<<<(s->ngroups + 127) / 128, 128, 0, s->st>>>(
          s->b, T.hX, s->gmeta, s->gmeta + s->ngroups, s->gmeta + 2 * s->ngroups + 1, s->ngroups,
          s->obs + (size_t)k * s->ng, s->lb, s->lA[0]);
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

int swe_adjoint_get_stream(swe_adjoint* s, void** stream) {
  if (!s || !stream) return fail(SWE_EINVAL, "null argument");
  *stream = (void*)s->st;
  return SWE_OK;
}

}  // extern "C"
