// swe_adjoint.cu -- discrete adjoint of the SSP-RK2 step: gradients of a
// gauge misfit with respect to the bed and the Manning-n field.
//
//   J = sum over steps s, gauges g of (b_g + h_g(s) - obs(s, g))^2
//
// Forward: the bit-exact step kernels of the library, dt = maxDt() each step
// (the dt sequence is recorded and then held fixed), the state stored every
// `checkpoint_every` steps.  Backward: for each segment, newest first, the
// segment's states are recomputed from its checkpoint; then each step is
// reversed: its two stages are recomputed (same kernels, so every branch is
// the branch the forward pass took) together with the residual's
// intermediates (velocities, slopes, face fluxes), and the hand-written
// reverse kernels run friction, dryClean, the stage combination, the
// residual and the ghost-cell maps backwards.  The initial depth
// h = max(0, eta0 - b) is part of the map from b to J.
//
// Scope: Cartesian grids, walls (reflect) on every side, any order and
// limiter, Coriolis, scalar or per-cell Manning n.  No sponge or Flather.
#include "../../include/swe_b200.h"
#include "swe_kernels.cuh"
#include "swe_adjoint_math.cuh"

#include <cuda_runtime.h>
#include <cmath>
#include <cstring>
#include <string>
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
  double *fx[5], *fy[5]; // M N T pL pR of the x face (k|k+1) and the y face (k|k+W)
};

struct Geo { int W, H, nx, ny; double minDepth, eps4, coriolis; int order, lim;
             const double *dxRow, *dyRowN, *dyRowS, *bedPhi; };

__global__ void k_vel(Geo g, const double* h, const double* hu, const double* hv, double* U, double* V) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < g.W * g.H; k += gridDim.x * blockDim.x) {
    const double hk = h[k];
    if (hk == 0) { U[k] = swe::vel_num(hu[k], hk); V[k] = swe::vel_num(hv[k], hk); continue; }
    const double den = swe::vel_den(hk, g.eps4);
    U[k] = swe::vel_num(hu[k], hk) / den;
    V[k] = swe::vel_num(hv[k], hk) / den;
  }
}

// src/swe.mjs:364-411
__global__ void k_slopes(Geo g, const double* b, const double* h, Inter it) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < g.W * g.H; k += gridDim.x * blockDim.x) {
    const int i = k % g.W, j = k / g.W;
    for (int d = 0; d < 2; d++) {
      double sE = 0, sB = 0, sU = 0, sV = 0;
      if (g.order >= 2 && i >= 1 && i < g.W - 1 && j >= 1 && j < g.H - 1) {
        const int kp = d == 0 ? k + 1 : k + g.W, km = d == 0 ? k - 1 : k - g.W;
        const double hk = h[k], bk = b[k], eC = bk + hk;
        if (!(hk <= g.minDepth || h[kp] <= g.minDepth || h[km] <= g.minDepth)) {
          const double eP = b[kp] + h[kp], eM = b[km] + h[km];
          sE = swe::limiter(g.lim, eC - eM, eP - eC);
          sB = swe::limiter(g.lim, bk - b[km], b[kp] - bk);
          sU = swe::limiter(g.lim, it.U[k] - it.U[km], it.U[kp] - it.U[k]);
          sV = swe::limiter(g.lim, it.V[k] - it.V[km], it.V[kp] - it.V[k]);
        }
      }
      it.s[4 * d][k] = sE; it.s[4 * d + 1][k] = sB; it.s[4 * d + 2][k] = sU; it.s[4 * d + 3][k] = sV;
    }
  }
}

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

// src/swe.mjs:414-475
__global__ void k_faces(Geo g, const double* b, const double* h, Inter it) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < g.W * g.H; k += gridDim.x * blockDim.x) {
    const int i = k % g.W, j = k / g.W;
    swe::Face fx = {0, 0, 0, 0, 0}, fy = {0, 0, 0, 0, 0};
    if (xface_on(g, i, j)) {
      const FaceIn x = xface_in(g, b, h, it, k);
      fx = swe::face_flux(x.bL, x.hL, x.nL, x.tL, x.sEL, x.sBL, x.sNL, x.sTL,
                          x.bR, x.hR, x.nR, x.tR, x.sER, x.sBR, x.sNR, x.sTR, g.minDepth);
    }
    if (yface_on(g, i, j)) {
      const FaceIn y = yface_in(g, b, h, it, k);
      fy = swe::face_flux(y.bL, y.hL, y.nL, y.tL, y.sEL, y.sBL, y.sNL, y.sTL,
                          y.bR, y.hR, y.nR, y.tR, y.sER, y.sBR, y.sNR, y.sTR, g.minDepth);
    }
    it.fx[0][k] = fx.M; it.fx[1][k] = fx.N; it.fx[2][k] = fx.T; it.fx[3][k] = fx.pL; it.fx[4][k] = fx.pR;
    it.fy[0][k] = fy.M; it.fy[1][k] = fy.N; it.fy[2][k] = fy.T; it.fy[3][k] = fy.pL; it.fy[4][k] = fy.pR;
  }
}

// ---- adjoint of the residual -------------------------------------------------
struct AdjBuf {
  double *lR[3];          // adjoints of rh, rhu, rhv (input)
  double *lFx[5], *lFy[5];// face-output adjoints (M N T pL pR)
  double *lthx, *lthy;    // theta adjoint a face sends to its upwind cell
  double *lout, *lhth;    // positivity limiter: adjoint of `out`, and the depth term
  double *gx[16], *gy[16];// face-input adjoints (FaceIn order)
  double *gs[16];         // per cell: (dslope/da, dslope/dc) x adjoint, 8 slopes
  double *dir[4];         // per cell: direct adjoints of b, h, U, V
};

// Face accumulation (src/swe.mjs:530-555) backwards.
__global__ void k_adj_faces_accum(Geo g, Inter it, const double* theta, AdjBuf a) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < g.W * g.H; k += gridDim.x * blockDim.x) {
    const int i = k % g.W, j = k / g.W;
    double lM = 0, lN = 0, lT = 0, lpL = 0, lpR = 0, lth = 0;
    if (xface_on(g, i, j)) {
      const int kL = k, kR = k + 1;
      const double M = it.fx[0][k], N = it.fx[1][k], T = it.fx[2][k], pL = it.fx[3][k], pR = it.fx[4][k];
      const double th = M >= 0 ? theta[kL] : theta[kR];
      const double inv = th / g.dxRow[j];
      lM = inv * (a.lR[0][kR] - a.lR[0][kL]);
      lN = inv * (a.lR[1][kR] - a.lR[1][kL]);
      lT = inv * (a.lR[2][kR] - a.lR[2][kL]);
      lpL = -inv * a.lR[1][kL];
      lpR = inv * a.lR[1][kR];
      const double linv = M * (a.lR[0][kR] - a.lR[0][kL]) + (N + pR) * a.lR[1][kR] - (N + pL) * a.lR[1][kL] +
                          T * (a.lR[2][kR] - a.lR[2][kL]);
      lth = linv / g.dxRow[j];
    }
    a.lFx[0][k] = lM; a.lFx[1][k] = lN; a.lFx[2][k] = lT; a.lFx[3][k] = lpL; a.lFx[4][k] = lpR; a.lthx[k] = lth;
    lM = 0; lN = 0; lT = 0; lpL = 0; lpR = 0; lth = 0;
    if (yface_on(g, i, j)) {
      const int kL = k, kR = k + g.W;
      const double M = it.fy[0][k], N = it.fy[1][k], T = it.fy[2][k], pL = it.fy[3][k], pR = it.fy[4][k];
      const double th = M >= 0 ? theta[kL] : theta[kR];
      const double invL = th / g.dyRowN[j], invR = th / g.dyRowS[j + 1];
      // rh[kL] -= M invL; rhv[kL] -= (N + pL) invL; rhu[kL] -= T invL; rh[kR] += M invR; ...
      lM = invR * a.lR[0][kR] - invL * a.lR[0][kL];
      lN = invR * a.lR[2][kR] - invL * a.lR[2][kL];
      lT = invR * a.lR[1][kR] - invL * a.lR[1][kL];
      lpL = -invL * a.lR[2][kL];
      lpR = invR * a.lR[2][kR];
      const double linvL = -(M * a.lR[0][kL] + (N + pL) * a.lR[2][kL] + T * a.lR[1][kL]);
      const double linvR = M * a.lR[0][kR] + (N + pR) * a.lR[2][kR] + T * a.lR[1][kR];
      lth = linvL / g.dyRowN[j] + linvR / g.dyRowS[j + 1];
    }
    a.lFy[0][k] = lM; a.lFy[1][k] = lN; a.lFy[2][k] = lT; a.lFy[3][k] = lpL; a.lFy[4][k] = lpR; a.lthy[k] = lth;
  }
}

// Positivity limiter (src/swe.mjs:511-529) backwards: theta's adjoint is
// gathered from the faces this cell is upwind of.
__global__ void k_adj_theta(Geo g, Inter it, const double* h, double dt, AdjBuf a) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < g.W * g.H; k += gridDim.x * blockDim.x) {
    const int i = k % g.W, j = k / g.W;
    double lout = 0, lh = 0;
    if (dt > 0 && i >= 1 && i < g.W - 1 && j >= 1 && j < g.H - 1) {
      double lth = 0;
      if (it.fx[0][k] >= 0) lth += a.lthx[k];              // east face, upwind = k
      if (it.fx[0][k - 1] < 0) lth += a.lthx[k - 1];       // west face
      if (it.fy[0][k] >= 0) lth += a.lthy[k];              // north face
      if (it.fy[0][k - g.W] < 0) lth += a.lthy[k - g.W];   // south face
      double out = 0;
      if (it.fx[0][k] > 0) out += it.fx[0][k] / g.dxRow[j];
      if (it.fx[0][k - 1] < 0) out -= it.fx[0][k - 1] / g.dxRow[j];
      if (it.fy[0][k] > 0) out += it.fy[0][k] / g.dyRowN[j];
      if (it.fy[0][k - g.W] < 0) out -= it.fy[0][k - g.W] / g.dyRowS[j];
      const double avail = h[k];
      if (out * dt > avail && avail > 0) {                 // theta = avail / (out dt)
        lh = lth / (out * dt);
        lout = -lth * avail / (out * out * dt);
      }
    }
    a.lout[k] = lout;
    a.lhth[k] = lh;
  }
}

// The faces backwards: limiter terms into the flux adjoint, then
// face_flux's reverse.
__global__ void k_adj_faces_core(Geo g, const double* b, const double* h, Inter it, AdjBuf a) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < g.W * g.H; k += gridDim.x * blockDim.x) {
    const int i = k % g.W, j = k / g.W;
    FaceIn gx = {}, gy = {};
    if (xface_on(g, i, j)) {
      double lM = a.lFx[0][k];
      const double M = it.fx[0][k];
      if (M > 0) lM += a.lout[k] / g.dxRow[j];
      if (M < 0) lM -= a.lout[k + 1] / g.dxRow[j];
      gx = swe::adj::face_rev(xface_in(g, b, h, it, k), g.minDepth, lM, a.lFx[1][k], a.lFx[2][k],
                              a.lFx[3][k], a.lFx[4][k]);
    }
    if (yface_on(g, i, j)) {
      double lM = a.lFy[0][k];
      const double M = it.fy[0][k];
      if (M > 0) lM += a.lout[k] / g.dyRowN[j];
      if (M < 0) lM -= a.lout[k + g.W] / g.dyRowS[j + 1];
      gy = swe::adj::face_rev(yface_in(g, b, h, it, k), g.minDepth, lM, a.lFy[1][k], a.lFy[2][k],
                              a.lFy[3][k], a.lFy[4][k]);
    }
    const double* px = &gx.bL;
    const double* py = &gy.bL;
    for (int q = 0; q < 16; q++) { a.gx[q][k] = px[q]; a.gy[q][k] = py[q]; }
  }
}

enum { F_BL, F_HL, F_NL, F_TL, F_SEL, F_SBL, F_SNL, F_STL, F_BR, F_HR, F_NR, F_TR, F_SER, F_SBR, F_SNR, F_STR };

// Per cell: gather the faces' adjoints, add the bed term and Coriolis
// backwards, then the limiter derivatives of each slope.
__global__ void k_adj_cells(Geo g, const double* b, const double* h, const double* hu, const double* hv,
                            Inter it, AdjBuf a, double* lhu, double* lhv) {
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
    dh += a.lhth[k];
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
// each ghost's adjoint moves to its source; one thread walks the ghosts in a
// fixed order so the sums are deterministic.
__global__ void k_adj_bc(int nx, int ny, double* lb, double* lh, double* lhu, double* lhv) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int W = nx + 4;
  auto clampi = [](int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); };
  auto move = [&](int gi, int gj, int si, int sj, double shu, double shv) {
    const int gk = (gj + 2) * W + (gi + 2), sk = (sj + 2) * W + (si + 2);
    if (lb) { lb[sk] += lb[gk]; lb[gk] = 0; }
    if (lh) {
      lh[sk] += lh[gk]; lh[gk] = 0;
      lhu[sk] += shu * lhu[gk]; lhu[gk] = 0;
      lhv[sk] += shv * lhv[gk]; lhv[gk] = 0;
    }
  };
  for (int i = -2; i < nx + 2; i++)                 // S/N rows (final values of the corners too)
    for (int gg = 0; gg < 2; gg++) {
      const int jS = -1 - gg, jN = ny + gg;
      move(i, jS, clampi(i, 0, nx - 1), clampi(-1 - jS, 0, ny - 1), 1, -1);
      move(i, jN, clampi(i, 0, nx - 1), clampi(2 * ny - 1 - jN, 0, ny - 1), 1, -1);
    }
  for (int j = 0; j < ny; j++)                      // W/E columns of the interior rows
    for (int gg = 0; gg < 2; gg++) {
      const int iW = -1 - gg, iE = nx + gg;
      move(iW, j, clampi(-1 - iW, 0, nx - 1), j, -1, 1);
      move(iE, j, clampi(2 * nx - 1 - iE, 0, nx - 1), j, -1, 1);
    }
}

// Stage outputs recomputed for their masks.
__global__ void k_stage1_pre(int N, const double* h, const double* hu, const double* hv, const double* rh,
                             const double* rhu, const double* rhv, double dt, double* oh, double* ohu, double* ohv) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    oh[k] = h[k] + dt * rh[k]; ohu[k] = hu[k] + dt * rhu[k]; ohv[k] = hv[k] + dt * rhv[k];
  }
}
__global__ void k_stage2_pre(int N, const double* h0, const double* hu0, const double* hv0, const double* h,
                             const double* hu, const double* hv, const double* rh, const double* rhu,
                             const double* rhv, double dt, double* oh, double* ohu, double* ohv) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    oh[k] = 0.5 * (h0[k] + h[k] + dt * rh[k]);
    ohu[k] = 0.5 * (hu0[k] + hu[k] + dt * rhu[k]);
    ohv[k] = 0.5 * (hv0[k] + hv[k] + dt * rhv[k]);
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
__global__ void k_misfit(const double* b, const double* h, const int* gk, const double* obs, int ng,
                         double* J, double* eta_out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = *J;
  for (int q = 0; q < ng; q++) {
    const double e = b[gk[q]] + h[gk[q]];
    if (eta_out) eta_out[q] = e;
    if (obs) { const double r = e - obs[q]; s += r * r; }
  }
  *J = s;
}
__global__ void k_adj_misfit(const double* b, const double* h, const int* gk, const double* obs, int ng,
                             double* lb, double* lh) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int q = 0; q < ng; q++) {
    const double r = b[gk[q]] + h[gk[q]] - obs[q];
    lh[gk[q]] += 2 * r;
    lb[gk[q]] += 2 * r;
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
__global__ void k_clean_interior(int W, int H, double minDepth, const double* h, const double* hu, const double* hv,
                                 double* oh, double* ohu, double* ohv) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < W * H; k += gridDim.x * blockDim.x) {
    const int i = k % W, j = k / W;
    double nh = h[k], nhu = hu[k], nhv = hv[k];
    if (i >= 2 && i < W - 2 && j >= 2 && j < H - 2) {
      if (nh < 0) nh = 0;
      if (nh <= minDepth) { nhu = 0; nhv = 0; }
    }
    oh[k] = nh; ohu[k] = nhu; ohv[k] = nhv;
  }
}
__global__ void k_axpy(int N, double a, const double* x, double* y) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) y[k] += a * x[k];
}
__global__ void k_scale(int N, double a, const double* x, double* y) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) y[k] = a * x[k];
}

}  // namespace

struct swe_adjoint {
  swe_options o;
  int W, H, N, steps, every, nseg, ng;
  double eps4;
  cudaStream_t st = nullptr;
  std::vector<double*> allocs;
  double *b, *eta0, *nfield = nullptr, *geom;
  double *A[3], *Bf[3], *W1[3], *Bp[3], *Ap[3], *Adc[3];  // state, stage buffers
  double *R[4];                                           // rh rhu rhv theta
  double *ckpt, *seg;                                     // checkpoints, one segment of states
  double *dts, *obs = nullptr, *J, *eta_series = nullptr;
  int* gk;
  double *lA[3], *lB[3], *lb, *ln;
  Inter it;
  AdjBuf ab;
  double *part;
  Control* ctl;
  int nblocks;
  dim3 grid;
  bool forward_done = false;
  bool fixed_dt = false;         // forward uses the given dt sequence instead of maxDt()
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
  a.part_max = s->part; a.part_fl1 = s->part + s->nblocks; a.part_fl2 = s->part + 2 * s->nblocks;
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
  swe::k_stage<1><<<s->grid, swe::BX, swe::STAGE_SMEM_BYTES, s->st>>>(stage_args(s, X, s->Bf), s->ctl);
  swe::k_apply_bc<<<bcb(s), 256, 0, s->st>>>(bc_args(s, s->Bf), s->ctl, 0);
  swe::k_stage<2><<<s->grid, swe::BX, swe::STAGE_SMEM_BYTES, s->st>>>(stage_args(s, s->Bf, X), s->ctl);
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
int residual_adjoint(swe_adjoint* s, double* const* X, const double* theta, double dt, double* const* lX) {
  const Geo g = geo_of(s);
  const int gb = G1(s);
  k_vel<<<gb, 256, 0, s->st>>>(g, X[0], X[1], X[2], s->it.U, s->it.V);
  k_slopes<<<gb, 256, 0, s->st>>>(g, s->b, X[0], s->it);
  k_faces<<<gb, 256, 0, s->st>>>(g, s->b, X[0], s->it);
  k_adj_faces_accum<<<gb, 256, 0, s->st>>>(g, s->it, theta, s->ab);
  k_adj_theta<<<gb, 256, 0, s->st>>>(g, s->it, X[0], dt, s->ab);
  k_adj_faces_core<<<gb, 256, 0, s->st>>>(g, s->b, X[0], s->it, s->ab);
  k_adj_cells<<<gb, 256, 0, s->st>>>(g, s->b, X[0], X[1], X[2], s->it, s->ab, lX[1], lX[2]);
  k_adj_cells_final<<<gb, 256, 0, s->st>>>(g, X[0], X[1], X[2], s->it, s->ab, s->lb, lX[0], lX[1], lX[2]);
  CU(cudaGetLastError());
  return SWE_OK;
}

// Reverse one step: on entry lA holds the adjoint of the step's output
// (interior), on exit the adjoint of its input state X0 (interior); lb and
// ln accumulate.
int step_adjoint(swe_adjoint* s, double* const* X0, int sidx) {
  const int N = s->N, gb = G1(s);
  double* lA[3] = {s->lA[0], s->lA[1], s->lA[2]};
  double* lB[3] = {s->lB[0], s->lB[1], s->lB[2]};
  double dt_h;
  CU(cudaMemcpyAsync(&dt_h, s->dts + sidx, sizeof(double), cudaMemcpyDeviceToHost, s->st));
  CU(cudaStreamSynchronize(s->st));
  const double dt = dt_h;
  k_set_dt<<<1, 32, 0, s->st>>>(s->ctl, s->dts, sidx);
  // recompute: W1 = BC(X0); R1; B pre/post clean; Bp = BC(B); R2; A pre/post clean
  copy3(s, s->W1, X0);
  swe::k_apply_bc<<<bcb(s), 256, 0, s->st>>>(bc_args(s, s->W1), s->ctl, 0);
  StageArgs r1 = stage_args(s, s->W1, nullptr);
  r1.rh = s->R[0]; r1.rhu = s->R[1]; r1.rhv = s->R[2]; r1.theta = s->R[3];
  swe::k_stage<0><<<s->grid, swe::BX, swe::STAGE_SMEM_BYTES, s->st>>>(r1, s->ctl);
  k_stage1_pre<<<gb, 256, 0, s->st>>>(N, s->W1[0], s->W1[1], s->W1[2], s->R[0], s->R[1], s->R[2], dt,
                                      s->Ap[0], s->Ap[1], s->Ap[2]);            // Ap = B before dryClean
  // stage-1 output after dryClean = the fused kernel's B
  swe::k_stage<1><<<s->grid, swe::BX, swe::STAGE_SMEM_BYTES, s->st>>>(stage_args(s, s->W1, s->Bf), s->ctl);
  copy3(s, s->Bp, s->Bf);
  swe::k_apply_bc<<<bcb(s), 256, 0, s->st>>>(bc_args(s, s->Bp), s->ctl, 0);
  // B before clean is needed for the stage-1 mask: keep it in Adc for now
  copy3(s, s->Adc, s->Ap);
  StageArgs r2 = stage_args(s, s->Bp, nullptr);
  r2.rh = s->R[0]; r2.rhu = s->R[1]; r2.rhv = s->R[2]; r2.theta = s->R[3];
  swe::k_stage<0><<<s->grid, swe::BX, swe::STAGE_SMEM_BYTES, s->st>>>(r2, s->ctl);
  k_stage2_pre<<<gb, 256, 0, s->st>>>(N, s->W1[0], s->W1[1], s->W1[2], s->Bp[0], s->Bp[1], s->Bp[2],
                                      s->R[0], s->R[1], s->R[2], dt, s->Ap[0], s->Ap[1], s->Ap[2]);
  // post-clean stage-2 state (friction's input): the fused kernel without friction
  // is not exposed, so clean Ap's copy here exactly as dryClean does
  CU(cudaGetLastError());
  {
    // Bf <- Ap cleaned (Bf is free now: stage 2's input lives in Bp)
    k_clean_interior<<<gb, 256, 0, s->st>>>(s->W, s->H, s->o.min_depth, s->Ap[0], s->Ap[1], s->Ap[2],
                                            s->Bf[0], s->Bf[1], s->Bf[2]);
  }
  // ---- reverse ----
  k_adj_friction<<<gb, 256, 0, s->st>>>(s->W, s->H, s->o.min_depth, s->eps4, s->o.manning, s->nfield, dt,
                                        s->Bf[0], s->Bf[1], s->Bf[2], lA[0], lA[1], lA[2], s->ln);
  k_adj_dryclean<<<gb, 256, 0, s->st>>>(s->W, s->H, s->o.min_depth, s->Ap[0], lA[0], lA[1], lA[2]);
  // A = 0.5 (W1 + Bp + dt R2): lW1 = lB = 0.5 lA, lR2 = 0.5 dt lA
  for (int q = 0; q < 3; q++) {
    k_scale<<<gb, 256, 0, s->st>>>(N, 0.5, lA[q], lB[q]);
    k_scale<<<gb, 256, 0, s->st>>>(N, 0.5 * dt, lA[q], s->ab.lR[q]);
    k_scale<<<gb, 256, 0, s->st>>>(N, 0.5, lA[q], lA[q]);       // lA now holds lW1
  }
  int rc = residual_adjoint(s, s->Bp, s->R[3], dt, lB);
  if (rc) return rc;
  k_adj_bc<<<1, 32, 0, s->st>>>(s->o.nx, s->o.ny, s->lb, lB[0], lB[1], lB[2]);
  // stage-1 dryClean backwards (mask from B before clean, kept in Adc)
  k_adj_dryclean<<<gb, 256, 0, s->st>>>(s->W, s->H, s->o.min_depth, s->Adc[0], lB[0], lB[1], lB[2]);
  // B = W1 + dt R1 (all cells): lW1 += lB, lR1 = dt lB
  StageArgs r1b = r1;
  swe::k_stage<0><<<s->grid, swe::BX, swe::STAGE_SMEM_BYTES, s->st>>>(r1b, s->ctl);   // theta of stage 1
  for (int q = 0; q < 3; q++) {
    k_axpy<<<gb, 256, 0, s->st>>>(N, 1.0, lB[q], lA[q]);
    k_scale<<<gb, 256, 0, s->st>>>(N, dt, lB[q], s->ab.lR[q]);
  }
  rc = residual_adjoint(s, s->W1, s->R[3], dt, lA);
  if (rc) return rc;
  k_adj_bc<<<1, 32, 0, s->st>>>(s->o.nx, s->o.ny, s->lb, lA[0], lA[1], lA[2]);
  CU(cudaGetLastError());
  return SWE_OK;
}

void free_adj(swe_adjoint* s) {
  for (double* p : s->allocs) cudaFree(p);
  if (s->gk) cudaFree(s->gk);
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
    s->A[q] = A(N); s->Bf[q] = A(N); s->W1[q] = A(N); s->Bp[q] = A(N); s->Ap[q] = A(N); s->Adc[q] = A(N);
    s->lA[q] = A(N); s->lB[q] = A(N);
  }
  for (int q = 0; q < 4; q++) s->R[q] = A(N);
  s->ckpt = A(3 * N * (size_t)s->nseg);
  s->seg = A(3 * N * (size_t)(checkpoint_every + 1));
  s->dts = A(steps);
  s->obs = A((size_t)steps * n_gauges);
  s->eta_series = A((size_t)steps * n_gauges);
  s->J = A(1);
  s->lb = A(N); s->ln = A(N);
  s->it.U = A(N); s->it.V = A(N);
  for (int q = 0; q < 8; q++) s->it.s[q] = A(N);
  for (int q = 0; q < 5; q++) { s->it.fx[q] = A(N); s->it.fy[q] = A(N); s->ab.lFx[q] = A(N); s->ab.lFy[q] = A(N); }
  for (int q = 0; q < 3; q++) s->ab.lR[q] = A(N);
  s->ab.lthx = A(N); s->ab.lthy = A(N); s->ab.lout = A(N); s->ab.lhth = A(N);
  for (int q = 0; q < 16; q++) { s->ab.gx[q] = A(N); s->ab.gy[q] = A(N); s->ab.gs[q] = A(N); }
  for (int q = 0; q < 4; q++) s->ab.dir[q] = A(N);
  const int gx = (s->W + swe::SX - 1) / swe::SX, gy = (s->H + 31) / 32;
  s->grid = dim3(gx, gy);
  s->nblocks = gx * gy;
  s->part = A(3 * (size_t)std::max(s->nblocks, 1024));
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
    k_misfit<<<1, 32, 0, s->st>>>(s->b, s->A[0], s->gk, s->obs + (size_t)k * s->ng, s->ng, s->J,
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
  auto slot = [&](int i) {
    double* p = s->seg + (size_t)i * 3 * N;
    return std::vector<double*>{p, p + N, p + 2 * N};
  };
  for (int sg = s->nseg - 1; sg >= 0; sg--) {
    const int k0 = sg * s->every, k1 = std::min(s->steps, k0 + s->every);
    // states A_k0 .. A_k1 of this segment
    {
      auto d0 = slot(0);
      double* src[3] = {s->ckpt + (size_t)sg * 3 * N, s->ckpt + ((size_t)sg * 3 + 1) * N, s->ckpt + ((size_t)sg * 3 + 2) * N};
      copy3(s, d0.data(), src);
    }
    for (int k = k0; k < k1; k++) {
      auto cur = slot(k - k0), nxt = slot(k - k0 + 1);
      copy3(s, nxt.data(), cur.data());
      int rc = fwd_step(s, nxt.data(), false, k);
      if (rc) return rc;
    }
    for (int k = k1 - 1; k >= k0; k--) {
      auto outp = slot(k - k0 + 1), inp = slot(k - k0);
      k_adj_misfit<<<1, 32, 0, s->st>>>(s->b, outp[0], s->gk, s->obs + (size_t)k * s->ng, s->ng, s->lb, s->lA[0]);
      int rc = step_adjoint(s, inp.data(), k);
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
