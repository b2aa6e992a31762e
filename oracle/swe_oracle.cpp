// swe_oracle.cpp -- CPU FP64 restatement of the reference shallow-water solver.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA library, never part of it.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU legs load this.
//
// Every function below cites the reference lines (Syntaxswine/water-simulator)
// whose arithmetic it restates.  Loop bounds, loop order, the order of the
// operands inside each expression, the zero-fill of the scratch arrays and
// the ghost-cell handling follow the reference, so that with
// -ffp-contract=off this produces the same doubles the JavaScript solver does
// (IEEE + - * / sqrt are correctly rounded in both).  The only library
// functions whose last bit is not pinned are pow (friction, src/swe.mjs:683,699),
// hypot (src/swe.mjs:681,697,904) and sin/cos/tan (metric and tide set-up):
// glibc here, V8's fdlibm port there.
//
// x ** 2 in hllc (src/swe.mjs:992) is written x * x (correctly rounded square).
//
// Threads: with threads == 1 every loop is the reference loop.  With
// threads > 1 (the CPU baseline arm) independent per-cell loops run under
// OpenMP and the two flux-accumulation scatter loops are run as a per-cell
// gather that applies the same additions to each cell in the same order,
// which gives bit-identical results (checked by a test).
#include "swe_oracle.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const double G = 9.80665;                       // src/swe.mjs:85
const double SQRT2 = 1.4142135623730951;        // Math.SQRT2
const double PI = 3.141592653589793;            // Math.PI
const double HALF_PI = PI / 2;                  // src/geometry.mjs:110
const double INF = INFINITY;

thread_local std::string g_err;

// A dual number: a value and its derivative along one direction.  Running
// the solver on Duals is its tangent-linear model; every comparison looks at
// the value only, so every branch is the branch the value takes.
struct Dual {
  double v, d;
  Dual(double x = 0) : v(x), d(0) {}
  Dual(double x, double dx) : v(x), d(dx) {}
};
inline Dual operator+(const Dual& a, const Dual& b) { return {a.v + b.v, a.d + b.d}; }
inline Dual operator-(const Dual& a, const Dual& b) { return {a.v - b.v, a.d - b.d}; }
inline Dual operator*(const Dual& a, const Dual& b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dual operator/(const Dual& a, const Dual& b) {
  const double q = a.v / b.v;
  return {q, (a.d - q * b.d) / b.v};
}
inline Dual operator-(const Dual& a) { return {-a.v, -a.d}; }
inline Dual operator+(const Dual& a, double b) { return {a.v + b, a.d}; }
inline Dual operator+(double a, const Dual& b) { return {a + b.v, b.d}; }
inline Dual operator-(const Dual& a, double b) { return {a.v - b, a.d}; }
inline Dual operator-(double a, const Dual& b) { return {a - b.v, -b.d}; }
inline Dual operator*(const Dual& a, double b) { return {a.v * b, a.d * b}; }
inline Dual operator*(double a, const Dual& b) { return {a * b.v, a * b.d}; }
inline Dual operator/(const Dual& a, double b) { return {a.v / b, a.d / b}; }
inline Dual operator/(double a, const Dual& b) { const double q = a / b.v; return {q, -q * b.d / b.v}; }
inline Dual& operator+=(Dual& a, const Dual& b) { a = a + b; return a; }
inline Dual& operator-=(Dual& a, const Dual& b) { a = a - b; return a; }
inline Dual& operator/=(Dual& a, const Dual& b) { a = a / b; return a; }
#define DUAL_CMP(op)                                                                 \
  inline bool operator op(const Dual& a, const Dual& b) { return a.v op b.v; }       \
  inline bool operator op(const Dual& a, double b) { return a.v op b; }              \
  inline bool operator op(double a, const Dual& b) { return a op b.v; }
DUAL_CMP(<) DUAL_CMP(>) DUAL_CMP(<=) DUAL_CMP(>=) DUAL_CMP(==) DUAL_CMP(!=)
#undef DUAL_CMP
inline double value(double x) { return x; }
inline double value(const Dual& x) { return x.v; }
inline double sqrtT(double x) { return std::sqrt(x); }
inline Dual sqrtT(const Dual& x) { const double r = std::sqrt(x.v); return {r, x.d == 0 ? 0 : x.d / (2 * r)}; }
inline double fabsT(double x) { return std::fabs(x); }
inline Dual fabsT(const Dual& x) { return std::signbit(x.v) ? -x : x; }
inline double hypotT(double a, double b) { return std::hypot(a, b); }
inline Dual hypotT(const Dual& a, const Dual& b) {
  const double r = std::hypot(a.v, b.v);
  return {r, r == 0 ? 0 : (a.v * a.d + b.v * b.d) / r};
}
inline double powT(double x, double p) { return std::pow(x, p); }
inline Dual powT(const Dual& x, double p) {
  const double r = std::pow(x.v, p);
  return {r, x.d == 0 ? 0 : p * std::pow(x.v, p - 1) * x.d};
}
inline bool isfiniteT(double x) { return std::isfinite(x); }
inline bool isfiniteT(const Dual& x) { return std::isfinite(x.v); }

// JavaScript Math.max / Math.min semantics: NaN if any operand is NaN, and
// +0 > -0.  (C fmax/fmin drop NaN operands, which would hide a blow-up.)
template <class T> inline T jmaxT(const T& a, const T& b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a > b) return a;
  if (b > a) return b;
  return std::signbit(value(a)) ? b : a;
}
template <class T> inline T jminT(const T& a, const T& b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a < b) return a;
  if (b < a) return b;
  return std::signbit(value(a)) ? a : b;
}
inline double jmax(double a, double b) { return jmaxT<double>(a, b); }
inline Dual jmax(const Dual& a, const Dual& b) { return jmaxT<Dual>(a, b); }
inline double jmin(double a, double b) { return jminT<double>(a, b); }
inline Dual jmin(const Dual& a, const Dual& b) { return jminT<Dual>(a, b); }

// src/swe.mjs:88-92
template <class T> inline T lim_minmod(const T& a, const T& b) {
  if (a > 0 && b > 0) return a < b ? a : b;
  if (a < 0 && b < 0) return a > b ? a : b;
  return T(0);
}
// src/swe.mjs:133-138
template <class T> inline T lim_mc(const T& a, const T& b) {
  if (a * b <= 0) return T(0);
  const T c = 0.5 * (a + b);
  const T m = jmin(jmin(fabsT(c), 2 * fabsT(a)), 2 * fabsT(b));
  return a > 0 ? m : -m;
}
// src/swe.mjs:141
template <class T> inline T lim_central(const T& a, const T& b) { return 0.5 * (a + b); }

// src/swe.mjs:1013-1018
template <class T> inline void flux1D(T* out, const T& h, const T& hu, const T& hv, const T& u) {
  out[0] = hu;
  out[1] = hu * u + 0.5 * G * h * h;
  out[2] = hv * u;
}

// src/swe.mjs:975-1011
template <class T>
void hllc(T* out, T hL, T huL, T hvL, T hR, T huR, T hvR, double dry) {
  const bool wetL = hL > dry, wetR = hR > dry;
  if (!wetL && !wetR) { out[0] = out[1] = out[2] = T(0); return; }
  const T uL = wetL ? huL / hL : T(0), vL = wetL ? hvL / hL : T(0);
  const T uR = wetR ? huR / hR : T(0), vR = wetR ? hvR / hR : T(0);
  const T cL = sqrtT(G * jmax(hL, T(0))), cR = sqrtT(G * jmax(hR, T(0)));
  T sL, sR;
  if (!wetL) { sL = uR - 2 * cR; sR = uR + cR; }
  else if (!wetR) { sL = uL - cL; sR = uL + 2 * cL; }
  else {
    const T a = (cL + cR) / 2 + (uL - uR) / 4;
    const T hStar = a * a / G;
    const T qL = hStar > hL ? sqrtT(0.5 * (hStar + hL) * hStar / (hL * hL)) : T(1);
    const T qR = hStar > hR ? sqrtT(0.5 * (hStar + hR) * hStar / (hR * hR)) : T(1);
    sL = uL - cL * qL;
    sR = uR + cR * qR;
  }
  if (sL >= 0) { flux1D(out, hL, huL, hvL, uL); return; }
  if (sR <= 0) { flux1D(out, hR, huR, hvR, uR); return; }
  const T num = sL * hR * (uR - sR) - sR * hL * (uL - sL);
  const T den = hR * (uR - sR) - hL * (uL - sL);
  const T sM = fabsT(den) > 1e-30 ? num / den : 0.5 * (sL + sR);
  T FL[3], FR[3];
  flux1D(FL, hL, huL, hvL, uL);
  flux1D(FR, hR, huR, hvR, uR);
  const T inv = 1 / (sR - sL);
  out[0] = (sR * FL[0] - sL * FR[0] + sL * sR * (hR - hL)) * inv;
  out[1] = (sR * FL[1] - sL * FR[1] + sL * sR * (huR - huL)) * inv;
  out[2] = out[0] * (sM >= 0 ? vL : vR);
}

// src/geometry.mjs:111-112
inline double clampLat(double p) { return p > HALF_PI ? HALF_PI : p < -HALF_PI ? -HALF_PI : p; }
inline double reflectLat(double p) { return p > HALF_PI ? PI - p : p < -HALF_PI ? -PI - p : p; }
// src/geometry.mjs:153-156
inline double cosLat(double p) {
  const double co = HALF_PI - std::fabs(p);
  return co <= 0 ? 0 : std::sin(co);
}

struct Tide {                 // src/tide.mjs:103-107 as a table
  double msl = 0, u_coef = 0;
  std::vector<double> amp, omega, phase;
  double eta(double t) const {
    double e = msl;
    for (size_t k = 0; k < amp.size(); k++) e += amp[k] * std::cos(omega[k] * t - phase[k] * PI / 180);
    return e;
  }
};

}  // namespace

template <class T>
struct SimT {
  int nx, ny, ng, W, H, N;
  double dx, dy, manning, minDepth, cfl, coriolis, eps4;
  int order, limiter, sphere;
  // metric
  std::vector<double> g[OG_NROWS];
  double R, dlam, dphi, totalArea, lat0, lat1, omega;
  // state and scratch, src/swe.mjs:200-220
  std::vector<T> b, h, hu, hv, h0, hu0, hv0, rh, rhu, rhv, sE, sU, sV, sB;
  std::vector<T> fxM, fxN, fxT, fyM, fyN, fyT, pxL, pxR, pyL, pyR, theta, uu, vv;
  std::vector<T> manningField;
  bool hasManning = false;
  int bc[4] = {OB_REFLECT, OB_REFLECT, OB_REFLECT, OB_REFLECT};
  double flEta[4] = {0, 0, 0, 0}, flU[4] = {0, 0, 0, 0};
  bool flTide[4] = {false, false, false, false};
  Tide tide[4];
  // sponge, src/swe.mjs:1174-1198
  bool hasSponge = false;
  double spongeRef = 0;
  std::vector<std::pair<int, double>> spongeCells;
  double t = 0, steps = 0;
  T massFloored = 0;
  int threads = 1;

  int idx(int i, int j) const { return (j + ng) * W + (i + ng); }

  // src/swe.mjs:282-285
  T vel(T hq, T hh) const {
    const T h4 = hh * hh * hh * hh;
    return (SQRT2 * hh * hq) / sqrtT(h4 + jmax(h4, eps4));
  }
  T limit(T a, T c) const {
    return limiter == 0 ? lim_mc(a, c) : limiter == 1 ? lim_minmod(a, c) : lim_central(a, c);
  }

  // ---- boundaries, src/swe.mjs:1026-1126 --------------------------------
  void bcReflect(int i, int j, int side) {
    int si = i, sj = j;
    if (side == 0) si = -1 - i; else if (side == 1) si = 2 * nx - 1 - i;
    else if (side == 2) sj = -1 - j; else sj = 2 * ny - 1 - j;
    si = std::max(0, std::min(nx - 1, si));
    sj = std::max(0, std::min(ny - 1, sj));
    const int gk = idx(i, j), s = idx(si, sj);
    b[gk] = b[s];
    h[gk] = h[s];
    const bool flipX = side == 0 || side == 1;
    hu[gk] = flipX ? -hu[s] : hu[s];
    hv[gk] = flipX ? hv[s] : -hv[s];
  }
  void bcOutflow(int i, int j) {
    const int si = std::max(0, std::min(nx - 1, i));
    const int sj = std::max(0, std::min(ny - 1, j));
    const int gk = idx(i, j), s = idx(si, sj);
    b[gk] = b[s]; h[gk] = h[s]; hu[gk] = hu[s]; hv[gk] = hv[s];
  }
  void bcFlather(int i, int j, int side) {
    const int si = std::max(0, std::min(nx - 1, i));
    const int sj = std::max(0, std::min(ny - 1, j));
    const int gk = idx(i, j), s = idx(si, sj);
    b[gk] = b[s];
    const T bed = b[gk];
    const T hInt = h[s];
    double e0, u0;
    if (flTide[side]) { e0 = tide[side].eta(t); u0 = tide[side].u_coef * tide[side].eta(t); }
    else { e0 = flEta[side]; u0 = flU[side]; }
    if (hInt <= minDepth) { h[gk] = jmax(0, e0 - bed); hu[gk] = 0; hv[gk] = 0; return; }
    const T etaInt = bed + hInt;
    const T r = sqrtT(G / hInt);
    const double sgn = (side == 0 || side == 2) ? 1 : -1;
    const T uInt = (side == 0 || side == 1) ? vel(hu[s], hInt) : vel(hv[s], hInt);
    const T Rin = u0 + sgn * e0 * r;
    const T Rout = uInt - sgn * etaInt * r;
    const T un = 0.5 * (Rin + Rout);
    const T en = sgn * (Rin - Rout) / (2 * r);
    h[gk] = jmax(0, en - bed);
    if (side == 0 || side == 1) { hu[gk] = h[gk] * un; hv[gk] = hv[s]; }
    else { hv[gk] = h[gk] * un; hu[gk] = hu[s]; }
  }
  void bcPeriodic(int i, int j, int side) {
    int si = i, sj = j;
    if (side == 0) si = i + nx; else if (side == 1) si = i - nx;
    else if (side == 2) sj = j + ny; else sj = j - ny;
    const int gk = idx(i, j), s = idx(si, sj);
    b[gk] = b[s]; h[gk] = h[s]; hu[gk] = hu[s]; hv[gk] = hv[s];
  }
  void bcCall(int side, int i, int j) {
    switch (bc[side]) {
      case OB_REFLECT: bcReflect(i, j, side); break;
      case OB_OUTFLOW: bcOutflow(i, j); break;
      case OB_PERIODIC: bcPeriodic(i, j, side); break;
      default: bcFlather(i, j, side); break;
    }
  }
  // src/swe.mjs:289-303
  void applyBC() {
    for (int j = 0; j < H; j++)
      for (int gg = 0; gg < ng; gg++) {
        bcCall(0, -1 - gg, j - ng);
        bcCall(1, nx + gg, j - ng);
      }
    for (int i = -ng; i < nx + ng; i++)
      for (int gg = 0; gg < ng; gg++) {
        bcCall(2, i, -1 - gg);
        bcCall(3, i, ny + gg);
      }
  }

  // ---- residual, src/swe.mjs:308-629 -------------------------------------
  void residual(double dt) {
    const std::vector<double>& dxRow = g[OG_DXROW];
    const std::vector<double>& dyRowN = g[OG_DYROWN];
    const std::vector<double>& dyRowS = g[OG_DYROWS];
    const std::vector<double>& bedPhi = g[OG_BEDPHI];
    const bool sph = sphere != 0;
    const int nthr = threads;
    std::fill(rh.begin(), rh.end(), 0.0);
    std::fill(rhu.begin(), rhu.end(), 0.0);
    std::fill(rhv.begin(), rhv.end(), 0.0);
    std::fill(fxM.begin(), fxM.end(), 0.0);
    std::fill(fyM.begin(), fyM.end(), 0.0);

    // cell velocities, src/swe.mjs:358-359
#pragma omp parallel for num_threads(nthr) if (nthr > 1) schedule(static)
    for (int k = 0; k < N; k++) { const T hk = h[k]; uu[k] = vel(hu[k], hk); vv[k] = vel(hv[k], hk); }
    const T* U = uu.data();
    const T* V = vv.data();

    // slopes, src/swe.mjs:362-411
    if (order >= 2) {
#pragma omp parallel for num_threads(nthr) if (nthr > 1) schedule(static)
      for (int j = 1; j < H - 1; j++) {
        for (int i = 1; i < W - 1; i++) {
          const int k = j * W + i, k2 = 2 * k;
          const T hk = h[k], bk = b[k], eC = bk + hk, uk = U[k], vk = V[k];
          for (int d = 0; d < 2; d++) {
            const int kp = d == 0 ? k + 1 : k + W;
            const int km = d == 0 ? k - 1 : k - W;
            if (hk <= minDepth || h[kp] <= minDepth || h[km] <= minDepth) {
              sE[k2 + d] = 0; sB[k2 + d] = 0; sU[k2 + d] = 0; sV[k2 + d] = 0;
              continue;
            }
            const T eP = b[kp] + h[kp], eM = b[km] + h[km];
            sE[k2 + d] = limit(eC - eM, eP - eC);
            sB[k2 + d] = limit(bk - b[km], b[kp] - bk);
            sU[k2 + d] = limit(uk - U[km], U[kp] - uk);
            sV[k2 + d] = limit(vk - V[km], V[kp] - vk);
          }
        }
      }
    } else {
      std::fill(sE.begin(), sE.end(), 0.0); std::fill(sU.begin(), sU.end(), 0.0);
      std::fill(sV.begin(), sV.end(), 0.0); std::fill(sB.begin(), sB.end(), 0.0);
    }

    // x interfaces, src/swe.mjs:414-445
#pragma omp parallel for num_threads(nthr) if (nthr > 1) schedule(static)
    for (int j = ng; j < H - ng; j++) {
      T flux[3];
      for (int i = ng - 1; i < W - ng; i++) {
        const int kL = j * W + i, kR = kL + 1, kL2 = 2 * kL, kR2 = 2 * kR;
        const T etaL = b[kL] + h[kL] + 0.5 * sE[kL2];
        const T etaR = b[kR] + h[kR] - 0.5 * sE[kR2];
        const T bL = b[kL] + 0.5 * sB[kL2];
        const T bR = b[kR] - 0.5 * sB[kR2];
        const T hLf = jmax(0, etaL - bL);
        const T hRf = jmax(0, etaR - bR);
        const T uL = U[kL] + 0.5 * sU[kL2];
        const T uR = U[kR] - 0.5 * sU[kR2];
        const T vL = V[kL] + 0.5 * sV[kL2];
        const T vR = V[kR] - 0.5 * sV[kR2];
        const T bStar = jmax(bL, bR);
        const T hsL = jmax(0, etaL - bStar);
        const T hsR = jmax(0, etaR - bStar);
        hllc(flux, hsL, hsL * uL, hsL * vL, hsR, hsR * uR, hsR * vR, minDepth);
        const T pL = 0.5 * G * (hLf * hLf - hsL * hsL);
        const T pR = 0.5 * G * (hRf * hRf - hsR * hsR);
        fxM[kL] = flux[0]; fxN[kL] = flux[1]; fxT[kL] = flux[2];
        pxL[kL] = pL; pxR[kL] = pR;
      }
    }

    // y interfaces, src/swe.mjs:447-475
#pragma omp parallel for num_threads(nthr) if (nthr > 1) schedule(static)
    for (int j = ng - 1; j < H - ng; j++) {
      T flux[3];
      for (int i = ng; i < W - ng; i++) {
        const int kL = j * W + i, kR = kL + W, kL2 = 2 * kL + 1, kR2 = 2 * kR + 1;
        const T etaL = b[kL] + h[kL] + 0.5 * sE[kL2];
        const T etaR = b[kR] + h[kR] - 0.5 * sE[kR2];
        const T bL = b[kL] + 0.5 * sB[kL2];
        const T bR = b[kR] - 0.5 * sB[kR2];
        const T hLf = jmax(0, etaL - bL);
        const T hRf = jmax(0, etaR - bR);
        const T uL = U[kL] + 0.5 * sU[kL2];
        const T uR = U[kR] - 0.5 * sU[kR2];
        const T vL = V[kL] + 0.5 * sV[kL2];
        const T vR = V[kR] - 0.5 * sV[kR2];
        const T bStar = jmax(bL, bR);
        const T hsL = jmax(0, etaL - bStar);
        const T hsR = jmax(0, etaR - bStar);
        hllc(flux, hsL, hsL * vL, hsL * uL, hsR, hsR * vR, hsR * uR, minDepth);
        const T pL = 0.5 * G * (hLf * hLf - hsL * hsL);
        const T pR = 0.5 * G * (hRf * hRf - hsR * hsR);
        fyM[kL] = flux[0]; fyN[kL] = flux[1]; fyT[kL] = flux[2];
        pyL[kL] = pL; pyR[kL] = pR;
      }
    }

    // positivity limiter, src/swe.mjs:511-529
    std::fill(theta.begin(), theta.end(), 1.0);
    if (dt > 0) {
#pragma omp parallel for num_threads(nthr) if (nthr > 1) schedule(static)
      for (int j = ng - 1; j < H - ng + 1; j++) {
        for (int i = ng - 1; i < W - ng + 1; i++) {
          const int k = j * W + i;
          T out = 0;
          if (fxM[k] > 0) out += fxM[k] / dxRow[j];
          if (fxM[k - 1] < 0) out -= fxM[k - 1] / dxRow[j];
          if (fyM[k] > 0) out += fyM[k] / dyRowN[j];
          if (fyM[k - W] < 0) out -= fyM[k - W] / dyRowS[j];
          const T avail = h[k];
          if (out * dt > avail) theta[k] = avail > 0 ? avail / (out * dt) : 0;
        }
      }
    }

    if (nthr <= 1) {
      // accumulate, src/swe.mjs:530-555, as the reference's scatter loops
      for (int j = ng; j < H - ng; j++) {
        for (int i = ng - 1; i < W - ng; i++) {
          const int kL = j * W + i, kR = kL + 1;
          const T th = fxM[kL] >= 0 ? theta[kL] : theta[kR];
          const T inv = th / dxRow[j];
          rh[kL] -= fxM[kL] * inv; rhu[kL] -= (fxN[kL] + pxL[kL]) * inv; rhv[kL] -= fxT[kL] * inv;
          rh[kR] += fxM[kL] * inv; rhu[kR] += (fxN[kL] + pxR[kL]) * inv; rhv[kR] += fxT[kL] * inv;
        }
      }
      for (int j = ng - 1; j < H - ng; j++) {
        for (int i = ng; i < W - ng; i++) {
          const int kL = j * W + i, kR = kL + W;
          const T th = fyM[kL] >= 0 ? theta[kL] : theta[kR];
          const T invL = th / dyRowN[j];
          const T invR = th / dyRowS[j + 1];
          rh[kL] -= fyM[kL] * invL; rhv[kL] -= (fyN[kL] + pyL[kL]) * invL; rhu[kL] -= fyT[kL] * invL;
          rh[kR] += fyM[kL] * invR; rhv[kR] += (fyN[kL] + pyR[kL]) * invR; rhu[kR] += fyT[kL] * invR;
        }
      }
    } else {
      // The same additions gathered per cell, in the order the scatter loops
      // apply them to that cell: west face, east face, south face, north face.
#pragma omp parallel for num_threads(nthr) schedule(static)
      for (int j = 0; j < H; j++) {
        for (int i = 0; i < W; i++) {
          const int k = j * W + i;
          T a = rh[k], au = rhu[k], av = rhv[k];
          const bool xrow = j >= ng && j < H - ng;
          if (xrow && i - 1 >= ng - 1 && i - 1 < W - ng) {
            const int kL = k - 1;
            const T th = fxM[kL] >= 0 ? theta[kL] : theta[k];
            const T inv = th / dxRow[j];
            a += fxM[kL] * inv; au += (fxN[kL] + pxR[kL]) * inv; av += fxT[kL] * inv;
          }
          if (xrow && i >= ng - 1 && i < W - ng) {
            const T th = fxM[k] >= 0 ? theta[k] : theta[k + 1];
            const T inv = th / dxRow[j];
            a -= fxM[k] * inv; au -= (fxN[k] + pxL[k]) * inv; av -= fxT[k] * inv;
          }
          const bool ycol = i >= ng && i < W - ng;
          if (ycol && j - 1 >= ng - 1 && j - 1 < H - ng) {
            const int kL = k - W;
            const T th = fyM[kL] >= 0 ? theta[kL] : theta[k];
            const T invR = th / dyRowS[j];
            a += fyM[kL] * invR; av += (fyN[kL] + pyR[kL]) * invR; au += fyT[kL] * invR;
          }
          if (ycol && j >= ng - 1 && j < H - ng) {
            const T th = fyM[k] >= 0 ? theta[k] : theta[k + W];
            const T invL = th / dyRowN[j];
            a -= fyM[k] * invL; av -= (fyN[k] + pyL[k]) * invL; au -= fyT[k] * invL;
          }
          rh[k] = a; rhu[k] = au; rhv[k] = av;
        }
      }
    }

    // centred bed term + spherical geometric source, src/swe.mjs:570-598
    if (order >= 2 || sph) {
      const std::vector<double>& geoCoef = g[OG_GEOCOEF];
#pragma omp parallel for num_threads(nthr) if (nthr > 1) schedule(static)
      for (int j = ng; j < H - ng; j++) {
        const double bedDiv1 = bedPhi[j], bedDiv0 = dxRow[j], gc = geoCoef[j];
        for (int i = ng; i < W - ng; i++) {
          const int k = j * W + i, k2 = 2 * k;
          const T bk = b[k];
          const T eC = bk + h[k];
          for (int d = 0; d < 2; d++) {
            const T hP = jmax(0, eC + 0.5 * sE[k2 + d] - (bk + 0.5 * sB[k2 + d]));
            const T hM = jmax(0, eC - 0.5 * sE[k2 + d] - (bk - 0.5 * sB[k2 + d]));
            const T db = sB[k2 + d];
            const T term = -G * 0.5 * (hP + hM) * db / (d == 0 ? bedDiv0 : bedDiv1);
            if (d == 0) rhu[k] += term;
            else {
              rhv[k] += term;
              if (sph) rhv[k] += gc * G * (hP * hP + hM * hM);
            }
          }
        }
      }
    }

    // Coriolis, src/swe.mjs:601-628
    if (sph) {
      const std::vector<double>& fRow = g[OG_FROW];
      const std::vector<double>& tanPhi = g[OG_TANPHI];
#pragma omp parallel for num_threads(nthr) if (nthr > 1) schedule(static)
      for (int j = ng; j < H - ng; j++) {
        const double f0 = fRow[j], tR = tanPhi[j] / R;
        for (int i = ng; i < W - ng; i++) {
          const int k = j * W + i;
          const T fe = f0 + U[k] * tR;
          rhu[k] += fe * hv[k];
          rhv[k] -= fe * hu[k];
        }
      }
    } else if (coriolis != 0 && coriolis == coriolis) {
      const double f = coriolis;
#pragma omp parallel for num_threads(nthr) if (nthr > 1) schedule(static)
      for (int j = ng; j < H - ng; j++) {
        for (int i = ng; i < W - ng; i++) {
          const int k = j * W + i;
          rhu[k] += f * hv[k];
          rhv[k] -= f * hu[k];
        }
      }
    }
  }

  // src/swe.mjs:632-647
  double maxDt() const {
    const std::vector<double>& dxRow = g[OG_DXROW];
    const std::vector<double>& dyCFL = g[OG_DYCFL];
    T inv = 0;
    for (int j = ng; j < H - ng; j++) {
      for (int i = ng; i < W - ng; i++) {
        const int k = j * W + i;
        const T hk = h[k];
        if (hk <= minDepth) continue;
        const T c = sqrtT(G * hk);
        const T u = fabsT(vel(hu[k], hk)), v = fabsT(vel(hv[k], hk));
        const T s = (u + c) / dxRow[j] + (v + c) / dyCFL[j];
        if (s > inv) inv = s;
      }
    }
    return inv > 0 ? cfl / value(inv) : INF;
  }

  // src/swe.mjs:659-704
  void applyFriction(double dt) {
    const double n = manning;
    const int nthr = threads;
    if (hasManning) {
      const T* nf = manningField.data();
#pragma omp parallel for num_threads(nthr) if (nthr > 1) schedule(static)
      for (int j = ng; j < H - ng; j++) {
        for (int i = ng; i < W - ng; i++) {
          const int k = j * W + i;
          const T hk = h[k];
          if (hk <= minDepth) { hu[k] = 0; hv[k] = 0; continue; }
          const T nk = nf[k];
          if (!(nk != 0 && nk == nk)) continue;
          const T u = vel(hu[k], hk), v = vel(hv[k], hk);
          const T speed = hypotT(u, v);
          if (speed < 1e-14) continue;
          const T denom = 1 + dt * G * nk * nk * speed / powT(hk, 4.0 / 3.0);
          hu[k] /= denom;
          hv[k] /= denom;
        }
      }
      return;
    }
    if (!(n != 0 && n == n)) return;
#pragma omp parallel for num_threads(nthr) if (nthr > 1) schedule(static)
    for (int j = ng; j < H - ng; j++) {
      for (int i = ng; i < W - ng; i++) {
        const int k = j * W + i;
        const T hk = h[k];
        if (hk <= minDepth) { hu[k] = 0; hv[k] = 0; continue; }
        const T u = vel(hu[k], hk), v = vel(hv[k], hk);
        const T speed = hypotT(u, v);
        if (speed < 1e-14) continue;
        const T denom = 1 + dt * G * n * n * speed / powT(hk, 4.0 / 3.0);
        hu[k] /= denom;
        hv[k] /= denom;
      }
    }
  }

  // src/swe.mjs:734-745
  T dryClean() {
    T added = 0;
    for (int j = ng; j < H - ng; j++) {
      for (int i = ng; i < W - ng; i++) {
        const int k = j * W + i;
        if (h[k] < 0) { added -= h[k]; h[k] = 0; }
        if (h[k] <= minDepth) { hu[k] = 0; hv[k] = 0; }
      }
    }
    return added;
  }

  // src/swe.mjs:1188-1197
  void sponge(double dt) {
    const double ref = spongeRef;
    for (const auto& c : spongeCells) {
      const int k = c.first;
      const double f = jmin(1.0, c.second * dt * 60);
      const T target = jmax(0, ref - b[k]);
      h[k] += (target - h[k]) * f;
      hu[k] -= hu[k] * f;
      hv[k] -= hv[k] * f;
    }
  }

  // src/swe.mjs:754-814
  double step(double dtIn, bool self) {
    applyBC();
    const double hh = self ? maxDt() : dtIn;
    if (!(hh > 0) || !std::isfinite(hh)) return 0;
    h0 = h; hu0 = hu; hv0 = hv;
    const int nthr = threads;
    residual(hh);
#pragma omp parallel for num_threads(nthr) if (nthr > 1) schedule(static)
    for (int k = 0; k < N; k++) {
      h[k] += hh * rh[k];
      hu[k] += hh * rhu[k];
      hv[k] += hh * rhv[k];
    }
    massFloored = dryClean();
    applyBC();
    residual(hh);
#pragma omp parallel for num_threads(nthr) if (nthr > 1) schedule(static)
    for (int k = 0; k < N; k++) {
      h[k] = 0.5 * (h0[k] + h[k] + hh * rh[k]);
      hu[k] = 0.5 * (hu0[k] + hu[k] + hh * rhu[k]);
      hv[k] = 0.5 * (hv0[k] + hv[k] + hh * rhv[k]);
    }
    massFloored += dryClean();
    applyFriction(hh);
    if (hasSponge) sponge(hh);
    t += hh;
    steps++;
    return hh;
  }

  // src/swe.mjs:819-836
  T volume() const {
    if (!sphere) {
      T v = 0;
      for (int j = 0; j < ny; j++) for (int i = 0; i < nx; i++) v += h[(j + ng) * W + (i + ng)];
      return v * dx * dy;
    }
    const std::vector<double>& area = g[OG_AREA];
    T v = 0;
    for (int j = 0; j < ny; j++) {
      T row = 0;
      for (int i = 0; i < nx; i++) row += h[(j + ng) * W + (i + ng)];
      v += row * area[j + ng];
    }
    return v;
  }
  // src/swe.mjs:862-877
  T energy() const {
    const std::vector<double>& area = g[OG_AREA];
    T e = 0;
    for (int j = 0; j < ny; j++) {
      T row = 0;
      for (int i = 0; i < nx; i++) {
        const int k = (j + ng) * W + (i + ng);
        const T hk = h[k];
        if (hk <= 0) continue;
        const T u = vel(hu[k], hk), v = vel(hv[k], hk);
        row += 0.5 * hk * (u * u + v * v) + 0.5 * G * hk * (hk + 2 * b[k]);
      }
      if (sphere) e += row * area[j + ng]; else e += row;
    }
    return sphere ? e : e * dx * dy;
  }
  // src/swe.mjs:880-892
  T maxSurfaceDeviation(double ref) const {
    T m = 0;
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        const int k = (j + ng) * W + (i + ng);
        if (h[k] <= minDepth) continue;
        const T d = fabsT(b[k] + h[k] - ref);
        if (d > m) m = d;
      }
    return m;
  }
  // src/swe.mjs:895-907
  T maxSpeed() const {
    T m = 0;
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        const int k = (j + ng) * W + (i + ng);
        const T hk = h[k];
        if (hk <= minDepth) continue;
        const T s = hypotT(vel(hu[k], hk), vel(hv[k], hk));
        if (s > m) m = s;
      }
    return m;
  }
  // src/swe.mjs:912-917
  bool finite() const {
    for (int k = 0; k < N; k++)
      if (!isfiniteT(h[k]) || !isfiniteT(hu[k]) || !isfiniteT(hv[k])) return false;
    return true;
  }
};

struct oracle_sim : SimT<double> {};

// ---- metric, src/geometry.mjs ------------------------------------------------
template <class S>
static void cartesianGeometry(S* s) {               // src/geometry.mjs:163-176
  s->R = INF;
  s->dlam = 0; s->dphi = 0;
  s->totalArea = s->nx * s->dx * s->ny * s->dy;
  for (int j = 0; j < s->H; j++) {
    s->g[OG_DXROW][j] = s->dx; s->g[OG_DYROWN][j] = s->dy; s->g[OG_DYROWS][j] = s->dy;
    s->g[OG_DYCFL][j] = s->dy; s->g[OG_BEDPHI][j] = s->dy;
    s->g[OG_AREA][j] = s->dx * s->dy; s->g[OG_LX][j] = s->dy; s->g[OG_LYN][j] = s->dx;
    s->g[OG_LYS][j] = s->dx; s->g[OG_FROW][j] = s->coriolis;
  }
}

static int sphericalGeometry(oracle_sim* s) {      // src/geometry.mjs:190-299
  const int nx = s->nx, ny = s->ny, ng = s->ng;
  const double R = s->R, lat0 = s->lat0, lat1 = s->lat1, omega = s->omega;
  char buf[256];
  if (!(lat1 > lat0)) {
    std::snprintf(buf, sizeof buf, "lat1 (%.17g) must exceed lat0 (%.17g)", lat1, lat0);
    g_err = buf; return -1;
  }
  if (lat0 < -90 || lat1 > 90) {
    std::snprintf(buf, sizeof buf, "latitudes must lie in [-90, 90]; got %.17g..%.17g", lat0, lat1);
    g_err = buf; return -1;
  }
  const bool touchesPole = lat0 <= -90 + 1e-12 || lat1 >= 90 - 1e-12;
  if (touchesPole && nx % 2 != 0) {
    std::snprintf(buf, sizeof buf, "nx must be even when the domain reaches a pole (got %d)", nx);
    g_err = buf; return -1;
  }
  const double dlam = 2 * PI / nx;
  const double p0 = lat0 * PI / 180, p1 = lat1 * PI / 180;
  const double dphi = (p1 - p0) / ny;
  s->dlam = dlam; s->dphi = dphi;
  const double gdy = R * dphi;
  s->dy = gdy;
  s->totalArea = 2 * PI * R * R * (std::sin(p1) - std::sin(p0));
  auto faceLat = [&](int k) { return k == 0 ? p0 : k == ny ? p1 : p0 + k * dphi; };
  for (int j = 0; j < s->H; j++) {
    const int jj = j - ng;
    const double rawS = faceLat(jj), rawN = faceLat(jj + 1);
    const double pS = clampLat(rawS), pN = clampLat(rawN);
    const double pC = 0.5 * (pS + pN);
    const double half = 0.5 * (pN - pS);
    s->g[OG_PHIC][j] = pC;
    s->g[OG_LYS][j] = R * dlam * cosLat(pS);
    s->g[OG_LYN][j] = R * dlam * cosLat(pN);
    s->g[OG_LX][j] = R * dphi;
    double A = 2 * R * R * dlam * cosLat(pC) * std::sin(half);
    if (!(A > 0)) {
      const double rS = reflectLat(rawS), rN = reflectLat(rawN);
      A = std::fabs(2 * R * R * dlam * cosLat(0.5 * (rS + rN)) * std::sin(0.5 * (rN - rS)));
    }
    s->g[OG_AREA][j] = A;
    const double lyN = s->g[OG_LYN][j], lyS = s->g[OG_LYS][j];
    s->g[OG_DXROW][j] = A / s->g[OG_LX][j];
    s->g[OG_DYROWN][j] = lyN > 0 ? A / lyN : INF;
    s->g[OG_DYROWS][j] = lyS > 0 ? A / lyS : INF;
    s->g[OG_DYCFL][j] = jmin(jmin(s->g[OG_DYROWN][j], s->g[OG_DYROWS][j]), gdy);
    s->g[OG_BEDPHI][j] = (lyN + lyS) > 0 ? 2 * A / (lyN + lyS) : INF;
    s->g[OG_TANPHI][j] = std::tan(pC);
    s->g[OG_FROW][j] = 2 * omega * std::sin(pC);
    s->g[OG_GEOCOEF][j] = (lyN - lyS) / (4 * A);
  }
  for (int j = 0; j < s->H; j++) {
    const double a = s->g[OG_AREA][j];
    if (!(a > 0) || !std::isfinite(a)) {
      std::snprintf(buf, sizeof buf, "row %d: area %.17g", j, a); g_err = buf; return -1;
    }
    if (!(s->g[OG_LYN][j] >= 0) || !(s->g[OG_LYS][j] >= 0)) {
      std::snprintf(buf, sizeof buf, "row %d: negative face length", j); g_err = buf; return -1;
    }
  }
  return 0;
}

// ---- C ABI ---------------------------------------------------------------
extern "C" {

const char* oracle_last_error(void) { return g_err.c_str(); }

int oracle_create(const oracle_options* o, const double* b, const double* h, oracle_sim** out) {
  *out = nullptr;
  if (!o || o->nx < 1 || o->ny < 1) { g_err = "nx and ny must be >= 1"; return -1; }
  if (o->limiter < 0 || o->limiter > 2) {
    g_err = "unknown limiter; have minmod,mc,central"; return -1;
  }
  oracle_sim* s = new oracle_sim();
  s->nx = o->nx; s->ny = o->ny; s->ng = 2;
  s->W = s->nx + 4; s->H = s->ny + 4; s->N = s->W * s->H;
  s->dx = o->dx; s->dy = o->dy;
  s->manning = o->manning; s->minDepth = o->min_depth; s->cfl = o->cfl; s->coriolis = o->coriolis;
  s->eps4 = std::pow(jmax(o->min_depth, 1e-12), 4.0);      // src/swe.mjs:190
  s->order = o->order; s->limiter = o->limiter; s->sphere = o->sphere;
  s->R = o->R; s->lat0 = o->lat0; s->lat1 = o->lat1; s->omega = o->omega;
  for (int r = 0; r < OG_NROWS; r++) s->g[r].assign(s->H, 0.0);
  if (s->sphere) {
    if (sphericalGeometry(s) != 0) { delete s; return -1; }
    s->dx = NAN;
  } else {
    cartesianGeometry(s);
  }
  const int N = s->N;
  for (auto* v : {&s->b, &s->h, &s->hu, &s->hv, &s->h0, &s->hu0, &s->hv0, &s->rh, &s->rhu, &s->rhv,
                  &s->fxM, &s->fxN, &s->fxT, &s->fyM, &s->fyN, &s->fyT, &s->pxL, &s->pxR, &s->pyL,
                  &s->pyR, &s->theta, &s->uu, &s->vv})
    v->assign(N, 0.0);
  for (auto* v : {&s->sE, &s->sU, &s->sV, &s->sB}) v->assign(2 * N, 0.0);
  if (b) std::memcpy(s->b.data(), b, sizeof(double) * N);
  if (h) std::memcpy(s->h.data(), h, sizeof(double) * N);
  if (s->sphere) { s->bc[0] = OB_PERIODIC; s->bc[1] = OB_PERIODIC; }     // src/swe.mjs:239-241
  *out = s;
  return 0;
}

void oracle_destroy(oracle_sim* s) { delete s; }

double* oracle_field(oracle_sim* s, int f) {
  switch (f) {
    case OF_B: return s->b.data();   case OF_H: return s->h.data();
    case OF_HU: return s->hu.data(); case OF_HV: return s->hv.data();
    case OF_H0: return s->h0.data(); case OF_HU0: return s->hu0.data();
    case OF_HV0: return s->hv0.data(); case OF_RH: return s->rh.data();
    case OF_RHU: return s->rhu.data(); case OF_RHV: return s->rhv.data();
    case OF_THETA: return s->theta.data();
    case OF_MANNING: return s->hasManning ? s->manningField.data() : nullptr;
    case OF_UU: return s->uu.data(); case OF_VV: return s->vv.data();
    default: return nullptr;
  }
}
double* oracle_geom(oracle_sim* s, int r) { return (r >= 0 && r < OG_NROWS) ? s->g[r].data() : nullptr; }

double oracle_get_scalar(oracle_sim* s, int w) {
  switch (w) {
    case 0: return s->dx; case 1: return s->dy; case 2: return s->R; case 3: return s->dlam;
    case 4: return s->dphi; case 5: return s->totalArea; case 6: return s->t; case 7: return s->steps;
    case 8: return s->massFloored; case 9: return s->eps4; case 10: return s->lat0;
    case 11: return s->lat1; case 12: return s->omega;
    default: return NAN;
  }
}
void oracle_set_scalar(oracle_sim* s, int w, double v) {
  if (w == 6) s->t = v; else if (w == 7) s->steps = v; else if (w == 8) s->massFloored = v;
}
void oracle_set_threads(oracle_sim* s, int threads) { s->threads = threads < 1 ? 1 : threads; }

int oracle_set_boundary(oracle_sim* s, int side, int kind) {
  if (side < 0 || side > 3 || kind < 0 || kind > 3) { g_err = "bad side or kind"; return -1; }
  s->bc[side] = kind;
  if (kind != OB_FLATHER) s->flTide[side] = false;
  return 0;
}
int oracle_set_flather_values(oracle_sim* s, int side, double eta_ext, double u_ext) {
  if (side < 0 || side > 3) { g_err = "bad side"; return -1; }
  s->bc[side] = OB_FLATHER; s->flTide[side] = false;
  s->flEta[side] = eta_ext; s->flU[side] = u_ext;
  return 0;
}
int oracle_set_flather_tide(oracle_sim* s, int side, double msl, int n, const double* amp,
                            const double* omega, const double* phase_deg, double u_coef) {
  if (side < 0 || side > 3 || n < 0) { g_err = "bad side"; return -1; }
  s->bc[side] = OB_FLATHER; s->flTide[side] = true;
  Tide& t = s->tide[side];
  t.msl = msl; t.u_coef = u_coef;
  t.amp.assign(amp, amp + n); t.omega.assign(omega, omega + n); t.phase.assign(phase_deg, phase_deg + n);
  return 0;
}
int oracle_set_manning_field(oracle_sim* s, const double* n) {   // src/swe.mjs:714-731
  if (!n) { s->hasManning = false; s->manningField.clear(); return 0; }
  for (int k = 0; k < s->N; k++) {
    const double v = n[k];
    if (!(v >= 0) || !std::isfinite(v)) {
      char buf[160];
      std::snprintf(buf, sizeof buf, "setManningField: n = %.17g at cell %d; Manning n must be finite and >= 0", v, k);
      g_err = buf; return -1;
    }
  }
  s->manningField.assign(n, n + s->N);
  s->hasManning = true;
  return 0;
}
int oracle_set_sponge(oracle_sim* s, int side, int width, double strength, double eta_ref) {
  // src/swe.mjs:1174-1186; side 0 west 1 east 2 south 3 north
  s->spongeCells.clear();
  for (int j = 0; j < s->ny; j++)
    for (int i = 0; i < s->nx; i++) {
      int d;
      if (side == 1) d = s->nx - 1 - i; else if (side == 0) d = i;
      else if (side == 3) d = s->ny - 1 - j; else d = j;
      if (d >= width) continue;
      const double c = std::cos(0.5 * PI * d / width);
      const double st = strength * (c * c);
      s->spongeCells.push_back({(j + s->ng) * s->W + (i + s->ng), st});
    }
  s->spongeRef = eta_ref;
  s->hasSponge = true;
  return 0;
}
int oracle_clear_sponge(oracle_sim* s) { s->hasSponge = false; s->spongeCells.clear(); return 0; }

void   oracle_apply_bc(oracle_sim* s) { s->applyBC(); }
void   oracle_residual(oracle_sim* s, double dt) { s->residual(dt); }
double oracle_max_dt(oracle_sim* s) { return s->maxDt(); }
void   oracle_apply_friction(oracle_sim* s, double dt) { s->applyFriction(dt); }
double oracle_dry_clean(oracle_sim* s) { return s->dryClean(); }
double oracle_step(oracle_sim* s, double dt) { return s->step(dt, false); }
double oracle_step_auto(oracle_sim* s) { return s->step(0, true); }
double oracle_volume(oracle_sim* s) { return s->volume(); }
double oracle_energy(oracle_sim* s) { return s->energy(); }
double oracle_max_surface_deviation(oracle_sim* s, double ref) { return s->maxSurfaceDeviation(ref); }
double oracle_max_speed(oracle_sim* s) { return s->maxSpeed(); }
int    oracle_finite(oracle_sim* s) { return s->finite() ? 1 : 0; }
double oracle_vel(oracle_sim* s, double hq, double h) { return s->vel(hq, h); }
void   oracle_hllc(double* out3, double hL, double huL, double hvL, double hR, double huR,
                   double hvR, double dry) { hllc(out3, hL, huL, hvL, hR, huR, hvR, dry); }

// Tangent-linear model of the gauge misfit J = sum_steps sum_gauges
// (b + h - obs)^2 over `steps` self-timed steps from h = max(0, eta0 - b)
// (Cartesian, walls): the solver run on Duals seeded with the directions db
// (bed) and dn (Manning field; NULL n means the scalar o->manning).  dt is
// each step's maxDt() of the value part, held as a constant, as the adjoint
// holds it.  Returns J, dJ = <grad J, (db, dn)>, and the dt sequence.
// oracle_tlm_misfit_bc: the same with a boundary kind per side (W, E, S, N:
// OB_REFLECT, OB_OUTFLOW, OB_PERIODIC, OB_FLATHER) and, for Flather sides,
// the constant exterior surface and normal velocity.

int oracle_tlm_misfit(const oracle_options* o, const double* b, const double* eta0, const double* n,
                      const double* db, const double* dn, int ng, const int* gauges, int steps,
                      const double* obs, int threads, double* J, double* dJ, double* dts) {
  return oracle_tlm_misfit_bc(o, b, eta0, n, db, dn, ng, gauges, steps, obs, threads, nullptr, nullptr, nullptr,
                              nullptr, J, dJ, dts);
}

int oracle_tlm_misfit_bc(const oracle_options* o, const double* b, const double* eta0, const double* n,
                         const double* db, const double* dn, int ng, const int* gauges, int steps,
                         const double* obs, int threads, const int* kinds, const double* fl_eta,
                         const double* fl_u, const oracle_tide_spec* tides, double* J, double* dJ,
                         double* dts) {
  if (!o || o->sphere || !b || !eta0 || !db || ng < 1 || !gauges || steps < 1 || !obs) {
    g_err = "oracle_tlm_misfit: Cartesian options, b, eta0, db, gauges, steps, obs"; return -1;
  }
  SimT<Dual> s;
  for (int q = 0; q < 4; q++) {
    const int kind = kinds ? kinds[q] : OB_REFLECT;
    if (kind < OB_REFLECT || kind > OB_FLATHER) { g_err = "oracle_tlm_misfit_bc: bad boundary kind"; return -1; }
    s.bc[q] = kind;
    s.flTide[q] = false;
    s.flEta[q] = fl_eta ? fl_eta[q] : 0.0;
    s.flU[q] = fl_u ? fl_u[q] : 0.0;
    if (tides && tides[q].n > 0 && kind == OB_FLATHER) {
      const oracle_tide_spec& ts = tides[q];
      s.flTide[q] = true;
      s.tide[q].msl = ts.msl; s.tide[q].u_coef = ts.u_coef;
      s.tide[q].amp.assign(ts.amp, ts.amp + ts.n);
      s.tide[q].omega.assign(ts.omega, ts.omega + ts.n);
      s.tide[q].phase.assign(ts.phase_deg, ts.phase_deg + ts.n);
    }
  }
  s.nx = o->nx; s.ny = o->ny; s.ng = 2; s.W = s.nx + 4; s.H = s.ny + 4; s.N = s.W * s.H;
  s.dx = o->dx; s.dy = o->dy; s.manning = o->manning; s.minDepth = o->min_depth; s.cfl = o->cfl;
  s.coriolis = o->coriolis; s.eps4 = std::pow(jmax(o->min_depth, 1e-12), 4.0);
  s.order = o->order; s.limiter = o->limiter; s.sphere = 0; s.threads = threads < 1 ? 1 : threads;
  for (int r = 0; r < OG_NROWS; r++) s.g[r].assign(s.H, 0.0);
  cartesianGeometry(&s);
  const int N = s.N;
  for (auto* v : {&s.b, &s.h, &s.hu, &s.hv, &s.h0, &s.hu0, &s.hv0, &s.rh, &s.rhu, &s.rhv, &s.fxM, &s.fxN,
                  &s.fxT, &s.fyM, &s.fyN, &s.fyT, &s.pxL, &s.pxR, &s.pyL, &s.pyR, &s.theta, &s.uu, &s.vv})
    v->assign(N, Dual(0));
  for (auto* v : {&s.sE, &s.sU, &s.sV, &s.sB}) v->assign(2 * N, Dual(0));
  for (int k = 0; k < N; k++) {
    s.b[k] = Dual(b[k], db[k]);
    s.h[k] = jmax(Dual(0), Dual(eta0[k]) - s.b[k]);
  }
  if (n) {
    s.manningField.resize(N);
    for (int k = 0; k < N; k++) s.manningField[k] = Dual(n[k], dn ? dn[k] : 0);
    s.hasManning = true;
  }
  Dual acc(0);
  for (int st = 0; st < steps; st++) {
    s.applyBC();
    const double dt = s.maxDt();
    if (dts) dts[st] = dt;
    s.step(dt, false);
    for (int q = 0; q < ng; q++) {
      const Dual r = s.b[gauges[q]] + s.h[gauges[q]] - obs[(size_t)st * ng + q];
      acc += r * r;
    }
  }
  *J = acc.v;
  *dJ = acc.d;
  return 0;
}

}  // extern "C"
