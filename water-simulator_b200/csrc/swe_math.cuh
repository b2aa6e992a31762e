// swe_math.cuh -- per-face and per-cell FP64 arithmetic of the shallow-water step.
//
// Every expression keeps the operand order of the reference (src/swe.mjs of
// Syntaxswine/water-simulator); the library is built with -fmad=false so no
// multiply-add is fused, which makes +, -, *, /, sqrt round exactly as the
// JavaScript engine's do.  Math.max / Math.min keep their JavaScript meaning
// (NaN in, NaN out; +0 above -0) so a blow-up propagates instead of being
// clipped away by IEEE maxNum.
#pragma once

#define SWE_G 9.80665                    // src/swe.mjs:85
#define SWE_SQRT2 1.4142135623730951     // Math.SQRT2

namespace swe {

__host__ __device__ __forceinline__ double jmax(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a > b) return a;
  if (b > a) return b;
  return signbit(a) ? b : a;
}
__host__ __device__ __forceinline__ double jmin(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a < b) return a;
  if (b < a) return b;
  return signbit(a) ? a : b;
}
// Math.max(0, x)
__host__ __device__ __forceinline__ double jmax0(double x) { return x > 0 ? x : (x == x ? 0.0 : x); }

// x / y correctly rounded (the operator's own PTX division), as an opaque
// operation: the compiler cannot see through it to rewrite its operands.
__device__ __forceinline__ double div_rn(double x, double y) {
  double q;
  asm("div.rn.f64 %0, %1, %2;" : "=d"(q) : "d"(x), "d"(y));
  return q;
}

// x / y, bit for bit, for a dividend that is often +-0 (the momentum of
// water at rest).  A zero dividend takes the division's slow path on B200
// (measured: 3.4x the time of a nonzero one).  +-0 / y with y finite and
// nonzero is the zero whose sign is the product of the signs, formed here
// from the bits; the division then gets the dividend 1 instead, so that lanes
// holding zeros stay on the fast path.  Every other case is the plain
// division.  The division is opaque because the compiler otherwise folds
// the substituted dividend back to x under the select.
// The tests are on the bit patterns (integer work, off the FP64 pipe).
__device__ __forceinline__ double qdiv(double x, double y) {
  const unsigned long long xb = __double_as_longlong(x), yb = __double_as_longlong(y);
  const bool z = (xb << 1) == 0 && (yb << 1) != 0 && ((yb >> 52) & 0x7ff) != 0x7ff;
  const double q = div_rn(z ? 1.0 : x, y);
  return z ? __longlong_as_double(xb ^ (yb & 0x8000000000000000ull)) : q;
}

// h^(4/3) of Manning friction (src/swe.mjs:683, 699: Math.pow(hk, 4 / 3)) as
// h * cbrt(h): within about 2 ulp of the power, as CUDA's pow is (the
// reference's Math.pow is not correctly rounded either, so friction is held
// to a tolerance rather than to the bits), at a fraction of pow's cost.
// Callers pass h > minDepth >= 0.
__device__ __forceinline__ double pow43(double h) { return h * cbrt(h); }

// Limiters, src/swe.mjs:88-141.  lim: 0 mc (default), 1 minmod, 2 central.
__device__ __forceinline__ double limiter(int lim, double a, double b) {
  if (lim == 0) {                                   // mc, src/swe.mjs:133-138
    const double p = a * b;
    if (p > 0) {
      // a, b are then non-NaN and nonzero of one sign, so c is too and the
      // three candidates are non-NaN and > +0: IEEE minNum is Math.min here.
      const double c = 0.5 * (a + b);
      const double m = fmin(fmin(fabs(c), 2 * fabs(a)), 2 * fabs(b));
      return a > 0 ? m : -m;
    }
    if (p <= 0) return 0;
    // a * b is NaN: Math.min's NaN rule decides
    const double c = 0.5 * (a + b);
    const double m = jmin(jmin(fabs(c), 2 * fabs(a)), 2 * fabs(b));
    return a > 0 ? m : -m;
  }
  if (lim == 1) {                                   // minmod, src/swe.mjs:88-92
    if (a > 0 && b > 0) return a < b ? a : b;
    if (a < 0 && b < 0) return a > b ? a : b;
    return 0;
  }
  return 0.5 * (a + b);                             // central, src/swe.mjs:141
}

// Desingularised velocity, src/swe.mjs:282-285.  The denominator depends on
// h only, so callers that need u and v of one cell share it (same double).
__device__ __forceinline__ double vel_den(double h, double eps4) {
  const double h4 = h * h * h * h;
  // h4 is +0, positive or NaN; for a NaN h4 the sum is NaN whichever maximum
  // is taken, so IEEE maxNum gives Math.max's result unless eps4 itself is
  // NaN (a NaN minDepth), where Math.max is NaN.
  return sqrt(h4 + (eps4 == eps4 ? fmax(h4, eps4) : eps4));
}
__device__ __forceinline__ double vel_num(double hq, double h) { return SWE_SQRT2 * h * hq; }
__device__ __forceinline__ double vel(double hq, double h, double eps4) {
  return qdiv(vel_num(hq, h), vel_den(h, eps4));
}

// HLLC with Einfeldt speeds and Toro's dry-state speeds, src/swe.mjs:975-1018.
// out = (mass, normal momentum, transverse momentum) flux.
__device__ __forceinline__ void hllc(double& o0, double& o1, double& o2,
                                     double hL, double huL, double hvL,
                                     double hR, double huR, double hvR, double dry) {
  const bool wetL = hL > dry, wetR = hR > dry;
  if (!wetL && !wetR) { o0 = 0; o1 = 0; o2 = 0; return; }
  const double uL = wetL ? qdiv(huL, hL) : 0, vL = wetL ? qdiv(hvL, hL) : 0;
  const double uR = wetR ? qdiv(huR, hR) : 0, vR = wetR ? qdiv(hvR, hR) : 0;
  const double cL = sqrt(SWE_G * jmax(hL, 0)), cR = sqrt(SWE_G * jmax(hR, 0));
  double sL, sR;
  if (!wetL) { sL = uR - 2 * cR; sR = uR + cR; }
  else if (!wetR) { sL = uL - cL; sR = uL + 2 * cL; }
  else {
    const double a = (cL + cR) / 2 + (uL - uR) / 4;
    const double hStar = a * a / SWE_G;
    const double qL = hStar > hL ? sqrt(0.5 * (hStar + hL) * hStar / (hL * hL)) : 1;
    const double qR = hStar > hR ? sqrt(0.5 * (hStar + hR) * hStar / (hR * hR)) : 1;
    sL = uL - cL * qL;
    sR = uR + cR * qR;
  }
  if (sL >= 0) {                                      // flux1D(left)
    o0 = huL; o1 = huL * uL + 0.5 * SWE_G * hL * hL; o2 = hvL * uL; return;
  }
  if (sR <= 0) {                                      // flux1D(right)
    o0 = huR; o1 = huR * uR + 0.5 * SWE_G * hR * hR; o2 = hvR * uR; return;
  }
  const double num = sL * hR * (uR - sR) - sR * hL * (uL - sL);
  const double den = hR * (uR - sR) - hL * (uL - sL);
  const double sM = fabs(den) > 1e-30 ? qdiv(num, den) : 0.5 * (sL + sR);
  const double FL0 = huL, FL1 = huL * uL + 0.5 * SWE_G * hL * hL;
  const double FR0 = huR, FR1 = huR * uR + 0.5 * SWE_G * hR * hR;
  const double inv = 1 / (sR - sL);
  o0 = (sR * FL0 - sL * FR0 + sL * sR * (hR - hL)) * inv;
  o1 = (sR * FL1 - sL * FR1 + sL * sR * (huR - huL)) * inv;
  o2 = o0 * (sM >= 0 ? vL : vR);
}

// One interface: MUSCL reconstruction from the two cells' slopes along the
// face normal, Audusse hydrostatic reconstruction against the higher bed,
// HLLC, and the two interface-local pressure corrections
// (src/swe.mjs:415-445 for x faces, :448-475 for y faces).  For a y face the
// caller passes (v, u) as (normal, transverse).
struct Face { double M, N, T, pL, pR; };

__device__ __forceinline__ Face face_flux(
    double bL_c, double hL_c, double nL_c, double tL_c,        // left cell b, h, normal vel, transverse vel
    double sEL, double sBL, double sNL, double sTL,            // left slopes along the normal
    double bR_c, double hR_c, double nR_c, double tR_c,
    double sER, double sBR, double sNR, double sTR, double dry) {
  const double etaL = bL_c + hL_c + 0.5 * sEL;
  const double etaR = bR_c + hR_c - 0.5 * sER;
  const double bL = bL_c + 0.5 * sBL;
  const double bR = bR_c - 0.5 * sBR;
  const double hLf = jmax0(etaL - bL);
  const double hRf = jmax0(etaR - bR);
  const double nL = nL_c + 0.5 * sNL;
  const double nR = nR_c - 0.5 * sNR;
  const double tL = tL_c + 0.5 * sTL;
  const double tR = tR_c - 0.5 * sTR;
  const double bStar = jmax(bL, bR);
  const double hsL = jmax0(etaL - bStar);
  const double hsR = jmax0(etaR - bStar);
  Face f;
  hllc(f.M, f.N, f.T, hsL, hsL * nL, hsL * tL, hsR, hsR * nR, hsR * tR, dry);
  f.pL = 0.5 * SWE_G * (hLf * hLf - hsL * hsL);
  f.pR = 0.5 * SWE_G * (hRf * hRf - hsR * hsR);
  return f;
}

}  // namespace swe
