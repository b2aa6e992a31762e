// swe_adjoint_math.cuh -- reverse-mode derivatives of the per-face and
// per-cell arithmetic in swe_math.cuh, written by hand.
//
// Every function recomputes the forward values it needs from the same
// inputs (so it takes exactly the branches the forward step took) and then
// runs the statements backwards.  At a kink -- max(0, x), Math.max of two
// beds, the limiter's choice, the wet/dry tests, HLLC's wave-speed branches,
// the positivity limiter -- the derivative is that of the branch the forward
// pass took, which is what the discrete adjoint of the implemented scheme
// is.
#pragma once
#include "swe_math.cuh"

namespace swe {
namespace adj {

// d/da, d/db of the limiter at (a, b), for the branch the forward takes.
__device__ __forceinline__ void limiter_grad(int lim, double a, double b, double& da, double& db) {
  da = 0; db = 0;
  if (lim == 0) {                                   // mc
    if (a * b <= 0) return;
    const double c = 0.5 * (a + b);
    const double x = fabs(c), y = 2 * fabs(a), z = 2 * fabs(b);
    // the operand jmin(jmin(x, y), z) returns (equal non-negatives: the 2nd)
    int which = x < y ? 0 : 1;                      // 0: |c|, 1: 2|a|, 2: 2|b|
    if (!((which == 0 ? x : y) < z)) which = 2;
    // s = a > 0 ? m : -m, with a, b of one sign: |c| branch is c itself,
    // 2|a| branch is 2a, 2|b| branch is 2b.
    if (which == 0) { da = 0.5; db = 0.5; }
    else if (which == 1) { da = 2; }
    else { db = 2; }
    return;
  }
  if (lim == 1) {                                   // minmod
    if (a > 0 && b > 0) { if (a < b) da = 1; else db = 1; return; }
    if (a < 0 && b < 0) { if (a > b) da = 1; else db = 1; return; }
    return;
  }
  da = 0.5; db = 0.5;                               // central
}

// vel(q, h) = sqrt2 h q / sqrt(h^4 + max(h^4, eps4)): partials.
__device__ __forceinline__ void vel_grad(double q, double h, double eps4, double& dq, double& dh) {
  const double h4 = h * h * h * h;
  const bool big = h4 > eps4 || (h4 == eps4 && !signbit(h4));     // jmax(h4, eps4) returns h4
  const double D = h4 + (big ? h4 : eps4);
  const double sD = sqrt(D);
  const double dD = 4 * h * h * h * (big ? 2 : 1);
  dq = SWE_SQRT2 * h / sD;
  dh = qdiv(SWE_SQRT2 * q, sD) - qdiv(0.5 * SWE_SQRT2 * h * q * dD, D * sD);   // q is often +-0
}

// Reverse of hllc(): given the output adjoints (gM, gN, gT), add the
// adjoints of the six inputs.
__device__ __forceinline__ void hllc_rev(double hL, double huL, double hvL, double hR, double huR, double hvR,
                                         double dry, double gM, double gN, double gT,
                                         double& ghL, double& ghuL, double& ghvL,
                                         double& ghR, double& ghuR, double& ghvR) {
  const bool wetL = hL > dry, wetR = hR > dry;
  if (!wetL && !wetR) return;
  // u decides the wave speeds and so every branch below: the forward's own
  // division.  v only scales the transverse flux, so a reciprocal (reused
  // by the reverse of u = hu / h at the end) serves.
  const double rL = wetL ? 1 / hL : 0, rR = wetR ? 1 / hR : 0;
  const double uL = wetL ? qdiv(huL, hL) : 0, vL = wetL ? hvL * rL : 0;
  const double uR = wetR ? qdiv(huR, hR) : 0, vR = wetR ? hvR * rR : 0;
  const double cL = sqrt(SWE_G * jmax(hL, 0)), cR = sqrt(SWE_G * jmax(hR, 0));
  double sL, sR, a = 0, hStar = 0, qL = 1, qR = 1;
  int speeds;                                       // 0 dry|wet, 1 wet|dry, 2 wet|wet
  if (!wetL) { sL = uR - 2 * cR; sR = uR + cR; speeds = 0; }
  else if (!wetR) { sL = uL - cL; sR = uL + 2 * cL; speeds = 1; }
  else {
    a = (cL + cR) / 2 + (uL - uR) / 4;
    hStar = a * a / SWE_G;
    qL = hStar > hL ? sqrt(0.5 * (hStar + hL) * hStar / (hL * hL)) : 1;
    qR = hStar > hR ? sqrt(0.5 * (hStar + hR) * hStar / (hR * hR)) : 1;
    sL = uL - cL * qL;
    sR = uR + cR * qR;
    speeds = 2;
  }
  double guL = 0, gvL = 0, guR = 0, gvR = 0, gsL = 0, gsR = 0, gcL = 0, gcR = 0;
  if (sL >= 0) {                                    // flux1D(left)
    ghuL += gM + gN * uL;
    guL += gN * huL + gT * hvL;
    ghL += gN * SWE_G * hL;
    ghvL += gT * uL;
  } else if (sR <= 0) {                             // flux1D(right)
    ghuR += gM + gN * uR;
    guR += gN * huR + gT * hvR;
    ghR += gN * SWE_G * hR;
    ghvR += gT * uR;
  } else {
    const double num = sL * hR * (uR - sR) - sR * hL * (uL - sL);
    const double den = hR * (uR - sR) - hL * (uL - sL);
    const double sM = fabs(den) > 1e-30 ? qdiv(num, den) : 0.5 * (sL + sR);
    const bool takeL = sM >= 0;
    const double FL0 = huL, FL1 = huL * uL + 0.5 * SWE_G * hL * hL;
    const double FR0 = huR, FR1 = huR * uR + 0.5 * SWE_G * hR * hR;
    const double inv = 1 / (sR - sL);
    const double P0 = sR * FL0 - sL * FR0 + sL * sR * (hR - hL);
    const double P1 = sR * FL1 - sL * FR1 + sL * sR * (huR - huL);
    const double M = P0 * inv;
    // T = M * v(selected)
    const double gMt = gM + gT * (takeL ? vL : vR);
    if (takeL) gvL += gT * M; else gvR += gT * M;
    const double gP0 = gMt * inv, gP1 = gN * inv;
    const double ginv = gMt * P0 + gN * P1;
    gsR += -ginv * inv * inv;
    gsL += ginv * inv * inv;
    gsR += gP0 * (FL0 + sL * (hR - hL));
    gsL += gP0 * (-FR0 + sR * (hR - hL));
    const double gFL0 = gP0 * sR, gFR0 = -gP0 * sL;
    ghR += gP0 * sL * sR;
    ghL -= gP0 * sL * sR;
    gsR += gP1 * (FL1 + sL * (huR - huL));
    gsL += gP1 * (-FR1 + sR * (huR - huL));
    const double gFL1 = gP1 * sR, gFR1 = -gP1 * sL;
    ghuR += gP1 * sL * sR;
    ghuL -= gP1 * sL * sR;
    ghuL += gFL0 + gFL1 * uL;
    guL += gFL1 * huL;
    ghL += gFL1 * SWE_G * hL;
    ghuR += gFR0 + gFR1 * uR;
    guR += gFR1 * huR;
    ghR += gFR1 * SWE_G * hR;
  }
  // wave speeds
  if (speeds == 0) {
    guR += gsL + gsR;
    gcR += -2 * gsL + gsR;
  } else if (speeds == 1) {
    guL += gsL + gsR;
    gcL += -gsL + 2 * gsR;
  } else {
    guL += gsL;
    gcL -= gsL * qL;
    const double gqL = -gsL * cL;
    guR += gsR;
    gcR += gsR * qR;
    const double gqR = gsR * cR;
    // q = sqrt(X), X = Y / Z: dX = dq / (2 q), dY = dX / Z, dZ = -dY X with
    // X = q^2.  The derivatives need no branch decision, so they take one
    // division where the chain rule as written takes three.
    double ghStar = 0;
    if (hStar > hL && gqL != 0) {
      const double Z = hL * hL, X = qL * qL;
      const double gY = gqL / (2 * qL * Z), gZ = -gY * X;
      ghStar += gY * (hStar + 0.5 * hL);
      ghL += gY * 0.5 * hStar + gZ * 2 * hL;
    }
    if (hStar > hR && gqR != 0) {
      const double Z = hR * hR, X = qR * qR;
      const double gY = gqR / (2 * qR * Z), gZ = -gY * X;
      ghStar += gY * (hStar + 0.5 * hR);
      ghR += gY * 0.5 * hStar + gZ * 2 * hR;
    }
    const double ga = ghStar * 2 * a * (1.0 / SWE_G);
    gcL += 0.5 * ga;
    gcR += 0.5 * ga;
    guL += 0.25 * ga;
    guR -= 0.25 * ga;
  }
  // c = sqrt(G h): dc/dh = G / (2c) = c / (2h).  c is only differentiated on
  // a wet side (the branches above give a dry side's c no adjoint), where
  // 1 / h is at hand.
  if (gcL != 0 && hL > 0) ghL += gcL * 0.5 * cL * rL;
  if (gcR != 0 && hR > 0) ghR += gcR * 0.5 * cR * rR;
  // u = hu / h backwards, one reciprocal per side
  if (wetL) { ghuL += guL * rL; ghvL += gvL * rL; ghL -= (guL * uL + gvL * vL) * rL; }
  if (wetR) { ghuR += guR * rR; ghvR += gvR * rR; ghR -= (guR * uR + gvR * vR) * rR; }
}

// Inputs of one face (swe_math.cuh face_flux) and their adjoints.
struct FaceIn { double bL, hL, nL, tL, sEL, sBL, sNL, sTL, bR, hR, nR, tR, sER, sBR, sNR, sTR; };

// Reverse of face_flux: output adjoints (gM, gN, gT, gpL, gpR) -> g (inputs).
__device__ __forceinline__ FaceIn face_rev(const FaceIn& x, double dry, double gM, double gN, double gT,
                                           double gpL, double gpR) {
  FaceIn g = {};
  const double etaL = x.bL + x.hL + 0.5 * x.sEL;
  const double etaR = x.bR + x.hR - 0.5 * x.sER;
  const double bL = x.bL + 0.5 * x.sBL;
  const double bR = x.bR - 0.5 * x.sBR;
  const double aLf = etaL - bL, aRf = etaR - bR;
  const double hLf = jmax0(aLf), hRf = jmax0(aRf);
  const double nL = x.nL + 0.5 * x.sNL, nR = x.nR - 0.5 * x.sNR;
  const double tL = x.tL + 0.5 * x.sTL, tR = x.tR - 0.5 * x.sTR;
  const double bStar = jmax(bL, bR);
  const bool starL = bL > bR || (bL == bR && !signbit(bL));   // the operand jmax(bL, bR) returns
  const double aL = etaL - bStar, aR = etaR - bStar;
  const double hsL = jmax0(aL), hsR = jmax0(aR);
  double ghsL = 0, ghsR = 0, ghLf = 0, ghRf = 0;
  // pressure corrections pL = 0.5 G (hLf^2 - hsL^2)
  ghLf += gpL * SWE_G * hLf;
  ghsL -= gpL * SWE_G * hsL;
  ghRf += gpR * SWE_G * hRf;
  ghsR -= gpR * SWE_G * hsR;
  // hllc(hsL, hsL nL, hsL tL, hsR, hsR nR, hsR tR)
  double g0 = 0, g1 = 0, g2 = 0, g3 = 0, g4 = 0, g5 = 0;
  hllc_rev(hsL, hsL * nL, hsL * tL, hsR, hsR * nR, hsR * tR, dry, gM, gN, gT, g0, g1, g2, g3, g4, g5);
  ghsL += g0 + g1 * nL + g2 * tL;
  const double gnL = g1 * hsL, gtL = g2 * hsL;
  ghsR += g3 + g4 * nR + g5 * tR;
  const double gnR = g4 * hsR, gtR = g5 * hsR;
  double getaL = 0, getaR = 0, gbL = 0, gbR = 0, gbStar = 0;
  if (aL > 0) { getaL += ghsL; gbStar -= ghsL; }
  if (aR > 0) { getaR += ghsR; gbStar -= ghsR; }
  if (starL) gbL += gbStar; else gbR += gbStar;
  if (aLf > 0) { getaL += ghLf; gbL -= ghLf; }
  if (aRf > 0) { getaR += ghRf; gbR -= ghRf; }
  g.nL += gnL; g.sNL += 0.5 * gnL;
  g.nR += gnR; g.sNR -= 0.5 * gnR;
  g.tL += gtL; g.sTL += 0.5 * gtL;
  g.tR += gtR; g.sTR -= 0.5 * gtR;
  g.bL += gbL; g.sBL += 0.5 * gbL;
  g.bR += gbR; g.sBR -= 0.5 * gbR;
  g.bL += getaL; g.hL += getaL; g.sEL += 0.5 * getaL;
  g.bR += getaR; g.hR += getaR; g.sER -= 0.5 * getaR;
  return g;
}

}  // namespace adj
}  // namespace swe
