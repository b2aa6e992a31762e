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
// Face arrays are indexed by their left / lower cell and are zero where no
// face exists, so the limiter reads them unconditionally.
#pragma once

#include "swe_kernels.cuh"

namespace swe {
namespace {

constexpr int SPX = 32, SPY = 8;                 // tile of owned cells
constexpr int SP_THREADS = SPX * SPY;
constexpr int SSX = SPX + 3, SSY = SPY + 3;     // state tile: cols i0-1 .. i0+SPX+1, rows j0-1 .. j0+SPY+1

struct SplitBufs {
  double* fx[5];        // x face (k|k+1): M N T pL pR
  double* fy[5];        // y face (k|k+W)
  double* tb[3];        // bed term x, bed term y, geometric source
  double* U;            // cell velocity u (spherical Coriolis)
};

__global__ void __launch_bounds__(SP_THREADS, 3) k_split_faces(StageArgs a, SplitBufs s, Control* ctl) {
  if (ctl->stop) return;
  __shared__ double s_b[SSY][SSX], s_h[SSY][SSX], s_U[SSY][SSX], s_V[SSY][SSX];
  __shared__ double s_xs[4][SPY][SPX + 1];      // x slopes of cols i0 .. i0+SPX, rows j0 .. j0+SPY-1
  __shared__ double s_ys[4][SPY + 1][SPX];      // y slopes of cols i0 .. i0+SPX-1, rows j0 .. j0+SPY
  const int W = a.W, H = a.H;
  const int i0 = blockIdx.x * SPX, j0 = blockIdx.y * SPY;
  const double dry = a.minDepth, eps4 = a.eps4;
  const bool order2 = a.order >= 2;
  const bool sph = a.sph != 0;
  const bool bedOn = order2 || sph;
  const int t = threadIdx.x;

  // state and velocities of the tile and its halo (zero outside the grid)
  for (int q = t; q < SSX * SSY; q += SP_THREADS) {
    const int ly = q / SSX, lx = q - ly * SSX;
    const int gi = i0 - 1 + lx, gj = j0 - 1 + ly;
    double b = 0, h = 0, U = 0, V = 0;
    if (gi >= 0 && gi < W && gj >= 0 && gj < H) {
      const int k = gj * W + gi;
      b = __ldg(a.b + k); h = __ldg(a.h + k);
      const double hu = __ldg(a.hu + k), hv = __ldg(a.hv + k);
      if (h == 0) {                  // +-0 / den == +-0 and NaN / den == NaN: no division needed
        U = vel_num(hu, h); V = vel_num(hv, h);
      } else {
        const double den = vel_den(h, eps4);
        U = vel_num(hu, h) / den; V = vel_num(hv, h) / den;
      }
    }
    s_b[ly][lx] = b; s_h[ly][lx] = h; s_U[ly][lx] = U; s_V[ly][lx] = V;
  }
  __syncthreads();

  // x slopes (src/swe.mjs:364-411, d = 0)
  for (int q = t; q < SPY * (SPX + 1); q += SP_THREADS) {
    const int ly = q / (SPX + 1), lx = q - ly * (SPX + 1);
    const int gi = i0 + lx, gj = j0 + ly;
    double sE = 0, sB = 0, sU = 0, sV = 0;
    if (order2 && gj >= 1 && gj < H - 1 && gi >= 1 && gi < W - 1) {
      const int cy = ly + 1, cx = lx + 1;
      const double hk = s_h[cy][cx], hp = s_h[cy][cx + 1], hm = s_h[cy][cx - 1];
      if (!(hk <= dry || hp <= dry || hm <= dry)) {
        const double bk = s_b[cy][cx], bp = s_b[cy][cx + 1], bm = s_b[cy][cx - 1];
        const double eC = bk + hk, eP = bp + hp, eM = bm + hm;
        const double uk = s_U[cy][cx], vk = s_V[cy][cx];
        sE = limiter(a.lim, eC - eM, eP - eC);
        sB = limiter(a.lim, bk - bm, bp - bk);
        sU = limiter(a.lim, uk - s_U[cy][cx - 1], s_U[cy][cx + 1] - uk);
        sV = limiter(a.lim, vk - s_V[cy][cx - 1], s_V[cy][cx + 1] - vk);
      }
    }
    s_xs[0][ly][lx] = sE; s_xs[1][ly][lx] = sB; s_xs[2][ly][lx] = sU; s_xs[3][ly][lx] = sV;
  }
  // y slopes (d = 1)
  for (int q = t; q < (SPY + 1) * SPX; q += SP_THREADS) {
    const int ly = q / SPX, lx = q - ly * SPX;
    const int gi = i0 + lx, gj = j0 + ly;
    double sE = 0, sB = 0, sU = 0, sV = 0;
    if (order2 && gj >= 1 && gj < H - 1 && gi >= 1 && gi < W - 1) {
      const int cy = ly + 1, cx = lx + 1;
      const double hk = s_h[cy][cx], hp = s_h[cy + 1][cx], hm = s_h[cy - 1][cx];
      if (!(hk <= dry || hp <= dry || hm <= dry)) {
        const double bk = s_b[cy][cx], bp = s_b[cy + 1][cx], bm = s_b[cy - 1][cx];
        const double eC = bk + hk, eP = bp + hp, eM = bm + hm;
        const double uk = s_U[cy][cx], vk = s_V[cy][cx];
        sE = limiter(a.lim, eC - eM, eP - eC);
        sB = limiter(a.lim, bk - bm, bp - bk);
        sU = limiter(a.lim, uk - s_U[cy - 1][cx], s_U[cy + 1][cx] - uk);
        sV = limiter(a.lim, vk - s_V[cy - 1][cx], s_V[cy + 1][cx] - vk);
      }
    }
    s_ys[0][ly][lx] = sE; s_ys[1][ly][lx] = sB; s_ys[2][ly][lx] = sU; s_ys[3][ly][lx] = sV;
  }
  __syncthreads();

  const int lx = t % SPX, ly = t / SPX;
  const int gi = i0 + lx, gj = j0 + ly;
  if (gi >= W || gj >= H) return;
  const int k = gj * W + gi;
  const int cx = lx + 1, cy = ly + 1;
  const double bk = s_b[cy][cx], hk = s_h[cy][cx], Uk = s_U[cy][cx], Vk = s_V[cy][cx];
  const double xsE = s_xs[0][ly][lx], xsB = s_xs[1][ly][lx];
  const double nsE = s_ys[0][ly][lx], nsB = s_ys[1][ly][lx];

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
  if (sph) s.U[k] = Uk;

  // east x face (k|k+1)
  Face fx = {0, 0, 0, 0, 0};
  if (gj >= 2 && gj < H - 2 && gi >= 1 && gi < W - 2) {
    fx = face_flux(bk, hk, Uk, Vk, xsE, xsB, s_xs[2][ly][lx], s_xs[3][ly][lx],
                   s_b[cy][cx + 1], s_h[cy][cx + 1], s_U[cy][cx + 1], s_V[cy][cx + 1],
                   s_xs[0][ly][lx + 1], s_xs[1][ly][lx + 1], s_xs[2][ly][lx + 1], s_xs[3][ly][lx + 1], dry);
  }
  s.fx[0][k] = fx.M; s.fx[1][k] = fx.N; s.fx[2][k] = fx.T; s.fx[3][k] = fx.pL; s.fx[4][k] = fx.pR;
  // north y face (k|k+W): v is normal, u transverse
  Face fy = {0, 0, 0, 0, 0};
  if (gj >= 1 && gj < H - 2 && gi >= 2 && gi < W - 2) {
    fy = face_flux(bk, hk, Vk, Uk, nsE, nsB, s_ys[3][ly][lx], s_ys[2][ly][lx],
                   s_b[cy + 1][cx], s_h[cy + 1][cx], s_V[cy + 1][cx], s_U[cy + 1][cx],
                   s_ys[0][ly + 1][lx], s_ys[1][ly + 1][lx], s_ys[3][ly + 1][lx], s_ys[2][ly + 1][lx], dry);
  }
  s.fy[0][k] = fy.M; s.fy[1][k] = fy.N; s.fy[2][k] = fy.T; s.fy[3][k] = fy.pL; s.fy[4][k] = fy.pR;
}

// Positivity limiter of cell (gi, gj) from its four faces' mass fluxes
// (src/swe.mjs:511-529), with the same conservative pre-test as stage_tile.
__device__ __forceinline__ double split_theta(const StageArgs& a, const SplitBufs& s, double dt, int gi, int gj) {
  const int W = a.W, H = a.H;
  if (!(dt > 0 && gj >= 1 && gj < H - 1 && gi >= 1 && gi < W - 1)) return 1;
  const int k = gj * W + gi;
  const double fxE = s.fx[0][k], fxW = s.fx[0][k - 1];
  const double fyN = s.fy[0][k], fyS = s.fy[0][k - W];
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

template <int MODE>
__global__ void __launch_bounds__(SP_THREADS) k_split_cells(StageArgs a, SplitBufs s, Control* ctl) {
  static_assert(MODE == 1 || MODE == 2, "stages only");
  if (ctl->stop) return;
  __shared__ double s_th[SPY + 2][SPX + 2];
  __shared__ double s_red[2][SP_THREADS / 32];
  __shared__ bool s_last;
  const int W = a.W, H = a.H;
  const int i0 = blockIdx.x * SPX, j0 = blockIdx.y * SPY;
  const int t = threadIdx.x;
  const double dt = ctl->dt;
  const double dry = a.minDepth, eps4 = a.eps4;
  const bool order2 = a.order >= 2;
  const bool sph = a.sph != 0;
  const bool bedOn = order2 || sph;
  const bool corOn = sph || (a.coriolis != 0 && a.coriolis == a.coriolis);

  for (int q = t; q < (SPX + 2) * (SPY + 2); q += SP_THREADS) {
    const int ly = q / (SPX + 2), lx = q - ly * (SPX + 2);
    s_th[ly][lx] = split_theta(a, s, dt, i0 - 1 + lx, j0 - 1 + ly);
  }
  __syncthreads();

  double locMax = 0, locFl = 0;
  const int lx = t % SPX, ly = t / SPX;
  const int gi = i0 + lx, gj = j0 + ly;
  if (gi < W && gj < H) {
    const int k = gj * W + gi;
    const double thC = s_th[ly + 1][lx + 1];
    const double rdx = a.m.rdxRow[gj], dxr = a.m.dxRow[gj];
    double ah = 0, ahu = 0, ahv = 0;
    if (gj >= 2 && gj < H - 2) {
      if (gi - 1 >= 1 && gi - 1 < W - 2) {            // west face, cell is its right side
        const double M = s.fx[0][k - 1];
        const double thf = M >= 0 ? s_th[ly + 1][lx] : thC;
        const double inv = thf == 1 ? rdx : thf / dxr;
        ah += M * inv; ahu += (s.fx[1][k - 1] + s.fx[4][k - 1]) * inv; ahv += s.fx[2][k - 1] * inv;
      }
      if (gi >= 1 && gi < W - 2) {                    // east face, cell is its left side
        const double M = s.fx[0][k];
        const double thf = M >= 0 ? thC : s_th[ly + 1][lx + 2];
        const double inv = thf == 1 ? rdx : thf / dxr;
        ah -= M * inv; ahu -= (s.fx[1][k] + s.fx[3][k]) * inv; ahv -= s.fx[2][k] * inv;
      }
    }
    if (gi >= 2 && gi < W - 2) {
      if (gj - 1 >= 1 && gj - 1 < H - 2) {            // south face, cell is its upper side
        const int kf = k - W;
        const double M = s.fy[0][kf];
        const double thf = M >= 0 ? s_th[ly][lx + 1] : thC;
        const double invR = thf == 1 ? a.m.rdyRowS[gj] : thf / a.m.dyRowS[gj];
        ah += M * invR; ahv += (s.fy[1][kf] + s.fy[4][kf]) * invR; ahu += s.fy[2][kf] * invR;
      }
      if (gj >= 1 && gj < H - 2) {                    // north face, cell is its lower side
        const double M = s.fy[0][k];
        const double thf = M >= 0 ? thC : s_th[ly + 2][lx + 1];
        const double invL = thf == 1 ? a.m.rdyRowN[gj] : thf / a.m.dyRowN[gj];
        ah -= M * invL; ahv -= (s.fy[1][k] + s.fy[3][k]) * invL; ahu -= s.fy[2][k] * invL;
      }
    }
    const bool interior = gi >= 2 && gi < W - 2 && gj >= 2 && gj < H - 2;
    const double hin = a.h[k], huin = a.hu[k], hvin = a.hv[k];
    if (interior) {
      if (bedOn) {
        ahu += s.tb[0][k];
        ahv += s.tb[1][k];
        if (sph) ahv += s.tb[2][k];
      }
      if (sph) {
        const double fe = a.m.fRow[gj] + s.U[k] * (a.m.tanPhi[gj] / a.m.R);
        ahu += fe * hvin;
        ahv -= fe * huin;
      } else if (corOn) {
        ahu += a.coriolis * hvin;
        ahv -= a.coriolis * huin;
      }
    }
    if (MODE == 1) {
      double nh = hin + dt * ah, nhu = huin + dt * ahu, nhv = hvin + dt * ahv;
      if (interior) {                                 // dryClean, src/swe.mjs:734-745
        if (nh < 0) { locFl -= nh; nh = 0; }
        if (nh <= dry) { nhu = 0; nhv = 0; }
      }
      a.oh[k] = nh; a.ohu[k] = nhu; a.ohv[k] = nhv;
    } else {
      const double h0 = a.oh[k], hu0 = a.ohu[k], hv0 = a.ohv[k];   // U0 (in place)
      if (a.h0c) { a.h0c[k] = h0; a.hu0c[k] = hu0; a.hv0c[k] = hv0; }
      double nh = 0.5 * (h0 + hin + dt * ah);
      double nhu = 0.5 * (hu0 + huin + dt * ahu);
      double nhv = 0.5 * (hv0 + hvin + dt * ahv);
      if (interior) {
        if (nh < 0) { locFl -= nh; nh = 0; }
        if (nh <= dry) { nhu = 0; nhv = 0; }
        // friction, src/swe.mjs:659-704
        const double n = a.nfield ? a.nfield[k] : a.manning;
        const bool fricOn = a.nfield ? true : (n != 0 && n == n);
        if (fricOn) {
          if (nh <= dry) { nhu = 0; nhv = 0; }
          else if (n != 0 && n == n) {
            const double den = vel_den(nh, eps4);
            const double u = vel_num(nhu, nh) / den, v = vel_num(nhv, nh) / den;
            const double speed = hypot(u, v);
            if (!(speed < 1e-14)) {
              const double denom = 1 + dt * SWE_G * n * n * speed / pow(nh, 4.0 / 3.0);
              nhu = nhu / denom;
              nhv = nhv / denom;
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
          const double u = fabs(vel_num(nhu, nh) / den), v = fabs(vel_num(nhv, nh) / den);
          const double sr5 = (u + cc) / dxr + (v + cc) / a.m.dyCFL[gj];
          if (sr5 > locMax) locMax = sr5;
        }
      }
      a.oh[k] = nh; a.ohu[k] = nhu; a.ohv[k] = nhv;
    }
  }

  // per-block partials, then the last block closes the step
  for (int o = 16; o > 0; o >>= 1) {
    locMax = fmax(locMax, __shfl_down_sync(0xffffffffu, locMax, o));
    locFl += __shfl_down_sync(0xffffffffu, locFl, o);
  }
  if ((t & 31) == 0) { s_red[0][t >> 5] = locMax; s_red[1][t >> 5] = locFl; }
  __syncthreads();
  const int bid = blockIdx.y * gridDim.x + blockIdx.x;
  const int nb = gridDim.x * gridDim.y;
  if (t == 0) {
    double m = s_red[0][0], f = s_red[1][0];
    for (int w = 1; w < SP_THREADS / 32; w++) { m = fmax(m, s_red[0][w]); f += s_red[1][w]; }
    if (MODE == 1) a.part_fl1[bid] = f;
    else { a.part_max[bid] = m; a.part_fl2[bid] = f; }
    __threadfence();
    const unsigned int ticket = atomicAdd(&ctl->counter, 1u);
    s_last = (ticket == (unsigned int)(nb - 1));
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // the whole last block reduces the partials in a fixed order (strided per
  // thread, then a fixed tree), so the sums are the same in every run
  double m = 0, f = 0;
  const volatile double* pf = MODE == 1 ? a.part_fl1 : a.part_fl2;
  for (int q = t; q < nb; q += SP_THREADS) {
    if (MODE == 2) m = fmax(m, ((volatile double*)a.part_max)[q]);
    f += pf[q];
  }
  for (int o = 16; o > 0; o >>= 1) {
    m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    f += __shfl_down_sync(0xffffffffu, f, o);
  }
  __syncthreads();
  if ((t & 31) == 0) { s_red[0][t >> 5] = m; s_red[1][t >> 5] = f; }
  __syncthreads();
  if (t == 0) {
    m = s_red[0][0]; f = s_red[1][0];
    for (int w = 1; w < SP_THREADS / 32; w++) { m = fmax(m, s_red[0][w]); f += s_red[1][w]; }
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

}  // namespace
}  // namespace swe
