// swe_kernels.cuh -- sm_100a FP64 kernels of the SSP-RK2 shallow-water step.
//
// Device layout (per simulation, row-major, padded grid W = nx+4, H = ny+4,
// index k = j*W + i as in src/swe.mjs:196-199,268):
//   b                 bed
//   A = (h, hu, hv)   the state; stage 2 overwrites it in place
//   B = (h, hu, hv)   the stage-1 state U1
//   metric rows       13 arrays of H doubles (src/geometry.mjs:301-309)
//
// One step (src/swe.mjs:754-814) is five launches:
//   k_prepare      dt, t, Flather values for this step (one warp)
//   k_apply_bc(A)  ghost rings of A (src/swe.mjs:289-303)
//   k_stage<1>     B = A + dt R(A); dryClean
//   k_apply_bc(B)
//   k_stage<2>     A = (A + B + dt R(B)) / 2; dryClean; friction; sponge;
//                  CFL rate of the result; the last CTA closes the step.
//
// k_stage is the whole residual (src/swe.mjs:308-629) fused with the stage
// update.  Each CTA owns a strip of SX output columns and RY output rows and
// marches down the rows, one thread per column; the dependency radius of the
// residual is 3 cells (slopes -> faces -> positivity factor of the upwind
// neighbour), so a strip carries 4 halo columns each side and a chunk starts
// 3 rows early.  Per row r the pipeline is
//   S1  load row r, velocities                      (publish to smem)
//   S2  slopes of row r-1, bed term of row r-1       (publish x slopes)
//   --  __syncthreads
//   S3  x face (c|c+1) of row r-1, y face (r-2|r-1)  (publish x faces)
//   S4  positivity factor theta of row r-2           (publish)
//   S5  accumulate + update of row r-3, gathering each cell's faces in the
//       order the reference's scatter loops apply them
// and same-column values ride in registers.  Ring depths (state 3, x slopes
// 2, x faces 3, theta 2) are what make one barrier per row sufficient.
#pragma once
#include "swe_math.cuh"

namespace swe {
namespace {   // every definition here is private to the including translation unit

constexpr int BX = 128;          // threads per CTA = columns per strip incl. halos
constexpr int HALO = 4;          // halo columns each side (left edge stays 16-byte aligned)
constexpr int SX = BX - 2 * HALO;
constexpr int MAX_TIDE = 16;

enum { BC_REFLECT = 0, BC_OUTFLOW = 1, BC_PERIODIC = 2, BC_FLATHER = 3 };

// Device control block: everything the step chain decides on the device.
struct Control {
  double dt;            // dt of the step in flight
  double t;             // simulation time at the start of the step in flight
  double steps;         // completed steps
  double next_max;      // max CFL rate over wet interior cells of the current state
  double floored1;      // mass floored by stage 1's dryClean
  double mass_floored;  // massFloored of the last completed step
  double fl_eta[4], fl_u[4];
  double diag;          // last diagnostic result
  int stop;             // 1: the prepared step was refused (dt not > 0 or not finite)
  // tiles the tiled cell kernels settled in the last step, one in 16
  // counted; beside `stop` and `dt`, in the line every kernel reads first
  int settled;
  int status;           // sticky status bits (4: a tile copy did not complete within its bound)
  unsigned int counter; // last-CTA ticket
  // Flather tide tables (src/tide.mjs:103-107), per side
  int tide_n[4];
  double tide_msl[4], tide_ucoef[4];
  double tide_amp[4][MAX_TIDE], tide_omega[4][MAX_TIDE], tide_phase[4][MAX_TIDE];
  int settled_next;     // the same count for the step in flight (k_prepare moves it to `settled`)
  int pad;
};

struct Metric {   // per-row divisors (src/geometry.mjs)
  const double* dxRow; const double* dyRowN; const double* dyRowS; const double* dyCFL;
  const double* bedPhi; const double* geoCoef; const double* fRow; const double* tanPhi;
  // 1/dxRow, 1/dyRowN, 1/dyRowS, formed on the host with the same IEEE
  // division, so theta/dxRow == rdxRow exactly when theta == 1
  const double* rdxRow; const double* rdyRowN; const double* rdyRowS;
  double R;
};

// x / d, skipping the division when the factor z of x is +-0: then x is
// +-0 or NaN, and +-0 / d == +-0, NaN / d == NaN for the finite or
// infinite positive divisors of the metric.
__device__ __forceinline__ double div_unless_zero(double x, double z, double d) {
  return z == 0 ? x : x / d;
}

struct StageArgs {
  int W, H, nx, ny;
  const double* b;
  const double* h; const double* hu; const double* hv;      // stage input (ghosts filled)
  double* oh; double* ohu; double* ohv;                     // stage output (stage 2: == U0)
  double* h0c; double* hu0c; double* hv0c;                  // optional copy of U0 (stage 2)
  double* rh; double* rhu; double* rhv; double* theta;       // residual mode outputs
  Metric m;
  double minDepth, eps4, coriolis;
  int sph, order, lim;
  // epilogue (stage 2)
  double manning; const double* nfield;
  int sponge_side, sponge_width; const double* sponge_str; double sponge_ref;
  double* part_max; double* part_fl1; double* part_fl2;     // one per CTA
  int nblocks;
  // optional tape of the tiled stage kernels (the adjoint's segment pass):
  // the cell's positivity limiter, its depth before dryClean and (stage 2)
  // the state after dryClean that friction takes
  double* tape_th; double* tape_hpre; double* tape_pre[3];
  // every reciprocal metric row (rdxRow, rdyRowN, rdyRowS) finite, so a
  // face value of +0 times any of them is +0
  int dryfold;
};

// ---------------------------------------------------------------------------
// prepare: dt of the next step (src/swe.mjs:783-784) and the Flather values.
// mode 0: dt = dt_host (checked on the host); 1: cfl / next_max (step());
// 2: a fixed dt clamped to t_end - t; 3: min(maxDt, t_end - t); 4: *dt_dev,
// a dt another kernel or a collective left in device memory.
struct PrepArgs {
  int mode; double dt_host; double cfl; double t_end; const double* dt_dev;
  int fl_kind[4];           // 0 host value, 1 tide table
  double fl_eta[4], fl_u[4];
};

__device__ __forceinline__ void prepare_one(Control* ctl, const PrepArgs& a) {
  double dt;
  if (a.mode == 0) dt = a.dt_host;
  else if (a.mode == 2) dt = jmin(a.dt_host, a.t_end - ctl->t);
  else if (a.mode == 4) dt = *a.dt_dev;
  else {
    const double inv = ctl->next_max;
    double md = inv > 0 ? a.cfl / inv : INFINITY;
    dt = (a.mode == 3) ? jmin(md, a.t_end - ctl->t) : md;
  }
  ctl->dt = dt;
  ctl->stop = (!(dt > 0) || !isfinite(dt)) ? 1 : 0;
  ctl->settled = ctl->settled_next;
  ctl->settled_next = 0;
  const double t = ctl->t;
  for (int s = 0; s < 4; s++) {
    if (a.fl_kind[s] == 1) {
      double e = ctl->tide_msl[s];
      for (int q = 0; q < ctl->tide_n[s]; q++)
        e += ctl->tide_amp[s][q] * cos(ctl->tide_omega[s][q] * t - ctl->tide_phase[s][q] * 3.141592653589793 / 180);
      ctl->fl_eta[s] = e;
      ctl->fl_u[s] = ctl->tide_ucoef[s] * e;
    } else {
      ctl->fl_eta[s] = a.fl_eta[s];
      ctl->fl_u[s] = a.fl_u[s];
    }
  }
}

// Programmatic dependent launch (sm_90+).  A kernel of the stepping loop
// lets the next one be scheduled as soon as all of its own CTAs have
// started, then waits until every grid it depends on has finished and its
// writes are visible, before it reads or writes anything.  Launched without
// the programmatic attribute, both are no-ops.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
}

__global__ void k_prepare(Control* ctl, PrepArgs a) {
  pdl_enter();
  if (threadIdx.x == 0) prepare_one(ctl, a);
}

// maxDt() of the current state (src/swe.mjs:632-647) into device memory, for
// a caller that combines it on the device (a row slab's all-reduce).
__global__ void k_dt_out(const Control* ctl, double cfl, double* out) {
  if (threadIdx.x == 0) {
    const double inv = ctl->next_max;
    *out = inv > 0 ? cfl / inv : INFINITY;
  }
}

// ---------------------------------------------------------------------------
// Boundary conditions, src/swe.mjs:289-303 and 1026-1126.
//
// The reference fills the W/E ghost columns for every row and then the S/N
// ghost rows for i in [-2, nx+2), so the corners come from the S/N pass and
// the W/E values at ghost rows are dead.  Every final ghost value is a pure
// function of interior cells: reflect/outflow/Flather read clamped interior
// sources, periodic reads the cell nx (ny) away -- which, for nx (ny) = 1,
// is the other ghost of the same side, i.e. the cell index taken modulo nx
// (ny) -- and a periodic S/N ghost in a ghost column reads the W/E ghost of
// an interior row.  So one thread per final ghost cell computes its value
// from interior cells only (W/E values needed by S/N are recomputed), with
// no ordering between threads.
struct BCArgs {
  int nx, ny, W, H;
  int kind[4];
  double minDepth, eps4;
  double* b; double* h; double* hu; double* hv;
};

struct Cell { double b, h, hu, hv; };

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ int modi(int v, int n) { int r = v % n; return r < 0 ? r + n : r; }

__device__ __forceinline__ Cell load_cell(const BCArgs& a, int i, int j) {
  const int k = (j + 2) * a.W + (i + 2);
  Cell c; c.b = a.b[k]; c.h = a.h[k]; c.hu = a.hu[k]; c.hv = a.hv[k];
  return c;
}

// src/swe.mjs:1085-1115: ghost (i,j) on `side` from interior source s.
__device__ __forceinline__ Cell flather_cell(const BCArgs& a, const Control* ctl, int side, Cell s) {
  Cell g;
  g.b = s.b;
  const double bed = g.b;
  const double hInt = s.h;
  const double e0 = ctl->fl_eta[side], u0 = ctl->fl_u[side];
  if (hInt <= a.minDepth) { g.h = jmax0(e0 - bed); g.hu = 0; g.hv = 0; return g; }
  const double etaInt = bed + hInt;
  const double r = sqrt(SWE_G / hInt);
  const double sgn = (side == 0 || side == 2) ? 1 : -1;
  const double uInt = (side == 0 || side == 1) ? vel(s.hu, hInt, a.eps4) : vel(s.hv, hInt, a.eps4);
  const double Rin = u0 + sgn * e0 * r;
  const double Rout = uInt - sgn * etaInt * r;
  const double un = 0.5 * (Rin + Rout);
  const double en = sgn * (Rin - Rout) / (2 * r);
  g.h = jmax0(en - bed);
  if (side == 0 || side == 1) { g.hu = g.h * un; g.hv = s.hv; }
  else { g.hv = g.h * un; g.hu = s.hu; }
  return g;
}

// Every final ghost value is one interior cell under one map (the ghost's
// source and transform): a copy, a copy with the x or the y momentum negated
// (reflect W/E, S/N), or the Flather state of one side.  ghost_source gives
// both for the ghost (i, j) -- W/E ghosts (i < 0 or i >= nx) of interior rows,
// S/N ghosts (j < 0 or j >= ny) of columns [-2, nx+2) -- for the forward fill
// here and for the adjoint's reverse of it.
enum { GT_COPY = 0, GT_FLIPU = 1, GT_FLIPV = 2, GT_FLATHER = 4 };   // GT_FLATHER + side
__host__ __device__ __forceinline__ int clampi_hd(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
__host__ __device__ __forceinline__ int modi_hd(int v, int n) { int r = v % n; return r < 0 ? r + n : r; }

__host__ __device__ __forceinline__ int we_source(const int* kind, int nx, int i, int j, int& si, int& sj) {
  const int side = i < 0 ? 0 : 1;
  sj = j;
  switch (kind[side]) {
    case BC_REFLECT: si = clampi_hd(side == 0 ? -1 - i : 2 * nx - 1 - i, 0, nx - 1); return GT_FLIPU;
    case BC_OUTFLOW: si = clampi_hd(i, 0, nx - 1); return GT_COPY;
    case BC_PERIODIC: si = modi_hd(i, nx); return GT_COPY;
    default: si = clampi_hd(i, 0, nx - 1); return GT_FLATHER + side;
  }
}
__host__ __device__ __forceinline__ int ghost_source(const int* kind, int nx, int ny, int i, int j, int& si,
                                                     int& sj) {
  if (j >= 0 && j < ny) return we_source(kind, nx, i, j, si, sj);
  const int side = j < 0 ? 2 : 3;
  switch (kind[side]) {
    case BC_REFLECT:
      si = clampi_hd(i, 0, nx - 1);
      sj = clampi_hd(side == 2 ? -1 - j : 2 * ny - 1 - j, 0, ny - 1);
      return GT_FLIPV;
    case BC_OUTFLOW: si = clampi_hd(i, 0, nx - 1); sj = clampi_hd(j, 0, ny - 1); return GT_COPY;
    case BC_PERIODIC: {
      const int pj = modi_hd(j, ny);
      if (i >= 0 && i < nx) { si = i; sj = pj; return GT_COPY; }
      return we_source(kind, nx, i, pj, si, sj);      // the W/E ghost of row pj, recomputed
    }
    default: si = clampi_hd(i, 0, nx - 1); sj = clampi_hd(j, 0, ny - 1); return GT_FLATHER + side;
  }
}

// Final value of the ghost (i, j).
__device__ __forceinline__ Cell ghost_cell(const BCArgs& a, const Control* ctl, int i, int j) {
  int si, sj;
  const int tr = ghost_source(a.kind, a.nx, a.ny, i, j, si, sj);
  Cell c = load_cell(a, si, sj);
  if (tr >= GT_FLATHER) return flather_cell(a, ctl, tr - GT_FLATHER, c);
  if (tr == GT_FLIPU) c.hu = -c.hu;
  else if (tr == GT_FLIPV) c.hv = -c.hv;
  return c;
}

// Ghost cells q0, q0 + stride, ... of one grid.
__device__ __forceinline__ void apply_bc_range(const BCArgs& a, const Control* ctl, int q0, int stride) {
  const int nwe = 4 * a.ny;                 // 2 sides x 2 rings x ny interior rows
  const int nsn = 4 * (a.nx + 4);           // 2 sides x 2 rings x (nx + 4) columns
  for (int q = q0; q < nwe + nsn; q += stride) {
    int i, j;
    Cell c;
    if (q < nwe) {
      j = q / 4;
      const int r = q % 4;                  // 0,1 west rings; 2,3 east rings
      i = r < 2 ? -1 - r : a.nx + (r - 2);
    } else {
      const int p = q - nwe;
      i = p / 4 - 2;
      const int r = p % 4;
      j = r < 2 ? -1 - r : a.ny + (r - 2);
    }
    c = ghost_cell(a, ctl, i, j);
    const int k = (j + 2) * a.W + (i + 2);
    a.b[k] = c.b; a.h[k] = c.h; a.hu[k] = c.hu; a.hv[k] = c.hv;
  }
}

__global__ void k_apply_bc(BCArgs a, const Control* ctl, int respect_stop) {
  pdl_enter();
  if (respect_stop && ctl->stop) return;
  apply_bc_range(a, ctl, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// ---------------------------------------------------------------------------
// Fused residual + stage update.  MODE 0: residual only (rh, rhu, rhv,
// theta for every cell, src/swe.mjs:308-629); MODE 1: stage 1
// (src/swe.mjs:790-796); MODE 2: stage 2 + epilogue (src/swe.mjs:798-813).
constexpr int RY_MAX = 64;                  // output rows per CTA, at most
constexpr int MROWS = RY_MAX + 6;           // metric rows a CTA touches
enum { M_DX, M_RDX, M_DYN, M_RDYN, M_DYS, M_RDYS, M_BED, M_GEO, M_F, M_TAN, M_CFL, M_COUNT };
// dynamic shared memory of k_stage: state ring 4x6 rows, x slopes 2x4,
// x faces 3x5, theta 2 (all BX wide), then the metric rows
constexpr int STAGE_SMEM_BYTES = (49 * BX + M_COUNT * MROWS) * 8;

#ifndef SWE_STAGE_MIN_BLOCKS
#define SWE_STAGE_MIN_BLOCKS 3
#endif
// One tile: output columns strip*SX .. +SX (padded), output rows [y0, y1).
// `part` is this tile's slot among the `a.nblocks` partial slots of its grid,
// whose last finisher closes the step.  Every thread of the CTA calls it.
template <int MODE>
__device__ __forceinline__ void stage_tile(const StageArgs& a, Control* ctl, int strip, int y0, int y1,
                                           int part, double* smem) {
  if (MODE != 0 && ctl->stop) return;
  // state ring, 4 rows deep: b, h, U, V are read by neighbours (rows r-1),
  // h, hu, hv, U of row r-3 by the cell's own thread in S5
  double (*s_b)[BX] = reinterpret_cast<double (*)[BX]>(smem);
  double (*s_h)[BX] = s_b + 4;
  double (*s_U)[BX] = s_b + 8;
  double (*s_V)[BX] = s_b + 12;
  double (*s_hu)[BX] = s_b + 16;
  double (*s_hv)[BX] = s_b + 20;
  double (*s_xs)[4][BX] = reinterpret_cast<double (*)[4][BX]>(smem + 24 * BX);   // x slopes ring (sE,sB,sU,sV)
  double (*s_fx)[5][BX] = reinterpret_cast<double (*)[5][BX]>(smem + 32 * BX);   // x faces ring (M,N,T,pL,pR)
  double (*s_th)[BX] = reinterpret_cast<double (*)[BX]>(smem + 47 * BX);         // theta ring
  double (*s_m)[MROWS] = reinterpret_cast<double (*)[MROWS]>(smem + 49 * BX);    // the CTA's metric rows
  __shared__ double s_red[2][BX / 32];

  const int c = threadIdx.x;
  const int W = a.W, H = a.H;
  const int gi = strip * SX - HALO + c;
  const bool colIn = gi >= 0 && gi < W;
  const int RY = y1 - y0;                    // <= RY_MAX (host)
  const int mbase = y0 - 3;                  // metric row m = j - mbase
  const double dt = ctl->dt;
  const double dry = a.minDepth, eps4 = a.eps4;
  const bool order2 = a.order >= 2;
  const bool sph = a.sph != 0;
  const bool bedOn = order2 || sph;
  const bool corOn = sph || (a.coriolis != 0 && a.coriolis == a.coriolis);
  const bool outCol = c >= HALO && c < HALO + SX && colIn;
  const bool interiorCol = gi >= 2 && gi < W - 2;

  // metric rows of this chunk into shared memory (broadcast reads later)
  for (int q = c; q < M_COUNT * MROWS; q += BX) {
    const int f = q / MROWS, m = q % MROWS, j = m + mbase;
    double v = 0;
    if (j >= 0 && j < H && m < RY + 6) {
      const double* src = f == M_DX ? a.m.dxRow : f == M_RDX ? a.m.rdxRow : f == M_DYN ? a.m.dyRowN :
                          f == M_RDYN ? a.m.rdyRowN : f == M_DYS ? a.m.dyRowS : f == M_RDYS ? a.m.rdyRowS :
                          f == M_BED ? a.m.bedPhi : f == M_GEO ? a.m.geoCoef : f == M_F ? a.m.fRow :
                          f == M_TAN ? a.m.tanPhi : a.m.dyCFL;
      v = src[j];
    }
    s_m[f][m] = v;
  }
  __syncthreads();

  // carried registers (same column)
  double b_m1 = 0, h_m1 = 0, U_m1 = 0, V_m1 = 0;     // row r-1
  double b_m2 = 0, h_m2 = 0, U_m2 = 0, V_m2 = 0;     // row r-2
  double ysE = 0, ysB = 0, ysU = 0, ysV = 0;         // y slopes of row r-2
  double tb0_m2 = 0, tb1_m2 = 0, tg_m2 = 0;          // bed terms of row r-2 (computed last row)
  double tb0_m3 = 0, tb1_m3 = 0, tg_m3 = 0;          // bed terms of row r-3
  Face fy1 = {0, 0, 0, 0, 0}, fy2 = {0, 0, 0, 0, 0}; // y faces (r-3|r-2), (r-4|r-3)
  double th_m3 = 1, th_m4 = 1;
  double locMax = 0, locFl = 0;

  // prefetch of the next row of the input state, and (stage 2) of U0 one
  // row ahead of its use in S5
  double pb = 0, ph = 0, phu = 0, phv = 0;
  double p0h = 0, p0hu = 0, p0hv = 0;
  {
    const int r = y0 - 3;
    if (colIn && r >= 0 && r < H) {
      const int k = r * W + gi;
      pb = __ldg(a.b + k); ph = __ldg(a.h + k); phu = __ldg(a.hu + k); phv = __ldg(a.hv + k);
    }
  }

  for (int r = y0 - 3; r <= y1 + 2; ++r) {
    // ---- S1: row r (prefetched), issue the loads of row r+1 -------------
    const double b_c = pb, h_c = ph, hu_c = phu, hv_c = phv;
    if (colIn && r + 1 >= 0 && r + 1 < H && r + 1 <= y1 + 2) {
      const int k = (r + 1) * W + gi;
      pb = __ldg(a.b + k); ph = __ldg(a.h + k); phu = __ldg(a.hu + k); phv = __ldg(a.hv + k);
    } else {
      pb = 0; ph = 0; phu = 0; phv = 0;
    }
    double U0h = 0, U0hu = 0, U0hv = 0;              // U0 of row r-3 (stage 2)
    if (MODE == 2) {
      U0h = p0h; U0hu = p0hu; U0hv = p0hv;
      const int jn = r - 2;
      if (outCol && jn >= y0 && jn < y1) {
        const int k = jn * W + gi;
        p0h = a.oh[k]; p0hu = a.ohu[k]; p0hv = a.ohv[k];
      }
    }
    double U_c = 0, V_c = 0;
    if (h_c == 0) {                 // +-0 / den == +-0 and NaN / den == NaN: no division needed
      U_c = vel_num(hu_c, h_c);
      V_c = vel_num(hv_c, h_c);
    } else {
      const double den = vel_den(h_c, eps4);
      U_c = qdiv(vel_num(hu_c, h_c), den);
      V_c = qdiv(vel_num(hv_c, h_c), den);
    }
    const int sr = (r + 4) & 3;     // ring slot of row r (r >= -3)
    s_b[sr][c] = b_c; s_h[sr][c] = h_c; s_U[sr][c] = U_c; s_V[sr][c] = V_c;
    s_hu[sr][c] = hu_c; s_hv[sr][c] = hv_c;

    // ---- S2: slopes and bed term of row r-1 --------------------------------
    const int j1 = r - 1;
    const int sr1 = (r + 3) & 3;    // slot of row r-1
    double xsE = 0, xsB = 0, xsU = 0, xsV = 0;
    double nsE = 0, nsB = 0, nsU = 0, nsV = 0;         // y slopes of row r-1
    if (order2 && j1 >= 1 && j1 < H - 1 && gi >= 1 && gi < W - 1 && c >= 1 && c < BX - 1) {
      const double hk = h_m1, bk = b_m1, eC = bk + hk, uk = U_m1, vk = V_m1;
      {   // d = 0 (x), neighbours from smem row r-1
        const double hp = s_h[sr1][c + 1], hm = s_h[sr1][c - 1];
        if (!(hk <= dry || hp <= dry || hm <= dry)) {
          const double bp = s_b[sr1][c + 1], bm = s_b[sr1][c - 1];
          const double eP = bp + hp, eM = bm + hm;
          xsE = limiter(a.lim, eC - eM, eP - eC);
          xsB = limiter(a.lim, bk - bm, bp - bk);
          xsU = limiter(a.lim, uk - s_U[sr1][c - 1], s_U[sr1][c + 1] - uk);
          xsV = limiter(a.lim, vk - s_V[sr1][c - 1], s_V[sr1][c + 1] - vk);
        }
      }
      {   // d = 1 (y), neighbours rows r-2 and r in registers
        const double hp = h_c, hm = h_m2;
        if (!(hk <= dry || hp <= dry || hm <= dry)) {
          const double eP = b_c + hp, eM = b_m2 + hm;
          nsE = limiter(a.lim, eC - eM, eP - eC);
          nsB = limiter(a.lim, bk - b_m2, b_c - bk);
          nsU = limiter(a.lim, uk - U_m2, U_c - uk);
          nsV = limiter(a.lim, vk - V_m2, V_c - vk);
        }
      }
    }
    const int xsr = (r + 4) & 1;    // slot of row r-1
    s_xs[xsr][0][c] = xsE; s_xs[xsr][1][c] = xsB; s_xs[xsr][2][c] = xsU; s_xs[xsr][3][c] = xsV;
    double tb0 = 0, tb1 = 0, tg = 0;
    if (bedOn && j1 >= 2 && j1 < H - 2 && interiorCol) {
      // src/swe.mjs:570-598
      const int m1 = j1 - mbase;
      const double bk = b_m1, eC = bk + h_m1;
      {
        const double hP = jmax0(eC + 0.5 * xsE - (bk + 0.5 * xsB));
        const double hM = jmax0(eC - 0.5 * xsE - (bk - 0.5 * xsB));
        tb0 = div_unless_zero(-SWE_G * 0.5 * (hP + hM) * xsB, xsB, s_m[M_DX][m1]);
      }
      {
        const double hP = jmax0(eC + 0.5 * nsE - (bk + 0.5 * nsB));
        const double hM = jmax0(eC - 0.5 * nsE - (bk - 0.5 * nsB));
        tb1 = div_unless_zero(-SWE_G * 0.5 * (hP + hM) * nsB, nsB, s_m[M_BED][m1]);
        if (sph) tg = s_m[M_GEO][m1] * SWE_G * (hP * hP + hM * hM);
      }
    }
    __syncthreads();

    // ---- S3: x face (c|c+1) of row r-1, y face (r-2|r-1) --------------------
    Face fx = {0, 0, 0, 0, 0};
    if (j1 >= 2 && j1 < H - 2 && gi >= 1 && gi < W - 2 && c < BX - 1 && j1 >= y0 - 1 && j1 <= y1) {
      fx = face_flux(b_m1, h_m1, U_m1, V_m1, xsE, xsB, xsU, xsV,
                     s_b[sr1][c + 1], s_h[sr1][c + 1], s_U[sr1][c + 1], s_V[sr1][c + 1],
                     s_xs[xsr][0][c + 1], s_xs[xsr][1][c + 1], s_xs[xsr][2][c + 1], s_xs[xsr][3][c + 1],
                     dry);
    }
    const int fsr = (r + 5) % 3;    // slot of row r-1
    s_fx[fsr][0][c] = fx.M; s_fx[fsr][1][c] = fx.N; s_fx[fsr][2][c] = fx.T;
    s_fx[fsr][3][c] = fx.pL; s_fx[fsr][4][c] = fx.pR;
    Face fy = {0, 0, 0, 0, 0};
    const int j2 = r - 2;
    if (j2 >= 1 && j2 < H - 2 && gi >= 2 && gi < W - 2 && j2 >= y0 - 2 && j2 <= y1) {
      // lower cell row r-2 (slopes ys*), upper cell row r-1 (slopes ns*); v is normal
      fy = face_flux(b_m2, h_m2, V_m2, U_m2, ysE, ysB, ysV, ysU,
                     b_m1, h_m1, V_m1, U_m1, nsE, nsB, nsV, nsU, dry);
    }

    // ---- S4: theta of row r-2 (src/swe.mjs:511-529) -------------------------
    double th = 1;
    if (dt > 0 && j2 >= 1 && j2 < H - 1 && gi >= 1 && gi < W - 1 && c >= 1 && c < BX - 1 &&
        j2 >= y0 - 1 && j2 <= y1) {
      const int f2 = (r + 4) % 3;   // slot of row r-2
      const int m2 = j2 - mbase;
      const double fxE = s_fx[f2][0][c], fxW = s_fx[f2][0][c - 1];
      const double fyN = fy.M, fyS = fy1.M;
      const double avail = h_m2;
      // The reference's out-budget is a sum of non-negative quotients.  The
      // same sum with reciprocal multiplies is within 1e-15 relative of it,
      // so when that estimate sits clearly below the water available the
      // limiter cannot fire and theta is 1 without forming the quotients.
      const double est = ((fxE > 0 ? fxE : 0) - (fxW < 0 ? fxW : 0)) * s_m[M_RDX][m2]
                       + (fyN > 0 ? fyN : 0) * s_m[M_RDYN][m2] - (fyS < 0 ? fyS : 0) * s_m[M_RDYS][m2];
      if (!(est * dt * (1 + 1e-12) < avail)) {
        double out = 0;
        if (fxE > 0) out += fxE / s_m[M_DX][m2];
        if (fxW < 0) out -= fxW / s_m[M_DX][m2];
        if (fyN > 0) out += fyN / s_m[M_DYN][m2];
        if (fyS < 0) out -= fyS / s_m[M_DYS][m2];
        if (out * dt > avail) th = avail > 0 ? avail / (out * dt) : 0;
      }
    }
    s_th[(r + 4) & 1][c] = th;      // slot of row r-2

    // ---- S5: accumulate + update row r-3 ------------------------------------
    const int j3 = r - 3;
    if (outCol && j3 >= y0 && j3 < y1) {
      const int k = j3 * W + gi;
      const int m3 = j3 - mbase;
      const int f3 = (r + 3) % 3;   // slot of row r-3
      const int ts = (r + 5) & 1;   // theta slot of row r-3
      const int s3 = (r + 1) & 3;   // state ring slot of row r-3
      double ah = 0, ahu = 0, ahv = 0;
      if (j3 >= 2 && j3 < H - 2) {
        // west face (c-1|c), cell is its right side
        if (gi - 1 >= 1 && gi - 1 < W - 2) {
          const double M = s_fx[f3][0][c - 1];
          const double thf = M >= 0 ? s_th[ts][c - 1] : th_m3;
          const double inv = thf == 1 ? s_m[M_RDX][m3] : thf / s_m[M_DX][m3];
          ah += M * inv; ahu += (s_fx[f3][1][c - 1] + s_fx[f3][4][c - 1]) * inv; ahv += s_fx[f3][2][c - 1] * inv;
        }
        // east face (c|c+1), cell is its left side
        if (gi >= 1 && gi < W - 2) {
          const double M = s_fx[f3][0][c];
          const double thf = M >= 0 ? th_m3 : s_th[ts][c + 1];
          const double inv = thf == 1 ? s_m[M_RDX][m3] : thf / s_m[M_DX][m3];
          ah -= M * inv; ahu -= (s_fx[f3][1][c] + s_fx[f3][3][c]) * inv; ahv -= s_fx[f3][2][c] * inv;
        }
      }
      if (gi >= 2 && gi < W - 2) {
        // south face (r-4|r-3), cell is its upper side
        if (j3 - 1 >= 1 && j3 - 1 < H - 2) {
          const double thf = fy2.M >= 0 ? th_m4 : th_m3;
          const double invR = thf == 1 ? s_m[M_RDYS][m3] : thf / s_m[M_DYS][m3];
          ah += fy2.M * invR; ahv += (fy2.N + fy2.pR) * invR; ahu += fy2.T * invR;
        }
        // north face (r-3|r-2), cell is its lower side
        if (j3 >= 1 && j3 < H - 2) {
          const double thf = fy1.M >= 0 ? th_m3 : th;
          const double invL = thf == 1 ? s_m[M_RDYN][m3] : thf / s_m[M_DYN][m3];
          ah -= fy1.M * invL; ahv -= (fy1.N + fy1.pL) * invL; ahu -= fy1.T * invL;
        }
      }
      const bool interior = interiorCol && j3 >= 2 && j3 < H - 2;
      const double hin = s_h[s3][c], huin = s_hu[s3][c], hvin = s_hv[s3][c];
      if (interior) {
        if (bedOn) {
          ahu += tb0_m3;
          ahv += tb1_m3;
          if (sph) ahv += tg_m3;
        }
        if (sph) {
          const double fe = s_m[M_F][m3] + s_U[s3][c] * (s_m[M_TAN][m3] / a.m.R);
          ahu += fe * hvin;
          ahv -= fe * huin;
        } else if (corOn) {
          ahu += a.coriolis * hvin;
          ahv -= a.coriolis * huin;
        }
      }
      if (MODE == 0) {
        a.rh[k] = ah; a.rhu[k] = ahu; a.rhv[k] = ahv; a.theta[k] = th_m3;
      } else if (MODE == 1) {
        double nh = hin + dt * ah, nhu = huin + dt * ahu, nhv = hvin + dt * ahv;
        if (interior) {                       // dryClean, src/swe.mjs:734-745
          if (nh < 0) { locFl -= nh; nh = 0; }
          if (nh <= dry) { nhu = 0; nhv = 0; }
        }
        a.oh[k] = nh; a.ohu[k] = nhu; a.ohv[k] = nhv;
      } else {
        const double h0 = U0h, hu0 = U0hu, hv0 = U0hv;   // U0 (in place)
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
            const int ii = gi - 2, jj = j3 - 2;
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
            const double sr5 = (u + cc) / s_m[M_DX][m3] + (v + cc) / s_m[M_CFL][m3];
            if (sr5 > locMax) locMax = sr5;
          }
        }
        a.oh[k] = nh; a.ohu[k] = nhu; a.ohv[k] = nhv;
      }
    }

    // ---- rotate ------------------------------------------------------------
    b_m2 = b_m1; h_m2 = h_m1; U_m2 = U_m1; V_m2 = V_m1;
    b_m1 = b_c; h_m1 = h_c; U_m1 = U_c; V_m1 = V_c;
    ysE = nsE; ysB = nsB; ysU = nsU; ysV = nsV;
    tb0_m3 = tb0_m2; tb1_m3 = tb1_m2; tg_m3 = tg_m2;   // bed terms computed at S2 are row r-1's
    tb0_m2 = tb0; tb1_m2 = tb1; tg_m2 = tg;
    fy2 = fy1; fy1 = fy;
    th_m4 = th_m3; th_m3 = th;
  }

  if constexpr (MODE != 0) {
    // ---- per-CTA partials, then the last CTA closes the step -----------------
    for (int o = 16; o > 0; o >>= 1) {
      locMax = fmax(locMax, __shfl_down_sync(0xffffffffu, locMax, o));
      locFl += __shfl_down_sync(0xffffffffu, locFl, o);
    }
    if ((c & 31) == 0) { s_red[0][c >> 5] = locMax; s_red[1][c >> 5] = locFl; }
    __syncthreads();
    __shared__ bool s_last;
    const int bid = part;
    if (c == 0) {
      double m = s_red[0][0], f = s_red[1][0];
      for (int w = 1; w < BX / 32; w++) { m = fmax(m, s_red[0][w]); f += s_red[1][w]; }
      if (MODE == 1) a.part_fl1[bid] = f;
      else { a.part_max[bid] = m; a.part_fl2[bid] = f; }
      __threadfence();
      const unsigned int ticket = atomicAdd(&ctl->counter, 1u);
      s_last = (ticket == (unsigned int)(a.nblocks - 1));
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (c == 0) {
      if (MODE == 1) {
        double f = 0;
        for (int q = 0; q < a.nblocks; q++) f += ((volatile double*)a.part_fl1)[q];
        ctl->floored1 = f;
      } else {
        double m = 0, f = 0;
        for (int q = 0; q < a.nblocks; q++) {
          m = fmax(m, ((volatile double*)a.part_max)[q]);
          f += ((volatile double*)a.part_fl2)[q];
        }
        ctl->next_max = m;
        ctl->mass_floored = ctl->floored1 + f;
        ctl->t = ctl->t + dt;
        ctl->steps = ctl->steps + 1;
      }
      ctl->counter = 0;
    }
  }
}

// The single-grid stage kernel: a 2D grid of tiles over one simulation.
template <int MODE>
__global__ void __launch_bounds__(BX, SWE_STAGE_MIN_BLOCKS) k_stage(StageArgs a, Control* ctl) {
  extern __shared__ double smem[];                                   // STAGE_SMEM_BYTES
  const int RY = (a.H + gridDim.y - 1) / gridDim.y;
  const int y0 = (int)blockIdx.y * RY;
  stage_tile<MODE>(a, ctl, blockIdx.x, y0, min(y0 + RY, a.H), blockIdx.y * gridDim.x + blockIdx.x, smem);
}

// ---------------------------------------------------------------------------
// Reductions and diagnostics.

// The last block's combine of the grid's per-block partials (a maximum, or
// a sum of whole numbers: exact in any order) by all of its threads, at L2
// (the other blocks wrote them); the result in thread 0.  One thread reading
// 16 384 partials in turn took most of a 0.49 ms launch.
__device__ __forceinline__ double combine_parts(const double* part, int n, bool sum, double* s_red) {
  double mm = 0;
  for (int q = threadIdx.x; q < n; q += blockDim.x) {
    const double x = __ldcg(part + q);
    mm = sum ? mm + x : fmax(mm, x);
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double x = __shfl_down_sync(0xffffffffu, mm, o);
    mm = sum ? mm + x : fmax(mm, x);
  }
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = mm;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int w = 1; w < (int)blockDim.x / 32; w++) mm = sum ? mm + s_red[w] : fmax(mm, s_red[w]);
  return mm;
}

// CFL rate max over wet interior cells (src/swe.mjs:632-647) -> ctl->next_max.
__global__ void k_cfl_rate(StageArgs a, Control* ctl, double* part) {
  __shared__ double s[BX / 32];
  __shared__ bool s_last;
  double m = 0;
  const int nx = a.nx, ny = a.ny, W = a.W;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nx * ny; q += gridDim.x * blockDim.x) {
    const int j = q / nx + 2, i = q % nx + 2, k = j * W + i;
    const double hk = a.h[k];
    if (hk <= a.minDepth) continue;
    const double cc = sqrt(SWE_G * hk);
    const double den = vel_den(hk, a.eps4);
    const double u = fabs(qdiv(vel_num(a.hu[k], hk), den)), v = fabs(qdiv(vel_num(a.hv[k], hk), den));
    const double sr = (u + cc) / a.m.dxRow[j] + (v + cc) / a.m.dyCFL[j];
    if (sr > m) m = sr;
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = s[0];
    for (int w = 1; w < (int)blockDim.x / 32; w++) mm = fmax(mm, s[w]);
    part[blockIdx.x] = mm;
    __threadfence();
    s_last = atomicAdd(&ctl->counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;                            // uniform per block
  __threadfence();
  const double mm = combine_parts(part, gridDim.x, false, s);
  if (threadIdx.x == 0) {
    ctl->next_max = mm;
    ctl->counter = 0;
  }
}

// dryClean over the interior alone (src/swe.mjs:734-745); sequential order
// for the floored sum, as the reference.
// Interior cells in the reference's row-major order, CHAIN_CELLS at a time,
// for the sums whose order is one running sum over every cell: the block
// stages a chunk into shared memory (coalesced within each row) while its
// first thread adds the previous chunk left to right.
constexpr int CHAIN_THREADS = 256, CHAIN_CELLS = 4 * CHAIN_THREADS;
__device__ __forceinline__ int chain_cell(const StageArgs& a, int q) {
  const int j = q / a.nx;
  return (j + 2) * a.W + (q - j * a.nx) + 2;
}

// dryClean() (src/swe.mjs:734-745): every cell's update in parallel; the
// floored mass is the running sum of -h over the floored cells in row-major
// order, which is the reference's sum (its other cells add nothing).  A
// chunk with no floored cell costs the first thread nothing.
__global__ void __launch_bounds__(CHAIN_THREADS) k_dry_clean(StageArgs a, Control* ctl) {
  __shared__ double buf[CHAIN_CELLS];
  const int n = a.nx * a.ny, t = threadIdx.x;
  double added = 0;
  for (int c0 = 0; c0 < n; c0 += CHAIN_CELLS) {
    int mine = 0;
    for (int r = 0; r < 4; r++) {
      const int q = c0 + r * CHAIN_THREADS + t;
      double add = 0;
      if (q < n) {
        const int k = chain_cell(a, q);
        double h = a.oh[k];
        if (h < 0) { add = -h; h = 0; a.oh[k] = 0; mine = 1; }
        if (h <= a.minDepth) { a.ohu[k] = 0; a.ohv[k] = 0; }
      }
      buf[r * CHAIN_THREADS + t] = add;
    }
    if (__syncthreads_or(mine) && t == 0) {
      const int m = min(CHAIN_CELLS, n - c0);
      for (int q = 0; q < m; q++)
        if (buf[q] != 0) added += buf[q];
    }
    __syncthreads();
  }
  if (t == 0) ctl->diag = added;
}

// The Cartesian volume() (src/swe.mjs:818-827): one running sum of h over
// every interior cell in row-major order, then one multiply by dx and dy.
// The order is the reference's exactly; the chunks of the next iteration are
// loaded by the whole block while the first thread adds.
__global__ void __launch_bounds__(CHAIN_THREADS) k_volume_chain(StageArgs a, double dx, double dy, Control* ctl) {
  __shared__ double buf[2][CHAIN_CELLS];
  const int n = a.nx * a.ny, t = threadIdx.x;
  const int chunks = (n + CHAIN_CELLS - 1) / CHAIN_CELLS;
  auto stage = [&](int c) {
    for (int r = 0; r < 4; r++) {
      const int q = c * CHAIN_CELLS + r * CHAIN_THREADS + t;
      buf[c & 1][r * CHAIN_THREADS + t] = q < n ? a.h[chain_cell(a, q)] : 0.0;
    }
  };
  double v = 0;
  if (chunks > 0) stage(0);
  __syncthreads();
  for (int c = 0; c < chunks; c++) {
    if (c + 1 < chunks) stage(c + 1);
    if (t == 0) {
      const int m = min(CHAIN_CELLS, n - c * CHAIN_CELLS);
      const double* b = buf[c & 1];
      for (int q = 0; q < m; q++) v += b[q];
    }
    __syncthreads();
  }
  if (t == 0) ctl->diag = v * dx * dy;
}

// applyFriction alone (src/swe.mjs:659-704).
__global__ void k_friction(StageArgs a, double dt) {
  const int nx = a.nx, ny = a.ny, W = a.W;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nx * ny; q += gridDim.x * blockDim.x) {
    const int k = (q / nx + 2) * W + (q % nx + 2);
    const double hk = a.oh[k];
    const double n = a.nfield ? a.nfield[k] : a.manning;
    if (!a.nfield && !(n != 0 && n == n)) return;
    if (hk <= a.minDepth) { a.ohu[k] = 0; a.ohv[k] = 0; continue; }
    if (!(n != 0 && n == n)) continue;
    const double den = vel_den(hk, a.eps4);
    const double u = qdiv(vel_num(a.ohu[k], hk), den), v = qdiv(vel_num(a.ohv[k], hk), den);
    const double speed = hypot(u, v);
    if (speed < 1e-14) continue;
    const double denom = 1 + dt * SWE_G * n * n * speed / pow43(hk);
    a.ohu[k] = qdiv(a.ohu[k], denom);
    a.ohv[k] = qdiv(a.ohv[k], denom);
  }
}

// Per-row sums in the reference's order (each row left to right from +0),
// one warp per row: the lanes load 32 consecutive cells of the row at a time
// (coalesced) and form each cell's term, lane 0 adds the 32 terms in order.
// what: 0 h (volume, src/swe.mjs:829-834), 1 the energy term
// (:862-877), 2 b + h (the eta projection of src/globe.mjs:1414-1421).
// A cell the energy skips (h <= 0) adds +0 here, which leaves a sum that
// started at +0 unchanged bit for bit (it can never be -0).
constexpr int ROWSUM_WARPS = 4;
__global__ void __launch_bounds__(32 * ROWSUM_WARPS) k_row_sums(StageArgs a, int what, double* rows) {
  __shared__ double buf[ROWSUM_WARPS][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int j = blockIdx.x * ROWSUM_WARPS + w;
  if (j >= a.ny) return;                            // the whole warp
  const size_t base = (size_t)(j + 2) * a.W + 2;
  double row = 0;
  for (int i0 = 0; i0 < a.nx; i0 += 32) {
    const int i = i0 + lane;
    double term = 0;
    if (i < a.nx) {
      const size_t k = base + i;
      const double hk = a.h[k];
      if (what == 0) term = hk;
      else if (what == 2) term = a.b[k] + hk;
      else if (!(hk <= 0)) {
        const double den = vel_den(hk, a.eps4);
        const double u = qdiv(vel_num(a.hu[k], hk), den), v = qdiv(vel_num(a.hv[k], hk), den);
        term = 0.5 * hk * (u * u + v * v) + 0.5 * SWE_G * hk * (hk + 2 * a.b[k]);
      }
    }
    buf[w][lane] = term;
    __syncwarp();
    if (lane == 0) {
      const int m = min(32, a.nx - i0);
      for (int q = 0; q < m; q++) row += buf[w][q];
    }
    __syncwarp();
  }
  if (lane == 0) rows[j] = row;
}

// The rows summed in order: mode 0 sum rows[j] * w[j] (the sphere's volume
// and energy with w = area, src/swe.mjs:829-836, 875), mode 1 (sum rows) *
// dx * dy (the Cartesian energy, :876; the Cartesian volume in the row
// order), mode 2 sum w[j] * rows[j] with the caller's weights (the
// projection).  One thread: ny terms.
__global__ void k_finish_sum(const double* rows, int ny, int mode, const double* w, double dx, double dy,
                             Control* ctl) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double v = 0;
  for (int j = 0; j < ny; j++) {
    if (mode == 1) v += rows[j];
    else v += rows[j] * w[j];
  }
  ctl->diag = mode == 1 ? v * dx * dy : v;
}

// what: 0 maxSurfaceDeviation(ref) (src/swe.mjs:880-892), 1 maxSpeed (:895-907),
// 2 finite count of non-finite cells over all N (:912-917).
__global__ void k_max_diag(StageArgs a, int what, double ref, double* part, Control* ctl) {
  __shared__ double s[BX / 32];
  __shared__ bool s_last;
  double m = 0;
  const int nx = a.nx, ny = a.ny, W = a.W;
  const int total = what == 2 ? a.W * a.H : nx * ny;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += gridDim.x * blockDim.x) {
    if (what == 2) {
      if (!isfinite(a.h[q]) || !isfinite(a.hu[q]) || !isfinite(a.hv[q])) m += 1;
      continue;
    }
    const int k = (q / nx + 2) * W + (q % nx + 2);
    const double hk = a.h[k];
    if (hk <= a.minDepth) continue;
    double d;
    if (what == 0) d = fabs(a.b[k] + hk - ref);
    else {
      const double den = vel_den(hk, a.eps4);
      d = hypot(qdiv(vel_num(a.hu[k], hk), den), qdiv(vel_num(a.hv[k], hk), den));
    }
    if (d > m) m = d;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double x = __shfl_down_sync(0xffffffffu, m, o);
    m = what == 2 ? m + x : fmax(m, x);
  }
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = s[0];
    for (int w = 1; w < (int)blockDim.x / 32; w++) mm = what == 2 ? mm + s[w] : fmax(mm, s[w]);
    part[blockIdx.x] = mm;
    __threadfence();
    s_last = atomicAdd(&ctl->counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;                            // uniform per block
  __threadfence();
  const double mm = combine_parts(part, gridDim.x, what == 2, s);
  if (threadIdx.x == 0) {
    ctl->diag = mm;
    ctl->counter = 0;
  }
}

// Standalone hllc over a batch (the reference exports hllc for direct calls,
// src/swe.mjs:975).  in: 7 doubles per case (hL huL hvL hR huR hvR dry).
__global__ void k_hllc_batch(int n, const double* in, double* out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const double* p = in + 7 * q;
  double o0, o1, o2;
  hllc(o0, o1, o2, p[0], p[1], p[2], p[3], p[4], p[5], p[6]);
  out[3 * q] = o0; out[3 * q + 1] = o1; out[3 * q + 2] = o2;
}

__global__ void k_vel_batch(int n, const double* hq, const double* h, double eps4, double* out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  out[q] = vel(hq[q], h[q], eps4);
}

}  // namespace
}  // namespace swe
