// swe_api.cu -- host side of libswe_b200.so: the C ABI declared in
// include/swe_b200.h.  Owns device buffers and one CUDA stream per
// simulation, sets up the metric (src/geometry.mjs), and sequences the
// kernels of swe_kernels.cuh.  No CPU solver path exists here: every field
// update runs on the GPU.
#include "../../include/swe_b200.h"
#include "swe_kernels.cuh"
#include "swe_split.cuh"

#include <cuda_runtime.h>
#include <cudaTypedefs.h>        // PFN_cuTensorMapEncodeTiled (fetched through the runtime, no -lcuda)
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstddef>
#include <cstdlib>
#include <string>
#include <vector>
#include <algorithm>

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) { g_err = msg; return code; }

#define CU(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return fail(SWE_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

const double PI = 3.141592653589793;
const double HALF_PI = PI / 2;

// ---- metric, src/geometry.mjs ------------------------------------------------
double js_max(double a, double b) { return swe::jmax(a, b); }
double js_min(double a, double b) { return swe::jmin(a, b); }
double clamp_lat(double p) { return p > HALF_PI ? HALF_PI : p < -HALF_PI ? -HALF_PI : p; }      // :111
double reflect_lat(double p) { return p > HALF_PI ? PI - p : p < -HALF_PI ? -PI - p : p; }    // :112
double cos_lat(double p) {                                                                     // :153
  const double co = HALF_PI - std::fabs(p);
  return co <= 0 ? 0 : std::sin(co);
}

}  // namespace

// The tiled pair measured faster than the fused kernel on every workload
// tried (2048^2 beach and all-wet, 1024^2, the 1440x720 sphere), with the
// same results bit for bit.
#ifndef SWE_DEFAULT_STAGE
#define SWE_DEFAULT_STAGE 1
#endif

namespace swe_host {
// Lets the other translation unit of the library report through swe_last_error().
void set_error(const std::string& msg) { g_err = msg; }
}  // namespace swe_host

struct swe_sim {
  swe_options o;
  int nx, ny, W, H, N;
  double dx, dy, eps4, R, dlam, dphi, totalArea;
  std::vector<double> geom[SWE_GEOM_NROWS];
  std::vector<double> recip[3];
  int dryfold = 0;                                 // every reciprocal row finite
  cudaStream_t st = nullptr;
  double* d_b = nullptr;
  double* d_A[3] = {nullptr, nullptr, nullptr};
  double* d_B[3] = {nullptr, nullptr, nullptr};
  double* d_h0[3] = {nullptr, nullptr, nullptr};
  double* d_res[4] = {nullptr, nullptr, nullptr, nullptr};
  double* d_nfield = nullptr;
  double* d_geom = nullptr;
  double* d_part = nullptr;
  double* d_rows = nullptr;
  double* d_coef = nullptr;                        // weights of swe_eta_projection (ny)
  int diag_order = SWE_DIAG_REFERENCE;
  double* d_sponge = nullptr;
  swe::Control* d_ctl = nullptr;
  int bc[4];
  int fl_kind[4] = {0, 0, 0, 0};
  double fl_eta[4] = {0, 0, 0, 0}, fl_u[4] = {0, 0, 0, 0};
  int sponge_side = 1, sponge_width = 0;
  double sponge_ref = 0;
  bool keep_h0 = false;
  bool cfl_valid = false;
  double t = 0, steps = 0;        // host mirror of the device clock
  bool clock_valid = true;
  dim3 grid;
  int nblocks = 0;
  int part_cap = 0;
  // device-resident loop graph
  // stage kernels: 0 the fused row-marching kernel, 1 the two tiled kernels
  int stage_impl = 0;
  int pdl = 1;                                     // programmatic dependent launch in the stepping loop
  double* d_split = nullptr;
  int* d_odry[2] = {nullptr, nullptr};             // per tile of A / B: all h == 0 (swe_split.cuh)
  swe::TileMaps tmaps[2];                          // the face kernel's tensor maps over A and B
  int tma = 0;                                     // 1: they are in use
  swe::CellMaps cmaps[2];                          // the cell kernel's, per stage
  int cell_tma = 0;                                // 1: they are in use
  int* d_flist = nullptr;                          // the face kernel's tile list and its two counters
  int* d_fcount = nullptr;
  int* d_clist = nullptr;                          // the cell kernel's tile list and its two counters
  int* d_ccount = nullptr;
  int face_list = 0;                               // 1: the face kernel takes the list
  swe::SplitBufs sb;
  dim3 sgrid;
  // Whether the tiled cell kernels may settle dry tiles (swe_split.cuh).
  // A swe_run of 128 steps or more keeps it on after its first chunk only
  // when a quarter or more of the tiles settled there, and remembers the
  // choice (settle_pref) for shorter runs; grids with little dry land run
  // the plain kernel faster.  The single-step entry points always settle.
  int settle = 1, settle_pref = 1;
  // device-resident loop graphs, one per value of `settle`
  struct LoopGraph {
    cudaGraphExec_t exec = nullptr;
    int steps = 0, mode = -1;
    double dt = 0, tend = 0;
    unsigned long long version = 0;
  } graphs[2];
  unsigned long long version = 1;
};

namespace {
// The state was written outside a stage: no tile is known dry any more.
int forget_dry(swe_sim* s) {
  if (!s->d_odry[0]) return SWE_OK;
  const size_t bytes = sizeof(int) * (size_t)s->sgrid.x * s->sgrid.y;
  CU(cudaMemsetAsync(s->d_odry[0], 0, bytes, s->st));
  CU(cudaMemsetAsync(s->d_odry[1], 0, bytes, s->st));
  return SWE_OK;
}
}  // namespace

namespace swe_host {
cudaStream_t stream_of(swe_sim* s) { return s->st; }

// Take b, h (and a Manning field, or none) from device arrays over the padded
// grid, in the handle's stream; used by importers that build the fields on
// the device.
int adopt_fields(swe_sim* s, const double* d_b, const double* d_h, const double* d_n) {
  const size_t nb = sizeof(double) * (size_t)s->N;
  cudaError_t e = cudaMemcpyAsync(s->d_b, d_b, nb, cudaMemcpyDeviceToDevice, s->st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_A[0], d_h, nb, cudaMemcpyDeviceToDevice, s->st);
  if (e == cudaSuccess && d_n) {
    if (!s->d_nfield) e = cudaMalloc(&s->d_nfield, nb);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_nfield, d_n, nb, cudaMemcpyDeviceToDevice, s->st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  if (e != cudaSuccess) { set_error(std::string("adopt_fields: ") + cudaGetErrorString(e)); return SWE_ECUDA; }
  if (forget_dry(s)) return SWE_ECUDA;
  s->version++;
  s->cfl_valid = false;
  return SWE_OK;
}
}  // namespace swe_host

namespace {

void cartesian_geometry(swe_sim* s) {            // src/geometry.mjs:163-176
  s->R = INFINITY; s->dlam = 0; s->dphi = 0;
  s->totalArea = s->nx * s->dx * s->ny * s->dy;
  for (int j = 0; j < s->H; j++) {
    s->geom[SWE_GEOM_DXROW][j] = s->dx;
    s->geom[SWE_GEOM_DYROWN][j] = s->dy;
    s->geom[SWE_GEOM_DYROWS][j] = s->dy;
    s->geom[SWE_GEOM_DYCFL][j] = s->dy;
    s->geom[SWE_GEOM_BEDPHI][j] = s->dy;
    s->geom[SWE_GEOM_AREA][j] = s->dx * s->dy;
    s->geom[SWE_GEOM_LX][j] = s->dy;
    s->geom[SWE_GEOM_LYN][j] = s->dx;
    s->geom[SWE_GEOM_LYS][j] = s->dx;
    s->geom[SWE_GEOM_FROW][j] = s->o.coriolis;
  }
}

int spherical_geometry(swe_sim* s) {             // src/geometry.mjs:190-299
  const int nx = s->nx, ny = s->ny;
  const double R = s->o.R, lat0 = s->o.lat0, lat1 = s->o.lat1, omega = s->o.omega;
  char buf[256];
  if (!(lat1 > lat0)) {
    std::snprintf(buf, sizeof buf, "lat1 (%.17g) must exceed lat0 (%.17g)", lat1, lat0);
    return fail(SWE_EINVAL, buf);
  }
  if (lat0 < -90 || lat1 > 90) {
    std::snprintf(buf, sizeof buf, "latitudes must lie in [-90, 90]; got %.17g..%.17g", lat0, lat1);
    return fail(SWE_EINVAL, buf);
  }
  const bool touches_pole = lat0 <= -90 + 1e-12 || lat1 >= 90 - 1e-12;
  if (touches_pole && nx % 2 != 0) {
    std::snprintf(buf, sizeof buf,
                  "nx must be even when the domain reaches a pole (got %d): a ghost row beyond the "
                  "pole is the row half a turn away in longitude.", nx);
    return fail(SWE_EINVAL, buf);
  }
  const double dlam = 2 * PI / nx;
  const double p0 = lat0 * PI / 180, p1 = lat1 * PI / 180;
  const double dphi = (p1 - p0) / ny;
  s->R = R; s->dlam = dlam; s->dphi = dphi;
  const double gdy = R * dphi;
  s->dy = gdy;
  s->totalArea = 2 * PI * R * R * (std::sin(p1) - std::sin(p0));
  for (int j = 0; j < s->H; j++) {
    const int jj = j - 2;
    // face latitudes; the domain edges are pinned exactly (src/geometry.mjs:216)
    const double rawS = jj == 0 ? p0 : jj == ny ? p1 : p0 + jj * dphi;
    const double rawN = jj + 1 == 0 ? p0 : jj + 1 == ny ? p1 : p0 + (jj + 1) * dphi;
    const double pS = clamp_lat(rawS), pN = clamp_lat(rawN);
    const double pC = 0.5 * (pS + pN);
    const double half = 0.5 * (pN - pS);
    const double lyS = R * dlam * cos_lat(pS);
    const double lyN = R * dlam * cos_lat(pN);
    const double lx = R * dphi;
    double A = 2 * R * R * dlam * cos_lat(pC) * std::sin(half);
    if (!(A > 0)) {
      const double rS = reflect_lat(rawS), rN = reflect_lat(rawN);
      A = std::fabs(2 * R * R * dlam * cos_lat(0.5 * (rS + rN)) * std::sin(0.5 * (rN - rS)));
    }
    s->geom[SWE_GEOM_PHIC][j] = pC;
    s->geom[SWE_GEOM_LYS][j] = lyS;
    s->geom[SWE_GEOM_LYN][j] = lyN;
    s->geom[SWE_GEOM_LX][j] = lx;
    s->geom[SWE_GEOM_AREA][j] = A;
    s->geom[SWE_GEOM_DXROW][j] = A / lx;
    const double dN = lyN > 0 ? A / lyN : INFINITY;
    const double dS = lyS > 0 ? A / lyS : INFINITY;
    s->geom[SWE_GEOM_DYROWN][j] = dN;
    s->geom[SWE_GEOM_DYROWS][j] = dS;
    s->geom[SWE_GEOM_DYCFL][j] = js_min(js_min(dN, dS), gdy);
    s->geom[SWE_GEOM_BEDPHI][j] = (lyN + lyS) > 0 ? 2 * A / (lyN + lyS) : INFINITY;
    s->geom[SWE_GEOM_TANPHI][j] = std::tan(pC);
    s->geom[SWE_GEOM_FROW][j] = 2 * omega * std::sin(pC);
    s->geom[SWE_GEOM_GEOCOEF][j] = (lyN - lyS) / (4 * A);
  }
  for (int j = 0; j < s->H; j++) {
    const double a = s->geom[SWE_GEOM_AREA][j];
    if (!(a > 0) || !std::isfinite(a)) {
      std::snprintf(buf, sizeof buf, "row %d: area %.17g", j, a);
      return fail(SWE_EINVAL, buf);
    }
    if (!(s->geom[SWE_GEOM_LYN][j] >= 0) || !(s->geom[SWE_GEOM_LYS][j] >= 0)) {
      std::snprintf(buf, sizeof buf, "row %d: negative face length", j);
      return fail(SWE_EINVAL, buf);
    }
  }
  return SWE_OK;
}

swe::Metric metric(const swe_sim* s) {
  swe::Metric m;
  const double* g = s->d_geom;
  const int H = s->H;
  m.dxRow = g + SWE_GEOM_DXROW * H; m.dyRowN = g + SWE_GEOM_DYROWN * H;
  m.dyRowS = g + SWE_GEOM_DYROWS * H; m.dyCFL = g + SWE_GEOM_DYCFL * H;
  m.bedPhi = g + SWE_GEOM_BEDPHI * H; m.geoCoef = g + SWE_GEOM_GEOCOEF * H;
  m.fRow = g + SWE_GEOM_FROW * H; m.tanPhi = g + SWE_GEOM_TANPHI * H;
  m.rdxRow = g + (SWE_GEOM_NROWS + 0) * H; m.rdyRowN = g + (SWE_GEOM_NROWS + 1) * H;
  m.rdyRowS = g + (SWE_GEOM_NROWS + 2) * H;
  m.R = s->R;
  return m;
}

// StageArgs reading `in` and writing `out`.
swe::StageArgs stage_args(const swe_sim* s, double* const* in, double* const* out) {
  swe::StageArgs a;
  std::memset(&a, 0, sizeof a);
  a.W = s->W; a.H = s->H; a.nx = s->nx; a.ny = s->ny;
  a.b = s->d_b;
  a.h = in[0]; a.hu = in[1]; a.hv = in[2];
  if (out) { a.oh = out[0]; a.ohu = out[1]; a.ohv = out[2]; }
  a.m = metric(s);
  a.minDepth = s->o.min_depth; a.eps4 = s->eps4; a.coriolis = s->o.coriolis;
  a.sph = s->o.sphere; a.order = s->o.order; a.lim = s->o.limiter;
  a.manning = s->o.manning; a.nfield = s->d_nfield;
  a.sponge_side = s->sponge_side; a.sponge_width = s->sponge_width;
  a.sponge_str = s->d_sponge; a.sponge_ref = s->sponge_ref;
  a.part_max = s->d_part; a.part_fl1 = s->d_part + s->part_cap; a.part_fl2 = s->d_part + 2 * s->part_cap;
  a.nblocks = s->nblocks;
  a.dryfold = s->dryfold;
  return a;
}

swe::BCArgs bc_args(const swe_sim* s, double* const* f) {
  swe::BCArgs a;
  a.nx = s->nx; a.ny = s->ny; a.W = s->W; a.H = s->H;
  for (int q = 0; q < 4; q++) a.kind[q] = s->bc[q];
  a.minDepth = s->o.min_depth; a.eps4 = s->eps4;
  a.b = s->d_b; a.h = f[0]; a.hu = f[1]; a.hv = f[2];
  return a;
}

swe::PrepArgs prep_args(const swe_sim* s, int mode, double dt, double t_end, const double* dt_dev = nullptr) {
  swe::PrepArgs p;
  p.mode = mode; p.dt_host = dt; p.cfl = s->o.cfl; p.t_end = t_end; p.dt_dev = dt_dev;
  for (int q = 0; q < 4; q++) { p.fl_kind[q] = s->fl_kind[q]; p.fl_eta[q] = s->fl_eta[q]; p.fl_u[q] = s->fl_u[q]; }
  return p;
}

int bc_blocks(const swe_sim* s) { return (4 * s->ny + 4 * (s->nx + 4) + 255) / 256; }

// A launch that, with `pdl`, may be scheduled before the previous kernel in
// the stream has finished (the kernel waits for it in pdl_enter).
template <typename... KArgs, typename... Args>
cudaError_t launch(bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

int launch_bc(swe_sim* s, double* const* f, int respect_stop, bool pdl = false) {
  CU(launch(pdl, swe::k_apply_bc, dim3(bc_blocks(s)), dim3(256), s->st, bc_args(s, f),
            (const swe::Control*)s->d_ctl, respect_stop));
  return SWE_OK;
}

// The driver's tensor-map encoder, or null; and whether the tile copies are
// on for this grid (SWE_B200_TMA=0 turns them off; a row stride that is not
// a multiple of 16 bytes cannot take them).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return nullptr;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  return encode;
}
bool tma_wanted(const swe_sim* s) {
  const char* env = std::getenv("SWE_B200_TMA");
  if (env && std::strcmp(env, "0") == 0) return false;
  return (sizeof(double) * (size_t)s->W) % 16 == 0;
}
// A 2-D map over one W x H field of doubles with the given box.
bool encode_field(PFN_cuTensorMapEncodeTiled_v12000 encode, const swe_sim* s, CUtensorMap* m, double* base,
                  int bx, int by) {
  const cuuint64_t dims[2] = {(cuuint64_t)s->W, (cuuint64_t)s->H};
  const cuuint64_t strides[1] = {(cuuint64_t)s->W * sizeof(double)};
  const cuuint32_t box[2] = {(cuuint32_t)bx, (cuuint32_t)by};
  const cuuint32_t estr[2] = {1, 1};
  return encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The cell kernel's maps: the face fields (one set of buffers for both
// stages) and the stage input's depth.
void make_cell_maps(swe_sim* s) {
  s->cell_tma = 0;
  if (!s->d_split || !tma_wanted(s)) return;
  PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  if (!encode) return;
  using swe::SPX;
  using swe::SPY;
  for (int st = 0; st < 2; st++) {
    swe::CellMaps& c = s->cmaps[st];
    bool ok = encode_field(encode, s, &c.m[swe::CM_XM], s->sb.fx[swe::F_M], SPX + 4, SPY + 2) &&
              encode_field(encode, s, &c.m[swe::CM_YM], s->sb.fy[swe::F_M], SPX + 4, SPY + 3) &&
              encode_field(encode, s, &c.m[swe::CM_H], st == 0 ? s->d_A[0] : s->d_B[0], SPX + 4, SPY + 2);
    for (int q = 0; q < 3 && ok; q++)
      ok = encode_field(encode, s, &c.m[swe::CM_XT + q], s->sb.fx[q + 1], SPX + 2, SPY) &&
           encode_field(encode, s, &c.m[swe::CM_YT + q], s->sb.fy[q + 1], SPX, SPY + 1) &&
           encode_field(encode, s, &c.m[swe::CM_TB + q], s->sb.tb[q], SPX, SPY);
    if (!ok) return;
  }
  s->cell_tma = 1;
}

// Tensor maps of the face kernel's state tile (swe_split.cuh, TileMaps):
// b, h, hu, hv of A (stage 1's input) and of B (stage 2's), each a 2-D
// W x H array of doubles, box SSXT x SSY, zeros outside.  A row stride that
// is not a multiple of 16 bytes (odd W), a driver without the encoder, or
// SWE_B200_TMA=0 leaves the per-element copies in use (the same bits).
void make_tile_maps(swe_sim* s) {
  s->tma = 0;
  if (!tma_wanted(s)) return;
  PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  if (!encode) return;
  double* src[2][4] = {{s->d_b, s->d_A[0], s->d_A[1], s->d_A[2]}, {s->d_b, s->d_B[0], s->d_B[1], s->d_B[2]}};
  for (int st = 0; st < 2; st++)
    for (int f = 0; f < 4; f++)
      if (!encode_field(encode, s, &s->tmaps[st].m[f], src[st][f], swe::SSXT, swe::SSY)) return;
  s->tma = 1;
}

// One SSP-RK2 step on the device; `mode`/`dt`/`t_end` as k_prepare.
// Buffers of the tiled stage kernels (faces and source terms).
int ensure_split(swe_sim* s) {
  if (s->d_split) return SWE_OK;
  const size_t N = s->N;
  const size_t ntiles = (size_t)s->sgrid.x * s->sgrid.y;
  // + three int flags per tile, and the face and cell kernels' tile lists
  // with two counters each
  const size_t doubles = swe::SPLIT_FIELDS * N + 3 * ((ntiles + 1) / 2) + (ntiles + 2);
  CU(cudaMalloc(&s->d_split, sizeof(double) * doubles));
  CU(cudaMemsetAsync(s->d_split, 0, sizeof(double) * doubles, s->st));
  s->sb = swe::split_bufs_at(s->d_split, N);
  s->sb.dry = reinterpret_cast<int*>(s->d_split + swe::SPLIT_FIELDS * N);
  s->sb.ntx = (int)s->sgrid.x;
  s->sb.nty = (int)s->sgrid.y;
  s->d_odry[0] = reinterpret_cast<int*>(s->d_split + swe::SPLIT_FIELDS * N + (ntiles + 1) / 2);
  s->d_odry[1] = reinterpret_cast<int*>(s->d_split + swe::SPLIT_FIELDS * N + 2 * ((ntiles + 1) / 2));
  s->d_flist = reinterpret_cast<int*>(s->d_split + swe::SPLIT_FIELDS * N + 3 * ((ntiles + 1) / 2));
  s->d_fcount = s->d_flist + ntiles;                // [2]
  s->d_clist = s->d_fcount + 2;
  s->d_ccount = s->d_clist + ntiles;               // [2]
  make_cell_maps(s);
  // The face kernel led by a tile list (swe_split.cuh, k_face_list), with
  // the tensor-map copies; SWE_B200_FACE_LIST=0 keeps every CTA testing its
  // own tile (the same bits).
  const char* fl = std::getenv("SWE_B200_FACE_LIST");
  s->face_list = s->tma && !(fl && std::strcmp(fl, "0") == 0) ? 1 : 0;
  return SWE_OK;
}


// The stage kernels' buffers of stage MODE (stage 1: A -> B, stage 2: B -> A).
template <int MODE>
swe::SplitBufs stage_bufs(const swe_sim* s) {
  swe::SplitBufs sb = s->sb;
  sb.odry_in = s->d_odry[MODE == 1 ? 0 : 1];
  sb.odry_out = s->d_odry[MODE == 1 ? 1 : 0];
  return sb;
}
// The tile lists pay where tiles settle: with the settling cell kernel
// (which swe_run keeps only where a quarter or more of the tiles settle).
bool stage_listed(const swe_sim* s) { return s->stage_impl == 1 && s->face_list && s->settle; }
// Whether the cell kernel takes its list: when tiles may be left out.
int cell_listed(const swe_sim* s, const swe::StageArgs& a) {
  return stage_listed(s) && s->cell_tma && a.dryfold && a.minDepth >= 0 && a.sponge_width <= 0 && !a.h0c &&
         !a.tape_th && !a.tape_hpre && !a.tape_pre[0];
}
template <int MODE>
swe::TileLists tile_lists(const swe_sim* s, const swe::StageArgs& a) {
  swe::TileLists L;
  L.list = s->d_flist; L.count = s->d_fcount + (MODE - 1); L.other_count = s->d_fcount + (2 - MODE);
  L.cell_skip = cell_listed(s, a);
  L.clist = s->d_clist; L.ccount = s->d_ccount + (MODE - 1); L.other_ccount = s->d_ccount + (2 - MODE);
  L.W = s->W; L.H = s->H;
  return L;
}

// One stage (MODE 1 or 2) with the selected kernels; list_done: its lists
// were made with the ghost fill (launch_bc_lists).
template <int MODE>
int launch_stage(swe_sim* s, const swe::StageArgs& a, bool pdl = false, bool list_done = false) {
  if (s->stage_impl == 1) {
    const swe::SplitBufs sb = stage_bufs<MODE>(s);
    const dim3 blk(swe::SP_THREADS);
    const bool listed = stage_listed(s);
    const int cell_list = cell_listed(s, a);
    if (listed) {
      const int ntiles = (int)(s->sgrid.x * s->sgrid.y);
      if (!list_done)
        CU(launch(pdl, swe::k_face_list, dim3((s->sgrid.x + swe::LX - 1) / swe::LX, (s->sgrid.y + swe::LY - 1) / swe::LY),
                  dim3(swe::LX * swe::LY), s->st, sb, s->d_ctl, tile_lists<MODE>(s, a)));
      CU(launch(pdl, swe::k_split_faces_tma_list, dim3(ntiles), blk, s->st, a, sb, s->d_ctl,
                s->tmaps[MODE - 1], (const int*)s->d_flist, (const int*)(s->d_fcount + (MODE - 1))));
    } else if (s->tma) {
      CU(launch(pdl, swe::k_split_faces_tma, s->sgrid, blk, s->st, a, sb, s->d_ctl, s->tmaps[MODE - 1]));
    }
    else CU(launch(pdl, swe::k_split_faces, s->sgrid, blk, s->st, a, sb, s->d_ctl));
    if (cell_list) {                               // only when tiles may be left out
      const swe::CellMaps& cm = s->cmaps[MODE - 1];
      const int ntiles = (int)(s->sgrid.x * s->sgrid.y);
      const int* cl = s->d_clist;
      const int* cc = s->d_ccount + (MODE - 1);
      if (s->settle) CU(launch(pdl, swe::k_split_cells_tma_list<MODE, true>, dim3(ntiles), blk, s->st, a, sb, s->d_ctl, cm, cl, cc));
      else CU(launch(pdl, swe::k_split_cells_tma_list<MODE, false>, dim3(ntiles), blk, s->st, a, sb, s->d_ctl, cm, cl, cc));
    } else if (s->cell_tma) {
      const swe::CellMaps& cm = s->cmaps[MODE - 1];
      if (s->settle) CU(launch(pdl, swe::k_split_cells_tma<MODE, true>, s->sgrid, blk, s->st, a, sb, s->d_ctl, cm));
      else CU(launch(pdl, swe::k_split_cells_tma<MODE, false>, s->sgrid, blk, s->st, a, sb, s->d_ctl, cm));
    } else if (s->settle) {
      CU(launch(pdl, swe::k_split_cells<MODE, true>, s->sgrid, blk, s->st, a, sb, s->d_ctl));
    } else {
      CU(launch(pdl, swe::k_split_cells<MODE, false>, s->sgrid, blk, s->st, a, sb, s->d_ctl));
    }
    // stage 2's close closes the whole step, stage 1's floored mass included
    if (MODE == 2)
      CU(launch(pdl, swe::k_split_close_multi<2>, dim3(swe::CLOSE_BLOCKS), blk, s->st, a, s->d_ctl,
                (int)(s->sgrid.x * s->sgrid.y), s->d_part + 3 * (size_t)s->part_cap));
  } else {
    swe::k_stage<MODE><<<s->grid, swe::BX, swe::STAGE_SMEM_BYTES, s->st>>>(a, s->d_ctl);
  }
  CU(cudaGetLastError());
  return SWE_OK;
}

// The ghost fill of f, and with tile lists the lists of stage MODE in the
// same launch (k_bc_face_list); returns through `listed` whether it made them.
template <int MODE>
int launch_bc_lists(swe_sim* s, double* const* f, int respect_stop, bool pdl, const swe::StageArgs& a,
                    bool& listed) {
  listed = stage_listed(s);
  if (!listed) return launch_bc(s, f, respect_stop, pdl);
  const int nbc = bc_blocks(s);
  const int nrx = (s->sgrid.x + swe::LX - 1) / swe::LX, nry = (s->sgrid.y + swe::LY - 1) / swe::LY;
  CU(launch(pdl, swe::k_bc_face_list, dim3(nbc + nrx * nry), dim3(swe::LX * swe::LY), s->st, bc_args(s, f),
            respect_stop, nbc, stage_bufs<MODE>(s), s->d_ctl, tile_lists<MODE>(s, a), nrx));
  return SWE_OK;
}

int enqueue_step(swe_sim* s, int mode, double dt, double t_end, const double* dt_dev = nullptr) {
  // The tiled kernels, the ghost fills and prepare enter through pdl_enter,
  // so each may be scheduled while its predecessor drains.
  const bool pdl = s->pdl && s->stage_impl == 1;
  CU(launch(pdl, swe::k_prepare, dim3(1), dim3(32), s->st, s->d_ctl, prep_args(s, mode, dt, t_end, dt_dev)));
  // Host-checked dt (mode 0) never reaches here refused.  In the device loop
  // a refused step (t reached t_end) changes nothing, ghosts included, as the
  // drivers' `while (sim.t < T)` loop stops calling step().
  swe::StageArgs a1 = stage_args(s, s->d_A, s->d_B);
  bool listed = false;
  int rc = launch_bc_lists<1>(s, s->d_A, mode == 0 ? 0 : 1, pdl, a1, listed);
  if (rc) return rc;
  rc = launch_stage<1>(s, a1, pdl, listed);
  if (rc) return rc;
  swe::StageArgs a2 = stage_args(s, s->d_B, s->d_A);
  if (s->keep_h0) { a2.h0c = s->d_h0[0]; a2.hu0c = s->d_h0[1]; a2.hv0c = s->d_h0[2]; }
  rc = launch_bc_lists<2>(s, s->d_B, 1, pdl, a2, listed);
  if (rc) return rc;
  return launch_stage<2>(s, a2, pdl, listed);
}

// Blocks of a grid-stride reduction over `cells` cells: one per 256 cells,
// at most 2368 (16 per SM of a B200), so that the last block's ticket is
// shared by a few thousand blocks and each thread strides over several cells.
int reduction_blocks(const swe_sim* s, int cells) {
  return std::min(s->part_cap, std::min(16 * 148, std::max(1, (cells + 255) / 256)));
}

int ensure_cfl(swe_sim* s) {
  if (s->cfl_valid) return SWE_OK;
  swe::StageArgs a = stage_args(s, s->d_A, nullptr);
  const int nb = reduction_blocks(s, s->nx * s->ny);
  swe::k_cfl_rate<<<nb, swe::BX, 0, s->st>>>(a, s->d_ctl, s->d_part);
  CU(cudaGetLastError());
  s->cfl_valid = true;
  return SWE_OK;
}

int read_ctl(swe_sim* s, swe::Control* out) {
  CU(cudaMemcpyAsync(out, s->d_ctl, sizeof(swe::Control), cudaMemcpyDeviceToHost, s->st));
  CU(cudaStreamSynchronize(s->st));
  return SWE_OK;
}

int sync_clock(swe_sim* s) {
  if (s->clock_valid) return SWE_OK;
  swe::Control c;
  int rc = read_ctl(s, &c);
  if (rc) return rc;
  s->t = c.t; s->steps = c.steps;
  s->clock_valid = true;
  return SWE_OK;
}

double* field_ptr(swe_sim* s, int f) {
  switch (f) {
    case SWE_FIELD_B: return s->d_b;
    case SWE_FIELD_H: return s->d_A[0];
    case SWE_FIELD_HU: return s->d_A[1];
    case SWE_FIELD_HV: return s->d_A[2];
    case SWE_FIELD_H0: return s->d_h0[0];
    case SWE_FIELD_HU0: return s->d_h0[1];
    case SWE_FIELD_HV0: return s->d_h0[2];
    case SWE_FIELD_RH: return s->d_res[0];
    case SWE_FIELD_RHU: return s->d_res[1];
    case SWE_FIELD_RHV: return s->d_res[2];
    case SWE_FIELD_THETA: return s->d_res[3];
    case SWE_FIELD_MANNING: return s->d_nfield;
    default: return nullptr;
  }
}

}  // namespace

namespace swe_host {
// Read-only view of a handle for the other translation units (frames).
void view_of(swe_sim* s, int* dims, double* opts, const double** b, const double** h, cudaStream_t* st) {
  dims[0] = s->nx; dims[1] = s->ny; dims[2] = s->W; dims[3] = s->H; dims[4] = s->o.sphere;
  opts[0] = s->o.min_depth; opts[1] = s->o.lat0; opts[2] = s->o.lat1; opts[3] = s->dx; opts[4] = s->dy;
  *b = field_ptr(s, SWE_FIELD_B);
  *h = field_ptr(s, SWE_FIELD_H);
  *st = s->st;
}
}  // namespace swe_host

namespace {

// Reciprocals of the three flux divisors (rows after the 13 metric rows).
void fill_reciprocals(swe_sim* s) {
  const int src[3] = {SWE_GEOM_DXROW, SWE_GEOM_DYROWN, SWE_GEOM_DYROWS};
  for (int q = 0; q < 3; q++) {
    s->recip[q].resize(s->H);
    for (int j = 0; j < s->H; j++) s->recip[q][j] = 1.0 / s->geom[src[q]][j];
  }
  s->dryfold = 1;
  for (int q = 0; q < 3; q++) s->dryfold &= swe::dry_fold_ok(s->recip[q].data(), s->recip[q].size());
}

int upload_geom(swe_sim* s) {
  fill_reciprocals(s);
  for (int r = 0; r < SWE_GEOM_NROWS; r++)
    CU(cudaMemcpyAsync(s->d_geom + (size_t)r * s->H, s->geom[r].data(), sizeof(double) * s->H,
                       cudaMemcpyHostToDevice, s->st));
  for (int q = 0; q < 3; q++)
    CU(cudaMemcpyAsync(s->d_geom + (size_t)(SWE_GEOM_NROWS + q) * s->H, s->recip[q].data(),
                       sizeof(double) * s->H, cudaMemcpyHostToDevice, s->st));
  return SWE_OK;
}

void free_all(swe_sim* s) {
  for (auto& g : s->graphs) if (g.exec) cudaGraphExecDestroy(g.exec);
  double** ptrs[] = {&s->d_b, &s->d_A[0], &s->d_A[1], &s->d_A[2], &s->d_B[0], &s->d_B[1], &s->d_B[2],
                     &s->d_h0[0], &s->d_h0[1], &s->d_h0[2], &s->d_res[0], &s->d_res[1], &s->d_res[2],
                     &s->d_res[3], &s->d_nfield, &s->d_geom, &s->d_part, &s->d_rows, &s->d_coef,
                     &s->d_sponge, &s->d_split};
  for (double** p : ptrs) if (*p) { cudaFree(*p); *p = nullptr; }
  if (s->d_ctl) cudaFree(s->d_ctl);
  if (s->st) cudaStreamDestroy(s->st);
}

int choose_rows_per_cta(const swe_sim* s) {
  const char* env = std::getenv("SWE_B200_ROWS_PER_CTA");
  if (env) { const int v = std::atoi(env); if (v >= 4) return std::min(v, swe::RY_MAX); }
  return 32;
}

}  // namespace

extern "C" {

const char* swe_last_error(void) { return g_err.c_str(); }

int swe_set_device(int ordinal) {
  CU(cudaSetDevice(ordinal));
  return SWE_OK;
}

int swe_options_init(swe_options* o) {
  if (!o) return fail(SWE_EINVAL, "null options");
  std::memset(o, 0, sizeof *o);
  o->dx = 1; o->dy = 1;
  o->manning = 0.025; o->min_depth = 1e-3; o->cfl = 0.45; o->coriolis = 0;
  o->order = 2; o->limiter = SWE_LIMITER_MC; o->sphere = 0;
  o->R = 6371e3; o->lat0 = -90; o->lat1 = 90; o->omega = 0;
  return SWE_OK;
}

int swe_create(const swe_options* o, const double* b, const double* h, swe_sim** out) {
  if (!out) return fail(SWE_EINVAL, "null output handle");
  *out = nullptr;
  if (!o) return fail(SWE_EINVAL, "null options");
  if (o->nx < 1 || o->ny < 1) return fail(SWE_EINVAL, "nx and ny must be >= 1");
  if (o->limiter < 0 || o->limiter > 2)
    return fail(SWE_EINVAL, "unknown limiter; have minmod,mc,central");   // src/swe.mjs:195
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
    return fail(SWE_ECUDA, "no CUDA device is available; this library has no CPU path");
  swe_sim* s = new swe_sim();
  s->o = *o;
  s->nx = o->nx; s->ny = o->ny; s->W = o->nx + 4; s->H = o->ny + 4; s->N = s->W * s->H;
  s->dx = o->dx; s->dy = o->dy;
  s->eps4 = std::pow(js_max(o->min_depth, 1e-12), 4.0);   // src/swe.mjs:190
  for (int r = 0; r < SWE_GEOM_NROWS; r++) s->geom[r].assign(s->H, 0.0);
  if (o->sphere) {
    const int rc = spherical_geometry(s);
    if (rc) { delete s; return rc; }
    s->dx = NAN;
  } else {
    cartesian_geometry(s);
  }
  // src/swe.mjs:239-241
  s->bc[0] = s->bc[1] = o->sphere ? SWE_BC_PERIODIC : SWE_BC_REFLECT;
  s->bc[2] = s->bc[3] = SWE_BC_REFLECT;

  const int gx = (s->W + swe::SX - 1) / swe::SX;
  const int ry = choose_rows_per_cta(s);
  const int gy = (s->H + ry - 1) / ry;
  s->grid = dim3(gx, gy, 1);
  s->nblocks = gx * gy;
  s->sgrid = dim3((s->W + swe::SPX - 1) / swe::SPX, (s->H + swe::SPY - 1) / swe::SPY, 1);
  s->part_cap = std::max(std::max(s->nblocks, (int)(s->sgrid.x * s->sgrid.y)), 1024);

  auto bail = [&](int rc) { free_all(s); delete s; return rc; };
  const size_t nb = sizeof(double) * (size_t)s->N;
#define CUB(call)                                                                           \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) return bail(fail(SWE_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_))); \
  } while (0)
  CUB(cudaFuncSetAttribute(swe::k_stage<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, swe::STAGE_SMEM_BYTES));
  CUB(cudaFuncSetAttribute(swe::k_stage<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, swe::STAGE_SMEM_BYTES));
  CUB(cudaFuncSetAttribute(swe::k_stage<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, swe::STAGE_SMEM_BYTES));
  CUB(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
  CUB(cudaMalloc(&s->d_b, nb));
  for (int q = 0; q < 3; q++) { CUB(cudaMalloc(&s->d_A[q], nb)); CUB(cudaMalloc(&s->d_B[q], nb)); }
  CUB(cudaMalloc(&s->d_geom, sizeof(double) * (SWE_GEOM_NROWS + 3) * s->H));
  CUB(cudaMalloc(&s->d_part, sizeof(double) * (3 * s->part_cap + 3 * swe::CLOSE_BLOCKS)));   // + the close's scratch
  CUB(cudaMalloc(&s->d_rows, sizeof(double) * std::max(1, s->ny)));
  CUB(cudaMalloc(&s->d_ctl, sizeof(swe::Control)));
  CUB(cudaMemsetAsync(s->d_ctl, 0, sizeof(swe::Control), s->st));
  CUB(cudaMemsetAsync(s->d_part, 0, sizeof(double) * (3 * s->part_cap + 3 * swe::CLOSE_BLOCKS), s->st));
  for (int q = 0; q < 3; q++) {
    CUB(cudaMemsetAsync(s->d_A[q], 0, nb, s->st));
    CUB(cudaMemsetAsync(s->d_B[q], 0, nb, s->st));
  }
  if (b) CUB(cudaMemcpyAsync(s->d_b, b, nb, cudaMemcpyHostToDevice, s->st));
  else CUB(cudaMemsetAsync(s->d_b, 0, nb, s->st));
  if (h) CUB(cudaMemcpyAsync(s->d_A[0], h, nb, cudaMemcpyHostToDevice, s->st));
  if (upload_geom(s)) return bail(SWE_ECUDA);
  make_tile_maps(s);
  {
    const char* env = std::getenv("SWE_B200_STAGE");
    s->stage_impl = (env && std::strcmp(env, "fused") == 0) ? 0 : (env && std::strcmp(env, "split") == 0) ? 1
                                                                  : SWE_DEFAULT_STAGE;
    if (s->stage_impl == 1 && ensure_split(s)) return bail(SWE_ECUDA);
    const char* pe = std::getenv("SWE_B200_PDL");
    s->pdl = (pe && std::strcmp(pe, "0") == 0) ? 0 : 1;
  }
  CUB(cudaStreamSynchronize(s->st));
#undef CUB
  *out = s;
  return SWE_OK;
}

int swe_destroy(swe_sim* s) {
  if (!s) return SWE_OK;
  if (s->st) cudaStreamSynchronize(s->st);
  free_all(s);
  delete s;
  return SWE_OK;
}

int swe_get_dims(swe_sim* s, int* d) {
  if (!s || !d) return fail(SWE_EINVAL, "null argument");
  d[0] = s->W; d[1] = s->H; d[2] = s->nx; d[3] = s->ny;
  return SWE_OK;
}

int swe_get_field(swe_sim* s, int field, double* out) {
  if (!s || !out) return fail(SWE_EINVAL, "null argument");
  if (field < 0 || field > SWE_FIELD_MANNING) return fail(SWE_EINVAL, "unknown field id");
  const size_t nb = sizeof(double) * (size_t)s->N;
  double* p = field_ptr(s, field);
  if (!p) {
    if (field == SWE_FIELD_MANNING) return fail(SWE_EINVAL, "no Manning field is set");
    std::memset(out, 0, nb);          // never written yet: a fresh Float64Array is zeros
    CU(cudaStreamSynchronize(s->st));
    return SWE_OK;
  }
  CU(cudaMemcpyAsync(out, p, nb, cudaMemcpyDeviceToHost, s->st));
  CU(cudaStreamSynchronize(s->st));
  return SWE_OK;
}

int swe_set_field(swe_sim* s, int field, const double* in) {
  if (!s || !in) return fail(SWE_EINVAL, "null argument");
  if (field != SWE_FIELD_B && field != SWE_FIELD_H && field != SWE_FIELD_HU && field != SWE_FIELD_HV)
    return fail(SWE_EINVAL, "only b, h, hu, hv are writable (use swe_set_manning_field for n)");
  const size_t nb = sizeof(double) * (size_t)s->N;
  CU(cudaMemcpyAsync(field_ptr(s, field), in, nb, cudaMemcpyHostToDevice, s->st));
  if (field != SWE_FIELD_B && forget_dry(s)) return SWE_ECUDA;
  s->cfl_valid = false;
  return SWE_OK;
}

int swe_get_rows(swe_sim* s, int field, int row0, int nrows, double* out) {
  if (!s || !out) return fail(SWE_EINVAL, "null argument");
  if (field != SWE_FIELD_B && field != SWE_FIELD_H && field != SWE_FIELD_HU && field != SWE_FIELD_HV)
    return fail(SWE_EINVAL, "swe_get_rows: b, h, hu or hv");
  if (row0 < 0 || nrows < 0 || row0 > s->H - nrows) return fail(SWE_EINVAL, "swe_get_rows: rows out of range");
  if (nrows == 0) return SWE_OK;
  const size_t off = (size_t)row0 * s->W, nb = sizeof(double) * (size_t)nrows * s->W;
  CU(cudaMemcpyAsync(out, field_ptr(s, field) + off, nb, cudaMemcpyDeviceToHost, s->st));
  CU(cudaStreamSynchronize(s->st));
  return SWE_OK;
}

int swe_set_rows(swe_sim* s, int field, int row0, int nrows, const double* in) {
  if (!s || !in) return fail(SWE_EINVAL, "null argument");
  if (field != SWE_FIELD_B && field != SWE_FIELD_H && field != SWE_FIELD_HU && field != SWE_FIELD_HV)
    return fail(SWE_EINVAL, "swe_set_rows: b, h, hu or hv");
  if (row0 < 0 || nrows < 0 || row0 > s->H - nrows) return fail(SWE_EINVAL, "swe_set_rows: rows out of range");
  if (nrows == 0) return SWE_OK;
  const size_t off = (size_t)row0 * s->W, nb = sizeof(double) * (size_t)nrows * s->W;
  CU(cudaMemcpyAsync(field_ptr(s, field) + off, in, nb, cudaMemcpyHostToDevice, s->st));
  if (field != SWE_FIELD_B && forget_dry(s)) return SWE_ECUDA;
  s->cfl_valid = false;
  return SWE_OK;
}

static int rows_args(swe_sim* s, int field, int row0, int nrows, const void* p, const char* who) {
  if (!s || !p) return fail(SWE_EINVAL, std::string(who) + ": null argument");
  if (field != SWE_FIELD_B && field != SWE_FIELD_H && field != SWE_FIELD_HU && field != SWE_FIELD_HV)
    return fail(SWE_EINVAL, std::string(who) + ": b, h, hu or hv");
  if (row0 < 0 || nrows < 0 || row0 > s->H - nrows) return fail(SWE_EINVAL, std::string(who) + ": rows out of range");
  return SWE_OK;
}

int swe_get_rows_async(swe_sim* s, int field, int row0, int nrows, double* dst) {
  int rc = rows_args(s, field, row0, nrows, dst, "swe_get_rows_async");
  if (rc || nrows == 0) return rc;
  const size_t off = (size_t)row0 * s->W, nb = sizeof(double) * (size_t)nrows * s->W;
  CU(cudaMemcpyAsync(dst, field_ptr(s, field) + off, nb, cudaMemcpyDefault, s->st));
  return SWE_OK;
}

int swe_set_rows_async(swe_sim* s, int field, int row0, int nrows, const double* src) {
  int rc = rows_args(s, field, row0, nrows, src, "swe_set_rows_async");
  if (rc || nrows == 0) return rc;
  const size_t off = (size_t)row0 * s->W, nb = sizeof(double) * (size_t)nrows * s->W;
  CU(cudaMemcpyAsync(field_ptr(s, field) + off, src, nb, cudaMemcpyDefault, s->st));
  if (field != SWE_FIELD_B && forget_dry(s)) return SWE_ECUDA;
  s->cfl_valid = false;
  return SWE_OK;
}

int swe_max_dt_to(swe_sim* s, double* dst) {
  if (!s || !dst) return fail(SWE_EINVAL, "swe_max_dt_to: null argument");
  int rc = ensure_cfl(s);
  if (rc) return rc;
  swe::k_dt_out<<<1, 32, 0, s->st>>>(s->d_ctl, s->o.cfl, dst);
  CU(cudaGetLastError());
  return SWE_OK;
}

int swe_step_dt_from(swe_sim* s, const double* dt) {
  if (!s || !dt) return fail(SWE_EINVAL, "swe_step_dt_from: null argument");
  int rc = sync_clock(s);
  if (rc) return rc;
  rc = enqueue_step(s, 4, 0, INFINITY, dt);
  if (rc) return rc;
  s->clock_valid = false;           // t and steps advanced on the device only
  s->cfl_valid = true;
  return SWE_OK;
}

int swe_get_geom(swe_sim* s, int row, double* out) {
  if (!s || !out) return fail(SWE_EINVAL, "null argument");
  if (row < 0 || row >= SWE_GEOM_NROWS) return fail(SWE_EINVAL, "unknown metric row id");
  std::memcpy(out, s->geom[row].data(), sizeof(double) * s->H);
  return SWE_OK;
}

int swe_set_geom(swe_sim* s, int row, const double* in) {
  if (!s || !in) return fail(SWE_EINVAL, "null argument");
  if (row < 0 || row >= SWE_GEOM_NROWS) return fail(SWE_EINVAL, "unknown metric row id");
  std::memcpy(s->geom[row].data(), in, sizeof(double) * s->H);
  const int rc = upload_geom(s);
  if (rc) return rc;
  CU(cudaStreamSynchronize(s->st));
  s->cfl_valid = false;
  return SWE_OK;
}

int swe_get_scalar(swe_sim* s, int which, double* out) {
  if (!s || !out) return fail(SWE_EINVAL, "null argument");
  switch (which) {
    case SWE_SCALAR_DX: *out = s->dx; return SWE_OK;
    case SWE_SCALAR_DY: *out = s->dy; return SWE_OK;
    case SWE_SCALAR_R: *out = s->R; return SWE_OK;
    case SWE_SCALAR_DLAM: *out = s->dlam; return SWE_OK;
    case SWE_SCALAR_DPHI: *out = s->dphi; return SWE_OK;
    case SWE_SCALAR_TOTAL_AREA: *out = s->totalArea; return SWE_OK;
    case SWE_SCALAR_EPS4: *out = s->eps4; return SWE_OK;
    case SWE_SCALAR_T: { int rc = sync_clock(s); if (rc) return rc; *out = s->t; return SWE_OK; }
    case SWE_SCALAR_STEPS: { int rc = sync_clock(s); if (rc) return rc; *out = s->steps; return SWE_OK; }
    case SWE_SCALAR_MASS_FLOORED: {
      swe::Control c; int rc = read_ctl(s, &c); if (rc) return rc;
      *out = c.mass_floored; return SWE_OK;
    }
    default: return fail(SWE_EINVAL, "unknown scalar id");
  }
}

int swe_set_scalar(swe_sim* s, int which, double v) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  int rc = sync_clock(s);
  if (rc) return rc;
  size_t off;
  if (which == SWE_SCALAR_T) { s->t = v; off = offsetof(swe::Control, t); }
  else if (which == SWE_SCALAR_STEPS) { s->steps = v; off = offsetof(swe::Control, steps); }
  else return fail(SWE_EINVAL, "only t and steps are settable");
  CU(cudaMemcpyAsync((char*)s->d_ctl + off, &v, sizeof(double), cudaMemcpyHostToDevice, s->st));
  CU(cudaStreamSynchronize(s->st));
  return SWE_OK;
}

int swe_set_boundary(swe_sim* s, int side, int kind) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  if (side < 0 || side > 3) return fail(SWE_EINVAL, "side must be 0..3 (west, east, south, north)");
  if (kind < 0 || kind > 3) return fail(SWE_EINVAL, "unknown boundary kind");
  s->bc[side] = kind;
  if (kind != SWE_BC_FLATHER) s->fl_kind[side] = 0;
  s->version++;
  return SWE_OK;
}

int swe_set_flather_values(swe_sim* s, int side, double eta_ext, double u_ext) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  if (side < 0 || side > 3) return fail(SWE_EINVAL, "side must be 0..3");
  s->bc[side] = SWE_BC_FLATHER;
  s->fl_kind[side] = 0;
  s->fl_eta[side] = eta_ext; s->fl_u[side] = u_ext;
  s->version++;
  return SWE_OK;
}

int swe_set_flather_tide(swe_sim* s, int side, double msl, int n, const double* amp,
                         const double* omega, const double* phase_deg, double u_coef) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  if (side < 0 || side > 3) return fail(SWE_EINVAL, "side must be 0..3");
  if (n < 0 || n > swe::MAX_TIDE) return fail(SWE_EINVAL, "tide tables hold at most 16 constituents");
  if (n > 0 && (!amp || !omega || !phase_deg)) return fail(SWE_EINVAL, "null tide table");
  swe::Control c;
  int rc = read_ctl(s, &c);
  if (rc) return rc;
  c.tide_n[side] = n; c.tide_msl[side] = msl; c.tide_ucoef[side] = u_coef;
  for (int q = 0; q < n; q++) {
    c.tide_amp[side][q] = amp[q]; c.tide_omega[side][q] = omega[q]; c.tide_phase[side][q] = phase_deg[q];
  }
  CU(cudaMemcpyAsync(s->d_ctl, &c, sizeof c, cudaMemcpyHostToDevice, s->st));
  CU(cudaStreamSynchronize(s->st));
  s->bc[side] = SWE_BC_FLATHER;
  s->fl_kind[side] = 1;
  s->version++;
  return SWE_OK;
}

int swe_set_manning_field(swe_sim* s, const double* n) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  s->version++;
  s->cfl_valid = false;
  if (!n) {
    if (s->d_nfield) { cudaStreamSynchronize(s->st); cudaFree(s->d_nfield); s->d_nfield = nullptr; }
    return SWE_OK;
  }
  for (int k = 0; k < s->N; k++) {                   // src/swe.mjs:723-725
    const double v = n[k];
    if (!(v >= 0) || !std::isfinite(v)) {
      char buf[200];
      std::snprintf(buf, sizeof buf, "setManningField: n = %.17g at cell %d; Manning n must be finite and >= 0", v, k);
      return fail(SWE_EINVAL, buf);
    }
  }
  if (!s->d_nfield) CU(cudaMalloc(&s->d_nfield, sizeof(double) * s->N));
  CU(cudaMemcpyAsync(s->d_nfield, n, sizeof(double) * s->N, cudaMemcpyHostToDevice, s->st));
  CU(cudaStreamSynchronize(s->st));
  return SWE_OK;
}

int swe_set_sponge(swe_sim* s, int side, int width, double strength, double eta_ref) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  if (side < 0 || side > 3) return fail(SWE_EINVAL, "side must be 0..3");
  if (width < 0) return fail(SWE_EINVAL, "sponge width must be >= 0");
  // per-distance strength, src/swe.mjs:1182-1183
  std::vector<double> str(std::max(1, width));
  for (int d = 0; d < width; d++) {
    const double c = std::cos(0.5 * PI * d / width);
    str[d] = strength * (c * c);
  }
  if (s->d_sponge) { cudaStreamSynchronize(s->st); cudaFree(s->d_sponge); s->d_sponge = nullptr; }
  CU(cudaMalloc(&s->d_sponge, sizeof(double) * str.size()));
  CU(cudaMemcpyAsync(s->d_sponge, str.data(), sizeof(double) * str.size(), cudaMemcpyHostToDevice, s->st));
  CU(cudaStreamSynchronize(s->st));
  s->sponge_side = side; s->sponge_width = width; s->sponge_ref = eta_ref;
  s->version++;
  return SWE_OK;
}

int swe_clear_sponge(swe_sim* s) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  s->sponge_width = 0;
  s->version++;
  return SWE_OK;
}

int swe_set_keep_h0(swe_sim* s, int on) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  if (on && !s->d_h0[0]) {
    for (int q = 0; q < 3; q++) {
      CU(cudaMalloc(&s->d_h0[q], sizeof(double) * s->N));
      CU(cudaMemsetAsync(s->d_h0[q], 0, sizeof(double) * s->N, s->st));
    }
  }
  s->keep_h0 = on != 0;
  s->version++;
  return SWE_OK;
}

int swe_apply_bc(swe_sim* s) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  swe::k_prepare<<<1, 32, 0, s->st>>>(s->d_ctl, prep_args(s, 0, 0, INFINITY));
  CU(cudaGetLastError());
  const int rc = launch_bc(s, s->d_A, 0);
  if (rc) return rc;
  CU(cudaStreamSynchronize(s->st));
  return SWE_OK;
}

int swe_residual(swe_sim* s, double dt) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  if (!s->d_res[0])
    for (int q = 0; q < 4; q++) {
      CU(cudaMalloc(&s->d_res[q], sizeof(double) * s->N));
      CU(cudaMemsetAsync(s->d_res[q], 0, sizeof(double) * s->N, s->st));
    }
  swe::k_prepare<<<1, 32, 0, s->st>>>(s->d_ctl, prep_args(s, 0, dt, INFINITY));
  CU(cudaGetLastError());
  swe::StageArgs a = stage_args(s, s->d_A, nullptr);
  a.rh = s->d_res[0]; a.rhu = s->d_res[1]; a.rhv = s->d_res[2]; a.theta = s->d_res[3];
  swe::k_stage<0><<<s->grid, swe::BX, swe::STAGE_SMEM_BYTES, s->st>>>(a, s->d_ctl);
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(s->st));
  return SWE_OK;
}

int swe_max_dt(swe_sim* s, double* out) {
  if (!s || !out) return fail(SWE_EINVAL, "null argument");
  int rc = ensure_cfl(s);
  if (rc) return rc;
  swe::Control c;
  rc = read_ctl(s, &c);
  if (rc) return rc;
  *out = c.next_max > 0 ? s->o.cfl / c.next_max : INFINITY;
  return SWE_OK;
}

int swe_apply_friction(swe_sim* s, double dt) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  swe::StageArgs a = stage_args(s, s->d_A, s->d_A);
  swe::k_friction<<<std::max(1, std::min(4096, (s->nx * s->ny + 255) / 256)), 256, 0, s->st>>>(a, dt);
  CU(cudaGetLastError());
  if (forget_dry(s)) return SWE_ECUDA;
  CU(cudaStreamSynchronize(s->st));
  s->cfl_valid = false;
  return SWE_OK;
}

int swe_dry_clean(swe_sim* s, double* added) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  swe::StageArgs a = stage_args(s, s->d_A, s->d_A);
  swe::k_dry_clean<<<1, swe::CHAIN_THREADS, 0, s->st>>>(a, s->d_ctl);
  CU(cudaGetLastError());
  if (forget_dry(s)) return SWE_ECUDA;
  swe::Control c;
  const int rc = read_ctl(s, &c);
  if (rc) return rc;
  if (added) *added = c.diag;
  s->cfl_valid = false;
  return SWE_OK;
}

int swe_step(swe_sim* s, double dt, double* taken) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  if (taken) *taken = 0;
  int rc = sync_clock(s);
  if (rc) return rc;
  if (!(dt > 0) || !std::isfinite(dt)) {   // src/swe.mjs:783-784, after applyBC
    swe::k_prepare<<<1, 32, 0, s->st>>>(s->d_ctl, prep_args(s, 0, 0, INFINITY));
    CU(cudaGetLastError());
    rc = launch_bc(s, s->d_A, 0);
    if (rc) return rc;
    CU(cudaStreamSynchronize(s->st));
    return SWE_OK;
  }
  rc = enqueue_step(s, 0, dt, INFINITY);
  if (rc) return rc;
  s->t = s->t + dt;
  s->steps = s->steps + 1;
  s->cfl_valid = true;
  if (taken) *taken = dt;
  return SWE_OK;
}

int swe_step_auto(swe_sim* s, double* taken) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  double dt;
  const int rc = swe_max_dt(s, &dt);
  if (rc) return rc;
  return swe_step(s, dt, taken);
}

int swe_run(swe_sim* s, int n, double dt_fixed, double t_end, int* done) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  if (done) *done = 0;
  if (n <= 0) return SWE_OK;
  int rc = sync_clock(s);
  if (rc) return rc;
  rc = ensure_cfl(s);
  if (rc) return rc;
  const double steps0 = s->steps;
  const int mode = dt_fixed > 0 ? 2 : 3;
  const double dtv = dt_fixed > 0 ? dt_fixed : 0;
  // Graphs of 32 steps; a shorter run (or remainder) is launched step by
  // step: a graph of 20 steps measured 12% slower per step than the same
  // steps launched directly, one of 32 as fast as them.
  const int chunk = 32;
  // The graph of `chunk` steps with the current value of s->settle, built
  // once per (chunk, mode, dt, tEnd, options) and kept.
  auto graph_for = [&](cudaGraphExec_t* out) -> int {
    swe_sim::LoopGraph& g = s->graphs[s->settle ? 1 : 0];
    if (!g.exec || g.steps != chunk || g.mode != mode || g.dt != dtv || g.tend != t_end || g.version != s->version) {
      if (g.exec) { cudaGraphExecDestroy(g.exec); g.exec = nullptr; }
      cudaGraph_t graph;
      CU(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
      for (int q = 0; q < chunk; q++) {
        const int rq = enqueue_step(s, mode, dtv, t_end);
        if (rq) { cudaStreamEndCapture(s->st, &graph); return rq; }
      }
      CU(cudaStreamEndCapture(s->st, &graph));
      const cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) return fail(SWE_ECUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
      g.steps = chunk; g.mode = mode; g.dt = dtv; g.tend = t_end; g.version = s->version;
    }
    *out = g.exec;
    return SWE_OK;
  };
  int left = n;
  cudaGraphExec_t exec = nullptr;
  s->settle = s->settle_pref;
  if (s->stage_impl == 1 && s->d_odry[0] && n >= 4 * chunk) {
    // the first chunk settles what it can; the settled-tile count of its
    // last step decides whether the rest (and later short runs) do
    s->settle = 1;
    rc = graph_for(&exec);
    if (rc) return rc;
    CU(cudaGraphLaunch(exec, s->st));
    left -= chunk;
    if (left > 0) {
      int counted = 0;
      CU(cudaMemcpyAsync(&counted, &s->d_ctl->settled_next, sizeof(int), cudaMemcpyDeviceToHost, s->st));
      CU(cudaStreamSynchronize(s->st));
      s->settle = s->settle_pref = 32 * counted >= (int)(s->sgrid.x * s->sgrid.y) ? 1 : 0;
    }
  }
  if (left >= chunk) {
    rc = graph_for(&exec);
    if (rc) return rc;
  }
  while (left >= chunk) {
    CU(cudaGraphLaunch(exec, s->st));
    left -= chunk;
  }
  for (int q = 0; q < left; q++) {
    rc = enqueue_step(s, mode, dtv, t_end);
    if (rc) return rc;
  }
  s->settle = 1;
  s->clock_valid = false;
  s->cfl_valid = true;
  rc = sync_clock(s);
  if (rc) return rc;
  if (done) *done = (int)(s->steps - steps0);
  return SWE_OK;
}

static int finish_diag(swe_sim* s, double* out) {
  swe::Control c;
  const int rc = read_ctl(s, &c);
  if (rc) return rc;
  *out = c.diag;
  return SWE_OK;
}

// Per-row sums (one warp per row) of `what`, then the rows in order.
static int row_diag(swe_sim* s, int what, int mode, const double* w, double* out) {
  swe::StageArgs a = stage_args(s, s->d_A, nullptr);
  swe::k_row_sums<<<(s->ny + swe::ROWSUM_WARPS - 1) / swe::ROWSUM_WARPS, 32 * swe::ROWSUM_WARPS, 0, s->st>>>(
      a, what, s->d_rows);
  CU(cudaGetLastError());
  swe::k_finish_sum<<<1, 1, 0, s->st>>>(s->d_rows, s->ny, mode, w, s->dx, s->dy, s->d_ctl);
  CU(cudaGetLastError());
  return finish_diag(s, out);
}

int swe_volume(swe_sim* s, double* out) {
  if (!s || !out) return fail(SWE_EINVAL, "null argument");
  if (s->o.sphere) return row_diag(s, 0, 0, s->d_geom + SWE_GEOM_AREA * s->H + 2, out);
  if (s->diag_order == SWE_DIAG_ROWS) return row_diag(s, 0, 1, nullptr, out);
  swe::StageArgs a = stage_args(s, s->d_A, nullptr);
  swe::k_volume_chain<<<1, swe::CHAIN_THREADS, 0, s->st>>>(a, s->dx, s->dy, s->d_ctl);
  CU(cudaGetLastError());
  return finish_diag(s, out);
}

int swe_energy(swe_sim* s, double* out) {
  if (!s || !out) return fail(SWE_EINVAL, "null argument");
  if (s->o.sphere) return row_diag(s, 1, 0, s->d_geom + SWE_GEOM_AREA * s->H + 2, out);
  return row_diag(s, 1, 1, nullptr, out);
}

int swe_set_diag_order(swe_sim* s, int order) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  if (order != SWE_DIAG_REFERENCE && order != SWE_DIAG_ROWS)
    return fail(SWE_EINVAL, "swe_set_diag_order: SWE_DIAG_REFERENCE or SWE_DIAG_ROWS");
  s->diag_order = order;
  return SWE_OK;
}

int swe_eta_projection(swe_sim* s, const double* coef, double* out) {
  if (!s || !coef || !out) return fail(SWE_EINVAL, "null argument");
  if (!s->d_coef) CU(cudaMalloc(&s->d_coef, sizeof(double) * std::max(1, s->ny)));
  CU(cudaMemcpyAsync(s->d_coef, coef, sizeof(double) * s->ny, cudaMemcpyHostToDevice, s->st));
  return row_diag(s, 2, 2, s->d_coef, out);
}

static int max_diag(swe_sim* s, int what, double ref, double* out) {
  swe::StageArgs a = stage_args(s, s->d_A, nullptr);
  const int total = what == 2 ? s->N : s->nx * s->ny;
  const int nb = reduction_blocks(s, total);
  swe::k_max_diag<<<nb, swe::BX, 0, s->st>>>(a, what, ref, s->d_part, s->d_ctl);
  CU(cudaGetLastError());
  return finish_diag(s, out);
}

int swe_max_surface_deviation(swe_sim* s, double ref, double* out) {
  if (!s || !out) return fail(SWE_EINVAL, "null argument");
  return max_diag(s, 0, ref, out);
}

int swe_max_speed(swe_sim* s, double* out) {
  if (!s || !out) return fail(SWE_EINVAL, "null argument");
  return max_diag(s, 1, 0, out);
}

int swe_finite(swe_sim* s, int* out) {
  if (!s || !out) return fail(SWE_EINVAL, "null argument");
  double bad = 0;
  const int rc = max_diag(s, 2, 0, &bad);
  if (rc) return rc;
  *out = bad == 0 ? 1 : 0;
  return SWE_OK;
}

int swe_compute_geometry(const swe_options* o, double* rows, double* scalars) {
  if (!o || !rows) return fail(SWE_EINVAL, "null argument");
  if (o->nx < 1 || o->ny < 1) return fail(SWE_EINVAL, "nx and ny must be >= 1");
  swe_sim tmp;
  tmp.o = *o;
  tmp.nx = o->nx; tmp.ny = o->ny; tmp.W = o->nx + 4; tmp.H = o->ny + 4; tmp.N = tmp.W * tmp.H;
  tmp.dx = o->dx; tmp.dy = o->dy;
  for (int r = 0; r < SWE_GEOM_NROWS; r++) tmp.geom[r].assign(tmp.H, 0.0);
  if (o->sphere) {
    const int rc = spherical_geometry(&tmp);
    if (rc) return rc;
    tmp.dx = NAN;
  } else {
    cartesian_geometry(&tmp);
  }
  for (int r = 0; r < SWE_GEOM_NROWS; r++)
    std::memcpy(rows + (size_t)r * tmp.H, tmp.geom[r].data(), sizeof(double) * tmp.H);
  if (scalars) {
    scalars[SWE_SCALAR_DX] = tmp.dx; scalars[SWE_SCALAR_DY] = tmp.dy; scalars[SWE_SCALAR_R] = tmp.R;
    scalars[SWE_SCALAR_DLAM] = tmp.dlam; scalars[SWE_SCALAR_DPHI] = tmp.dphi;
    scalars[SWE_SCALAR_TOTAL_AREA] = tmp.totalArea;
  }
  return SWE_OK;
}

int swe_get_stream(swe_sim* s, void** stream) {
  if (!s || !stream) return fail(SWE_EINVAL, "null argument");
  *stream = (void*)s->st;
  return SWE_OK;
}

int swe_step_timed(swe_sim* s, double dt, double* ms) {
  if (!s || !ms) return fail(SWE_EINVAL, "null argument");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(SWE_EINVAL, "swe_step_timed needs a valid dt");
  int rc = sync_clock(s);
  if (rc) return rc;
  cudaEvent_t ev[6];
  for (int q = 0; q < 6; q++) CU(cudaEventCreate(&ev[q]));
  CU(cudaEventRecord(ev[0], s->st));
  swe::k_prepare<<<1, 32, 0, s->st>>>(s->d_ctl, prep_args(s, 0, dt, INFINITY));
  CU(cudaEventRecord(ev[1], s->st));
  rc = launch_bc(s, s->d_A, 0);
  if (rc) return rc;
  CU(cudaEventRecord(ev[2], s->st));
  rc = launch_stage<1>(s, stage_args(s, s->d_A, s->d_B));
  if (rc) return rc;
  CU(cudaEventRecord(ev[3], s->st));
  rc = launch_bc(s, s->d_B, 1);
  if (rc) return rc;
  CU(cudaEventRecord(ev[4], s->st));
  swe::StageArgs a2 = stage_args(s, s->d_B, s->d_A);
  if (s->keep_h0) { a2.h0c = s->d_h0[0]; a2.hu0c = s->d_h0[1]; a2.hv0c = s->d_h0[2]; }
  rc = launch_stage<2>(s, a2);
  if (rc) return rc;
  CU(cudaEventRecord(ev[5], s->st));
  CU(cudaEventSynchronize(ev[5]));
  for (int q = 0; q < 5; q++) {
    float f = 0;
    CU(cudaEventElapsedTime(&f, ev[q], ev[q + 1]));
    ms[q] = f;
  }
  for (int q = 0; q < 6; q++) cudaEventDestroy(ev[q]);
  s->t = s->t + dt;
  s->steps = s->steps + 1;
  s->cfl_valid = true;
  return SWE_OK;
}

int swe_get_launch_config(swe_sim* s, int* cfg) {
  if (!s || !cfg) return fail(SWE_EINVAL, "null argument");
  if (s->stage_impl == 1) {
    cfg[0] = (int)s->sgrid.x; cfg[1] = (int)s->sgrid.y; cfg[2] = swe::SP_THREADS; cfg[3] = swe::SPX;
    cfg[4] = swe::SPY;
  } else {
    cfg[0] = (int)s->grid.x; cfg[1] = (int)s->grid.y; cfg[2] = swe::BX; cfg[3] = swe::SX;
    cfg[4] = (s->H + (int)s->grid.y - 1) / (int)s->grid.y;
  }
  return SWE_OK;
}

int swe_set_stage_kernels(swe_sim* s, int impl) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  if (impl != SWE_STAGE_FUSED && impl != SWE_STAGE_SPLIT) return fail(SWE_EINVAL, "unknown stage kernels");
  if (impl == SWE_STAGE_SPLIT) {
    int rc = ensure_split(s);
    if (rc) return rc;
  }
  // the fused kernels write no dry flags: whatever a switch leaves is stale
  if (forget_dry(s)) return SWE_ECUDA;
  s->stage_impl = impl;
  s->version++;                     // the cached graph holds the other kernels
  return SWE_OK;
}

int swe_get_stage_kernels(swe_sim* s, int* impl) {
  if (!s || !impl) return fail(SWE_EINVAL, "null argument");
  *impl = s->stage_impl;
  return SWE_OK;
}

int swe_synchronize(swe_sim* s) {
  if (!s) return fail(SWE_EINVAL, "null argument");
  CU(cudaStreamSynchronize(s->st));
  // A tile copy that did not complete within its bound left its tile
  // unwritten and set bit 4 of the control block's status
  // (swe_split.cuh): reported here once, then cleared.
  int st = 0;
  CU(cudaMemcpyAsync(&st, &s->d_ctl->status, sizeof st, cudaMemcpyDeviceToHost, s->st));
  CU(cudaStreamSynchronize(s->st));
  if (st & 4) {
    const int cleared = st & ~4;
    CU(cudaMemcpyAsync(&s->d_ctl->status, &cleared, sizeof cleared, cudaMemcpyHostToDevice, s->st));
    CU(cudaStreamSynchronize(s->st));
    return fail(SWE_ETIMEOUT, "swe_synchronize: a tile copy did not complete within its time bound; the steps "
                              "since the last synchronize are incomplete");
  }
  return SWE_OK;
}

int swe_hllc_batch(int n, const double* in, double* out) {
  if (n < 0 || (n > 0 && (!in || !out))) return fail(SWE_EINVAL, "bad arguments");
  if (n == 0) return SWE_OK;
  double *d_in = nullptr, *d_out = nullptr;
  CU(cudaMalloc(&d_in, sizeof(double) * 7 * n));
  cudaError_t e = cudaMalloc(&d_out, sizeof(double) * 3 * n);
  if (e == cudaSuccess) e = cudaMemcpy(d_in, in, sizeof(double) * 7 * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    swe::k_hllc_batch<<<(n + 127) / 128, 128>>>(n, d_in, d_out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, d_out, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost);
  cudaFree(d_in);
  if (d_out) cudaFree(d_out);
  if (e != cudaSuccess) return fail(SWE_ECUDA, std::string("hllc batch: ") + cudaGetErrorString(e));
  return SWE_OK;
}

int swe_vel_batch(swe_sim* s, int n, const double* hq, const double* h, double* out) {
  if (!s || n < 0 || (n > 0 && (!hq || !h || !out))) return fail(SWE_EINVAL, "bad arguments");
  if (n == 0) return SWE_OK;
  double* d = nullptr;
  CU(cudaMalloc(&d, sizeof(double) * 3 * n));
  cudaError_t e = cudaMemcpyAsync(d, hq, sizeof(double) * n, cudaMemcpyHostToDevice, s->st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d + n, h, sizeof(double) * n, cudaMemcpyHostToDevice, s->st);
  if (e == cudaSuccess) {
    swe::k_vel_batch<<<(n + 127) / 128, 128, 0, s->st>>>(n, d, d + n, s->eps4, d + 2 * n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d + 2 * n, sizeof(double) * n, cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  cudaFree(d);
  if (e != cudaSuccess) return fail(SWE_ECUDA, std::string("vel batch: ") + cudaGetErrorString(e));
  return SWE_OK;
}

}  // extern "C"
