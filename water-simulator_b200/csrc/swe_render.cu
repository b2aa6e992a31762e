// swe_render.cu -- headless frames of the solver's state, written as RGBA
// bytes into a device buffer (and optionally copied to the host).
//
//   swe_render_map    the map panel of WaterView.draw() (src/render.mjs:220-247):
//                     one pixel per interior cell, +y up, the diverging L*a*b*
//                     ramp about mean sea level over water (darkened by the STILL
//                     depth when the bed is shown), the land ramp over dry cells.
//   swe_render_globe  renderGlobe() (src/globe.mjs:770-812): an orthographic view
//                     of a spherical grid through a pixel -> cell table baked
//                     once per (size, tilt, margin, grid) by buildGlobeLut()
//                     (src/globe.mjs:554-629); the frame is a copy of the baked
//                     background plus one thread per modelled pixel.
//
// Bytes are stored as a Uint8ClampedArray stores a double (clamp to [0, 255],
// round half to even, NaN to 0), which is how the reference's ImageData holds
// them.  The colour tables are built on the host with the reference's
// formulas (src/render.mjs:98-131, src/globe.mjs:644-652).
#include "../../include/swe_b200.h"

#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace swe_host {
void set_error(const std::string& msg);
void view_of(swe_sim* s, int* dims, double* opts, const double** b, const double** h, cudaStream_t* st);
}  // namespace swe_host

struct swe_globe_lut {
  int size = 0, count = 0, inside = 0, capped = 0;
  double tilt = 0, margin = 0;
  int nx = 0, ny = 0;
  double lat0 = 0, lat1 = 0;
  int* d_px = nullptr;           // byte offset of the pixel in the frame
  double* d_lon = nullptr;       // longitude of the pixel centre at rotation 0 [deg]
  int* d_rowbase = nullptr;      // padded index of the row's first interior cell
  float* d_lit = nullptr;        // cos(incidence) of the viewer-fixed light
  unsigned char* d_bg = nullptr; // everything that is not modelled ocean or land
  double* d_stats = nullptr;     // frame reduction scratch
  unsigned int* d_ticket = nullptr;
  int nblocks = 0;
};

namespace {

int fail(int code, const std::string& m) { swe_host::set_error(m); return code; }

#define RCU(call)                                                                          \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) return fail(SWE_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

constexpr int RAMP_N = 1025;                    // odd: entry (N-1)/2 is mean sea level exactly
constexpr int RAMP_MID = (RAMP_N - 1) >> 1;
constexpr double PI_D = 3.141592653589793;

__constant__ double c_ramp[3 * RAMP_N];         // src/render.mjs RAMP (unclamped sRGB)
__constant__ unsigned char c_cbytes[3 * RAMP_N]; // src/globe.mjs CBYTES

// ---- the colour tables (host) ------------------------------------------------
// CIE L*a*b* (D65) -> sRGB, unclamped (src/render.mjs:98-110).
void lab_to_srgb_raw(double L, double a, double bb, double* out) {
  const double fy = (L + 16) / 116, fx = fy + a / 500, fz = fy - bb / 200;
  auto g = [](double f) { return f * f * f > 0.008856 ? f * f * f : (f - 16.0 / 116) / 7.787; };
  const double X = 0.95047 * g(fx), Y = g(fy), Z = 1.08883 * g(fz);
  auto enc = [](double u) {
    return 255 * (u <= 0.0031308 ? 12.92 * u : 1.055 * std::pow(u > 0 ? u : 0.0, 1 / 2.4) - 0.055);
  };
  out[0] = enc(3.2406 * X - 1.5372 * Y - 0.4986 * Z);
  out[1] = enc(-0.9689 * X + 1.8758 * Y + 0.0415 * Z);
  out[2] = enc(0.0557 * X - 0.2040 * Y + 1.0570 * Z);
}

// Uint8ClampedArray's conversion of a double (ToUint8Clamp).
__host__ __device__ __forceinline__ unsigned char clamp_u8(double x) {
  if (!(x > 0)) return 0;                       // NaN, negative, zero
  if (x >= 255) return 255;
  const double f = floor(x);
  const double d = x - f;
  if (d > 0.5) return (unsigned char)(f + 1);
  if (d < 0.5) return (unsigned char)f;
  const int fi = (int)f;
  return (unsigned char)((fi & 1) ? fi + 1 : fi);
}

// JavaScript Math.max / Math.min / Math.round.
__host__ __device__ __forceinline__ double js_max(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a > b) return a;
  if (b > a) return b;
  return signbit(a) ? b : a;
}
__host__ __device__ __forceinline__ double js_min(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a < b) return a;
  if (b < a) return b;
  return signbit(a) ? a : b;
}
__host__ __device__ __forceinline__ double js_round(double x) {
  const double f = floor(x);
  return (x - f >= 0.5) ? f + 1 : f;
}

struct Tables {
  double ramp[3 * RAMP_N];
  unsigned char cbytes[3 * RAMP_N];
};

void build_tables(Tables* t) {
  const double TROUGH[3] = {20, 8, -34}, MSL[3] = {53, -4, -14}, CREST[3] = {86, 6, 44};
  for (int i = 0; i < RAMP_N; i++) {                          // buildRamp, src/render.mjs:118-131
    const double tt = -1 + (2.0 * i) / (RAMP_N - 1);
    const double* end = tt >= 0 ? CREST : TROUGH;
    const double q = std::fabs(tt);
    lab_to_srgb_raw(MSL[0] + (end[0] - MSL[0]) * q, MSL[1] + (end[1] - MSL[1]) * q,
                    MSL[2] + (end[2] - MSL[2]) * q, t->ramp + 3 * i);
  }
  for (int i = 0; i < RAMP_N; i++) {                          // CBYTES, src/globe.mjs:644-652
    const double v = -1 + (2.0 * i) / (RAMP_N - 1);
    const double tt = js_max(-1, js_min(1, v / 1));           // surfaceColour(v, 1)
    const double q = js_round(std::fabs(tt) * RAMP_MID);
    const int o = 3 * (tt >= 0 ? RAMP_MID + (int)q : RAMP_MID - (int)q);
    for (int c = 0; c < 3; c++) t->cbytes[3 * i + c] = clamp_u8(t->ramp[o + c]);
  }
}

int ensure_tables() {
  static int done = -1;                        // per process; the constant banks are per device
  static int done_dev = -1;
  int dev = 0;
  RCU(cudaGetDevice(&dev));
  if (done == 1 && done_dev == dev) return SWE_OK;
  static Tables t;
  build_tables(&t);
  RCU(cudaMemcpyToSymbol(c_ramp, t.ramp, sizeof t.ramp));
  RCU(cudaMemcpyToSymbol(c_cbytes, t.cbytes, sizeof t.cbytes));
  done = 1;
  done_dev = dev;
  return SWE_OK;
}

// ---- WaterView map panel -------------------------------------------------------
// surfaceColour (src/render.mjs:142-153): the RAMP entry for elevation v.
__device__ __forceinline__ int ramp_offset(double v, double scale) {
  const double t = js_max(-1, js_min(1, v / scale));
  if (t != t) return -1;                       // NaN: the reference reads undefined -> 0
  const double q = js_round(fabs(t) * RAMP_MID);
  return 3 * (t >= 0 ? RAMP_MID + (int)q : RAMP_MID - (int)q);
}

__global__ void k_render_map(int nx, int ny, int W, const double* __restrict__ b, const double* __restrict__ h,
                             double minDepth, double msl, double scale, int showBed,
                             unsigned char* __restrict__ out) {
  const long long n = (long long)nx * ny;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(p / nx), i = (int)(p - (long long)j * nx);
    const long long k = (long long)(j + 2) * W + (i + 2);
    const long long o = 4 * ((long long)(ny - 1 - j) * nx + i);     // +y up on screen
    const double depth = h[k], bk = b[k];
    double c0, c1, c2;
    if (depth <= minDepth) {                    // landColour, src/render.mjs:193-196
      const double t = js_max(0, js_min(1, bk / 6));
      c0 = 96 + 70 * t; c1 = 88 + 62 * t; c2 = 74 + 52 * t;
    } else {
      const int ro = ramp_offset(bk + depth - msl, scale);
      if (ro < 0) { c0 = c1 = c2 = NAN; }
      else { c0 = c_ramp[ro]; c1 = c_ramp[ro + 1]; c2 = c_ramp[ro + 2]; }
      if (showBed) {                            // STILL depth shading, src/render.mjs:238-245
        const double still = js_max(0, msl - bk);
        const double shade = 0.55 + 0.45 * exp(-still / 12);
        c0 = c0 * shade; c1 = c1 * shade; c2 = c2 * shade;
      }
    }
    out[o] = clamp_u8(c0); out[o + 1] = clamp_u8(c1); out[o + 2] = clamp_u8(c2); out[o + 3] = 255;
  }
}

// ---- renderGlobe ------------------------------------------------------------------
constexpr int FRAME_THREADS = 256;
constexpr double LAND_SAT = 2500;               // src/globe.mjs:680-682
__constant__ double c_land_lo[3] = {92, 84, 70};
__constant__ double c_land_hi[3] = {188, 172, 144};

// colOfLon (src/globe.mjs:547-550), with the rotation applied as frameLon()'s
// addition (src/globe.mjs:741).
__device__ __forceinline__ long long col_of_lon(double lonDeg, int nx) {
  const double i = floor((lonDeg + 180) * nx / 360);
  const long long ii = (long long)i;
  return ((ii % nx) + nx) % nx;
}

__global__ void k_render_globe(int count, const int* __restrict__ px, const double* __restrict__ lon,
                               const int* __restrict__ rowbase, const float* __restrict__ lit, int nx,
                               const double* __restrict__ b, const double* __restrict__ h, double minDepth,
                               double rot, double scale, double msl, int landLight, unsigned char* __restrict__ out,
                               double* __restrict__ part, unsigned int* ticket, double* __restrict__ stats) {
  __shared__ double s_lo[FRAME_THREADS], s_hi[FRAME_THREADS];
  __shared__ unsigned int s_wet[FRAME_THREADS], s_dry[FRAME_THREADS], s_sat[FRAME_THREADS];
  __shared__ bool s_last;
  double lo = INFINITY, hi = -INFINITY;
  unsigned int wet = 0, dry = 0, sat = 0;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < count; p += gridDim.x * blockDim.x) {
    const long long k = rowbase[p] + col_of_lon(lon[p] + rot, nx);
    const int o = px[p];
    const double hk = h[k];
    if (hk <= minDepth) {
      dry++;
      const double t = js_max(0, js_min(1, b[k] / LAND_SAT));
      const double s = landLight ? 0.30 + 0.70 * (double)lit[p] : 1;
      for (int c = 0; c < 3; c++) out[o + c] = clamp_u8((c_land_lo[c] + (c_land_hi[c] - c_land_lo[c]) * t) * s);
      out[o + 3] = 255;
    } else {
      wet++;
      const double e = b[k] + hk - msl;
      if (e < lo) lo = e;
      if (e > hi) hi = e;
      if (e >= scale || e <= -scale) sat++;
      const int co = ramp_offset(e, scale);     // colourOffset, src/globe.mjs:665-669
      for (int c = 0; c < 3; c++) out[o + c] = co < 0 ? 0 : c_cbytes[co + c];
      out[o + 3] = 255;
    }
  }
  s_lo[threadIdx.x] = lo; s_hi[threadIdx.x] = hi;
  s_wet[threadIdx.x] = wet; s_dry[threadIdx.x] = dry; s_sat[threadIdx.x] = sat;
  __syncthreads();
  for (int w = FRAME_THREADS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s_lo[threadIdx.x] = fmin(s_lo[threadIdx.x], s_lo[threadIdx.x + w]);
      s_hi[threadIdx.x] = fmax(s_hi[threadIdx.x], s_hi[threadIdx.x + w]);
      s_wet[threadIdx.x] += s_wet[threadIdx.x + w];
      s_dry[threadIdx.x] += s_dry[threadIdx.x + w];
      s_sat[threadIdx.x] += s_sat[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double* q = part + 5 * blockIdx.x;
    q[0] = s_lo[0]; q[1] = s_hi[0]; q[2] = s_wet[0]; q[3] = s_dry[0]; q[4] = s_sat[0];
    __threadfence();
    s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {             // the last block closes the frame (no waiting)
    __threadfence();
    double L = INFINITY, Hh = -INFINITY, Wt = 0, D = 0, S = 0;
    for (unsigned int g = 0; g < gridDim.x; g++) {
      const volatile double* q = part + 5 * g;
      L = fmin(L, q[0]); Hh = fmax(Hh, q[1]); Wt += q[2]; D += q[3]; S += q[4];
    }
    stats[0] = Wt; stats[1] = D; stats[4] = L; stats[5] = Hh; stats[6] = S;
    stats[7] = Wt > 0 ? S / Wt : 0;
    *ticket = 0;
  }
}

// ---- the LUT bake (host) --------------------------------------------------------------
struct Cam { double size, margin, r, cx, cy, tilt, sinT, cosT; };

Cam globe_camera(int size, double tilt, double margin) {     // src/globe.mjs:460-466
  Cam c;
  c.size = size; c.margin = margin; c.r = 0.5 * size * margin; c.cx = 0.5 * size; c.cy = 0.5 * size;
  c.tilt = tilt;
  const double D2R = PI_D / 180;
  c.sinT = std::sin(tilt * D2R); c.cosT = std::cos(tilt * D2R);
  return c;
}

int row_of_lat(double latDeg, double lat0, double lat1, int ny) {   // src/globe.mjs:561-568
  if (latDeg < lat0 || latDeg > lat1) return -1;
  int j = (int)std::floor((latDeg - lat0) * ny / (lat1 - lat0));
  if (j >= ny) j = ny - 1;
  else if (j < 0) j = 0;
  return j;
}

}  // namespace

extern "C" {

int swe_render_tables(double* ramp, unsigned char* cbytes) {
  static Tables t;
  build_tables(&t);
  if (ramp) std::memcpy(ramp, t.ramp, sizeof t.ramp);
  if (cbytes) std::memcpy(cbytes, t.cbytes, sizeof t.cbytes);
  return SWE_OK;
}

int swe_render_map(swe_sim* s, double msl, double scale, int show_bed, unsigned char* rgba_host, void* rgba_device) {
  if (!s || (!rgba_host && !rgba_device)) return fail(SWE_EINVAL, "swe_render_map: null handle or no output");
  int dims[5];
  double opts[5];
  const double *b, *h;
  cudaStream_t st;
  swe_host::view_of(s, dims, opts, &b, &h, &st);
  const int nx = dims[0], ny = dims[1], W = dims[2];
  int rc = ensure_tables();
  if (rc) return rc;
  const size_t bytes = (size_t)4 * nx * ny;
  unsigned char* out = static_cast<unsigned char*>(rgba_device);
  bool own = false;
  if (!out) { RCU(cudaMallocAsync(reinterpret_cast<void**>(&out), bytes, st)); own = true; }
  long long blocks = ((long long)nx * ny + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  k_render_map<<<(int)blocks, 256, 0, st>>>(nx, ny, W, b, h, opts[0], msl, scale, show_bed ? 1 : 0, out);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && rgba_host) e = cudaMemcpyAsync(rgba_host, out, bytes, cudaMemcpyDeviceToHost, st);
  if (own) cudaFreeAsync(out, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(SWE_ECUDA, std::string("swe_render_map: ") + cudaGetErrorString(e));
  return SWE_OK;
}

int swe_globe_lut_create(swe_sim* s, int size, double tilt_deg, double margin, const double* sun,
                         const double* bg, const double* halo, swe_globe_lut** out) {
  if (!out) return fail(SWE_EINVAL, "null output");
  *out = nullptr;
  if (!s || size < 1) return fail(SWE_EINVAL, "swe_globe_lut_create: null handle or size < 1");
  int dims[5];
  double opts[5];
  const double *b, *h;
  cudaStream_t st;
  swe_host::view_of(s, dims, opts, &b, &h, &st);
  if (!dims[4])
    return fail(SWE_EINVAL, "globe.mjs draws spherical fields only: sim.geom.kind is cartesian. "
                            "Use the map panel (swe_render_map).");
  const int nx = dims[0], ny = dims[1], W = dims[2];
  const double lat0 = opts[1], lat1 = opts[2];
  double sv[3] = {-0.42, 0.48, 0.77};
  if (sun) { sv[0] = sun[0]; sv[1] = sun[1]; sv[2] = sun[2]; }
  const double m = std::sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);   // normalise()
  const double su[3] = {sv[0] / m, sv[1] / m, sv[2] / m};
  const double B[3] = {bg ? bg[0] : 8, bg ? bg[1] : 11, bg ? bg[2] : 16};
  const double HALO[3] = {halo ? halo[0] : 36, halo ? halo[1] : 58, halo ? halo[2] : 84};
  const Cam cam = globe_camera(size, tilt_deg, margin);
  const double R2D = 180 / PI_D;
  const size_t NP = (size_t)size * size;
  std::vector<unsigned char> bgb(4 * NP, 0);
  std::vector<int> px, rowbase;
  std::vector<double> lon;
  std::vector<float> lit;
  int inside = 0, capped = 0;
  for (int y = 0; y < size; y++) {
    for (int x = 0; x < size; x++) {
      const size_t p = (size_t)y * size + x, o = 4 * p;
      // orthoInversePixel at rotation 0 (src/globe.mjs:500-520)
      const double X = (x + 0.5 - cam.cx) / cam.r, Y = (cam.cy - y - 0.5) / cam.r;
      const double ss = X * X + Y * Y;
      if (ss > 1) {
        const double g = std::exp(-(ss - 1) * 5.5);            // limb halo
        for (int c = 0; c < 3; c++) bgb[o + c] = clamp_u8(B[c] + (HALO[c] - B[c]) * g);
        bgb[o + 3] = 255;
        continue;
      }
      inside++;
      const double z = std::sqrt(1 - ss);
      const double phi = std::asin(z * cam.sinT + Y * cam.cosT);
      const double lam = std::atan2(X, z * cam.cosT - Y * cam.sinT);
      const double lonDeg = 0 + lam * R2D, latDeg = phi * R2D;
      const int j = row_of_lat(latDeg, lat0, lat1, ny);
      if (j < 0) {                                             // unmodelled cap: hatched
        capped++;
        const int t = ((x + y) & 7) < 3 ? 1 : 0;
        bgb[o] = 52 + 14 * t; bgb[o + 1] = 56 + 14 * t; bgb[o + 2] = 62 + 14 * t; bgb[o + 3] = 255;
        continue;
      }
      px.push_back((int)o);
      lon.push_back(lonDeg);
      rowbase.push_back((j + 2) * W + 2);
      const double l = X * su[0] + Y * su[1] + z * su[2];
      lit.push_back((float)js_max(0, l));
    }
  }
  swe_globe_lut* L = new swe_globe_lut();
  L->size = size; L->count = (int)px.size(); L->inside = inside; L->capped = capped;
  L->tilt = tilt_deg; L->margin = margin; L->nx = nx; L->ny = ny; L->lat0 = lat0; L->lat1 = lat1;
  const int n = std::max(1, L->count);
  L->nblocks = std::max(1, std::min(148 * 8, (L->count + FRAME_THREADS - 1) / FRAME_THREADS));
  cudaError_t e = cudaSuccess;
  auto M = [&](void** p, size_t bytes) { if (e == cudaSuccess) e = cudaMalloc(p, bytes); };
  M(reinterpret_cast<void**>(&L->d_px), sizeof(int) * n);
  M(reinterpret_cast<void**>(&L->d_lon), sizeof(double) * n);
  M(reinterpret_cast<void**>(&L->d_rowbase), sizeof(int) * n);
  M(reinterpret_cast<void**>(&L->d_lit), sizeof(float) * n);
  M(reinterpret_cast<void**>(&L->d_bg), 4 * NP);
  M(reinterpret_cast<void**>(&L->d_stats), sizeof(double) * (5 * L->nblocks + 8));
  M(reinterpret_cast<void**>(&L->d_ticket), sizeof(unsigned int));
  if (e == cudaSuccess && L->count) {
    e = cudaMemcpy(L->d_px, px.data(), sizeof(int) * L->count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(L->d_lon, lon.data(), sizeof(double) * L->count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(L->d_rowbase, rowbase.data(), sizeof(int) * L->count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(L->d_lit, lit.data(), sizeof(float) * L->count, cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMemcpy(L->d_bg, bgb.data(), 4 * NP, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(L->d_ticket, 0, sizeof(unsigned int));
  if (e != cudaSuccess) {
    swe_globe_lut_destroy(L);
    return fail(SWE_ECUDA, std::string("swe_globe_lut_create: ") + cudaGetErrorString(e));
  }
  *out = L;
  return SWE_OK;
}

int swe_globe_lut_destroy(swe_globe_lut* L) {
  if (!L) return SWE_OK;
  cudaFree(L->d_px); cudaFree(L->d_lon); cudaFree(L->d_rowbase); cudaFree(L->d_lit);
  cudaFree(L->d_bg); cudaFree(L->d_stats); cudaFree(L->d_ticket);
  delete L;
  return SWE_OK;
}

int swe_globe_lut_get(swe_globe_lut* L, int* counts, int* px, double* lon_base, int* row_base, float* lit,
                      unsigned char* bg) {
  if (!L) return fail(SWE_EINVAL, "null LUT");
  if (counts) { counts[0] = L->count; counts[1] = L->inside; counts[2] = L->capped; counts[3] = L->size; }
  const size_t n = L->count;
  if (px && n) RCU(cudaMemcpy(px, L->d_px, sizeof(int) * n, cudaMemcpyDeviceToHost));
  if (lon_base && n) RCU(cudaMemcpy(lon_base, L->d_lon, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (row_base && n) RCU(cudaMemcpy(row_base, L->d_rowbase, sizeof(int) * n, cudaMemcpyDeviceToHost));
  if (lit && n) RCU(cudaMemcpy(lit, L->d_lit, sizeof(float) * n, cudaMemcpyDeviceToHost));
  if (bg) RCU(cudaMemcpy(bg, L->d_bg, (size_t)4 * L->size * L->size, cudaMemcpyDeviceToHost));
  return SWE_OK;
}

int swe_render_globe(swe_sim* s, swe_globe_lut* L, double rot_deg, double scale, double msl, int land_light,
                     unsigned char* rgba_host, void* rgba_device, double* stats) {
  if (!s || !L) return fail(SWE_EINVAL, "swe_render_globe: null handle or LUT");
  if (!rgba_host && !rgba_device) return fail(SWE_EINVAL, "swe_render_globe: no output");
  int dims[5];
  double opts[5];
  const double *b, *h;
  cudaStream_t st;
  swe_host::view_of(s, dims, opts, &b, &h, &st);
  if (!dims[4]) return fail(SWE_EINVAL, "globe.mjs draws spherical fields only: sim.geom.kind is cartesian.");
  if (dims[0] != L->nx || dims[1] != L->ny || opts[1] != L->lat0 || opts[2] != L->lat1) {
    char buf[240];
    std::snprintf(buf, sizeof buf, "LUT was baked for %d|%.17g|%.17g|%d|%d|%.17g|%.17g, grid is now %d|%d|%.17g|%.17g",
                  L->size, L->tilt, L->margin, L->nx, L->ny, L->lat0, L->lat1, dims[0], dims[1], opts[1], opts[2]);
    return fail(SWE_EINVAL, buf);
  }
  int rc = ensure_tables();
  if (rc) return rc;
  const size_t bytes = (size_t)4 * L->size * L->size;
  unsigned char* out = static_cast<unsigned char*>(rgba_device);
  bool own = false;
  if (!out) { RCU(cudaMallocAsync(reinterpret_cast<void**>(&out), bytes, st)); own = true; }
  cudaError_t e = cudaMemcpyAsync(out, L->d_bg, bytes, cudaMemcpyDeviceToDevice, st);   // out.set(lut.bg)
  double* part = L->d_stats + 8;
  if (e == cudaSuccess && L->count > 0) {
    k_render_globe<<<L->nblocks, FRAME_THREADS, 0, st>>>(L->count, L->d_px, L->d_lon, L->d_rowbase, L->d_lit,
                                                        dims[0], b, h, opts[0], rot_deg, scale, msl,
                                                        land_light ? 1 : 0, out, part, L->d_ticket, L->d_stats);
    e = cudaGetLastError();
  }
  double st8[8] = {0, 0, 0, 0, INFINITY, -INFINITY, 0, 0};
  if (e == cudaSuccess && L->count > 0) e = cudaMemcpyAsync(st8, L->d_stats, sizeof st8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && rgba_host) e = cudaMemcpyAsync(rgba_host, out, bytes, cudaMemcpyDeviceToHost, st);
  if (own) cudaFreeAsync(out, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(SWE_ECUDA, std::string("swe_render_globe: ") + cudaGetErrorString(e));
  st8[2] = L->capped; st8[3] = L->inside;
  if (stats) std::memcpy(stats, st8, sizeof st8);
  return SWE_OK;
}

}  // extern "C"
