// swe_gridlands.cu -- gridlands-terrain v1 import straight to the device.
//
// The export's float32 layers arrive as base64 text and are decoded by a
// kernel (decodeF32, src/gridlands.mjs:82-98); a second kernel samples the
// terrain functions of gridlandsTerrain() (src/gridlands.mjs:262-291) at
// every padded cell centre of the new grid, exactly as the ShallowWater
// constructor samples bed() and eta0() (src/swe.mjs:222-232), and the
// per-cell Manning field the way tools/verify-gridlands.mjs:330-331 samples
// it for setManningField().  Arithmetic is FP64 operation for operation
// (the library is built with -fmad=false), so the fields are bit-identical
// to sampling the same functions on the host.
#include "../../include/swe_b200.h"

#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

namespace swe_host {
void set_error(const std::string& msg);
cudaStream_t stream_of(swe_sim* s);
int adopt_fields(swe_sim* s, const double* d_b, const double* d_h, const double* d_n);
}  // namespace swe_host

namespace {

int fail(int code, const std::string& m) { swe_host::set_error(m); return code; }

// Math.max / Math.min with JavaScript's NaN and signed-zero meaning.
__device__ __forceinline__ double js_max(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a > b) return a;
  if (b > a) return b;
  return signbit(a) ? b : a;
}
__device__ __forceinline__ double js_min(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a < b) return a;
  if (b < a) return b;
  return signbit(a) ? a : b;
}
// Math.round: the nearest integer, ties towards +Infinity.  x - floor(x) is
// exact for every double, so the tie test is exact too.
__device__ __forceinline__ double js_round(double x) {
  const double f = floor(x);
  return (x - f >= 0.5) ? f + 1.0 : f;
}

__device__ __forceinline__ int b64_value(unsigned char c) {
  if (c >= 'A' && c <= 'Z') return c - 'A';
  if (c >= 'a' && c <= 'z') return c - 'a' + 26;
  if (c >= '0' && c <= '9') return c - '0' + 52;
  if (c == '+' || c == '-') return 62;
  if (c == '/' || c == '_') return 63;
  return -1;
}

// One thread per 4-character quantum of the unpadded text (`len` characters):
// 3 bytes out, fewer for a short last quantum.  A character outside both
// alphabets sets *bad and the lowest such position.
__global__ void k_b64_decode(const unsigned char* __restrict__ txt, long long len, long long nbytes,
                             unsigned char* __restrict__ out, int* bad, long long* bad_pos) {
  const long long nq = (len + 3) / 4;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    int v[4] = {0, 0, 0, 0};
    for (int c = 0; c < 4; c++) {
      const long long p = 4 * q + c;
      if (p >= len) break;
      const int x = b64_value(txt[p]);
      if (x < 0) {
        atomicExch(bad, 1);
        atomicMin(reinterpret_cast<unsigned long long*>(bad_pos), (unsigned long long)p);
        v[c] = 0;
      } else {
        v[c] = x;
      }
    }
    const unsigned char o[3] = {(unsigned char)((v[0] << 2) | (v[1] >> 4)),
                                (unsigned char)(((v[1] & 15) << 4) | (v[2] >> 2)),
                                (unsigned char)(((v[2] & 3) << 6) | v[3])};
    for (int c = 0; c < 3; c++) {
      const long long k = 3 * q + c;
      if (k < nbytes) out[k] = o[c];
    }
  }
}

struct SampleArgs {
  const float* bedM;
  const float* surfM;
  const float* nM;           // nullptr: no Manning field
  int Wg, Hg;                // export grid
  double C;                  // cellMeters
  int flip;
  int W, H;                  // padded sim grid
  double dx, dy;
  double* b;
  double* h;
  double* n;
  int* bad_n;
  long long* bad_k;
};

// rowOf / colOf of src/gridlands.mjs:262-265
__device__ __forceinline__ double row_of(const SampleArgs& a, double y) {
  const double r = js_min(a.Hg - 1, js_max(0, y / a.C - 0.5));
  return a.flip ? (a.Hg - 1) - r : r;
}
__device__ __forceinline__ double col_of(const SampleArgs& a, double x) {
  return js_min(a.Wg - 1, js_max(0, x / a.C - 0.5));
}

__global__ void k_gridlands_sample(SampleArgs a) {
  const long long N = (long long)a.W * a.H;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < N;
       k += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(k / a.W), i = (int)(k - (long long)j * a.W);
    const double x = ((i - 2) + 0.5) * a.dx;          // cellCentre(i - ng, j - ng), src/swe.mjs:251
    const double y = ((j - 2) + 0.5) * a.dy;
    const double fc = col_of(a, x), fr = row_of(a, y);
    // bed: bilinear, src/gridlands.mjs:271-279
    const int c0 = (int)floor(fc), r0 = (int)floor(fr);
    const int c1 = min(a.Wg - 1, c0 + 1), r1 = min(a.Hg - 1, r0 + 1);
    const double tc = fc - c0, tr = fr - r0;
    const double v00 = a.bedM[(long long)r0 * a.Wg + c0], v10 = a.bedM[(long long)r0 * a.Wg + c1];
    const double v01 = a.bedM[(long long)r1 * a.Wg + c0], v11 = a.bedM[(long long)r1 * a.Wg + c1];
    const double bed = (v00 * (1 - tc) + v10 * tc) * (1 - tr) + (v01 * (1 - tc) + v11 * tc) * tr;
    // surface: nearest, src/gridlands.mjs:289
    const long long kn = (long long)js_round(fr) * a.Wg + (long long)js_round(fc);
    const double e = a.surfM[kn];
    a.b[k] = bed;
    const double d = e - bed;                           // Math.max(0, e - b), src/swe.mjs:230
    a.h[k] = d > 0 ? d : (d == d ? 0.0 : d);
    if (a.nM) {
      const double v = a.nM[kn];
      if (!(v >= 0) || !isfinite(v)) {                  // src/swe.mjs:723-725
        atomicExch(a.bad_n, 1);
        atomicMin(reinterpret_cast<unsigned long long*>(a.bad_k), (unsigned long long)k);
      }
      a.n[k] = v;
    }
  }
}

int grid_blocks(long long work) {
  long long b = (work + 255) / 256;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return (int)b;
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
};

#define GL_CU(call)                                                                        \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) return fail(SWE_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Decode `len` characters of base64 into `out` (device, >= 4n bytes), which
// must come to exactly 4n bytes.
int decode_layer(const char* b64, size_t len, long long n, float* out, cudaStream_t st, const char* name) {
  if (!b64) return fail(SWE_EINVAL, std::string("gridlands: layer ") + name + " is missing");
  size_t L = len;
  int pad = 0;
  while (L > 0 && b64[L - 1] == '=' && pad < 2) { L--; pad++; }
  long long nbytes = (long long)(L / 4) * 3;
  const int rem = (int)(L % 4);
  if (rem == 1) nbytes = -1;
  else if (rem == 2) nbytes += 1;
  else if (rem == 3) nbytes += 2;
  if (nbytes != 4 * n) {
    char buf[320];
    std::snprintf(buf, sizeof buf,
                  "gridlands: layer %s decoded to %lld bytes, expected %lld (%lld cells x 4). "
                  "A truncated layer would otherwise read as terrain.",
                  name, nbytes < 0 ? 0LL : nbytes, 4 * n, n);
    return fail(SWE_EINVAL, buf);
  }
  DevBuf txt, flag;
  GL_CU(cudaMalloc(&txt.p, L > 0 ? L : 1));
  GL_CU(cudaMalloc(&flag.p, 16));
  GL_CU(cudaMemsetAsync(flag.p, 0, 8, st));
  GL_CU(cudaMemsetAsync(static_cast<char*>(flag.p) + 8, 0xff, 8, st));
  if (L > 0) GL_CU(cudaMemcpyAsync(txt.p, b64, L, cudaMemcpyHostToDevice, st));
  const long long nq = (long long)(L + 3) / 4;
  if (nq > 0)
    k_b64_decode<<<grid_blocks(nq), 256, 0, st>>>(static_cast<const unsigned char*>(txt.p), (long long)L, nbytes,
                                                  reinterpret_cast<unsigned char*>(out),
                                                  static_cast<int*>(flag.p),
                                                  reinterpret_cast<long long*>(static_cast<char*>(flag.p) + 8));
  GL_CU(cudaGetLastError());
  long long hflag[2];
  GL_CU(cudaMemcpyAsync(hflag, flag.p, 16, cudaMemcpyDeviceToHost, st));
  GL_CU(cudaStreamSynchronize(st));
  if (hflag[0] & 0xffffffffLL) {
    char buf[200];
    std::snprintf(buf, sizeof buf, "gridlands: layer %s is not base64: character %lld is outside the alphabet",
                  name, hflag[1]);
    return fail(SWE_EINVAL, buf);
  }
  return SWE_OK;
}

// ---- connected waterbodies (src/gridlands.mjs:107-139) ----------------------
// Wet cells (surface - bed > 0, in double) are grouped into 4-connected
// bodies by a lock-free union-find over the grid: every wet cell unites
// with its wet east and south neighbours.  A union always hangs the larger
// root under the smaller, so parent[k] <= k holds throughout and every root
// is its body's lowest cell index -- the cell the reference's row-major
// scan starts that body's flood fill from.  find() walks strictly
// decreasing indices, so it ends; a union retries only when another thread
// has just hung its root (lock-free progress), and gives up after
// CCL_TRIES attempts with an error flag rather than spin.
constexpr int CCL_TRIES = 1 << 20;

__device__ __forceinline__ bool ccl_wet(const float* bed, const float* srf, long long k) {
  return (double)srf[k] - (double)bed[k] > 0;
}

__device__ __forceinline__ int ccl_find(int* parent, int x) {
  volatile int* p = parent;
  int up = p[x];
  while (up != x) {
    const int upup = p[up];
    if (upup != up) p[x] = upup;                  // path halving: an ancestor, never a root's slot
    x = up;
    up = upup;
  }
  return x;
}

__global__ void k_ccl_init(const float* bed, const float* srf, long long n, int* parent) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    parent[k] = ccl_wet(bed, srf, k) ? (int)k : -1;
}

__global__ void k_ccl_merge(int W, int H, int* parent, int* bad) {
  const long long n = (long long)W * H;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    if (parent[k] < 0) continue;
    const int c = (int)(k % W), r = (int)(k / W);
    for (int d = 0; d < 2; d++) {
      const long long m = d == 0 ? k + 1 : k + W;
      if ((d == 0 && c + 1 >= W) || (d == 1 && r + 1 >= H) || parent[m] < 0) continue;
      int a = (int)k, b = (int)m;
      bool done = false;
      for (int it = 0; it < CCL_TRIES && !done; it++) {
        a = ccl_find(parent, a);
        b = ccl_find(parent, b);
        if (a == b) { done = true; break; }
        if (a > b) { const int t = a; a = b; b = t; }
        const int old = atomicCAS(&parent[b], b, a);   // b still a root: hang it under a
        if (old == b) done = true;
        else b = old;                                 // b was just hung elsewhere
      }
      if (!done) atomicExch(bad, 1);
    }
  }
}

// After the merge the forest no longer changes: each wet cell's root, by a
// walk that writes nothing (a shortcut written here could overwrite the
// root another thread just stored).
__global__ void k_ccl_flatten(long long n, const int* __restrict__ parent, int* __restrict__ label) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    int x = parent[k];
    if (x >= 0)
      while (parent[x] != x) x = parent[x];
    label[k] = x;
  }
}

int load_layer(const char* b64, size_t len, const float* host, long long n, float* out, cudaStream_t st,
               const char* name) {
  if (host) {
    GL_CU(cudaMemcpyAsync(out, host, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    return SWE_OK;
  }
  return decode_layer(b64, len, n, out, st, name);
}

}  // namespace

extern "C" {

int swe_gridlands_decode(const char* b64, size_t len, int n, float* out) {
  if (!out || n < 0) return fail(SWE_EINVAL, "swe_gridlands_decode: null output or negative n");
  cudaStream_t st;
  GL_CU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  DevBuf d;
  int rc = SWE_OK;
  if (cudaMalloc(&d.p, sizeof(float) * (size_t)(n > 0 ? n : 1)) != cudaSuccess) rc = fail(SWE_ECUDA, "cudaMalloc");
  if (rc == SWE_OK) rc = decode_layer(b64, len, n, static_cast<float*>(d.p), st, "data");
  if (rc == SWE_OK && n > 0) {
    if (cudaMemcpyAsync(out, d.p, sizeof(float) * n, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      rc = fail(SWE_ECUDA, "swe_gridlands_decode: copy back failed");
  }
  cudaStreamDestroy(st);
  return rc;
}

int swe_gridlands_bodies(int W, int H, const float* bed, const float* surface, int* label) {
  if (W < 1 || H < 1 || !bed || !surface || !label)
    return fail(SWE_EINVAL, "swe_gridlands_bodies: W, H >= 1 and non-null arrays");
  const long long n = (long long)W * H;
  if (n > 0x7fffffffLL) return fail(SWE_EINVAL, "swe_gridlands_bodies: more than 2^31 - 1 cells");
  cudaStream_t st;
  GL_CU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard { cudaStream_t s; ~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); } } sg{st};
  DevBuf layers, links, flag;
  GL_CU(cudaMalloc(&layers.p, sizeof(float) * n * 2));
  GL_CU(cudaMalloc(&links.p, sizeof(int) * n * 2));
  GL_CU(cudaMalloc(&flag.p, sizeof(int)));
  float* d_bed = static_cast<float*>(layers.p);
  float* d_srf = d_bed + n;
  int* parent = static_cast<int*>(links.p);
  int* d_label = parent + n;
  GL_CU(cudaMemcpyAsync(d_bed, bed, sizeof(float) * n, cudaMemcpyHostToDevice, st));
  GL_CU(cudaMemcpyAsync(d_srf, surface, sizeof(float) * n, cudaMemcpyHostToDevice, st));
  GL_CU(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
  const int nb = grid_blocks(n);
  k_ccl_init<<<nb, 256, 0, st>>>(d_bed, d_srf, n, parent);
  k_ccl_merge<<<nb, 256, 0, st>>>(W, H, parent, static_cast<int*>(flag.p));
  k_ccl_flatten<<<nb, 256, 0, st>>>(n, parent, d_label);
  GL_CU(cudaGetLastError());
  int bad = 0;
  GL_CU(cudaMemcpyAsync(&bad, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  GL_CU(cudaMemcpyAsync(label, d_label, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  GL_CU(cudaStreamSynchronize(st));
  if (bad) return fail(SWE_ETIMEOUT, "swe_gridlands_bodies: a union did not settle within its retry limit");
  return SWE_OK;
}

int swe_gridlands_create(const swe_options* o, const swe_gridlands* g, swe_sim** out) {
  if (!out) return fail(SWE_EINVAL, "null output handle");
  *out = nullptr;
  if (!o || !g) return fail(SWE_EINVAL, "null options or terrain");
  if (o->sphere) return fail(SWE_EINVAL, "gridlands terrain is Cartesian; a spherical grid cannot take it");
  if (!(g->width > 0 && g->height > 0 && g->cell_m > 0)) {
    char buf[160];
    std::snprintf(buf, sizeof buf, "gridlands: bad grid {\"width\":%d,\"height\":%d,\"cellMeters\":%.17g}",
                  g->width, g->height, g->cell_m);
    return fail(SWE_EINVAL, buf);
  }
  if (o->nx < 1 || o->ny < 1) return fail(SWE_EINVAL, "nx and ny must be >= 1");
  const long long n = (long long)g->width * g->height;
  const bool want_n = g->manning_field != 0;
  if (want_n && !g->manning_b64 && !g->manning_f32)
    return fail(SWE_EINVAL, "gridlands: layer manningN is missing");
  cudaStream_t st;
  GL_CU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard { cudaStream_t s; ~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); } } sg{st};
  DevBuf layers, fields, flags;
  GL_CU(cudaMalloc(&layers.p, sizeof(float) * n * 3));
  float* bedM = static_cast<float*>(layers.p);
  float* surfM = bedM + n;
  float* nM = surfM + n;
  int rc = load_layer(g->bed_b64, g->bed_len, g->bed_f32, n, bedM, st, "bedM");
  if (rc == SWE_OK) rc = load_layer(g->surface_b64, g->surface_len, g->surface_f32, n, surfM, st, "surfaceM");
  if (rc == SWE_OK && want_n) rc = load_layer(g->manning_b64, g->manning_len, g->manning_f32, n, nM, st, "manningN");
  if (rc != SWE_OK) return rc;

  const int W = o->nx + 4, H = o->ny + 4;
  const long long N = (long long)W * H;
  GL_CU(cudaMalloc(&fields.p, sizeof(double) * N * 3));
  GL_CU(cudaMalloc(&flags.p, 16));
  GL_CU(cudaMemsetAsync(flags.p, 0, 8, st));
  GL_CU(cudaMemsetAsync(static_cast<char*>(flags.p) + 8, 0xff, 8, st));
  SampleArgs a;
  a.bedM = bedM; a.surfM = surfM; a.nM = want_n ? nM : nullptr;
  a.Wg = g->width; a.Hg = g->height; a.C = g->cell_m; a.flip = g->flip_rows ? 1 : 0;
  a.W = W; a.H = H; a.dx = o->dx; a.dy = o->dy;
  a.b = static_cast<double*>(fields.p); a.h = a.b + N; a.n = a.h + N;
  a.bad_n = static_cast<int*>(flags.p);
  a.bad_k = reinterpret_cast<long long*>(static_cast<char*>(flags.p) + 8);
  k_gridlands_sample<<<grid_blocks(N), 256, 0, st>>>(a);
  GL_CU(cudaGetLastError());
  long long hflag[2];
  GL_CU(cudaMemcpyAsync(hflag, flags.p, 16, cudaMemcpyDeviceToHost, st));
  GL_CU(cudaStreamSynchronize(st));
  if (want_n && (hflag[0] & 0xffffffffLL)) {
    const long long k = hflag[1];
    double v = 0;
    GL_CU(cudaMemcpy(&v, a.n + k, sizeof(double), cudaMemcpyDeviceToHost));
    const int j = (int)(k / W), i = (int)(k % W);
    char buf[240];
    std::snprintf(buf, sizeof buf, "setManningField: n = %.17g at (%.17g, %.17g); Manning n must be finite and >= 0",
                  v, ((i - 2) + 0.5) * o->dx, ((j - 2) + 0.5) * o->dy);
    return fail(SWE_EINVAL, buf);
  }
  swe_sim* s = nullptr;
  rc = swe_create(o, nullptr, nullptr, &s);
  if (rc != SWE_OK) return rc;
  rc = swe_host::adopt_fields(s, a.b, a.h, want_n ? a.n : nullptr);
  if (rc != SWE_OK) { swe_destroy(s); return rc; }
  *out = s;
  return SWE_OK;
}

}  // extern "C"
