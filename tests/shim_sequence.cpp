// shim_sequence.cpp -- drives the Node drop-in's host side (swe_shim.h, the
// class the N-API addon wraps) through the call sequences the reference's
// suites make on a ShallowWater, next to the oracle, and checks
//   - every result bit for bit against the oracle (no friction here, so
//     every operation is the same IEEE operation in the same order);
//   - what crosses PCIe: a plain step() loop moves no field, a field the
//     caller touched is uploaded and refreshed around each device call, a
//     metric row the caller holds is uploaded before each call.
// Test infrastructure: it links the oracle (oracle/liboracle_swe.so).
// Built and run by tests/test_shim_gpu.py; prints one line per check and
// exits 1 on the first failure.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "../oracle/swe_oracle.h"
#include "../water-simulator_b200/node/swe_shim.h"

namespace {

int failures = 0;

void check(bool ok, const std::string& what) {
  std::printf("%s %s\n", ok ? "PASS" : "FAIL", what.c_str());
  if (!ok) {
    failures++;
    std::fflush(stdout);
    std::exit(1);
  }
}

struct Pair {
  swe_shim::Sim* gpu = nullptr;
  oracle_sim* ref = nullptr;
  size_t N = 0;
  ~Pair() {
    delete gpu;
    if (ref) oracle_destroy(ref);
  }
};

// b and h sampled at padded cell centres as the reference's constructor does.
void make(Pair& p, const swe_options& o, const std::function<double(double, double)>& bed,
          const std::function<double(double, double)>& eta0) {
  const int W = o.nx + 4, H = o.ny + 4;
  std::vector<double> b(W * H), h(W * H);
  for (int j = 0; j < H; j++)
    for (int i = 0; i < W; i++) {
      const double x = (i - 2 + 0.5) * o.dx, y = (j - 2 + 0.5) * o.dy;
      const int k = j * W + i;
      b[k] = bed(x, y);
      const double d = eta0(x, y) - b[k];
      h[k] = d > 0 ? d : 0.0;
    }
  p.gpu = new swe_shim::Sim(o, b.data(), h.data());
  oracle_options oo;
  std::memset(&oo, 0, sizeof oo);
  oo.nx = o.nx; oo.ny = o.ny; oo.dx = o.dx; oo.dy = o.dy;
  oo.manning = o.manning; oo.min_depth = o.min_depth; oo.cfl = o.cfl; oo.coriolis = o.coriolis;
  oo.order = o.order; oo.limiter = o.limiter; oo.sphere = o.sphere;
  oo.R = o.R; oo.lat0 = o.lat0; oo.lat1 = o.lat1; oo.omega = o.omega;
  check(oracle_create(&oo, b.data(), h.data(), &p.ref) == 0, "oracle created");
  p.N = static_cast<size_t>(W) * H;
}

bool same(const double* a, const double* b, size_t n) { return std::memcmp(a, b, n * sizeof(double)) == 0; }

bool same_state(Pair& p) {
  for (int f : {SWE_FIELD_H, SWE_FIELD_HU, SWE_FIELD_HV})
    if (!same(p.gpu->field(f, false), oracle_field(p.ref, f), p.N)) return false;
  return true;
}

void bounds(Pair& p, int w, int e, int s, int n) {
  const int k[4] = {w, e, s, n};
  for (int side = 0; side < 4; side++) {
    p.gpu->setBoundary(side, k[side]);
    oracle_set_boundary(p.ref, side, k[side]);
  }
}

// tools/verify.mjs:124-136: a 200 x 4 lake at eta = 2 m over a smooth bump.
void lake_sequence() {
  swe_options o;
  swe_options_init(&o);
  o.nx = 200; o.ny = 4; o.dx = o.dy = 5; o.manning = 0;
  Pair p;
  make(p, o, [](double x, double y) { return 0.8 * std::exp(-std::pow((x - 500) / 120, 2)) + 0.15 * std::sin(y * 0.05); },
       [](double, double) { return 2.0; });
  bounds(p, SWE_BC_REFLECT, SWE_BC_REFLECT, SWE_BC_PERIODIC, SWE_BC_PERIODIC);
  const double v0 = p.gpu->volume();
  check(v0 == oracle_volume(p.ref), "lake: volume() equals the oracle's");
  const uint64_t up0 = p.gpu->bytesUp(), down0 = p.gpu->bytesDown();
  for (int s = 0; s < 400; s++) {
    const double a = p.gpu->stepAuto(), b = oracle_step_auto(p.ref);
    if (a != b) check(false, "lake: step() took the oracle's dt");
  }
  check(p.gpu->bytesUp() == up0 && p.gpu->bytesDown() == down0,
        "lake: 400 plain step() calls moved no field");
  check(same_state(p), "lake: state after 400 steps is the oracle's, bit for bit");
  check(p.gpu->maxSurfaceDeviation(2.0) <= 4 * 4.440892098500626e-16, "lake: |eta - 2| within 4 ulp");
  check(p.gpu->t() == oracle_get_scalar(p.ref, 6) && p.gpu->steps() == 400, "lake: t and steps");
}

// A disturbance written into a caller-held array between steps
// (tools/verify.mjs:264-266), then residual() / theta read back
// (tools/verify-physics.mjs:470-498), a dryClean, and the device loop.
void written_field_sequence() {
  swe_options o;
  swe_options_init(&o);
  o.nx = 90; o.ny = 40; o.dx = o.dy = 4; o.manning = 0;
  Pair p;
  make(p, o, [](double x, double y) { return -2 + x / 50 + 0.2 * std::sin(y / 13); },
       [](double x, double) { return x < 60 ? 1.0 : 0.0; });
  bounds(p, SWE_BC_REFLECT, SWE_BC_OUTFLOW, SWE_BC_REFLECT, SWE_BC_REFLECT);
  const size_t N = p.N;
  double* h = p.gpu->expose(SWE_FIELD_H);           // held like `const h = sim.h`
  double* hr = oracle_field(p.ref, OF_H);
  const int W = o.nx + 4;
  for (int s = 0; s < 10; s++) {
    const int k = (10 + s) * W + 20 + s;
    h[k] += 0.05;                                   // the caller writes the array it holds
    hr[k] += 0.05;
    const uint64_t up = p.gpu->bytesUp(), down = p.gpu->bytesDown();
    const double dt = oracle_max_dt(p.ref);
    check(p.gpu->maxDt() == dt, "written: maxDt sees the write");
    p.gpu->step(dt);
    oracle_step(p.ref, dt);
    // a held field goes up before every device call: maxDt(), then step()
    check(p.gpu->bytesUp() - up == 2 * N * sizeof(double), "written: the held field went up before each call");
    check(p.gpu->bytesDown() - down == N * sizeof(double), "written: and came back once");
    check(same(h, hr, N), "written: the held array is the current state");
  }
  check(same_state(p), "written: state is the oracle's");
  for (double mult : {1.0, 5.0}) {
    const double dt = mult * oracle_max_dt(p.ref);
    p.gpu->applyBC();
    oracle_apply_bc(p.ref);
    p.gpu->residual(dt);
    oracle_residual(p.ref, dt);
    bool ok = true;
    for (int f : {SWE_FIELD_RH, SWE_FIELD_RHU, SWE_FIELD_RHV, SWE_FIELD_THETA})
      ok = ok && same(p.gpu->field(f, false), oracle_field(p.ref, f), N);
    check(ok, "residual: rh, rhu, rhv, theta are the oracle's at " + std::to_string(mult) + "x the CFL step");
  }
  check(p.gpu->dryClean() == oracle_dry_clean(p.ref), "dryClean: the same floored mass");
  check(same(h, hr, N), "dryClean: the held array is current");
  const int done = p.gpu->run(25, 0, INFINITY);
  for (int s = 0; s < 25; s++) oracle_step_auto(p.ref);
  check(done == 25 && same_state(p), "run(25): the device loop equals 25 oracle steps");
  check(p.gpu->energy() == oracle_energy(p.ref), "energy() equals the oracle's");
}

// Flather values evaluated at sim.t before each step (src/swe.mjs:1093).
void flather_sequence() {
  swe_options o;
  swe_options_init(&o);
  o.nx = 120; o.ny = 6; o.dx = o.dy = 5; o.manning = 0;
  Pair p;
  make(p, o, [](double x, double) { return -10 + x / 100; }, [](double, double) { return 0.0; });
  bounds(p, SWE_BC_FLATHER, SWE_BC_FLATHER, SWE_BC_PERIODIC, SWE_BC_PERIODIC);
  const uint64_t up0 = p.gpu->bytesUp(), down0 = p.gpu->bytesDown();
  for (int s = 0; s < 40; s++) {
    const double t = p.gpu->t();
    const double e = 0.4 * std::sin(2 * M_PI * t / 60), u = std::sqrt(9.80665 / 10) * e;
    p.gpu->setFlatherValues(SWE_SIDE_WEST, e, u);
    p.gpu->setFlatherValues(SWE_SIDE_EAST, 0, 0);
    oracle_set_flather_values(p.ref, SWE_SIDE_WEST, e, u);
    oracle_set_flather_values(p.ref, SWE_SIDE_EAST, 0, 0);
    const double dt = oracle_max_dt(p.ref);
    p.gpu->step(dt);
    oracle_step(p.ref, dt);
  }
  check(p.gpu->bytesUp() == up0 && p.gpu->bytesDown() == down0, "flather: 40 steps moved no field");
  check(same_state(p), "flather: state is the oracle's after 40 steps");
}

// A metric row written by the caller (tools/verify-sphere.mjs:569-572).
void geometry_sequence() {
  swe_options o;
  swe_options_init(&o);
  o.nx = 60; o.ny = 30; o.sphere = 1; o.lat0 = -60; o.lat1 = 60; o.manning = 0;
  o.omega = 7.292115e-5;
  Pair p;
  // sample at (lon, lat) from the library's own metric
  {
    double rows[13 * 34], sc[6];
    check(swe_compute_geometry(&o, rows, sc) == SWE_OK, "sphere: geometry computed");
    const int W = o.nx + 4, H = o.ny + 4;
    std::vector<double> b(W * H), h(W * H);
    for (int j = 0; j < H; j++)
      for (int i = 0; i < W; i++) {
        const double lon = std::fmod(std::fmod((i - 2 + 0.5) * sc[3] * 180 / M_PI, 360) + 360, 360) - 180;
        const double lat = rows[9 * H + j] * 180 / M_PI;
        const int k = j * W + i;
        b[k] = -4000 + 900 * std::sin(3 * lon * M_PI / 180) * std::cos(2 * lat * M_PI / 180);
        const double e = 2 * std::exp(-((lon - 20) * (lon - 20) + (lat - 30) * (lat - 30)) / 300);
        h[k] = e - b[k] > 0 ? e - b[k] : 0;
      }
    p.gpu = new swe_shim::Sim(o, b.data(), h.data());
    oracle_options oo;
    std::memset(&oo, 0, sizeof oo);
    oo.nx = o.nx; oo.ny = o.ny; oo.dx = o.dx; oo.dy = o.dy; oo.manning = 0; oo.min_depth = o.min_depth;
    oo.cfl = o.cfl; oo.order = o.order; oo.limiter = o.limiter; oo.sphere = 1;
    oo.R = o.R; oo.lat0 = o.lat0; oo.lat1 = o.lat1; oo.omega = o.omega;
    check(oracle_create(&oo, b.data(), h.data(), &p.ref) == 0, "sphere: oracle created");
    p.N = static_cast<size_t>(W) * H;
  }
  check(same(p.gpu->geom(SWE_GEOM_BEDPHI, false), oracle_geom(p.ref, OG_BEDPHI), o.ny + 4),
        "sphere: bedPhi row equals the oracle's");
  double* row = p.gpu->geom(SWE_GEOM_DYCFL, true);
  double* rref = oracle_geom(p.ref, OG_DYCFL);
  for (int j = 0; j < o.ny + 4; j++) { row[j] *= 0.5; rref[j] *= 0.5; }
  check(p.gpu->maxDt() == oracle_max_dt(p.ref), "sphere: a written dyCFL row reaches maxDt");
  for (int s = 0; s < 12; s++) {
    row[7] = rref[7] = row[7] * (1 + 1e-3);       // written again while held
    const double dt = oracle_max_dt(p.ref);
    check(p.gpu->maxDt() == dt, "sphere: the held row is uploaded before each call");
    p.gpu->step(dt);
    oracle_step(p.ref, dt);
  }
  check(same_state(p), "sphere: state is the oracle's after 12 steps");
  check(p.gpu->volume() == oracle_volume(p.ref), "sphere: volume() equals the oracle's");
}

// Errors the reference throws come back as exceptions with its message.
void error_sequence() {
  swe_options o;
  swe_options_init(&o);
  o.nx = 8; o.ny = 8; o.dx = o.dy = 1; o.limiter = 7;
  std::vector<double> z(12 * 12, 0.0);
  bool threw = false;
  try {
    swe_shim::Sim s(o, z.data(), z.data());
  } catch (const swe_shim::Error& e) {
    threw = e.code == SWE_EINVAL;
  }
  check(threw, "errors: an unknown limiter throws EINVAL");
  o.limiter = SWE_LIMITER_MC;
  swe_shim::Sim s(o, z.data(), z.data());
  threw = false;
  try {
    s.field(SWE_FIELD_THETA, true);
  } catch (const swe_shim::Error&) {
    threw = true;
  }
  check(threw, "errors: theta is read-only");
  check(s.step(-1.0) == 0 && s.step(NAN) == 0, "errors: step() refuses a bad dt with 0");
}

}  // namespace

int main() {
  lake_sequence();
  written_field_sequence();
  flather_sequence();
  geometry_sequence();
  error_sequence();
  std::printf("ALL PASS\n");
  return failures ? 1 : 0;
}
