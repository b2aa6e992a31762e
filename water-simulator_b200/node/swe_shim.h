// swe_shim.h -- the host side of the Node drop-in: one ShallowWater's host
// mirrors over the C ABI, with per-field dirty tracking.
//
// The reference's callers (tools/verify*.mjs, src/globe.mjs, index.html)
// treat a ShallowWater (src/swe.mjs:145-918) as a bag of Float64Array
// fields they read and write between calls: sim.h[k] = ..., then
// sim.step(); sim.theta[k] after sim.residual(dt); sim.geom.bedPhi[j] = ...
// (tools/verify-physics.mjs:79-97, tools/verify-sphere.mjs:569-572).  The
// library owns the state on the device, so this class keeps one host copy
// of each field and knows, per field, whether that copy is
//   fresh  -- equal to the device's (nothing to download before a read),
//   dirty  -- written by the caller (upload before the next device call).
// A device call that changes a field makes its host copy stale; a read
// downloads it once; a write marks it dirty.  A plain step() loop whose
// caller touches no field therefore moves no field across PCIe at all; the
// byte counters below let a test check exactly that.
//
// JavaScript holds a field as one Float64Array for the life of the object
// (`const h = sim.h;` before a loop of steps) and writes it without telling
// anyone.  A field handed out that way is "exposed": it is uploaded before
// every device call (it may have been written) and downloaded again after
// every device call that changes it, so the array the caller holds is always
// the current state.  Only the fields a caller actually touched pay for it.
//
// It is plain C++ over include/swe_b200.h (no Node types), so the N-API glue
// in swe_napi.cc stays a thin wrapper and this part is compiled and tested
// without a JS engine (tests/shim_sequence.cpp).
#pragma once

#include "../../include/swe_b200.h"

#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace swe_shim {

// The reference throws; the addon turns this into a JS exception.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
  if (rc != SWE_OK) {
    const char* m = swe_last_error();
    throw Error(rc, m ? m : "swe_b200 error");
  }
}

// Field ids of include/swe_b200.h; the first four are writable state.
enum Field { kB = SWE_FIELD_B, kH = SWE_FIELD_H, kHU = SWE_FIELD_HU, kHV = SWE_FIELD_HV,
             kH0 = SWE_FIELD_H0, kHU0 = SWE_FIELD_HU0, kHV0 = SWE_FIELD_HV0,
             kRH = SWE_FIELD_RH, kRHU = SWE_FIELD_RHU, kRHV = SWE_FIELD_RHV, kTHETA = SWE_FIELD_THETA,
             kNFIELDS = 11 };

class Sim {
 public:
  // new ShallowWater(opts) with the sampled bed and depth over the padded
  // grid (the addon samples bed()/eta0() per cell, src/swe.mjs:222-232).
  Sim(const swe_options& o, const double* b, const double* h) {
    check(swe_create(&o, b, h, &s_));
    int d[4];
    check(swe_get_dims(s_, d));
    W_ = d[0]; H_ = d[1]; nx_ = d[2]; ny_ = d[3];
    N_ = static_cast<size_t>(W_) * H_;
    for (int f = 0; f < kNFIELDS; f++) {
      host_[f].assign(N_, 0.0);
      fresh_[f] = false; dirty_[f] = false; exposed_[f] = false;
    }
    // the state just given is what the device holds
    std::copy(b, b + N_, host_[kB].begin()); fresh_[kB] = true;
    std::copy(h, h + N_, host_[kH].begin()); fresh_[kH] = true;
    fresh_[kHU] = fresh_[kHV] = true;                       // zero on both sides
    for (int r = 0; r < SWE_GEOM_NROWS; r++) {
      geom_[r].assign(H_, 0.0);
      check(swe_get_geom(s_, r, geom_[r].data()));
      geom_dirty_[r] = false;
    }
  }
  ~Sim() { if (s_) swe_destroy(s_); }
  Sim(const Sim&) = delete;
  Sim& operator=(const Sim&) = delete;

  int W() const { return W_; }
  int H() const { return H_; }
  int nx() const { return nx_; }
  int ny() const { return ny_; }
  size_t N() const { return N_; }
  swe_sim* handle() { return s_; }

  // ---- field access ------------------------------------------------------
  // The host copy of a field, downloaded first if stale.  `write`: the
  // caller may change it (only b, h, hu, hv), so it is uploaded before the
  // next device call.  The pointer stays valid for the life of the Sim.
  double* field(int f, bool write) {
    if (f < 0 || f >= kNFIELDS) throw Error(SWE_EINVAL, "unknown field id");
    if (write && f > kHV) throw Error(SWE_EINVAL, "only b, h, hu and hv are writable");
    if (f >= kH0 && f <= kHV0 && !keep_h0_) { check(swe_set_keep_h0(s_, 1)); keep_h0_ = true; }
    if (!fresh_[f] && !dirty_[f]) {
      check(swe_get_field(s_, f, host_[f].data()));
      bytes_down_ += N_ * sizeof(double);
      fresh_[f] = true;
    }
    if (write) dirty_[f] = true;
    return host_[f].data();
  }
  // The field as a caller-held array (see the header comment): current now
  // and after every later device call, uploaded before each one.
  double* expose(int f) {
    double* p = field(f, false);
    exposed_[f] = true;
    return p;
  }
  // A metric row (sim.geom.<row>).  Only the caller changes the metric, so
  // the host copy is always current; a row handed out writable is uploaded
  // before every later device call (H doubles), as the caller may write it
  // at any time (tools/verify-sphere.mjs:569-572).
  double* geom(int row, bool write) {
    if (row < 0 || row >= SWE_GEOM_NROWS) throw Error(SWE_EINVAL, "unknown geometry row");
    if (write) geom_dirty_[row] = true;
    return geom_[row].data();
  }

  // ---- the solver (src/swe.mjs) -------------------------------------------
  void setBoundary(int side, int kind) { check(swe_set_boundary(s_, side, kind)); }
  // flather(etaExt, uExt) with the two values the caller evaluated at t.
  void setFlatherValues(int side, double eta, double u) { check(swe_set_flather_values(s_, side, eta, u)); }
  void setFlatherTide(int side, double msl, int n, const double* amp, const double* omega,
                      const double* phase_deg, double u_coef) {
    check(swe_set_flather_tide(s_, side, msl, n, amp, omega, phase_deg, u_coef));
  }
  void setManningField(const double* n) { push(); check(swe_set_manning_field(s_, n)); }
  void setSponge(int side, int width, double strength, double eta_ref) {
    check(swe_set_sponge(s_, side, width, strength, eta_ref));
  }
  void clearSponge() { check(swe_clear_sponge(s_)); }

  void applyBC() { push(); check(swe_apply_bc(s_)); stale({kB, kH, kHU, kHV}); }
  void residual(double dt) { push(); check(swe_residual(s_, dt)); stale({kRH, kRHU, kRHV, kTHETA}); }
  double maxDt() { push(); double v = 0; check(swe_max_dt(s_, &v)); return v; }
  void applyFriction(double dt) { push(); check(swe_apply_friction(s_, dt)); stale({kHU, kHV}); }
  double dryClean() { push(); double v = 0; check(swe_dry_clean(s_, &v)); stale({kH, kHU, kHV}); return v; }
  // step(dt) / step(): the dt taken, 0 when refused (src/swe.mjs:783-784).
  double step(double dt) {
    push();
    double taken = 0;
    check(swe_step(s_, dt, &taken));
    if (taken != 0) stale({kB, kH, kHU, kHV, kH0, kHU0, kHV0});
    return taken;
  }
  double stepAuto() {
    push();
    double taken = 0;
    check(swe_step_auto(s_, &taken));
    if (taken != 0) stale({kB, kH, kHU, kHV, kH0, kHU0, kHV0});
    return taken;
  }
  // The drivers' loop kept on the device (swe_run).
  int run(int n, double dt_fixed, double t_end) {
    push();
    int done = 0;
    check(swe_run(s_, n, dt_fixed, t_end, &done));
    if (done) stale({kB, kH, kHU, kHV, kH0, kHU0, kHV0});
    return done;
  }
  double volume() { push(); double v = 0; check(swe_volume(s_, &v)); return v; }
  double energy() { push(); double v = 0; check(swe_energy(s_, &v)); return v; }
  double maxSurfaceDeviation(double ref) {
    push(); double v = 0; check(swe_max_surface_deviation(s_, ref, &v)); return v;
  }
  double maxSpeed() { push(); double v = 0; check(swe_max_speed(s_, &v)); return v; }
  bool finite() { push(); int v = 0; check(swe_finite(s_, &v)); return v != 0; }
  double vel(double hq, double h) { double v = 0; check(swe_vel_batch(s_, 1, &hq, &h, &v)); return v; }

  double scalar(int which) { double v = 0; check(swe_get_scalar(s_, which, &v)); return v; }
  void setScalar(int which, double v) { check(swe_set_scalar(s_, which, v)); }
  double t() { return scalar(SWE_SCALAR_T); }
  double steps() { return scalar(SWE_SCALAR_STEPS); }
  double massFloored() { return scalar(SWE_SCALAR_MASS_FLOORED); }

  // bytes moved between the host copies and the device so far
  uint64_t bytesUp() const { return bytes_up_; }
  uint64_t bytesDown() const { return bytes_down_; }

 private:
  // Upload what the caller wrote; the device copy then equals the host's.
  void push() {
    for (int f = kB; f <= kHV; f++) {
      if (!dirty_[f] && !exposed_[f]) continue;
      check(swe_set_field(s_, f, host_[f].data()));
      bytes_up_ += N_ * sizeof(double);
      dirty_[f] = false;
      fresh_[f] = true;
    }
    for (int r = 0; r < SWE_GEOM_NROWS; r++) {
      if (!geom_dirty_[r]) continue;              // stays set: the caller holds the row
      check(swe_set_geom(s_, r, geom_[r].data()));
      bytes_up_ += geom_[r].size() * sizeof(double);
    }
  }
  void stale(std::initializer_list<int> fs) {
    for (int f : fs) {
      fresh_[f] = false;
      if (exposed_[f]) field(f, false);          // keep the caller's array current
    }
  }

  swe_sim* s_ = nullptr;
  int W_ = 0, H_ = 0, nx_ = 0, ny_ = 0;
  size_t N_ = 0;
  std::vector<double> host_[kNFIELDS];
  bool fresh_[kNFIELDS];
  bool dirty_[kNFIELDS];
  bool exposed_[kNFIELDS];
  std::vector<double> geom_[SWE_GEOM_NROWS];
  bool geom_dirty_[SWE_GEOM_NROWS];
  bool keep_h0_ = false;
  uint64_t bytes_up_ = 0, bytes_down_ = 0;
};

}  // namespace swe_shim
