// swe_napi.cc -- the Node N-API addon behind swe-gpu.mjs.
//
// A thin wrapper: each method unwraps the swe_shim::Sim held by the JS
// object, calls it, and turns a swe_shim::Error into a JS exception with
// the library's message (the reference's own texts, e.g. "unknown limiter"
// from src/swe.mjs:195).  Fields are handed to JS as Float64Arrays over the
// shim's host copies (external ArrayBuffers, no copy); the shim keeps those
// arrays current (swe_shim.h, "exposed" fields).
//
// Built with node-gyp (binding.gyp) against libswe_b200.so.  There is no
// JS engine and no node_api.h on the machine this repository is built on,
// so this file is not compiled here; the logic it wraps is swe_shim.h,
// which tests/shim_sequence.cpp compiles and runs on the GPU.
#include <node_api.h>

#include <string>
#include <vector>

#include "swe_shim.h"

namespace {

#define NAPI_OK(call)                                                  \
  do {                                                                 \
    if ((call) != napi_ok) {                                           \
      napi_throw_error(env, nullptr, "swe_napi: N-API call failed");   \
      return nullptr;                                                  \
    }                                                                  \
  } while (0)

struct Args {
  napi_value self = nullptr;
  napi_value argv[8] = {};
  size_t argc = 8;
};

napi_value args(napi_env env, napi_callback_info info, Args* a) {
  NAPI_OK(napi_get_cb_info(env, info, &a->argc, a->argv, &a->self, nullptr));
  return a->self;
}

swe_shim::Sim* unwrap(napi_env env, napi_value self) {
  void* p = nullptr;
  if (napi_unwrap(env, self, &p) != napi_ok || !p) {
    napi_throw_error(env, nullptr, "ShallowWater: the native simulation is gone");
    return nullptr;
  }
  return static_cast<swe_shim::Sim*>(p);
}

double num(napi_env env, napi_value v, double dflt) {
  napi_valuetype t;
  if (!v || napi_typeof(env, v, &t) != napi_ok || t != napi_number) return dflt;
  double d = dflt;
  napi_get_value_double(env, v, &d);
  return d;
}

double prop(napi_env env, napi_value obj, const char* name, double dflt) {
  napi_value v;
  bool has = false;
  if (napi_has_named_property(env, obj, name, &has) != napi_ok || !has) return dflt;
  if (napi_get_named_property(env, obj, name, &v) != napi_ok) return dflt;
  return num(env, v, dflt);
}

double* f64(napi_env env, napi_value v, size_t* n) {
  napi_typedarray_type t;
  void* data = nullptr;
  size_t len = 0;
  if (napi_get_typedarray_info(env, v, &t, &len, &data, nullptr, nullptr) != napi_ok ||
      t != napi_float64_array) {
    napi_throw_type_error(env, nullptr, "expected a Float64Array");
    return nullptr;
  }
  if (n) *n = len;
  return static_cast<double*>(data);
}

napi_value dbl(napi_env env, double d) {
  napi_value r;
  napi_create_double(env, d, &r);
  return r;
}

// Run f(sim); a library error becomes a JS Error carrying its message.
template <class F>
napi_value guarded(napi_env env, napi_callback_info info, F f) {
  Args a;
  if (!args(env, info, &a)) return nullptr;
  swe_shim::Sim* s = unwrap(env, a.self);
  if (!s) return nullptr;
  try {
    return f(s, a);
  } catch (const swe_shim::Error& e) {
    napi_throw_error(env, std::to_string(e.code).c_str(), e.what());
    return nullptr;
  }
}

// new Native(options, b, h): options carries nx, ny, dx, dy, manning,
// minDepth, cfl, coriolis, order, limiter (0 mc, 1 minmod, 2 central),
// sphere (0/1), R, lat0, lat1, omega; b and h are Float64Arrays over the
// padded grid, sampled by the JS side as the reference's constructor does.
napi_value Construct(napi_env env, napi_callback_info info) {
  Args a;
  if (!args(env, info, &a)) return nullptr;
  if (a.argc < 3) {
    napi_throw_type_error(env, nullptr, "Native(options, b, h)");
    return nullptr;
  }
  swe_options o;
  swe_options_init(&o);
  napi_value opt = a.argv[0];
  o.nx = static_cast<int>(prop(env, opt, "nx", 0));
  o.ny = static_cast<int>(prop(env, opt, "ny", 0));
  o.dx = prop(env, opt, "dx", o.dx);
  o.dy = prop(env, opt, "dy", o.dx);
  o.manning = prop(env, opt, "manning", o.manning);
  o.min_depth = prop(env, opt, "minDepth", o.min_depth);
  o.cfl = prop(env, opt, "cfl", o.cfl);
  o.coriolis = prop(env, opt, "coriolis", o.coriolis);
  o.order = static_cast<int>(prop(env, opt, "order", o.order));
  o.limiter = static_cast<int>(prop(env, opt, "limiter", o.limiter));
  o.sphere = static_cast<int>(prop(env, opt, "sphere", 0));
  o.R = prop(env, opt, "R", o.R);
  o.lat0 = prop(env, opt, "lat0", o.lat0);
  o.lat1 = prop(env, opt, "lat1", o.lat1);
  o.omega = prop(env, opt, "omega", o.omega);
  size_t nb = 0, nh = 0;
  double* b = f64(env, a.argv[1], &nb);
  double* h = f64(env, a.argv[2], &nh);
  if (!b || !h) return nullptr;
  if (nb != nh || nb != static_cast<size_t>(o.nx + 4) * static_cast<size_t>(o.ny + 4)) {
    napi_throw_range_error(env, nullptr, "b and h must hold (nx + 4) * (ny + 4) values");
    return nullptr;
  }
  swe_shim::Sim* s = nullptr;
  try {
    s = new swe_shim::Sim(o, b, h);
  } catch (const swe_shim::Error& e) {
    napi_throw_error(env, std::to_string(e.code).c_str(), e.what());
    return nullptr;
  }
  NAPI_OK(napi_wrap(env, a.self, s, [](napi_env, void* p, void*) { delete static_cast<swe_shim::Sim*>(p); },
                    nullptr, nullptr));
  return a.self;
}

// field(id): the field as a Float64Array over the shim's host copy.
napi_value Field(napi_env env, napi_callback_info info) {
  return guarded(env, info, [env](swe_shim::Sim* s, Args& a) -> napi_value {
    const int id = static_cast<int>(num(env, a.argv[0], -1));
    double* p = s->expose(id);
    napi_value buf, arr;
    NAPI_OK(napi_create_external_arraybuffer(env, p, s->N() * sizeof(double), nullptr, nullptr, &buf));
    NAPI_OK(napi_create_typedarray(env, napi_float64_array, s->N(), buf, 0, &arr));
    return arr;
  });
}

// geom(row): a metric row as a Float64Array; writes reach the device at the
// next call (the shim uploads rows handed out this way).
napi_value Geom(napi_env env, napi_callback_info info) {
  return guarded(env, info, [env](swe_shim::Sim* s, Args& a) -> napi_value {
    const int row = static_cast<int>(num(env, a.argv[0], -1));
    double* p = s->geom(row, true);
    napi_value buf, arr;
    NAPI_OK(napi_create_external_arraybuffer(env, p, s->H() * sizeof(double), nullptr, nullptr, &buf));
    NAPI_OK(napi_create_typedarray(env, napi_float64_array, s->H(), buf, 0, &arr));
    return arr;
  });
}

#define METHOD0(NAME, EXPR)                                                          \
  napi_value NAME(napi_env env, napi_callback_info info) {                           \
    return guarded(env, info, [env](swe_shim::Sim* s, Args& a) -> napi_value {       \
      (void)a;                                                                       \
      return EXPR;                                                                   \
    });                                                                              \
  }

METHOD0(ApplyBC, (s->applyBC(), nullptr))
METHOD0(MaxDt, dbl(env, s->maxDt()))
METHOD0(DryClean, dbl(env, s->dryClean()))
METHOD0(StepAuto, dbl(env, s->stepAuto()))
METHOD0(Volume, dbl(env, s->volume()))
METHOD0(Energy, dbl(env, s->energy()))
METHOD0(MaxSpeed, dbl(env, s->maxSpeed()))
METHOD0(T, dbl(env, s->t()))
METHOD0(Steps, dbl(env, s->steps()))
METHOD0(MassFloored, dbl(env, s->massFloored()))
METHOD0(ClearSponge, (s->clearSponge(), nullptr))

napi_value Finite(napi_env env, napi_callback_info info) {
  return guarded(env, info, [env](swe_shim::Sim* s, Args&) -> napi_value {
    napi_value r;
    napi_get_boolean(env, s->finite(), &r);
    return r;
  });
}

#define METHOD_D(NAME, CALL)                                                         \
  napi_value NAME(napi_env env, napi_callback_info info) {                           \
    return guarded(env, info, [env](swe_shim::Sim* s, Args& a) -> napi_value {       \
      const double x = num(env, a.argv[0], 0);                                       \
      return CALL;                                                                   \
    });                                                                              \
  }

METHOD_D(Residual, (s->residual(x), nullptr))
METHOD_D(ApplyFriction, (s->applyFriction(x), nullptr))
METHOD_D(Step, dbl(env, s->step(x)))
METHOD_D(MaxSurfaceDeviation, dbl(env, s->maxSurfaceDeviation(x)))
METHOD_D(SetT, (s->setScalar(SWE_SCALAR_T, x), nullptr))
METHOD_D(SetSteps, (s->setScalar(SWE_SCALAR_STEPS, x), nullptr))

// vel(hq, h)
napi_value Vel(napi_env env, napi_callback_info info) {
  return guarded(env, info, [env](swe_shim::Sim* s, Args& a) -> napi_value {
    return dbl(env, s->vel(num(env, a.argv[0], 0), num(env, a.argv[1], 0)));
  });
}

// run(n, dtFixed, tEnd): steps taken
napi_value Run(napi_env env, napi_callback_info info) {
  return guarded(env, info, [env](swe_shim::Sim* s, Args& a) -> napi_value {
    const int n = static_cast<int>(num(env, a.argv[0], 0));
    const double dt = num(env, a.argv[1], 0);
    const double tEnd = num(env, a.argv[2], INFINITY);
    return dbl(env, s->run(n, dt, tEnd));
  });
}

// setBoundary(side, kind)
napi_value SetBoundary(napi_env env, napi_callback_info info) {
  return guarded(env, info, [env](swe_shim::Sim* s, Args& a) -> napi_value {
    s->setBoundary(static_cast<int>(num(env, a.argv[0], -1)), static_cast<int>(num(env, a.argv[1], -1)));
    return nullptr;
  });
}

// setFlatherValues(side, etaExt(t), uExt(t))
napi_value SetFlatherValues(napi_env env, napi_callback_info info) {
  return guarded(env, info, [env](swe_shim::Sim* s, Args& a) -> napi_value {
    s->setFlatherValues(static_cast<int>(num(env, a.argv[0], -1)), num(env, a.argv[1], 0),
                        num(env, a.argv[2], 0));
    return nullptr;
  });
}

// setFlatherTide(side, msl, amp[], omega[], phaseDeg[], uCoef)
napi_value SetFlatherTide(napi_env env, napi_callback_info info) {
  return guarded(env, info, [env](swe_shim::Sim* s, Args& a) -> napi_value {
    size_t n1 = 0, n2 = 0, n3 = 0;
    double* amp = f64(env, a.argv[2], &n1);
    double* om = f64(env, a.argv[3], &n2);
    double* ph = f64(env, a.argv[4], &n3);
    if (!amp || !om || !ph) return nullptr;
    if (n1 != n2 || n1 != n3) {
      napi_throw_range_error(env, nullptr, "tide tables of unequal length");
      return nullptr;
    }
    s->setFlatherTide(static_cast<int>(num(env, a.argv[0], -1)), num(env, a.argv[1], 0), static_cast<int>(n1),
                      amp, om, ph, num(env, a.argv[5], 0));
    return nullptr;
  });
}

// setManningField(Float64Array | null)
napi_value SetManningField(napi_env env, napi_callback_info info) {
  return guarded(env, info, [env](swe_shim::Sim* s, Args& a) -> napi_value {
    napi_valuetype t;
    napi_typeof(env, a.argv[0], &t);
    if (t == napi_null || t == napi_undefined) {
      s->setManningField(nullptr);
      return nullptr;
    }
    size_t n = 0;
    double* p = f64(env, a.argv[0], &n);
    if (!p) return nullptr;
    if (n != s->N()) {
      napi_throw_range_error(env, nullptr, "a Manning field holds (nx + 4) * (ny + 4) values");
      return nullptr;
    }
    s->setManningField(p);
    return nullptr;
  });
}

// setSponge(side, width, strength, etaRef)
napi_value SetSponge(napi_env env, napi_callback_info info) {
  return guarded(env, info, [env](swe_shim::Sim* s, Args& a) -> napi_value {
    s->setSponge(static_cast<int>(num(env, a.argv[0], 1)), static_cast<int>(num(env, a.argv[1], 20)),
                 num(env, a.argv[2], 0.06), num(env, a.argv[3], 0));
    return nullptr;
  });
}

// dims(): [W, H, nx, ny]
napi_value Dims(napi_env env, napi_callback_info info) {
  return guarded(env, info, [env](swe_shim::Sim* s, Args&) -> napi_value {
    napi_value arr;
    NAPI_OK(napi_create_array_with_length(env, 4, &arr));
    const int v[4] = {s->W(), s->H(), s->nx(), s->ny()};
    for (uint32_t q = 0; q < 4; q++) {
      napi_value x;
      napi_create_int32(env, v[q], &x);
      napi_set_element(env, arr, q, x);
    }
    return arr;
  });
}

// scalar(id): SWE_SCALAR_* (dx, dy, R, dlam, dphi, totalArea, ...)
napi_value Scalar(napi_env env, napi_callback_info info) {
  return guarded(env, info, [env](swe_shim::Sim* s, Args& a) -> napi_value {
    return dbl(env, s->scalar(static_cast<int>(num(env, a.argv[0], -1))));
  });
}

// hllc(hL, huL, hvL, hR, huR, hvR, dry) -> [mass, normal, transverse]
// (the module-level export of src/swe.mjs:975; no simulation needed)
napi_value Hllc(napi_env env, napi_callback_info info) {
  size_t argc = 7;
  napi_value argv[7];
  NAPI_OK(napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr));
  double in[7];
  for (int q = 0; q < 7; q++) in[q] = q < static_cast<int>(argc) ? num(env, argv[q], 0) : 1e-4;
  double out[3] = {0, 0, 0};
  if (swe_hllc_batch(1, in, out) != SWE_OK) {
    napi_throw_error(env, nullptr, swe_last_error());
    return nullptr;
  }
  napi_value arr;
  NAPI_OK(napi_create_array_with_length(env, 3, &arr));
  for (uint32_t q = 0; q < 3; q++) napi_set_element(env, arr, q, dbl(env, out[q]));
  return arr;
}

}  // namespace

NAPI_MODULE_INIT() {
  const napi_property_descriptor methods[] = {
      {"field", nullptr, Field, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"geom", nullptr, Geom, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"applyBC", nullptr, ApplyBC, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"residual", nullptr, Residual, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"maxDt", nullptr, MaxDt, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"applyFriction", nullptr, ApplyFriction, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"dryClean", nullptr, DryClean, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"step", nullptr, Step, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"stepAuto", nullptr, StepAuto, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"run", nullptr, Run, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"volume", nullptr, Volume, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"energy", nullptr, Energy, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"maxSurfaceDeviation", nullptr, MaxSurfaceDeviation, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"maxSpeed", nullptr, MaxSpeed, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"finite", nullptr, Finite, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"vel", nullptr, Vel, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setBoundary", nullptr, SetBoundary, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setFlatherValues", nullptr, SetFlatherValues, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setFlatherTide", nullptr, SetFlatherTide, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setManningField", nullptr, SetManningField, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setSponge", nullptr, SetSponge, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"clearSponge", nullptr, ClearSponge, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"t", nullptr, T, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setT", nullptr, SetT, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"steps", nullptr, Steps, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setSteps", nullptr, SetSteps, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"massFloored", nullptr, MassFloored, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"dims", nullptr, Dims, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"scalar", nullptr, Scalar, nullptr, nullptr, nullptr, napi_default, nullptr},
  };
  napi_value cls;
  if (napi_define_class(env, "Native", NAPI_AUTO_LENGTH, Construct, nullptr, sizeof methods / sizeof *methods,
                        methods, &cls) != napi_ok)
    return nullptr;
  napi_set_named_property(env, exports, "Native", cls);
  napi_value fn;
  napi_create_function(env, "hllc", NAPI_AUTO_LENGTH, Hllc, nullptr, &fn);
  napi_set_named_property(env, exports, "hllc", fn);
  return exports;
}
