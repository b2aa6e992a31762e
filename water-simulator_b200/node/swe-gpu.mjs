// swe-gpu.mjs -- ShallowWater on the B200 library, with the reference's API.
//
// A drop-in for the class and exports of src/swe.mjs (Syntaxswine/
// water-simulator): the same constructor options, fields, methods, errors
// and module exports, with the arithmetic in libswe_b200.so (CUDA, FP64)
// through the N-API addon built from swe_napi.cc.  The suites switch with
// one import line (or an import map):
//     import { ShallowWater, reflect, flather, G } from './swe-gpu.mjs';
//
// Fields (sim.h, sim.hu, ..., sim.theta) are Float64Arrays over the addon's
// host copies.  A field the caller has touched is kept current after every
// device call and uploaded before the next one (swe_shim.h); fields nobody
// touches never cross PCIe, so a plain `sim.step()` loop moves no field.
// Boundaries are recognised by identity (reflect, outflow, periodic) or as
// a flather() of this module; their values are evaluated on the host at
// sim.t before each step, as the reference evaluates them
// (src/swe.mjs:1085-1115).  Any other forcing function runs on the host
// after the step, on the current fields (src/swe.mjs:809).
//
// Not compiled or run where this repository is built (no JS engine there);
// the class logic underneath it, swe_shim.h, is what tests/ exercises.
import { createRequire } from 'node:module';

const require = createRequire(import.meta.url);
const addon = require('./build/Release/swe_napi.node');

export const G = 9.80665;                       // src/swe.mjs:85
const FIELD = { b: 0, h: 1, hu: 2, hv: 3, h0: 4, hu0: 5, hv0: 6, rh: 7, rhu: 8, rhv: 9, theta: 10 };
const GEOM = ['dxRow', 'dyRowN', 'dyRowS', 'dyCFL', 'area', 'lx', 'lyN', 'lyS', 'bedPhi', 'phiC',
  'tanPhi', 'fRow', 'geoCoef'];
const SIDE = { west: 0, east: 1, south: 2, north: 3 };
const LIMITER = { mc: 0, minmod: 1, central: 2 };
const SCALAR = { dx: 0, dy: 1, R: 2, dlam: 3, dphi: 4, totalArea: 5 };

// Built-in boundaries: identity tokens.  Calling one per cell is not how the
// device applies them, so they refuse, as the Python mirror's do.
const builtin = (name, kind) => {
  const fn = () => { throw new Error(`${name}() is applied on the device by sim.applyBC()`); };
  fn.kind = kind;
  fn.boundaryName = name;
  return fn;
};
export const reflect = builtin('reflect', 0);
export const outflow = builtin('outflow', 1);
export const periodic = builtin('periodic', 2);

// flather(etaExt, uExt) (src/swe.mjs:1085-1115): the two signals ride on
// the returned function so the class can evaluate them at sim.t.
export function flather(etaExt, uExt = () => 0) {
  const fn = () => { throw new Error('flather() is applied on the device by sim.applyBC()'); };
  fn.kind = 3;
  fn.etaExt = etaExt;
  fn.uExt = uExt;
  return fn;
}

// makeSponge(sim, {side, width, strength, etaRef}) (src/swe.mjs:1174-1198):
// a forcing the device runs inside step(); a time-varying etaRef is not
// supported on the device and is refused.
export function makeSponge(sim, { side = 'east', width = 20, strength = 0.06, etaRef = 0 } = {}) {
  if (typeof etaRef === 'function') throw new Error('makeSponge: a time-varying etaRef is not supported on the device');
  const fn = () => {};
  fn.sponge = { side: side in SIDE ? side : 'south', width, strength, etaRef };
  return fn;
}

// hllc(out, hL, huL, hvL, hR, huR, hvR, dry) (src/swe.mjs:975): on the device.
export function hllc(out, hL, huL, hvL, hR, huR, hvR, dry = 1e-4) {
  const r = addon.hllc(hL, huL, hvL, hR, huR, hvR, dry);
  out[0] = r[0]; out[1] = r[1]; out[2] = r[2];
  return out;
}

export class ShallowWater {
  constructor({ nx, ny, dx, dy = dx, bed = () => 0, eta0 = 0, manning = 0.025, minDepth = 1e-3, cfl = 0.45,
    coriolis = 0, order = 2, limiter = 'mc', sphere = null } = {}) {
    const lim = LIMITER[limiter];
    if (lim === undefined) throw new Error(`ShallowWater: unknown limiter "${limiter}"`);
    const opts = { nx, ny, dx, dy, manning, minDepth, cfl, coriolis, order, limiter: lim, sphere: sphere ? 1 : 0 };
    if (sphere) Object.assign(opts, { R: sphere.R ?? 6371e3, lat0: sphere.lat0 ?? -90, lat1: sphere.lat1 ?? 90,
      omega: sphere.omega ?? 0 });
    const W = nx + 4, H = ny + 4;
    // Sample bed and eta0 at every padded cell centre, ghosts included
    // (src/swe.mjs:222-232); a sphere samples at (lon, lat).  The metric
    // comes from a probe with flat state, which has the same geometry.
    const zeros = new Float64Array(W * H);
    const probe = new addon.Native(opts, zeros, zeros);
    const phiC = probe.geom(9);
    const dlam = probe.scalar(SCALAR.dlam);
    const at = (i, j) => (sphere
      ? [((((i + 0.5) * dlam * 180 / Math.PI) % 360) + 360) % 360 - 180, phiC[j + 2] * 180 / Math.PI]
      : [(i + 0.5) * dx, (j + 0.5) * dy]);
    const b = new Float64Array(W * H), h = new Float64Array(W * H);
    for (let j = -2; j < ny + 2; j++) {
      for (let i = -2; i < nx + 2; i++) {
        const k = (j + 2) * W + (i + 2);
        const [x, y] = at(i, j);
        b[k] = bed(x, y);
        const e = typeof eta0 === 'function' ? eta0(x, y) : eta0;
        h[k] = Math.max(0, e - b[k]);
      }
    }
    this._n = new addon.Native(opts, b, h);
    Object.assign(this, { nx, ny, ng: 2, W, H, manning, minDepth, cfl, coriolis, order, limiterName: limiter });
    this.dx = sphere ? NaN : dx;
    this.dy = sphere ? this._n.scalar(SCALAR.dy) : dy;
    this.geom = this._geometry(!!sphere);
    this.manningField = null;
    this.forcing = null;
    this.boundaries = sphere
      ? { west: periodic, east: periodic, south: reflect, north: reflect }
      : { west: reflect, east: reflect, south: reflect, north: reflect };
  }

  _geometry(sphere) {
    const n = this._n;
    const g = { kind: sphere ? 'sphere' : 'cartesian', nx: this.nx, ny: this.ny, ng: 2, H: this.H };
    for (const [name, id] of Object.entries(SCALAR)) g[name] = n.scalar(id);
    GEOM.forEach((name, row) => {
      Object.defineProperty(g, name, { get: () => n.geom(row), enumerable: true });
    });
    return g;
  }

  // ---- fields (src/swe.mjs:200-220) ---------------------------------------
  get b() { return this._n.field(FIELD.b); }
  get h() { return this._n.field(FIELD.h); }
  get hu() { return this._n.field(FIELD.hu); }
  get hv() { return this._n.field(FIELD.hv); }
  get h0() { return this._n.field(FIELD.h0); }
  get hu0() { return this._n.field(FIELD.hu0); }
  get hv0() { return this._n.field(FIELD.hv0); }
  get rh() { return this._n.field(FIELD.rh); }
  get rhu() { return this._n.field(FIELD.rhu); }
  get rhv() { return this._n.field(FIELD.rhv); }
  get theta() { return this._n.field(FIELD.theta); }

  get t() { return this._n.t(); }
  set t(v) { this._n.setT(v); }
  get steps() { return this._n.steps(); }
  set steps(v) { this._n.setSteps(v); }
  get massFloored() { return this._n.massFloored(); }

  idx(i, j) { return (j + 2) * this.W + (i + 2); }
  eta(i, j) { const k = this.idx(i, j); return this.b[k] + this.h[k]; }
  depth(i, j) { return this.h[this.idx(i, j)]; }
  cellCentre(i, j) {
    if (this.geom.kind !== 'cartesian') throw new Error('cellCentre() on a sphere: use cellLonLat()');
    return [(i + 0.5) * this.dx, (j + 0.5) * this.dy];
  }
  cellLonLat(i, j) {
    if (this.geom.kind !== 'sphere') throw new Error('cellLonLat() needs a sphere geometry');
    const lon = (i + 0.5) * this.geom.dlam * 180 / Math.PI;
    return [((lon % 360) + 360) % 360 - 180, this.geom.phiC[j + 2] * 180 / Math.PI];
  }
  vel(hq, h) { return this._n.vel(hq, h); }

  // ---- boundaries and forcing ---------------------------------------------
  _bc() {
    for (const [side, s] of Object.entries(SIDE)) {
      const fn = this.boundaries[side];
      if (fn && fn.kind === 3) {
        const t = this.t;
        this._n.setFlatherValues(s, fn.etaExt(t), fn.uExt(t));
      } else if (fn && fn.kind !== undefined) {
        this._n.setBoundary(s, fn.kind);
      } else {
        throw new Error(`boundaries.${side}: reflect, outflow, periodic or flather(...) of swe-gpu.mjs`);
      }
    }
    const f = this.forcing;
    if (f && f.sponge) this._n.setSponge(SIDE[f.sponge.side], f.sponge.width, f.sponge.strength, f.sponge.etaRef);
    else this._n.clearSponge();
  }

  // ---- the solver (src/swe.mjs:289-814) -------------------------------------
  applyBC() { this._bc(); this._n.applyBC(); }
  residual(dt) { this._n.residual(dt); }
  maxDt() { return this._n.maxDt(); }
  applyFriction(dt) { this._n.applyFriction(dt); }
  dryClean() { return this._n.dryClean(); }
  setManningField(fn) {
    if (fn == null) { this._n.setManningField(null); this.manningField = null; return this; }
    const n = new Float64Array(this.W * this.H);
    for (let j = -2; j < this.ny + 2; j++) {
      for (let i = -2; i < this.nx + 2; i++) {
        const [x, y] = this.geom.kind === 'sphere' ? this.cellLonLat(i, j) : this.cellCentre(i, j);
        const v = typeof fn === 'function' ? fn(x, y) : fn[this.idx(i, j)];
        if (!(v >= 0) || !Number.isFinite(v)) {
          throw new Error(`setManningField: n = ${v} at (${x}, ${y}); Manning n must be finite and >= 0`);
        }
        n[this.idx(i, j)] = v;
      }
    }
    this._n.setManningField(n);
    this.manningField = n;
    return this;
  }
  step(dt) {
    this._bc();
    const t0 = this.t;
    const taken = dt === undefined ? this._n.stepAuto() : this._n.step(dt);
    const f = this.forcing;
    if (taken && f && !f.sponge) {              // user code, on the current fields
      const t1 = this.t;
      this._n.setT(t0);
      try { f(this, taken); } finally { this._n.setT(t1); }
    }
    return taken;
  }
  // The drivers' loop kept on the device when nothing needs the host each
  // step (no Flather signal, no host forcing); otherwise step by step.
  run(n, { dt = 0, tEnd = Infinity } = {}) {
    const hostEachStep = Object.values(this.boundaries).some((fn) => fn.kind === 3) ||
      (this.forcing && !this.forcing.sponge);
    if (!hostEachStep) { this._bc(); return this._n.run(n, dt, tEnd); }
    let done = 0;
    for (; done < n; done++) {
      const d = Math.min(dt > 0 ? dt : this.maxDt(), tEnd - this.t);
      if (!this.step(d)) break;
    }
    return done;
  }

  // ---- diagnostics (src/swe.mjs:819-917) ------------------------------------
  volume() { return this._n.volume(); }
  energy() { return this._n.energy(); }
  maxSurfaceDeviation(ref) { return this._n.maxSurfaceDeviation(ref); }
  maxSpeed() { return this._n.maxSpeed(); }
  finite() { return this._n.finite(); }
}
