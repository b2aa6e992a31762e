"""Harmonic tide for Flather boundaries (src/tide.mjs:33-114 of the reference).

Tide.eta(t) = msl + sum_k amp_k cos(omega_k t - phase_k pi/180), with the
terms sorted by amplitude as the reference's constructor sorts them.
`Tide.signal()` returns a callable that a Flather boundary evaluates on the
GPU each step (so `ShallowWater.run` keeps the whole loop on the device);
calling it on the host gives the same sum.
"""
import math

import numpy as np

# Constituent periods in hours (src/tide.mjs:17-27).
CONSTITUENTS = {
    "M2": {"period": 12.4206012, "name": "principal lunar semidiurnal"},
    "S2": {"period": 12.0, "name": "principal solar semidiurnal"},
    "N2": {"period": 12.65834751, "name": "larger lunar elliptic semidiurnal"},
    "K2": {"period": 11.96723606, "name": "lunisolar semidiurnal"},
    "K1": {"period": 23.93447213, "name": "lunisolar diurnal"},
    "O1": {"period": 25.81933871, "name": "principal lunar diurnal"},
    "P1": {"period": 24.06588766, "name": "principal solar diurnal"},
    "Q1": {"period": 26.868350, "name": "larger lunar elliptic diurnal"},
    "Mf": {"period": 327.8599387, "name": "lunar fortnightly"},
}

ATLANTIC_MESO = {"M2": [1.35, 0], "S2": [0.45, 42], "N2": [0.28, -18], "K2": [0.12, 40],
                 "K1": [0.09, 190], "O1": [0.07, 175], "P1": [0.03, 188]}
DIURNAL_COAST = {"K1": [0.55, 20], "O1": [0.38, 5], "P1": [0.18, 18], "M2": [0.16, 250], "S2": [0.05, 280]}


class Tide:
    def __init__(self, constituents=None, msl=0.0, periods_hours=None):
        """constituents: {name: [amp m, phase deg]}; names from CONSTITUENTS,
        or any name whose period (hours) is given in periods_hours."""
        constituents = ATLANTIC_MESO if constituents is None else constituents
        self.msl = float(msl)
        self.terms = []
        for name, (amp, phase) in constituents.items():
            if periods_hours and name in periods_hours:
                period = periods_hours[name]
            elif name in CONSTITUENTS:
                period = CONSTITUENTS[name]["period"]
            else:
                raise ValueError(f"Tide: unknown constituent {name}")
            self.terms.append({"name": name, "amp": float(amp), "phase": float(phase),
                               "omega": 2 * math.pi / (period * 3600), "period": period * 3600})
        self.terms.sort(key=lambda k: -k["amp"])   # stable, as Array.prototype.sort

    def eta(self, t):
        e = self.msl
        for k in self.terms:
            e += k["amp"] * math.cos(k["omega"] * t - k["phase"] * math.pi / 180)
        return e

    def rate(self, t):
        d = 0.0
        for k in self.terms:
            d -= k["amp"] * k["omega"] * math.sin(k["omega"] * t - k["phase"] * math.pi / 180)
        return d

    @staticmethod
    def resonantPeriod(length, depth, g=9.80665):
        return 4 * length / math.sqrt(g * depth)

    def signal(self):
        return TideSignal(self)


class TideSignal:
    """eta(t) of a Tide, evaluable on the device by a Flather boundary."""

    def __init__(self, tide, coef=None):
        self.tide, self.coef = tide, coef

    def __call__(self, t):
        e = self.tide.eta(t)
        return e if self.coef is None else self.coef * e

    def scaled(self, coef):
        """u(t) = coef * eta(t), e.g. sqrt(G/h) * tide.eta(t) (tools/verify-tide.mjs:1137-1140)."""
        return TideSignal(self.tide, float(coef))

    def device_table(self):
        tr = self.tide.terms
        return (self.tide.msl, np.array([k["amp"] for k in tr], dtype=np.float64),
                np.array([k["omega"] for k in tr], dtype=np.float64),
                np.array([k["phase"] for k in tr], dtype=np.float64))
