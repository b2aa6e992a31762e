"""B200-native shallow-water step (Syntaxswine/water-simulator's hot path).

The public API mirrors the reference's JavaScript modules:
  ShallowWater, G, hllc, reflect, outflow, periodic, flather, makeSponge  (src/swe.mjs)
  cartesianGeometry, sphericalGeometry, interiorArea, cellLonLat,
  R_EARTH, OMEGA_EARTH                                                    (src/geometry.mjs)
  Tide, CONSTITUENTS                                                      (src/tide.mjs)
  gridlandsTerrain, loadGridlandsTerrain, verifyInvariants, settleLakes,
  waterbodies                                                             (src/gridlands.mjs)
  renderMap, globeCamera, buildGlobeLut, renderGlobe, colourTables        (src/render.mjs, src/globe.mjs)
All solver arithmetic runs in libswe_b200.so (CUDA, sm_100a, FP64).
"""
from .swe import (G, R_EARTH, OMEGA_EARTH, ShallowWater, Flather, Sponge, hllc, hllc_batch,
                  reflect, outflow, periodic, flather, makeSponge, cartesianGeometry,
                  sphericalGeometry, interiorArea, cellLonLat, Geometry)
from .tide import Tide, TideSignal, CONSTITUENTS, ATLANTIC_MESO, DIURNAL_COAST
from ._lib import SweError, load as load_library, LIB_PATH
from .batch import Ensemble
from .adjoint import MisfitAdjoint
from .gridlands import gridlandsTerrain, loadGridlandsTerrain, verifyInvariants, settleLakes, waterbodies
from .render import renderMap, globeCamera, buildGlobeLut, renderGlobe, colourTables

__all__ = ["G", "R_EARTH", "OMEGA_EARTH", "ShallowWater", "Flather", "Sponge", "hllc", "hllc_batch",
           "reflect", "outflow", "periodic", "flather", "makeSponge", "cartesianGeometry",
           "sphericalGeometry", "interiorArea", "cellLonLat", "Geometry", "Tide", "TideSignal",
           "CONSTITUENTS", "ATLANTIC_MESO", "DIURNAL_COAST", "SweError", "load_library", "LIB_PATH",
           "Ensemble", "MisfitAdjoint", "gridlandsTerrain", "loadGridlandsTerrain", "verifyInvariants",
           "settleLakes", "waterbodies", "renderMap", "globeCamera", "buildGlobeLut", "renderGlobe",
           "colourTables"]
