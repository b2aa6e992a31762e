"""The gridlands import (src/gridlands.mjs): document checks that throw
before anything is decoded (no GPU), and waterbodies / verifyInvariants /
settleLakes on a synthetic export, whose bodies are labelled by the
device's connected-components pass (GPU) and checked against a flood-fill
oracle and the export's known lakes."""
import numpy as np
import pytest

from gridlands_doc import make_doc, terrain_arrays
from gridlands_oracle import flood_bodies


def test_document_checks(swe):
    from water_simulator_b200 import gridlands as gl
    doc = make_doc()
    with pytest.raises(ValueError, match="not a document"):
        gl.gridlandsTerrain(None)
    with pytest.raises(ValueError, match="unsupported terrain something-else v1"):
        gl.gridlandsTerrain(dict(doc, format="something-else"))
    with pytest.raises(ValueError, match="unsupported terrain gridlands-terrain v2"):
        gl.gridlandsTerrain(dict(doc, version=2))
    with pytest.raises(ValueError, match="bad grid"):
        gl.gridlandsTerrain(dict(doc, grid=dict(doc["grid"], width=0)))
    with pytest.raises(ValueError, match="rowOrder is south-first"):
        gl.gridlandsTerrain(dict(doc, grid=dict(doc["grid"], rowOrder="south-first")))


def test_layer_checks_before_decoding(swe):
    from water_simulator_b200 import gridlands as gl
    with pytest.raises(ValueError, match="layer bedM is missing"):
        gl.decodeF32(None, 4, "bedM")
    with pytest.raises(ValueError, match="encoding b64f16le, expected b64f32le"):
        gl.decodeF32({"encoding": "b64f16le", "data": ""}, 4, "bedM")


def _same_bodies(got, want):
    assert len(got) == len(want)
    for g, w in zip(got, want):
        assert g["level"] == w["level"] and g["spread"] == w["spread"]
        assert g["ringMin"] == w["ringMin"] and g["perch"] == w["perch"] and g["isOcean"] == w["isOcean"]
        assert list(g["cells"]) == w["cells"]


@pytest.mark.gpu
def test_device_bodies_match_the_flood_fill(swe):
    """Random wet/dry maps with many bodies of every shape (spirals of one
    cell, bodies touching the edges, one body over the whole grid)."""
    from water_simulator_b200 import gridlands as gl
    rng = np.random.default_rng(4)
    for W, H, p in ((64, 48, 0.55), (200, 150, 0.6), (1, 37, 0.5), (41, 1, 0.5), (9, 7, 1.0), (128, 96, 0.45)):
        bed = rng.uniform(-5, 5, (H, W)).astype(np.float32)
        srf = np.where(rng.uniform(0, 1, (H, W)) < p, bed + rng.uniform(0.01, 2, (H, W)), bed).astype(np.float32)
        _same_bodies(gl.waterbodies(bed, srf, W, H), flood_bodies(bed, srf, W, H))
    # a one-cell-wide spiral: the longest chain a union-find can meet
    W = H = 61
    wet = np.zeros((H, W), bool)
    r0, c0, r1, c1 = 0, 0, H - 1, W - 1
    while r0 <= r1 and c0 <= c1:
        wet[r0, c0:c1 + 1] = True
        wet[r0:r1 + 1, c1] = True
        wet[r1, c0:c1 + 1] = True
        if c0 + 2 <= c1:
            wet[r0 + 2:r1 + 1, c0] = True
        r0, c0, r1, c1 = r0 + 2, c0 + 2, r1 - 2, c1 - 2
    bed = np.zeros((H, W), np.float32)
    srf = np.where(wet, 1.0, 0.0).astype(np.float32)
    _same_bodies(gl.waterbodies(bed, srf, W, H), flood_bodies(bed, srf, W, H))
    assert gl.waterbodies(np.zeros((3, 3), np.float32), np.zeros((3, 3), np.float32), 3, 3) == []


@pytest.mark.gpu
def test_waterbodies_and_invariants(swe):
    from water_simulator_b200 import gridlands as gl
    W, H = 64, 48
    b, s, _ = terrain_arrays(W, H)
    b, s = b.reshape(-1), s.reshape(-1)
    bodies = gl.waterbodies(b, s, W, H)
    assert len(bodies) == 3
    lakes = sorted([x for x in bodies if not x["isOcean"]], key=lambda x: x["level"])
    ocean = [x for x in bodies if x["isOcean"]]
    assert [x["level"] for x in lakes] == [32.0, 38.5]
    assert lakes[0]["ringMin"] == 30.0 and lakes[0]["perch"] == 2.0     # perched 2 m above its spill
    assert lakes[1]["perch"] < 0                                          # seated below its rim
    assert all(x["spread"] == 0 for x in bodies)
    assert ocean[0]["perch"] <= 1e-6
    # every wet cell belongs to exactly one body
    wet = set(np.nonzero(s.astype(np.float64) - b > 0)[0].tolist())
    cells = [k for x in bodies for k in x["cells"]]
    assert len(cells) == len(set(cells)) and set(cells) == wet

    class T:
        pass
    t = T()
    t.bedM, t.surfaceM, t.W, t.H = b, s, W, H
    inv = gl.verifyInvariants(t)
    assert inv["surfaceBelowBed"] == 0 and inv["lakesNotFlat"] == 0
    assert inv["lakeBodies"] == 2 and inv["perchedLakes"] == 1 and inv["worstPerch"] == 2.0
    assert inv["perchedCells"] == len(lakes[0]["cells"])
    assert inv["perchedVolumeCells"] == len(lakes[0]["cells"]) * 2.0
    assert inv["wet"] == len(wet) and inv["cells"] == W * H


@pytest.mark.gpu
def test_settle_lowers_only_the_perched_lake(swe):
    from water_simulator_b200 import gridlands as gl
    W, H = 64, 48
    b, s, _ = terrain_arrays(W, H)
    b, s = b.reshape(-1), s.reshape(-1)
    before = s.copy()
    lakes = [x for x in gl.waterbodies(b, s, W, H) if not x["isOcean"]]
    perched = [x for x in lakes if x["perch"] > 1e-6][0]
    rep = gl.settleLakes(b, s, W, H)
    assert rep["bodiesMoved"] == 1 and rep["worstDrop"] == 2.0
    changed = np.nonzero(s != before)[0]
    assert set(changed.tolist()) <= set(perched["cells"])
    for k in perched["cells"]:
        assert s[k] == max(float(b[k]), 30.0)
    assert s.dtype == np.float32
    # after settling nothing is perched
    assert all(x["perch"] <= 1e-6 for x in gl.waterbodies(b, s, W, H) if not x["isOcean"])
