"""Extract the reference's own recorded numbers for the step into
tests/golden/reference_pins.json (run where the reference tree is present).

Sources, all inside Syntaxswine/water-simulator:
  tools/sphere-baseline.json     resting-ocean, area-identity and Merian rows
                                 recorded by `node tools/verify-sphere.mjs --bless`
  README.md (lake-at-rest table) max |eta - 2| and max speed for four beds,
                                 200x4 cells, 400 steps
  tools/verify-physics.mjs       the positivity factor the solver returns in the
                                 one-wet-cell rig ("the solver returns 0.6666...")
  README.md (claims table)       closed-basin mass drift over 600 steps
Usage: python tests/golden/make_golden.py /path/to/the/reference/tree
"""
import json
import os
import re
import sys

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_pins.json")


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py /path/to/the/reference/tree")
    REF = sys.argv[1]
    with open(os.path.join(REF, "tools", "sphere-baseline.json")) as f:
        base = json.load(f)
    with open(os.path.join(REF, "README.md")) as f:
        readme = f.read()
    with open(os.path.join(REF, "tools", "verify-physics.mjs")) as f:
        physics = f.read()

    lake = {}
    for m in re.finditer(r"lake at rest, ([a-z ()]+?)\s{2,}(\S+)( m)?\s+(\S+) m/s", readme):
        name = m.group(1).strip()
        lake[name] = {"max_eta_dev": float(m.group(2)), "max_speed": float(m.group(4))}
    theta = re.search(r"the solver returns (0\.\d+)", physics).group(1)
    mass = re.search(r"mass conservation, closed basin, 600 steps \| (\S+) relative", readme).group(1)

    pins = {
        "source": "Syntaxswine/water-simulator: tools/sphere-baseline.json, README.md, "
                  "tools/verify-physics.mjs",
        "sphere_baseline": {"recorded": base["recorded"], "node": base["node"],
                            "constants": base["constants"],
                            "restingOcean": base["restingOcean"],
                            "areaIdentity": base["areaIdentity"], "merian": base["merian"]},
        "lake_at_rest_200x4_400steps": lake,
        "positivity_theta_one_wet_cell": theta,
        "closed_basin_mass_drift_600_steps": float(mass),
    }
    with open(OUT, "w") as f:
        json.dump(pins, f, indent=1)
    print(f"wrote {OUT}: {len(lake)} lake rows, theta {theta}, mass {mass}, "
          f"{len(base['restingOcean'])}/{len(base['areaIdentity'])}/{len(base['merian'])} sphere rows")


if __name__ == "__main__":
    main()
