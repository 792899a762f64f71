"""Writes tests/golden/grown_colony_1e6_profile.json: the radial density, volume
and growth-rate histograms of the configured 3D colony grown on the device
from 10^4 agents to 10^6 (needs a CUDA device and the built library).

    python tests/golden/make_grown_colony_profile.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import conftest  # noqa: E402  (loads the package)
from scenarios import growing_colony_3d  # noqa: E402


def main():
    cbm = conftest.cbm
    abi = cbm._abi
    kw, st = growing_colony_3d(abi, 1_000_000, precision=abi.F32)
    g = cbm.Context(abi.make_config(**kw))
    g.upload(st)
    steps = 0
    while g.counters()["N"] < 1_000_000:
        g.step(10)
        steps += 10
    s = g.download()
    p = np.stack([s["x"], s["y"], s["z"]], 1).astype(np.float64) - 200.0
    r = np.linalg.norm(p, axis=1)
    r_edges = np.arange(0, np.ceil(r.max()) + 1.0, 1.0)
    v_edges = np.linspace(1.0, 2.0, 21)
    g_edges = np.linspace(0.8, 1.2, 21)
    out = {"what": "histograms of the 3D growing colony grown on the device from 10^4 agents (seed 2, "
                   "Float32) until N >= 10^6: radius from the box centre (200,200,200) in unit shells, "
                   "volume v in 20 bins on [1,2], growth rate g in 20 bins on [0.8,1.2]; made by "
                   "tests/golden/make_grown_colony_profile.py",
           "N": int(s["N"]), "grow_steps": steps,
           "r_edges": r_edges.tolist(), "r_counts": np.histogram(r, r_edges)[0].tolist(),
           "v_edges": v_edges.tolist(),
           "v_counts": np.histogram(np.clip(s["v"], 1.0, 2.0 - 1e-9), v_edges)[0].tolist(),
           "g_edges": g_edges.tolist(),
           "g_counts": np.histogram(np.clip(s["g"], 0.8, 1.2 - 1e-9), g_edges)[0].tolist()}
    with open(os.path.join(HERE, "grown_colony_1e6_profile.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
