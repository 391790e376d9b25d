"""The small CPU configuration, frozen from the reference program
(tests/golden/c1_plane200.npz, made by tests/golden/make_golden.py): 200 x
200 cells of 2 m, a plane sloping 0.01 with smoothed Gaussian bumps (seed 0),
dry start, 20 mm/day of melt at 1 mg/L for 6 h, D = 0.01 m^2/s, ROUGNESS_HEIGHT
(the dry threshold) 0.001 m, output every 600 s: 36 Results files, the
reference's whole loop (main.cpp:271-470)."""
import hashlib
import json
import os

import numpy as np

from fluxos_cpp_b200 import scenarios as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c1_plane200.npz")


def load():
    z = np.load(GOLDEN)
    return z, json.loads(str(z["meta"]))


def write_inputs(folder: str):
    """Regenerate the case's input files; return (scenario, modset path)
    after checking they are the bytes the reference read."""
    z, meta = load()
    sc = S.plane_scenario()
    mp = sc.write(folder)
    for fn, sha in meta["inputs"].items():
        with open(os.path.join(folder, fn), "rb") as f:
            assert hashlib.sha256(f.read()).hexdigest() == sha, f"{fn} differs from the reference's input"
    return sc, mp


def digest_of(z, meta, fn):
    t = fn.split(".")[0]
    d = dict(meta["digest"][fn])
    d.update(mask=z[f"mask_{t}"], sums=z[f"sums_{t}"], samples=z[f"samples_{t}"])
    return d
