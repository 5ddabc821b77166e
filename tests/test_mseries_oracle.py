"""The CPU restatement of the benchmark driver's random-number generator
(RandomNumbers_parallel<RandomNumbers_Mseries>, oracle/mseries.py) against the
reference corelib's own draws (tests/golden/mseries_parallel.npz): the
uniform stream and the Gaussian fields bit for bit, across calls and after a
reset."""
import json
import os

import numpy as np

from oracle.mseries import MseriesParallel

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mseries_parallel.npz")


def test_oracle_matches_reference_stream():
    g = np.load(GOLD)
    meta = json.loads(str(g["meta"]))
    lat, ls, seed = meta["lattice"], meta["Ls"], meta["seed"]
    r = MseriesParallel(lat, seed)
    assert np.array_equal(r.uniform_lex_global(2, 1), g["u"])
    assert np.array_equal(r.gauss_lex_global(8, 4), g["h"])
    assert np.array_equal(r.gauss_lex_global(24, ls), g["x"])
    r.reset(seed + 1)
    assert np.array_equal(r.gauss_lex_global(8, 4), g["h2"])


def test_reference_draw_statistics():
    """Gaussians of variance 1/2 and uniforms on [0, 1): a check on the
    fixture itself, independent of the restatement."""
    g = np.load(GOLD)
    x = np.concatenate([g["h"], g["x"], g["h2"]])
    assert abs(x.mean()) < 0.02 and abs(x.var() - 0.5) < 0.02
    u = g["u"][0::2]
    assert u.min() >= 0.0 and u.max() < 1.0 and abs(u.mean() - 0.5) < 0.05
    assert np.all(g["u"][1::2] == 0.0)
