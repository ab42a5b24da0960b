"""Index construction (medoid, Vamana build, PQ training and encode, exact kNN)
runs from libdgbuild.so: a process that only prepares an index maps that
library and never the search library, and its graph equals the one the
oracle builds."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
sys.path.insert(0, {root!r})
import numpy as np
import pydiskann_b200 as dg
from pydiskann_b200 import synth
X = synth.mixture(2000, 128, 16, seed=9)
Q = synth.mixture(20, 128, 16, seed=9, stream=synth.STREAM_QUERY)
adj, med = dg.build_graph(X, 32, 64, 1.2, seed=3)
cb = dg.pq_train(X, 16, 256, 3, 2000, seed=1)
codes = dg.pq_encode(X, cb)
gt, _ = dg.exact_knn(X, Q, 10)
np.save({out!r}, adj)
maps = open("/proc/self/maps").read()
print(json.dumps({{"med": int(med), "libdgann": "libdgann.so" in maps, "libdgbuild": "libdgbuild.so" in maps}}))
"""


def test_construction_maps_only_the_builder_library(tmp_path, oracle):
    import numpy as np

    from pydiskann_b200 import synth

    out = str(tmp_path / "adj.npy")
    r = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT, out=out)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    info = json.loads(r.stdout.strip().splitlines()[-1])
    assert info["libdgbuild"] and not info["libdgann"]
    X = synth.mixture(2000, 128, 16, seed=9)
    oadj, _ = oracle.build_vamana(X, 32, 64, 1.2, seed=3, medoid_id=info["med"])
    assert np.array_equal(np.load(out), oadj)
