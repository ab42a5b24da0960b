"""bench.py --impl reference on CPU: the arm times the oracle's search of the
headline variant (BF16 traversal + FP32 rerank) on the cached workload, prints
the config object the GPU arm prints for the same beam, and its process maps no
library of this repository other than the oracle."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
sys.argv = ["bench.py", "--impl", "reference", "--n", "3000", "--nq", "200", "--steps", "2", "--warmup", "1"]
sys.path.insert(0, {root!r})
import bench
bench.main()
maps = open("/proc/self/maps").read()
print(json.dumps({{"libdgann": "libdgann.so" in maps, "libdgbuild": "libdgbuild.so" in maps,
                  "oracle": "libdgoracle.so" in maps}}))
"""


def _fill_cache(cache):
    """The workload cache of a 3000-vector case, built by the oracle (so no GPU
    is needed): graph, medoid, PQ codebooks and codes, exact ground truth."""
    sys.path.insert(0, ROOT)
    import bench
    import oracle
    from pydiskann_b200 import synth

    class A:
        n, nq, seed = 3000, 200, 0

    d, files = bench._cache_files(A)
    X, Q = synth.pq_config(A.n, A.nq, 128, A.seed)
    med = oracle.medoid(X)
    adj, _ = oracle.build_vamana(X, bench.R, bench.L_BUILD, bench.ALPHA, seed=A.seed, medoid_id=med)
    cb = np.ascontiguousarray(X[:256].reshape(256, bench.M, 128 // bench.M).transpose(1, 0, 2))
    codes = oracle.pq_encode(X, cb)
    gt, _ = oracle.exact_knn(X, Q, bench.K)
    os.makedirs(d, exist_ok=True)
    for k, v in (("adj", adj), ("meta", np.array([med])), ("cb", cb), ("codes", codes), ("gt", gt)):
        np.save(files[k], v)
    return bench, A, X, Q, adj, med, gt


def test_reference_arm_line_and_libraries(tmp_path):
    cache = str(tmp_path / "cache")
    os.environ["DGANN_BENCH_CACHE"] = cache
    try:
        import importlib

        sys.path.insert(0, ROOT)
        import bench

        importlib.reload(bench)
        bench, A, X, Q, adj, med, gt = _fill_cache(cache)
        env = dict(os.environ, DGANN_BENCH_CACHE=cache)
        env.pop("RANK", None)
        r = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT)], env=env, capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-3000:]
        lines = [json.loads(x) for x in r.stdout.strip().splitlines()]
        line, maps = lines[0], lines[1]
        assert maps == {"libdgann": False, "libdgbuild": False, "oracle": True}
        assert line["impl"] == "reference" and line["metric"] == bench.METRIC
        L = line["config"]["L"]
        assert line["config"] == bench.config_of(A, 1, L)
        assert line["config"]["variant"] == "bf16_rerank"
        assert line["recall_at_10"] >= 0.95 or L == bench.L_SWEEP[-1]
        # the beam is the smallest of the sweep reaching the target on the whole batch
        curve = line["recall_curve"]
        assert curve[-1][0] == L and all(rc < 0.95 for _, rc in curve[:-1])
        assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
    finally:
        os.environ.pop("DGANN_BENCH_CACHE", None)
        importlib.reload(bench)
