#!/usr/bin/env python
"""QPS at recall@10 >= 0.95 on the 1M x 128 workload, plain FP32 vs BF16 + FP32
rerank, on one B200 (or N replicas).

Workload: 1M x 128 FP32 base vectors from a 256-centre clipped Gaussian mixture
(seeded synthetic data with the configuration's shapes and value distribution),
10k queries per batch, Vamana graph R=64, L_build=128, alpha=1.2, PQ M=16 x
K=256 trained with 25 Lloyd iterations on a 100k sample, k=10.  A step is one
batched search of the 10k queries.  Each variant is timed at the smallest beam
L whose recall@10 against the exact FP64 ground truth reaches 0.95:
  bf16_rerank-- BF16 rows during the search, FP32 rerank of the top L: the
                headline `value`
  fp32       -- plain FP32 beam search (DiskANN::search), reported beside it
  int8_rerank-- int8 SQ codes (global scale/offset, src/sq.rs) + FP32 rerank
  fp8_rerank -- e4m3 rows with per-vector scales + FP32 rerank
  pq_rerank  -- PQ ADC + FP32 rerank of the top L
The graph, codebooks and ground truth are inputs of the search: `--prepare`
builds them once into a cache, in a process of its own that loads only the
index-construction library (libdgbuild.so), and both arms read that cache.

`--impl reference` times the CPU restatement of the reference search (the
oracle, all host threads) on the same graph, queries and variant: BF16 rows
during the traversal and an FP32 rerank of the top L, at the beam the oracle's
own recall sweep picks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

CACHE = os.environ.get("DGANN_BENCH_CACHE", os.path.join(tempfile.gettempdir(), "dgann_bench_cache"))
R, L_BUILD, ALPHA, M, K_PQ, PQ_ITERS, PQ_SAMPLE, K = 64, 128, 1.2, 16, 256, 25, 100_000, 10
L_SWEEP = (16, 24, 32, 40, 48, 56, 64, 80, 96, 128, 160, 192, 256, 384, 512, 768, 1024)
COSINE_SWEEP = (256, 384, 512, 768, 1024)  # fixed beams of the cosine recall-target sweep
METRIC = "QPS @ recall@10=0.95, plain FP32 vs BF16+FP32-rerank, 1 B200; p99 ms"
HEADLINE = "bf16_rerank"
PARITY_QUERIES = 1000  # queries of the batch compared with the oracle for every timed variant


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--prepare", action="store_true",
                    help="only build the cached graph, codebooks and ground truth (index-construction library)")
    ap.add_argument("--device", type=int, default=0, help="device of --prepare")
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--nq", type=int, default=10_000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--target-recall", type=float, default=0.95)
    ap.add_argument("--beam", type=int, default=0,
                    help="time this beam instead of sweeping for the target recall (profiling runs)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="time the default launch schedule (profiling runs: fewer launches before the timed ones)")
    ap.add_argument("--variants", default="bf16_rerank,fp32,fp8_rerank,int8_rerank,pq_rerank")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serve-rates", default="100000,1000000,3000000,0",
                    help="Poisson arrival rates (req/s) for the serving loop; 0 = all requests at once")
    ap.add_argument("--serve-requests", type=int, default=200_000)
    ap.add_argument("--no-filtered", action="store_true")
    ap.add_argument("--no-spfresh", action="store_true")
    ap.add_argument("--spfresh-n", type=int, default=2_000_000)
    ap.add_argument("--spfresh-batches", type=int, default=3,
                    help="update batches (1%% inserts, 0.5%% deletes, then searches at n_probe 64) after the load")
    ap.add_argument("--filtered-queries", type=int, default=5000)
    ap.add_argument("--cosine", action="store_true",
                    help="also run the quantized cosine workload (1M x 768, 20k queries, uneven beams)")
    ap.add_argument("--cosine-n", type=int, default=1_000_000)
    ap.add_argument("--filtered-serving", action="store_true",
                    help="run the filtered serving workload (1M x 256, labels, R=48, Poisson 5k-200k req/s) on its "
                         "whole grid (k in {10, 100} x L in {64, 200} x 5 rates); by default a short grid runs")
    ap.add_argument("--no-filtered-serving", action="store_true")
    ap.add_argument("--fs-n", type=int, default=1_000_000)
    ap.add_argument("--cosine-nq", type=int, default=20_000)
    return ap.parse_args()


# ------------------------------------------------------------------ setup
def _cache_files(args):
    key = f"pq_n{args.n}_q{args.nq}_R{R}_L{L_BUILD}_a{ALPHA}_M{M}_s{args.seed}"
    d = os.path.join(CACHE, key)
    return d, {k: os.path.join(d, k + ".npy") for k in ("adj", "meta", "cb", "codes", "gt")}


def prepare(args):
    """Builds the cached inputs of the search (graph, medoid, PQ codebooks and
    codes, FP64 ground truth) with the index-construction library only."""
    from pydiskann_b200 import synth

    import pydiskann_b200 as dg

    d, files = _cache_files(args)
    if all(os.path.exists(f) for f in files.values()):
        return {"cached": True}
    X, Q = synth.pq_config(args.n, args.nq, 128, args.seed)
    dev = args.device
    times = {}
    t0 = time.time()
    med = dg.medoid(X, device=dev)
    times["medoid_s"] = round(time.time() - t0, 2)
    t0 = time.time()
    adj, _ = dg.build_graph(X, R, L_BUILD, ALPHA, seed=args.seed, medoid_id=med, device=dev)
    times["graph_build_s"] = round(time.time() - t0, 2)
    t0 = time.time()
    cb = dg.pq_train(X, M, K_PQ, PQ_ITERS, PQ_SAMPLE, seed=args.seed, device=dev)
    times["pq_train_s"] = round(time.time() - t0, 2)
    codes = dg.pq_encode(X, cb, device=dev)
    t0 = time.time()
    gt, _ = dg.exact_knn(X, Q, K, device=dev)
    times["ground_truth_s"] = round(time.time() - t0, 2)
    os.makedirs(d, exist_ok=True)
    for k, v in (("adj", adj), ("meta", np.array([med])), ("cb", cb), ("codes", codes), ("gt", gt)):
        tmp = files[k] + f".tmp{os.getpid()}.npy"
        np.save(tmp, v)
        os.replace(tmp, files[k])
    with open(os.path.join(d, "setup.json"), "w") as f:
        json.dump(times, f)
    return times


def _run_prepare(args, device):
    """`bench.py --prepare` in a child process (it loads libdgbuild.so only)."""
    cmd = [sys.executable, os.path.abspath(__file__), "--prepare", "--device", str(device), "--n", str(args.n),
           "--nq", str(args.nq), "--seed", str(args.seed)]
    t0 = time.time()
    subprocess.run(cmd, check=True)
    log(f"[setup] prepared the cached graph, codebooks and ground truth in {time.time() - t0:.1f}s")


def workload(args, device=0, build=True):
    """Data (regenerated from the seed) and the cached graph, codebooks and
    ground truth; builds the cache first (in a child process) when missing."""
    from pydiskann_b200 import synth

    d, files = _cache_files(args)
    if not all(os.path.exists(f) for f in files.values()):
        if not build:
            return None
        _run_prepare(args, device)
    t0 = time.time()
    X, Q = synth.pq_config(args.n, args.nq, 128, args.seed)
    log(f"[setup] data {X.shape} + {Q.shape} in {time.time() - t0:.1f}s")
    adj = np.load(files["adj"])
    med = int(np.load(files["meta"])[0])
    cb = np.load(files["cb"])
    codes = np.load(files["codes"])
    gt = np.load(files["gt"])
    setup = {"cache": d}
    try:
        setup.update(json.load(open(os.path.join(d, "setup.json"))))
    except (OSError, ValueError):
        pass
    return X, Q, adj, med, (cb, codes), gt, setup


def recall(ids, gt, k=K):
    ids = np.asarray(ids)[:, :k]
    hits = sum(len(set(ids[i].tolist()) & set(gt[i, :k].tolist())) for i in range(len(gt)))
    return hits / (len(gt) * k)


def config_of(args, world, L, variant=HEADLINE):
    """The `config` object both arms print (same workload, variant and beam)."""
    return {"workload": f"pq-1Mx128 M={M} R={R} L_build={L_BUILD} alpha={ALPHA} k={K} nq={args.nq} n={args.n}",
            "variant": variant, "L": L, "global_batch": args.nq * world, "parallelism": f"replicas{world}",
            "l2_policy": "inputs larger than L2 (512 MB f32 + 256 MB bf16 rows + 256 MB adjacency)"}


# ------------------------------------------------------------ clock probe
def _nvml_index(cuda_index):
    """NVML's ordinal of a CUDA device (they differ under CUDA_VISIBLE_DEVICES)."""
    try:
        import torch

        return int(torch.cuda._get_nvml_device_index(cuda_index))
    except Exception:
        return cuda_index


class Clocks:
    """Samples SM clocks and throttle reasons while the timed region runs.

    nvidia-smi polls every 200 ms from 0.3 s before the region; a thread polls
    NVML (read-only queries) about every half millisecond from the moment the
    context is entered until it exits, so a timed region of a few milliseconds
    still has samples taken under load.  Without NVML the nvidia-smi samples
    are reported."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clocks-event reason bits (nvmlClocksThrottleReason*)
    REASON_BITS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
                   ("sw_power_cap", 0x4))

    def __init__(self, gpu_index, nvml=None):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.fast = []  # (SM MHz, reason bits) from NVML inside the region
        self.fast_max = None
        self._nvml = nvml  # a stand-in module for tests; pynvml otherwise
        self._go = threading.Event()
        self._stop = threading.Event()
        self._thr = None

    def _poll(self):
        try:
            nv = self._nvml
            if nv is None:
                import pynvml as nv
            nv.nvmlInit()
        except Exception:
            return
        try:
            h = nv.nvmlDeviceGetHandleByIndex(_nvml_index(self.gpu) if self._nvml is None else self.gpu)
            reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            self.fast_max = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            if not self._go.wait(timeout=10.0):
                return
            while not self._stop.is_set():
                self.fast.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), int(reasons(h))))
                time.sleep(0.0005)
        except Exception:
            pass
        finally:
            try:
                nv.nvmlShutdown()
            except Exception:
                pass

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        try:
            self._thr = threading.Thread(target=self._poll, daemon=True)
            self._thr.start()
        except Exception:
            self._thr = None
        time.sleep(0.3)
        self._go.set()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._go.set()
        if self._thr is not None:
            self._thr.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        try:
            for line in open(self.path):
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    mx.append(float(p[2]))
                except ValueError:
                    continue
                for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), p[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(name)
        except OSError:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.remove(self.path)
        fast = list(self.fast)
        if fast:
            for name, bit in self.REASON_BITS:
                if any(r & bit for _, r in fast):
                    reasons.add(name)
            top = max(mx) if mx else self.fast_max
            return {"sm_mhz": float(np.median([c for c, _ in fast])), "sm_max_mhz": top, "reasons": sorted(reasons),
                    "samples": len(fast), "source": "nvml, inside the timed region"}
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi"}


# ------------------------------------------------------------ GPU timing
# DRAM bytes of one launch of the dominant kernel (dram__bytes_read.sum +
# dram__bytes_write.sum) from one ncu capture of this bench's command on a
# smaller batch, keyed by (variant, L, base vectors): (queries captured,
# bytes).  The line scales it to the batch by queries.
NCU_TRAFFIC = {("bf16_rerank", 40, 1_000_000): (2000, 623.473408e6 + 5.54752e6)}
NCU_TRAFFIC_SOURCE = ("scaled by queries from one ncu --set full capture of a 2000-query launch of the same "
                      "kernel (python bench.py --nq 2000 --beam 40 --no-autotune --variants bf16_rerank ...)")

VARIANTS = {
    # name: (traversal, rerank = L?)
    "fp32": ("f32", False),
    "bf16_rerank": ("bf16", True),
    "int8_rerank": ("int8", True),
    "fp8_rerank": ("fp8", True),
    "pq_rerank": ("codes", True),
}


def max_over_ranks(ms, dist, device):
    """The slowest rank's time (every rank calls this at the same step)."""
    if dist is None:
        return ms
    import torch

    tt = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def run_variant(idx, qidx, name, Qd, L, out=None, with_stats=False, stream=None, rerank=True):
    """idx: the FP32/BF16 index; qidx: {"pq": QuantizedDiskANN, "int8": ...}.
    rerank=False returns the traversal's own distances (no FP32 rerank)."""
    from pydiskann_b200 import _lib

    trav, rr = VARIANTS[name]
    t = {"f32": _lib.TRAVERSE_F32, "bf16": _lib.TRAVERSE_BF16, "codes": _lib.TRAVERSE_CODES,
         "int8": _lib.TRAVERSE_CODES, "fp8": _lib.TRAVERSE_FP8}[trav]
    target = qidx["pq"] if trav == "codes" else qidx["int8"] if trav == "int8" else idx
    return target.search_arrays(Qd, K, L, traversal=t, rerank_size=L if rr and rerank else 0, out=out,
                                with_stats=with_stats, stream=stream)


def autotune_variant(idx, qidx, name, Qd, L):
    """dg_index_autotune on the variant's own search (same queries, k, L)."""
    from pydiskann_b200 import _lib

    trav, rr = VARIANTS[name]
    t = {"f32": _lib.TRAVERSE_F32, "bf16": _lib.TRAVERSE_BF16, "codes": _lib.TRAVERSE_CODES,
         "int8": _lib.TRAVERSE_CODES, "fp8": _lib.TRAVERSE_FP8}[trav]
    target = qidx["pq"] if trav == "codes" else qidx["int8"] if trav == "int8" else idx
    return target.autotune(Qd, K, L, traversal=t, rerank_size=L if rr else 0, reps=3)


def distance_error(X, Q, ids, ds):
    """Relative error of returned distances against FP64 squared L2 of the same
    (query, id) pairs: {"max", "mean"} over every returned neighbour."""
    ids = np.asarray(ids)
    ds = np.asarray(ds, dtype=np.float64)
    ok = ids != 0xFFFFFFFF
    errs = []
    for q0 in range(0, len(Q), 1000):
        sl = slice(q0, q0 + 1000)
        I = np.where(ok[sl], ids[sl], 0).astype(np.int64)
        diff = X[I].astype(np.float64) - Q[sl, None, :].astype(np.float64)
        exact = (diff * diff).sum(-1)
        e = np.abs(ds[sl] - exact) / np.maximum(exact, 1e-30)
        errs.append(e[ok[sl]])
    e = np.concatenate(errs) if errs else np.zeros(0)
    return {"max": float(e.max()) if e.size else 0.0, "mean": float(e.mean()) if e.size else 0.0}


def algorithmic_bytes(name, nq, L, E, N, d=128):
    """Bytes the algorithm must read per launch of nq queries: adjacency rows,
    distance operands, rerank rows, queries and results (per query E*4R +
    N*bytes per evaluation + L*4d + 4d + 8k).  E (expansions) and N (distance
    evaluations) are per-query means of an exact visited set (the oracle's
    counts); the kernel's own N also counts ids its small visited table forgot
    and evaluated again."""
    adj = E * 4 * R
    if name == "fp32":
        dist, rr = N * 4 * d, 0.0
    elif name == "bf16_rerank":
        dist, rr = N * 2 * d, L * 4 * d
    elif name == "int8_rerank":
        dist, rr = N * d, L * 4 * d
    elif name == "fp8_rerank":
        dist, rr = N * (d + 8), L * 4 * d  # e4m3 row + (scale, norm)
    else:
        dist, rr = N * M, L * 4 * d
    return nq * (adj + dist + rr + 4 * d + 8 * K)


def _oracle_variant(X, adj, med, pq, name, native=False):
    """The oracle index of a variant (test infrastructure, run only as the checker
    of the parity leg and, built for the host's own CPU, as the CPU baseline)."""
    import oracle

    o = oracle.OracleIndex(X, adj, med, native=native)
    if name == "pq_rerank":
        o.set_pq(*pq)
    elif name == "int8_rerank":
        from pydiskann_b200 import int8_params

        sc, off = int8_params(X)
        o.set_int8(sc, off, oracle.int8_encode(X, sc, off))
    elif name == "bf16_rerank":
        o.set_bf16()
    elif name == "fp8_rerank":
        o.set_fp8(*oracle.fp8_encode(X))
    return o


def _oracle_run(o, name, Qs, L, threads, with_stats=False):
    if name == "fp32":
        return o.search(Qs, K, L, threads=threads, with_stats=with_stats)
    return o.search(Qs, K, L, rerank=L, use_codes=True, threads=threads, with_stats=with_stats)


def parity_leg(X, Q, adj, med, pq, name, L, got, threads):
    """Compares the GPU's results for the first PARITY_QUERIES queries of the
    batch with the oracle's search of the same variant and beam: positions
    whose id or distance differ, and queries whose result count differs.  Also
    returns the oracle's per-query expansions and distance evaluations (an
    exact visited set)."""
    nq = min(PARITY_QUERIES, len(Q))
    o = _oracle_variant(X, adj, med, pq, name)
    oi, od, oc, st = _oracle_run(o, name, Q[:nq], L, threads, with_stats=True)
    gi, gd, gc = (np.asarray(a)[:nq] for a in got)
    return ({"queries": nq, "id_mismatch": int((gi != oi).sum()), "dist_mismatch": int((gd != od).sum()),
             "count_mismatch": int((gc != oc).sum())},
            {"expansions": float(st[:, 0].mean()), "dist_evals": float(st[:, 1].mean())})


def main():
    args = parse()
    if args.prepare:
        log(f"[prepare] {json.dumps(prepare(args))}")
        return 0
    if args.impl == "reference":
        return reference_arm(args)
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import pydiskann_b200 as dg

    # rank 0 fills the cache, the others read it (no data-path collective)
    wl = None
    if rank == 0:
        wl = workload(args, local)
    if dist is not None:
        dist.barrier()
    if wl is None:
        wl = workload(args, local)
    X, Q, adj, med, (cb, codes), gt, setup_times = wl
    t0 = time.time()
    wanted = args.variants.split(",")
    idx, qidx = None, {}
    if "fp32" in wanted or "bf16_rerank" in wanted or "fp8_rerank" in wanted:
        idx = dg.DiskANN.from_graph(X, adj, med, device=local)
        if "bf16_rerank" in wanted:
            idx.enable_bf16()
        if "fp8_rerank" in wanted:
            idx.enable_fp8()
    if "pq_rerank" in wanted:
        qidx["pq"] = dg.QuantizedDiskANN(X, adj, med, device=local)
        qidx["pq"].attach_pq(cb, codes)
    if "int8_rerank" in wanted:
        qidx["int8"] = dg.QuantizedDiskANN(X, adj, med, device=local)
        qidx["int8"].attach_int8(*dg.int8_params(X))
    log(f"[setup] index upload + encodes {time.time() - t0:.1f}s")
    Qd = torch.from_numpy(Q).to(dev)
    stream = torch.cuda.current_stream(dev)

    # ---- recall sweep: smallest L reaching the target for each variant
    chosen, curves = {}, {}
    for name in wanted:
        curves[name] = []
        for L in ((args.beam,) if args.beam else L_SWEEP):
            ids, _, _ = run_variant(idx, qidx, name, Qd, L)
            torch.cuda.synchronize()
            rec = recall(ids.cpu().numpy().view(np.uint32), gt)
            curves[name].append((L, round(rec, 4)))
            if rec >= args.target_recall or args.beam:
                chosen[name] = (L, rec)
                break
        log(f"[sweep] {name}: {chosen.get(name)} curve {curves[name]}")

    # ---- timing per variant (device-resident queries and results), after the
    # autotuner picked the visited-table size for this exact search
    results, outs = {}, {}
    tuned = {}
    for name, (L, rec) in chosen.items():
        tuned[name] = ({"hbits": 10 if L <= 64 else 11 if L <= 128 else 12, "order": 0, "occ_pct": 100,
                        "warps_per_cta": 4, "default": True}
                       if args.no_autotune else autotune_variant(idx, qidx, name, Qd, L))
        log(f"[autotune] {name}: {tuned[name]}")
        out = run_variant(idx, qidx, name, Qd, L)
        for _ in range(args.warmup):
            run_variant(idx, qidx, name, Qd, L, out=out)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        with Clocks(local) as ck:
            torch.cuda.synchronize()
            t_start = torch.cuda.Event(enable_timing=True)
            t_end = torch.cuda.Event(enable_timing=True)
            t_start.record(stream)
            for s in range(args.steps):
                ev[s][0].record(stream)
                run_variant(idx, qidx, name, Qd, L, out=out)
                ev[s][1].record(stream)
            t_end.record(stream)
            torch.cuda.synchronize()
        total_ms = t_start.elapsed_time(t_end)
        steps_ms = np.array([a.elapsed_time(b) for a, b in ev])
        total_ms = max_over_ranks(total_ms, dist, dev)
        outs[name] = tuple(t.cpu().numpy() for t in out)
        outs[name] = (outs[name][0].view(np.uint32), outs[name][1], outs[name][2].view(np.uint32))
        _, _, _, st = run_variant(idx, qidx, name, Qd, L, with_stats=True)
        stats = st.cpu().numpy().view(np.uint32)
        # accuracy against the FP64 oracle: returned distances, the traversal's
        # own distances (rerank off) and the recall shortfall
        ti, td, _ = run_variant(idx, qidx, name, Qd, L, rerank=False)
        acc = {"dist_rel_err": distance_error(X, Q, outs[name][0], outs[name][1]),
               "traversal_dist_rel_err": distance_error(X, Q, ti.cpu().numpy().view(np.uint32), td.cpu().numpy()),
               "recall_delta_vs_fp64": round(1.0 - rec, 4)}
        results[name] = {
            "L": L, "recall_at_10": round(rec, 4), "qps": world * args.nq * args.steps / (total_ms / 1e3),
            "ms_per_step": total_ms / args.steps, "p50_ms": float(np.percentile(steps_ms, 50)),
            "p99_ms": float(np.percentile(steps_ms, 99)), "launch_ms": float(steps_ms.mean()),
            "kernel_expansions_per_query": float(stats[:, 0].mean()),
            "kernel_dist_evals_per_query": float(stats[:, 1].mean()),
            **acc, "visited_table_bits": tuned[name]["hbits"],
            "schedule": {k: v for k, v in tuned[name].items() if k != "ms"}, "clocks": ck.summary(),
        }
        log(f"[time] {name}: {json.dumps(results[name])}")

    # ---- parity with the oracle on the first queries of the batch (rank 0),
    # and the oracle's exact-visited work counts for the algorithmic bytes
    parity = {}
    if rank == 0:
        threads = os.cpu_count() or 1
        for name, r in results.items():
            parity[name], work = parity_leg(X, Q, adj, med, (cb, codes), name, r["L"], outs[name], threads)
            r["expansions_per_query"] = work["expansions"]
            r["dist_evals_per_query"] = work["dist_evals"]
            r["alg_bytes_per_launch"] = algorithmic_bytes(name, args.nq, r["L"], work["expansions"],
                                                          work["dist_evals"])
            log(f"[parity] {name}: {parity[name]} {work}")

    head = HEADLINE if HEADLINE in results else (max(results, key=lambda n: results[n]["qps"]) if results else None)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    extra = {n: {"qps": r["qps"], "L": r["L"], "recall_at_10": r["recall_at_10"]} for n, r in results.items()
             if n not in (HEADLINE, "fp32")}
    for n in extra:
        if n in ("int8_rerank",):
            extra[n]["note"] = "int8 codes are lossless on this integer-valued 0-255 data (scale 1, offset 0)"
    line = {
        "metric": METRIC,
        "value": results[head]["qps"] if head else None,
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": results[head]["ms_per_step"] if head else None,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"fp32": "f32", "bf16_rerank": "bf16+f32", "int8_rerank": "u8+f32",
                  "fp8_rerank": "e4m3+f32"}.get(head, "u8-pq+f32"),
        "data": "synthetic (seeded 256-centre Gaussian mixture, 1M x 128, 10k queries)",
        "config": config_of(args, world, results[head]["L"] if head else None, head or HEADLINE),
        "fp32_qps": results["fp32"]["qps"] if "fp32" in results else None,
        "bf16_rerank_over_fp32": (round(results[HEADLINE]["qps"] / results["fp32"]["qps"], 3)
                                  if HEADLINE in results and "fp32" in results else None),
        "extra_variants": extra,
        "parity_vs_oracle": parity,
        "variants": results,
        "recall_curves": curves,
        "p99_ms": results[head]["p99_ms"] if head else None,
        "setup": setup_times,
    }
    if head:
        r = results[head]
        if "alg_bytes_per_launch" in r:
            ach = r["alg_bytes_per_launch"] / (r["launch_ms"] / 1e3) / 1e9
            cap = NCU_TRAFFIC.get((head, r["L"], args.n))
            tr = cap[1] * args.nq / cap[0] if cap else None
            line["roofline"] = {"bound": "hbm", "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
                                "frac": round(ach / hbm, 4), "traffic": tr,
                                "traffic_source": NCU_TRAFFIC_SOURCE if tr else None,
                                "peak_source": ("measured: MEASURED_PEAKS.json hbm_gbs (burst)" if peaks
                                                else "fallback 6650 GB/s"),
                                "kernel": f"beam_search_kernel {head} L={r['L']}",
                                "alg_bytes_per_launch": r["alg_bytes_per_launch"]}
        line["clocks"] = r["clocks"]
        line["gpu_launches"] = args.steps
        line["e2e"] = e2e(args, idx, qidx, head, r["L"], Q, gt, dist, world, dev)
        if not args.no_serving:
            line["serving"] = {n: serving(args, idx, qidx, n, results[n]["L"], Q, gt)
                               for n in dict.fromkeys([head, "fp32"]) if n in results}
            # headline p99: the highest Poisson load (the saturation run measures queue drain)
            loaded = [x for x in line["serving"][head]["rates"] if x["offered_rps"]]
            if loaded:
                line["p99_ms"] = loaded[-1]["p99_ms"]
                line["p99_load_rps"] = loaded[-1]["offered_rps"]
        if not args.no_filtered:
            line["filtered"] = filtered(args, X, Q, adj, med, dev, dist)
        if args.cosine and rank == 0:
            line["quantized_cosine"] = quantized_cosine(args, dev)
        if not args.no_filtered_serving and rank == 0:
            try:
                line["filtered_serving"] = filtered_serving(args, dev, full=args.filtered_serving)
            except Exception as e:  # a secondary workload: keep the headline line
                line["filtered_serving"] = {"error": repr(e)[:400]}
                log(f"[filtered serving] failed: {e!r}")
        if not args.no_spfresh and rank == 0:
            # one replica is enough for this secondary measurement (it stages
            # several GB of posting blocks on the host)
            line["spfresh"] = spfresh_scan(args, dev, None)
    if rank == 0 and head and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, X, Q, adj, med, (cb, codes), head, results[head]["L"])
    if rank == 0:
        print(json.dumps(line), flush=True)
    if idx is not None:
        idx.close()
    for q in qidx.values():
        q.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def e2e(args, idx, qidx, name, L, Q, gt, dist, world, dev):
    """The same search through the public API with host buffers: the queries
    are copied from pinned host memory and the results read back every step."""
    import torch

    Qh = torch.from_numpy(Q).pin_memory()
    Qn = Qh.numpy()
    outs = (torch.empty((args.nq, K), dtype=torch.int32).pin_memory().numpy().view(np.uint32),
            torch.empty((args.nq, K), dtype=torch.float32).pin_memory().numpy(),
            torch.empty((args.nq,), dtype=torch.int32).pin_memory().numpy().view(np.uint32))
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        run_variant(idx, qidx, name, Qn, L, out=outs, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(args.steps):
        run_variant(idx, qidx, name, Qn, L, out=outs, stream=stream.cuda_stream)
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    ms = max_over_ranks(ms, dist, dev)
    rec = recall(outs[0], gt)
    return {"value": world * args.nq * args.steps / (ms / 1e3), "unit": "queries/s",
            "h2d_bytes_per_step": int(Q.nbytes), "d2h_bytes_per_step": int(args.nq * (K * 8 + 4)),
            "recall_at_10": round(rec, 4)}


def filtered(args, X, Q, adj, med, dev, dist):
    """Label-filtered search on the same graph (the reference has no
    filter-aware build): every vector carries 1-3 of 100 labels drawn Zipf(1.0);
    query i asks Or(Eq(0, l), Eq(1, l), Eq(2, l)) for a uniform label l, so the
    selectivity spans ~0.5 % to ~35 %.  Ground truth: exact kNN inside each
    label's subset.  For FP32 and int8 + FP32 rerank: the smallest L reaching
    recall@10 >= the target, and the device-timed QPS at it."""
    import torch

    import pydiskann_b200 as dg
    from pydiskann_b200 import _lib, synth

    t0 = time.time()
    labels = synth.label_sets(len(X), seed=args.seed)
    nqf = min(args.filtered_queries, len(Q))
    Qf = Q[:nqf]
    ql = np.random.default_rng(args.seed + 7).integers(1, 101, nqf)
    flist = [dg.Filter.or_([dg.Filter.eq(0, int(l)), dg.Filter.eq(1, int(l)), dg.Filter.eq(2, int(l))]) for l in ql]
    filt = dg.pack_filters(flist)
    gt = np.zeros((nqf, K), dtype=np.int64)
    sel = np.zeros(nqf)
    for l in np.unique(ql):
        sub = np.nonzero((labels == np.uint64(l)).any(1))[0]
        qi = np.nonzero(ql == l)[0]
        ids, _ = dg.exact_knn(X[sub], Qf[qi], K, device=dev.index)
        gt[qi] = sub[ids.astype(np.int64)]
        sel[qi] = len(sub) / len(X)
    setup_s = time.time() - t0
    f32 = dg.FilteredDiskANN(X, adj, med, labels, device=dev.index)
    f32.enable_bf16()
    q8 = dg.QuantizedDiskANN(X, adj, med, device=dev.index)
    q8.attach_int8(*dg.int8_params(X))
    q8.attach_labels(labels)
    Qd = torch.from_numpy(Qf).to(dev)
    stream = torch.cuda.current_stream(dev)
    out = {"queries": nqf, "labels": "1-3 of 100 per vector, Zipf(1.0)", "selectivity_min": float(sel.min()),
           "selectivity_max": float(sel.max()), "setup_s": round(setup_s, 1), "variants": {}}
    variants = (("fp32", f32, {"traversal": _lib.TRAVERSE_F32}),
                ("bf16_rerank", f32, {"traversal": _lib.TRAVERSE_BF16}),
                ("int8_rerank", q8, {"traversal": _lib.TRAVERSE_CODES}))
    for name, ix, kw in variants:
        chosen = None
        curve = []
        for L in L_SWEEP:
            rr = L if name != "fp32" else 0
            ids, _, _ = ix.search_arrays(Qd, K, L, rerank_size=rr, filters=filt, **kw)
            torch.cuda.synchronize()
            rec = recall(ids.cpu().numpy().view(np.uint32), gt)
            curve.append((L, round(rec, 4)))
            if rec >= args.target_recall:
                chosen = (L, rec)
                break
        if chosen is None:
            out["variants"][name] = {"recall_curve": curve}
            continue
        L, rec = chosen
        rr = L if name != "fp32" else 0
        tune = ix.autotune(Qd, K, L, rerank_size=rr, filters=filt, reps=2, **kw)
        log(f"[filtered] autotune {name}: {tune}")
        res = ix.search_arrays(Qd, K, L, rerank_size=rr, filters=filt, **kw)
        for _ in range(args.warmup):
            ix.search_arrays(Qd, K, L, rerank_size=rr, filters=filt, out=res, **kw)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            ix.search_arrays(Qd, K, L, rerank_size=rr, filters=filt, out=res, **kw)
        b.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(a.elapsed_time(b), dist, dev)
        _, _, _, st = ix.search_arrays(Qd, K, L, rerank_size=rr, filters=filt, with_stats=True, **kw)
        stats = st.cpu().numpy().view(np.uint32)
        out["variants"][name] = {"L": L, "recall_at_10": round(rec, 4), "qps": nqf * args.steps / (ms / 1e3),
                                 "ms_per_step": ms / args.steps, "recall_curve": curve,
                                 "expansions_per_query": float(stats[:, 0].mean()),
                                 "dist_evals_per_query": float(stats[:, 1].mean()),
                                 "visited_table_bits": tune["hbits"]}
        log(f"[filtered] {name}: {json.dumps(out['variants'][name])}")
    # filtered serving: Poisson arrivals, each request with its own label filter
    n_srv, rate = 50_000, 200_000.0
    qi = np.arange(n_srv) % nqf
    out["serving"] = {"requests": n_srv, "offered_rps": rate, "variants": {}}
    for name, ix, kw in variants:
        v = out["variants"].get(name, {})
        if "L" not in v or name == "int8_rerank":
            continue
        L = v["L"]
        with dg.Server(ix, max_batch=512, streams=16, max_k=K) as srv:
            srv.run_trace(Qf[:2000], np.zeros(2000), k=K, beam_width=L, rerank_size=L if name != "fp32" else 0,
                          traversal=kw["traversal"], filters=flist[:2000])
            res = srv.run_trace(Qf[qi], dg.poisson_arrivals(n_srv, rate, seed=5), k=K, beam_width=L,
                                rerank_size=L if name != "fp32" else 0, traversal=kw["traversal"],
                                filters=[flist[i] for i in qi])
        lat = res["latency_us"] / 1e3
        hits = [len(set(res["ids"][i].tolist()) & set(gt[qi[i]].tolist())) for i in range(0, n_srv, 5)]
        out["serving"]["variants"][name] = {
            "L": L, "achieved_qps": n_srv / (res["wall_us"] / 1e6), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "recall_at_10": round(float(np.mean(hits)) / K, 4)}
        log(f"[filtered serve] {name}: {json.dumps(out['serving']['variants'][name])}")
    f32.close()
    q8.close()
    return out


def filtered_serving(args, dev, full=True):
    """The filtered serving workload: 1M x 256 Gaussian mixture (512 centres),
    each vector with 1-3 of 100 labels drawn Zipf(1.0); a Vamana graph with
    R = 48 (the reference has no filter-aware build); queries ask Or(Eq(0, l),
    Eq(1, l), Eq(2, l)) for a uniform label l (selectivity ~0.5 % to ~35 %).
    Requests with their own filters arrive as Poisson streams at 5k-200k req/s
    through the serving loop, for k in {10, 100} and L in {64, 200} (full) or
    for (k, L) = (10, 64) and (100, 200) at 5k, 50k and 200k req/s (short), FP32
    and BF16 + FP32 rerank; p50 / p99 latency, achieved QPS and recall@10
    against exact kNN inside each label's subset."""
    import pydiskann_b200 as dg
    from pydiskann_b200 import _lib, synth

    t0 = time.time()
    nq = 5000
    X, Q, labels = synth.filtered(args.fs_n, nq, 256, args.seed)
    adj, med = dg.build_graph(X, 48, 128, 1.2, seed=args.seed, device=dev.index or 0)
    setup = {"data_and_graph_s": round(time.time() - t0, 1)}
    ql = np.random.default_rng(args.seed + 11).integers(1, 101, nq)
    flist = [dg.Filter.or_([dg.Filter.eq(0, int(l)), dg.Filter.eq(1, int(l)), dg.Filter.eq(2, int(l))]) for l in ql]
    t0 = time.time()
    gt = np.zeros((nq, K), dtype=np.int64)
    for l in np.unique(ql):
        sub = np.nonzero((labels == np.uint64(l)).any(1))[0]
        qi = np.nonzero(ql == l)[0]
        ids, _ = dg.exact_knn(X[sub], Q[qi], K, device=dev.index or 0)
        gt[qi] = sub[ids.astype(np.int64)]
    setup["ground_truth_s"] = round(time.time() - t0, 1)
    log(f"[filtered serving] setup {setup}")
    ix = dg.FilteredDiskANN(X, adj, med, labels, device=dev.index or 0)
    ix.enable_bf16()
    out = {"n": len(X), "dim": 256, "R": 48, "queries": nq, "setup": setup, "grid": "full" if full else "short",
           "runs": []}
    rates = (5_000, 20_000, 50_000, 100_000, 200_000) if full else (5_000, 50_000, 200_000)
    kls = [(k, L) for k in (10, 100) for L in (64, 200)] if full else [(10, 64), (100, 200)]
    for name, trav in (("fp32", _lib.TRAVERSE_F32), ("bf16_rerank", _lib.TRAVERSE_BF16)):
        for k, L in kls:
            rr = L if name != "fp32" else 0
            tune = ix.autotune(Q[:2000], k, L, traversal=trav, rerank_size=rr, filters=flist[:2000], reps=1)
            with dg.Server(ix, max_batch=512, streams=16, max_k=100) as srv:
                srv.run_trace(Q[:1000], np.zeros(1000), k=k, beam_width=L, rerank_size=rr, traversal=trav,
                              filters=flist[:1000])
                for rate in rates:
                    n = int(max(2000, rate * 1.0))
                    qi = np.arange(n) % nq
                    res = srv.run_trace(Q[qi], dg.poisson_arrivals(n, rate, seed=rate), k=k, beam_width=L,
                                        rerank_size=rr, traversal=trav, filters=[flist[i] for i in qi])
                    lat = res["latency_us"] / 1e3
                    hits = [len(set(res["ids"][i][:K].tolist()) & set(gt[qi[i]].tolist()))
                            for i in range(0, n, max(1, n // 2000))]
                    r = {"variant": name, "k": k, "L": L, "offered_rps": rate,
                         "achieved_qps": round(n / (res["wall_us"] / 1e6)), "p50_ms": round(float(np.percentile(lat, 50)), 3),
                         "p99_ms": round(float(np.percentile(lat, 99)), 3),
                         "recall_at_10": round(float(np.mean(hits)) / K, 4), "visited_table_bits": tune["hbits"],
                         "schedule": {a: b for a, b in tune.items() if a != "ms"}}
                    out["runs"].append(r)
                    log(f"[filtered serving] {json.dumps(r)}")
    ix.close()
    return out


def cosine_distance_error(X, Q, ids, ds):
    """Relative error of returned cosine distances against FP64 1 - cos of the
    same (query, id) pairs."""
    ids = np.asarray(ids)
    ok = ids != 0xFFFFFFFF
    errs = []
    qn = np.linalg.norm(Q.astype(np.float64), axis=1)
    for q0 in range(0, len(Q), 1000):
        sl = slice(q0, q0 + 1000)
        I = np.where(ok[sl], ids[sl], 0).astype(np.int64)
        V = X[I].astype(np.float64)
        dot = np.einsum("qkd,qd->qk", V, Q[sl].astype(np.float64))
        exact = 1.0 - dot / (np.linalg.norm(V, axis=2) * qn[sl, None])
        e = np.abs(np.asarray(ds[sl], np.float64) - exact) / np.maximum(np.abs(exact), 1e-12)
        errs.append(e[ok[sl]])
    e = np.concatenate(errs)
    return {"max": float(e.max()), "mean": float(e.mean())}


def quantized_cosine(args, dev):
    """The quantized cosine workload: 1M x 768 embeddings with an anisotropic
    power-law spectrum (exponent -0.5), unit norm, BF16 values; 20k queries
    whose beams are drawn uniformly from {32..256} and run in one launch; k =
    10 and an FP32 rerank of the top 4k = 40 candidates.  Vamana R = 64, L_build
    = 128 (cosine).  FP32 (exact) traversal beside BF16, FP8, int8 (global
    min/max) and RaBitQ codes; recall against FP64 exact kNN and the relative
    error of the returned and of the traversal distances against FP64."""
    import torch

    import pydiskann_b200 as dg
    from pydiskann_b200 import _lib, synth

    t0 = time.time()
    X, Q = synth.cosine(args.cosine_n, args.cosine_nq, 768, args.seed)
    setup = {"data_s": round(time.time() - t0, 1)}
    key = f"cos_n{args.cosine_n}_q{args.cosine_nq}_s{args.seed}"
    d = os.path.join(CACHE, key)
    fa, fm, fg = (os.path.join(d, f + ".npy") for f in ("adj", "meta", "gt"))
    if all(os.path.exists(f) for f in (fa, fm, fg)):
        adj, med, gt = np.load(fa), int(np.load(fm)[0]), np.load(fg)
    else:
        t0 = time.time()
        adj, med = dg.build_graph(X, 64, 128, 1.2, metric="cosine", seed=args.seed, device=dev.index or 0)
        setup["graph_build_s"] = round(time.time() - t0, 1)
        t0 = time.time()
        gt, _ = dg.exact_knn(X, Q, K, metric="cosine", device=dev.index or 0)
        setup["ground_truth_s"] = round(time.time() - t0, 1)
        os.makedirs(d, exist_ok=True)
        for f, v in ((fa, adj), (fm, np.array([med])), (fg, gt)):
            np.save(f, v)
    log(f"[cosine] setup {setup}")
    beams = np.random.default_rng([args.seed, 77]).integers(32, 257, size=len(Q)).astype(np.uint32)
    base = dg.DiskANN.from_graph(X, adj, med, metric="cosine", device=dev.index or 0)
    base.enable_bf16()
    base.enable_fp8()
    q8 = dg.QuantizedDiskANN(X, adj, med, metric="cosine", device=dev.index or 0)
    q8.attach_int8(*dg.int8_params(X))
    rq = dg.QuantizedDiskANN(X, adj, med, metric="cosine", device=dev.index or 0)
    cen, signs = dg.rabitq_params(X, args.seed)
    rq.attach_rabitq(cen, signs)
    Qd = torch.from_numpy(Q).to(dev)
    variants = (("fp32", base, _lib.TRAVERSE_F32, 0), ("bf16_rerank", base, _lib.TRAVERSE_BF16, 4 * K),
                ("fp8_rerank", base, _lib.TRAVERSE_FP8, 4 * K), ("int8_rerank", q8, _lib.TRAVERSE_CODES, 4 * K),
                ("rabitq_rerank", rq, _lib.TRAVERSE_CODES, 4 * K))
    out = {"n": len(X), "dim": 768, "queries": len(Q), "beams": "uniform 32..256 per query",
           "rerank": 4 * K, "setup": setup, "variants": {}}
    stream = torch.cuda.current_stream(dev)
    for name, ix, trav, rr in variants:
        run = lambda rerank=rr, o=None: ix.search_arrays(Qd, K, 256, traversal=trav, rerank_size=rerank,
                                                         per_query_beam=beams, out=o)
        tune = ix.autotune(Qd, K, 256, traversal=trav, rerank_size=rr, per_query_beam=beams, reps=1)
        log(f"[cosine] autotune {name}: {tune}")
        res = run()
        for _ in range(max(args.warmup, 1)):
            run(o=res)
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for a, b in ev:
            a.record(stream)
            run(o=res)
            b.record(stream)
        torch.cuda.synchronize()
        ms = np.array([a.elapsed_time(b) for a, b in ev])
        ids = res[0].cpu().numpy().view(np.uint32)
        rec = recall(ids, gt)
        ti, td, _ = run(rerank=0)
        out["variants"][name] = {
            "recall_at_10": round(rec, 4), "recall_delta_vs_fp64": round(1.0 - rec, 4),
            "qps": len(Q) / (ms.mean() / 1e3), "ms_per_step": float(ms.mean()), "p99_ms": float(np.percentile(ms, 99)),
            "dist_rel_err": cosine_distance_error(X, Q, ids, res[1].cpu().numpy()),
            "traversal_dist_rel_err": cosine_distance_error(X, Q, ti.cpu().numpy().view(np.uint32), td.cpu().numpy()),
            "visited_table_bits": tune["hbits"],
        }
        log(f"[cosine] {name}: {json.dumps(out['variants'][name])}")
    # The per-query beams above (32..256) stop near recall 0.38 on this spectrum;
    # one fixed beam for the whole batch is swept upwards to the smallest that
    # reaches the target recall, then timed there.
    out["at_target"] = {"target_recall": args.target_recall, "variants": {}}
    for name, ix, trav, rr in variants[:4]:
        curve, hit = [], None
        for L in COSINE_SWEEP:
            ids = ix.search_arrays(Qd, K, L, traversal=trav, rerank_size=rr)[0]
            torch.cuda.synchronize()
            rec = recall(ids.cpu().numpy().view(np.uint32), gt)
            curve.append((L, round(rec, 4)))
            if rec >= args.target_recall:
                hit = (L, rec)
                break
        row = {"recall_curve": curve}
        if hit:
            L = hit[0]
            tune = ix.autotune(Qd, K, L, traversal=trav, rerank_size=rr, reps=1)
            res = ix.search_arrays(Qd, K, L, traversal=trav, rerank_size=rr)
            for _ in range(max(args.warmup, 1)):
                ix.search_arrays(Qd, K, L, traversal=trav, rerank_size=rr, out=res)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(args.steps):
                ix.search_arrays(Qd, K, L, traversal=trav, rerank_size=rr, out=res)
            b.record(stream)
            torch.cuda.synchronize()
            ms = a.elapsed_time(b) / args.steps
            row.update({"L": L, "recall_at_10": round(hit[1], 4), "qps": len(Q) / (ms / 1e3), "ms_per_step": ms,
                        "visited_table_bits": tune["hbits"]})
        out["at_target"]["variants"][name] = row
        log(f"[cosine] at target {name}: {json.dumps(row)}")
    for ix in (base, q8, rq):
        ix.close()
    return out


def spfresh_scan(args, dev, dist):
    """SPFresh posting scans: Zipf(1.1)-weighted 1024-centre mixture, 96
    dims, max posting 250 (n / 125 postings), 10k queries, k = 10.  Postings
    are bulk-loaded (exact nearest-centroid assignment + 2-means splits); the
    smallest n_probe reaching the recall target is timed on the device."""
    import torch

    import pydiskann_b200 as dg
    from pydiskann_b200 import synth

    t0 = time.time()
    Xs, Qs = synth.spfresh(args.spfresh_n, 10_000, seed=args.seed)
    gt, _ = dg.exact_knn(Xs, Qs, K, device=dev.index)
    t1 = time.time()
    s = dg.SPFresh.bulk_load(Xs, max_posting_size=250, seed=args.seed, device=dev.index)
    load_s = time.time() - t1
    st = s.stats()
    out = {"n": len(Xs), "dim": Xs.shape[1], "queries": len(Qs), "postings": st["postings"],
           "max_posting": st["max_posting"], "bulk_load_s": round(load_s, 1), "setup_s": round(time.time() - t0, 1)}
    Qd = torch.from_numpy(Qs).to(dev)
    stream = torch.cuda.current_stream(dev)
    curve = []
    for nprobe in (16, 64, 256, 1024):
        ids, _, _ = s.search_arrays(Qd, K, nprobe)
        for _ in range(args.warmup):
            s.search_arrays(Qd, K, nprobe)
        torch.cuda.synchronize()
        rec = recall(ids.cpu().numpy().astype(np.int64), gt.astype(np.int64))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            s.search_arrays(Qd, K, nprobe)
        b.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(a.elapsed_time(b), dist, dev) / args.steps
        curve.append({"nprobe": nprobe, "recall_at_10": round(rec, 4), "qps": len(Qs) / (ms / 1e3), "ms_per_step": ms})
        if rec >= args.target_recall:
            break
    out["curve"] = curve
    out["stream"] = spfresh_stream(args, s, Xs, Qs, Qd, dev)
    log(f"[spfresh] {json.dumps(out)}")
    s.close()
    return out


def spfresh_stream(args, s, Xs, Qs, Qd, dev, nprobe=64):
    """The update stream of the SPFresh workload: each batch inserts 1 % fresh
    vectors of the same mixture and deletes 0.5 % of the live ids (uniformly),
    then searches the query batch at n_probe 64 (device-timed); recall@10 is
    against exact kNN over the live vectors after the batch."""
    import torch

    import pydiskann_b200 as dg
    from pydiskann_b200 import synth

    stream = torch.cuda.current_stream(dev)
    n0 = len(Xs)
    rng = np.random.default_rng([args.seed, 0x5F])
    allX = [Xs]
    rows = []
    for b in range(args.spfresh_batches):
        new = synth.mixture(n0 // 100, Xs.shape[1], 1024, args.seed, stream=synth.STREAM_MISC + 100 + b, clip=False,
                            zipf=1.1)
        t0 = time.time()
        s.insert(new)
        t_ins = time.time() - t0
        allX.append(new)
        live = np.setdiff1d(np.arange(s.next_id, dtype=np.int64), np.fromiter(s.deleted, dtype=np.int64))
        gone = rng.choice(live, size=n0 // 200, replace=False)
        t0 = time.time()
        s.delete(gone.tolist())
        t_del = time.time() - t0
        live = np.setdiff1d(live, gone)
        X = np.concatenate(allX)
        gt, _ = dg.exact_knn(X[live], Qs, K, device=dev.index)
        gt = live[gt.astype(np.int64)]
        ids, _, _ = s.search_arrays(Qd, K, nprobe)
        for _ in range(args.warmup):
            s.search_arrays(Qd, K, nprobe)
        torch.cuda.synchronize()
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            s.search_arrays(Qd, K, nprobe)
        e.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(e) / args.steps
        st = s.stats()
        row = {"batch": b, "inserted": len(new), "deleted": len(gone), "insert_s": round(t_ins, 2),
               "delete_s": round(t_del, 3), "live": st["live"], "postings": st["postings"], "nprobe": nprobe,
               "qps": len(Qs) / (ms / 1e3), "ms_per_step": ms,
               "recall_at_10": round(recall(ids.cpu().numpy().astype(np.int64), gt), 4)}
        rows.append(row)
        log(f"[spfresh stream] {json.dumps(row)}")
    return rows


def serving(args, idx, qidx, name, L, Q, gt):
    """Continuous batching: requests arrive one at a time (Poisson) and are
    admitted into batches as stream slots free up; p50/p99 is measured from
    each request's scheduled arrival to its result in host memory."""
    import pydiskann_b200 as dg
    from pydiskann_b200 import _lib

    trav, rr = VARIANTS[name]
    target = qidx["pq"] if trav == "codes" else qidx["int8"] if trav == "int8" else idx
    t = {"f32": _lib.TRAVERSE_F32, "bf16": _lib.TRAVERSE_BF16, "codes": _lib.TRAVERSE_CODES,
         "int8": _lib.TRAVERSE_CODES, "fp8": _lib.TRAVERSE_FP8}[trav]
    n = args.serve_requests
    qi = np.arange(n) % len(Q)
    Qn = Q[qi]
    out = {"variant": name, "L": L, "max_batch": 512, "streams": 16, "requests": n, "rates": []}
    with dg.Server(target, max_batch=512, streams=16, max_k=K, max_wait_us=0) as srv:
        srv.run_trace(Qn[:5000], np.zeros(5000), k=K, beam_width=L, rerank_size=L if rr else 0, traversal=t)
        for rate in [float(x) for x in args.serve_rates.split(",")]:
            arr = dg.poisson_arrivals(n, rate, seed=3) if rate > 0 else np.zeros(n)
            b0 = srv.stats()["batches"]
            res = srv.run_trace(Qn, arr, k=K, beam_width=L, rerank_size=L if rr else 0, traversal=t)
            lat = res["latency_us"] / 1e3
            ids = np.full((n, K), 0xFFFFFFFF, np.uint32)
            for i, r in enumerate(res["ids"]):
                ids[i, : len(r)] = r
            hit = [len(set(ids[i].tolist()) & set(gt[qi[i]][:K].tolist())) for i in range(0, n, 7)]
            row = {"offered_rps": rate or None, "achieved_qps": n / (res["wall_us"] / 1e6),
                   "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                   "mean_batch": n / max(1, srv.stats()["batches"] - b0),
                   "recall_at_10": round(float(np.mean(hit)) / K, 4)}
            out["rates"].append(row)
            log(f"[serve] {name} L={L}: {json.dumps(row)}")
        out["max_in_flight"] = srv.stats()["max_in_flight"]
    return out


# ------------------------------------------------------------ CPU legs
def cpu_baseline(args, X, Q, adj, med, pq, name, L, threads=None):
    """The oracle's search of the same variant and beam on the host cores, over
    about cpu_seconds of queries (the batch, cycled)."""
    threads = threads or os.cpu_count() or 1
    o = _oracle_variant(X, adj, med, pq, name, native=True)
    t0 = time.time()
    _oracle_run(o, name, Q[:200], L, threads)
    rate = 200 / max(time.time() - t0, 1e-6)
    ns = int(min(20 * len(Q), max(200, rate * args.cpu_seconds)))
    Qs = Q[np.arange(ns) % len(Q)]
    t0 = time.time()
    _oracle_run(o, name, Qs, L, threads)
    dt = time.time() - t0
    return {"value": ns / dt, "unit": "queries/s", "cores": threads, "kind": "port",
            "sample": f"{ns} queries (the {len(Q)} bench queries, cycled), variant {name} at L={L}, "
                      f"same graph and rows", "seconds": round(dt, 2)}


def reference_arm(args):
    """The reference search (CPU restatement, all host threads) of the headline
    variant -- BF16 rows during the traversal, FP32 rerank of the top L -- at
    the smallest beam whose recall@10 over the whole batch reaches the target,
    on the workload of the GPU arm.  A step searches the whole batch.  This
    process loads the oracle library only; a missing workload cache is built
    by `bench.py --prepare` in a child process.  Under torchrun only rank 0
    works."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    world = int(os.environ.get("WORLD_SIZE", "1"))
    X, Q, adj, med, pq, gt, _ = workload(args, int(os.environ.get("LOCAL_RANK", "0")))
    threads = os.cpu_count() or 1
    name = HEADLINE
    o = _oracle_variant(X, adj, med, pq, name, native=True)
    L, curve = L_SWEEP[-1], []
    for Lc in L_SWEEP:
        ids, _, _ = _oracle_run(o, name, Q, Lc, threads)
        rec = recall(ids, gt)
        curve.append((Lc, round(rec, 4)))
        if rec >= args.target_recall:
            L = Lc
            break
    for _ in range(args.warmup):
        _oracle_run(o, name, Q[:1000], L, threads)
    step_s = []
    for _ in range(args.steps):
        t0 = time.time()
        ids, _, _ = _oracle_run(o, name, Q, L, threads)
        step_s.append(time.time() - t0)
    dt = float(np.sum(step_s))
    qps = len(Q) * args.steps / dt
    rec = recall(ids, gt)
    line = {
        "impl": "reference", "metric": METRIC, "value": qps, "unit": "queries/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16+f32",
        "data": "synthetic (seeded 256-centre Gaussian mixture, 1M x 128, 10k queries)",
        "config": config_of(args, world, L),
        "recall_at_10": round(rec, 4), "recall_curve": curve,
        "p99_ms": float(np.percentile(np.array(step_s) * 1e3, 99)),
        "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": threads, "kind": "port",
                         "sample": f"the {len(Q)}-query batch per step: BF16 traversal + FP32 rerank of the top "
                                   f"{L} (CPU restatement of the reference's quantized search, -O3 -march=native, "
                                   f"OpenMP over queries)"},
        "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main() or 0)
