#!/usr/bin/env python
"""Benchmark of the B200 VIA server answer path.

Workload (one step = one answer of one query): the paper VIA-C preset
(n1=2048, n2=512, q1 two 37/38-bit primes, q2 34-bit) over a 1 GiB database of
4-bit records laid out I=2^8 x J=2^12 (the reference's docs/params.html Table 4
dimensions for 1 GiB). The prepared database is 8.5 GiB in HBM (four byte
planes and a two-bit plane per eval-form residue, the operand layout of the
tensor-core scan), far larger
than L2, so every step streams it from DRAM. Every step answers a distinct
query for a seeded index.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). `value` is whole-job answers/s with the query
already resident on the device; `e2e` is the same through the host-buffer C ABI
call via_server_answer (query upload and answer download inside the timed
region). With N > 1 (torchrun) every rank answers on its own full replica
("replicas only": the answer path does not shard), timed as the max over ranks.

Further legs (1 GPU): 64-query shared-scan batches and a Poisson-served stream
at 1 GiB; VIA-B (T = 8); kernel micro-benchmarks; the scan's roofline; then the
64-query batched workload at 4 GiB and the served VIA-C / VIA-B mix at 8 GiB;
last, the CPU oracle on one full-size answer (`cpu_baseline`).
"""
import argparse
import ctypes
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "answers/s and DB GB/s scanned, batched vs plain, 1 GiB DB; p50/p99 answer ms"
# ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_fd_tc launch on the
# I=64, J=4096 paper case (packed planes, q2 < 2^34): 2.284716288 GB read,
# 130.85696 MB written. Reads scale with the database cells (each cell's
# 4.25 * n1 plane bytes are read once, plus the selection chunks that miss L2),
# writes with the columns (2 * n1 u64 residues per column).
SCAN_READ_BYTES_PER_CELL = 2.284716288e9 / (64 * 4096)
SCAN_WRITE_BYTES_PER_COLUMN = 130.85696e6 / 4096


def prepared_db_bytes(prm):
    """Bytes of the byte-plane database: rows padded to 64, columns to 128; five
    planes per residue, or four and a two-bit plane for q2 below 2^34 (34816 bytes
    per 128 x 64 chunk instead of 40960)."""
    ru = lambda v, a: (v + a - 1) // a * a
    chunks = ru(prm.num_rows, 64) // 64 * (ru(prm.num_cols, 128) // 128) * prm.n1
    return chunks * (34816 if prm.q2 < (1 << 34) else 40960)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rows", type=int, default=256)
    ap.add_argument("--cols", type=int, default=4096)
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU oracle leg (for profiling)")
    ap.add_argument("--scan-launches", type=int, default=10)
    ap.add_argument("--batch", type=int, default=64, help="queries per shared-scan batch (0 = skip)")
    ap.add_argument("--served", type=int, default=384,
                    help="requests of the served leg (Poisson arrivals, continuous batching; 0 = skip)")
    ap.add_argument("--via-b", type=int, default=1, help="run the VIA-B leg (T = 8, records of degree 64)")
    ap.add_argument("--mixed", type=int, default=32,
                    help="requests in the mixed VIA-C / VIA-B served leg at 8 GiB (0 = skip)")
    ap.add_argument("--mixed-rate", type=float, default=2.0, help="arrival rate (requests/s) of the mixed leg")
    ap.add_argument("--big", type=int, default=1,
                    help="run the 4 GiB batched and 8 GiB mixed legs after the 1 GiB legs (0 = skip)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default scan tiles (skip the autotuner)")
    ap.add_argument("--microbench", type=int, default=1, help="run the kernel micro-benchmark leg (NTT, external "
                    "product, key switch at n = 2048)")
    ap.add_argument("--scan-tile", default="",
                    help="n_max,stages,order: force this scan tile for --batch queries (after any autotuning)")
    ap.add_argument("--profile-batch", action="store_true",
                    help="set up, answer one batch of --batch queries and exit (a short target for ncu)")
    return ap.parse_args()


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_tensor_peak():
    """Dense bf16 tensor TFLOP/s (burst), measured when MEASURED_PEAKS.json holds it."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        if "bf16_tflops" in d:
            return float(d["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


# ---------------------------------------------------------------------------
# Synthetic inputs (seeded). Key and query residues are uniform: the answer's
# cost does not depend on their values; correctness is covered by the tests.
# ---------------------------------------------------------------------------
def make_inputs(prm, seed):
    from via_rs_b200.server import PublicKeys

    rng = np.random.default_rng(seed)
    qmin = min(prm.q1)
    records = rng.integers(0, 256, size=prm.capacity * prm.n_rec // 2, dtype=np.uint8)
    keys = PublicKeys(rng.integers(0, qmin, size=prm.cascade_key_len, dtype=np.uint64),
                      rng.integers(0, qmin, size=prm.conv_key_len, dtype=np.uint64),
                      rng.integers(0, prm.q3, size=prm.rsk_len, dtype=np.uint64))
    query = rng.integers(0, qmin, size=prm.n_lwe * prm.lwe_len, dtype=np.uint64)
    return records, keys, query


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (a restatement of the reference's Rust server, with
# its threading: FirstDim over all host threads, the rest serial) answering
# full-size queries of the same workload. Setup (Server::setup) is not timed.
# ---------------------------------------------------------------------------
def cpu_server(prm, seed):
    from oracle import pyoracle

    records, keys, _ = make_inputs(prm, seed)
    threads = os.cpu_count() or 1
    srv = pyoracle.Server(prm, keys.cascade_key, keys.conv_key, keys.rsk, records, threads)
    del records
    return srv, threads


def cpu_answer_times(srv, prm, count, seed):
    """Wall seconds of `count` full answers, each of a fresh seeded query."""
    rng = np.random.default_rng(seed)
    qmin = min(prm.q1)
    times = []
    for _ in range(count):
        q = rng.integers(0, qmin, size=prm.n_lwe * prm.lwe_len, dtype=np.uint64)
        t0 = time.perf_counter()
        srv.answer(q)
        times.append(time.perf_counter() - t0)
    return times


def cpu_sample_text(prm, threads, n, seconds):
    return (f"{n} full oracle answer(s) of the workload itself (I={prm.num_rows}, J={prm.num_cols}, "
            f"{prm.n_lwe} query LWEs, every stage run, no extrapolation): {seconds:.2f} s on {threads} threads; "
            "setup not timed")


def reference_arm(args, prm):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    try:
        srv, threads = cpu_server(prm, seed=7)
    except (MemoryError, RuntimeError) as e:
        print(json.dumps({"impl": "reference", "unavailable": f"the oracle could not prepare the database: {e}"}),
              flush=True)
        return
    cpu_answer_times(srv, prm, args.warmup, seed=70)
    times = cpu_answer_times(srv, prm, args.steps, seed=71)
    t_step = sum(times) / len(times)
    value = 1.0 / t_step
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "answers/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": config_dict(prm),
        "cpu_baseline": {"value": value, "unit": "answers/s", "cores": threads, "kind": "port",
                         "sample": cpu_sample_text(prm, threads, len(times), sum(times))
                         + "; Rust toolchain unavailable, so the C++ oracle restatement is timed"},
        "e2e": {"value": value, "unit": "answers/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_dict(prm):
    gib = prm.capacity * prm.n_rec // 2 / (1 << 30)
    return {"workload": f"paper VIA-C answer, {gib:g} GiB DB (I={prm.num_rows}, J={prm.num_cols}, n1={prm.n1}), "
                        "one query per step",
            "preset": "paper (q1=137438822401*274810798081, q2=17175674881, q3=8380417, q4=4096, p=16)",
            "db_raw_bytes": prm.capacity * prm.n_rec // 2, "db_prepared_bytes": prepared_db_bytes(prm),
            "l2": f"inputs larger than L2: the {prepared_db_bytes(prm) / (1 << 30):g} GiB prepared DB "
                  "is streamed every step"}


# ---------------------------------------------------------------------------
# GPU arm.
# ---------------------------------------------------------------------------
def max_over_ranks(seconds, dist, device):
    """The job's time: the slowest rank's (replicas run in parallel; the job ends
    with the last one). Every rank calls this at the same point."""
    if dist is None:
        return seconds
    import torch

    t = torch.tensor([seconds], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def load_client(prm, seed):
    """The device client (via_client_*) with seeded ternary secrets: the load
    generator for distinct, well-formed queries at seeded indices. The server's
    public keys are seeded residues, not this client's, so the answers do not
    decrypt; the answer's cost does not depend on key or query values."""
    from via_rs_b200.client import Client

    rng = np.random.default_rng(seed)
    t1 = rng.integers(-1, 2, size=prm.nl * prm.n1)
    sk1 = np.concatenate([np.where(t1[l * prm.n1:(l + 1) * prm.n1] < 0, q + t1[l * prm.n1:(l + 1) * prm.n1],
                                   t1[l * prm.n1:(l + 1) * prm.n1]).astype(np.uint64)
                          for l, q in enumerate(prm.q1)])
    t2 = rng.integers(-1, 2, size=prm.n2)
    sk2 = np.where(t2 < 0, prm.q3 + t2, t2).astype(np.uint64)
    return Client(prm, sk1, sk2)


def distinct_queries(prm, n, seed, client=None):
    """n queries for seeded uniform indices, each from its own PRG seed."""
    own = client is None
    c = load_client(prm, seed) if own else client
    idx = np.random.default_rng(seed + 1).integers(prm.capacity, size=n)
    parts = []
    for k in range(0, n, 64):
        chunk = idx[k:k + 64]
        parts.append(c.queries(chunk, [b"q-%08d-%08d" % (seed, k + j) for j in range(len(chunk))]))
    if own:
        c.close()
    return np.concatenate(parts)


def served_leg(args, prm, server, queries, rate):
    """Seeded Poisson arrivals at `rate` requests/s into a 2-lane service, each
    request a distinct query; returns throughput and the service's p50/p99
    submit-to-answer latency."""
    from via_rs_b200.service import Service

    rng = np.random.default_rng(7)
    gaps = rng.exponential(1.0 / rate, size=args.served)
    # Scan tiles tuned for batch sizes 1, 2, 4, ..., 64 and the graphs of every
    # batch size captured up front.
    svc = Service(server, lanes=2, max_batch=64, warm=True, autotune=not args.no_autotune)
    try:
        for t in [svc.submit(queries[k]) for k in range(4)]:
            svc.wait(t)
        svc.reset_stats()
        tickets = []
        t0 = time.perf_counter()
        due = t0
        for k, g in enumerate(gaps):
            due += g
            while time.perf_counter() < due:
                time.sleep(min(0.0005, max(0.0, due - time.perf_counter())))
            tickets.append(svc.submit(queries[k % len(queries)]))
        for t in tickets:
            svc.wait(t)
        wall = time.perf_counter() - t0
        st = svc.stats()
        tuning = svc.tuning()
    finally:
        svc.close()
    return {"requests": args.served, "distinct_queries": min(args.served, len(queries)), "offered_rate_hz": rate,
            "answers_s": st["answers_per_s"], "wall_answers_s": args.served / wall, "p50_ms": st["p50_ms"],
            "p99_ms": st["p99_ms"], "mean_batch": st["mean_batch"], "batches": st["batches"], "lanes": st["lanes"],
            "max_in_flight": st["max_in_flight"], "arrivals": "seeded Poisson (numpy PCG64 seed 7)",
            "scan_tiles": [{"batch": e["batch"], **e["tile"]} for e in tuning]}


def timed_answers(L, server, prm, queries, steps, warmup, stream):
    """Device-resident answers: one query per step (queries cycled), CUDA events
    on `stream`. Returns (answers/s, per-step ms)."""
    import torch

    from via_rs_b200.server import check

    d_q = torch.from_numpy(np.ascontiguousarray(queries).view(np.int64)).cuda()
    d_m = torch.empty(prm.n2, dtype=torch.int64, device="cuda")
    d_b = torch.empty(prm.n2, dtype=torch.int64, device="cuda")
    qlen = prm.n_lwe * prm.lwe_len
    sptr = ctypes.c_void_p(stream.cuda_stream)

    def one(k):
        check(L.via_server_answer_dev(server._h, ctypes.c_void_p(d_q.data_ptr() + (k % len(queries)) * qlen * 8),
                                      prm.n_lwe, ctypes.c_void_p(d_m.data_ptr()), ctypes.c_void_p(d_b.data_ptr()),
                                      sptr))

    for k in range(warmup):
        one(k)
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    evs[0].record(stream)
    for k in range(steps):
        one(k)
        evs[k + 1].record(stream)
    torch.cuda.synchronize()
    ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(steps)]
    return steps / (evs[0].elapsed_time(evs[-1]) / 1e3), ms


def timed_batches(L, server, prm, queries, steps, warmup, stream):
    """Device-resident shared-scan batches of len(queries) distinct queries per
    step (via_server_answer_many_dev). Returns (answers/s, per-batch ms)."""
    import torch

    from via_rs_b200.server import check

    B = len(queries)
    check(L.via_server_reserve(server._h, B))
    d_qb = torch.from_numpy(np.ascontiguousarray(queries).view(np.int64)).cuda()
    d_mb = torch.empty(B * prm.n2, dtype=torch.int64, device="cuda")
    d_bb = torch.empty(B * prm.n2, dtype=torch.int64, device="cuda")
    sptr = ctypes.c_void_p(stream.cuda_stream)

    def one():
        check(L.via_server_answer_many_dev(server._h, ctypes.c_void_p(d_qb.data_ptr()), B, prm.n_lwe,
                                           ctypes.c_void_p(d_mb.data_ptr()), ctypes.c_void_p(d_bb.data_ptr()), sptr))

    for _ in range(warmup):
        one()
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    evs[0].record(stream)
    for k in range(steps):
        one()
        evs[k + 1].record(stream)
    torch.cuda.synchronize()
    ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(steps)]
    return steps * B / (evs[0].elapsed_time(evs[-1]) / 1e3), ms


def batched_4gib_leg(args, seed):
    """The batched workload at 4 GiB (I = 2^9, J = 2^13): plain answers, then
    shared-scan batches of `--batch` distinct seeded-index queries, tuned scan."""
    import torch

    from via_rs_b200 import _lib
    from via_rs_b200.params import paper_preset
    from via_rs_b200.server import VIA_RECORDS_NIBBLE, Server

    prm = paper_preset(512, 8192)
    L = _lib.lib()
    records, keys, _ = make_inputs(prm, seed)
    server = Server.setup(prm, keys, records, VIA_RECORDS_NIBBLE)
    del records
    B = args.batch
    queries = distinct_queries(prm, B, seed=seed + 1)
    tuning = [] if args.no_autotune else server.autotune([1, B])
    stream = torch.cuda.Stream()
    plain, plain_ms = timed_answers(L, server, prm, queries, steps=8, warmup=3, stream=stream)
    batched, b_ms = timed_batches(L, server, prm, queries, steps=3, warmup=1, stream=stream)
    db = prepared_db_bytes(prm)
    server.close()
    del server
    torch.cuda.empty_cache()
    return {"db_raw_bytes": prm.capacity * prm.n_rec // 2, "rows": prm.num_rows, "cols": prm.num_cols,
            "db_prepared_bytes": db, "batch": B, "distinct_queries": B,
            "plain_answers_s": plain, "plain_p50_ms": float(np.percentile(plain_ms, 50)),
            "plain_db_gbs": plain * db / 1e9,
            "answers_s": batched, "ms_per_batch": float(np.mean(b_ms)), "p50_ms": float(np.percentile(b_ms, 50)),
            "p99_ms": float(np.percentile(b_ms, 99)), "db_gbs": batched * db / 1e9 / B,
            "vs_plain": batched / plain, "autotune": tuning}


def mixed_8gib_leg(args, seed):
    """The served mixed load at 8 GiB (I = 2^10, J = 2^13): a seeded Poisson
    stream of VIA-C queries and VIA-B requests of 1..256 indices (log-uniform),
    each VIA-B request padded to the smallest power-of-two batch T >= m and
    served from views of the one prepared database (a continuous-batching
    service per view, admitted by an HBM budget). Every request carries
    distinct queries; one request per route is re-answered alone and compared."""
    import torch

    from via_rs_b200 import _lib
    from via_rs_b200.mixed import MixedService, poisson_mix, via_b_route
    from via_rs_b200.params import paper_preset
    from via_rs_b200.server import VIA_RECORDS_NIBBLE, Server

    prm = paper_preset(1024, 8192)
    L = _lib.lib()
    records, keys, _ = make_inputs(prm, seed)
    server = Server.setup(prm, keys, records, VIA_RECORDS_NIBBLE)
    del records
    stream = torch.cuda.Stream()
    plain_q = distinct_queries(prm, 4, seed=seed + 1)
    if not args.no_autotune:
        server.autotune([1])
    plain, _ = timed_answers(L, server, prm, plain_q, steps=4, warmup=2, stream=stream)
    free, _ = torch.cuda.mem_get_info()
    budget = int(free * 0.6)
    t_build = time.perf_counter()
    mix = MixedService(server, lanes=2, hbm_budget=budget, autotune=not args.no_autotune)
    t_build = time.perf_counter() - t_build
    clients = {}

    def queries(route, n_req):
        pv = mix.params(route)
        if route not in clients:
            clients[route] = load_client(pv, seed + 100 + (0 if route == "c" else route))
        return distinct_queries(pv, 1 if route == "c" else route, seed=seed + 1000 + n_req, client=clients[route])

    plan = []
    for k, (gap, kind, m) in enumerate(poisson_mix(args.mixed, args.mixed_rate, seed=22)):
        route = "c" if kind == "c" else via_b_route(m)
        plan.append((gap, route, m, queries(route, k)))
    for c in clients.values():
        c.close()
    routes = sorted({p[1] for p in plan}, key=str)
    try:
        for route in routes:  # one warm request per route in the stream
            mix.wait(mix.submit(route, next(p[3] for p in plan if p[1] == route)))
        mix.reset_stats()
        handles = []
        t0 = time.perf_counter()
        due = t0
        for gap, route, m, q in plan:
            due += gap
            while time.perf_counter() < due:
                time.sleep(min(0.0005, max(0.0, due - time.perf_counter())))
            handles.append(mix.submit(route, q))
        answers = [mix.wait(h) for h in handles]
        wall = time.perf_counter() - t0
        lat = mix.latencies()
        mix.close_services()  # frees the lanes before the views answer alone
        exact = True
        for route in routes:
            k = next(i for i, p in enumerate(plan) if p[1] == route)
            srv = mix.servers[route]
            alone = srv.answer(plan[k][3]) if route == "c" else srv.answer_batch(plan[k][3].reshape(route, -1))
            exact = exact and np.array_equal(alone[0], answers[k][0]) and np.array_equal(alone[1], answers[k][1])
            if route != "c":  # each view's own workspace goes before the next view answers
                mix.servers.pop(route).close()
    finally:
        mix.close()
        server.close()
        del server
        torch.cuda.empty_cache()
    n_c = sum(1 for p in plan if p[1] == "c")
    b = [p for p in plan if p[1] != "c"]
    records_n = n_c + sum(p[2] for p in b)
    slots = sum(p[1] for p in b)
    all_lat = np.concatenate([v for v in lat.values() if len(v)])

    def pct(v, q):
        return float(np.percentile(v, q)) if len(v) else None

    return {"db_raw_bytes": prm.capacity * prm.n_rec // 2, "rows": prm.num_rows, "cols": prm.num_cols,
            "db_prepared_bytes": prepared_db_bytes(prm), "plain_answers_s": plain,
            "requests": len(plan), "via_c": n_c, "via_b": len(b),
            "via_b_by_t": {str(t): sum(1 for p in b if p[1] == t) for t in routes if t != "c"},
            "offered_rate_hz": args.mixed_rate, "requests_s": len(plan) / wall, "answers_s": len(plan) / wall,
            "records_s": records_n / wall, "padding_frac": (slots - sum(p[2] for p in b)) / max(1, slots),
            "p50_ms": pct(all_lat, 50), "p99_ms": pct(all_lat, 99),
            "p50_ms_by_route": {str(k): pct(v, 50) for k, v in lat.items() if len(v)},
            "p99_ms_by_route": {str(k): pct(v, 99) for k, v in lat.items() if len(v)},
            "hbm_budget_bytes": budget, "services_build_s": t_build, "sampled_bit_exact": bool(exact),
            "arrivals": "seeded Poisson (numpy PCG64 seed 22), half VIA-C, VIA-B sizes log-uniform in 1..256"}


def microbench_leg(args, prm, peak):
    """Kernel micro-benchmarks on seeded uniform residues at n = 2048: the NTT of
    65536 polynomials over both q1 primes, 16384 external products (DMux gadget
    55879, L = 2 at q1; CMux gadget 81, L = 2 at q2) and 16384 key switches of
    rotated ciphertexts (conversion-key gadget 18, L = 18 at q1). CUDA events on
    the launching stream; each call is one whole batch."""
    import torch

    from via_rs_b200 import prims
    from via_rs_b200.params import PAPER_Q1, PAPER_Q2

    n = 2048
    gen = torch.Generator(device="cuda").manual_seed(11)
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream

    def rand(q, count):
        parts = [torch.randint(0, int(qi), (count, 1, n), dtype=torch.int64, device="cuda", generator=gen) for qi in q]
        return torch.cat(parts, dim=1).contiguous()

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {"n": n, "data": "seeded uniform residues (torch Philox seed 11)"}
    q1 = tuple(PAPER_Q1)
    r1 = prims.ring(n, q1)
    polys = 65536
    x = rand(q1, polys)
    ntt_bytes = 2 * x.numel() * 8  # read + write of every residue
    for name, fn in (("ntt_forward", prims.ntt_forward_dev), ("ntt_inverse", prims.ntt_inverse_dev)):
        ms = timed(lambda: fn(r1, x.data_ptr(), polys, sp))
        out[name] = {"polys": polys, "primes": 2, "ms": ms, "limb_transforms_s": polys * 2 / ms * 1e3,
                     "gbs": ntt_bytes / ms / 1e6, "hbm_frac": ntt_bytes / ms / 1e6 / peak}
    del x
    pairs = 16384
    for name, q, base, L in (("external_product_q1", q1, 55879, 2), ("external_product_q2", (PAPER_Q2,), 81, 2)):
        r = prims.ring(n, q)
        rg = rand(q, pairs * 2 * L * 2)
        ct = rand(q, pairs * 2)
        o = torch.empty_like(ct)
        ms = timed(lambda: prims.external_product_dev(r, base, L, rg.data_ptr(), ct.data_ptr(), pairs, o.data_ptr(), sp))
        out[name] = {"pairs": pairs, "base": base, "levels": L, "ms": ms, "per_s": pairs / ms * 1e3}
        del rg, ct, o
    L = 18
    key = rand(q1, L * 2)
    ct = rand(q1, pairs * 2)
    shifts = torch.from_numpy(np.random.default_rng(12).integers(0, 2 * n, size=pairs).astype(np.int64)).cuda()
    o = torch.empty_like(ct)
    ms = timed(lambda: prims.key_switch_dev(r1, 18, L, key.data_ptr(), ct.data_ptr(), shifts.data_ptr(), pairs,
                                            o.data_ptr(), sp))
    out["key_switch_q1"] = {"ciphertexts": pairs, "base": 18, "levels": L, "rotation": "X^k, k uniform in [0, 2n)",
                            "ms": ms, "per_s": pairs / ms * 1e3}
    del key, ct, o
    torch.cuda.empty_cache()
    out["client"] = client_microbench(prm)
    return out


def client_microbench(prm):
    """Device client at the bench's preset and grid: 64 queries generated per call
    (one seeded PRG stream each) and 256 answers recovered per call."""
    rng = np.random.default_rng(13)
    c = load_client(prm, 13)
    n = 64
    idx = rng.integers(prm.capacity, size=n)
    seeds = [b"bench-%04d" % k for k in range(n)]
    c.queries(idx[:2], seeds[:2])
    t0 = time.perf_counter()
    c.queries(idx, seeds)
    tq = time.perf_counter() - t0
    masks = rng.integers(0, prm.q3, size=(256, prm.n2), dtype=np.uint64)
    bodies = rng.integers(0, prm.q4, size=(256, prm.n2), dtype=np.uint64)
    c.recover_many(masks[:2], bodies[:2])
    t0 = time.perf_counter()
    c.recover_many(masks, bodies)
    tr = time.perf_counter() - t0
    c.close()
    return {"queries": n, "query_ms": tq * 1e3, "queries_s": n / tq, "query_bytes": int(prm.n_lwe * prm.lwe_len * 8),
            "recovers": 256, "recover_ms": tr * 1e3, "recovers_s": 256 / tr,
            "timing": "host wall clock around the synchronous call (host buffers, copies included)"}


def via_b_leg(args, prm, rank):
    """answer_batch with T = n2 / n3 = 8 queries per answer over the same number
    of database cells (records of degree 64: 8x the records of the VIA-C leg)."""
    import torch

    from via_rs_b200.params import paper_preset
    from via_rs_b200.server import VIA_RECORDS_NIBBLE, Server, check
    from via_rs_b200 import _lib

    pb = paper_preset(prm.num_rows, prm.num_cols, n_rec=64)
    T = pb.n2 // pb.n_rec
    records, keys, _ = make_inputs(pb, seed=100 + rank)
    srv = Server.setup(pb, keys, records, VIA_RECORDS_NIBBLE)
    del records
    L = _lib.lib()
    qs = torch.from_numpy(distinct_queries(pb, T, seed=200 + rank).view(np.int64)).cuda()
    dm = torch.empty(pb.n2, dtype=torch.int64, device="cuda")
    db = torch.empty(pb.n2, dtype=torch.int64, device="cuda")
    stream = torch.cuda.Stream()
    sptr = ctypes.c_void_p(stream.cuda_stream)

    def one():
        check(L.via_server_answer_batch_dev(srv._h, ctypes.c_void_p(qs.data_ptr()), T, pb.n_lwe,
                                            ctypes.c_void_p(dm.data_ptr()), ctypes.c_void_p(db.data_ptr()), sptr))

    for _ in range(2):
        one()
    torch.cuda.synchronize()
    k = max(2, args.steps // 4)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(k):
        one()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / k
    srv.close()
    return {"T": T, "record_degree": pb.n_rec, "ms_per_answer": ms, "answers_s": 1e3 / ms,
            "records_s": T * 1e3 / ms, "db_raw_bytes": pb.capacity * pb.n_rec // 2}


def log_leg(name, result):
    """Each finished leg on stderr (the JSON line on stdout comes at the end)."""
    print(json.dumps({"leg": name, "result": result}), file=sys.stderr, flush=True)


def gpu_arm(args, prm):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from via_rs_b200 import _lib
    from via_rs_b200.server import VIA_RECORDS_NIBBLE, Server, check

    L = _lib.lib()
    records, keys, query = make_inputs(prm, seed=rank)
    server = Server.setup(prm, keys, records, VIA_RECORDS_NIBBLE)
    del records
    stream = torch.cuda.Stream()
    sptr = ctypes.c_void_p(stream.cuda_stream)
    # Distinct well-formed queries at seeded indices (the device client).
    n_distinct = max(args.steps, args.batch, min(args.served, 384), 1)
    queries = distinct_queries(prm, n_distinct, seed=1000 + rank)
    qlen = prm.n_lwe * prm.lwe_len
    d_q = torch.from_numpy(queries[:args.steps].view(np.int64)).cuda()
    d_m = torch.empty(prm.n2, dtype=torch.int64, device="cuda")
    d_b = torch.empty(prm.n2, dtype=torch.int64, device="cuda")

    def answer_dev(k):
        check(L.via_server_answer_dev(server._h, ctypes.c_void_p(d_q.data_ptr() + (k % args.steps) * qlen * 8),
                                      prm.n_lwe, ctypes.c_void_p(d_m.data_ptr()), ctypes.c_void_p(d_b.data_ptr()),
                                      sptr))

    # Scan autotuner: the fastest tile for one query and for the batched leg.
    tuning = []
    if not args.no_autotune:
        tuning = server.autotune([1] + ([args.batch] if args.batch > 1 else []))
    if args.scan_tile:
        nm, st, od = (int(v) for v in args.scan_tile.split(","))
        server.set_scan_tile(max(1, args.batch), {"n_max": nm, "stages": st, "order": od})

    if args.profile_batch:
        B = max(1, args.batch)
        mb, bb = server.answer_many(queries[:B])
        torch.cuda.synchronize()
        print(json.dumps({"profile_batch": B, "answers": int(mb.shape[0])}), flush=True)
        server.close()
        return

    for k in range(args.warmup):
        answer_dev(k)
    torch.cuda.synchronize()

    # ---- timed region: K device-resident answers, one distinct query each.
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = L.via_kernel_launches()
    with torch.cuda.stream(stream):
        evs[0].record(stream)
        for k in range(args.steps):
            answer_dev(k)
            evs[k + 1].record(stream)
    torch.cuda.synchronize()
    launches = L.via_kernel_launches() - l0
    if dist:
        dist.barrier()
    clk = clocks.stop()
    step_ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(args.steps)]
    elapsed = evs[0].elapsed_time(evs[-1]) / 1e3
    elapsed = max_over_ranks(elapsed, dist, "cuda")
    n_answers = args.steps * world
    value = n_answers / elapsed
    db_bytes = prepared_db_bytes(prm)

    # ---- e2e: the reference-facing host-buffer call, copies inside the region;
    # the queries sit in pinned host memory.
    q_host = torch.from_numpy(np.ascontiguousarray(queries[:min(n_distinct, args.steps)]).view(np.int64))
    q_host = q_host.pin_memory().numpy().view(np.uint64)
    for k in range(2):
        server.answer(q_host[k % len(q_host)])
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(args.steps):
        server.answer(q_host[k % len(q_host)])
    e2e_el = time.perf_counter() - t0
    e2e_el = max_over_ranks(e2e_el, dist, "cuda")
    e2e_value = n_answers / e2e_el

    # ---- batched: B distinct queries per step share one database pass.
    batched = None
    if args.batch > 1:
        B = args.batch
        kb = max(2, args.steps // 4)
        if dist:
            dist.barrier()
        b_value, b_ms = timed_batches(L, server, prm, queries[:B], steps=kb, warmup=2, stream=stream)
        b_el = max_over_ranks(kb * B / b_value, dist, "cuda")
        b_value = kb * B * world / b_el
        batched = {"answers_s": b_value, "batch": B, "distinct_queries": B, "steps": kb,
                   "ms_per_batch": b_el / kb * 1e3, "db_gbs": b_value * db_bytes / 1e9 / B,
                   "p50_ms": float(np.percentile(b_ms, 50)), "p99_ms": float(np.percentile(b_ms, 99)),
                   "vs_plain": b_value / value}

    # ---- served: Poisson arrivals of distinct queries through the service.
    served = None
    if args.served > 0:
        served = served_leg(args, prm, server, queries, rate=0.85 * (batched["answers_s"] if batched else value))

    # ---- VIA-B: T = 8 records of degree 64 per answer on a second (1 GiB) server.
    via_b = None
    if args.via_b and world == 1:
        via_b = via_b_leg(args, prm, rank)

    # ---- kernel micro-benchmarks (NTT, external product, key switch).
    micro = None
    if args.microbench and world == 1:
        micro = microbench_leg(args, prm, load_peaks()[0])

    # ---- roofline of the dominant kernel: the FirstDim scan alone, timed live.
    sel = torch.randint(0, prm.q2, (prm.num_rows * 2 * prm.n1,), dtype=torch.int64, device="cuda")
    out = torch.empty(prm.num_cols * 2 * prm.n1, dtype=torch.int64, device="cuda")
    for _ in range(2):
        check(L.via_first_dim_scan_dev(server._h, ctypes.c_void_p(sel.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                       sptr))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.scan_launches):
        check(L.via_first_dim_scan_dev(server._h, ctypes.c_void_p(sel.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                       sptr))
    e1.record(stream)
    torch.cuda.synchronize()
    scan_s = e0.elapsed_time(e1) / 1e3 / args.scan_launches
    scan_bytes = db_bytes + sel.numel() * 8 + out.numel() * 8
    peak, peak_kind = load_peaks()
    achieved = scan_bytes / scan_s / 1e9

    # ---- the batched scan as a tensor-core contraction: B queries' selections
    # against the byte planes, 25 byte-product GEMMs per eval slot (kind::i8).
    # Its time is the autotuner's live CUDA-event measurement of the kept tile
    # (three timed scans on preallocated buffers).
    roofline_batched = None
    tuned_b = next((e for e in tuning if e["batch"] == args.batch), None) if args.batch > 1 else None
    if tuned_b:
        B = args.batch
        bscan_s = tuned_b["ms"] / 1e3
        macs = 25.0 * prm.n1 * prm.num_rows * prm.num_cols * 2 * B  # byte products, all 25 limb pairs
        tpeak, tpeak_kind = load_tensor_peak()
        i8_peak = 2.0 * tpeak  # dense int8 = 2x dense bf16 on this tensor core
        achieved_tops = 2.0 * macs / bscan_s / 1e12
        roofline_batched = {"bound": "tensor", "kernel": f"k_fd_split + k_fd_tc, {B} queries (tcgen05 kind::i8)",
                            "achieved": achieved_tops, "peak": i8_peak, "unit": "TOP/s (int8)",
                            "frac": achieved_tops / i8_peak, "peak_kind": f"2x {tpeak_kind} bf16 TFLOP/s",
                            "launch_ms": bscan_s * 1e3, "tile": tuned_b["tile"], "int8_ops": 2.0 * macs,
                            "db_gbs": db_bytes / bscan_s / 1e9}
    server.close()
    del server, d_q, sel, out
    torch.cuda.empty_cache()

    # ---- the configs' larger databases (1 GPU): 4 GiB batched, 8 GiB served mix.
    log_leg("plain", {"answers_s": value, "e2e": e2e_value, "scan_ms": scan_s * 1e3})
    log_leg("batched", batched)
    log_leg("served", served)
    big4 = batched_4gib_leg(args, seed=40 + rank) if args.big and world == 1 and args.batch > 1 else None
    log_leg("batched_4gib", big4)
    mixed8 = mixed_8gib_leg(args, seed=80 + rank) if args.big and world == 1 and args.mixed > 0 else None
    log_leg("mixed_8gib", mixed8)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "answers/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic: seeded uniform 4-bit records (numpy PCG64), seeded key residues, distinct device-client "
                    "queries at seeded indices",
            "config": config_dict(prm),
            "plain": {"answers_s": value, "db_gbs": value * db_bytes / 1e9, "db_raw_gbs": value * (1 << 30) / 1e9,
                      "p50_ms": float(np.percentile(step_ms, 50)), "p99_ms": float(np.percentile(step_ms, 99))},
            "batched": batched,
            "served": served,
            "via_b": via_b,
            "batched_4gib": big4,
            "mixed_8gib": mixed8,
            "microbench": micro,
            "roofline": {"bound": "hbm", "kernel": "k_fd_split + k_fd_tc (tcgen05 FirstDim scan)", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": (SCAN_READ_BYTES_PER_CELL * prm.num_rows * prm.num_cols
                                     + SCAN_WRITE_BYTES_PER_COLUMN * prm.num_cols),
                         "launch_ms": scan_s * 1e3, "algorithmic_bytes": scan_bytes},
            "roofline_batched": roofline_batched,
            "e2e": {"value": e2e_value, "unit": "answers/s", "h2d_bytes_per_step": int(query.nbytes),
                    "d2h_bytes_per_step": int(2 * prm.n2 * 8)},
            "autotune": tuning,
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        if world == 1 and not args.no_cpu_baseline:
            srv, threads = cpu_server(prm, seed=7)
            t = cpu_answer_times(srv, prm, 1, seed=71)
            del srv
            line["cpu_baseline"] = {"value": 1.0 / t[0], "unit": "answers/s", "cores": threads, "kind": "port",
                                    "sample": cpu_sample_text(prm, threads, 1, t[0])}
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def main():
    args = parse()
    from via_rs_b200.params import paper_preset

    prm = paper_preset(args.rows, args.cols)
    if args.impl == "reference":
        reference_arm(args, prm)
    else:
        gpu_arm(args, prm)


if __name__ == "__main__":
    main()
