"""Benchmark of the flat TurboQuant FastScan search on B200.

Workload (default): 1,000,000 x 1536 database, 4-bit codes, TQ+ calibrated on
10,000 rows, 10,000 queries, k = 10 — vectors drawn (seeded) from a Gaussian
with power-law variances lambda_i ~ i^-0.8, a Haar-random rotation and L2
normalization (vectorcache_b200.synthetic.power_law_torch). One step = one
search of the whole query batch against the index.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). Multi-GPU (torchrun, one rank per GPU): every
rank holds its own 1M-vector shard (weak scaling), all ranks search the same
queries, and the per-shard top-k lists are exchanged with one NCCL all-gather
and merged (score desc, id asc) — the only collective of the path.

--impl reference times the reference's own CPU implementation
(oracle/_ref/libtqref.so: encode + repack + search_flat compiled in place from
the reference sources) on this host's cores, on a bounded sample of the same
workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "QPS at fixed Recall@10 (1Mx1536 4-bit, k=10)"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--n", type=int, default=1_000_000, help="vectors per GPU shard")
    p.add_argument("--nq", type=int, default=10_000)
    p.add_argument("--dim", type=int, default=1536)
    p.add_argument("--bits", type=int, default=4)
    p.add_argument("--k", type=int, default=10)
    p.add_argument("--calib", type=int, default=10_000)
    p.add_argument("--recall-queries", type=int, default=1000)
    p.add_argument("--cpu-queries", type=int, default=64, help="queries per CPU-baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-variants", action="store_true", help="skip the (bits, k) variants of the flat workload")
    p.add_argument("--ref-gpu-queries", type=int, default=2368,
                   help="queries the reference's own GPU index searches beside ours (0: skip)")
    p.add_argument("--workload", choices=["flat", "bucketed", "serving", "multi", "encode"], default="flat",
                   help="flat: the 1M x 1536 flat search (default); bucketed: the 1.2M x 100 bucketed index, "
                        "learned n_probe against fixed n_probe; serving: the continuous-batching server over a "
                        "10M x 768 flat index and the bucketed index; multi: 32 flat indexes in one persistent "
                        "graph-captured launch; encode: the encode kernels alone")
    p.add_argument("--serving-flat-n", type=int, default=10_000_000)
    p.add_argument("--bucketed-n", type=int, default=1_200_000)
    p.add_argument("--bucketed-train", type=int, default=50_000, help="training queries of the learned probe")
    p.add_argument("--rerank", type=int, default=100, help="bucketed: candidates re-ranked exactly (0 = off)")
    p.add_argument("--epochs", type=int, default=30)
    p.add_argument("--probe-objective", choices=("recall", "classes"), default="recall",
                   help="learned n_probe: fit each class's recall (trade-off rule) or one label class per query "
                        "(cumulative-probability rule)")
    p.add_argument("--bucketed-fixed-only", type=int, default=0,
                   help="bucketed: time the plain path at this n_probe only (no sweep, no learned probe)")
    p.add_argument("--extra-classes", type=str, default="",
                   help="learned n_probe: comma-separated candidate n_probe values added below the operating point")
    p.add_argument("--learned-above", type=str, default=",".join(str(c) for c in LEARNED_ABOVE),
                   help="learned n_probe: comma-separated candidate n_probe values above the operating point")
    return p.parse_args()


def _int_list(text):
    return tuple(int(v) for v in text.split(",") if v.strip())


def learned_classes(args, p_op):
    """Candidate n_probe values of the learned probe: the listed ones (and any
    --extra-classes) below the fixed operating point, the operating point,
    and the --learned-above values above it."""
    below = sorted({c for c in PROBE_CLASSES + _int_list(args.extra_classes) if c < p_op})
    above = sorted({c for c in _int_list(args.learned_above) if c > p_op})
    return tuple(below) + (p_op,) + tuple(above)


def load_peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    """Per-launch DRAM bytes of the scan kernel from the committed ncu summary."""
    f = ROOT / "profiles" / "scan_traffic.json"
    if not f.exists():
        return None
    try:
        return json.loads(f.read_text())
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.tmp, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        self.tmp.flush()
        rows = []
        for line in Path(self.tmp.name).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.tmp.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(world, value: float) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def merge_shards(world, scores, ids, k):
    """All-gather every rank's top-k and merge: score desc, equal scores by lower id."""
    if world == 1:
        return scores, ids
    from vectorcache_b200.sharded import allgather_merge

    return allgather_merge(scores, ids, k)


def exact_topk(db, q, k):
    """Exact inner-product top-k on the device in fp32 (no TF32)."""
    import torch

    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        best_s = None
        best_i = None
        chunk = 262144
        for s0 in range(0, db.shape[0], chunk):
            sc = q @ db[s0:s0 + chunk].T
            ts, ti = torch.topk(sc, min(k, sc.shape[1]), dim=1)
            ti = ti + s0
            if best_s is None:
                best_s, best_i = ts, ti
            else:
                cs = torch.cat([best_s, ts], 1)
                ci = torch.cat([best_i, ti], 1)
                top = torch.topk(cs, k, dim=1)
                best_s, best_i = top.values, torch.gather(ci, 1, top.indices)
        return best_i
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def recall_at(approx_ids, exact_ids, t):
    a = approx_ids[:, :t]
    e = exact_ids[:, :t]
    hits = sum(len(set(a[r].tolist()) & set(e[r].tolist())) for r in range(a.shape[0]))
    return hits / (t * a.shape[0])


def reference_index(db_host, calib_host, bits):
    """The reference's own CPU index (fit_calibration + encode + repack on all
    host cores); returns (index, threads, build_seconds)."""
    from oracle.oracle import Reference, ReferenceIndex

    ref = Reference()
    t0 = time.perf_counter()
    idx = ReferenceIndex(ref, db_host, bits, calib_rows=calib_host)
    return idx, ref.max_threads(), time.perf_counter() - t0


def time_reference(idx, q_host, k, sample_queries, steps, warmup):
    """QPS of the reference's search_flat per step of `sample_queries` queries."""
    qps = []
    nq = q_host.shape[0]
    for step in range(warmup + steps):
        s0 = (step * sample_queries) % max(1, nq - sample_queries + 1)
        qs = q_host[s0:s0 + sample_queries]
        t = time.perf_counter()
        idx.search(qs, k)
        dt = time.perf_counter() - t
        if step >= warmup:
            qps.append(qs.shape[0] / dt)
    return qps


def cpu_reference_run(db_host, q_host, calib_host, bits, k, sample_queries, steps, warmup):
    """Times the reference's own CPU search_flat (all host cores) on the same
    index; returns (qps_list, threads, build_seconds)."""
    idx, threads, build_s = reference_index(db_host, calib_host, bits)
    qps = time_reference(idx, q_host, k, sample_queries, steps, warmup)
    idx.close()
    return qps, threads, build_s


def reference_gpu_run(db_h, q_h, exact_np, dim, bits, k, nq_time):
    """The reference's own GPU flat index (gpu::FlatIndex from src/gpu, built
    by `make -C oracle refgpu` with the one cast kernels.cu needs) on the same
    B200, data and queries: its host-buffer search of nq_time queries (query
    upload and result download included, as in our e2e number), timed with
    the host clock around the synchronous call; Recall@10 against the same
    exact top-10. It has no TQ+ and keeps an approximate top-k."""
    from oracle.oracle import REF_GPU_SO, ReferenceGpuIndex

    if not REF_GPU_SO.exists():
        return {"unavailable": "oracle/_ref/libtqrefgpu.so was not built"}
    idx = ReferenceGpuIndex(dim, bits)
    try:
        t0 = time.perf_counter()
        idx.add(db_h)
        idx.prepare()
        build_s = time.perf_counter() - t0
        idx.search(q_h[:4], k)  # first launch (module load, buffers)
        qs = q_h[:nq_time]
        t0 = time.perf_counter()
        _, ids = idx.search(qs, k)
        dt = time.perf_counter() - t0
        nr = min(exact_np.shape[0], nq_time)
        return {"impl": "reference gpu::FlatIndex (src/gpu/kernels.cu scan_mq_topk, float ADC, no TQ+)",
                "qps": nq_time / dt, "seconds": dt, "queries": nq_time, "k": k,
                "recall_at_10": recall_at(ids[:nr], exact_np[:nr], min(10, k)), "recall_queries": nr,
                "prepare_s": build_s, "timing": "host clock around the synchronous search (H2D/D2H included)",
                "top_k": "approximate: a few candidates per thread and query (kernels.cu:393-516)"}
    finally:
        idx.close()


def search_parity(ref_idx, q_host, k, got_scores, got_ids):
    """Top-k of our search against the reference's search_flat on the same
    queries: ids identical and scores bit-equal (score desc, ties by lower id)."""
    ws, wi = ref_idx.search(q_host, k)
    got_ids = np.asarray(got_ids).astype(np.uint64)
    got_scores = np.ascontiguousarray(got_scores, np.float32)
    rows_ids = int(np.count_nonzero(np.any(got_ids != wi, axis=1)))
    rows_sc = int(np.count_nonzero(np.any(got_scores.view(np.uint32) != ws.view(np.uint32), axis=1)))
    return {"queries": int(q_host.shape[0]), "k": int(k), "ids_equal": rows_ids == 0,
            "scores_bitequal": rows_sc == 0, "rows_with_id_mismatch": rows_ids,
            "rows_with_score_mismatch": rows_sc}


def code_parity(ref_idx, index):
    """Codes, alpha and TQ+ calibration of our index against the reference's
    encode of the same rows. A code row that differs would be a rounding
    difference at a codebook boundary (allowed within 1e-6 relative); it is
    counted, not hidden."""
    rp, ra = ref_idx.packed()
    gp, ga = index.packed(), index.alpha()
    out = {"rows": int(rp.shape[0]),
           "code_rows_differing": int(np.count_nonzero(np.any(gp != rp, axis=1))),
           "alpha_bitequal": bool(np.array_equal(ga.view(np.uint32), ra.view(np.uint32)))}
    try:
        rsh, rsc = ref_idx.calibration()
        gsh, gsc = index.calibration()
        out["calibration_bitequal"] = bool(np.array_equal(gsh.view(np.uint32), rsh.view(np.uint32)) and
                                           np.array_equal(gsc.view(np.uint32), rsc.view(np.uint32)))
    except RuntimeError:
        out["calibration_bitequal"] = None
    return out


def make_data(args, rank, device):
    import torch

    from vectorcache_b200.synthetic import power_law_torch

    db = power_law_torch(args.n, args.dim, seed=1000 + rank, device=device)
    q = power_law_torch(args.nq, args.dim, seed=7, device=device)
    torch.cuda.synchronize()
    return db, q


def run_reference(args, world, rank):
    if rank != 0:
        return
    import torch

    device = torch.device("cuda", 0) if torch.cuda.is_available() else None
    if device is not None:
        db, q = make_data(args, 0, device)
        db_h, q_h = db.cpu().numpy(), q.cpu().numpy()
        del db, q
    else:
        from vectorcache_b200.synthetic import power_law

        db_h, q_h = power_law(args.n, args.dim, 1000), power_law(args.nq, args.dim, 7)
    calib = db_h[: args.calib]
    qps, threads, build_s = cpu_reference_run(db_h, q_h, calib, args.bits, args.k, args.cpu_queries,
                                              args.steps, args.warmup)
    value = statistics.mean(qps)
    sample = (f"{args.cpu_queries} queries per step against the full {args.n}x{args.dim} {args.bits}-bit "
              f"TQ+ index built by the reference's encode/repack ({build_s:.1f}s); avx2_perm0 backend")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * args.cpu_queries / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": f"flat TurboQuant search {args.n}x{args.dim} {args.bits}-bit TQ+, k={args.k}",
                   "n": args.n, "dim": args.dim, "bits": args.bits, "k": args.k, "nq": args.nq,
                   "queries_per_step": args.cpu_queries,
                   "batch_note": f"steps of {args.cpu_queries} queries (our arm: {args.nq} per step) so that "
                                 "the run ends within minutes; QPS is per query"},
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# Other (bits, k) points of the 1M x 1536 configuration, timed and checked
# against the reference beside the headline (4-bit, k = 10).
VARIANTS = ((4, 64), (2, 10), (2, 64))


def device_timed(fn, stream, steps, warmup):
    """Mean ms per call of fn on `stream`, CUDA events, after `warmup` calls."""
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def run_ours(args, world, rank, local):
    import torch

    import vectorcache_b200 as vcb
    from vectorcache_b200.sharded import ShardedIndex

    device = torch.device("cuda", local)
    db, q = make_data(args, rank, device)
    # Shard r holds global ids [r * n, (r + 1) * n). One TQ+ calibration for
    # every shard: rank 0's first rows, broadcast to the other ranks.
    shard = ShardedIndex(args.dim, args.bits, device=local, shard_base=rank * args.n)
    index = shard.index
    idx_stream = torch.cuda.ExternalStream(index.stream(), device=device)

    # Build: calibrate, stage, encode (timed as encode vectors/s).
    sample = db[: args.calib].clone() if rank == 0 else torch.empty((args.calib, args.dim), device=device)
    shard.calibrate_shared(sample)
    del sample
    index.add_device(db)
    index.set_profiling(True)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(idx_stream)
    index.prepare()
    ev1.record(idx_stream)
    ev1.synchronize()
    prof_build = index.read_profile()
    prepare_ms = ev0.elapsed_time(ev1)  # includes growing the layout buffers
    encode_vps = args.n / (prof_build["encode_ms"] / 1e3)  # encode + relayout kernels
    encode_kernels_ms = prof_build["encode_ms"]

    k = args.k
    # An explicit stream: NULL would mean the index's own (non-blocking) stream.
    stream = torch.cuda.Stream(device=device)
    torch.cuda.set_stream(stream)
    d_scores = torch.empty((args.nq, k), dtype=torch.float32, device=device)
    d_ids = torch.empty((args.nq, k), dtype=torch.int64, device=device)

    def step():
        if world > 1:
            return shard.search_device(q, k, d_scores, d_ids, stream=stream)
        index.search_device(q, k, d_scores, d_ids, stream=stream)
        return d_scores, d_ids

    # Recall@10 of the returned top-k against exact fp32 inner-product top-k.
    nr = min(args.recall_queries, args.nq)
    step()
    torch.cuda.synchronize()
    exact = exact_topk(db, q[:nr], 10)
    exact_np = exact.cpu().numpy()
    recall10 = recall_at(d_ids[:nr].cpu().numpy(), exact_np, min(10, k))
    keep_rows = world == 1 and not (args.no_variants and args.no_cpu_baseline)
    if not keep_rows:
        # Nothing later reads the float rows: free them, so a profiler run of
        # this command holds only the index and the queries on the device.
        del db
        torch.cuda.empty_cache()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    index.read_profile()  # reset counters
    barrier(world)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t0.record(stream)
        for _ in range(args.steps):
            step()
        t1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    elapsed_ms = max_over_ranks(world, t0.elapsed_time(t1))
    prof = index.read_profile()
    clocks = clk.summary()
    plan = index.scan_plan(args.nq, k)

    queries_scanned = args.nq * args.steps * world  # one query against one 1M-vector shard = one unit
    value = queries_scanned / (elapsed_ms / 1e3)
    # this shard's own top-k of the first queries, for the reference comparison
    n_par = min(args.cpu_queries, args.nq)
    dev_top = (d_scores[:n_par].cpu().numpy(), d_ids[:n_par].cpu().numpy()) if world == 1 else None

    # Latency of small batches (device-resident queries): p50 / p99 over repeats.
    latency = {}
    one_query = None
    if world == 1:
        for bsz, reps in ((1, 50), (16, 30), (256, 15)):
            times = []
            sub = q[:bsz]
            for r in range(reps + 3):
                if r == 3:
                    index.read_profile()  # per-kernel times of the timed repeats only
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                index.search_device(sub, k, d_scores, d_ids, stream=stream)
                e1.record(stream)
                e1.synchronize()
                if r >= 3:
                    times.append(e0.elapsed_time(e1))
            p = index.read_profile()
            latency[f"nq={bsz}"] = {"p50_ms": float(np.percentile(times, 50)),
                                    "p99_ms": float(np.percentile(times, 99)),
                                    "qps": bsz / (float(np.median(times)) / 1e3),
                                    "kernel_ms": {"prep": p["prep_ms"] / reps, "scan": p["scan_ms"] / reps,
                                                  "merge": p["merge_ms"] / reps}}
            if bsz == 1 and p["scan_launches"]:
                # One query per pass: the scan's memory-bound regime.
                ms = p["scan_ms"] / p["scan_launches"]
                gbs = args.n * (args.dim // (8 // args.bits) + 4) / (ms / 1e3) / 1e9
                one_query = {"kernel": "scan_kernel (1 query per pass)", "bound": "hbm", "achieved": gbs,
                             "unit": "GB/s", "ms_per_launch": ms}

    # End to end through the public host-buffer API: pinned host queries in,
    # host top-k out, copies inside the timed region.
    q_host = q.cpu().pin_memory()
    out_s = np.empty(args.nq * k, np.float32)
    out_i = np.empty(args.nq * k, np.uint64)
    import ctypes as C

    lib = vcb.load_library()
    ke = C.c_size_t(0)

    def host_step():
        rc = lib.tq_index_search(index._h, C.c_void_p(q_host.data_ptr()), args.nq, k,
                                 out_s.ctypes.data_as(C.c_void_p), out_i.ctypes.data_as(C.c_void_p), C.byref(ke))
        if rc != 0:
            raise RuntimeError(lib.tq_last_error().decode())
        if world > 1:
            s = torch.from_numpy(out_s).view(args.nq, k).to(device)
            i = torch.from_numpy(out_i.view(np.int64)).view(args.nq, k).to(device) + rank * args.n
            ms, mi = merge_shards(world, s, i, k)
            ms.cpu(), mi.cpu()

    for _ in range(max(1, args.warmup)):
        host_step()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk_e2e:
        e0.record(idx_stream)
        for _ in range(args.steps):
            host_step()
        e1.record(idx_stream)
        e1.synchronize()
    barrier(world)
    e2e_ms = max_over_ranks(world, e0.elapsed_time(e1))
    e2e_value = args.nq * args.steps * world / (e2e_ms / 1e3)
    e2e_top = (out_s.reshape(args.nq, k)[:n_par].copy(), out_i.reshape(args.nq, k)[:n_par].copy())

    # Roofline of the dominant kernel (scan): algorithmic bytes per launch over
    # its mean event-timed duration.
    peak, peak_kind = load_peaks()
    scan_launches = max(1, prof["scan_launches"])
    scan_ms_avg = prof["scan_ms"] / scan_launches
    bytes_per_launch = prof["scan_stream_bytes"] / scan_launches
    achieved = bytes_per_launch / (scan_ms_avg / 1e3) / 1e9
    traffic = load_traffic()
    tr = None
    if traffic and traffic.get("n") and traffic.get("dram_bytes_per_launch"):
        # Captured on a smaller case; DRAM traffic scales with the vectors streamed.
        tr = traffic["dram_bytes_per_launch"] * (args.n / traffic["n"]) * (args.nq / traffic.get("nq", args.nq))
    nbg = args.dim // (8 // args.bits)
    lookups = 2.0 * args.nq * args.n * nbg
    total_kernel_ms = prof["prep_ms"] + prof["scan_ms"] + prof["merge_ms"]
    encode_bytes = args.n * (args.dim * 4 + nbg + 4)  # rows read, codes + alpha written

    # The other (bits, k) points of the same data: device-timed QPS, Recall@10,
    # and their top-k for the reference comparison below.
    variants = []
    if keep_rows and not args.no_variants:
        second = {}
        with ClockSampler(local) as clk_var:
            for bits, kv in VARIANTS:
                if (bits, kv) == (args.bits, k):
                    continue
                if bits == args.bits:
                    vidx = index
                else:
                    if bits not in second:
                        second[bits] = vcb.TurboQuantIndex(args.dim, bits, device=local)
                        second[bits].calibrate_device(db[: args.calib])
                        second[bits].add_device(db)
                        second[bits].prepare()
                    vidx = second[bits]
                vs = torch.empty((args.nq, kv), dtype=torch.float32, device=device)
                vi = torch.empty((args.nq, kv), dtype=torch.int64, device=device)
                steps_v = max(2, min(args.steps, 3))
                ms = device_timed(lambda: vidx.search_device(q, kv, vs, vi, stream=stream), stream, steps_v, 3)
                variants.append({"bits": bits, "k": kv, "qps": args.nq / (ms / 1e3), "ms_per_step": ms,
                                 "steps": steps_v, "warmup": 3,
                                 "recall_at_10": recall_at(vi[:nr].cpu().numpy(), exact.cpu().numpy(), 10),
                                 "_top": (vs[:n_par].cpu().numpy(), vi[:n_par].cpu().numpy())})
        var_clocks = clk_var.summary()
        for v in variants:
            v["clocks"] = var_clocks
    del exact

    cpu_base = None
    parity = None
    ref_gpu = None
    if rank == 0 and keep_rows and not args.no_cpu_baseline:
        try:
            db_h = db.cpu().numpy()
            q_h = q.cpu().numpy()
            del db
            torch.cuda.empty_cache()
            if args.ref_gpu_queries > 0:
                try:
                    ref_gpu = reference_gpu_run(db_h, q_h, exact_np, args.dim, args.bits, k, args.ref_gpu_queries)
                except Exception as exc:  # reported, never required
                    ref_gpu = {"unavailable": f"{type(exc).__name__}: {exc}"}
            ref_idx, threads, build_s = reference_index(db_h, db_h[: args.calib], args.bits)
            qps = time_reference(ref_idx, q_h, k, args.cpu_queries, 2, 1)
            cpu_base = {"value": statistics.mean(qps), "unit": "queries/s", "cores": threads, "kind": "reference",
                        "sample": f"{args.cpu_queries} queries x 2 timed steps against the same "
                                  f"{args.n}x{args.dim} {args.bits}-bit TQ+ data, index built by the "
                                  f"reference's own encode/repack on the host ({build_s:.1f}s), avx2_perm0"}
            # Parity at the headline size: our codes and top-k against the
            # reference's own encode and search_flat of the same rows.
            qp = q_h[:n_par]
            parity = {"reference": "search_flat, avx2_perm0 backend (oracle/_ref)",
                      "codes": code_parity(ref_idx, index),
                      "device_search": search_parity(ref_idx, qp, k, *dev_top),
                      "host_abi_search": search_parity(ref_idx, qp, k, *e2e_top)}
            for v in variants:
                if v["bits"] == args.bits:
                    v["parity"] = search_parity(ref_idx, qp, v["k"], *v["_top"])
            ref_idx.close()
            for bits in sorted({v["bits"] for v in variants} - {args.bits}):
                ref2, _, _ = reference_index(db_h, db_h[: args.calib], bits)
                codes2 = code_parity(ref2, second[bits])
                for v in variants:
                    if v["bits"] == bits:
                        v["parity"] = dict(search_parity(ref2, qp, v["k"], *v["_top"]), codes=codes2)
                ref2.close()
        except Exception as exc:  # the baseline is reported, never required
            cpu_base = {"value": None, "unit": "queries/s", "cores": os.cpu_count(), "kind": "reference",
                        "sample": f"unavailable: {exc}"}
    for v in variants:
        v.pop("_top", None)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {
                "workload": f"flat TurboQuant search {args.n}x{args.dim} {args.bits}-bit TQ+, k={k}, "
                            f"{args.nq} queries per step",
                "n_per_gpu": args.n, "dim": args.dim, "bits": args.bits, "k": k, "nq": args.nq,
                "calibration_rows": args.calib, "recall_at_10": recall10,
                "recall_queries": nr, "l2": "inputs larger than L2 (codes %.0f MB per shard)"
                                           % (args.n * (nbg + 4) / 1e6),
                "parallelism": f"shard{world}" if world > 1 else "single",
                "scan_plan": plan,
                "encode_vectors_per_s": encode_vps, "prepare_ms": prepare_ms,
                "kernel_ms_per_step": {"prep": prof["prep_ms"] / args.steps, "scan": prof["scan_ms"] / args.steps,
                                       "merge": prof["merge_ms"] / args.steps},
                "nibble_lookups_per_s": lookups * args.steps / (prof["scan_ms"] / 1e3) if prof["scan_ms"] else None,
                "encode_kernel_ms": encode_kernels_ms,
                "encode_roofline": {"bytes": encode_bytes, "achieved_gbs": encode_bytes / (encode_kernels_ms / 1e3) / 1e9,
                                    "peak": peak, "frac": encode_bytes / (encode_kernels_ms / 1e3) / 1e9 / peak},
                "latency_ms": latency,
            },
            "roofline": {"kernel": "scan_kernel", "bound": "hbm", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": tr,
                         "bytes_per_launch": bytes_per_launch, "ms_per_launch": scan_ms_avg,
                         "share_of_kernel_time": prof["scan_ms"] / total_kernel_ms if total_kernel_ms else None,
                         "nibble_lookups_per_s": lookups * args.steps / (prof["scan_ms"] / 1e3)
                         if prof["scan_ms"] else None,
                         "one_query_pass": (dict(one_query, peak=peak, frac=one_query["achieved"] / peak)
                                            if one_query else None)},
            "cpu_baseline": cpu_base,
            "parity": parity,
            "variants": variants,
            "reference_gpu": ref_gpu,
            "e2e": {"value": e2e_value, "unit": "queries/s", "h2d_bytes_per_step": args.nq * args.dim * 4,
                    "d2h_bytes_per_step": args.nq * k * 12, "clocks": clk_e2e.summary()},
            "gpu_launches": prof["prep_launches"] + prof["scan_launches"] + prof["merge_launches"],
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    for extra in (second.values() if keep_rows and not args.no_variants else ()):
        extra.close()
    index.close()


BUCKETED_METRIC = "QPS at Recall@10 >= 0.95 (bucketed 1.2Mx100 4-bit cosine, learned n_probe vs fixed n_probe)"
# Candidate n_probe values of the learned probe below the fixed operating
# point (finer steps from 128 on: 1.48x -> 1.52x over the fixed n_probe in one
# call, mean 252 -> 245 probes at Recall@10 0.95), and above it: only 512, so
# the top-p selection still sorts 512 keys (1.52x as well; 512..768 cost
# 0.21 ms more per 10k queries in the selection for no gain).
PROBE_CLASSES = (1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 160, 192, 224, 256, 320, 352, 384, 416, 512,
                 768, 1024, 1536, 2048)
FIXED_PROBES = (64, 128, 256, 384, 512, 768, 1024, 1536, 2048)
FINE_STEP = 16  # fixed n_probe grid step below the first coarse point reaching the target
LEARNED_ABOVE = (512,)  # learned-probe classes above the fixed operating point
RECALL_TARGET = 0.95
BISECT_STEPS = 5  # trade-off bisection steps of the learned n_probe
# Prediction-rule sweeps of the learned n_probe, fewest buckets first:
# trade-offs (recall objective) and coverages (classes objective).
PROBE_RULES = {"recall": (0.3, 0.2, 0.15, 0.12, 0.1, 0.08, 0.06, 0.04, 0.03, 0.02, 0.015, 0.01, 0.005),
               "classes": (0.5, 0.7, 0.8, 0.9, 0.95, 0.98)}


def train_probe_mlp(idx, train_q, labels, rec, classes, objective, epochs, device, local, stream=None):
    """Routes the training queries, standardizes their features and trains the
    probe MLP on the GPU (batches of 512, Adam lr 2e-3) against label classes
    or per-class recall targets. Returns (model, mean loss of the last 50 steps)."""
    import torch

    from vectorcache_b200.probe import ProbeMLP

    mlp = ProbeMLP(classes=classes, hidden=128, layers=2, seed=17, device=local, objective=objective)
    d_train = torch.from_numpy(train_q).to(device)
    tr_s = torch.empty((train_q.shape[0], 256), dtype=torch.float32, device=device)
    tr_i = torch.empty((train_q.shape[0], 256), dtype=torch.int32, device=device)
    idx.route_device(d_train, 256, tr_s, tr_i, stream=stream)
    torch.cuda.synchronize()
    raw = mlp.features(tr_s.cpu().numpy())
    mlp.set_normalization(raw.mean(axis=0), raw.std(axis=0) + 1e-6)
    if objective == "recall":
        d_tgt = torch.from_numpy(np.ascontiguousarray(rec, np.float32)).to(device)
    else:
        d_tgt = torch.from_numpy(labels.astype(np.int32)).to(device)
    gen = torch.Generator(device=device)
    gen.manual_seed(5)
    losses = []
    for epoch in range(epochs):
        perm = torch.randperm(train_q.shape[0], device=device, generator=gen)
        for s in range(0, train_q.shape[0], 512):
            sel = perm[s:s + 512]
            losses.append(mlp.train_step_device(tr_s[sel].contiguous(), d_tgt[sel].contiguous(), sel.numel(), 256,
                                                2e-3, stream=stream))
    return mlp, float(np.mean(losses[-50:]))


def run_bucketed(args, world, rank, local):
    """The bucketed index workload: a von Mises-Fisher mixture (2000 clusters,
    kappa log-uniform in [20, 200], Zipf(1.1) sizes), dim 100, 4-bit, cosine;
    max_bucket_size 800, energy_soft 400, expected_n = corpus size. One step =
    one search of 10,000 queries (k = 10). The plain path scans the fixed
    n_probe = 64 best-routed buckets; the learned path routes, runs the probe
    MLP (trained here on the GPU on the recall at every candidate n_probe that
    the plain index reaches against exact top-10 for 50,000 training queries,
    or on label classes with --probe-objective classes) and scans each query's
    predicted number of buckets. Both re-rank their top `--rerank` candidates
    exactly."""
    import torch

    import vectorcache_b200 as vcb
    from vectorcache_b200.probe import probe_labels, recall_rows
    from vectorcache_b200.synthetic import vmf_mixture

    if world > 1:
        raise SystemExit("--workload bucketed runs on one GPU")
    device = torch.device("cuda", local)
    dim, n, nq, k = 100, args.bucketed_n, args.nq, 10
    t0 = time.perf_counter()
    db = vmf_mixture(n, dim, seed=31)
    test_q = vmf_mixture(nq, dim, seed=32)
    train_q = vmf_mixture(args.bucketed_train, dim, seed=33)
    gen_s = time.perf_counter() - t0
    params = vcb.BucketParams(n_probe=64, max_bucket_size=800, energy_soft=400, expected_n=n, rerank_k=args.rerank)
    idx = vcb.BucketedTurboQuantIndex(dim, 4, params, device=local)
    idx.add(db)
    t0 = time.perf_counter()
    idx.prepare()
    build_s = time.perf_counter() - t0
    info = idx.info()

    # exact top-10 (fp32 brute force on the normalized rows, no TF32)
    torch.backends.cuda.matmul.allow_tf32 = False
    x = torch.from_numpy(db).to(device)
    x = x / torch.linalg.vector_norm(x, dim=1, keepdim=True)

    def exact(q):
        out = []
        for s in range(0, q.shape[0], 4096):
            qq = torch.from_numpy(q[s:s + 4096]).to(device)
            qq = qq / torch.linalg.vector_norm(qq, dim=1, keepdim=True)
            out.append(torch.topk(qq @ x.T, k, dim=1).indices.cpu().numpy())
        return np.concatenate(out)

    ex_test, ex_train = exact(test_q), exact(train_q)
    del x
    torch.cuda.empty_cache()

    stream = torch.cuda.Stream(device=device)
    torch.cuda.set_stream(stream)
    d_q = torch.from_numpy(test_q).to(device)
    d_s = torch.empty((nq, k), dtype=torch.float32, device=device)
    d_i = torch.empty((nq, k), dtype=torch.int64, device=device)

    def timed(step_fn):
        for _ in range(args.warmup):
            step_fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step_fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    # The plain path at fixed n_probe: QPS and Recall@10 per n_probe; the
    # operating point is the smallest n_probe reaching the recall target,
    # found on a coarse grid and then in steps of 16 below the first coarse
    # point that reaches it.
    clk = ClockSampler(local).__enter__()
    sweep = {}

    def fixed_point(p):
        ms = timed(lambda: idx.search_device(d_q, k, d_s, d_i, n_probe=p, stream=stream))
        sweep[p] = {"n_probe": p, "ms_per_step": ms, "qps": nq / (ms / 1e3),
                    "recall_at_10": float(recall_rows(d_i.cpu().numpy(), ex_test, k).mean())}

    for p in ([args.bucketed_fixed_only] if args.bucketed_fixed_only else FIXED_PROBES):
        fixed_point(p)
    if args.bucketed_fixed_only:
        # the plain path at one n_probe only (profiling runs)
        clk.__exit__()
        print(json.dumps({"metric": BUCKETED_METRIC, "fixed_only": sweep[args.bucketed_fixed_only],
                          "clocks": clk.summary()}), flush=True)
        idx.close()
        return
    reach = [p for p in FIXED_PROBES if sweep[p]["recall_at_10"] >= RECALL_TARGET]
    p_coarse = reach[0] if reach else FIXED_PROBES[-1]
    below = [p for p in FIXED_PROBES if p < p_coarse]
    for p in range((below[-1] if below else 0) + FINE_STEP, p_coarse, FINE_STEP):
        fixed_point(p)
    grid = sorted(sweep)
    reach = [p for p in grid if sweep[p]["recall_at_10"] >= RECALL_TARGET]
    p_op = reach[0] if reach else p_coarse
    fixed = sweep[p_op]
    recall_fixed = fixed["recall_at_10"]
    fixed_ms = fixed["ms_per_step"]
    # Candidate n_probe values: the listed ones below the operating point, the
    # operating point itself, and a few above it, so that the recall objective
    # can spend more buckets on hard queries than the fixed path does.
    classes = learned_classes(args, p_op)
    p_max = classes[-1]

    # labels from the plain index (reference n_probe = the operating point) and GPU training
    t0 = time.perf_counter()
    labels, rec = probe_labels(lambda q, p: idx.search(q, k, n_probe=p).ids, train_q, ex_train, classes, k, p_op)
    label_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    objective = args.probe_objective
    mlp, final_loss = train_probe_mlp(idx, train_q, labels, rec, classes, objective, args.epochs, device, local,
                                      stream)
    train_s = time.perf_counter() - t0

    te_s = torch.empty((nq, 256), dtype=torch.float32, device=device)
    te_i = torch.empty((nq, 256), dtype=torch.int32, device=device)
    npq = torch.empty(nq, dtype=torch.int32, device=device)
    best = None
    learned_sweep = []
    target = min(RECALL_TARGET, recall_fixed)

    def learned_point(rule):
        nonlocal best

        def learned_step():
            # one routing pass feeds the network and the probes
            idx.search_learned_device(d_q, k, mlp, d_s, d_i, coverage=rule, min_confidence=0.0,
                                      fallback_n_probe=p_max, stream=stream)

        ms = timed(learned_step)
        r = float(recall_rows(d_i.cpu().numpy(), ex_test, k).mean())
        # the per-query probe counts of that search (recomputed outside the timed region)
        idx.route_device(d_q, 256, te_s, te_i, stream=stream)
        mlp.predict_device(te_s, nq, 256, npq, coverage=rule, min_confidence=0.0, fallback=p_max, stream=stream)
        mean_probe = float(npq.float().mean().item())
        counts = np.bincount(np.searchsorted(classes, npq.cpu().numpy()), minlength=len(classes))
        cand = {"rule": rule, "ms_per_step": ms, "qps": nq / (ms / 1e3), "recall_at_10": r,
                "mean_n_probe": mean_probe, "n_probe_histogram": counts.tolist()}
        learned_sweep.append(cand)
        if r >= target and (best is None or cand["qps"] > best["qps"]):
            best = cand
        return cand

    for rule in PROBE_RULES[objective]:
        learned_point(rule)
    # The recall falls as the trade-off grows: bisect between the largest grid
    # value that meets the target and the next larger one that misses it.
    meets = [c["rule"] for c in learned_sweep if c["recall_at_10"] >= target]
    misses = [c["rule"] for c in learned_sweep if c["recall_at_10"] < target]
    if meets and misses and objective == "recall":
        lo = max(meets)
        above = [r for r in misses if r > lo]
        if above:
            hi = min(above)
            for _ in range(BISECT_STEPS):
                mid = 0.5 * (lo + hi)
                if learned_point(mid)["recall_at_10"] >= target:
                    lo = mid
                else:
                    hi = mid
    qps_fixed = nq / (fixed_ms / 1e3)

    # Device time per kernel class of one search at each operating point.
    eng = idx.engine()

    def kernel_ms(step_fn):
        step_fn()
        torch.cuda.synchronize()
        eng.set_profiling(True)
        eng.read_profile()
        step_fn()
        torch.cuda.synchronize()
        prof = eng.read_profile()
        eng.set_profiling(False)
        return {"prep_route_pairs": prof["prep_ms"], "bucket_scan": prof["scan_ms"], "merge_rerank": prof["merge_ms"],
                "by_launch": {name: round(ms, 4) for name, (ms, _) in prof["by_launch"].items()}}

    fixed["kernel_ms"] = kernel_ms(lambda: idx.search_device(d_q, k, d_s, d_i, n_probe=p_op, stream=stream))
    if best:
        best["kernel_ms"] = kernel_ms(lambda: idx.search_learned_device(
            d_q, k, mlp, d_s, d_i, coverage=best["rule"], min_confidence=0.0, fallback_n_probe=p_max,
            stream=stream))
        # the plain path at the swept n_probe nearest the learned mean: what the
        # per-query counts cost beyond their mean
        near = min(sweep, key=lambda p: abs(p - best["mean_n_probe"]))
        sweep[near]["kernel_ms"] = kernel_ms(
            lambda: idx.search_device(d_q, k, d_s, d_i, n_probe=near, stream=stream))
    clk.__exit__()
    line = {
        "metric": BUCKETED_METRIC, "value": best["qps"] if best else None, "unit": "queries/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": f"bucketed TurboQuant {n}x{dim} 4-bit cosine vMF mixture, k={k}, {nq} queries per "
                               f"step, rerank {args.rerank}",
                   "n_buckets": info["n_buckets"], "n_slots": info["n_slots"], "build_s": build_s, "gen_s": gen_s,
                   "label_s": label_s, "train_s": train_s, "train_queries": train_q.shape[0],
                   "label_histogram": np.bincount(labels, minlength=len(classes)).tolist(),
                   "classes": list(classes), "final_loss": final_loss, "probe_objective": objective,
                   "recall_target": RECALL_TARGET},
        "fixed": fixed, "learned": best, "speedup_vs_fixed": (best["qps"] / qps_fixed) if best else None,
        "fixed_sweep": [sweep[p] for p in sorted(sweep)], "learned_sweep": learned_sweep,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    mlp.close()
    idx.close()


SERVING_RATES = (5_000, 20_000, 50_000, 100_000, 200_000)


def run_serving(args, world, rank, local):
    """Serving loop workload: a resident flat index (10M x 768, 3-bit, power-law
    vectors) plus the bucketed index of the bucketed workload (1.2M x 100 vMF,
    4-bit, re-rank 100) behind one server (HBM budget 120 GB, 4 slots,
    max_batch 1024). Requests arrive as a Poisson process in bursts of 1-256
    queries (k = 10 or 64 at equal odds; 1% of the queries go to the flat
    index); each rate is replayed open-loop twice: bucketed requests at the
    fixed n_probe that reaches Recall@10 >= 0.95, then with the learned probe.
    Reported per rate: p50/p99 latency, achieved QPS, bucketed Recall@10."""
    import torch

    import vectorcache_b200 as vcb
    from vectorcache_b200.probe import probe_labels, recall_rows
    from vectorcache_b200.synthetic import power_law_torch, vmf_mixture

    if world > 1:
        raise SystemExit("--workload serving runs on one GPU")
    device = torch.device("cuda", local)
    torch.backends.cuda.matmul.allow_tf32 = False
    t0 = time.perf_counter()
    flat_n, flat_dim = args.serving_flat_n, 768
    flat = vcb.TurboQuantIndex(flat_dim, 3, device=local)
    chunk = 1_000_000
    for s in range(0, flat_n, chunk):
        x = power_law_torch(min(chunk, flat_n - s), flat_dim, seed=2000 + s // chunk, device=device)
        if s == 0:
            flat.calibrate_device(x[:10_000])
        flat.add_device(x)
        del x
    flat.prepare()
    torch.cuda.empty_cache()
    flat_q = power_law_torch(2048, flat_dim, seed=77, device=device).cpu().numpy()
    flat_build_s = time.perf_counter() - t0

    dim, n, nq, k = 100, args.bucketed_n, args.nq, 10
    db = vmf_mixture(n, dim, seed=31)
    test_q = vmf_mixture(nq, dim, seed=32)
    train_q = vmf_mixture(args.bucketed_train, dim, seed=33)
    bkt = vcb.BucketedTurboQuantIndex(dim, 4, vcb.BucketParams(max_bucket_size=800, energy_soft=400, expected_n=n,
                                                               rerank_k=args.rerank), device=local)
    bkt.add(db)
    bkt.prepare()
    x = torch.from_numpy(db).to(device)

    def exact(q):
        out = []
        for s in range(0, q.shape[0], 4096):
            qq = torch.from_numpy(q[s:s + 4096]).to(device)
            out.append(torch.topk(qq @ x.T, k, dim=1).indices.cpu().numpy())
        return np.concatenate(out)

    ex_test, ex_train = exact(test_q), exact(train_q)
    del x
    torch.cuda.empty_cache()
    # fixed operating point: smallest n_probe with Recall@10 >= 0.95 (the
    # coarse grid, then steps of FINE_STEP below its first point reaching it)
    def fixed_recall(p):
        return recall_rows(bkt.search(test_q, k, n_probe=p).ids, ex_test, k).mean()

    p_op = FIXED_PROBES[-1]
    for p in FIXED_PROBES:
        if fixed_recall(p) >= RECALL_TARGET:
            p_op = p
            break
    below = [p for p in FIXED_PROBES if p < p_op]
    for p in range((below[-1] if below else 0) + FINE_STEP, p_op, FINE_STEP):
        if fixed_recall(p) >= RECALL_TARGET:
            p_op = p
            break
    classes = learned_classes(args, p_op)
    p_max = classes[-1]
    labels, rec = probe_labels(lambda q, p: bkt.search(q, k, n_probe=p).ids, train_q, ex_train, classes, k, p_op)
    objective = args.probe_objective
    mlp, _ = train_probe_mlp(bkt, train_q, labels, rec, classes, objective, args.epochs, device, local)
    # learned operating point: the rule with the fewest buckets whose Recall@10
    # reaches the target (grid, then bisection of the recall objective's trade-off)
    d_q = torch.from_numpy(test_q).to(device)
    d_s = torch.empty((nq, k), dtype=torch.float32, device=device)
    d_i = torch.empty((nq, k), dtype=torch.int64, device=device)

    def learned_recall(rule):
        bkt.search_learned_device(d_q, k, mlp, d_s, d_i, coverage=rule, fallback_n_probe=p_max)
        torch.cuda.synchronize()
        return recall_rows(d_i.cpu().numpy(), ex_test, k).mean()

    rules = PROBE_RULES[objective]
    cov_op, missed = rules[-1], None
    for rule in rules:
        if learned_recall(rule) >= RECALL_TARGET:
            cov_op = rule
            break
        missed = rule
    if objective == "recall" and missed is not None:
        lo, hi = cov_op, missed
        for _ in range(BISECT_STEPS):
            mid = 0.5 * (lo + hi)
            if learned_recall(mid) >= RECALL_TARGET:
                lo = mid
            else:
                hi = mid
        cov_op = lo

    srv = vcb.Server(device=local, hbm_budget_bytes=120 << 30, max_slots=4, max_batch=1024)
    t_flat = srv.add_flat(flat, 64)
    t_fixed = srv.add_bucketed(bkt, 64, p_op)
    t_learn = srv.add_bucketed(bkt, 64, p_max, mlp=mlp, coverage=cov_op)
    srv.start()
    info = srv.info()
    rng = np.random.default_rng(11)
    per_rate = []
    clk = ClockSampler(local).__enter__()
    for rate in SERVING_RATES:
        budget_q = min(40_000, int(rate * 2.0))
        t, base = 0.0, []
        total = 0
        while total < budget_q:
            nb_q = int(rng.integers(1, 257))
            t += rng.exponential(nb_q / rate * 1e6)
            kk = int(rng.choice([10, 64]))
            if rng.random() < 0.01:
                rows = rng.integers(0, flat_q.shape[0], nb_q)
                base.append((t, "flat", rows, kk))
            else:
                rows = rng.integers(0, nq, nb_q)
                base.append((t, "bkt", rows, kk))
            total += nb_q
        row = {"rate_qps": rate, "queries": total, "requests": len(base)}
        for mode, target in (("fixed", t_fixed), ("learned", t_learn)):
            # bucketed requests: the fixed n_probe, or the learned probe's own
            # largest class (a request's n_probe caps the learned counts)
            cap = p_op if mode == "fixed" else p_max
            trace = [(tt, t_flat if kind == "flat" else target, (flat_q if kind == "flat" else test_q)[rows], kk,
                      0 if kind == "flat" else cap) for tt, kind, rows, kk in base]
            lat, wall, results = srv.replay(trace)
            lat_ms = lat / 1e3
            is_b = np.array([kind == "bkt" for _, kind, _, _ in base])
            hits = tot = 0
            for (tt, kind, rows, kk), (s_, i_) in zip(base, results):
                if kind == "bkt":
                    hits += recall_rows(i_[:, :k], ex_test[rows], k).sum() * k
                    tot += rows.size * k
            row[mode] = {"qps": total / wall, "wall_s": wall, "p50_ms": float(np.percentile(lat_ms, 50)),
                         "p99_ms": float(np.percentile(lat_ms, 99)),
                         "bucketed_p50_ms": float(np.percentile(lat_ms[is_b], 50)),
                         "bucketed_p99_ms": float(np.percentile(lat_ms[is_b], 99)),
                         "flat_p99_ms": float(np.percentile(lat_ms[~is_b], 99)) if (~is_b).any() else None,
                         "bucketed_recall_at_10": hits / max(tot, 1)}
        per_rate.append(row)
    clk.__exit__()
    best = max(per_rate, key=lambda r: r["learned"]["qps"])
    line = {
        "metric": "serving QPS and p50/p99 latency (10Mx768 3-bit flat + 1.2Mx100 bucketed, Poisson bursts 1-256)",
        "value": best["learned"]["qps"], "unit": "queries/s", "n_gpus": 1, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": f"serving: flat {flat_n}x{flat_dim} 3-bit + bucketed {n}x{dim} 4-bit, HBM budget "
                               f"120 GB, rates {list(SERVING_RATES)} q/s", "slots": info["slots"],
                   "slot_bytes": info["slot_bytes"], "resident_bytes": info["resident_bytes"],
                   "fixed_n_probe": p_op, "learned_max_n_probe": p_max, "learned_rule": cov_op,
                   "probe_objective": objective, "flat_build_s": flat_build_s},
        "per_rate": per_rate, "server_stats": srv.stats(), "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    srv.close()
    mlp.close()
    bkt.close()
    flat.close()


def run_multi(args, world, rank, local):
    """Multi-index workload: 32 flat indexes with n log-uniform in [10k, 2M],
    dim in {128, 384, 768, 1536}, bits in {2, 3, 4} (power-law vectors at each
    dim), query batches log-uniform in [1, 4096], k in {10, 64}. One step =
    one search of every index's batch: (a) index by index on one stream, (b)
    the one persistent graph-captured multi-index launch (autotuned). Results
    of (b) are checked against (a) for every index."""
    import torch

    import vectorcache_b200 as vcb
    from vectorcache_b200.multi import MultiIndex
    from vectorcache_b200.synthetic import power_law_torch

    if world > 1:
        raise SystemExit("--workload multi runs on one GPU")
    device = torch.device("cuda", local)
    rng = np.random.default_rng(3)
    n_idx = 32
    specs = []
    for j in range(n_idx):
        n = int(np.exp(rng.uniform(np.log(1e4), np.log(2e6))))
        dim = int(rng.choice([128, 384, 768, 1536]))
        bits = int(rng.choice([2, 3, 4]))
        nq = int(np.exp(rng.uniform(0.0, np.log(4096))))
        k = int(rng.choice([10, 64]))
        specs.append((n, dim, bits, nq, k))
    t0 = time.perf_counter()
    idxs, queries = [], []
    for j, (n, dim, bits, nq, k) in enumerate(specs):
        idx = vcb.TurboQuantIndex(dim, bits, device=local)
        for s in range(0, n, 1 << 20):
            x = power_law_torch(min(1 << 20, n - s), dim, seed=5000 + 97 * j + s, device=device)
            idx.add_device(x)
            del x
        idx.prepare()
        idxs.append(idx)
        queries.append(power_law_torch(nq, dim, seed=9000 + j, device=device))
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    total_q = sum(s[3] for s in specs)
    stream = torch.cuda.Stream(device=device)
    torch.cuda.set_stream(stream)
    outs = [(torch.empty((s[3], s[4]), dtype=torch.float32, device=device),
             torch.empty((s[3], s[4]), dtype=torch.int64, device=device)) for s in specs]

    def seq_step():
        for idx, q, (o_s, o_i), s in zip(idxs, queries, outs, specs):
            idx.search_device(q, s[4], o_s, o_i, stream=stream)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    clk = ClockSampler(local).__enter__()
    seq_ms = timed(seq_step)
    multi = MultiIndex(idxs)
    t0 = time.perf_counter()
    multi.plan([s[3] for s in specs], [s[4] for s in specs], autotune=True)
    plan_s = time.perf_counter() - t0
    for j, q in enumerate(queries):
        multi.set_queries(j, q.cpu().numpy())
    multi_ms = timed(lambda: multi.launch(stream=stream))
    clk.__exit__()
    # exactness: every index's result equals its own search
    seq_step()
    torch.cuda.synchronize()
    exact = True
    for j, (o_s, o_i) in enumerate(outs):
        ms_, mi_ = multi.results(j)
        exact &= bool(np.array_equal(mi_, o_i.cpu().numpy().view(np.uint64)))
        exact &= bool(np.array_equal(ms_.view(np.uint32), o_s.cpu().numpy().view(np.uint32)))
    cfg = multi.config()
    multi.close()

    # The same 32 indexes with interactive-size batches (at most 16 queries
    # each): every separate search is latency-bound there, which is where one
    # persistent launch over all indexes pays.
    small = [min(s[3], 16) for s in specs]
    small_q = [q[:m] for q, m in zip(queries, small)]
    small_outs = [(o_s[:m], o_i[:m]) for (o_s, o_i), m in zip(outs, small)]

    def seq_small():
        for idx, q, (o_s, o_i), s in zip(idxs, small_q, small_outs, specs):
            idx.search_device(q, s[4], o_s, o_i, stream=stream)

    clk2 = ClockSampler(local).__enter__()
    seq_small_ms = timed(seq_small)
    multi2 = MultiIndex(idxs)
    multi2.plan(small, [s[4] for s in specs], autotune=True)
    for j, q in enumerate(small_q):
        multi2.set_queries(j, q.cpu().numpy())
    multi_small_ms = timed(lambda: multi2.launch(stream=stream))
    clk2.__exit__()
    seq_small()
    torch.cuda.synchronize()
    exact_small = True
    for j, (o_s, o_i) in enumerate(small_outs):
        ms_, mi_ = multi2.results(j)
        exact_small &= bool(np.array_equal(mi_, o_i.cpu().numpy().view(np.uint64)))
        exact_small &= bool(np.array_equal(ms_.view(np.uint32), o_s.cpu().numpy().view(np.uint32)))
    small_line = {"queries": sum(small), "per_index_sequential_ms": seq_small_ms, "multi_ms": multi_small_ms,
                  "qps": sum(small) / (multi_small_ms / 1e3), "speedup_vs_sequential": seq_small_ms / multi_small_ms,
                  "identical_to_per_index_search": exact_small, "autotuned": multi2.config(),
                  "clocks": clk2.summary()}
    multi2.close()
    line = {
        "metric": "multi-index QPS (32 flat indexes, uneven n/dim/bits/batches, one persistent graph launch)",
        "value": total_q / (multi_ms / 1e3), "unit": "queries/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": multi_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": "32 flat TurboQuant indexes: n log-uniform [1e4, 2e6], dim {128,384,768,1536}, "
                               "bits {2,3,4}, batches log-uniform [1, 4096], k {10,64}",
                   "indexes": [{"n": s[0], "dim": s[1], "bits": s[2], "nq": s[3], "k": s[4]} for s in specs],
                   "total_queries": total_q, "total_vectors": sum(s[0] for s in specs), "build_s": build_s,
                   "plan_and_autotune_s": plan_s, "autotuned": cfg},
        "per_index_sequential": {"ms_per_step": seq_ms, "qps": total_q / (seq_ms / 1e3)},
        "speedup_vs_sequential": seq_ms / multi_ms, "identical_to_per_index_search": exact,
        "clocks": clk.summary(), "small_batches": small_line,
    }
    print(json.dumps(line), flush=True)
    for idx in idxs:
        idx.close()


def run_encode(args, world, rank, local):
    """Encode workload: n x dim power-law rows (TQ+ calibrated on the first
    `--calib` rows) encoded into a fresh index per step (calibrate excluded):
    the encode kernel and the relayout into the scan layout. Reports encode
    vectors/s and the encode kernel's HBM roofline (rows read, codes and alpha
    written)."""
    import torch

    import vectorcache_b200 as vcb
    from vectorcache_b200.synthetic import power_law_torch

    if world > 1:
        raise SystemExit("--workload encode runs on one GPU")
    device = torch.device("cuda", local)
    db = power_law_torch(args.n, args.dim, seed=1000, device=device)
    torch.cuda.synchronize()
    nbg = args.dim // (8 // args.bits)
    peak, peak_kind = load_peaks()
    times = {"encode": [], "relayout": []}
    with ClockSampler(local) as clk:
        for step in range(args.warmup + args.steps):
            idx = vcb.TurboQuantIndex(args.dim, args.bits, device=local)
            idx.calibrate_device(db[: args.calib])
            idx.add_device(db)
            idx.set_profiling(True)
            idx.read_profile()
            idx.prepare()
            prof = idx.read_profile()
            if step >= args.warmup:
                times["encode"].append(prof["encode_ms"])
            idx.close()
    ms = statistics.mean(times["encode"])
    bytes_alg = args.n * (args.dim * 4 + nbg + 4)
    line = {
        "metric": "encode vectors/s", "value": args.n / (ms / 1e3), "unit": "vectors/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"encode {args.n}x{args.dim} {args.bits}-bit TQ+ (calibration on "
                               f"{args.calib} rows, excluded)", "n": args.n, "dim": args.dim, "bits": args.bits},
        "roofline": {"kernel": "encode + relayout", "bound": "hbm", "achieved": bytes_alg / (ms / 1e3) / 1e9,
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": bytes_alg / (ms / 1e3) / 1e9 / peak, "bytes_per_launch": bytes_alg},
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.workload == "encode":
        world, rank, local = dist_setup(args)
        run_encode(args, world, rank, local)
        return
    if args.workload == "multi":
        world, rank, local = dist_setup(args)
        run_multi(args, world, rank, local)
        return
    if args.workload == "bucketed":
        world, rank, local = dist_setup(args)
        run_bucketed(args, world, rank, local)
        return
    if args.workload == "serving":
        world, rank, local = dist_setup(args)
        run_serving(args, world, rank, local)
        return
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        if world > 1 and rank != 0:
            return
        if not (ROOT / "oracle" / "_ref" / "libtqref.so").exists():
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libtqref.so was not built"}))
            return
        run_reference(args, world, rank)
        return
    world, rank, local = dist_setup(args)
    try:
        run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
