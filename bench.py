#!/usr/bin/env python
"""SyN-CC throughput on the 3-D 182x218x182 workload (voxel-iterations per second).

One step = one complete SyN stage on one fixed/moving pair:
  SyN[0.1,3,0], CC radius 4, shrink 8x4x2x1, smoothing 3x2x1x0 vox, iterations 100x70x50x20,
  convergence [.., 1e-12, 10] (the fixed-schedule setting; the iterations actually run per level
  are counted from the stage log and reported).
A voxel-iteration is one voxel of a level grid processed by one full SyN iteration.

  value    -- inputs resident in HBM (device-to-device image upload, device field output), each
              level's iteration replayed as a CUDA graph, CUDA events on the stage's stream, L2
              flushed (256 MB write) between steps.
  e2e      -- the same stage through the C ABI with pinned host buffers: host->device images and
              device->host forward and inverse fields inside the timed region.
  roofline -- the dominant unit of the step: one full-resolution SyN iteration, replayed as one CUDA
              graph (warp, CC, xy and z smoothing, compose, and the two fixed-point inverses as
              conditional loops: 56 % of the step), timed with CUDA events on the stage's stream
              around the level inside the timed region and divided by its iterations.
              Algorithmic bytes = voxels x (176 B + inverse half-field sub-iterations x 36 B) per
              iteration, the compulsory traffic of each step (BYTES_PER_ITER_VOXEL below);
              `achieved_whole_step` applies the same model to all levels over the step time.
  --impl reference -- the CPU path (the oracle restatement of the reference arithmetic, all host
              threads) on the same workload: the K timed steps together run one complete registration,
              each advancing it by up to ceil(240 / K) SyN iterations.

Multi-GPU (torchrun): independent replicas, one pair per rank (no data-path collective);
value = voxel-iterations of all ranks / max over ranks of the timed region.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SyN-CC voxel-iters/s at 182x218x182"
UNIT = "voxel-iter/s"
SIZE = (182, 218, 182)
STAGE = dict(cc_radius=4, iterations=(100, 70, 50, 20), shrink_factors=(8, 4, 2, 1), smoothing_sigmas=(3.0, 2.0, 1.0, 0.0),
             learning_rate=0.1, update_variance=3.0, total_variance=0.0, convergence_threshold=1e-12,
             convergence_window=10)
WORKLOAD = ("3-D SyN[0.1,3,0] + CC[r=4], 182x218x182 at 1 mm, shrink 8x4x2x1, sigmas 3x2x1x0 vox, "
            "iterations 100x70x50x20, convergence [1e-12,10]")
# Compulsory (algorithmic) bytes of one 3-D SyN iteration per voxel, f32 fields of 12 B, every
# operand counted once per step:
#   warp both images + CC + derivatives: read 2 inverse half-fields, 2 image samples,
#     write 2 derivative fields                                                   4c + 8 =  56
#   smooth both update fields + max norm: read 2, write 2                          4c     =  48
#   scale + compose both halves: read 2 updates, read + write 2 half-fields        6c     =  72
# plus 3c = 36 B per voxel for each fixed-point inverse sub-iteration of one half-field
# (read psi, gather phi, write psi).
BYTES_PER_ITER_VOXEL = 176
BYTES_PER_INV_VOXEL = 36  # one fixed-point sub-iteration, one half-field voxel: read psi, gather phi, write psi
ROOF_LEVEL = 3  # the 182x218x182 level: one iteration graph per replay
# DRAM bytes (read + write) of one replay of that iteration graph, from the ncu capture summarised
# in profiles/iteration_graph_182x218x182.md (one pass per graph, every replay of two registrations)
ITER_GRAPH_TRAFFIC_BYTES = 2.665e9  # 1.607 GB read + 1.058 GB written (mean of 40 replays)


DATA = "synthetic: seeded layered-ellipsoid phantom pair, moving = fixed warped by a smooth field"


def workload_config(iterations_per_level, voxel_iterations, replicas_n):
    """The `config` object both arms print: the workload and what one registration of it ran."""
    return {"workload": WORKLOAD, "iterations_run_per_level": list(iterations_per_level),
            "voxel_iterations_per_registration": int(voxel_iterations), "l2": "flushed between steps (256 MB)",
            "parallelism": f"replicas x{replicas_n}"}


def dist_env():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed region.

    NVML is read every 20 ms from a host thread (read-only queries: current and maximum SM clock,
    active clock-event reasons), on the device matched by UUID, then PCI bus id.  Without NVML the
    sampler falls back to an `nvidia-smi -lms 200` process."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    PERIOD_S = 0.02
    # NVML clock-event reason bits
    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.out = None
        self.nvml = None
        self.handle = None
        self.thread = None
        self.stop = None
        self.rows = []  # (sm MHz, max sm MHz, reason bits)

    def _nvml_handle(self):
        import pynvml as N
        N.nvmlInit()
        self.nvml = N
        try:
            import torch
            p = torch.cuda.get_device_properties(self.index)
            try:
                return N.nvmlDeviceGetHandleByUUID("GPU-" + str(p.uuid))
            except Exception:
                bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
                return N.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return N.nvmlDeviceGetHandleByIndex(self.index)

    def _sample(self):
        N, h = self.nvml, self.handle
        while not self.stop.is_set():
            try:
                self.rows.append((float(N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)),
                                  float(N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)),
                                  int(N.nvmlDeviceGetCurrentClocksEventReasons(h))))
            except Exception:
                pass
            self.stop.wait(self.PERIOD_S)

    def __enter__(self):
        try:
            import threading
            self.handle = self._nvml_handle()
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._sample, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.handle = None
        try:
            self.out = open(os.path.join("/tmp", f"synx_clocks_{os.getpid()}.csv"), "w+")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        if self.thread is not None:
            sm = [r[0] for r in self.rows]
            reasons = sorted(n for n, bit in self.REASON_BITS.items() if any(r[2] & bit for r in self.rows))
            return {"sm_mhz": statistics.median(sm) if sm else None,
                    "sm_max_mhz": max(r[1] for r in self.rows) if self.rows else None,
                    "reasons": reasons, "samples": len(sm), "source": "nvml, 20 ms"}
        if self.out is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.out.seek(0)
        rows = [r.split(",") for r in self.out.read().strip().splitlines() if r.strip()]
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 200 ms"}


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def level_sizes(g):
    from ants_b200.synx import shrink_geom
    return [shrink_geom(g, f).count for f in STAGE["shrink_factors"]]


def voxel_iterations(log, sizes) -> int:
    return int(sum(sizes[r.level] for r in log))


# ---------------------------------------------------------------------------------------------
def cpu_sample(fixed, moving, g, threads: int, min_seconds: float = 0.0, max_iterations: int = 1):
    """Full-resolution SyN iterations of the CPU path (oracle restatement, `threads` host threads)
    from zero fields on the preprocessed, unsmoothed images (sigma = 0 at level 4): at least one,
    repeated until `min_seconds` have passed or `max_iterations` have run.  Returns
    (voxel-iterations per second, seconds, iterations)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from ants_b200.synx import SyNParams
    O.set_threads(threads)
    P = SyNParams(dim=3, **STAGE)
    Fp, Mp = O.preprocess(fixed), O.preprocess(moving)
    z = np.zeros((3,) + g.shape, np.float32)
    n, t0 = 0, time.perf_counter()
    while True:
        O.syn_iteration(Fp, g, Mp, g, P, g, z, z, z, z)
        n += 1
        dt = time.perf_counter() - t0
        if dt >= min_seconds or n >= max_iterations:
            break
    return g.count * n / dt, dt, n


SCHEDULE_MAX_ITERATIONS = sum(STAGE["iterations"])  # 240: the schedule's iterations without early stops


def run_reference(args, fixed, moving, g):
    """The CPU path on the same configuration as the device arm: the K timed steps together run ONE
    complete registration of the 182x218x182 pair with the full schedule (preprocessing, the four
    levels with their set-ups and the convergence monitor at 1e-12, the final composition).  Each
    step advances that registration by up to ceil(240 / K) SyN iterations (240 = the schedule's
    iterations without early stops), so the registration is complete within the K steps; steps left
    after it completes do nothing.  The W warm-up steps advance a separate registration the same way.
    value = voxel-iterations of the complete registration / the sum of the K step times, the same
    quantity the device arm reports per registration."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from ants_b200.synx import SyNParams
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    P = SyNParams(dim=3, **STAGE)
    per_step = -(-SCHEDULE_MAX_ITERATIONS // max(args.steps, 1))
    warm = O.SynRun(fixed, g, moving, g, P)
    for _ in range(args.warmup):
        warm.advance(per_step)
    warm.close()
    run = O.SynRun(fixed, g, moving, g, P)
    times, vox = [], 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        vox += run.advance(per_step)
        times.append(time.perf_counter() - t0)
    assert run.done, "the complete registration did not finish within the timed steps"
    levels = run.levels()
    run.close()
    total = sum(times)
    value = vox / total
    sample = (f"one complete registration of the workload split over the {args.steps} timed steps "
              f"(up to {per_step} SyN iterations per step); {threads} host threads, CPU restatement of the "
              f"reference arithmetic, {total:.1f} s")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": DATA, "config": workload_config([lv[2] for lv in levels], vox, 1),
            "cpu_level_seconds": [round(lv[1], 3) for lv in levels],
            "cpu_level_voxel_iterations": [lv[0] for lv in levels],
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
BATCH_PAIRS = 32
BATCH_STAGE = dict(cc_radius=4, iterations=(50, 30, 15), shrink_factors=(4, 2, 1), smoothing_sigmas=(2.0, 1.0, 0.0),
                   learning_rate=0.1, update_variance=3.0, total_variance=0.0, convergence_threshold=1e-12,
                   convergence_window=10)
BATCH_WORKLOAD = ("32 independent 3-D phantom pairs, per-axis dims U{96..192} (seeded), SyN[0.1,3,0] + CC[r=4], "
                  "shrink 4x2x1, sigmas 2x1x0 vox, iterations 50x30x15, convergence [1e-12,10]")


def batch_dims(k: int):
    rng = np.random.default_rng(0x5EED0000 + 1000 + k)
    return tuple(int(x) for x in rng.integers(96, 193, size=3))


def _batch_pair(k: int):
    from ants_b200 import phantoms
    return phantoms.pair_3d(batch_dims(k), seed=0x5EED0000 + 1000 + k)


def run_batched(args) -> int:
    """32 pairs: all advanced together through synx_batch_* (one step = every pair's next level,
    the small levels of all pairs in shared cooperative launches) vs the same pairs one after the
    other through the plain single-pair path.  One timed step = all 32 pairs registered, device
    inputs, fields to device memory; contexts are created (and their arenas allocated) before
    the timed region in both arms."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    ws, rank, local = dist_env()
    # generate the phantoms in spawned worker processes before any GPU work
    with ProcessPoolExecutor(max_workers=min(16, os.cpu_count() or 1), mp_context=mp.get_context("spawn")) as ex:
        pairs = list(ex.map(_batch_pair, [rank * BATCH_PAIRS + k for k in range(BATCH_PAIRS)]))
    import torch
    from ants_b200 import replicas
    from ants_b200 import synx as S

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    geoms = [S.Geom(f.shape[::-1]) for f, _ in pairs]
    dev_pairs = [(torch.from_numpy(np.ascontiguousarray(f)).to(dev), torch.from_numpy(np.ascontiguousarray(m)).to(dev))
                 for f, m in pairs]
    outs = [(torch.empty((3,) + g.shape, device=dev), torch.empty((3,) + g.shape, device=dev)) for g in geoms]
    # both arms replay their per-kernel levels from CUDA graphs (the faster single-pair setting)
    P = S.SyNParams(dim=3, flags=S.SYNX_F_USE_GRAPHS, **BATCH_STAGE)
    seq = [S.SyNStage(P, device=local, stream=stream.cuda_stream) for _ in range(BATCH_PAIRS)]
    bat = [S.SyNStage(P, device=local, stream=stream.cuda_stream) for _ in range(BATCH_PAIRS)]
    batch = S.Batch(local)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def sequential():
        for st, (f, m), g, (a, b) in zip(seq, dev_pairs, geoms, outs):
            st.set_images(f, g, m, g)
            st.run()
            st.fields_device(a, b)

    def batched():
        for st, (f, m), g in zip(bat, dev_pairs, geoms):
            st.set_images(f, g, m, g)
        batch.run(bat, stream.cuda_stream)
        for st, (a, b) in zip(bat, outs):
            st.fields_device(a, b)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ms = []
        for k in range(args.steps):
            flush.fill_(float(k))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return sum(ms) / 1000.0

    launches0 = S.launch_count()
    with ClockSampler(local) as clk:
        t_bat = timed(batched)
    launches = (S.launch_count() - launches0) // max(args.warmup + args.steps, 1) * args.steps
    for st in seq:
        st.reset_profile()
    t_seq = timed(sequential)
    # the sequential arm's time per pyramid level (all pairs, per step): what batching can remove is
    # bounded by the share of the levels whose launches leave the GPU idle
    seq_level_ms = [0.0] * len(BATCH_STAGE["iterations"])
    for st in seq:
        for lv in st.level_profile():
            seq_level_ms[lv["level"]] += lv["iterate_ms"] / (args.warmup + args.steps)
    # the two arms compute the same fields (each pair's result does not depend on the batch)
    same = all(bool(torch.equal(torch.from_numpy(x.fields()[0]), torch.from_numpy(y.fields()[0])))
               for x, y in zip(seq, bat))
    vi = 0
    for st, g in zip(bat, geoms):
        sizes = [S.shrink_geom(g, f).count for f in BATCH_STAGE["shrink_factors"]]
        vi += sum(sizes[r.level] for r in st.log())
    t_bat_all, n_all = replicas.aggregate(t_bat, BATCH_PAIRS * args.steps, dev)
    t_seq_all, _ = replicas.aggregate(t_seq, BATCH_PAIRS * args.steps, dev)
    if rank == 0:
        pph = n_all / t_bat_all * 3600.0
        pph_seq = n_all / t_seq_all * 3600.0
        line = {"metric": "batched pairs/hour (32 pairs, 3-D, dims U{96..192})", "value": pph, "unit": "pairs/h",
                "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1000.0 * t_bat_all / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32",
                "data": "synthetic: seeded layered-ellipsoid phantom pairs, moving = fixed warped by a smooth field",
                "config": {"workload": BATCH_WORKLOAD, "pairs_per_step": BATCH_PAIRS,
                           "dims": [list(g.size) for g in geoms], "voxel_iterations_per_step": vi,
                           "l2": "flushed between steps (256 MB)", "parallelism": f"replicas x{ws}",
                           "sequential_pairs_per_hour": pph_seq, "speedup_vs_sequential": pph / pph_seq,
                           "sequential_ms_per_step": 1000.0 * t_seq_all / args.steps,
                           "sequential_level_ms_per_step": [round(x, 2) for x in seq_level_ms],
                           "fields_identical_to_sequential": same},
                "clocks": clk.summary(), "gpu_launches": int(launches)}
        print(json.dumps(line), flush=True)
    for st in seq + bat:
        st.close()
    batch.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------------------------
# Serving mix: (dimension, size, weight); 3-level schedule, CC r=2 (2-D) / r=4 (3-D)
SERVE_MIX = [(2, (256, 256), 0.3), (2, (512, 512), 0.1), (3, (128, 128, 128), 0.3), (3, (182, 218, 182), 0.2),
             (3, (256, 256, 256), 0.1)]
SERVE_STAGE = dict(iterations=(40, 20, 10), shrink_factors=(4, 2, 1), smoothing_sigmas=(2.0, 1.0, 0.0),
                   learning_rate=0.1, update_variance=3.0, total_variance=0.0, convergence_threshold=1e-12,
                   convergence_window=10)
SERVE_POOL = 2  # distinct seeded pairs per size class (requests reuse them)


def _serve_pair(job):
    from ants_b200 import phantoms
    cls, k = job
    dim, size, _ = SERVE_MIX[cls]
    seed = 0x5EED0000 + 2000 + 10 * cls + k
    return phantoms.pair_2d(size, seed=seed) if dim == 2 else phantoms.pair_3d(size, seed=seed)


def run_serving(args) -> int:
    """Poisson arrivals of registration requests (the 2-D/3-D mix above) into the serving loop
    (synx_server_*): continuous batching, admission by device footprint, every resident request
    advanced one level per step.  Latency = completion - submission on the server's clock; one
    rate after another on the same server."""
    import multiprocessing as mp
    import threading
    from concurrent.futures import ProcessPoolExecutor

    ws, rank, local = dist_env()
    jobs = [(c, k) for c in range(len(SERVE_MIX)) for k in range(SERVE_POOL)]
    with ProcessPoolExecutor(max_workers=min(16, os.cpu_count() or 1), mp_context=mp.get_context("spawn")) as ex:
        pool = dict(zip(jobs, ex.map(_serve_pair, jobs)))
    import torch
    from ants_b200 import synx as S

    # pinned host memory for request inputs and results (as a serving front end would hold them)
    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.float32, pin_memory=True)
        t.numpy()[...] = a
        return t.numpy()

    pool = {k: (pinned(f), pinned(m)) for k, (f, m) in pool.items()}
    outs = {}
    for c, (d, size, _) in enumerate(SERVE_MIX):
        shp = tuple(reversed(size)) + (d,)
        outs[c] = [(torch.empty(shp, pin_memory=True).numpy(), torch.empty(shp, pin_memory=True).numpy())
                   for _ in range(4)]
    out_next = {c: 0 for c in outs}

    rates = [float(x) for x in args.rates.split(",") if x]
    rng = np.random.default_rng(0x5EED0000 + 3000 + rank)
    weights = np.array([w for _, _, w in SERVE_MIX])
    params = {d: S.SyNParams(dim=d, cc_radius=2 if d == 2 else 4, **SERVE_STAGE) for d in (2, 3)}
    geoms = [S.Geom(size) for _, size, _ in SERVE_MIX]
    srv = S.Server(local)

    def request(cls, k):
        f, m = pool[(cls, k)]
        o = outs[cls][out_next[cls] % len(outs[cls])]  # results are not inspected; buffers rotate
        out_next[cls] += 1
        return srv.submit(params[SERVE_MIX[cls][0]], f, geoms[cls], m, geoms[cls], out=o)

    # service time of each class alone (also warms every code path)
    alone_ms = []
    for cls in range(len(SERVE_MIX)):
        for _ in range(2):
            _, _, info = srv.wait(request(cls, 0), timeout=600)
        alone_ms.append(round(1000.0 * (info["t_done"] - info["t_submit"]), 2))
    launches0 = S.launch_count()
    per_rate = []
    with ClockSampler(local) as clk:
        for lam in rates:
            n = int(min(60, max(8, round(lam * args.window))))
            classes = rng.choice(len(SERVE_MIX), size=n, p=weights)
            gaps = rng.exponential(1.0 / lam, size=n)
            st0 = srv.stats()
            ids, results = [], {}

            def collect():
                for i in range(n):
                    while len(ids) <= i:
                        time.sleep(0.0005)
                    results[i] = srv.wait(ids[i], timeout=900)[2]

            th = threading.Thread(target=collect)
            th.start()
            t_next = time.perf_counter()
            for i in range(n):
                t_next += gaps[i]
                d = t_next - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                ids.append(request(int(classes[i]), i % SERVE_POOL))
            th.join()
            st1 = srv.stats()
            lat = np.array([1000.0 * (results[i]["t_done"] - results[i]["t_submit"]) for i in range(n)])
            wait_q = np.array([1000.0 * (results[i]["t_admit"] - results[i]["t_submit"]) for i in range(n)])
            span = max(r["t_done"] for r in results.values()) - min(r["t_submit"] for r in results.values())
            occ = (st1["resident_byte_seconds"] - st0["resident_byte_seconds"]) / max(st1["elapsed"] - st0["elapsed"], 1e-9)
            per_rate.append({"rate_per_s": lam, "requests": n, "p50_ms": float(np.percentile(lat, 50)),
                             "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
                             "p99_admission_wait_ms": float(np.percentile(wait_q, 99)),
                             "pairs_per_hour": n / span * 3600.0,
                             "hbm_mean_resident_gb": occ / 1e9, "hbm_peak_resident_gb": st1["bytes_peak"] / 1e9,
                             "steps": st1["steps"] - st0["steps"],
                             "mix_counts": [int((classes == c).sum()) for c in range(len(SERVE_MIX))]})
    launches = S.launch_count() - launches0
    stats = srv.stats()
    srv.close()
    if rank == 0:
        top = per_rate[-1]
        line = {"metric": "serving p50/p99 latency (Poisson arrivals, 2-D/3-D mix)", "value": top["p99_ms"],
                "unit": "ms (p99 at the highest rate)", "n_gpus": ws, "steps": len(rates), "warmup": len(SERVE_MIX) * 2,
                "ms_per_step": None, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic: seeded phantom pairs (2 per size class, reused by requests)",
                "config": {"workload": "mix 2-D 256^2 (0.3) / 512^2 (0.1), 3-D 128^3 (0.3) / 182x218x182 (0.2) / "
                                       "256^3 (0.1); CC r=2 (2-D) / r=4 (3-D); SyN[0.1,3,0], f 4x2x1, s 2x1x0 vox, "
                                       "c 40x20x10 [1e-12,10]",
                           "hbm_budget_gb": stats["budget"] / 1e9, "alone_service_ms_per_class": alone_ms,
                           "per_rate": per_rate},
                "clocks": clk.summary(), "gpu_launches": int(launches)}
        print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------------
PREC_SIZE = (256, 256, 256)
PREC_SPACING = (0.7, 0.7, 0.7)
PREC_STAGE = dict(cc_radius=5, iterations=(70, 50, 20), shrink_factors=(4, 2, 1), smoothing_sigmas=(2.0, 1.0, 0.0),
                  learning_rate=0.1, update_variance=3.0, total_variance=0.0, convergence_threshold=1e-12,
                  convergence_window=10)


def _twelve_bit(a):
    a = a.astype(np.float64)
    return ((a - a.min()) / (a.max() - a.min()) * 4095.0).astype(np.float32)


def run_precision(args) -> int:
    """Precision study on a 256^3 pair at 0.7 mm with intensities in [0, 4095] (CC r=5):
    step level, the CC value and derivative fields with window sums in double (default) and in
    float, on the raw 12-bit intensities and after antsRegistration's [0,1] rescaling; the other
    steps (warp, update smoothing, compose, inverse) in float against the double oracle; end to
    end, the final fields of each variant (double or float CC sums, float or half-precision field
    storage) against the double-precision oracle registration, with each variant's throughput."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from ants_b200 import phantoms

    f, m = phantoms.pair_3d(PREC_SIZE, seed=0x5EED0000 + 4000)
    f, m = _twelve_bit(f), _twelve_bit(m)
    import torch
    from ants_b200 import synx as S

    O.set_threads(os.cpu_count() or 1)
    g = S.Geom(PREC_SIZE, spacing=PREC_SPACING)
    dev = torch.device("cuda", 0)
    out = {"workload": "256^3 at 0.7 mm, layered-ellipsoid phantom pair scaled to [0,4095], CC r=5, SyN[0.1,3,0], "
                       "f 4x2x1, s 2x1x0 vox, c 70x50x20 [1e-12,10]", "host_threads": os.cpu_count()}

    def rel_rms(a, b):
        return float(np.sqrt(((a - b) ** 2).mean() / max((b ** 2).mean(), 1e-300)))

    def event_ms(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        b.synchronize()
        return a.elapsed_time(b) / reps

    # ---- step level: CC ----
    cc_rows = []
    fp, mp = O.preprocess(f, dtype=np.float64).astype(np.float32), O.preprocess(m, dtype=np.float64).astype(np.float32)
    for label, (a, b) in (("raw 12-bit", (f, m)), ("rescaled to [0,1]", (fp, mp))):
        t0 = time.perf_counter()
        v64, gF64, gM64, _ = O.cc_metric(a, b, g, 5, dtype=np.float64)
        t_or = time.perf_counter() - t0
        A, B = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
        gF = torch.empty((3,) + g.shape, device=dev)
        gM = torch.empty_like(gF)
        for fp32 in (False, True):
            v = S.cc_metric(A, B, g, 5, gF, gM, fp32_sums=fp32)
            hF, hM = gF.cpu().numpy(), gM.cpu().numpy()
            ms = event_ms(lambda: S.cc_metric(A, B, g, 5, gF, gM, fp32_sums=fp32))
            cc_rows.append({"data": label, "window_sums": "float" if fp32 else "double",
                            "metric_abs_err": abs(v - v64), "metric": v, "metric_fp64_oracle": v64,
                            "grad_rel_rms_err": max(rel_rms(hF, gF64), rel_rms(hM, gM64)),
                            "grad_max_abs_err": float(max(np.abs(hF - gF64).max(), np.abs(hM - gM64).max())),
                            "ms_per_call": ms, "oracle_fp64_s": t_or})
    out["cc_step"] = cc_rows

    # ---- step level: the float steps against the double oracle ----
    rng = np.random.default_rng(0x5EED0000 + 4001)
    u = np.moveaxis(phantoms.smooth_field(g.shape, 8.0, 4.0, rng), -1, 0).astype(np.float32).copy()
    w = np.moveaxis(phantoms.smooth_field(g.shape, 10.0, 5.0, rng), -1, 0).astype(np.float32).copy()
    U, W = torch.from_numpy(u).to(dev), torch.from_numpy(w).to(dev)
    steps = {}
    Fp = torch.from_numpy(fp).to(dev)
    o1 = torch.empty(g.shape, device=dev)
    S.warp_image(Fp, g, U, g, o1)
    ref = O.warp_image(fp, g, u, g, dtype=np.float64)
    h = o1.cpu().numpy()
    steps["warp"] = {"max_abs_err": float(np.abs(h - ref).max()), "rel_rms_err": rel_rms(h, ref)}
    o3 = torch.empty_like(U)
    S.smooth_field(U, o3, g, 3.0)
    ref = O.smooth_field(u, g, 3.0, dtype=np.float64)
    h = o3.cpu().numpy()
    steps["update_smoothing"] = {"max_abs_err": float(np.abs(h - ref).max()), "rel_rms_err": rel_rms(h, ref)}
    S.compose(U, W, g, o3)
    ref = O.compose(u, w, g, dtype=np.float64)
    h = o3.cpu().numpy()
    steps["compose"] = {"max_abs_err": float(np.abs(h - ref).max()), "rel_rms_err": rel_rms(h, ref)}
    psi = torch.zeros_like(W)
    it = S.invert_field(W, psi, g)
    ref, it_ref, _, _ = O.invert(w, np.zeros_like(w), g, dtype=np.float64)
    h = psi.cpu().numpy()
    steps["inverse"] = {"max_abs_err": float(np.abs(h - ref).max()), "rel_rms_err": rel_rms(h, ref),
                        "iterations": it, "iterations_fp64": it_ref}
    out["float_steps_vs_fp64_oracle"] = steps

    # ---- end to end ----
    sizes = [S.shrink_geom(g, k).count for k in PREC_STAGE["shrink_factors"]]
    Fd, Md = torch.from_numpy(f).to(dev), torch.from_numpy(m).to(dev)

    def e2e(preprocess, flags):
        P = S.SyNParams(dim=3, preprocess=preprocess, flags=flags, **PREC_STAGE)
        st = S.SyNStage(P)
        st.set_images(Fd, g, Md, g)
        st.run()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        st.set_images(Fd, g, Md, g)
        st.run()
        b.record()
        b.synchronize()
        fw, iv = st.fields()
        vi = sum(sizes[r.level] for r in st.log())
        res = (np.moveaxis(fw, -1, 0).copy(), np.moveaxis(iv, -1, 0).copy(), vi / (a.elapsed_time(b) / 1e3),
               [r.metric for r in st.log()][-1])
        st.close()
        return res

    def rms_vox(a, b):
        sp = np.asarray(PREC_SPACING).reshape(3, 1, 1, 1)
        return float(np.sqrt((((a - b) / sp) ** 2).sum(0).mean()))

    variants = [("double CC sums, float fields (default)", S.SYNX_F_USE_GRAPHS),
                ("float CC sums", S.SYNX_F_USE_GRAPHS | S.SYNX_F_CC_FP32_SUMS),
                ("half-precision field storage", S.SYNX_F_USE_GRAPHS | S.SYNX_F_FIELDS_FP16),
                ("float CC sums + half-precision fields",
                 S.SYNX_F_USE_GRAPHS | S.SYNX_F_CC_FP32_SUMS | S.SYNX_F_FIELDS_FP16)]
    rows = []
    for preprocess, vlist in ((True, variants), (False, variants[:2])):
        P = S.SyNParams(dim=3, preprocess=preprocess, **PREC_STAGE)
        t0 = time.perf_counter()
        rf, ri, _, rlog = O.syn_register(f, g, m, g, P, dtype=np.float64)
        t_or = time.perf_counter() - t0
        for name, flags in vlist:
            fw, iv, vis, last = e2e(preprocess, flags)
            rows.append({"intensities": "rescaled to [0,1] (antsRegistration)" if preprocess else "raw 12-bit",
                         "variant": name, "forward_rms_vox_vs_fp64": rms_vox(fw, rf),
                         "inverse_rms_vox_vs_fp64": rms_vox(iv, ri), "final_metric": last,
                         "final_metric_fp64": rlog[-1]["metric"], "voxel_iter_per_s": vis,
                         "oracle_fp64_s": t_or})
    out["end_to_end"] = rows
    line = {"metric": "precision study (error vs FP64 oracle, per variant)", "value": rows[0]["forward_rms_vox_vs_fp64"],
            "unit": "voxel RMS (default variant, forward field)", "n_gpus": 1, "steps": 1, "warmup": 1,
            "higher_is_better": False, "dtype": "f32", "data": "synthetic: seeded phantom pair",
            "config": out}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------------
APPLY_BYTES_PER_VOXEL = 20  # field 12 B + output 4 B + one sample of the input 4 B


def run_apply(args) -> int:
    """antsApplyTransforms through the standard stack `-t 1Warp.nii.gz -t 0GenericAffine.mat` onto a
    182x218x182 reference grid.  The command line's scheme for this stack is one warp of the input
    through the field, with the affine folded into the input's geometry (synx_warp_image), so a step
    is that warp.  value = reference voxels per second with inputs resident (CUDA events on the
    launching stream, L2 flushed between steps); e2e = the same with the input image and the field
    copied host->device and the output device->host inside each timed step; roofline = the warp,
    20 B per voxel (field 12, output 4, one input sample 4); cpu_baseline = the oracle's warp on all
    host threads; the device output is checked against it."""
    import torch
    from ants_b200 import phantoms
    from ants_b200 import synx as S

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    g = S.Geom(SIZE)                                        # the reference (fixed) grid, 1 mm
    gi = S.Geom(SIZE, (1.0, 1.0, 1.0), (-2.0, 1.5, -1.0))   # the input (moving) image's own grid
    rng = np.random.default_rng(0x5EED0000 + 5000)
    _, moving = phantoms.pair_3d(SIZE, seed=0x5EED0000 + 5001)
    img = np.ascontiguousarray(moving, dtype=np.float32)
    u = np.ascontiguousarray(np.moveaxis(phantoms.smooth_field(g.shape, 8.0, 3.0, rng), -1, 0).astype(np.float32))
    A = S.LinearTransform(np.array([[1.02, 0.03, -0.01], [-0.02, 0.98, 0.02], [0.01, -0.015, 1.01]]),
                          np.array([1.5, -2.0, 0.75]), np.array([91.0, 109.0, 91.0]))
    gi_fold = S.fold_moving_geometry(gi, A)  # sampling at q reads the input at A(q)
    N = g.count
    Id, Ud = torch.from_numpy(img).to(dev), torch.from_numpy(u).to(dev)
    out = torch.empty(g.shape, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2
    stream = torch.cuda.current_stream()

    def step():
        S.warp_image(Id, gi_fold, Ud, g, out, stream=stream.cuda_stream)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    launches0 = S.launch_count()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(0) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))
            evs[k][0].record(stream)
            step()
            evs[k][1].record(stream)
        torch.cuda.synchronize()
    launches = S.launch_count() - launches0
    ms = [a.elapsed_time(b) for a, b in evs]
    t = sum(ms) / 1000.0
    value = N * args.steps / t
    got = out.cpu().numpy()

    # end to end: host input image and field in, warped image out, every step
    img_h = torch.from_numpy(img).pin_memory()
    u_h = torch.from_numpy(u).pin_memory()
    out_h = torch.empty(g.shape, dtype=torch.float32).pin_memory()
    e2e_ms = []
    for k in range(args.steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        Id.copy_(img_h, non_blocking=True)
        Ud.copy_(u_h, non_blocking=True)
        step()
        out_h.copy_(out, non_blocking=True)
        b.record(stream)
        b.synchronize()
        e2e_ms.append(a.elapsed_time(b))
    t_e2e = sum(e2e_ms) / 1000.0

    peak, peak_kind = measured_peak_hbm()
    achieved = APPLY_BYTES_PER_VOXEL * N / (t / args.steps) / 1e9
    cpu, mismatch = None, None
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        threads = os.cpu_count() or 1
        O.set_threads(threads)
        n_cpu, t0 = 0, time.perf_counter()
        while True:
            ref = O.warp_image(img, gi_fold, u, g)
            n_cpu += 1
            dt = time.perf_counter() - t0
            if dt >= 5.0 or n_cpu >= 50:
                break
        cpu = {"value": N * n_cpu / dt, "unit": "voxel/s", "cores": threads, "kind": "port",
               "sample": f"{n_cpu} warps of the 182x218x182 workload by the oracle ({dt:.1f} s of CPU work)"}
        mismatch = float((np.abs(got - ref) > 1e-5).mean())
    line = {"metric": "antsApplyTransforms voxels/s (182x218x182, -t warp -t affine)", "value": value,
            "unit": "voxel/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3),
            "ms_per_step": 1000.0 * t / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic: seeded phantom image, smooth field, fixed affine",
            "config": {"workload": "warp of a 182x218x182 image through a displacement field and an affine "
                                   "(folded into the input geometry), linear interpolation",
                       "l2": "flushed between steps (256 MB)", "parity_mismatch_fraction_vs_oracle": mismatch},
            "e2e": {"value": N * args.steps / t_e2e, "unit": "voxel/s", "h2d_bytes_per_step": int(img.nbytes + u.nbytes),
                    "d2h_bytes_per_step": int(N * 4), "ms_per_step": 1000.0 * t_e2e / args.steps},
            "roofline": {"kernel": "k_warp_image<3>", "bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind, "traffic": None,
                         "algorithmic_bytes_per_launch": APPLY_BYTES_PER_VOXEL * N,
                         "launch_ms": t / args.steps * 1000.0},
            "cpu_baseline": cpu, "clocks": clk.summary(), "gpu_launches": int(launches)}
    print(json.dumps(line), flush=True)
    return 0


def run_kernels(args) -> int:
    """Each full-resolution step of a SyN iteration once per step through the C ABI, on the
    182x218x182 phantom pair and a smooth synthetic field (about 3 voxels at most): image warp, CC
    value + both update directions (r = 4), update smoothing (variance 3 voxels^2), composition, and
    a field inversion from a zero start.  Few launches and a few hundred MB on the device, so a
    profiler capture of one of these kernels stays short.  Prints one JSON line with the mean time
    of each call (CUDA events on the launching stream around the call, L2 flushed before each; the
    calls that return a value or allocate scratch synchronise inside, which the times include)."""
    import torch
    from ants_b200 import phantoms, replicas
    from ants_b200 import synx as S

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    g = S.Geom(SIZE)
    N = g.count
    fixed, moving = phantoms.pair_3d(SIZE, seed=replicas.pair_seed(0))
    rng = np.random.default_rng(0x5EED0000 + 6000)
    u = np.ascontiguousarray(np.moveaxis(phantoms.smooth_field(g.shape, 6.0, 3.0, rng), -1, 0).astype(np.float32))
    F, M = torch.from_numpy(fixed).to(dev), torch.from_numpy(moving).to(dev)
    U = torch.from_numpy(u).to(dev)
    W = 0.5 * U
    out1 = torch.empty(g.shape, device=dev)
    gF, gM, out3 = (torch.empty((3,) + g.shape, device=dev) for _ in range(3))
    psi = torch.zeros_like(U)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2
    stream = torch.cuda.current_stream()
    calls = {
        "warp_image": (lambda: S.warp_image(F, g, U, g, out1, stream=stream.cuda_stream), 20),
        "cc_metric_r4": (lambda: S.cc_metric(F, M, g, 4, gF, gM, stream=stream.cuda_stream), 32),
        "smooth_field_var3": (lambda: S.smooth_field(U, out3, g, 3.0, stream=stream.cuda_stream), 48),
        "compose": (lambda: S.compose(U, W, g, out3, 0.5, stream=stream.cuda_stream), 72),
        "invert_field": (lambda: (psi.zero_(), S.invert_field(U, psi, g, stream=stream.cuda_stream)), None),
    }
    for _ in range(max(args.warmup, 0)):
        for fn, _b in calls.values():
            fn()
    torch.cuda.synchronize()
    launches0 = S.launch_count()
    res = {}
    with ClockSampler(0) as clk:
        for name, (fn, bytes_per_voxel) in calls.items():
            ms = []
            for k in range(args.steps):
                flush.fill_(float(k))
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                fn()
                b.record(stream)
                b.synchronize()
                ms.append(a.elapsed_time(b))
            t = sum(ms) / len(ms)
            res[name] = {"call_us": 1000.0 * t}
            if bytes_per_voxel:
                res[name]["algorithmic_gbs"] = bytes_per_voxel * N / (t / 1000.0) / 1e9
    launches = S.launch_count() - launches0
    peak, peak_kind = measured_peak_hbm()
    line = {"metric": "per-call time at 182x218x182", "value": res["cc_metric_r4"]["call_us"], "unit": "us",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
            "dtype": "f32", "data": "synthetic: seeded phantom pair, smooth field",
            "config": {"workload": "one call of each full-resolution step (182x218x182) through the C ABI",
                       "l2": "flushed before each call (256 MB)"},
            "kernels": res, "peak_hbm_gbs": peak, "peak_source": peak_kind, "clocks": clk.summary(),
            "gpu_launches": int(launches)}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------------
def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="synx", choices=["synx", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-launches", action="store_true",
                    help="launch every kernel directly instead of replaying per-level CUDA graphs (the same "
                         "work; profilers see each kernel, which they do not inside graphs with conditional nodes)")
    ap.add_argument("--config", default="single",
                    choices=["single", "batched", "serving", "precision", "apply", "kernels"],
                    help="single: the 182x218x182 pair (default); batched: 32 pairs of uneven sizes, "
                         "batched vs sequential pairs/hour; serving: Poisson arrivals of a 2-D/3-D mix, "
                         "p50/p99 latency; precision: the error study; apply: antsApplyTransforms warp + affine; "
                         "kernels: each full-resolution step once (short profiler captures)")
    ap.add_argument("--rates", default="0.5,2,5,10,20", help="serving: arrival rates (requests/s)")
    ap.add_argument("--window", type=float, default=12.0, help="serving: seconds of arrivals per rate")
    args = ap.parse_args(argv)
    if args.config == "batched":
        return run_batched(args)
    if args.config == "serving":
        return run_serving(args)
    if args.config == "precision":
        return run_precision(args)
    if args.config == "apply":
        return run_apply(args)
    if args.config == "kernels":
        return run_kernels(args)

    ws, rank, local = dist_env()
    from ants_b200 import phantoms, replicas
    from ants_b200.synx import Geom

    g = Geom(SIZE)
    if args.impl == "reference":
        if rank != 0:
            return 0
        fixed, moving = phantoms.pair_3d(SIZE, seed=replicas.pair_seed(0))
        run_reference(args, fixed, moving, g)
        return 0

    import torch
    from ants_b200 import synx as S

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    fixed, moving = phantoms.pair_3d(SIZE, seed=replicas.pair_seed(rank))
    sizes = level_sizes(g)

    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    stage = S.SyNStage(S.SyNParams(dim=3, flags=0 if args.plain_launches else S.SYNX_F_USE_GRAPHS, **STAGE),
                       device=local, stream=stream.cuda_stream)
    Fd = torch.from_numpy(fixed).to(dev)
    Md = torch.from_numpy(moving).to(dev)
    fwd_d = torch.empty((3,) + g.shape, device=dev)
    inv_d = torch.empty_like(fwd_d)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2

    def step_device(st):
        st.set_images(Fd, g, Md, g)
        st.run()
        st.fields_device(fwd_d, inv_d)

    for _ in range(args.warmup):
        step_device(stage)
    torch.cuda.synchronize()

    # ---- timed region (device-resident inputs, graph replay) ----
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = S.launch_count()
    stage.reset_profile()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    vox_iters = 0
    its = {}
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            step_device(stage)
            ev[k][1].record(stream)
            log = stage.log()
            vox_iters += voxel_iterations(log, sizes)
        torch.cuda.synchronize()
    for r in log:
        its[r.level] = its.get(r.level, 0) + 1
    launches = S.launch_count() - launches0
    step_ms = [a.elapsed_time(b) for a, b in ev]
    t_total, vox_all = replicas.aggregate(sum(step_ms) / 1000.0, vox_iters, dev)
    value = vox_all / t_total

    prof_levels = stage.level_profile()

    # ---- end to end through the C ABI with pinned host buffers ----
    Fh = torch.from_numpy(fixed).pin_memory().numpy()
    Mh = torch.from_numpy(moving).pin_memory().numpy()
    shp = g.shape + (3,)
    fwd_h = torch.empty(shp, dtype=torch.float32).pin_memory().numpy()
    inv_h = torch.empty(shp, dtype=torch.float32).pin_memory().numpy()
    e2e_ms, e2e_vi = [], 0
    if dist:
        dist.barrier()
    for k in range(args.steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        stage.set_images(Fh, g, Mh, g)
        stage.run()
        stage.fields(fwd_h, inv_h)
        b.record(stream)
        b.synchronize()
        e2e_ms.append(a.elapsed_time(b))
        e2e_vi += voxel_iterations(stage.log(), sizes)
    t_e2e, e2e_vi = replicas.aggregate(sum(e2e_ms) / 1000.0, e2e_vi, dev)
    e2e_value = e2e_vi / t_e2e

    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        lv = prof_levels[ROOF_LEVEL]
        alg = lv["voxels"] * (lv["iterations"] * BYTES_PER_ITER_VOXEL + lv["inverse_subiterations"] * BYTES_PER_INV_VOXEL)
        achieved = alg / (lv["iterate_ms"] / 1000.0) / 1e9
        n_iter = max(lv["iterations"], 1)

        def level_gbs(l):
            b = l["voxels"] * (l["iterations"] * BYTES_PER_ITER_VOXEL + l["inverse_subiterations"] * BYTES_PER_INV_VOXEL)
            return round(b / (l["iterate_ms"] / 1000.0) / 1e9, 1) if l["iterate_ms"] > 0 else None

        roof = {"kernel": "full-resolution SyN iteration graph (182x218x182: warp, CC, smoothing, compose, "
                          "fixed-point inverse loops)", "bound": "hbm",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": ITER_GRAPH_TRAFFIC_BYTES,
                "algorithmic_bytes_per_launch": alg / n_iter, "launch_ms": lv["iterate_ms"] / n_iter,
                "bytes_per_voxel_iteration": BYTES_PER_ITER_VOXEL, "bytes_per_inverse_subiteration_voxel": BYTES_PER_INV_VOXEL,
                "achieved_gbs_per_level": [level_gbs(l) for l in prof_levels],
                "level_ms_per_step": [round(l["iterate_ms"] / args.steps, 3) for l in prof_levels],
                "level_voxels": [l["voxels"] for l in prof_levels],
                "achieved_whole_step": sum(
                    l["voxels"] * (l["iterations"] * BYTES_PER_ITER_VOXEL + l["inverse_subiterations"] * BYTES_PER_INV_VOXEL)
                    for l in prof_levels) / t_total / 1e9}
        cpu = None
        if not args.no_cpu_baseline and ws == 1:
            threads = os.cpu_count() or 1
            v_cpu, dt, n_cpu = cpu_sample(fixed, moving, g, threads, min_seconds=10.0, max_iterations=20)
            cpu = {"value": v_cpu, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"{n_cpu} full-resolution (182x218x182) SyN-CC iterations from zero fields "
                             f"({dt:.1f} s of CPU work)"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * t_total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": DATA,
            "config": workload_config([its.get(l, 0) for l in range(4)], vox_iters // args.steps, ws),
            "cuda_graphs": not args.plain_launches,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(Fh.nbytes + Mh.nbytes),
                    "d2h_bytes_per_step": int(fwd_h.nbytes + inv_h.nbytes),
                    "ms_per_step": 1000.0 * t_e2e / args.steps},
            "roofline": roof, "cpu_baseline": cpu, "clocks": clk.summary(), "gpu_launches": int(launches),
        }
        print(json.dumps(line), flush=True)
    stage.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
