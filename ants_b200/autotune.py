"""The project's tile autotuner: measures candidate tile plans per level grid and writes the winners
to the tuning table that libsynx loads at synx_create (tuning_b200.txt beside the library).

For a set of representative workloads (the benchmark's image pairs and pyramids) every candidate
plan runs the whole registration through the C ABI; the level profile gives each level's iteration
time, so one registration per candidate times every level of the pyramid under that candidate.  A
level grid keeps the candidate with the least time per iteration.  Candidates:

* the persistent level kernel (every phase of every iteration in one cooperative launch), where the
  level kernel implements the stage's options;
* the per-kernel path with the update smoothing as the fused slab kernel (8- or 16-row column tiles),
  as an xy kernel plus a z kernel, or as the pipelined xy kernel (32- or 64-row tiles) plus the z
  kernel, crossed with the CC kernel's z chunk count (its cost model, or 4 or 8 chunks);
* the built-in cost models (the plan without a table), timed for comparison.

    python -m ants_b200.autotune --out ants_b200/tuning_b200.txt [--workloads single,batched,...]

The plans change the launch decomposition only: the smoothing variants give identical bits, the
CC chunking changes the order of the FP64 window sums' rounding, and the persistent kernel agrees
with the per-kernel path within the stage tolerances (tests/test_gpu_syn.py).
"""
from __future__ import annotations

import argparse
import os
import sys
import time
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if os.path.dirname(HERE) not in sys.path:
    sys.path.insert(0, os.path.dirname(HERE))

from ants_b200 import phantoms  # noqa: E402
from ants_b200 import synx as S  # noqa: E402

BIG = 2 ** 31 - 1

STAGE_SINGLE = dict(cc_radius=4, iterations=(100, 70, 50, 20), shrink_factors=(8, 4, 2, 1),
                    smoothing_sigmas=(3.0, 2.0, 1.0, 0.0))
STAGE_3LEVEL = dict(cc_radius=4, iterations=(50, 30, 15), shrink_factors=(4, 2, 1), smoothing_sigmas=(2.0, 1.0, 0.0))
STAGE_SERVING_3D = dict(cc_radius=4, iterations=(40, 20, 10), shrink_factors=(4, 2, 1),
                        smoothing_sigmas=(2.0, 1.0, 0.0))
STAGE_SERVING_2D = dict(cc_radius=2, iterations=(40, 20, 10), shrink_factors=(4, 2, 1),
                        smoothing_sigmas=(2.0, 1.0, 0.0))
STAGE_PRECISION = dict(cc_radius=5, iterations=(70, 50, 20), shrink_factors=(4, 2, 1), smoothing_sigmas=(2.0, 1.0, 0.0))


def workloads(names):
    """(label, dim, size, stage) per representative pair."""
    out = []
    if "single" in names:
        out.append(("182x218x182 single pair", 3, (182, 218, 182), STAGE_SINGLE))
        out.append(("256x256 blobs", 2, (256, 256), dict(cc_radius=2, iterations=(40, 20, 10), shrink_factors=(4, 2, 1),
                                                         smoothing_sigmas=(2.0, 1.0, 0.0))))
    if "batched" in names:
        for k in range(32):  # the dims of the batched benchmark's pairs
            dims = tuple(int(x) for x in np.random.default_rng(0x5EED0000 + 1000 + k).integers(96, 193, size=3))
            out.append((f"batched pair {k} {dims}", 3, dims, STAGE_3LEVEL))
    if "serving" in names:
        out += [("serving 2-D 256^2", 2, (256, 256), STAGE_SERVING_2D),
                ("serving 2-D 512^2", 2, (512, 512), STAGE_SERVING_2D),
                ("serving 3-D 128^3", 3, (128, 128, 128), STAGE_SERVING_3D),
                ("serving 3-D 182x218x182", 3, (182, 218, 182), STAGE_SERVING_3D),
                ("serving 3-D 256^3", 3, (256, 256, 256), STAGE_SERVING_3D)]
    if "precision" in names:
        out.append(("precision 256^3 r=5", 3, (256, 256, 256), STAGE_PRECISION))
    return out


def candidates(dim):
    """(name, SyNParams overrides) per candidate plan."""
    cands = [("models", dict(tuning=1)),
             ("persistent", dict(tuning=1, persistent_max_voxels=BIG))]
    if dim == 2:
        cands.append(("kernels", dict(tuning=1, flags=S.SYNX_F_NO_PERSISTENT)))
        return cands
    for rows in (8, 16, -1, -2, -3):
        for chunks in (0, 4, 8):
            cands.append((f"kernels rows={rows} chunks={chunks}",
                          dict(tuning=1, flags=S.SYNX_F_NO_PERSISTENT, smooth_tile_rows=rows, cc_z_chunks=chunks)))
    return cands


def time_levels(f, m, g, dim, stage, over, reps):
    """Per level: (ms per iteration, plan) of the best of `reps` timed registrations (one untimed
    registration first captures the graphs)."""
    flags = S.SYNX_F_USE_GRAPHS | over.get("flags", 0)
    kw = {k: v for k, v in over.items() if k != "flags"}
    P = S.SyNParams(dim=dim, flags=flags, convergence_threshold=1e-12, **stage, **kw)
    best = None
    with S.SyNStage(P) as st:
        st.set_images(f, g, m, g)
        plans = [st.level_plan(l) for l in range(len(stage["iterations"]))]
        st.run()
        for _ in range(reps):
            st.reset_profile()
            st.set_images(f, g, m, g)
            st.run()
            prof = st.level_profile()
            per = [p["iterate_ms"] / max(p["iterations"], 1) for p in prof]
            best = per if best is None else [min(a, b) for a, b in zip(best, per)]
    return best, plans


def level_key(g: S.Geom, factor: int, dim: int, radius: int, uvar: float):
    gl = S.shrink_geom(g, factor)
    rs = 1
    for n in gl.size[:dim]:
        rs = max(rs, len(S.gaussian_kernel(uvar, 0.001, n)) // 2)
    size3 = tuple(gl.size) + (1,) * (3 - len(gl.size))
    return (dim,) + size3 + (radius, rs)


def tune(names, reps=2, log=print):
    table = {}
    for label, dim, size, stage in workloads(names):
        t0 = time.perf_counter()
        seed = phantoms.SEED_BASE + (zlib.crc32(label.encode()) & 0xFFFF)
        f, m = phantoms.pair_2d(size, seed=seed) if dim == 2 else phantoms.pair_3d(size, seed=seed)
        g = S.Geom(size)
        results = {}
        for name, over in candidates(dim):
            try:
                results[name] = time_levels(f, m, g, dim, stage, over, reps)
            except S.SynxError as e:  # a candidate the device cannot run (e.g. too large for the level kernel)
                log(f"  {label}: {name} skipped: {e}")
        for name, (ms, _) in results.items():
            log(f"    {label} {name}: " + " ".join(f"{x:.4f}" for x in ms) + " ms/iteration per level")
        for lv, factor in enumerate(stage["shrink_factors"]):
            key = level_key(g, factor, dim, stage["cc_radius"], 3.0)
            default_ms = results["models"][0][lv]
            best_name = min(results, key=lambda n: results[n][0][lv])
            ms, plans = results[best_name]
            plan = plans[lv]
            entry = (plan["persistent"], plan["smooth_rows"] if plan["smooth_rows"] != 0 else 8,
                     plan["cc_z_chunks"], ms[lv], default_ms)
            old = table.get(key)
            if old is None or entry[3] < old[3]:
                table[key] = entry
            log(f"  {label} level {lv} {key[1:1 + 3]}: best {best_name} {ms[lv]:.4f} ms/iteration "
                f"(cost models {default_ms:.4f})")
        log(f"{label}: {len(results)} candidates in {time.perf_counter() - t0:.1f} s")
    return table


def write_table(table, path):
    with open(path, "w") as fh:
        fh.write("# synx tile plans measured by ants_b200.autotune on one B200 (sm_100a)\n")
        fh.write("# dim nx ny nz r_cc r_smooth  persistent smooth_rows cc_z_chunks  ms_per_iteration "
                 "ms_per_iteration_cost_models\n")
        for key in sorted(table):
            p, rows, chunks, ms, dms = table[key]
            fh.write(" ".join(str(x) for x in key) + f"  {p} {rows} {chunks}  {ms:.5f} {dms:.5f}\n")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "tuning_b200.txt"))
    ap.add_argument("--workloads", default="single,batched,serving,precision")
    ap.add_argument("--reps", type=int, default=2)
    a = ap.parse_args(argv)
    import torch
    assert torch.cuda.is_available(), "the autotuner times candidates on a CUDA device"
    table = tune(set(a.workloads.split(",")), a.reps)
    write_table(table, a.out)
    print(f"wrote {len(table)} entries to {a.out}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
