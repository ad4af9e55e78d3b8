"""End-to-end parity at the benchmarked configurations: the CUDA stage (through the C ABI) against
the CPU oracle (float) on the same seeded inputs, with the full schedules.

* 3-D 182x218x182 at 1 mm: SyN[0.1,3,0], CC r=4, shrink 8x4x2x1, sigmas 3x2x1x0 vox,
  iterations 100x70x50x20 at threshold 1e-12 (the single-pair throughput workload), on the
  axis-aligned grid and on the same arrays placed on an oblique, anisotropic grid.
* 2-D 256x256 blobs at 1 mm: SyN[0.1,3,0], CC r=2, shrink 4x2x1, sigmas 2x1x0 vox,
  iterations 40x20x10 at 1e-12.

Asserted: the same iterations run per level (the convergence monitor stops the same levels at the
same iteration), the per-iteration metric within 2e-3, and the final forward and inverse fields
within an RMS of 0.05 voxel.  The measured figures are printed (run with -s to see them).
Reference stage replaced: Examples/itkantsRegistrationHelper.hxx:1983-2220; final composition
Examples/antsDisplacementAndVelocityFieldRegistrationCommandIterationUpdate.h:415-432.
"""
import os
from collections import Counter

import numpy as np
import pytest
from scipy.spatial.transform import Rotation

import oracle as O
from ants_b200 import phantoms
from ants_b200.synx import SYNX_F_USE_GRAPHS, Geom, SyNParams, SyNStage

pytestmark = pytest.mark.gpu

C2 = dict(cc_radius=4, iterations=(100, 70, 50, 20), shrink_factors=(8, 4, 2, 1), smoothing_sigmas=(3.0, 2.0, 1.0, 0.0),
          learning_rate=0.1, update_variance=3.0, total_variance=0.0, convergence_threshold=1e-12,
          convergence_window=10)
C1 = dict(cc_radius=2, iterations=(40, 20, 10), shrink_factors=(4, 2, 1), smoothing_sigmas=(2.0, 1.0, 0.0),
          learning_rate=0.1, update_variance=3.0, total_variance=0.0, convergence_threshold=1e-12,
          convergence_window=10)


def planes(interleaved):
    return np.moveaxis(interleaved, -1, 0)


def rms_vox(a, b, spacing):
    sp = np.asarray(spacing, dtype=np.float64).reshape((-1,) + (1,) * (a.ndim - 1))
    return float(np.sqrt((((a - b) / sp) ** 2).sum(0).mean()))


def compare(f, gf, m, gm, stage, dim, label):
    O.set_threads(os.cpu_count() or 1)
    P = SyNParams(dim=dim, flags=SYNX_F_USE_GRAPHS, **stage)
    with SyNStage(P) as st:
        st.set_images(f, gf, m, gm)
        st.run()
        fwd, inv = (planes(a) for a in st.fields())
        go = st.output_geom()
        log = st.log()
    rf, ri, rg, rlog = O.syn_register(f, gf, m, gm, P)
    assert go.size == rg.size
    its = Counter(r.level for r in log)
    rits = Counter(r["level"] for r in rlog)
    per_level = [its.get(l, 0) for l in range(len(stage["iterations"]))]
    ref_per_level = [rits.get(l, 0) for l in range(len(stage["iterations"]))]
    dmetric = float(np.max(np.abs(np.array([r.metric for r in log]) - np.array([r["metric"] for r in rlog]))))
    e_fwd, e_inv = rms_vox(fwd, rf, go.spacing), rms_vox(inv, ri, go.spacing)
    size = rms_vox(fwd, np.zeros_like(fwd), go.spacing)
    print(f"\n[{label}] iterations per level {per_level} (oracle {ref_per_level}); max |metric difference| "
          f"{dmetric:.2e}; forward-field RMS difference {e_fwd:.2e} voxel, inverse {e_inv:.2e} voxel; "
          f"forward-field RMS {size:.3f} voxel", flush=True)
    assert per_level == ref_per_level
    assert dmetric < 2e-3
    assert e_fwd <= 0.05 and e_inv <= 0.05
    assert size > 0.1  # a real deformation was recovered


@pytest.fixture(scope="module")
def pair_c2():
    return phantoms.pair_3d((182, 218, 182), seed=phantoms.SEED_BASE)


def test_c2_single_pair_workload(cuda, pair_c2):
    f, m = pair_c2
    g = Geom((182, 218, 182))
    compare(f, g, m, g, C2, 3, "3-D 182x218x182, axis-aligned")


def test_c2_on_an_oblique_grid(cuda, pair_c2):
    f, m = pair_c2
    R = Rotation.from_euler("xyz", [0.2, -0.15, 0.3]).as_matrix()
    g = Geom((182, 218, 182), (1.0, 0.9, 1.2), (-90.0, 110.0, -70.0), R)
    compare(f, g, m, g, C2, 3, "3-D 182x218x182, oblique and anisotropic")


def test_c1_blobs_2d(cuda):
    f, m = phantoms.pair_2d((256, 256), seed=phantoms.SEED_BASE)
    g = Geom((256, 256))
    compare(f, g, m, g, C1, 2, "2-D 256x256 blobs")
