"""Parity with the unmodified reference CUDA build, run live on the same GPU, at the two
configurations the step is specified on:

* the granular column collapse (24 x 24 x 48 = 27,648 soil particles at dx = 5 mm,
  seed 1), FP64 as the reference builds it (``-DDOUBLE_PRECISION``) and FP32, 100 steps;
* the translating retaining wall (200 x 80 x 120 = 1,920,000 soil particles at
  dx = 2.5 mm, seed 2), FP32, 5 steps.

Both programs read the same case files (written by the project's generator in the
reference's layout).  The reference is driven by ``oracle/ref_driver.cu``, which steps
``LoquatSph`` as ``RunSimulation`` does (src/loquat.cu:548-561) and dumps its device
arrays.  Bars: sort permutation, cell ranges and cell coordinates bit-exact (integer
work); positions, velocities, density and stress within 1e-5 relative L2.  The column
has no contact wall, so its bar holds over the whole state.  The wall's bar holds beyond
one kernel support (2h) of the contact zone, where the reference's contact
redistribution reads state other threads are rewriting
(src/particle_interaction.cu:147-166); the error inside the zone is printed."""
import os

import numpy as np
import pytest

from retainwall_code_b200 import LoquatSph, cases as C
from tests._refrun import dumps, run_reference
from tests._util import far_from_contact, rel

pytestmark = pytest.mark.gpu

INT_KEYS = ("part_idx", "cell_beg", "cell_end", "cellpos")
INIT_KEYS = INT_KEYS + ("pospres",)  # the loader's in-cell positions too, bit for bit
KEYS = INT_KEYS + ("pospres", "velrhop", "str", "contact_var")


def fields(a_pos, a_vel, a_str):
    """The compared quantities: in-cell position, pressure, velocity, density, stress."""
    return {"position": a_pos[:, :3], "pressure": a_pos[:, 3], "velocity": a_vel[:, :3], "density": a_vel[:, 3],
            "stress": a_str}


def compare_state(sim, g, rows, tol, tag, report):
    """Relative L2 of each field over `rows`; failures are collected in `report`."""
    ours = fields(sim.get("pospres"), sim.get("velrhop"), sim.get("str"))
    refs = fields(g["pospres"], g["velrhop"], g["str"])
    out = {}
    for k in ours:
        r = rel(ours[k][rows], refs[k][rows])
        out[k] = r
        if not r < tol:
            report.append(f"{tag} {k}: {r:.3e} >= {tol:g}")
    return out


def compare_ints(sim, g, tag, report, keys=INT_KEYS):
    for k in keys:
        a, b = sim.get(k), g[k]
        if not np.array_equal(a, b):
            report.append(f"{tag} {k}: {int(np.sum(a != b))} entries differ")


@pytest.mark.parametrize("prec", [8, 4], ids=["fp64", "fp32"])
def test_config1_column_collapse_vs_reference_build(tmp_path, prec):
    case = C.column_collapse()
    assert case.npm == 27_648
    proj = str(tmp_path / "column")
    C.write_case(case, proj)
    dd = str(tmp_path / "dump")
    steps = (1, 10, 100)
    run_reference(proj, prec, 100, dump_dir=dd, dump_steps=steps, keys=KEYS)
    sim = LoquatSph(proj, precision=prec)
    report = []
    compare_ints(sim, dumps(dd, "init.rwd", prec), "init", report, INIT_KEYS)
    every = np.ones(case.np_, bool)
    done = 0
    for st in steps:
        sim.step(st - done)
        done = st
        g = dumps(dd, f"step_{st}.rwd", prec)
        compare_ints(sim, g, f"step {st}", report)
        errs = compare_state(sim, g, every, 1e-5, f"step {st}", report)
        print(f"config1 {'fp64' if prec == 8 else 'fp32'} step {st}: " +
              ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    assert sim.info().device_err == 0
    assert not report, "\n".join(report)


def test_config2_retaining_wall_vs_reference_build(tmp_path):
    case = C.retaining_wall(wall_friction=C.REFERENCE_WALL_FRICTION)
    assert case.npm == 1_920_000
    proj = str(tmp_path / "wall")
    C.write_case(case, proj)
    dd = str(tmp_path / "dump")
    run_reference(proj, 4, 5, dump_dir=dd, dump_steps=(5,), keys=KEYS)
    sim = LoquatSph(proj, precision=4)
    report = []
    compare_ints(sim, dumps(dd, "init.rwd", 4), "init", report, INIT_KEYS)
    sim.step(5)
    g = dumps(dd, "step_5.rwd", 4)
    compare_ints(sim, g, "step 5", report)
    far = far_from_contact(case, g["cellpos"], g["pospres"], g["contact_var"])
    mat = np.arange(case.np_) >= case.npb
    zone = mat & ~far
    errs_far = compare_state(sim, g, far, 1e-5, "step 5 (beyond 2h of the contact zone)", report)
    errs_all = compare_state(sim, g, mat, 1.0, "step 5 (all soil)", [])
    errs_zone = compare_state(sim, g, zone, 1.0, "step 5 (contact zone)", [])
    print(f"config2 step 5: {int(far.sum())} soil particles beyond 2h of the contact zone, {int(zone.sum())} "
          f"within; far: " + ", ".join(f"{k} {v:.2e}" for k, v in errs_far.items()) +
          "; within: " + ", ".join(f"{k} {v:.2e}" for k, v in errs_zone.items()) +
          "; all soil: " + ", ".join(f"{k} {v:.2e}" for k, v in errs_all.items()))
    assert sim.info().device_err == 0
    assert not report, "\n".join(report)
