"""Runs the unmodified reference CUDA build on a case, for parity tests on a GPU machine.

The driver binaries are ``oracle/_ref/ref_driver_f32`` / ``ref_driver_f64``: the
reference's own ``src/*.cu`` compiled from where they lie by ``oracle/build_ref.sh``,
linked with ``oracle/ref_driver.cu`` in place of the reference's ``main.cpp``.  The
driver steps ``LoquatSph`` exactly as ``RunSimulation`` does (src/loquat.cu:511-565) and
dumps its device arrays (RWD1 files, read by ``read_rwd``), saves its own output files,
or records its wall-strip force."""
from __future__ import annotations

import os
import subprocess

import pytest

from tests.golden.make_golden import read_rwd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def driver(precision: int) -> str:
    path = os.path.join(REF_DIR, "ref_driver_f64" if precision == 8 else "ref_driver_f32")
    if not os.path.exists(path):
        pytest.skip(f"{path} missing: build it with oracle/build_ref.sh where the reference sources are")
    return path


def run_reference(project: str, precision: int, steps: int, *, dump_dir: str | None = None,
                  dump_steps=(), keys=(), stage_step: int = -1, save_steps=(), wall_force_every: int = 0,
                  timeout: float = 1800.0) -> str:
    """Runs the reference on ``<project>.xml/.dat[/.motion]`` for ``steps`` steps; returns
    its console output.  Dumps go to ``dump_dir`` (``init.rwd``, ``step_<s>.rwd``,
    ``stage/<tag>.rwd``); saves go to ``<project>/`` as the reference writes them."""
    cmd = [driver(precision), project, "--steps", str(steps)]
    if dump_dir:
        os.makedirs(os.path.join(dump_dir, "stage"), exist_ok=True)
        cmd += ["--dump-dir", dump_dir]
        if dump_steps:
            cmd += ["--dump-steps", ",".join(map(str, dump_steps))]
        if keys:
            cmd += ["--dump-keys", ",".join(keys)]
        if stage_step >= 0:
            cmd += ["--stage-step", str(stage_step)]
        if wall_force_every:
            cmd += ["--wall-force-every", str(wall_force_every)]
    if save_steps:
        cmd += ["--save-steps", ",".join(map(str, save_steps))]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference driver failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout[-2000:]}\n"
                           f"{r.stderr[-2000:]}")
    return r.stdout


def dumps(dump_dir: str, name: str, precision: int) -> dict:
    return read_rwd(os.path.join(dump_dir, name), 8 if precision == 8 else 4)
