"""Generate the golden fixtures of this directory from the UNMODIFIED reference build.

Runs on a machine with a CUDA GPU and the prebuilt reference driver
(``oracle/_ref/ref_driver_f32``, made by ``oracle/build_ref.sh`` from the reference's
own sources).  For each mini case it:

1. writes the case in the reference's file layout with the project's generator
   (``retainwall_code_b200.cases``; seeded, so the inputs are reproducible);
2. runs the reference step for ``STEPS`` steps, dumping every device array
   (RWD1 format, see ``read_rwd``) after step 1, after every stage of step index 1,
   and after steps 10 and 100, plus the reference's wall-strip force every step;
3. packs the arrays the parity tests compare into ``<case>_ref.npz``.

Usage:  python tests/golden/make_golden.py OUTDIR_FOR_RAW_DUMPS [CASE ...]
(no CASE: every case; the fixtures are written next to this script and copied into
OUTDIR_FOR_RAW_DUMPS)
"""
from __future__ import annotations

import hashlib
import os
import shutil
import struct
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from retainwall_code_b200 import cases as C  # noqa: E402

STEPS = 100
DUMP_STEPS = [1, 10, 100]
STAGE_STEP = 1
STAGES = ["p0_sorted", "p1_adami", "p2_corner", "p3_interaction", "p4_predictor",
          "c0_sorted", "c1_adami", "c2_corner", "c3_interaction", "c4_corrector"]


def mini_cases():
    """The fixture cases: a column collapse, a retaining wall with a contact wall, and
    the same wall periodic in y (no side walls, period-bound planes).  The wall cases
    use the reference's hard-coded wall friction (0.58108)."""
    return {
        "col_mini": C.column_collapse(nx=8, ny=8, nz=16, runout=1.0, name="col_mini"),
        "wall_mini": C.retaining_wall(nx=16, ny=8, nz=12, dx=0.005, wall_friction=C.REFERENCE_WALL_FRICTION,
                                      name="wall_mini"),
        "per_mini": C.retaining_wall(nx=16, ny=8, nz=12, dx=0.005, wall_friction=C.REFERENCE_WALL_FRICTION,
                                     periodic_y=True, name="per_mini"),
    }


def case_digest(case) -> str:
    h = hashlib.sha256()
    for a in (case.codes, case.pospres, case.velrhop, case.idmassidx, case.stress, case.strain, case.normal):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:16]


_DT = {("codes", 16): ("<i4", 4), ("cellpos", 16): ("<i4", 4), ("part_idx", 4): ("<i4", 1),
       ("part_cel", 4): ("<i4", 1), ("cell_beg", 4): ("<i4", 1), ("cell_end", 4): ("<i4", 1)}


def read_rwd(path: str, scalar_bytes: int = 4) -> dict:
    """Reader of the RWD1 dumps written by oracle/ref_driver.cu."""
    out = {}
    with open(path, "rb") as f:
        assert f.read(4) == b"RWD1"
        (n,) = struct.unpack("<i", f.read(4))
        for _ in range(n):
            name = f.read(32).split(b"\0", 1)[0].decode()
            (elem,) = struct.unpack("<i", f.read(4))
            (count,) = struct.unpack("<q", f.read(8))
            raw = f.read(elem * count)
            if name == "meta":
                out[name] = np.frombuffer(raw, "<f8")
                continue
            key = (name, elem)
            if key in _DT:
                dt, w = _DT[key]
            else:
                dt = "<f4" if scalar_bytes == 4 else "<f8"
                w = elem // scalar_bytes
            a = np.frombuffer(raw, dt)
            out[name] = a.reshape(count, w) if w > 1 else a
    return out


STATE_KEYS = ["codes", "cellpos", "pospres", "pospres_ori", "velrhop", "idmassidx", "str", "stn", "normal_m",
              "contact_mag", "contact_var"]
STAGE_KEYS = {
    "p0_sorted": ["part_idx", "cell_beg", "cell_end", "cellpos", "pospres", "velrhop", "str"],
    "p1_adami": ["velrhop", "str", "contact_mag"],
    "p2_corner": ["contact_var", "contact_mag"],
    "p3_interaction": ["accad", "acestn", "spin", "contact_var", "contact_mag"],
    "p4_predictor": ["pospres", "velrhop", "str", "stn", "idmassidx"],
    "c0_sorted": ["part_idx", "cell_beg", "cell_end"],
    "c1_adami": ["velrhop", "str", "contact_mag"],
    "c2_corner": ["contact_var", "contact_mag"],
    "c3_interaction": ["accad", "acestn", "spin", "contact_var", "contact_mag"],
    "c4_corrector": ["pospres", "cellpos", "velrhop", "str", "stn", "idmassidx", "pospres_ori", "accad"],
}
STEP_KEYS = ["cellpos", "pospres", "velrhop", "str", "idmassidx", "contact_mag", "contact_var"]


def main(raw_dir: str, only=None) -> None:
    drv = os.path.join(ROOT, "oracle", "_ref", "ref_driver_f32")
    if not os.path.exists(drv):
        raise SystemExit(f"missing {drv}; run oracle/build_ref.sh where the reference sources exist")
    for name, case in mini_cases().items():
        if only and name not in only:
            continue
        d = os.path.join(raw_dir, name)
        os.makedirs(os.path.join(d, "stage"), exist_ok=True)
        proj = os.path.join(d, name)
        C.write_case(case, proj)
        cmd = [drv, proj, "--steps", str(STEPS), "--dump-dir", d, "--dump-steps", ",".join(map(str, DUMP_STEPS)),
               "--stage-step", str(STAGE_STEP), "--wall-force-every", "1"]
        with open(os.path.join(d, "driver.log"), "w") as log:
            subprocess.run(cmd, check=True, stdout=log, stderr=subprocess.STDOUT)
        fx = {"digest": np.array(case_digest(case)), "steps": np.array(STEPS)}
        init = read_rwd(os.path.join(d, "init.rwd"))
        for k in ("part_idx", "cell_beg", "cell_end", "cellpos", "pospres"):
            fx[f"init/{k}"] = init[k]
        for st in DUMP_STEPS:
            s = read_rwd(os.path.join(d, f"step_{st}.rwd"))
            fx[f"step{st}/meta"] = s["meta"]
            keys = STATE_KEYS if st == STAGE_STEP else STEP_KEYS
            for k in keys:
                fx[f"step{st}/{k}"] = s[k]
        for sg in STAGES:
            s = read_rwd(os.path.join(d, "stage", f"{sg}.rwd"))
            fx[f"{sg}/meta"] = s["meta"]
            for k in STAGE_KEYS[sg]:
                fx[f"{sg}/{k}"] = s[k]
        th = np.loadtxt(os.path.join(d, "time_history.txt"))
        fx["wall_force_kN"] = th.reshape(-1, 2)
        out = os.path.join(HERE, f"{name}_ref.npz")
        np.savez_compressed(out, **fx)
        shutil.copy(out, os.path.join(raw_dir, f"{name}_ref.npz"))
        print(name, case.np_, case.npb, case.npm, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    if len(sys.argv) < 2:
        raise SystemExit(__doc__)
    main(sys.argv[1], sys.argv[2:])
