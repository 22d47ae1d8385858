"""Python mirror of the reference's ``LoquatSph`` (src/loquat.h:44-126) over the C ABI.

Method names follow the reference's (``PredictorSection`` -> ``predictor_section`` ...);
each one is one C-ABI call into librw.so.  ``run_simulation`` is the reference's
``RunSimulation`` loop (src/loquat.cu:511-565) with whole steps replayed from a captured
CUDA graph between saves."""
from __future__ import annotations

import ctypes as ct
import os
from typing import Optional, Sequence

import numpy as np

from . import _abi
from ._lib import check, lib


class LoquatSph:
    def __init__(self, project: Optional[str] = None, device: int = 0, precision: int = 4, case=None):
        """Open ``project`` (reads ``<project>.xml/.dat/.motion``) or an in-memory
        ``cases.Case``.  precision 4 = float (the reference's default build), 8 = double."""
        L = lib()
        h = ct.c_void_p()
        if case is not None:
            keep: list = []
            c = _abi.case_struct(case, keep)
            st = L.rw_create_from_case(ct.byref(c), device, precision, ct.byref(h))
        else:
            if project is None:
                raise ValueError("need a project name or a case")
            st = L.rw_create(project.encode(), device, precision, ct.byref(h))
        check(st, "rw_create", None)
        self._h = h
        self.project = project
        self.precision = precision

    # -- lifetime ---------------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().rw_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, st: int, what: str) -> None:
        check(st, what, self._h)

    @property
    def handle(self):
        return self._h

    # -- learned closure ----------------------------------------------------------------
    def set_closure(self, net=None, margin: float = 0.0) -> None:
        """Use ``net`` (closure.Mlp) for the HypoCS objective stress rate (None: exact)."""
        self._c(lib().rw_set_closure(self._h, net.handle if net is not None else None, margin), "rw_set_closure")

    def list_stats(self):
        """(entries, soil particles) of the kept candidate lists."""
        out = (ct.c_int64 * 2)()
        self._c(lib().rw_list_stats(self._h, out), "rw_list_stats")
        return out[0], out[1]

    def closure_stats(self) -> dict:
        out = (ct.c_double * 4)()
        self._c(lib().rw_closure_stats(self._h, out), "rw_closure_stats")
        return {"offered": out[0], "used": out[1], "mean_rel_err": out[2], "max_rel_err": out[3]}

    # -- the reference's stage methods --------------------------------------------------
    def step_calculation(self):
        self._c(lib().rw_begin_step(self._h), "rw_begin_step")

    def neighbor_search(self, section: int):
        self._c(lib().rw_neighbor_search(self._h, section), "rw_neighbor_search")

    def rigid_body_update(self):
        self._c(lib().rw_rigid_body_update(self._h), "rw_rigid_body_update")

    def adami_boundary(self):
        self._c(lib().rw_adami_boundary(self._h), "rw_adami_boundary")

    def find_corner_particle(self):
        self._c(lib().rw_find_corner(self._h), "rw_find_corner")

    def stress_regularization(self):
        self._c(lib().rw_shepard_filter(self._h), "rw_shepard_filter")

    def particle_interaction(self):
        self._c(lib().rw_particle_interaction(self._h), "rw_particle_interaction")

    def predictor(self):
        self._c(lib().rw_predictor(self._h), "rw_predictor")

    def corrector(self):
        self._c(lib().rw_corrector(self._h), "rw_corrector")

    def end_step(self):
        self._c(lib().rw_end_step(self._h), "rw_end_step")

    def predictor_section(self, shepard: bool = False):
        """src/loquat.cu:376-406 (Shepard only when the caller's step schedule asks)."""
        self.neighbor_search(0)
        self.rigid_body_update()
        self.adami_boundary()
        self.find_corner_particle()
        if shepard:
            self.stress_regularization()
        self.particle_interaction()
        self.predictor()

    def corrector_section(self):
        """src/loquat.cu:408-436."""
        self.neighbor_search(1)
        self.adami_boundary()
        self.find_corner_particle()
        self.particle_interaction()
        self.corrector()

    def step(self, n: int = 1):
        """n whole steps from the captured CUDA graph (asynchronous)."""
        self._c(lib().rw_step(self._h, n), "rw_step")

    def step_timed(self, n: int) -> float:
        """n whole steps; returns their device time in ms (CUDA events on the context's
        stream; the graph is captured before the first event if needed)."""
        ms = ct.c_double(0.0)
        self._c(lib().rw_step_timed(self._h, n, ct.byref(ms)), "rw_step_timed")
        return ms.value

    def synchronize(self):
        self._c(lib().rw_synchronize(self._h), "rw_synchronize")

    def profile(self, nsteps: int = 5):
        """Mean device time per stage [ms] over nsteps per-stage steps, and the number
        of kernels one whole step launches."""
        from ._lib import STAGE_NAMES

        ms = (ct.c_double * len(STAGE_NAMES))()
        kps = ct.c_int(0)
        self._c(lib().rw_profile(self._h, nsteps, ms, len(STAGE_NAMES), ct.byref(kps)), "rw_profile")
        return dict(zip(STAGE_NAMES, ms[:])), kps.value

    def autotune(self, steps: int = 2) -> int:
        """Pick the faster interaction kernel for this case by timing (the case advances)."""
        ch = ct.c_int(-1)
        self._c(lib().rw_autotune(self._h, steps, ct.byref(ch)), "rw_autotune")
        return ch.value

    # -- state ----------------------------------------------------------------------------
    def info(self) -> _abi.Info:
        inf = _abi.Info()
        self._c(lib().rw_get_info(self._h, ct.byref(inf)), "rw_get_info")
        return inf

    def get(self, name: str) -> np.ndarray:
        rows, cols, dt = _abi.array_spec(name, self.info())
        a = np.zeros((rows, cols), dt) if cols > 1 else np.zeros(rows, dt)
        self._c(lib().rw_get_array(self._h, _abi.ARRAYS[name], a.ctypes.data, a.nbytes), f"rw_get_array({name})")
        return a

    def set(self, name: str, a: np.ndarray) -> None:
        rows, cols, dt = _abi.array_spec(name, self.info())
        a = np.ascontiguousarray(a, dtype=dt)
        self._c(lib().rw_set_array(self._h, _abi.ARRAYS[name], a.ctypes.data, a.nbytes), f"rw_set_array({name})")

    def set_counters(self, time: float, step: int, npm: int, np_delete_m: int) -> None:
        self._c(lib().rw_set_counters(self._h, time, step, npm, np_delete_m), "rw_set_counters")

    def set_option(self, opt: int, value: float) -> None:
        self._c(lib().rw_set_option(self._h, opt, value), "rw_set_option")

    def wall_force(self, mode: int = 0, wall_id: int = 10, strip: Optional[Sequence[float]] = None) -> np.ndarray:
        """Lateral wall force [N], FP64 accumulation (mode 0: by nearest wall id; 1: strip)."""
        out = (ct.c_double * 3)()
        sp = None
        if strip is not None:
            sa = (ct.c_double * 3)(*strip)
            sp = ct.cast(sa, ct.c_void_p)
        self._c(lib().rw_wall_force(self._h, mode, wall_id, sp, out), "rw_wall_force")
        return np.array(out[:])

    def wall_profile(self, x_wall: float = float("nan"), z_top: float = float("nan"), dz: float = float("nan"),
                     nbins: int = 0) -> np.ndarray:
        """Earth-pressure profile along the wall: rows (depth, band 1, band 2, band 3).
        Defaults are the reference's: (int)(1/dr) bins of dr below its hard-coded top."""
        if nbins <= 0:
            nbins = max(1, int(np.float32(1.0) / np.float32(self.info().dr)))
        out = (ct.c_double * (4 * nbins))()
        self._c(lib().rw_wall_profile(self._h, x_wall, z_top, dz, nbins, out), "rw_wall_profile")
        return np.array(out[:]).reshape(nbins, 4)

    def save(self, outdir: Optional[str] = None) -> None:
        d = outdir or self.project or "."
        self._c(lib().rw_save(self._h, d.encode()), "rw_save")

    # -- RunSimulation ---------------------------------------------------------------------
    def run_simulation(self, outdir: Optional[str] = None, time_max: Optional[float] = None,
                       output_frequency: Optional[float] = None) -> None:
        """The reference's main loop (src/loquat.cu:533-561): the initial output, then
        steps, with Saving inside the step in which output_time exceeds output-frequency
        (time-max and output-frequency default to the parameter file's).  The steps
        between two saves run as one captured-graph call."""
        inf = self.info()
        tmax = float(inf.time_max if time_max is None else time_max)
        freq = float(inf.output_frequency if output_frequency is None else output_frequency)
        out = outdir or self.project or "."
        os.makedirs(out, exist_ok=True)
        self.save(out)
        t, ot, dt = inf.time, 0.0, inf.dt
        while t < tmax:
            n, save = 0, False
            while t < tmax and not save:
                n += 1
                save = ot > freq
                if save:
                    ot = 0.0
                t += dt
                ot += dt
            self.step(n)
            self.synchronize()
            if save:
                self.save(out)


class Batch:
    """Several cases on one device advanced by one graph launch per step
    (rw_batch_*).  The LoquatSph objects must stay alive while the batch is used."""

    def __init__(self, sims):
        self.sims = list(sims)
        arr = (ct.c_void_p * len(self.sims))(*[s._h.value for s in self.sims])
        h = ct.c_void_p()
        check(lib().rw_batch_create(arr, len(self.sims), ct.byref(h)), "rw_batch_create", None)
        self._h = h

    def step(self, n: int = 1) -> None:
        check(lib().rw_batch_step(self._h, n, None), "rw_batch_step", None)

    def step_timed(self, n: int) -> float:
        ms = ct.c_double(0.0)
        check(lib().rw_batch_step(self._h, n, ct.byref(ms)), "rw_batch_step", None)
        return ms.value

    def synchronize(self) -> None:
        check(lib().rw_batch_synchronize(self._h), "rw_batch_synchronize", None)

    def wall_force(self, mode: int = 0, wall_id: int = 10, strip: Optional[Sequence[float]] = None) -> np.ndarray:
        """LoquatSph.wall_force of every case (rows in the batch's order), one copy back."""
        out = (ct.c_double * (3 * len(self.sims)))()
        sp = None
        if strip is not None:
            sa = (ct.c_double * 3)(*strip)
            sp = ct.cast(sa, ct.c_void_p)
        check(lib().rw_batch_wall_force(self._h, mode, wall_id, sp, out), "rw_batch_wall_force", None)
        return np.array(out[:]).reshape(len(self.sims), 3)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().rw_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
