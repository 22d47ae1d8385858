"""ctypes mirror of the structs and constants of include/retainwall.h."""
from __future__ import annotations

import ctypes as ct
from typing import Dict

import numpy as np

RW_OK, RW_EINVAL, RW_ENOENT, RW_EIO, RW_EFORMAT, RW_ECUDA, RW_ENOMEM, RW_EDEVICE, RW_ETIMEDOUT, RW_ESTATE = range(10)
STATUS_NAMES = {0: "RW_OK", 1: "RW_EINVAL", 2: "RW_ENOENT", 3: "RW_EIO", 4: "RW_EFORMAT", 5: "RW_ECUDA",
                6: "RW_ENOMEM", 7: "RW_EDEVICE", 8: "RW_ETIMEDOUT", 9: "RW_ESTATE"}
MODEL_MAX, MATERIAL_SIZE, MOTION_MAX, TABLE_MAX = 10, 15, 10, 10
OPT_WALL_FRICTION, OPT_COMPAT_CONTACT, OPT_INTERACTION_KERNEL, OPT_STRICT_FP, OPT_MIXED_PRECISION = 0, 1, 2, 3, 4
OPT_LIST_SKIN = 5
OPT_GRAPH_GATES = 6
OPT_CLOSURE_MAX_ERR = 7
OPT_WALK_THREADS = 8
OPT_INTEGRATOR_THREADS = 9
OPT_ASYNC_SAVE = 10

# rw_array ids and their row shapes (columns, integer?)
ARRAYS: Dict[str, int] = {
    "codes": 0, "cellpos": 1, "pospres": 2, "pospres_ori": 3, "velrhop": 4, "idmassidx": 5, "str": 6, "stn": 7,
    "normal_m": 8, "contact_mag": 9, "contact_var": 10, "accad": 11, "spin": 12, "acestn": 13, "pospres_ini": 14,
    "velrhop_ini": 15, "str_ini": 16, "stn_ini": 17, "part_idx": 18, "cell_beg": 19, "cell_end": 20, "pos_abs": 21,
}
_COLS = {"codes": 4, "cellpos": 4, "str": 6, "stn": 6, "acestn": 6, "str_ini": 6, "stn_ini": 6, "contact_mag": 9,
         "part_idx": 1, "cell_beg": 1, "cell_end": 1}
_INT = {"codes", "cellpos", "part_idx", "cell_beg", "cell_end"}


def array_spec(name: str, info: "Info"):
    """(rows, cols, dtype) of an exported array for a context described by ``info``."""
    cols = _COLS.get(name, 4)
    if name == "normal_m":
        rows = info.npb
    elif name in ("cell_beg", "cell_end"):
        rows = info.ncell
    else:
        rows = info.np
    if name in _INT:
        dt = np.int32
    else:
        dt = np.float32 if info.scalar_bytes == 4 else np.float64
    return rows, cols, dt


class Motion(ct.Structure):
    _fields_ = [
        ("is_translation", ct.c_int32), ("n_trans", ct.c_int32),
        ("trans_time", ct.c_double * TABLE_MAX), ("trans_vel", (ct.c_double * 3) * TABLE_MAX),
        ("trans_acc", (ct.c_double * 3) * TABLE_MAX),
        ("is_rotation", ct.c_int32), ("pattern", ct.c_int32), ("n_rot", ct.c_int32), ("pad_", ct.c_int32),
        ("pos_rp", ct.c_double * 3), ("rotat_vel", ct.c_double * 3), ("rotat_time", ct.c_double * TABLE_MAX),
        ("rotat_acc", (ct.c_double * 3) * TABLE_MAX),
    ]


class CaseParams(ct.Structure):
    _fields_ = [
        ("dim", ct.c_int32), ("periodbound", ct.c_int32), ("n_motion", ct.c_int32), ("np", ct.c_int32),
        ("npb", ct.c_int32), ("npm", ct.c_int32), ("n_model", ct.c_int32),
        ("stress_shepard_filter", ct.c_int32), ("dynamic_time_step", ct.c_int32),
        ("integration_method", ct.c_int32), ("viscosity_type", ct.c_int32),
        ("output_number", ct.c_int32), ("output_format", ct.c_int32), ("pad_", ct.c_int32),
        ("planeleft", ct.c_double * 4), ("planeright", ct.c_double * 4),
        ("domain_size", ct.c_double * 3), ("domain_min", ct.c_double * 3),
        ("dr", ct.c_double), ("hdr", ct.c_double), ("gravity", ct.c_double * 3), ("rho0_m", ct.c_double),
        ("damping", ct.c_double), ("model_par", (ct.c_double * MATERIAL_SIZE) * MODEL_MAX),
        ("artificial_viscosity_alpha_m", ct.c_double), ("cs_m", ct.c_double), ("cfl", ct.c_double),
        ("artificial_pressure_coefficient_material", ct.c_double),
        ("time_max", ct.c_double), ("time", ct.c_double), ("dt", ct.c_double), ("output_frequency", ct.c_double),
        ("wall_friction", ct.c_double),
        ("motion", Motion * MOTION_MAX),
    ]


class Case(ct.Structure):
    _fields_ = [
        ("params", CaseParams),
        ("codes", ct.POINTER(ct.c_int32)), ("pospres", ct.POINTER(ct.c_double)),
        ("velrhop", ct.POINTER(ct.c_double)), ("idmassidx", ct.POINTER(ct.c_double)),
        ("stress", ct.POINTER(ct.c_double)), ("strain", ct.POINTER(ct.c_double)),
        ("normal", ct.POINTER(ct.c_double)),
    ]


class Info(ct.Structure):
    _fields_ = [
        ("np", ct.c_int32), ("npb", ct.c_int32), ("npm", ct.c_int32), ("np_delete_m", ct.c_int32),
        ("ncell", ct.c_int32), ("step", ct.c_int32), ("scalar_bytes", ct.c_int32), ("device_err", ct.c_int32),
        ("cell_num", ct.c_int32 * 3), ("n_motion", ct.c_int32),
        ("time", ct.c_double), ("dt", ct.c_double), ("h", ct.c_double), ("dr", ct.c_double),
        ("n_sorts", ct.c_int32), ("n_list_reuse", ct.c_int32),
        ("n_search_skipped", ct.c_int32), ("n_scan_skipped", ct.c_int32), ("n_build_skipped", ct.c_int32),
        ("graph_kernels", ct.c_int32), ("search_body_kernels", ct.c_int32), ("n_list_updates", ct.c_int32),
        ("time_max", ct.c_double), ("output_frequency", ct.c_double),
        ("ix_kernel", ct.c_int32), ("walk_threads", ct.c_int32), ("integrator_threads", ct.c_int32),
        ("n_lists_rebuilt", ct.c_int32), ("build_body_kernels", ct.c_int32), ("pad_", ct.c_int32),
    ]


def case_struct(case, keep: list) -> Case:
    """Fill an rw_case from a ``cases.Case``; ``keep`` receives the numpy buffers that
    must stay alive while the struct is in use."""
    p = case.params
    c = Case()
    q = c.params
    q.dim = int(p["dim"])
    q.periodbound = int(p["periodbound"])
    q.n_motion = int(p["n_motion"])
    q.np, q.npb, q.npm = case.np_, case.npb, case.npm
    q.n_model = int(p["n_model"])
    for k in ("stress_shepard_filter", "dynamic_time_step", "integration_method", "viscosity_type",
              "output_number", "output_format"):
        setattr(q, k, int(p[k]))
    if q.periodbound:
        for k in range(4):
            q.planeleft[k] = float(p["planeleft"][k])
            q.planeright[k] = float(p["planeright"][k])
    for k, ax in enumerate("xyz"):
        q.domain_size[k] = float(p[f"domain_size_{ax}"])
        q.domain_min[k] = float(p[f"domain_min_{ax}"])
        q.gravity[k] = float(p[f"gravity_{ax}"])
    q.dr, q.hdr = float(p["dr"]), float(p["hdr"])
    q.rho0_m, q.damping = float(p["rho0_m"]), float(p["damping"])
    for i in range(int(p["n_model"])):
        for j in range(MATERIAL_SIZE):
            q.model_par[i][j] = float(p[f"model-{i}-par-{j}"])
    q.artificial_viscosity_alpha_m = float(p.get("artificial_viscosity_alpha_m", 0.0))
    for k in ("cs_m", "cfl", "artificial_pressure_coefficient_material", "time_max", "time", "dt",
              "output_frequency"):
        setattr(q, k, float(p[k]))
    q.wall_friction = float(p.get("wall-friction-coefficient", 0.58108))
    for i, m in enumerate(case.motions[:MOTION_MAX]):
        mm = q.motion[i]
        mm.is_translation = int(m.is_translation)
        mm.n_trans = len(m.trans_time)
        for j in range(mm.n_trans):
            mm.trans_time[j] = m.trans_time[j]
            for k in range(3):
                mm.trans_vel[j][k] = m.trans_vel[j][k]
                mm.trans_acc[j][k] = m.trans_acc[j][k]
        mm.is_rotation = int(m.is_rotation)
        mm.pattern = int(m.pattern)
        mm.n_rot = len(m.rotat_time)
        for k in range(3):
            mm.pos_rp[k] = m.pos_rp[k]
            mm.rotat_vel[k] = m.rotat_vel[k]
        for j in range(mm.n_rot):
            mm.rotat_time[j] = m.rotat_time[j]
            for k in range(3):
                mm.rotat_acc[j][k] = m.rotat_acc[j][k]

    def buf(a, dt, ptr):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data_as(ct.POINTER(ptr))

    c.codes = buf(case.codes, np.int32, ct.c_int32)
    c.pospres = buf(case.pospres, np.float64, ct.c_double)
    c.velrhop = buf(case.velrhop, np.float64, ct.c_double)
    c.idmassidx = buf(case.idmassidx, np.float64, ct.c_double)
    c.stress = buf(case.stress, np.float64, ct.c_double)
    c.strain = buf(case.strain, np.float64, ct.c_double)
    c.normal = buf(case.normal if case.npb else np.zeros((1, 4)), np.float64, ct.c_double)
    return c
