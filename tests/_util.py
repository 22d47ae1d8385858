"""Shared helpers of the test suite."""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

STATE_KEYS = ["codes", "cellpos", "pospres", "pospres_ori", "velrhop", "idmassidx", "str", "stn", "normal_m",
              "contact_mag", "contact_var"]
# Stage order of one step, with the golden stage tag each stage is compared with.
STEP_STAGES = [("begin_step", None), ("neighbor_search_p", "p0_sorted"), ("rigid_body_update", None),
               ("adami", "p1_adami"), ("find_corner", "p2_corner"), ("interaction", "p3_interaction"),
               ("predictor", "p4_predictor"), ("neighbor_search_c", "c0_sorted"), ("adami", "c1_adami"),
               ("find_corner", "c2_corner"), ("interaction", "c3_interaction"), ("corrector", "c4_corrector")]


def rel(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a))


def far_from_contact(case, cellpos, pospres, contact_var):
    """Material rows farther than one kernel support (2h) from every particle of the
    contact zone (contact_var.y <= 2h).  Inside the zone the reference's contact
    redistribution reads state that other threads are rewriting
    (src/particle_interaction.cu:147-166), which the oracle and the product resolve as
    a start-of-stage snapshot; its rounding-level differences reach the first ring of
    neighbours through the SPH sums."""
    from scipy.spatial import cKDTree

    h = case.params["dr"] * case.params["hdr"]
    mat = np.arange(case.np_) >= case.npb
    zone = mat & (contact_var[:, 1] <= 2.0 * h + 1e-12)
    if not zone.any():
        return mat
    pabs = pospres[:, :3].astype(np.float64) + cellpos[:, :3].astype(np.float64) * (2.0 * h)
    d, _ = cKDTree(pabs[zone]).query(pabs)
    return mat & ~zone & (d > 2.0 * h)


def golden(name: str):
    return np.load(os.path.join(GOLDEN, f"{name}_ref.npz"))


def mini_cases():
    from tests.golden.make_golden import mini_cases as mc

    return mc()


def load_state(sim, g, prefix="step1"):
    """Restart a simulator (oracle or GPU) from a golden full-state dump."""
    for k in STATE_KEYS:
        sim.set(k, g[f"{prefix}/{k}"])
    m = g[f"{prefix}/meta"]
    sim.set_counters(float(m[0]), int(m[1]), int(m[2]), int(m[3]))


def boundary_normal_mask(contact_mag_ref, npb, codes):
    """Rows/columns of contact_mag that are compared: everything except the Adami
    normals (columns 3..5) of contact-wall boundary particles.  Those normals are the
    direction of a sum that nearly cancels inside a 3-layer wall, i.e. rounding noise
    in the reference itself (src/adami_boundary.cu:39-41,106-110)."""
    m = np.ones(contact_mag_ref.shape, bool)
    wall = (np.arange(len(m)) < npb) & (codes[:, 0] >= 10)
    m[wall, 3:6] = False
    return m
