"""Case generators and the reference's case-file formats.

The reference reads a project as three text files (``<project>.xml``,
``<project>.dat``, ``<project>.motion``) through ``LoquatIo::LoadParameters`` /
``LoadParticles`` (src/loquat_io.cu:75-312) and its own generator writes them with
``SaveXmlFile`` / ``SaveDatFile`` / ``SaveMotionFile`` (src/GenCase.cu:70-227).
This module builds the retaining-wall and column-collapse cases used for parity and
measurement and reads/writes that exact layout:

* ``.xml``: ``<parameters>`` with typed children (``int``, ``scalar``, ``model_mat``,
  ``dimension``, ``bool``), same tag names as src/GenCase.cu:119-204;
* ``.dat``: one particle per line, boundary first (31 columns incl. the normal), then
  material (27 columns): ``codes(4) pos(4) velrhop(4) id mass idx.w str(6) stn(6)``;
* ``.motion``: per body ``is_trans is_rot``, translation table, rotation header/table.

Particle codes follow src/GenCase.cu:473,494: ``codes.x`` block id (>= 10 is a contact
wall), ``.y`` status (0 Fix, 1 NonFix), ``.z`` model, ``.w`` material or motion index.
All floating values are rounded to float32 before they are written, and written with
9 significant digits, so a float build reads back exactly the generated values.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, List, Optional

import numpy as np

INT_MIN = -2147483648
FIX, NONFIX = 0, 1
RIGID, DP_EPP, MUI_DP_EPP, HYPO_BASIC, HYPO_CS = 0, 1, 2, 3, 4
CUBOID, CIRCLE = 0, 1

# Tag order and types of the parameter file (src/GenCase.cu:119-204, read back by
# src/loquat_io.cu:132-197).
_XML_HEAD = [
    ("dimension-of-problem", "dimension", "dim"),
    ("number-of-motion", "int", "n_motion"),
    ("period-bound", "bool", "periodbound"),
]
_XML_PLANES = [
    ("planeleft-A", "planeleft", 0), ("planeleft-B", "planeleft", 1),
    ("planeleft-C", "planeleft", 2), ("planeleft-D", "planeleft", 3),
    ("planeright-A", "planeright", 0), ("planeright-B", "planeright", 1),
    ("planeright-C", "planeright", 2), ("planeright-D", "planeright", 3),
]
_XML_BODY = [
    ("number-of-particles", "int", "np"),
    ("number-of-boundary-particles", "int", "npb"),
    ("number-of-material-particles", "int", "npm"),
    ("domain-size-x", "scalar", "domain_size_x"),
    ("domain-size-y", "scalar", "domain_size_y"),
    ("domain-size-z", "scalar", "domain_size_z"),
    ("domain-min-x", "scalar", "domain_min_x"),
    ("domain-min-y", "scalar", "domain_min_y"),
    ("domain-min-z", "scalar", "domain_min_z"),
    ("particle-size", "scalar", "dr"),
    ("h-over-dr", "scalar", "hdr"),
    ("acceleration-x", "scalar", "gravity_x"),
    ("acceleration-y", "scalar", "gravity_y"),
    ("acceleration-z", "scalar", "gravity_z"),
    ("reference-density-material", "scalar", "rho0_m"),
    ("damping", "scalar", "damping"),
    ("number-of-model", "int", "n_model"),
]
_XML_TAIL = [
    ("stress-shepard-filter", "int", "stress_shepard_filter"),
    ("dynamic-time-step", "int", "dynamic_time_step"),
    ("integration-method", "int", "integration_method"),
    ("viscosity-type", "int", "viscosity_type"),
]
_XML_TAIL2 = [
    ("speed-of-sound-material", "scalar", "cs_m"),
    ("cfl-number", "scalar", "cfl"),
    ("artificial-pressure-coefficient-material", "scalar", "artificial_pressure_coefficient_material"),
    ("time-max", "scalar", "time_max"),
    ("time", "scalar", "time"),
    ("time-step", "scalar", "dt"),
    ("output-frequency", "scalar", "output_frequency"),
    ("output-number", "int", "output_number"),
    ("output-format", "int", "output_format"),
]
# Project extension (optional, typed, ignored by the reference's loader which parses and
# drops unknown typed tags): wall-soil Coulomb coefficient of the contact wall.  The
# reference hard-codes 0.58108 (src/particle_interaction.cu:188-189).
WALL_FRICTION_TAG = "wall-friction-coefficient"
REFERENCE_WALL_FRICTION = 0.58108


def f32(x) -> float:
    return float(np.float32(x))


@dataclasses.dataclass
class MotionTable:
    """One rigid body's motion table (``MotionTable``, src/types.h:77-97)."""

    is_translation: bool = False
    trans_time: List[float] = dataclasses.field(default_factory=list)
    trans_vel: List[List[float]] = dataclasses.field(default_factory=list)
    trans_acc: List[List[float]] = dataclasses.field(default_factory=list)
    is_rotation: bool = False
    pattern: int = CUBOID
    pos_rp: List[float] = dataclasses.field(default_factory=lambda: [0.0, 0.0, 0.0])
    rotat_vel: List[float] = dataclasses.field(default_factory=lambda: [0.0, 0.0, 0.0])
    rotat_time: List[float] = dataclasses.field(default_factory=list)
    rotat_acc: List[List[float]] = dataclasses.field(default_factory=list)


@dataclasses.dataclass
class Case:
    """A project: parameters (XML) + particles (.dat) + motion tables (.motion).

    Arrays use the reference's per-particle layout (np rows; boundary first):
    ``codes`` int32 (np,4); ``pospres``/``velrhop``/``idmassidx`` float64 (np,4);
    ``stress``/``strain`` (np,6) as xx yy zz xy xz yz; ``normal`` (npb,4).
    ``idmassidx[:,2]`` is the original index, as LoadParticles sets it.
    """

    params: Dict[str, object]
    codes: np.ndarray
    pospres: np.ndarray
    velrhop: np.ndarray
    idmassidx: np.ndarray
    stress: np.ndarray
    strain: np.ndarray
    normal: np.ndarray
    motions: List[MotionTable]
    name: str = "case"

    @property
    def np_(self) -> int:
        return int(self.codes.shape[0])

    @property
    def npb(self) -> int:
        return int(self.normal.shape[0])

    @property
    def npm(self) -> int:
        return self.np_ - self.npb


def hypocs_model(phi_c_deg: float, e0: float, rho0: float, *, h_s: float = 2.6e9, n: float = 0.27,
                 e_d0: float = 0.61, e_c0: float = 0.98, e_i0: float = 1.10, alpha: float = 0.18,
                 p_ref: float = 1.0e5, Ei: float = 5.0e7, Vi: float = 0.3, cohesion: float = 0.0) -> List[float]:
    """The 15-slot HypoCS parameter vector (``GetMaterial_HypoCS``, src/GenCase.cu:52-68).

    The von Wolffersdorff-style inputs map onto Wu's HypoCS slots as follows:
    e_c0 -> void_co, e_d0 -> void_min, e_i0 -> void_max, n -> xi, and the Bauer
    compression law gives lambda = (3 p_ref / h_s)^n.  beta has no counterpart.
    Ei, Vi default to the reference case's values (src/GenCase.cu:387).
    Slots 13, 14 are the density clamps rho_min = 0.8 rho0, rho_max = 1.2 rho0.
    """
    lam = (3.0 * p_ref / h_s) ** n
    m = [0.0] * 15
    m[0], m[1], m[2], m[3], m[4] = Ei, Vi, math.radians(phi_c_deg), cohesion, p_ref
    m[5], m[6], m[7], m[8] = e_c0, lam, n, alpha
    m[9], m[10], m[11], m[12] = e_d0, e_i0, e0, rho0
    m[13], m[14] = rho0 * 0.8, rho0 * 1.2
    return [f32(v) for v in m]


def hypo_basic_model(rho0: float, *, Ei: float = 20.0e6, Vi: float = 0.3, phi_c_deg: float = 35.0,
                     cohesion: float = 0.0, p_ref: float = 1.0e5) -> List[float]:
    """HypoBasic slots (``GetMaterial_HypoBasic``, src/GenCase.cu:42-50): Ei, Vi, phi_c
    [rad], cohesion, p_ref; density clamps 0.8 / 1.2 rho0 in slots 13, 14.  Defaults are
    the reference generator's HypoBasic material (src/GenCase.cu:380-383)."""
    m = [0.0] * 15
    m[0], m[1], m[2], m[3], m[4] = Ei, Vi, math.radians(phi_c_deg), cohesion, p_ref
    m[13], m[14] = rho0 * 0.8, rho0 * 1.2
    return [f32(v) for v in m]


def _dp_fit(tan_x: float) -> float:
    """Drucker-Prager coefficient matched to Mohr-Coulomb in plane strain:
    3 tan x / sqrt(9 + 12 tan^2 x)."""
    return 3.0 * tan_x / math.sqrt(9.0 + 12.0 * tan_x * tan_x)


def dp_model(rho0: float, *, E: float = 1.5e6, V: float = 0.2, phi_deg: float = 25.0, psi_deg: float = 0.0,
             cohesion: float = 0.0) -> List[float]:
    """Elastic-perfectly-plastic Drucker-Prager slots (``GetMaterial_DP_EPP``,
    src/GenCase.cu:16-25): bulk modulus E / 3(1 - 2V), shear modulus E / 2(1 + V), the
    friction, dilatancy and cohesion coefficients of the plane-strain fit, density clamps
    in slots 13, 14.  Defaults are the reference generator's DP material
    (src/GenCase.cu:308-312)."""
    tp, ts = math.tan(math.radians(phi_deg)), math.tan(math.radians(psi_deg))
    m = [0.0] * 15
    m[0] = E / (3.0 * (1.0 - 2.0 * V))
    m[1] = E / (2.0 * (1.0 + V))
    m[2], m[3] = _dp_fit(tp), _dp_fit(ts)
    m[4] = 3.0 * cohesion / math.sqrt(9.0 + 12.0 * tp * tp)
    m[13], m[14] = rho0 * 0.8, rho0 * 1.2
    return [f32(v) for v in m]


def mui_dp_model(rho0: float, *, E: float = 1.5e6, V: float = 0.3, phi1_deg: float = 20.9, phi2_deg: float = 32.76,
                 I0: float = 0.279, rho_g: float = 2650.0, d_grain: float = 0.5e-3, lam: float = 0.1) -> List[float]:
    """mu(I)-enhanced Drucker-Prager slots (``GetMaterial_MuI_DP_EPP``,
    src/GenCase.cu:27-40): bulk and shear modulus, mu_s = tan phi1, mu_2 = tan phi2, I0,
    grain density, grain diameter, the rate regularisation lambda [1/s]; density clamps in
    slots 13, 14.  The defaults are common granular-flow values (mu_s, mu_2, I0 of
    glass-bead flows); the reference's generator sets none."""
    m = [0.0] * 15
    m[0] = E / (3.0 * (1.0 - 2.0 * V))
    m[1] = E / (2.0 * (1.0 + V))
    m[2], m[3] = math.tan(math.radians(phi1_deg)), math.tan(math.radians(phi2_deg))
    m[4], m[5], m[6], m[7] = I0, rho_g, d_grain, lam
    m[13], m[14] = rho0 * 0.8, rho0 * 1.2
    return [f32(v) for v in m]


MODELS = {"hypo_cs": HYPO_CS, "hypo_basic": HYPO_BASIC, "dp": DP_EPP, "mui_dp": MUI_DP_EPP}


def _base_params(dr: float, hdr: float, cs: float, cfl: float, rho0: float, model: List[float]) -> Dict[str, object]:
    p: Dict[str, object] = dict(
        dim=3, n_motion=0, periodbound=0,
        dr=f32(dr), hdr=f32(hdr), gravity_x=0.0, gravity_y=0.0, gravity_z=f32(-9.81),
        rho0_m=f32(rho0), damping=0.0, n_model=1,
        stress_shepard_filter=0, dynamic_time_step=1, integration_method=1, viscosity_type=1,
        artificial_viscosity_alpha_m=f32(1.5), cs_m=f32(cs), cfl=f32(cfl),
        artificial_pressure_coefficient_material=f32(0.01),
        time_max=1.0, time=0.0, dt=f32(1e-6), output_frequency=f32(0.01), output_number=0, output_format=2,
        domain_min_x=0.0, domain_min_y=0.0, domain_min_z=0.0,
    )
    for j in range(15):
        p[f"model-0-par-{j}"] = model[j]
    return p


class _Builder:
    def __init__(self):
        self.codes: List[np.ndarray] = []
        self.pos: List[np.ndarray] = []
        self.normal: List[np.ndarray] = []
        self.mcodes: List[np.ndarray] = []
        self.mpos: List[np.ndarray] = []
        self.mstr: List[np.ndarray] = []

    def box(self, lo, hi, dr, code, normal):
        """Boundary lattice filling [lo, hi) with spacing dr (cell centres)."""
        n = [max(1, int(round((hi[k] - lo[k]) / dr))) for k in range(3)]
        ax = [lo[k] + dr * (np.arange(n[k]) + 0.5) for k in range(3)]
        g = np.stack(np.meshgrid(*ax, indexing="ij"), -1).reshape(-1, 3)
        self.pos.append(g)
        self.codes.append(np.tile(np.asarray(code, np.int64), (len(g), 1)))
        self.normal.append(np.tile(np.asarray(normal, np.float64), (len(g), 1)))

    def case(self, params, motions, name, rho0, mass, seed_dummy=None) -> Case:
        bpos = np.concatenate(self.pos) if self.pos else np.zeros((0, 3))
        bcodes = np.concatenate(self.codes) if self.codes else np.zeros((0, 4), np.int64)
        bnorm = np.concatenate(self.normal) if self.normal else np.zeros((0, 4))
        mpos = np.concatenate(self.mpos)
        mcodes = np.concatenate(self.mcodes)
        mstr = np.concatenate(self.mstr)
        npb, npm = len(bpos), len(mpos)
        npt = npb + npm
        codes = np.concatenate([bcodes, mcodes]).astype(np.int32)
        pospres = np.zeros((npt, 4))
        pospres[:npb, :3] = bpos
        pospres[npb:, :3] = mpos
        velrhop = np.zeros((npt, 4))
        velrhop[npb:, 3] = rho0
        idm = np.zeros((npt, 4))
        idm[npb:, 0] = 100.0
        idm[npb:, 1] = mass
        idm[npb:, 3] = 100.0
        idm[:, 2] = np.arange(npt)
        stress = np.zeros((npt, 6))
        stress[npb:] = mstr
        strain = np.zeros((npt, 6))
        f = lambda a: a.astype(np.float32).astype(np.float64)
        params = dict(params)
        params.update(np=npt, npb=npb, npm=npm)
        return Case(params, codes, f(pospres), f(velrhop), f(idm), f(stress), strain, f(bnorm), motions, name)


def _soil(b: _Builder, x0, y0, z0, nx, ny, nz, dr, rng, jitter, rho0, g, K0, model_id=0, model_type=HYPO_CS):
    """Soil lattice with uniform jitter and geostatic stress sigma_zz = rho g depth."""
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    pos = np.stack([x0 + (ix + 0.5) * dr, y0 + (iy + 0.5) * dr, z0 + (iz + 0.5) * dr], -1).reshape(-1, 3)
    if jitter > 0:
        pos = pos + rng.uniform(-jitter * dr, jitter * dr, size=pos.shape)
    top = z0 + nz * dr
    szz = rho0 * g * (top - pos[:, 2])  # g < 0: compressive (negative) stress
    s = np.zeros((len(pos), 6))
    s[:, 0] = szz * K0
    s[:, 1] = szz * K0
    s[:, 2] = szz
    b.mpos.append(pos)
    b.mcodes.append(np.tile(np.asarray([6, NONFIX, model_type, model_id], np.int64), (len(pos), 1)))
    b.mstr.append(s)


def column_collapse(nx=24, ny=24, nz=48, dx=0.005, seed=1, phi_c=30.0, e0=0.70, rho0=1850.0,
                    hdr=1.2, jitter=0.05, cs=60.0, cfl=0.1, runout=4.0, name="column", model="hypo_cs") -> Case:
    """Granular column collapse: soil column in a box whose +x wall is absent at t = 0.

    Frictionless (free-slip, normal.w = +1) Adami walls on -x, -y, +y around the column,
    a no-slip floor (normal.w = -1) extending ``runout`` column widths in +x.  Geostatic
    stress with K0 = 1 - sin(phi_c).  dt = cfl h / cs (src/loquat.cu:366-374).
    ``model`` selects the soil's constitutive law (a key of ``MODELS``): HypoCS with the
    configuration's parameters (default), or the reference generator's HypoBasic, DP or
    a mu(I)-DP material.
    """
    rng = np.random.default_rng(seed)
    h = dx * hdr
    bt = math.ceil(2.0 * hdr) * dx
    margin = 4.0 * h
    W, D, H = nx * dx, ny * dx, nz * dx
    x0, y0, z0 = margin + bt, margin + bt + W, margin + bt  # room in -y for lateral spreading
    L = W * (1.0 + runout)
    if model not in MODELS:
        raise ValueError(f"unknown model {model!r}")
    mat = {"hypo_cs": lambda: hypocs_model(phi_c, e0, rho0), "hypo_basic": lambda: hypo_basic_model(rho0),
           "dp": lambda: dp_model(rho0), "mui_dp": lambda: mui_dp_model(rho0)}[model]()
    p = _base_params(dx, hdr, cs, cfl, rho0, mat)
    b = _Builder()
    # floor (no slip), wide enough for run-out and lateral spreading
    b.box((x0 - bt, y0 - D - bt, z0 - bt), (x0 + L, y0 + 2 * D + bt, z0), dx, (0, FIX, INT_MIN, INT_MIN), (0, 0, 1, -1))
    # -x wall and the two y walls around the column (free slip)
    b.box((x0 - bt, y0 - bt, z0), (x0, y0 + D + bt, z0 + H + 2 * h), dx, (1, FIX, INT_MIN, INT_MIN), (1, 0, 0, 1))
    b.box((x0, y0 - bt, z0), (x0 + W, y0, z0 + H + 2 * h), dx, (2, FIX, INT_MIN, INT_MIN), (0, 1, 0, 1))
    b.box((x0, y0 + D, z0), (x0 + W, y0 + D + bt, z0 + H + 2 * h), dx, (3, FIX, INT_MIN, INT_MIN), (0, -1, 0, 1))
    K0 = 1.0 - math.sin(math.radians(phi_c))
    _soil(b, x0, y0, z0, nx, ny, nz, dx, rng, jitter, rho0, -9.81, K0, model_type=MODELS[model])
    p["domain_size_x"] = f32(x0 + L + margin)
    p["domain_size_y"] = f32(y0 + 2 * D + bt + margin)
    p["domain_size_z"] = f32(z0 + H + 2 * h + margin)
    return b.case(p, [], name, rho0, f32(rho0 * dx ** 3))


def retaining_wall(nx=200, ny=80, nz=120, dx=0.0025, seed=2, phi_c=30.0, e0=0.65, rho0=1850.0, hdr=1.2,
                   jitter=0.05, cs=60.0, cfl=0.1, mode="active", wall_speed=1.0e-3, rot_speed=0.005,
                   wall_friction: Optional[float] = None, periodic_y: bool = False, name="wall") -> Case:
    """Rigid retaining wall against hypoplastic sand.

    The soil block starts at x = 0.04 + bt, z = 0.04 + bt, the placement of the
    reference's own case (src/GenCase.cu:418-477), so the reference's hard-coded wall
    strip (src/utilities.cu:619-621) covers the soil next to the moving wall.
    The moving wall is a contact block (codes.x = 10, NonFix, motion 0); the far wall
    and the y side walls are free-slip Adami walls; the floor is no-slip.
    ``mode``: ``active`` (wall moves -x at wall_speed), ``passive`` (+x), or
    ``rotation`` (about the toe, top moving away from the soil at rot_speed rad/s).
    Wall friction defaults to delta = 2/3 phi_c (mu = tan delta).
    ``periodic_y``: no y side walls; the planes y = y0 and y = y0 + W are periodic
    (``period-bound``, planeleft = (0, 1, 0, -y0), planeright = (0, -1, 0, y0 + W)), and
    the floor and both x walls span exactly one period in y.
    """
    rng = np.random.default_rng(seed)
    h = dx * hdr
    bt = math.ceil(2.0 * hdr) * dx
    L, W, H = nx * dx, ny * dx, nz * dx
    x0 = y0 = z0 = 0.04 + bt
    top = z0 + H + 2 * h
    model = hypocs_model(phi_c, e0, rho0)
    p = _base_params(dx, hdr, cs, cfl, rho0, model)
    b = _Builder()
    yb = 0.0 if periodic_y else bt  # y extent of the floor and x walls beyond the soil
    b.box((x0 - bt, y0 - yb, z0 - bt), (x0 + L + bt, y0 + W + yb, z0), dx, (0, FIX, INT_MIN, INT_MIN), (0, 0, 1, -1))
    if not periodic_y:
        b.box((x0, y0 - bt, z0), (x0 + L, y0, top), dx, (2, FIX, INT_MIN, INT_MIN), (0, 1, 0, 1))
        b.box((x0, y0 + W, z0), (x0 + L, y0 + W + bt, top), dx, (3, FIX, INT_MIN, INT_MIN), (0, -1, 0, 1))
    b.box((x0 + L, y0 - yb, z0), (x0 + L + bt, y0 + W + yb, top), dx, (4, FIX, INT_MIN, INT_MIN), (-1, 0, 0, 1))
    b.box((x0 - bt, y0 - yb, z0), (x0, y0 + W + yb, top), dx, (10, NONFIX, INT_MIN, 0), (1, 0, 0, 1))
    if periodic_y:
        p["periodbound"] = 1
        p["planeleft"] = [0.0, 1.0, 0.0, -f32(y0)]
        p["planeright"] = [0.0, -1.0, 0.0, f32(y0 + W)]
    K0 = 1.0 - math.sin(math.radians(phi_c))
    _soil(b, x0, y0, z0, nx, ny, nz, dx, rng, jitter, rho0, -9.81, K0)
    margin = 0.04
    p["domain_size_x"] = f32(x0 + L + bt + margin)
    p["domain_size_y"] = f32(y0 + W + bt + margin)
    p["domain_size_z"] = f32(top + margin)
    tmax = 1.0
    mt = MotionTable()
    if mode in ("active", "passive"):
        v = -wall_speed if mode == "active" else wall_speed
        mt.is_translation = True
        mt.trans_time = [tmax]
        mt.trans_vel = [[f32(v), 0.0, 0.0]]
        mt.trans_acc = [[0.0, 0.0, 0.0]]
    elif mode == "rotation":
        mt.is_rotation = True
        mt.pattern = CUBOID
        mt.pos_rp = [f32(x0), 0.0, f32(z0)]
        mt.rotat_vel = [0.0, f32(-rot_speed), 0.0]
        mt.rotat_time = [tmax]
        mt.rotat_acc = [[0.0, 0.0, 0.0]]
    else:
        raise ValueError(f"unknown wall mode {mode!r}")
    p["n_motion"] = 1
    p["time_max"] = tmax
    mu = math.tan(2.0 / 3.0 * math.radians(phi_c)) if wall_friction is None else wall_friction
    p[WALL_FRICTION_TAG] = f32(mu)
    return b.case(p, [mt], name, rho0, f32(rho0 * dx ** 3))


def batch_sweep(n_cases=64, seed=5, n_lo=50_000, n_hi=400_000, dx_lo=0.0025, dx_hi=0.005):
    """Specs of the batched sweep: sizes U[n_lo, n_hi] particles, dx U[dx_lo, dx_hi],
    phi_c U[28, 40] deg, e0 U[0.55, 0.80], wall mode uniform over
    {active, passive, rotation}.  The soil block keeps the 5:2:3 aspect of the single
    retaining-wall case and is scaled so that nx*ny*nz is close to the drawn size."""
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(n_cases):
        n = rng.uniform(n_lo, n_hi)
        dx = rng.uniform(dx_lo, dx_hi)
        phi = rng.uniform(28.0, 40.0)
        e0 = rng.uniform(0.55, 0.80)
        mode = ("active", "passive", "rotation")[int(rng.integers(0, 3))]
        s = (n / 30.0) ** (1.0 / 3.0)  # nx:ny:nz = 5:2:3 -> 30 s^3 particles
        nx, ny, nz = max(4, int(round(5 * s))), max(4, int(round(2 * s))), max(4, int(round(3 * s)))
        specs.append(dict(nx=nx, ny=ny, nz=nz, dx=float(dx), phi_c=float(phi), e0=float(e0), mode=mode,
                          seed=int(seed * 1000 + k), name=f"case{k:02d}"))
    return specs


# ----------------------------------------------------------------------------------------
# Reference file formats
# ----------------------------------------------------------------------------------------

def _fmt(v) -> str:
    if isinstance(v, (bool, np.bool_)):
        return str(int(v))
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    return "%.9g" % float(v)


def write_xml(path: str, params: Dict[str, object]) -> None:
    """``SaveXmlFile`` layout (src/GenCase.cu:119-204)."""
    p = params
    out = ['<?xml version="1.0" encoding="utf-8" ?>', "<parameters>"]

    def tag(name, typ, val):
        out.append(f'  <{name} type="{typ}">{_fmt(val)}</{name}>')

    for name, typ, key in _XML_HEAD:
        tag(name, typ, p[key])
    if int(p.get("periodbound", 0)):
        for name, key, k in _XML_PLANES:
            tag(name, "scalar", p[key][k])
    for name, typ, key in _XML_BODY:
        tag(name, typ, p[key])
    for i in range(int(p["n_model"])):
        for j in range(15):
            tag(f"model-{i}-par-{j}", "scalar", p[f"model-{i}-par-{j}"])
    for name, typ, key in _XML_TAIL:
        tag(name, typ, p[key])
    if int(p["viscosity_type"]) == 1:
        tag("artificial-viscosity-alpha-material", "scalar", p["artificial_viscosity_alpha_m"])
    for name, typ, key in _XML_TAIL2:
        tag(name, typ, p[key])
    if WALL_FRICTION_TAG in p:
        tag(WALL_FRICTION_TAG, "scalar", p[WALL_FRICTION_TAG])
    out.append("</parameters>")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def read_xml(path: str) -> Dict[str, object]:
    """Typed parameter map (src/loquat_io.cu:97-127); unknown typed tags are kept."""
    import xml.etree.ElementTree as ET

    root = ET.parse(path).getroot()
    raw: Dict[str, object] = {}
    for el in root:
        typ = el.get("type")
        txt = (el.text or "").strip()
        if typ in ("int", "model_mat", "dimension"):
            raw[el.tag] = int(float(txt)) if txt else 0
        elif typ == "scalar":
            raw[el.tag] = float(txt)
        elif typ == "bool":
            raw[el.tag] = int(bool(float(txt)))
        else:
            raise ValueError(f"Wrong data type for {el.tag}")
    p: Dict[str, object] = {}
    for name, _, key in _XML_HEAD + _XML_BODY + _XML_TAIL + _XML_TAIL2:
        if name not in raw:
            raise KeyError(f"{name} does not exist in the xml file")
        p[key] = raw[name]
    if p["periodbound"]:
        p["planeleft"] = [raw[n] for n, key, _ in _XML_PLANES if key == "planeleft"]
        p["planeright"] = [raw[n] for n, key, _ in _XML_PLANES if key == "planeright"]
    for i in range(int(p["n_model"])):
        for j in range(15):
            p[f"model-{i}-par-{j}"] = raw[f"model-{i}-par-{j}"]
    if int(p["viscosity_type"]) == 1:
        p["artificial_viscosity_alpha_m"] = raw["artificial-viscosity-alpha-material"]
    if WALL_FRICTION_TAG in raw:
        p[WALL_FRICTION_TAG] = raw[WALL_FRICTION_TAG]
    return p


def write_dat(path: str, case: Case) -> None:
    """``SaveDatFile`` layout (src/GenCase.cu:70-116): boundary rows carry the normal."""
    npb = case.npb
    ints = case.codes.astype(np.int64)
    fl = np.concatenate([case.pospres, case.velrhop, case.idmassidx[:, [0, 1, 3]], case.stress, case.strain], 1)
    with open(path, "w") as f:
        for lo, hi, with_n in ((0, npb, True), (npb, case.np_, False)):
            if hi <= lo:
                continue
            cols = [ints[lo:hi, k].astype(str) for k in range(4)]
            cols += [np.char.mod("%.9g", fl[lo:hi, k]) for k in range(fl.shape[1])]
            if with_n:
                cols += [np.char.mod("%.9g", case.normal[:, k]) for k in range(4)]
            rows = cols[0]
            for c in cols[1:]:
                rows = np.char.add(np.char.add(rows, " "), c)
            f.write("\n".join(rows.tolist()))
            f.write("\n")


def read_dat(path: str, np_: int, npb: int):
    """Inverse of write_dat (src/loquat_io.cu:229-254)."""
    with open(path) as f:
        lines = f.read().split("\n")
    b = np.array([l.split() for l in lines[:npb]], dtype=np.float64).reshape(npb, 31)
    m = np.array([l.split() for l in lines[npb:np_]], dtype=np.float64).reshape(np_ - npb, 27)
    allr = np.concatenate([b[:, :27], m], 0)
    codes = allr[:, 0:4].astype(np.int64).astype(np.int32)
    pospres = allr[:, 4:8]
    velrhop = allr[:, 8:12]
    idm = np.zeros((np_, 4))
    idm[:, 0] = allr[:, 12]
    idm[:, 1] = allr[:, 13]
    idm[:, 3] = allr[:, 14]
    idm[:, 2] = np.arange(np_)
    return codes, pospres, velrhop, idm, allr[:, 15:21], allr[:, 21:27], b[:, 27:31]


def write_motion(path: str, motions: List[MotionTable]) -> None:
    """``SaveMotionFile`` layout (src/GenCase.cu:206-227)."""
    out = []
    for m in motions:
        out.append(f"{int(m.is_translation)} {int(m.is_rotation)}")
        if m.is_translation:
            out.append(str(len(m.trans_time)))
            for t, v, a in zip(m.trans_time, m.trans_vel, m.trans_acc):
                out.append(" ".join(_fmt(x) for x in [t, *v, *a]))
        if m.is_rotation:
            out.append(" ".join([str(int(m.pattern))] + [_fmt(x) for x in [*m.pos_rp, *m.rotat_vel]]
                                + [str(len(m.rotat_time))]))
            for t, a in zip(m.rotat_time, m.rotat_acc):
                out.append(" ".join(_fmt(x) for x in [t, *a]))
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def read_motion(path: str, n_motion: int) -> List[MotionTable]:
    """src/loquat_io.cu:266-303."""
    with open(path) as f:
        tok = f.read().split()
    it = iter(tok)
    nxt = lambda: next(it)
    out = []
    for _ in range(n_motion):
        m = MotionTable()
        m.is_translation = bool(int(nxt()))
        m.is_rotation = bool(int(nxt()))
        if m.is_translation:
            n = int(nxt())
            for _ in range(n):
                vals = [float(nxt()) for _ in range(7)]
                m.trans_time.append(vals[0])
                m.trans_vel.append(vals[1:4])
                m.trans_acc.append(vals[4:7])
        if m.is_rotation:
            m.pattern = int(nxt())
            m.pos_rp = [float(nxt()) for _ in range(3)]
            m.rotat_vel = [float(nxt()) for _ in range(3)]
            n = int(nxt())
            for _ in range(n):
                vals = [float(nxt()) for _ in range(4)]
                m.rotat_time.append(vals[0])
                m.rotat_acc.append(vals[1:4])
        out.append(m)
    return out


def write_dat_native(path: str, case: Case) -> None:
    """write_dat through the native library (rw_write_case_dat: the same bytes, rows
    formatted by several host threads); for cases of millions of particles."""
    import ctypes as ct

    from . import _abi
    from ._lib import check, lib

    keep: list = []
    c = _abi.case_struct(case, keep)
    check(lib().rw_write_case_dat(ct.byref(c), path.encode()), "rw_write_case_dat", None)


def write_case(case: Case, project: str, native: Optional[bool] = None) -> None:
    """Write ``<project>.xml/.dat[/.motion]`` in the reference layout.  ``native``: write
    the particle file through the native library (default: for cases above 100k
    particles)."""
    d = os.path.dirname(project)
    if d:
        os.makedirs(d, exist_ok=True)
    write_xml(project + ".xml", case.params)
    if native is None:
        native = case.np_ > 100_000
    if native:
        write_dat_native(project + ".dat", case)
    else:
        write_dat(project + ".dat", case)
    if int(case.params.get("n_motion", 0)) > 0:
        write_motion(project + ".motion", case.motions)


def read_case(project: str) -> Case:
    p = read_xml(project + ".xml")
    codes, pos, vel, idm, s, e, nrm = read_dat(project + ".dat", int(p["np"]), int(p["npb"]))
    mot = read_motion(project + ".motion", int(p["n_motion"])) if int(p["n_motion"]) > 0 else []
    return Case(p, codes, pos, vel, idm, s, e, nrm, mot, os.path.basename(project))
