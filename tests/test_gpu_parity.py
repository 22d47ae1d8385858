"""Parity of the native sm_100a step (through the C ABI) with the CPU oracle and with
the reference's own GPU outputs (tests/golden).  Tolerances as in
tests/test_oracle_golden.py: integer work bit-exact; relative L2 <= 1e-5 per stage and
over 100 steps away from the contact zone; wall force within 0.5 %."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from retainwall_code_b200 import LoquatSph
from tests._util import STEP_STAGES, boundary_normal_mask, far_from_contact, golden, load_state, mini_cases, rel

pytestmark = pytest.mark.gpu

CASES = ["col_mini", "wall_mini", "per_mini"]
GPU_STAGE = {
    "begin_step": lambda s: s.step_calculation(),
    "neighbor_search_p": lambda s: s.neighbor_search(0),
    "neighbor_search_c": lambda s: s.neighbor_search(1),
    "rigid_body_update": lambda s: s.rigid_body_update(),
    "adami": lambda s: s.adami_boundary(),
    "find_corner": lambda s: s.find_corner_particle(),
    "interaction": lambda s: s.particle_interaction(),
    "predictor": lambda s: s.predictor(),
    "corrector": lambda s: s.corrector(),
}


@pytest.fixture(scope="module")
def cases():
    return mini_cases()


def _cmp(a, b, key, tag, npb=None, codes=None, tol=1e-5):
    if a.dtype.kind == "i":
        np.testing.assert_array_equal(a, b, err_msg=f"{tag}/{key}")
    elif key == "contact_mag" and npb is not None:
        m = boundary_normal_mask(b, npb, codes)
        assert rel(a[m], b[m]) < tol, (tag, key, rel(a[m], b[m]))
    else:
        assert rel(a, b) < tol, (tag, key, rel(a, b))


@pytest.mark.parametrize("name", CASES)
def test_initial_cell_list_bit_exact(cases, name):
    g = golden(name)
    s = LoquatSph(case=cases[name])
    o = Oracle(cases[name], 4)
    for k in ("part_idx", "cell_beg", "cell_end", "cellpos", "codes"):
        np.testing.assert_array_equal(s.get(k), g[f"init/{k}"] if f"init/{k}" in g else o.get(k), err_msg=k)
        np.testing.assert_array_equal(s.get(k), o.get(k), err_msg=k)
    np.testing.assert_array_equal(s.get("pospres"), o.get("pospres"))
    # the in-cell positions of the reference's own loader, bit for bit
    np.testing.assert_array_equal(s.get("pospres"), g["init/pospres"])


@pytest.mark.parametrize("name", CASES)
def test_stage_by_stage(cases, name):
    """GPU and oracle restarted from the reference's state after step 1; every stage of
    step index 1 compared with the oracle and with the reference's stage dump."""
    g = golden(name)
    c = cases[name]
    s = LoquatSph(case=c)
    o = Oracle(c, 4)
    load_state(s, g)
    load_state(o, g)
    codes = g["step1/codes"]
    for st, tag in STEP_STAGES:
        GPU_STAGE[st](s)
        o.stage(st)
        if tag is None:
            continue
        for key in [k.split("/", 1)[1] for k in g.files if k.startswith(tag + "/") and not k.endswith("/meta")]:
            a = s.get(key)
            _cmp(a, o.get(key), key, tag + "[oracle]", c.npb, codes)
            _cmp(a, g[f"{tag}/{key}"], key, tag + "[reference]", c.npb, codes)
    assert s.info().device_err == 0


@pytest.mark.parametrize("name", CASES)
def test_trajectory_100_steps_graph(cases, name):
    """100 whole steps from the captured CUDA graph against the reference's dumps."""
    g = golden(name)
    c = cases[name]
    s = LoquatSph(case=c)
    s.set_option(0, 0.58108)
    wf = []
    for st in range(1, 101):
        s.step(1)
        wf.append(s.wall_force(1)[0] * 1e-3)
        if st in (1, 10, 100):
            np.testing.assert_array_equal(s.get("cellpos"), g[f"step{st}/cellpos"])
            far = far_from_contact(c, g[f"step{st}/cellpos"], g[f"step{st}/pospres"], g[f"step{st}/contact_var"])
            for key in ("pospres", "velrhop", "str"):
                a, b = s.get(key), g[f"step{st}/{key}"]
                assert rel(a[far], b[far]) < 1e-5, (st, key, rel(a[far], b[far]))
                assert rel(a, b) < 1e-4, (st, key, rel(a, b))
    s.synchronize()
    ref = g["wall_force_kN"][:, 1]
    assert np.max(np.abs(np.asarray(wf) - ref)) / max(np.abs(ref).max(), 1e-30) < 5e-3


@pytest.mark.parametrize("name", CASES)
def test_graph_equals_stage_calls(cases, name):
    """The captured whole-step graph and the per-stage C-ABI calls are the same program."""
    c = cases[name]
    a = LoquatSph(case=c)
    b = LoquatSph(case=c)
    a.step(5)
    for _ in range(5):
        b.step_calculation()
        b.predictor_section()
        b.corrector_section()
        b.end_step()
    for key in ("cellpos", "pospres", "velrhop", "str", "stn", "contact_var", "contact_mag", "idmassidx"):
        np.testing.assert_array_equal(a.get(key), b.get(key), err_msg=key)
    assert a.info().step == b.info().step == 5


@pytest.mark.parametrize("name", CASES)
def test_oracle_trajectory(cases, name):
    """GPU vs oracle over 50 steps, float and double.  The device contracts products into
    fused multiply-adds and the oracle does not, so even in double the two drift apart
    at the rounding level.  Next to a contact wall, discrete decisions (closing test,
    Coulomb cap, slide flag) can flip on such rounding differences and the flip spreads
    by up to one kernel support per step, so with a contact wall the bound is the float
    one even in double, away from the contact zone, and 1e-4 for the whole state."""
    c = cases[name]
    for prec, tol in ((4, 1e-5), (8, 1e-9 if name == "col_mini" else 1e-5)):
        s = LoquatSph(case=c, precision=prec)
        o = Oracle(c, prec)
        s.step(50)
        o.step(50)
        np.testing.assert_array_equal(s.get("cellpos"), o.get("cellpos"))
        cv = o.get("contact_var")
        far = (np.arange(c.np_) >= c.npb) & ~(cv[:, 1] <= 2.0 * c.params["dr"] * c.params["hdr"] + 1e-12)
        for key in ("pos_abs", "velrhop", "str"):
            a, b = s.get(key), o.get(key)
            assert rel(a[far], b[far]) < tol, (prec, key, rel(a[far], b[far]))
            assert rel(a, b) < 1e-4, (prec, key, rel(a, b))
        fs, fo = s.wall_force(0), o.wall_force(0)
        assert abs(fs[0] - fo[0]) <= 5e-3 * max(abs(fo[0]), 1e-12), (prec, fs, fo)


def test_device_error_word_on_wall_leaving_grid():
    """A rigid wall driven out of the grid: the reference would write out of bounds;
    here the cell key is clamped, RW_DERR_CELL_RANGE is raised, and rw_synchronize
    reports RW_EDEVICE without any device fault."""
    from retainwall_code_b200 import cases as C, RwError

    c = C.retaining_wall(nx=8, ny=4, nz=6, dx=0.005, mode="active", wall_speed=400.0)
    s = LoquatSph(case=c)
    with pytest.raises(RwError) as ei:
        s.step(400)
        s.synchronize()
    assert ei.value.status == 7
    assert s.info().device_err & 1


@pytest.mark.parametrize("build", ["col_mini", "wall_mini", "per_mini", "thin_column", "wall_medium"])
def test_chunked_interaction_equals_global_path(cases, build):
    """The chunked interaction (neighbour tile in shared memory) and the global-memory
    path run the same arithmetic in the same order: states must be bit-identical.
    The thin column (one particle per layer) makes chunks span more z cells than the
    tile holds, so it exercises the chunked kernel's fallback as well."""
    from retainwall_code_b200 import _abi, cases as C

    if build in cases:
        c = cases[build]
    elif build == "thin_column":
        c = C.column_collapse(nx=1, ny=1, nz=150, runout=0.2)
    else:
        c = C.retaining_wall(nx=48, ny=24, nz=36, dx=0.0025, wall_friction=0.58108)
    a = LoquatSph(case=c)
    b = LoquatSph(case=c)
    a.set_option(_abi.OPT_INTERACTION_KERNEL, 1)
    b.set_option(_abi.OPT_INTERACTION_KERNEL, 0)
    a.step(10)
    b.step(10)
    for key in ("cellpos", "pospres", "velrhop", "str", "stn", "contact_var", "contact_mag", "accad", "acestn"):
        np.testing.assert_array_equal(a.get(key), b.get(key), err_msg=key)
    assert a.info().device_err == 0 and b.info().device_err == 0


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("ix_kernel", [0, 1])
def test_interaction_strict_bit_exact_vs_oracle(cases, name, ix_kernel):
    """With RW_OPT_STRICT_FP every product and sum of the interaction is rounded
    separately, the written order of the reference's expressions.  Given the same input
    state, the GPU interaction stage (either kernel) then equals the CPU restatement bit
    for bit, which pins the summation order of every particle's sums (27 cells in
    cz, cy, cx order, boundary before material, ascending j) and the contact rule."""
    from retainwall_code_b200 import _abi

    g = golden(name)
    c = cases[name]
    s = LoquatSph(case=c)
    s.set_option(_abi.OPT_STRICT_FP, 1)
    s.set_option(_abi.OPT_INTERACTION_KERNEL, ix_kernel)
    o = Oracle(c, 4)
    load_state(s, g)
    load_state(o, g)
    for st in ("begin_step", "neighbor_search_p", "rigid_body_update", "adami", "find_corner"):
        GPU_STAGE[st](s)
        o.stage(st)
    # identical interaction inputs: hand the GPU's post-corner state to the oracle
    for key in ("velrhop", "str", "contact_mag", "contact_var", "pospres", "idmassidx"):
        o.set(key, s.get(key))
    s.particle_interaction()
    o.stage("interaction")
    for key in ("accad", "acestn", "spin", "contact_var", "contact_mag"):
        a, b = s.get(key), o.get(key)
        np.testing.assert_array_equal(a, b, err_msg=key)


def _pq(stress):
    """Mean stress p = -tr(s)/3 and deviator invariant q = sqrt(3/2 s':s') per row
    (columns xx, yy, zz, xy, xz, yz)."""
    s = np.asarray(stress, dtype=np.float64)
    p = -(s[:, 0] + s[:, 1] + s[:, 2]) / 3.0
    d = s[:, :3] + p[:, None]
    q = np.sqrt(1.5 * ((d * d).sum(1) + 2.0 * (s[:, 3:6] ** 2).sum(1)))
    return p, q


def test_precision_form_runs_close_to_fp64(cases):
    """Precision form (compensated integration, FP64 strain-rate norm) against the
    oracle's FP64 step (the CPU restatement in double) over 200 steps of the column:
    positions and the stress invariants p and q stay within rounding-level distance and
    no further than plain FP32's; the GPU's own FP64 step matches the oracle to 1e-9.
    Rows are matched by the original index the loader keeps (idmassidx[:, 2])."""
    from retainwall_code_b200 import _abi

    c = cases["col_mini"]
    o = Oracle(c, 8)
    o.step(200)

    def by_orig(get):
        idx = get("idmassidx")[:, 2].astype(np.int64)
        out = {}
        for k in ("pos_abs", "str"):
            a = np.asarray(get(k), dtype=np.float64)
            b = np.empty_like(a)
            b[idx[:len(a)]] = a
            out[k] = b
        return out

    ref = by_orig(o.get)
    ref_p, ref_q = _pq(ref["str"][c.npb:])
    soil = slice(c.npb, None)
    errs = {}
    for mode in ("f64", "f32", "mixed"):
        sim = LoquatSph(case=c, precision=8 if mode == "f64" else 4)
        if mode == "mixed":
            sim.set_option(_abi.OPT_MIXED_PRECISION, 1)
        sim.step(200)
        assert sim.info().device_err == 0
        got = by_orig(sim.get)
        p, q = _pq(got["str"][soil])
        errs[mode] = (rel(got["pos_abs"][:, :3], ref["pos_abs"][:, :3]), rel(p, ref_p), rel(q, ref_q))
    print({k: [f"{x:.2e}" for x in v] for k, v in errs.items()})
    assert max(errs["f64"]) < 1e-9, errs["f64"]
    for mode in ("f32", "mixed"):
        assert errs[mode][0] < 1e-6 and errs[mode][1] < 1e-4 and errs[mode][2] < 1e-4, (mode, errs[mode])
    assert errs["mixed"][0] <= 2.0 * errs["f32"][0] + 1e-9


def test_batch_equals_individual_runs():
    """Cases advanced together by one graph launch per step (rw_batch_*) end in exactly
    the states they reach when stepped alone."""
    from retainwall_code_b200 import Batch, cases as C

    specs = C.batch_sweep(n_cases=3, seed=7, n_lo=2000, n_hi=6000)
    cs = [C.retaining_wall(nx=s["nx"], ny=s["ny"], nz=s["nz"], dx=s["dx"], phi_c=s["phi_c"], e0=s["e0"],
                           mode=s["mode"], seed=s["seed"]) for s in specs]
    together = [LoquatSph(case=c) for c in cs]
    b = Batch(together)
    b.step(6)
    b.synchronize()
    forces = b.wall_force(0)
    strips = b.wall_force(1)
    assert forces.shape == (3, 3) and strips.shape == (3, 3)
    # the batch graph keeps each step's gates: quiet sections skip their search
    assert sum(t.info().n_search_skipped for t in together) > 0
    for k, (c, t) in enumerate(zip(cs, together)):
        alone = LoquatSph(case=c)
        alone.step(6)
        for key in ("cellpos", "pospres", "velrhop", "str", "contact_mag"):
            np.testing.assert_array_equal(t.get(key), alone.get(key), err_msg=key)
        assert t.info().step == 6
        np.testing.assert_array_equal(forces[k], alone.wall_force(0))
        np.testing.assert_array_equal(strips[k], alone.wall_force(1))
    b.close()


def test_batch_sees_options_set_after_creation():
    """An option set on a context after rw_batch_create (here the wall friction and the
    list skin) takes effect at the next batch step: the batch equals runs stepped alone
    with the same option changes at the same step."""
    from retainwall_code_b200 import Batch, _abi, cases as C

    cs = [C.retaining_wall(nx=14, ny=6, nz=10, dx=0.005, seed=s, mode=m) for s, m in ((1, "active"), (2, "passive"))]
    together = [LoquatSph(case=c) for c in cs]
    b = Batch(together)
    b.step(2)
    together[0].set_option(_abi.OPT_WALL_FRICTION, 0.1)
    together[1].set_option(_abi.OPT_LIST_SKIN, 0.0)
    b.step(3)
    b.synchronize()
    for k, c in enumerate(cs):
        alone = LoquatSph(case=c)
        alone.step(2)
        alone.set_option(*((_abi.OPT_WALL_FRICTION, 0.1) if k == 0 else (_abi.OPT_LIST_SKIN, 0.0)))
        alone.step(3)
        for key in ("cellpos", "pospres", "velrhop", "str", "contact_mag"):
            np.testing.assert_array_equal(together[k].get(key), alone.get(key), err_msg=f"case {k} {key}")
    plain = LoquatSph(case=cs[0])
    plain.step(5)
    assert not np.array_equal(plain.get("contact_mag"), together[0].get("contact_mag"))  # the friction acted
    b.close()


def test_autotune_picks_shapes():
    """The autotuner times five shapes (walk at 64/128 threads, chunked kernel, then
    integrators at 256/128 threads), three steps each, and keeps the fastest."""
    from retainwall_code_b200 import cases as C

    s = LoquatSph(case=C.retaining_wall(nx=16, ny=8, nz=12, dx=0.005))
    k = s.autotune(2)
    inf = s.info()
    assert k in (0, 1) and inf.ix_kernel == k
    assert inf.walk_threads in (64, 128) and inf.integrator_threads in (128, 256)
    assert inf.step == 15 and inf.device_err == 0


def test_block_shapes_do_not_change_the_result(cases):
    """Walk and integrator block sizes are launch shapes only: bit-identical states."""
    from retainwall_code_b200 import _abi

    c = cases["wall_mini"]
    ref = LoquatSph(case=c)
    ref.step(6)
    for wt, it in ((64, 128), (64, 256), (128, 128)):
        s = LoquatSph(case=c)
        s.set_option(_abi.OPT_WALK_THREADS, wt)
        s.set_option(_abi.OPT_INTEGRATOR_THREADS, it)
        s.step(6)
        for key in ("cellpos", "pospres", "velrhop", "str", "stn", "contact_var", "accad"):
            np.testing.assert_array_equal(s.get(key), ref.get(key), err_msg=f"{wt}/{it} {key}")


def test_periodic_wrap_matches_oracle():
    """Particles leaving through a periodic plane re-enter through the other one; after
    the wraps the GPU's cell coordinates equal the oracle's and no particle is lost."""
    from tests.test_oracle_golden import _periodic_drift_case

    c = _periodic_drift_case()
    s = LoquatSph(case=c)
    o = Oracle(c, 4)
    s.step(10)
    o.step(10)
    yl, yr = -c.params["planeleft"][3], c.params["planeright"][3]
    for sim in (s, o):
        inf = sim.info()
        assert inf.npm == c.npm and inf.np_delete_m == 0
        y = sim.get("pos_abs")[c.npb:, 1]
        assert y.min() >= yl - 1e-6 and y.max() <= yr + 1e-6
    np.testing.assert_array_equal(s.get("cellpos"), o.get("cellpos"))
    assert rel(s.get("pos_abs"), o.get("pos_abs")) < 1e-5
    assert s.info().device_err == 0


def test_kept_candidate_lists_reused_and_dropped(cases):
    """Interactions walk the candidate lists kept by an earlier scan while no particle
    changed cell or moved more than the skin allows (a quasi-static case: every
    interaction after the first); in a fast case (a half step beyond the skin's share)
    every interaction scans the cells again.  Either way the result equals the chunked
    kernel, which never keeps lists, bit for bit."""
    from retainwall_code_b200 import _abi

    c = cases["wall_mini"]
    s = LoquatSph(case=c)
    s.step(5)
    assert s.info().n_list_reuse == 9
    b = LoquatSph(case=c)
    b.set_option(_abi.OPT_INTERACTION_KERNEL, 1)
    b.step(5)
    d = LoquatSph(case=c)
    d.set_option(_abi.OPT_LIST_SKIN, 0.0)
    d.step(5)
    assert d.info().n_list_reuse == 0
    for key in ("cellpos", "pospres", "velrhop", "str", "contact_var", "accad"):
        np.testing.assert_array_equal(s.get(key), b.get(key), err_msg=key)
        np.testing.assert_array_equal(s.get(key), d.get(key), err_msg=key)
    fast = mini_cases()["wall_mini"]
    fast.velrhop[fast.npb:, 0] = 40.0  # a half step of 0.2 mm > 0.45 x skin (0.054 mm)
    a = LoquatSph(case=fast)
    b = LoquatSph(case=fast)
    b.set_option(_abi.OPT_INTERACTION_KERNEL, 1)
    a.step(3)
    b.step(3)
    assert a.info().n_list_reuse == 0
    for key in ("cellpos", "pospres", "velrhop", "str", "contact_var", "accad"):
        np.testing.assert_array_equal(a.get(key), b.get(key), err_msg=key)


def test_graph_gates_skip_idle_work_only(cases):
    """The step graph's conditional nodes skip a search in which no particle changed
    cell and the scan launch of an interaction that walks every kept list; the device
    counts what it skipped.  Results equal a plain graph (every kernel launched) bit for
    bit, in a quasi-static case (searches skipped) and in a fast one (none skipped)."""
    from retainwall_code_b200 import _abi

    fast = mini_cases()["wall_mini"]
    fast.velrhop[fast.npb:, 0] = 40.0
    for c, quiet in ((cases["wall_mini"], True), (fast, False)):
        g = LoquatSph(case=c)
        p = LoquatSph(case=c)
        p.set_option(_abi.OPT_GRAPH_GATES, 0)
        g.step(6)
        p.step(6)
        for key in ("cellpos", "pospres", "velrhop", "str", "contact_var", "accad"):
            np.testing.assert_array_equal(g.get(key), p.get(key), err_msg=key)
        gi, pi = g.info(), p.info()
        assert pi.n_search_skipped == 0 and pi.n_scan_skipped == 0 and pi.n_build_skipped == 0
        assert gi.graph_kernels - pi.graph_kernels == 6  # gates: 2 searches, 2 list builds, 2 scans
        if quiet:  # every interaction walks a list; lists rebuilt once
            assert gi.n_scan_skipped == 12 and gi.n_build_skipped == 11 and gi.n_search_skipped > 0
        else:
            assert gi.n_build_skipped == 0
        assert gi.device_err == 0


def test_options_changed_between_steps_keep_the_state(cases):
    """Options that rebuild the step graph (gates, list skin, interaction kernel) can be
    changed between steps; the state carries over and the run equals one that kept the
    defaults, bit for bit."""
    from retainwall_code_b200 import _abi

    c = cases["wall_mini"]
    ref = LoquatSph(case=c)
    ref.step(8)
    s = LoquatSph(case=c)
    s.step(2)
    s.set_option(_abi.OPT_GRAPH_GATES, 0)
    s.step(2)
    s.set_option(_abi.OPT_LIST_SKIN, 0.0)
    s.step(2)
    s.set_option(_abi.OPT_GRAPH_GATES, 1)
    s.set_option(_abi.OPT_LIST_SKIN, 0.02)
    s.set_option(_abi.OPT_INTERACTION_KERNEL, 1)
    s.step(1)
    s.set_option(_abi.OPT_INTERACTION_KERNEL, 0)
    s.step(1)
    for key in ("cellpos", "pospres", "velrhop", "str", "contact_var", "accad"):
        np.testing.assert_array_equal(s.get(key), ref.get(key), err_msg=key)
    assert s.info().step == 8 and s.info().device_err == 0


def test_overflowing_lists_fall_back_to_the_scan(cases):
    """With a skin wide enough that some candidate lists exceed their 96 entries, the
    list build marks those lists and counts them; the scan launch takes exactly those
    particles while the walk takes the rest.  The result equals scanning every
    particle (skin 0), bit for bit."""
    from retainwall_code_b200 import _abi

    c = cases["wall_mini"]
    a = LoquatSph(case=c)
    a.set_option(_abi.OPT_LIST_SKIN, 0.45)
    b = LoquatSph(case=c)
    b.set_option(_abi.OPT_LIST_SKIN, 0.0)
    a.step(4)
    b.step(4)
    ent, parts = a.list_stats()
    assert 0 < parts < a.info().npm  # some lists kept, some overflowed
    for key in ("cellpos", "pospres", "velrhop", "str", "contact_var", "accad"):
        np.testing.assert_array_equal(a.get(key), b.get(key), err_msg=key)
    assert a.info().device_err == 0


def test_deletion_matches_oracle():
    """Soil thrown out through the open +x side of the grid is moved to the deleted cell
    (cuCheckOutDomain, src/predictor_corrector.cu:183-187; the count bookkeeping of
    src/loquat_grid.cu:164-190): live and deleted counts, the cell coordinates of every
    slot and the state of the remaining soil match the oracle step after step."""
    from retainwall_code_b200 import cases as C

    c = C.column_collapse(nx=8, ny=8, nz=16, runout=0.0)
    c.velrhop[c.npb:, 0] = 40.0
    s = LoquatSph(case=c)
    o = Oracle(c, 4)
    deleted = []
    for _ in range(11):
        s.step(10)
        o.step(10)
        a, b = s.info(), o.info()
        assert (a.npm, a.np_delete_m) == (b.npm, b.np_delete_m)
        np.testing.assert_array_equal(s.get("cellpos"), o.get("cellpos"))
        live = slice(a.npb, a.npb + a.npm)
        assert rel(s.get("pos_abs")[live], o.get("pos_abs")[live]) < 1e-5
        deleted.append(a.np_delete_m)
    assert deleted[-1] > 0 and deleted[0] == 0
    assert s.info().device_err == 0


def test_no_boundary_particles_matches_oracle():
    """A case without boundary particles (npb = 0: soil in free fall)."""
    from retainwall_code_b200 import cases as C

    b = C._Builder()
    C._soil(b, 0.05, 0.05, 0.05, 6, 6, 6, 0.005, np.random.default_rng(1), 0.05, 1850.0, -9.81, 0.5)
    p = C._base_params(0.005, 1.2, 60.0, 0.1, 1850.0, C.hypocs_model(30.0, 0.7, 1850.0))
    p["domain_size_x"] = p["domain_size_y"] = p["domain_size_z"] = 0.15
    c = b.case(p, [], "free", 1850.0, C.f32(1850.0 * 0.005 ** 3))
    assert c.npb == 0
    s = LoquatSph(case=c)
    o = Oracle(c, 4)
    s.step(20)
    o.step(20)
    np.testing.assert_array_equal(s.get("cellpos"), o.get("cellpos"))
    for key in ("pos_abs", "velrhop", "str"):
        assert rel(s.get(key), o.get(key)) < 1e-5, key
    assert s.info().device_err == 0
