"""Kept candidate lists updated in part when particles change cell.

The candidate lists stand in for the 27-cell scans of cuParticleInteractionMaterial
(src/particle_interaction.cu:117-140) and cuAdamiBoundaryMaterial
(src/adami_boundary.cu:26-158).  After a step in which particles entered or left cells,
the next predictor section rebuilds only the lists of the particles next to those cells
and carries every other list through the section's sort permutation.  A run with list
updates must equal scanning the cells at every interaction (list skin 0), the chunked
kernel (no lists) and the ungated graph, bit for bit, at every checkpoint of a run with
many cell changes and sorts."""
import numpy as np
import pytest

from retainwall_code_b200 import LoquatSph, _abi, cases as C

pytestmark = pytest.mark.gpu

KEYS = ("cellpos", "idmassidx", "pospres", "velrhop", "str", "contact_var", "accad", "normal_m")


def _column(vx=3.0):
    """The column thrown along +x at vx (m/s): at 3 m/s about four particles cross a cell
    face per step, most crossings need a sort (an x step moves a key by ny x nz), and a
    half step stays within the displacement share of a 0.6 h skin for about 50 steps."""
    c = C.column_collapse(nx=8, ny=8, nz=16, runout=1.0, name="col")
    c.velrhop[c.npb:, 0] = vx
    return c


def _passive_wall():
    """The wall pushed into the soil at 2 m/s: its particle layers cross cell faces."""
    return C.retaining_wall(nx=16, ny=8, nz=12, dx=0.005, wall_friction=C.REFERENCE_WALL_FRICTION, mode="passive",
                            wall_speed=2.0, name="passive")


def _run_with_updates(case, steps, every, skin):
    """Steps one at a time with list updates on (list skin `skin`), a twin with every
    option at its default (skin 0.02 h, set at creation), a lists-off twin and a
    chunked-kernel twin; compares the four at every `every` steps and returns per-step
    counters of the first."""
    s = LoquatSph(case=case)
    s.set_option(_abi.OPT_LIST_SKIN, skin)
    dflt = LoquatSph(case=case)
    scan = LoquatSph(case=case)
    scan.set_option(_abi.OPT_LIST_SKIN, 0.0)
    chunk = LoquatSph(case=case)
    chunk.set_option(_abi.OPT_INTERACTION_KERNEL, 1)
    rows = []
    prev = s.info()
    for k in range(1, steps + 1):
        for x in (s, dflt, scan, chunk):
            x.step(1)
        cur = s.info()
        rows.append((cur.n_sorts - prev.n_sorts, cur.n_list_updates - prev.n_list_updates,
                     cur.n_lists_rebuilt - prev.n_lists_rebuilt))
        prev = cur
        if k % every == 0 or k == steps:
            for key in KEYS:
                a = s.get(key)
                np.testing.assert_array_equal(a, dflt.get(key), err_msg=f"step {k} {key} vs default skin")
                np.testing.assert_array_equal(a, scan.get(key), err_msg=f"step {k} {key} vs scan")
                np.testing.assert_array_equal(a, chunk.get(key), err_msg=f"step {k} {key} vs chunked")
    assert all(x.info().device_err == 0 for x in (s, dflt, scan, chunk))
    assert np.isfinite(s.get("pospres")).all()
    return s, np.array(rows)


def test_column_collapse_list_updates_equal_scans():
    """A moving column: particles change cell in most steps.  With a skin of 0.6 h the
    displacement bound forces a full build only every few dozen steps, so most steps
    after a cell change update the lists in part, most of them after a sort."""
    case = _column()
    s, rows = _run_with_updates(case, 300, 25, 0.6)
    sorts, updates, rebuilt = rows[:, 0], rows[:, 1], rows[:, 2]
    inf = s.info()
    assert updates.sum() >= 20, updates.sum()
    assert ((sorts > 0) & (updates > 0)).sum() >= 5  # updates that carried lists through a sort
    # the updates rebuilt a part of the lists (soil and boundary), not all of them
    assert 0 < rebuilt.sum() < 0.8 * updates.sum() * inf.np
    full = 2 * inf.step - inf.n_build_skipped - inf.n_list_updates
    assert full < updates.sum()
    print(f"column: {updates.sum()} updates ({((sorts > 0) & (updates > 0)).sum()} after a sort), "
          f"{full} full builds, {rebuilt.sum() / max(updates.sum(), 1):.0f} of {inf.np} lists rebuilt per update")


def test_passive_wall_list_updates_equal_scans():
    """A wall pushed into the soil: boundary particles change cell too (their cells are
    marked from the corrector's rigid-wall rows) and the boundary lists of the Adami
    extrapolation are updated with the soil's."""
    case = _passive_wall()
    s, rows = _run_with_updates(case, 200, 20, 0.6)
    assert rows[:, 1].sum() > 0
    assert s.info().n_list_reuse > 0


def test_list_updates_gated_graph_equals_plain_graph():
    """The mark dilation sits in the gated search body and the rebuild of the lists next
    to marked cells in the gated list build: the gated graph equals the plain one (every
    kernel launched)."""
    case = _column()
    g = LoquatSph(case=case)
    p = LoquatSph(case=case)
    for x in (g, p):
        x.set_option(_abi.OPT_LIST_SKIN, 0.6)
    p.set_option(_abi.OPT_GRAPH_GATES, 0)
    g.step(150)
    p.step(150)
    for key in KEYS:
        np.testing.assert_array_equal(g.get(key), p.get(key), err_msg=key)
    gi, pi = g.info(), p.info()
    assert gi.n_list_updates == pi.n_list_updates > 0
    assert gi.n_lists_rebuilt == pi.n_lists_rebuilt
    assert gi.device_err == 0 and pi.device_err == 0


def test_list_updates_under_the_default_skin_fp64():
    """The default skin (0.02 h) and FP64: updates and full builds interleave; the run
    equals the lists-off run bit for bit."""
    case = _column()
    a = LoquatSph(case=case, precision=8)
    b = LoquatSph(case=case, precision=8)
    b.set_option(_abi.OPT_LIST_SKIN, 0.0)
    a.step(120)
    b.step(120)
    for key in KEYS:
        np.testing.assert_array_equal(a.get(key), b.get(key), err_msg=key)
    assert a.info().n_list_updates > 0 and a.info().device_err == 0


def test_too_many_marked_cells_make_a_full_build():
    """More than 8192 cells marked in one step (the capacity of the marked-cell list) turn
    the next update into a full build.  A 384k-particle wall whose soil block is moved
    onto the cell faces (dx/10 along x: the generator's lattice otherwise keeps every
    particle 0.05 dx from them) and thrown at 10 m/s: in each step about 7,500 particles
    change cell.  The run equals the lists-off run bit for bit, and its interactions
    rebuilt every list instead of updating them."""
    c = C.retaining_wall(nx=40, ny=80, nz=120, name="burst")
    c.pospres[c.npb:, 0] += 0.1 * c.params["dr"]
    c.velrhop[c.npb:, 0] = 10.0
    a = LoquatSph(case=c)
    a.set_option(_abi.OPT_LIST_SKIN, 1.0)
    b = LoquatSph(case=c)
    b.set_option(_abi.OPT_LIST_SKIN, 0.0)
    for _ in range(3):
        a.step(1)
        b.step(1)
    for key in KEYS:
        np.testing.assert_array_equal(a.get(key), b.get(key), err_msg=key)
    inf = a.info()
    full = 2 * inf.step - inf.n_build_skipped - inf.n_list_updates
    assert inf.n_sorts >= 3 and full >= 3, (inf.n_sorts, full, inf.n_list_updates)
    assert inf.device_err == 0


@pytest.mark.parametrize("every", [1, 3])
def test_shepard_filter_on_lists_equals_scan(every):
    """The Shepard stress filter inside the step (src/field_smoothing.cu:26-101, applied
    every `stress-shepard-filter` steps) walks the candidate lists when they are kept:
    the moving column with the filter on equals the runs that filter by scanning the
    cells (list skin 0, chunked kernel), bit for bit, through cell changes and list
    updates."""
    case = _column()
    case.params["stress_shepard_filter"] = every
    runs = {}
    for name, opt in (("lists", None), ("scan", (_abi.OPT_LIST_SKIN, 0.0)), ("chunk", (_abi.OPT_INTERACTION_KERNEL, 1))):
        s = LoquatSph(case=case)
        if opt:
            s.set_option(*opt)
        s.step(120)
        runs[name] = s
    plain = LoquatSph(case=_column())
    plain.step(120)
    for key in KEYS:
        np.testing.assert_array_equal(runs["lists"].get(key), runs["scan"].get(key), err_msg=key)
        np.testing.assert_array_equal(runs["lists"].get(key), runs["chunk"].get(key), err_msg=key)
    assert not np.array_equal(runs["lists"].get("str"), plain.get("str"))  # the filter acted
    assert runs["lists"].info().n_list_updates > 0 and runs["lists"].info().device_err == 0


def test_periodic_wraps_update_lists():
    """Periodic y planes (src/loquat_grid.cu's periodic images, `period_wrap` in the
    corrector): the soil thrown along +y at 3 m/s crosses cell faces and, near the +y
    plane, wraps to the other end of the grid.  Both cells of each wrap are marked and
    the lists next to them rebuilt; the run equals scanning the cells, bit for bit."""
    c = C.retaining_wall(nx=16, ny=8, nz=12, dx=0.005, wall_friction=C.REFERENCE_WALL_FRICTION, periodic_y=True,
                         name="periodic")
    c.velrhop[c.npb:, 1] = 3.0
    s, rows = _run_with_updates(c, 150, 25, 0.6)
    assert rows[:, 1].sum() > 0 and rows[:, 0].sum() > 0  # updates, sorts
    idx = s.get("idmassidx")[:, 2].astype(np.int64)
    y0 = c.pospres[idx[c.npb:], 1]
    y1 = s.get("pos_abs")[c.npb:, 1]
    assert (y1 < y0 - 0.01).any()  # some particles wrapped to the low side


def test_precision_form_with_list_updates_equals_scan():
    """The precision form permutes its compensation terms with the state; through list
    updates after sorts it equals the same form scanning the cells, bit for bit."""
    case = _column()
    a, b = LoquatSph(case=case), LoquatSph(case=case)
    for x in (a, b):
        x.set_option(_abi.OPT_MIXED_PRECISION, 1)
    a.set_option(_abi.OPT_LIST_SKIN, 0.6)
    b.set_option(_abi.OPT_LIST_SKIN, 0.0)
    a.step(150)
    b.step(150)
    for key in KEYS:
        np.testing.assert_array_equal(a.get(key), b.get(key), err_msg=key)
    assert a.info().n_list_updates > 0 and a.info().n_sorts > 10 and a.info().device_err == 0
