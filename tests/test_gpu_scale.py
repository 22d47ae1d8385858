"""Full-size retaining wall (1.92M soil particles): size-independent properties of the
cell list and of the step, and one step against the CPU oracle at full size."""
import numpy as np
import pytest

from retainwall_code_b200 import LoquatSph, cases as C
from tests._util import rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def wall2():
    return C.retaining_wall()


def test_cell_list_invariants(wall2):
    s = LoquatSph(case=wall2)
    inf = s.info()
    assert inf.npm == 1_920_000
    perm = s.get("part_idx")
    cell = s.get("cellpos")
    key = cell[:, 3]
    assert np.array_equal(np.sort(perm), np.arange(inf.np))  # a permutation
    assert (np.diff(key) >= 0).all()                          # sorted by cell key
    beg, end = s.get("cell_beg"), s.get("cell_end")
    occ = beg >= 0
    assert (end[occ] - beg[occ]).sum() == inf.np
    k = np.nonzero(occ)[0]
    assert (key[beg[k]] == k).all() and (key[end[k] - 1] == k).all()
    assert (beg[~occ] == -1).all() and (end[~occ] == -1).all()
    # stable: within a cell the original order is kept
    same = np.diff(key) == 0
    assert (np.diff(perm)[same] > 0).all()


def test_steps_conserve_mass_and_stay_finite(wall2):
    s = LoquatSph(case=wall2)
    m0 = s.get("idmassidx")[:, 1].astype(np.float64).sum()
    s.step(20)
    s.synchronize()
    inf = s.info()
    assert inf.device_err == 0 and inf.np_delete_m == 0 and inf.step == 20
    idm = s.get("idmassidx")
    assert abs(idm[:, 1].astype(np.float64).sum() - m0) <= 1e-9 * m0
    for k in ("pos_abs", "velrhop", "str"):
        assert np.isfinite(s.get(k)).all(), k
    f = s.wall_force(0)
    assert np.isfinite(f).all()


@pytest.mark.slow
def test_one_step_against_oracle_full_size(wall2):
    from oracle.oracle import Oracle

    s = LoquatSph(case=wall2)
    o = Oracle(wall2, 4)
    s.step(1)
    o.step(1)
    np.testing.assert_array_equal(s.get("cellpos"), o.get("cellpos"))
    for k in ("pos_abs", "velrhop", "str", "contact_var"):
        assert rel(s.get(k), o.get(k)) < 1e-5, k
