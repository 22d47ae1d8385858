"""Output layout (src/loquat_io.cu:315-680, src/loquat.cu:439-482, src/utilities.cu:266-367)
through the C ABI and the `loquat` command line."""
import os
import subprocess

import numpy as np
import pytest

from retainwall_code_b200 import LoquatSph, cases as C

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _wall_case():
    return C.retaining_wall(nx=16, ny=8, nz=12, dx=0.005, wall_friction=C.REFERENCE_WALL_FRICTION, name="io")


def test_wall_profile_matches_reference_loop_semantics():
    """Per (band, depth bin): value of the highest-index particle in it, as the
    reference's sequential loop leaves it; the depth of a bin only where the first band
    has a particle (the reference writes it together with that band's value)."""
    s = LoquatSph(case=_wall_case())
    s.step(40)
    inf = s.info()
    dr = inf.dr
    x_wall, z_top, nb = 0.04 + 0.015 + 1e-4, 0.04 + 0.015 + 0.07, 30
    prof = s.wall_profile(x_wall, z_top, dr, nb)
    pos = s.get("pos_abs").astype(np.float32)
    cm = s.get("contact_mag")
    exp = np.zeros((nb, 4))
    for i in range(inf.npb, inf.np):
        px, pz = float(pos[i, 0]), float(pos[i, 2])
        if not (z_top - 1.0 <= pz <= z_top):
            continue
        for band in range(3):
            if x_wall + dr * band <= px <= x_wall + dr * (band + 1):
                b = int((z_top - pz) / dr)
                if 0 <= b < nb:
                    exp[b, 1 + band] = float(np.float32(cm[i, 0]) / np.float32(dr))
                    if band == 0:  # the depth is written with the first band's value
                        exp[b, 0] = b * np.float64(np.float32(dr))
    np.testing.assert_allclose(prof, exp, rtol=1e-6, atol=1e-9)
    assert (prof[:, 1] != 0).any()


def test_save_writes_reference_layout(tmp_path):
    case = _wall_case()
    s = LoquatSph(case=case)
    out = str(tmp_path / "out")
    s.save(out)  # initial configuration: output_0, particles only
    assert set(os.listdir(out)) == {"output_0.xml", "0_0.vtu", "100_0.vtu"}
    s.step(5)
    s.save(out)
    files = set(os.listdir(out))
    assert {"output_1.xml", "time_history.txt", "stress_zz1.txt", "0_1.vtu", "100_1.vtu"} <= files
    p = C.read_xml(os.path.join(out, "output_1.xml"))
    assert p["np"] == case.np_ and p["output_number"] == 1
    th = np.loadtxt(os.path.join(out, "time_history.txt")).reshape(-1, 2)
    assert th.shape[0] == 1 and np.isfinite(th).all()
    zz = np.loadtxt(os.path.join(out, "stress_zz1.txt"))
    assert zz.shape == (int(np.float32(1.0) / np.float32(s.info().dr)), 4)
    vtu = open(os.path.join(out, "100_1.vtu")).read()
    assert f'NumberOfPoints="{case.npm}"' in vtu and 'Name="Stress" NumberOfComponents="6"' in vtu


def test_save_dat_format_roundtrips(tmp_path):
    case = _wall_case()
    case.params["output_format"] = 1
    s = LoquatSph(case=case)
    out = str(tmp_path / "o")
    s.save(out)
    s.step(3)
    s.save(out)
    rows = open(os.path.join(out, "1.dat")).read().strip().split("\n")
    assert len(rows) == case.np_
    assert all(len(r.split()) == 31 for r in rows)  # every live row carries the normal columns
    pos = np.array([list(map(float, r.split()[4:7])) for r in rows])
    np.testing.assert_allclose(pos, s.get("pos_abs")[:, :3], rtol=5e-6, atol=1e-9)  # 6 significant digits


def test_cli_runs_project(tmp_path):
    exe = os.path.join(ROOT, "retainwall_code_b200", "loquat")
    case = _wall_case()
    case.params["output_frequency"] = 2e-4
    proj = str(tmp_path / "wall")
    C.write_case(case, proj)
    env = dict(os.environ, RW_TIME_MAX="5e-4")
    r = subprocess.run([exe, proj, "0"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr
    files = os.listdir(proj)
    assert "output_0.xml" in files and "output_1.xml" in files and "time_history.txt" in files
    th = np.loadtxt(os.path.join(proj, "time_history.txt")).reshape(-1, 2)
    assert th.shape[0] >= 2


def test_case_ingest_matches_host_conversion():
    """rw_create_from_case copies the caller's double arrays as they are and converts them
    on the device (LoadParticles' values, PositionFromAbsolute2Relative's absolute ->
    in-cell split with the fused product of src/loquat_grid.cu:253-271).  The state after
    creation equals the same conversion done on the host in float32, bit for bit, row by row (rows are matched through the original index that the
    loader keeps in idmassidx[:, 2], since creation also sorts by cell)."""
    c = C.retaining_wall(nx=24, ny=12, nz=16, dx=0.004, name="ingest")
    s = LoquatSph(case=c)
    f32 = np.float32
    h = f32(c.params["dr"]) * f32(c.params["hdr"])
    half_ih = f32(0.5 * float(f32(1.0) / h))
    two_h = f32(2.0 * float(h))
    pa = c.pospres.astype(f32)
    cell = (pa[:, :3] * half_ih).astype(np.int32)  # truncation toward zero
    pos = pa.copy()
    # x - c 2h with one rounding (exact in double, then rounded once to float)
    pos[:, :3] = (pa[:, :3].astype(np.float64) - cell.astype(np.float64) * np.float64(two_h)).astype(f32)
    idx = s.get("idmassidx")[:, 2].astype(np.int64)
    assert np.array_equal(np.sort(idx), np.arange(c.np_))
    np.testing.assert_array_equal(s.get("pospres"), pos[idx].astype(np.float64))
    np.testing.assert_array_equal(s.get("cellpos")[:, :3], cell[idx])
    np.testing.assert_array_equal(s.get("codes"), c.codes[idx])
    np.testing.assert_array_equal(s.get("velrhop"), c.velrhop.astype(f32)[idx].astype(np.float64))
    np.testing.assert_array_equal(s.get("str"), c.stress.astype(f32)[idx].astype(np.float64))
    np.testing.assert_array_equal(s.get("stn"), c.strain.astype(f32)[idx].astype(np.float64))
    m = s.get("idmassidx")
    np.testing.assert_array_equal(m[:, 1], c.idmassidx[:, 1].astype(f32)[idx].astype(np.float64))
    assert np.all(idx[:c.npb] < c.npb)  # boundary rows stay in front
    np.testing.assert_array_equal(s.get("normal_m"), c.normal.astype(f32)[idx[:c.npb]].astype(np.float64))
    assert s.info().device_err == 0


def test_async_save_writes_the_same_files(tmp_path):
    """RW_OPT_ASYNC_SAVE: rw_save returns while a background task writes the files; the
    next save or rw_synchronize waits for it.  The files equal those of synchronous saves
    byte for byte (both formats), and a write that fails is reported by rw_synchronize."""
    from retainwall_code_b200 import _abi

    for fmt in (1, 2):
        case = _wall_case()
        case.params["output_format"] = fmt
        a, b = LoquatSph(case=case), LoquatSph(case=case)
        b.set_option(_abi.OPT_ASYNC_SAVE, 1)
        da, db = str(tmp_path / f"sync{fmt}"), str(tmp_path / f"async{fmt}")
        for s, d in ((a, da), (b, db)):
            s.save(d)
            for _ in range(3):
                s.step(4)
                s.save(d)
            s.synchronize()
        assert sorted(os.listdir(da)) == sorted(os.listdir(db))
        for name in os.listdir(da):
            assert open(os.path.join(da, name), "rb").read() == open(os.path.join(db, name), "rb").read(), name
    c = LoquatSph(case=_wall_case())
    c.set_option(_abi.OPT_ASYNC_SAVE, 1)
    c.save("/proc/no_such_dir/out")  # the directory cannot be made: the background write fails
    with pytest.raises(RuntimeError):
        c.synchronize()
