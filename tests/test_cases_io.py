"""Case generator and the reference's case-file formats (src/GenCase.cu:70-227,
src/loquat_io.cu:75-312)."""
import numpy as np

from retainwall_code_b200 import cases as C


def test_generator_is_deterministic():
    a = C.retaining_wall(nx=10, ny=6, nz=8, dx=0.005)
    b = C.retaining_wall(nx=10, ny=6, nz=8, dx=0.005)
    assert np.array_equal(a.pospres, b.pospres) and np.array_equal(a.codes, b.codes)


def test_counts_and_layout():
    c = C.retaining_wall(nx=10, ny=6, nz=8, dx=0.005)
    assert c.npm == 10 * 6 * 8
    assert c.np_ == c.npb + c.npm
    assert (c.idmassidx[: c.npb, 0] == 0).all() and (c.idmassidx[c.npb:, 0] == 100).all()
    assert (c.codes[c.npb:, 2] == C.HYPO_CS).all()
    assert ((c.codes[: c.npb, 0] == 10) == (c.codes[: c.npb, 1] == C.NONFIX)).all()
    # every particle strictly inside the grid, with margin
    pos = c.pospres[:, :3]
    dom = np.array([c.params["domain_size_x"], c.params["domain_size_y"], c.params["domain_size_z"]])
    assert (pos > 0).all() and (pos < dom).all()


def test_config_sizes():
    c = C.column_collapse()
    assert c.npm == 27648
    specs = C.batch_sweep()
    assert len(specs) == 64
    n = [s["nx"] * s["ny"] * s["nz"] for s in specs]
    assert 40_000 < min(n) and max(n) < 450_000


def test_geostatic_stress_and_k0():
    c = C.column_collapse(nx=4, ny=4, nz=10)
    m = c.stress[c.npb:]
    assert (m[:, 2] < 0).all()
    k0 = 1 - np.sin(np.radians(30.0))
    np.testing.assert_allclose(m[:, 0] / m[:, 2], k0, rtol=1e-6)


def test_hypocs_mapping():
    m = C.hypocs_model(30.0, 0.7, 1850.0)
    assert abs(m[6] - (3e5 / 2.6e9) ** 0.27) < 1e-7
    assert m[9] == np.float32(0.61) and m[10] == np.float32(1.10) and m[5] == np.float32(0.98)
    assert abs(m[13] - 0.8 * 1850) < 1e-3 and abs(m[14] - 1.2 * 1850) < 1e-3


def test_roundtrip_files(tmp_path):
    c = C.retaining_wall(nx=6, ny=4, nz=5, dx=0.005, mode="rotation")
    proj = str(tmp_path / "w")
    C.write_case(c, proj)
    r = C.read_case(proj)
    assert np.array_equal(r.codes, c.codes)
    for a, b in ((r.pospres, c.pospres), (r.velrhop, c.velrhop), (r.stress, c.stress), (r.normal, c.normal)):
        assert np.array_equal(a.astype(np.float32), b.astype(np.float32))
    assert r.params["npb"] == c.npb
    assert np.float32(r.params[C.WALL_FRICTION_TAG]) == np.float32(c.params[C.WALL_FRICTION_TAG])
    m = r.motions[0]
    assert m.is_rotation and not m.is_translation and m.rotat_vel[1] == np.float32(-0.005)


def test_native_dat_writer_matches_python(tmp_path):
    """rw_write_case_dat (native, threaded) writes the same bytes as write_dat, on a
    wall case (boundary rows with normals) and a case without boundary particles."""
    import filecmp

    import numpy as np

    from retainwall_code_b200 import cases as C

    wall = C.retaining_wall(nx=12, ny=6, nz=8, dx=0.005, mode="rotation")
    b = C._Builder()
    C._soil(b, 0.05, 0.05, 0.05, 3, 3, 3, 0.005, np.random.default_rng(3), 0.05, 1850.0, -9.81, 0.5)
    p = C._base_params(0.005, 1.2, 60.0, 0.1, 1850.0, C.hypocs_model(30.0, 0.7, 1850.0))
    p["domain_size_x"] = p["domain_size_y"] = p["domain_size_z"] = 0.15
    free = b.case(p, [], "free", 1850.0, C.f32(1850.0 * 0.005 ** 3))
    for k, c in enumerate((wall, free)):
        a, n = str(tmp_path / f"py{k}"), str(tmp_path / f"nat{k}")
        C.write_case(c, a, native=False)
        C.write_case(c, n, native=True)
        assert filecmp.cmp(a + ".dat", n + ".dat", shallow=False)
        r = C.read_case(n)
        np.testing.assert_array_equal(r.pospres.astype(np.float32), c.pospres.astype(np.float32))


def test_project_reader_reports_malformed_and_short_particle_files(tmp_path):
    """rw_create reads <project>.dat (src/loquat_io.cu:222-264) on several host threads
    before it touches the GPU: a malformed line deep in a large file is reported with
    its index, as a line-by-line read would, and so is a file that ends early."""
    import ctypes as ct

    from retainwall_code_b200 import _lib, cases as C

    case = C.column_collapse()  # 27,648 soil particles: the reader splits the file across threads
    proj = str(tmp_path / "col")
    C.write_case(case, proj)
    lines = open(proj + ".dat").read().split("\n")
    L = _lib.lib()

    def create_error():
        ctx = ct.c_void_p()
        st = L.rw_create(proj.encode(), 0, 4, ct.byref(ctx))
        assert st != 0
        return L.rw_last_error(None).decode()

    bad = list(lines)
    bad[20000] = bad[20000].split(" ")[0] + " 1 2 x"
    open(proj + ".dat", "w").write("\n".join(bad))
    assert "malformed particle line 20000" in create_error()
    open(proj + ".dat", "w").write("\n".join(lines[:30000]) + "\n")
    assert "ends before particle 30000" in create_error()
