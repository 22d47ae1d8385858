"""The oracle's constitutive restatement against the reference's own functions
(src/constitutive_model.h, src/functions.h compiled on the host by oracle/build_ref.sh;
known answers in tests/golden/hypo_ref.npz, made by tests/golden/make_hypo_golden.py).

Float build: bit-exact.  Double build: the reference's FP64 build still takes sqrtf of
the strain-rate norm and of the deviatoric invariant (src/constitutive_model.h:177,254,290);
the project's FP64 path is true double, so agreement is to float rounding (1e-7)."""
import numpy as np
import pytest

from oracle import oracle as O
from retainwall_code_b200.cases import hypocs_model

G = np.load("tests/golden/hypo_ref.npz")
N = len(G["rho"])


def _args(i, npt):
    par = np.asarray(hypocs_model(G["phi"][i], G["e0"][i], 1850.0), npt).astype(np.float64)
    f = lambda a: np.asarray(a, npt).astype(np.float64)
    return par, f(G["om"][i]), f(G["rate"][i]), f(G["sig"][i]), float(npt(G["dt"][i])), float(npt(G["rho"][i]))


def test_hypo_cs_float_bit_exact():
    for i in range(N):
        par, om, rate, sig, dt, rho = _args(i, np.float32)
        s, m = O.hypo_cs(4, dt, rho, om, rate, sig, par)
        np.testing.assert_array_equal(s.astype(np.float32), G["f32/hypo_cs"][i], err_msg=str(i))
        assert np.float32(m) == G["f32/m_crt"][i], i


def test_hypo_basic_float_bit_exact():
    for i in range(N):
        par, om, rate, sig, dt, _ = _args(i, np.float32)
        s = O.hypo_basic(4, dt, om, rate, sig, par)
        np.testing.assert_array_equal(s.astype(np.float32), G["f32/hypo_basic"][i], err_msg=str(i))


@pytest.mark.parametrize("prec,tag,npt", [(4, "f32", np.float32), (8, "f64", np.float64)])
def test_wendland_kernel_bit_exact(prec, tag, npt):
    L = O.lib()
    for i in range(N):
        q = float(npt(G["q"][i]))
        assert npt(L.orc_kernel_w(prec, float(npt(1234.5)), q)) == G[f"{tag}/kernel_w"][i]
        assert npt(L.orc_kernel_f(prec, float(npt(-98765.4)), q)) == G[f"{tag}/kernel_f"][i]


def test_hypo_cs_double_to_float_sqrt_rounding():
    worst = 0.0
    for i in range(N):
        par, om, rate, sig, dt, rho = _args(i, np.float64)
        s, m = O.hypo_cs(8, dt, rho, om, rate, sig, par)
        r = G["f64/hypo_cs"][i]
        worst = max(worst, np.linalg.norm(s - r) / max(np.linalg.norm(r), 1e-300))
        assert m == G["f64/m_crt"][i]
    assert worst < 1e-7


@pytest.mark.parametrize("prec,tag,npt", [(4, "f32", np.float32), (8, "f64", np.float64)])
def test_drucker_prager_models(prec, tag, npt):
    """Drucker-Prager (cuMatModDP, src/constitutive_model.h:38-84) and mu(I)-DP
    (cuMatModMuIDP, :90-130), restated by the oracle, against the reference's own
    functions on every third sample (cohesion, dilatancy, tension and shear yield
    among them).  Float: bit-exact, yield flags included.  Double: mu(I)-DP bit-exact;
    DP to float rounding, because the reference's FP64 build takes sqrtf of the
    equivalent shear stress (:69) where the project's FP64 path is true double."""
    from tests.golden.make_hypo_golden import plastic_params

    worst = 0.0
    for i in range(0, N, 3):
        _, om, rate, sig, dt, _ = _args(i, npt)
        pdp, pmu = (np.asarray(v, npt).astype(np.float64) for v in plastic_params(i, G["phi"][i]))
        s, y = O.dp(prec, dt, om, rate, sig, pdp)
        r = G[f"{tag}/dp"][i]
        if prec == 4:
            np.testing.assert_array_equal(s.astype(npt), r, err_msg=f"dp {i}")
            assert y == G[f"{tag}/dp_yield"][i], i
        else:
            worst = max(worst, np.linalg.norm(s - r) / max(np.linalg.norm(r), 1e-300))
        s, _ = O.dp(prec, dt, om, rate, sig, pmu, mui=True)
        np.testing.assert_array_equal(s.astype(npt), G[f"{tag}/mui_dp"][i], err_msg=f"mui_dp {i}")
    assert worst < 1e-7
