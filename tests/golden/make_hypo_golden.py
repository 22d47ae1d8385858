"""Known answers of the reference's own constitutive functions.

Loads oracle/_ref/libref_hypo_{f32,f64}.so (src/functions.h + src/constitutive_model.h
compiled on the host by oracle/build_ref.sh, where the reference sources exist) and
evaluates HypoCS, HypoBasic, Drucker-Prager, mu(I)-DP and the Wendland kernel on seeded
inputs covering compression, tension cut-off, the I1 > -4 reset, shear yielding and the
void-ratio clamps.  Writes tests/golden/hypo_ref.npz.

Usage: python tests/golden/make_hypo_golden.py
"""
import ctypes as ct
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from retainwall_code_b200.cases import dp_model, hypocs_model, mui_dp_model  # noqa: E402


def inputs(n=4000, seed=11):
    rng = np.random.default_rng(seed)
    p = 10 ** rng.uniform(0.0, 5.5, n)                     # mean pressure 1 Pa .. 300 kPa
    dev = rng.normal(0, 1, (n, 6)) * (p[:, None] * rng.uniform(0, 1.2, (n, 1)))
    sig = dev.copy()
    sig[:, :3] -= p[:, None]
    sig[rng.uniform(size=n) < 0.05, :3] *= -1.0           # some tensile states
    rate = rng.normal(0, 1, (n, 6)) * 10 ** rng.uniform(-6, 0, (n, 1))
    om = np.zeros((n, 4))
    om[:, :3] = rng.normal(0, 1, (n, 3)) * 10 ** rng.uniform(-6, 0, (n, 1))
    rho = 1850.0 * rng.uniform(0.78, 1.22, n)
    dt = 10 ** rng.uniform(-7, -4, n)
    phi = rng.uniform(28, 40, n)
    e0 = rng.uniform(0.55, 0.80, n)
    q = rng.uniform(0.0, 2.2, n)
    return sig, rate, om, rho, dt, phi, e0, q


def plastic_params(i, phi):
    """DP and mu(I)-DP parameter vectors of sample i: friction angles from the sample's
    phi (28-40 deg), a cohesion on every third DP sample, a dilatancy on every fifth."""
    dp = dp_model(1850.0, phi_deg=phi - 5.0, psi_deg=5.0 if i % 5 == 0 else 0.0,
                  cohesion=2000.0 if i % 3 == 0 else 0.0)
    mui = mui_dp_model(1850.0, phi1_deg=phi - 10.0, phi2_deg=phi + 2.0)
    return dp, mui


def main():
    out = {}
    sig, rate, om, rho, dt, phi, e0, q = inputs()
    out.update(sig=sig, rate=rate, om=om, rho=rho, dt=dt, phi=phi, e0=e0, q=q)
    for tag, ctype, npt in (("f32", ct.c_float, np.float32), ("f64", ct.c_double, np.float64)):
        L = ct.CDLL(os.path.join(ROOT, "oracle", "_ref", f"libref_hypo_{tag}.so"))
        P = ct.POINTER(ctype)
        L.ref_hypo_cs.argtypes = [ctype, ctype, P, P, P, P, P]
        L.ref_hypo_basic.argtypes = [ctype, P, P, P, P]
        L.ref_dp.argtypes = [ctype, P, P, P, P, ct.POINTER(ct.c_int)]
        L.ref_mui_dp.argtypes = [ctype, P, P, P, P]
        L.ref_kernel_w.restype = ctype
        L.ref_kernel_w.argtypes = [ctype, ctype]
        L.ref_kernel_f.restype = ctype
        L.ref_kernel_f.argtypes = [ctype, ctype]
        n = len(rho)
        cs = np.zeros((n, 6), npt)
        mc = np.zeros(n, npt)
        hb = np.zeros((n, 6), npt)
        kw = np.zeros(n, npt)
        kf = np.zeros(n, npt)
        dpo = np.zeros((n, 6), npt)
        dpy = np.zeros(n, np.int32)
        muo = np.zeros((n, 6), npt)
        for i in range(n):
            par = np.asarray(hypocs_model(phi[i], e0[i], 1850.0), npt)
            s = np.asarray(sig[i], npt).copy()
            r = np.asarray(rate[i], npt)
            o = np.asarray(om[i], npt)
            m = ctype(0)
            L.ref_hypo_cs(npt(dt[i]), npt(rho[i]), o.ctypes.data_as(P), r.ctypes.data_as(P), s.ctypes.data_as(P),
                          par.ctypes.data_as(P), ct.byref(m))
            cs[i], mc[i] = s, m.value
            s = np.asarray(sig[i], npt).copy()
            L.ref_hypo_basic(npt(dt[i]), o.ctypes.data_as(P), r.ctypes.data_as(P), s.ctypes.data_as(P),
                             par.ctypes.data_as(P))
            hb[i] = s
            pdp, pmu = (np.asarray(v, npt) for v in plastic_params(i, phi[i]))
            s = np.asarray(sig[i], npt).copy()
            y = ct.c_int(0)
            L.ref_dp(npt(dt[i]), o.ctypes.data_as(P), r.ctypes.data_as(P), s.ctypes.data_as(P),
                     pdp.ctypes.data_as(P), ct.byref(y))
            dpo[i], dpy[i] = s, y.value
            s = np.asarray(sig[i], npt).copy()
            L.ref_mui_dp(npt(dt[i]), o.ctypes.data_as(P), r.ctypes.data_as(P), s.ctypes.data_as(P),
                         pmu.ctypes.data_as(P))
            muo[i] = s
            kw[i] = L.ref_kernel_w(npt(1234.5), npt(q[i]))
            kf[i] = L.ref_kernel_f(npt(-98765.4), npt(q[i]))
        out.update({f"{tag}/hypo_cs": cs, f"{tag}/m_crt": mc, f"{tag}/hypo_basic": hb, f"{tag}/kernel_w": kw,
                    f"{tag}/kernel_f": kf, f"{tag}/dp": dpo, f"{tag}/dp_yield": dpy, f"{tag}/mui_dp": muo})
    np.savez_compressed(os.path.join(HERE, "hypo_ref.npz"), **out)
    print("wrote", os.path.join(HERE, "hypo_ref.npz"))


if __name__ == "__main__":
    main()
