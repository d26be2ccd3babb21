"""Viscoelastic (GSLS-3) Born operators in the CPU oracle: the relaxation fit,
attenuation of the modelled data, adjointness and the misfit gradient."""
import numpy as np

from _born_case import VISCO, born_case, oracle_shot, visco_case


def test_visco_fit_gives_near_constant_q(orc):
    ts, tp, tsh = orc.visco_fit(*VISCO)
    assert len(ts) == 3 and tp > 0 and tsh > 0
    assert abs(tsh / tp - 2.0) < 1e-12                   # Qs = Qp / 2
    w = 2 * np.pi * np.geomspace(15.0 / 4, 15.0 * 4, 50)
    S = sum(w * t / (1 + (w * t) ** 2) for t in ts)
    q = 1.0 / (tp * S)
    assert np.all(np.abs(q / 100.0 - 1.0) < 0.15), q    # within 15 % of Qp over two octaves


def test_attenuation_reduces_the_recorded_energy(orc):
    ce, cv = born_case(orc), visco_case(orc)
    s = oracle_shot(orc, ce)
    de = orc.visco_model(ce["g"], ce["vp"], ce["vs"], ce["rho"], s, ce["nt"])
    dv = orc.visco_model(cv["g"], cv["vp"], cv["vs"], cv["rho"], s, cv["nt"])
    # elastic background scheme = the modelling pass of the main oracle
    dr = orc.run_pass(ce["g"], ce["vp"], ce["vs"], ce["rho"], s, orc.MODEL, ce["nt"])["data"]
    assert np.linalg.norm(de - dr) <= 1e-6 * np.linalg.norm(dr)
    ee, ev = float(np.sum(de.astype(np.float64) ** 2)), float(np.sum(dv.astype(np.float64) ** 2))
    assert 0.5 * ee < ev < ee


def test_visco_dot_product(orc):
    c = visco_case(orc)
    s = oracle_shot(orc, c)
    rng = c["rng"]
    m = [(0.05 * rng.standard_normal(c["shape"])).astype(np.float32) for _ in range(3)]
    d = orc.born_forward(c["g"], c["vp"], c["vs"], c["rho"], s, c["nt"], *m)
    dh = rng.standard_normal(d.shape).astype(np.float32)
    dh[1] = 0
    gm = orc.born_adjoint(c["g"], c["vp"], c["vs"], c["rho"], s, c["nt"], dh)
    lhs = float(np.sum(d.astype(np.float64) * dh))
    rhs = sum(float(np.sum(a.astype(np.float64) * b)) for a, b in zip(m, gm))
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)


def _perturbed(c, dirn, eps):
    return [(b.astype(np.float64) * (1 + eps * d)).astype(np.float32)
            for b, d in zip((c["vp"], c["vs"], c["rho"]), dirn)]


def test_visco_born_is_the_derivative_of_modelling(orc):
    c = visco_case(orc)
    s = oracle_shot(orc, c)
    rng = c["rng"]
    m = [(0.05 * rng.standard_normal(c["shape"])).astype(np.float32) for _ in range(3)]
    d = orc.born_forward(c["g"], c["vp"], c["vs"], c["rho"], s, c["nt"], *m).astype(np.float64)
    errs = []
    for eps in (4e-2, 2e-2):
        dp = orc.visco_model(c["g"], *_perturbed(c, m, eps), s, c["nt"])
        dm = orc.visco_model(c["g"], *_perturbed(c, m, -eps), s, c["nt"])
        fd = (dp.astype(np.float64) - dm) / (2 * eps)
        errs.append(np.linalg.norm(fd - d) / np.linalg.norm(d))
    assert errs[1] < 1e-4, errs
    assert errs[1] < errs[0] / 2.5, errs


def test_visco_misfit_gradient_matches_finite_differences(orc):
    c = visco_case(orc)
    s = oracle_shot(orc, c)
    rng = c["rng"]
    true = [(0.5 * rng.standard_normal(c["shape"])).astype(np.float32) for _ in range(3)]
    dobs = orc.visco_model(c["g"], *_perturbed(c, true, 0.1), s, c["nt"]).astype(np.float64)
    d0 = orc.visco_model(c["g"], c["vp"], c["vs"], c["rho"], s, c["nt"])
    grad = orc.born_adjoint(c["g"], c["vp"], c["vs"], c["rho"], s, c["nt"],
                            (d0.astype(np.float64) - dobs).astype(np.float32))
    dirn = [rng.standard_normal(c["shape"]).astype(np.float32) for _ in range(3)]
    gdot = sum(float(np.sum(a.astype(np.float64) * b)) for a, b in zip(grad, dirn))

    def J(eps):
        dd = orc.visco_model(c["g"], *_perturbed(c, dirn, eps), s, c["nt"])
        return 0.5 * float(np.sum((dd.astype(np.float64) - dobs) ** 2))

    errs = [abs((J(e) - J(-e)) / (2 * e) - gdot) / abs(gdot) for e in (1e-2, 5e-3)]
    assert errs[1] < 5e-3, errs
    assert errs[1] < errs[0] / 2.5, errs
