"""Born modelling and its adjoint in the CPU oracle: adjointness and linearisation."""
import numpy as np

from _born_case import born_case, oracle_shot


def test_dot_product(orc):
    c = born_case(orc)
    s = oracle_shot(orc, c)
    rng = c["rng"]
    m = [(0.05 * rng.standard_normal(c["shape"])).astype(np.float32) for _ in range(3)]
    d = orc.born_forward(c["g"], c["vp"], c["vs"], c["rho"], s, c["nt"], *m)
    dh = rng.standard_normal(d.shape).astype(np.float32)
    dh[1] = 0
    gm = orc.born_adjoint(c["g"], c["vp"], c["vs"], c["rho"], s, c["nt"], dh)
    lhs = float(np.sum(d.astype(np.float64) * dh))
    rhs = sum(float(np.sum(a.astype(np.float64) * b)) for a, b in zip(m, gm))
    # inputs and outputs are float32, so agreement is at float32 rounding
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)


def _perturbed(c, dirn, eps):
    out = []
    for base, d in zip((c["vp"], c["vs"], c["rho"]), dirn):
        out.append((base.astype(np.float64) * (1 + eps * d)).astype(np.float32))
    return out


def test_born_is_the_derivative_of_modelling(orc):
    c = born_case(orc)
    s = oracle_shot(orc, c)
    rng = c["rng"]
    m = [(0.05 * rng.standard_normal(c["shape"])).astype(np.float32) for _ in range(3)]
    d = orc.born_forward(c["g"], c["vp"], c["vs"], c["rho"], s, c["nt"], *m).astype(np.float64)
    errs = []
    for eps in (4e-2, 2e-2):
        dp = orc.run_pass(c["g"], *_perturbed(c, m, eps), s, orc.MODEL, c["nt"])["data"]
        dm = orc.run_pass(c["g"], *_perturbed(c, m, -eps), s, orc.MODEL, c["nt"])["data"]
        fd = (dp.astype(np.float64) - dm) / (2 * eps)
        errs.append(np.linalg.norm(fd - d) / np.linalg.norm(d))
    assert errs[1] < 1e-4
    assert errs[1] < errs[0] / 2.5          # second-order convergence of the centred difference


def test_misfit_gradient_matches_finite_differences(orc):
    c = born_case(orc)
    s = oracle_shot(orc, c)
    rng = c["rng"]
    true = [(0.5 * rng.standard_normal(c["shape"])).astype(np.float32) for _ in range(3)]
    dobs = orc.run_pass(c["g"], *_perturbed(c, true, 0.1), s, orc.MODEL, c["nt"])["data"].astype(
        np.float64)
    d0 = orc.run_pass(c["g"], c["vp"], c["vs"], c["rho"], s, orc.MODEL, c["nt"])["data"]
    grad = orc.born_adjoint(c["g"], c["vp"], c["vs"], c["rho"], s, c["nt"],
                            (d0.astype(np.float64) - dobs).astype(np.float32))
    dirn = [rng.standard_normal(c["shape"]).astype(np.float32) for _ in range(3)]
    gdot = sum(float(np.sum(a.astype(np.float64) * b)) for a, b in zip(grad, dirn))

    def J(eps):
        dd = orc.run_pass(c["g"], *_perturbed(c, dirn, eps), s, orc.MODEL, c["nt"])["data"]
        return 0.5 * float(np.sum((dd.astype(np.float64) - dobs) ** 2))

    errs = [abs((J(e) - J(-e)) / (2 * e) - gdot) / abs(gdot) for e in (1e-2, 5e-3)]
    assert errs[1] < 5e-3, errs
    assert errs[1] < errs[0] / 2.5, errs
