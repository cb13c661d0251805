"""Tangent-linear model (uwshcu_tangent_device) against central finite differences of the FP64 path.

Objective per column, as the differentiation targets define it: J = precip + sum_k sten(k) dp0(k)/g.
Directions: relative perturbations of t0, qv0, tke and pblh (uniform in +-1e-3 of each value per
element), and each tuning parameter rpen, rle, rkm, criqc.  98 % of the columns whose central
quotients at two step sizes agree to 1e-3 (no branch switch inside the step) are within 1e-4; and
every convecting column whose central and one-sided quotients agree to 1 % is within 1e-4 + 5 x
their disagreement (the rest, at most 5 % at 30 levels and 15 % at 51, have a jump, a kink or strong
curvature inside the step).  At 51 levels (the 64-level unit) the input steps are 10x smaller: a
column makes more saturation evaluations, so a step crosses more of their kinks."""
import numpy as np
import pytest

import soundings

G = 9.80616
PARAMS = np.array([10.0, 0.1, 14.0, 0.7e-3])   # rpen, rle, rkm, criqc (uwshcu_init_default)


def _J(out, dp0):
    return out["precip"] + (out["sten"] * dp0).sum(0) / G


def _run(uw, s):
    import torch
    c = uw.DeviceCase(s)
    assert c.launch() == 0
    torch.cuda.synchronize()
    return c.outputs_numpy()


def _compare(tl, f1, f2, conv, one_sided, what=""):
    """f1, f2: central difference quotients at steps h and h/4; one_sided: the forward and backward
    quotients at h/4.  Returns the columns where the quotients are smooth, the relative error of the
    tangent against f2, and the columns whose error the difference quotients do not account for.

    The finite differences are their own error bar: where a branch switches inside the step (a jump)
    the two central quotients disagree, and where the objective has a kink (MX, MN, a limiter) the
    forward and backward quotients disagree.  A column whose quotients disagree by more than 1 % is
    not differentiable at this step; every other convecting column must have a tangent within
    1e-4 + 5 x (that disagreement) of f2."""
    scale = max(float(np.abs(f2[conv]).max()), 1e-300)
    den = np.maximum(np.abs(f2), 1e-6 * scale)
    smooth = conv & (np.abs(f1 - f2) <= 1e-3 * den)
    rel = np.abs(tl - f2) / den
    fw, bw = one_sided
    spread = np.maximum(np.abs(f1 - f2), np.abs(fw - bw)) / den
    rough = conv & (spread > 1e-2)
    unexplained = conv & ~rough & (rel > 1e-4 + 5.0 * spread)
    print("%s: %d convecting, %d off by > 1e-4, %d not differentiable at this step, %d unexplained" % (
        what, int(conv.sum()), int((conv & (rel > 1e-4)).sum()), int(rough.sum()), int(unexplained.sum())))
    return smooth, rel, unexplained, rough


@pytest.mark.gpu
# (levels, the two relative steps of the input direction, the share of the convecting columns allowed
# to be non-differentiable at that step): 51 levels make more saturation evaluations per column, so
# they take smaller steps
@pytest.mark.parametrize("pver,steps,rough_max,smooth_min", [(30, (1e-4, 2.5e-5), 0.05, 0.9),
                                                             (51, (1e-5, 2.5e-6), 0.15, 0.85)])
def test_tangent_linear_model(uw, cuda, pver, steps, rough_max, smooth_min):
    import torch
    assert uw.init_default() == 0
    s = soundings.make_soundings(4096, pver, seed=201, rh_pbl=(0.675, 0.93))
    rng = np.random.default_rng(5)
    dirs = {k: s[k] * rng.uniform(-1e-3, 1e-3, s[k].shape) for k in ("t0", "qv0", "tke", "pblh")}
    base = _run(uw, s)
    conv = base["cush"] != -1.0

    # a tangent run computes the FP64 outputs bit for bit
    tc = uw.DeviceCase(s)
    tout = uw.tangent_launch(tc, {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in dirs.items()})
    torch.cuda.synchronize()
    vals = tc.outputs_numpy()
    assert all(np.array_equal(vals[k], base[k]) for k in base)
    tl = tout["precip"].cpu().numpy() + (tout["sten"].cpu().numpy() * s["dp0"]).sum(0) / G

    j0 = _J(base, s["dp0"])

    def fd(h):
        sp, sm = dict(s), dict(s)
        for k, v in dirs.items():
            sp[k], sm[k] = s[k] + h * v, s[k] - h * v
        jp, jm = _J(_run(uw, sp), s["dp0"]), _J(_run(uw, sm), s["dp0"])
        return (jp - jm) / (2 * h), ((jp - j0) / h, (j0 - jm) / h)

    (f1, _), (f2, sided) = fd(steps[0]), fd(steps[1])
    fails = []

    def judge(name, smooth, rel, unexplained, rough):
        within = float(np.mean(rel[smooth] <= 1e-4))
        print("   %s: smooth %d, within 1e-4 on them %.4f" % (name, int(smooth.sum()), within))
        if unexplained.any():
            fails.append((name, "unexplained", np.flatnonzero(unexplained)[:8]))
        if rough.sum() > rough_max * conv.sum():
            fails.append((name, "not differentiable", int(rough.sum())))
        if smooth.sum() < smooth_min * conv.sum():
            fails.append((name, "smooth", int(smooth.sum())))
        if within < 0.98:
            fails.append((name, "within 1e-4", within, np.percentile(rel[smooth], [50, 90, 99])))

    judge("inputs", *_compare(tl, f1, f2, conv, sided, "inputs %d levels" % pver))

    # tuning parameters, one at a time
    try:
        for j, name in enumerate(("rpen", "rle", "rkm", "criqc")):
            dp = [0.0] * 4
            dp[j] = PARAMS[j] * 1e-3
            tc = uw.DeviceCase(s)
            to = uw.tangent_launch(tc, None, dp)
            torch.cuda.synchronize()
            tlp = to["precip"].cpu().numpy() + (to["sten"].cpu().numpy() * s["dp0"]).sum(0) / G
            fds = []
            for h in (1e-3, 2.5e-4):
                pp, pm = PARAMS.copy(), PARAMS.copy()
                pp[j] += h * dp[j]
                pm[j] -= h * dp[j]
                assert uw.set_params(*pp) == 0
                jp = _J(_run(uw, s), s["dp0"])
                assert uw.set_params(*pm) == 0
                jm = _J(_run(uw, s), s["dp0"])
                fds.append(((jp - jm) / (2 * h), ((jp - j0) / h, (j0 - jm) / h)))
            assert uw.set_params(*PARAMS) == 0
            judge(name, *_compare(tlp, fds[0][0], fds[1][0], conv, fds[1][1], name))
    finally:
        assert uw.init_default() == 0
    assert not fails, fails
