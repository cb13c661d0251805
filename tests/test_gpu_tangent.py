"""Tangent-linear model (uwshcu_tangent_device) against central finite differences of the FP64 path.

Objective per column, as the differentiation targets define it: J = precip + sum_k sten(k) dp0(k)/g.
Directions: relative perturbations of t0, qv0, tke and pblh (uniform in +-1e-3 of each value per
element), and each tuning parameter rpen, rle, rkm, criqc.  A column is compared only where the
finite-difference quotients at two step sizes agree to 1e-3 (no branch switch inside the step); the
scheme's decisions make the others non-differentiable there."""
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


def _compare(tl, f1, f2, conv):
    scale = max(float(np.abs(f2[conv]).max()), 1e-300)
    smooth = conv & (np.abs(f1 - f2) <= 1e-3 * np.maximum(np.abs(f2), 1e-6 * scale))
    rel = np.abs(tl - f2) / np.maximum(np.abs(f2), 1e-6 * scale)
    return smooth, rel


@pytest.mark.gpu
def test_tangent_linear_model(uw, cuda):
    import torch
    assert uw.init_default() == 0
    s = soundings.make_soundings(4096, 30, seed=201, rh_pbl=(0.675, 0.93))
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

    def fd(h):
        sp, sm = dict(s), dict(s)
        for k, v in dirs.items():
            sp[k], sm[k] = s[k] + h * v, s[k] - h * v
        return (_J(_run(uw, sp), s["dp0"]) - _J(_run(uw, sm), s["dp0"])) / (2 * h)

    smooth, rel = _compare(tl, fd(1e-4), fd(2.5e-5), conv)
    assert smooth.sum() >= 0.9 * conv.sum()
    assert np.mean(rel[smooth] <= 1e-4) >= 0.98, np.percentile(rel[smooth], [50, 90, 99])

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
                fds.append((jp - jm) / (2 * h))
            assert uw.set_params(*PARAMS) == 0
            smooth, rel = _compare(tlp, fds[0], fds[1], conv)
            assert smooth.sum() >= 0.9 * conv.sum(), name
            assert np.mean(rel[smooth] <= 1e-4) >= 0.98, (name, np.percentile(rel[smooth], [50, 90, 99]))
    finally:
        assert uw.init_default() == 0
