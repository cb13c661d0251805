"""The adjoint gradient against central finite differences of the FP64 path (no tangent-linear model
in between), for the objective of the adjoint benchmark: per column
    J = precip + column-integrated heating = precip + sum_k sten(k) dp0(k) / g,
with respect to t0, qv0, tke and pblh (a random direction per column) and to the tuning parameters
rpen, rle, rkm and criqc, at their defaults and at the defaults perturbed by -10 % and +10 %.

Central differences with a relative step h = 1e-6 of the perturbed quantities.  The scheme is only
piecewise smooth (trigger, cloud base and top, the many limiters), so a column counts only where it
is away from a branch switch in the step: its decisions and level indices are the same at x - h d,
x and x + h d, and the differences with steps h and h/4 agree to 1e-3.  On those columns the
adjoint's <grad J, d> must match the central difference within 1e-4 relative (of |J| + the size of
the directional derivative) on at least 98 % of the columns, with a median below 1e-6."""
import numpy as np
import pytest

import soundings

pytestmark = pytest.mark.gpu

G = 9.80616
PARAMS = ("rpen", "rle", "rkm", "criqc")
DEFAULTS = (10.0, 0.1, 14.0, 0.7e-3)


def _j(case):
    o = case.out
    return o["precip"] + (o["sten"] * case.inp["dp0"]).sum(0) / G


def _run(uw, case, params, inputs=None):
    assert uw.set_params(*params) == 0
    c = uw.DeviceCase.__new__(uw.DeviceCase)
    c.__dict__.update(case.__dict__)
    if inputs is not None:
        c.inp = inputs
    c.out = {k: v.clone() for k, v in case.out.items()}
    c.diag_int = case.diag_int.clone()
    c.reset_cush()
    assert c.launch() in (0, 4)
    return _j(c), c.diag_int.clone()


def _check(fd1, fd2, dirg, jj, same):
    scale = jj.abs() + dirg.abs() + 1e-30
    smooth = same & ((fd1 - fd2).abs() <= 1e-3 * scale)
    err = ((fd1 - dirg).abs() / scale)[smooth].cpu().numpy()
    return int(smooth.sum()), err


@pytest.mark.parametrize("pscale", [1.0, 0.9, 1.1])
def test_adjoint_against_central_differences(uw, cuda, pscale):
    torch = cuda
    assert uw.init_default() == 0
    params = tuple(p * pscale for p in DEFAULTS)
    s = soundings.make_soundings(4096, 30, seed=401, rh_pbl=(0.6, 0.95))
    case = uw.DeviceCase(s, diag=True)
    assert uw.set_params(*params) == 0
    case.reset_cush()
    assert case.launch() == 0 and case.status() == 0
    conv = case.out["cush"] != -1.0
    j0 = _j(case)
    n, mkx = case.n, case.mkx
    cot = {"precip": torch.ones(n, dtype=torch.float64, device="cuda"),
           "sten": (case.inp["dp0"] / G).clone()}
    try:
        rc, grads = uw.adjoint_launch(case, cot)
        assert rc == 0, (rc, uw.last_cuda_error())
        gen = torch.Generator(device="cpu").manual_seed(17)

        def rnd(t):
            return torch.randn(t.shape, generator=gen, dtype=torch.float64).to(t.device)

        # a relative direction in the four input fields
        d = {k: rnd(case.inp[k]) * case.inp[k].abs() for k in ("t0", "qv0", "tke", "pblh")}
        dirg = sum((grads[k] * d[k]).reshape(-1, n).sum(0) for k in d)

        def shifted(h):
            return {k: (v + h * d[k] if k in d else v) for k, v in case.inp.items()}

        def fd(h):
            jp, dp = _run(uw, case, params, shifted(h))
            jm, dm = _run(uw, case, params, shifted(-h))
            same = (dp == case.diag_int).all(0) & (dm == case.diag_int).all(0)
            return (jp - jm) / (2 * h), same
        fd1, same1 = fd(1e-6)
        fd2, same2 = fd(2.5e-7)
        nsm, err = _check(fd1, fd2, dirg, j0, conv & same1 & same2)
        assert nsm >= 0.8 * int(conv.sum()), (nsm, int(conv.sum()))
        assert np.mean(err <= 1e-4) >= 0.98, (np.mean(err <= 1e-4), np.sort(err)[-5:])
        assert np.median(err) <= 1e-6, np.median(err)
        # each tuning parameter (per-column gradients; the parameter is one scalar for all columns)
        for p, name in enumerate(PARAMS):
            dirp = grads[name] * params[p]
            out = []
            for h in (1e-6, 2.5e-7):
                pp = list(params)
                pp[p] = params[p] * (1 + h)
                jp, dp = _run(uw, case, pp)
                pp[p] = params[p] * (1 - h)
                jm, dm = _run(uw, case, pp)
                out.append(((jp - jm) / (2 * h), (dp == case.diag_int).all(0) & (dm == case.diag_int).all(0)))
            nsm, err = _check(out[0][0], out[1][0], dirp, j0, conv & out[0][1] & out[1][1])
            assert nsm >= 0.8 * int(conv.sum()), (name, nsm)
            assert np.mean(err <= 1e-4) >= 0.98, (name, np.mean(err <= 1e-4), np.sort(err)[-5:])
    finally:
        assert uw.set_params(*DEFAULTS) == 0
