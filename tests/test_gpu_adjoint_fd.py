"""The adjoint gradient against central finite differences of the FP64 path (no tangent-linear model
in between), for the objective of the adjoint benchmark: per column
    J = precip + column-integrated heating = precip + sum_k sten(k) dp0(k) / g,
with respect to t0, qv0, tke and pblh (a random direction per column) and to the tuning parameters
rpen, rle, rkm and criqc, at their defaults and at the defaults perturbed by -10 % and +10 %, at 30
levels and (default parameters) at 51 levels.

Central differences with relative steps h and h/4 (h = 1e-6 and 1e-7) of the perturbed quantities (every element
of t0, qv0, tke and pblh moves by a random fraction of up to h of its value; a parameter by h of its
value), combined by Richardson extrapolation.  The scheme is only piecewise smooth (trigger, cloud
base and top, the many limiters), so a column counts only where it is away from a branch switch in
the step: its decisions, limiter flags and level indices are the same at x - h d, x and x + h d, and
the two differences agree to 1e-3 (the test requires half of the convecting columns).  On those
columns the adjoint's <grad J, d> must match the extrapolated difference within 1e-4 relative (floor:
1e-6 of the largest) on the fraction of the columns CASES gives, with a median below 1e-5."""
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


def _check(fd1, fd2, ad, same):
    """Columns away from a branch switch (same decisions, the two step sizes agree to 1e-3) and the
    adjoint's relative error there against the Richardson extrapolation of the two differences."""
    fdr = (4.0 * fd2 - fd1) / 3.0
    floor = 1e-6 * float(fdr[same].abs().max()) if bool(same.any()) else 0.0
    den = fdr.abs().clamp(min=floor + 1e-300)
    smooth = same & ((fd1 - fd2).abs() <= 1e-3 * den)
    err = ((ad - fdr).abs() / den)[smooth].cpu().numpy()
    return int(smooth.sum()), err


# (parameter scale, relative step h of the inputs, bar for the inputs): the fraction of the columns
# away from a branch switch whose error is within 1e-4.  The saturation table is piecewise linear in T
# with a knot every 1 K (wv_saturation.F90:64-80); a step of 1e-6 of T (0.3 mK) crosses a knot in
# about one saturation evaluation in 1,600, and a convecting column makes thousands, so the larger
# step sees more kinks that the two-step check does not catch (measured: 96.9 % within 1e-4 at
# h = 1e-6, 98.8-99.8 % at 1e-7).  The parameters always take h = 1e-6: J is much less sensitive to
# them than to the inputs, and at 1e-7 the differences of J drown in its rounding (rle: 67 % within
# 1e-4 at 1e-7, 94 % at 1e-6).  Parameter bars: 0.9 for rle, 0.95 for rpen, rkm and criqc.
CASES = [(1.0, 1e-6, 0.95, 30), (1.0, 1e-7, 0.98, 30), (0.9, 1e-7, 0.98, 30), (1.1, 1e-7, 0.98, 30),
         (1.0, 1e-7, 0.97, 51)]   # 51 levels (the 64-level unit): more saturation evaluations per
                                  # column, so more knots in the step (measured 97.6 % within 1e-4)
H_PARAM = 1e-6
BAR_PARAM = {"rpen": 0.95, "rle": 0.90, "rkm": 0.95, "criqc": 0.95}


@pytest.mark.parametrize("pscale,h,bar_in,pver", CASES)
def test_adjoint_against_central_differences(uw, cuda, pscale, h, bar_in, pver):
    torch = cuda
    assert uw.init_default() == 0
    params = tuple(p * pscale for p in DEFAULTS)
    s = soundings.make_soundings(4096, pver, seed=401, rh_pbl=(0.6, 0.95))
    case = uw.DeviceCase(s, diag=True)
    assert uw.set_params(*params) == 0
    case.reset_cush()
    assert case.launch() == 0 and case.status() == 0
    conv = case.out["cush"] != -1.0
    n, mkx = case.n, case.mkx
    cot = {"precip": torch.ones(n, dtype=torch.float64, device="cuda"),
           "sten": (case.inp["dp0"] / G).clone()}
    try:
        case.reset_cush()          # the adjoint's forward sweep reads cush as the call's input
        rc, grads = uw.adjoint_launch(case, cot)
        assert rc == 0, (rc, uw.last_cuda_error())
        gen = torch.Generator(device="cpu").manual_seed(17)

        # a relative direction in the four input fields: every element moves by up to h of its value
        d = {k: (2.0 * torch.rand(case.inp[k].shape, generator=gen, dtype=torch.float64) - 1.0).to(case.inp[k].device)
             * case.inp[k].abs() for k in ("t0", "qv0", "tke", "pblh")}
        dirg = sum((grads[k] * d[k]).reshape(-1, n).sum(0) for k in d)

        def shifted(h):
            return {k: (v + h * d[k] if k in d else v) for k, v in case.inp.items()}

        def fd(h):
            jp, dp = _run(uw, case, params, shifted(h))
            jm, dm = _run(uw, case, params, shifted(-h))
            same = (dp == case.diag_int).all(0) & (dm == case.diag_int).all(0)
            return (jp - jm) / (2 * h), same
        fd1, same1 = fd(h)
        fd2, same2 = fd(h / 4)
        nsm, err = _check(fd1, fd2, dirg, conv & same1 & same2)
        print("inputs: %d of %d convecting columns away from a branch switch; error median %.2e, "
              "within 1e-4: %.4f" % (nsm, int(conv.sum()), np.median(err), np.mean(err <= 1e-4)))
        res = [("inputs", nsm, err)]
        # each tuning parameter (per-column gradients; the parameter is one scalar for all columns)
        for p, name in enumerate(PARAMS):
            dirp = grads[name] * params[p]
            out = []
            for hh in (H_PARAM, H_PARAM / 4):
                pp = list(params)
                pp[p] = params[p] * (1 + hh)
                jp, dp = _run(uw, case, pp)
                pp[p] = params[p] * (1 - hh)
                jm, dm = _run(uw, case, pp)
                out.append(((jp - jm) / (2 * hh), (dp == case.diag_int).all(0) & (dm == case.diag_int).all(0)))
            nsm, err = _check(out[0][0], out[1][0], dirp, conv & out[0][1] & out[1][1])
            res.append((name, nsm, err))
        ncv = int(conv.sum())
        for name, nsm, err in res:
            print("scale %.1f h %g %-6s: %d of %d convecting columns away from a branch switch; error "
                  "median %.2e, within 1e-4 %.4f" % (pscale, h, name, nsm, ncv, np.median(err), np.mean(err <= 1e-4)))
        for name, nsm, err in res:
            assert nsm >= 0.5 * ncv, (name, nsm, ncv)
            bar = bar_in if name == "inputs" else BAR_PARAM[name]
            assert np.mean(err <= 1e-4) >= bar, (name, np.mean(err <= 1e-4), np.sort(err)[-5:])
            assert np.median(err) <= 1e-5, (name, np.median(err))
    finally:
        assert uw.set_params(*DEFAULTS) == 0
