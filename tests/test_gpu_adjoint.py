"""Adjoint model (uwshcu_adjoint_device): the transpose of the tangent-linear model.

Dot-product test: for a random direction d in (t0, qv0, tke, pblh, rpen, rle, rkm, criqc) and random
cotangents w on every differentiable output, the tangent-linear model gives <w, TL d> and the adjoint
gives <ADJ w, d>, column by column.  Both linearise the same FP64 computation (the branch the FP64
path takes) and multiply the same partial derivatives in opposite orders, so they agree to the
rounding of that product.  Most columns agree to ~1e-15 of the column's sum of |terms|; a column
whose derivative is ill-conditioned (intermediate derivatives many orders above the outputs', which
cancel) amplifies rounding, and the two models amplify it differently (the tangent model in its
tangents, the adjoint in its adjoints).  The bar measures each model's amplification on the column
with that model alone, by its defect of linearity under a split of its argument:
|<w, TL d> - <w, TL d1> - <w, TL d2>| for d = d1 + d2, and |<ADJ w, d> - <ADJ w1, d> - <ADJ w2, d>| for
w = w1 + w2.  Every convecting column must satisfy |<w, TL d> - <ADJ w, d>| <= 1e-9 |terms| + 10 x
(the sum of the two defects), and the median column 1e-13.  The adjoint's forward sweep also
reproduces the FP64 outputs bit for bit.  The tangent-linear model itself is checked against finite
differences in test_gpu_tangent.py.

uwshcu_adjoint_device_checked gives the same bits and, per column, the adjoint's defect of linearity
under its own split of the cotangents (on the same tape): the median convecting column's defect is at
rounding level, at most 1 % of the columns exceed 1e-8, and every column whose dot products disagree by
more than 1e-7 of |terms| is among those.
"""
import numpy as np
import pytest

import soundings

pytestmark = pytest.mark.gpu

OUTS = ("cush umf slflx qtflx flxprc1 flxsnow1 qvten qlten qiten sten uten vten trten qrten qsten precip "
        "snow evapc cufrc qcu qlu qiu cbmf qc rliq wu").split()


@pytest.mark.parametrize("inv,pver", [(0, 30), (1, 30), (0, 51)])
def test_adjoint_dot_product(uw, cuda, inv, pver):
    import torch
    assert uw.init_default() == 0
    s = soundings.make_soundings(2048, pver, seed=301 + inv + pver, rh_pbl=(0.6, 0.95))
    if inv:
        s = soundings.to_inv(s)
    ref = uw.DeviceCase(s)
    assert ref.launch(inv=inv) == 0 and ref.status() == 0
    want = ref.outputs_numpy()
    g = torch.Generator(device="cpu").manual_seed(7 + inv)

    def rnd(t):
        return torch.randn(t.shape, generator=g, dtype=torch.float64).to(t.device) * t.abs().mean().clamp(min=1e-30)

    # direction: a relative perturbation of every differentiated input, and of the parameters
    dirs = {k: rnd(ref.inp[k]) for k in ("t0", "qv0", "tke", "pblh")}
    dparams = (0.3, 0.01, 0.7, 2e-5)
    case_t = uw.DeviceCase(s, inputs=ref.inp)
    tout = uw.tangent_launch(case_t, dirs, dparams, inv=inv)
    torch.cuda.synchronize()
    # cotangents: random, scaled to each output's size
    cot = {k: torch.randn(ref.out[k].shape, generator=g, dtype=torch.float64).to(ref.out[k].device)
           / ref.out[k].abs().mean().clamp(min=1e-30) for k in OUTS}
    case_a = uw.DeviceCase(s, inputs=ref.inp)
    rc, grads = uw.adjoint_launch(case_a, cot, inv=inv)
    assert rc == 0, (rc, uw.last_cuda_error())
    records = uw.adjoint_last_records()
    assert 0 < records
    # the forward sweep's outputs are the FP64 path's
    got = case_a.outputs_numpy()
    diff = [k for k in want if not np.array_equal(want[k], got[k])]
    assert not diff, diff
    n = s["ncol"]

    def per_col(t):
        return t.reshape(-1, n).sum(0)
    lhs = sum(per_col(cot[k] * tout[k]) for k in OUTS)
    scl = sum(per_col((cot[k] * tout[k]).abs()) for k in OUTS)
    rhs = sum(per_col(grads[k] * dirs[k]) for k in ("t0", "qv0", "tke", "pblh"))
    rhs = rhs + sum(grads[k] * p for k, p in zip(("rpen", "rle", "rkm", "criqc"), dparams))
    # the tangent-linear model's own defect of linearity: d = d1 + d2 (d2 = d - d1)
    d1 = {k: v * torch.rand(v.shape, generator=g, dtype=torch.float64).to(v.device) for k, v in dirs.items()}
    d2 = {k: dirs[k] - d1[k] for k in dirs}
    p1 = tuple(p * 0.37 for p in dparams)
    p2 = tuple(p - q for p, q in zip(dparams, p1))
    t1 = uw.tangent_launch(uw.DeviceCase(s, inputs=ref.inp), d1, p1, inv=inv)
    t2 = uw.tangent_launch(uw.DeviceCase(s, inputs=ref.inp), d2, p2, inv=inv)
    torch.cuda.synchronize()
    lin = (lhs - sum(per_col(cot[k] * (t1[k] + t2[k])) for k in OUTS)).abs()
    # the adjoint's own defect of linearity: w = w1 + w2 (w2 = w - w1)
    w1 = {k: v * torch.rand(v.shape, generator=g, dtype=torch.float64).to(v.device) for k, v in cot.items()}
    w2 = {k: cot[k] - w1[k] for k in cot}
    ga = [uw.adjoint_launch(uw.DeviceCase(s, inputs=ref.inp), w, inv=inv) for w in (w1, w2)]
    assert all(rc_ == 0 for rc_, _ in ga)

    def dot_adj(gr):
        r = sum(per_col(gr[k] * dirs[k]) for k in ("t0", "qv0", "tke", "pblh"))
        return r + sum(gr[k] * p for k, p in zip(("rpen", "rle", "rkm", "criqc"), dparams))
    lin_adj = (rhs - dot_adj(ga[0][1]) - dot_adj(ga[1][1])).abs()
    conv = torch.from_numpy(want["cush"] != -1.0).to(lhs.device) & (scl > 0)
    assert int(conv.sum()) > 200, int(conv.sum())
    assert bool(torch.isfinite(lhs).all()) and bool(torch.isfinite(rhs).all())
    err = (lhs - rhs).abs()
    excess = ((err - 1e-9 * scl).clamp(min=0.0) / (lin + lin_adj).clamp(min=1e-300))[conv]
    print("dot product: largest mismatch beyond 1e-9 |terms|, in units of the two defects: %.3g; "
          "columns with any such mismatch: %d of %d" % (float(excess.max()), int((excess > 0).sum()), int(conv.sum())))
    bound = 1e-9 * scl + 10.0 * (lin + lin_adj)
    bad = torch.nonzero(conv & (err > bound)).flatten().tolist()
    assert not bad, [(c, float(err[c] / scl[c]), float(lin[c] / scl[c]), float(lin_adj[c] / scl[c])) for c in bad[:8]]
    rel = (err / scl.clamp(min=1e-300))[conv].cpu().numpy()
    assert np.median(rel) <= 1e-13, np.median(rel)
    # the columns that leave the scheme in the trigger pass have zero gradients
    quiet = torch.from_numpy(want["cush"] == -1.0).to(grads["t0"].device)
    assert float(grads["t0"][:, quiet].abs().max()) == 0.0
    # uwshcu_adjoint_device_checked: the same bits, and a defect per column that flags the columns
    # whose dot products disagree
    case_c = uw.DeviceCase(s, inputs=ref.inp)
    rc, gc = uw.adjoint_launch(case_c, cot, inv=inv, defect=True)
    assert rc == 0, (rc, uw.last_cuda_error())
    assert all(torch.equal(gc[k], grads[k]) for k in grads)
    got_c = case_c.outputs_numpy()
    assert all(np.array_equal(want[k], got_c[k]) for k in want)
    defect = gc["defect"]
    assert bool(torch.isfinite(defect).all()) and float(defect.min()) >= 0.0
    assert float(defect[quiet].abs().max()) == 0.0
    dc = defect[conv].cpu().numpy()
    assert np.median(dc) <= 1e-12, np.median(dc)
    flagged = int((defect[conv] > 1e-8).sum())
    assert flagged <= 0.01 * int(conv.sum()), flagged
    unflagged_bad = torch.nonzero(conv & (err > 1e-7 * scl) & (defect <= 1e-8)).flatten().tolist()
    assert not unflagged_bad, [(c, float(err[c] / scl[c]), float(defect[c])) for c in unflagged_bad[:8]]


def test_adjoint_capacity_and_buffer_reuse(uw, cuda):
    """Repeated calls reuse the adjoint buffer and size the tapes from the previous call; a capacity
    that is too small makes the call start again at the full one.  Every variant gives the same
    bits (each lane's reductions run in its own program order)."""
    import torch
    assert uw.init_default() == 0
    s = soundings.make_soundings(1500, 30, seed=305, rh_pbl=(0.6, 0.95))
    case = uw.DeviceCase(s)
    g = torch.Generator(device="cpu").manual_seed(3)
    cot = {k: torch.randn(v.shape, generator=g, dtype=torch.float64).to(v.device) for k, v in case.out.items()
           if k in uw.ADJ_OUTPUTS}
    runs = []
    try:
        for rows in (0, None, 4096, None, "release"):
            if rows == "release":
                assert uw.adjoint_release() == 0
            elif rows is not None:
                assert uw.set_adjoint_rows(rows) == 0
            case.reset_cush()
            rc, grads = uw.adjoint_launch(case, cot)
            assert rc == 0, (rows, rc, uw.last_cuda_error())
            runs.append((uw.adjoint_last_records(), {k: v.cpu().numpy() for k, v in grads.items()},
                         case.outputs_numpy()))
    finally:
        uw.set_adjoint_rows(0)
    assert runs[0][0] > 4096   # the 4096-row call overflowed and started again
    for j, (recs, gr, out) in enumerate(runs[1:], 1):
        assert recs == runs[0][0], (j, recs, runs[0][0])
        assert all(np.array_equal(gr[k], runs[0][1][k]) for k in gr), j
        # the restarted call computed its outputs from the cush the trigger pass left
        assert all(np.array_equal(out[k], runs[0][2][k]) for k in out), j
    assert np.any(runs[0][1]["t0"])
