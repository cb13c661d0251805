"""Pin the CPU oracle to the reference.

The reference has no tests or golden data, and no Fortran compiler exists here, so the oracle is
pinned against the reference's own C++ restatement of the same Fortran: the in-model drop-in
src/physics/bxcompute_uwshcu_inv.cpp, compiled unchanged for the host (oracle/ref).  The fixtures
in tests/golden were produced by that code (tests/golden/make_golden.py).  Agreement is required
bit for bit.  The one known deviation of the drop-in from uwshcu.F90 (it treats every tracer as
'dry' in the positivity fluxes, bxcompute_uwshcu_inv.cpp:4251,4280,4295 vs uwshcu.F90:4024-4028)
is checked to be the only difference when wet tracers are present.
"""
import glob
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "oracle", "ref"))
sys.path.insert(0, os.path.join(HERE, "golden"))

import refdropin  # noqa: E402
import soundings  # noqa: E402

OUTS = ("umf", "slflx", "qtflx", "flxprc1", "flxsnow1", "wu", "qvten", "qlten", "qiten", "sten",
        "uten", "vten", "qrten", "qsten", "evapc", "cufrc", "qcu", "qlu", "qiu", "qc", "trten",
        "precip", "snow", "cbmf", "rliq", "cnt", "cnb", "cush")
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def load_golden(path):
    z = np.load(path)
    n, mkx, nc, seed, dt = z["meta"]
    si = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    si.update(ncol=int(n), mkx=int(mkx), ncnst=int(nc), dt=float(dt))
    ref = {k[4:]: z[k] for k in z.files if k.startswith("out_")}
    return si, ref, z["qmin"], z["wet"], z["consts"], z["estbl"]


def init_oracle(oracle, qmin, wet):
    c = oracle.consts()
    oracle.init(c[0], c[3], c[1], c[4], c[5], c[6], c[7], c[10], 173.16, 375.16, 20.0, 1, c[14],
                c[15], c[16], qmin, wet, 4, 5)


@pytest.fixture
def oracle25(oracle):
    yield oracle
    oracle.init_default()


def test_golden_fixtures_exist():
    assert len(GOLDEN) >= 2


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_reproduces_reference_fixture_bit_for_bit(oracle25, path):
    si, ref, qmin, wet, consts, estbl = load_golden(path)
    init_oracle(oracle25, qmin, wet)
    assert np.array_equal(oracle25.consts(), consts)
    assert np.array_equal(oracle25.estbl(), estbl)
    out = oracle25.compute(si, inv=True)
    for f in OUTS:
        assert np.array_equal(out[f], ref[f]), f


def test_constants_match_the_reference_ports(oracle):
    """Constants as the reference prints them into its ports (src/doubleGPUUWshcu/mpiuwshcu.cpp:36-46
    and the wv_saturation values of src/physics/bxcompute_uwshcu_inv.cpp:64-75)."""
    c = oracle.consts()
    xlv, xlf, xls, cp, zvir, r, g, ep2, p00, rovcp, rpen, tmin, tmax, ttrice, epsqs, rgasv, tmelt = c[:17]
    assert (xlv, xlf, xls, cp, g, p00, rpen) == (2501000.0, 333700.0, 2834700.0, 1004.64, 9.80616, 1e5, 10.0)
    assert abs(zvir - 0.607793072824156) < 5e-16
    assert abs(r - 287.042311365049) < 5e-13
    assert abs(ep2 - 0.621970586204516) < 5e-16
    assert epsqs == float("0.6219705862045155076")
    assert rgasv == float("461.5046398201599231470")
    assert tmin == float("173.1599999999999965894") and tmax == float("375.1600000000000250111")
    assert tmelt == float("273.1499999999999772626") and ttrice == 20.0
    # r/cp, not the 1.2857 the standalone ports hardcode (mpiuwshcu.cpp:96)
    assert abs(rovcp - r / cp) == 0.0 and abs(rovcp - 0.2857165864041) < 1e-12


@pytest.mark.skipif(not refdropin.available(), reason="reference drop-in not built (needs the reference tree)")
@pytest.mark.parametrize("seed", [201, 202])
def test_oracle_matches_live_reference_dropin(oracle25, seed):
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden
    qmin, wet = make_golden.config()
    init_oracle(oracle25, qmin, wet)
    refdropin.init(oracle25.consts(), oracle25.estbl(), qmin, wet)
    s = soundings.make_soundings(256, 30, seed=seed, ncnst=25)
    si = soundings.to_inv(s)
    ref = refdropin.compute_inv(si)
    out = oracle25.compute(si, inv=True)
    for f in OUTS:
        assert np.array_equal(out[f], ref[f]), f
    # with wet tracers the drop-in differs from uwshcu.F90 only in those tracers' tendencies
    wet2 = wet.copy()
    wet2[6::2] = 1
    init_oracle(oracle25, qmin, wet2)
    refdropin.init(oracle25.consts(), oracle25.estbl(), qmin, wet2)
    ref2 = refdropin.compute_inv(si)
    out2 = oracle25.compute(si, inv=True)
    for f in OUTS:
        if f != "trten":
            assert np.array_equal(out2[f], ref2[f]), f
    same = np.all(out2["trten"] == ref2["trten"], axis=(1, 2))
    assert np.all(same[wet2 == 0])
    assert not np.all(same[wet2 == 1][5:])
