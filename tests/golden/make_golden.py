"""Generate the golden fixtures from the reference's own code.

Runs src/physics/bxcompute_uwshcu_inv.cpp of the reference (compiled unchanged for the host by
oracle/ref/Makefile into oracle/_ref/libuwref_dropin.so; needs the reference tree) on seeded
soundings and stores inputs and outputs as compressed .npz files next to this script.

The drop-in's compile-time shape is 30 levels and 25 tracers, and it always weighs the tracer
positivity fluxes with the dry pressure thickness (its 'wet' test is `if(false)`,
bxcompute_uwshcu_inv.cpp:4251,4280,4295), so the fixtures declare every tracer past NUMICE 'dry':
for that configuration the drop-in computes what uwshcu.F90 computes.

Usage: python tests/golden/make_golden.py
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(REPO, "oracle"), os.path.join(REPO, "oracle", "ref"),
                os.path.join(REPO, "hpc-and-climate-model_b200")]

import oracle  # noqa: E402
import refdropin  # noqa: E402
import soundings  # noqa: E402

NCNST = 25
CASES = [("dropin_96x30x25_seed101", 96, 101, (0.70, 0.95)),
         ("dropin_64x30x25_seed102_moist", 64, 102, (0.85, 0.99))]


def config():
    """Tracer metadata of the fixtures: qmin(1) = 1e-12, all others 0; Q, CLDLIQ, CLDICE, NUMLIQ,
    NUMICE wet, the rest dry; ixnumliq = 4, ixnumice = 5."""
    qmin = np.zeros(NCNST)
    qmin[0] = 1e-12
    wet = np.array([1] * 5 + [0] * (NCNST - 5), dtype=np.int32)
    return qmin, wet


def init_oracle_25():
    oracle.init_default()
    c = oracle.consts()
    qmin, wet = config()
    oracle.init(c[0], c[3], c[1], c[4], c[5], c[6], c[7], c[10], 173.16, 375.16, 20.0, 1, c[14],
                c[15], c[16], qmin, wet, 4, 5)
    return qmin, wet


def main():
    # the reference checkout: UWSHCU_REFERENCE_ROOT, else "reference" beside this repository
    ref_root = os.environ.get("UWSHCU_REFERENCE_ROOT") or os.path.join(os.path.dirname(REPO), "reference")
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle", "ref"), "REF_ROOT=" + ref_root],
                   check=True)
    qmin, wet = init_oracle_25()
    refdropin.init(oracle.consts(), oracle.estbl(), qmin, wet)
    for name, n, seed, rh in CASES:
        s = soundings.make_soundings(n, 30, seed=seed, ncnst=NCNST, rh_pbl=rh)
        si = soundings.to_inv(s)
        out = refdropin.compute_inv(si)
        arrays = {"in_" + k: v for k, v in si.items() if isinstance(v, np.ndarray)}
        arrays.update({"out_" + k: v for k, v in out.items()})
        arrays.update(meta=np.array([n, 30, NCNST, seed, si["dt"]]), qmin=qmin, wet=wet,
                      consts=oracle.consts(), estbl=oracle.estbl())
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **arrays)
        print("wrote %s (%d bytes), trigger fraction %.3f"
              % (path, os.path.getsize(path), float(np.mean(out["cush"] != -1.0))))


if __name__ == "__main__":
    main()
