"""The mixed-precision, tangent-linear and adjoint kernels are generated from the FP64 column code
(csrc/gen_mixed.py, csrc/gen_tangent.py, csrc/gen_adjoint.py).  The committed generated files must be what the
generators produce from the committed FP64 kernel, so that a change to the column code cannot
leave them behind silently."""
import os
import shutil
import subprocess
import sys

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                    "hpc-and-climate-model_b200", "csrc")
INPUTS = ("gen_mixed.py", "gen_tangent.py", "gen_adjoint.py", "uwshcu_fp64_kernel.cuh", "uwshcu_mixed_kernel.cuh",
          "mixed_positive_moisture.inc")


def test_generated_kernels_are_up_to_date(tmp_path):
    for f in INPUTS:
        shutil.copy(os.path.join(CSRC, f), tmp_path / f)
    for gen in ("gen_mixed.py", "gen_tangent.py", "gen_adjoint.py"):
        subprocess.run([sys.executable, str(tmp_path / gen)], check=True, capture_output=True)
    for out in ("uwshcu_mixed_kernel.cuh", "uwshcu_tl_kernel.cuh", "uwshcu_adj_kernel.cuh"):
        assert (tmp_path / out).read_text() == open(os.path.join(CSRC, out)).read(), out
