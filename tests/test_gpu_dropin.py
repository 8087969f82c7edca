"""The drop-in: the reference's own CellPoissonFACSolver and
FACPreconditioner running the B200 operators.

oracle/_ref/fac_dropin_driver is the reference's solver (its C++ built from
its sources by oracle/ref/build_ref.py) with CellPoissonFACOps replaced by
samrai_b200.dropin's B200CellPoissonFACOps, which routes every
FACOperatorStrategy operation through the C ABI to the GPU.  Solving the
golden cases with it must reproduce the reference's own solves
(tests/golden/ref_*.npz): the same cycle count and convergence flag, the
same residual norm after every cycle to 1e-11 of the first cycle's norm,
and the
same solution on every level to 1e-12 relative and, on the interior, bit
for bit.
"""
import os

import numpy as np
import pytest

import ref_cases
from oracle.ref import refio

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DRIVER = os.path.join(os.path.dirname(refio.DRIVER), "fac_dropin_driver")
CASES = ["config1_tight", "config3_tight", "mixed_parity_2d", "robin_2d", "robin_faces_2d",
         "c_field_2d", "small_3d"]


@pytest.mark.parametrize("name", CASES)
def test_reference_solver_on_b200_operators(name, require_gpu):
    if not refio.available(DRIVER):
        pytest.skip("fac_dropin_driver not built (the reference's sources were absent at build)")
    fx = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    build, prm, bc, full = ref_cases.CASES[name]
    p = build()
    out = refio.run_reference(p, prm, bc, driver=DRIVER)
    assert int(out["iterations"][0]) == int(fx["iterations"][0])
    assert int(out["converged"][0]) == int(fx["converged"][0])
    # late norms are differences of O(1) terms: compared on the scale of
    # the first cycle's norm
    assert np.abs(out["hist"] - fx["hist"]).max() <= 1e-11 * fx["hist"][0]
    bit = []
    for ln in range(p.nlev):
        u = out[f"u{ln}"]
        m = ref_cases.interior_mask(p, ln)
        want = fx[f"u{ln}"] if full else None
        if want is not None:
            scale = max(np.abs(want[m]).max(), 1e-300)
            assert np.abs(u[m] - want[m]).max() <= 1e-12 * scale, ln
        else:
            s = fx[f"u{ln}_sample"]
            assert np.abs(u[::ref_cases.SAMPLE] - s).max() <= 1e-12 * np.abs(s).max(), ln
        bit.append(bool(np.array_equal(ref_cases.digest(u[m]), fx[f"u{ln}_sha_interior"])))
    print(f"{name} through B200CellPoissonFACOps: interior bit-identical per level: {bit}")
    assert all(bit), bit
