"""The oracle against the reference's own FAC solver.

tests/golden/ref_<case>.npz hold full solves by SAMRAI's CellPoissonFACSolver
itself -- its FACPreconditioner loop, CellPoissonFACOps, RefineSchedule and
CoarsenSchedule data motion, CoarseFineBoundary, CartesianRobinBcHelper,
norms and weights, with its Fortran kernels translated to C -- built from the
reference's sources by oracle/ref/build_ref.py and run by
tests/golden/make_ref_fixtures.py.  The oracle (a C restatement of the same
path) must reproduce every one bit for bit: the cycle count, the residual
norm after every cycle, and the solution on every level (interior cells;
with the ghost cells too where the boundary is the solver's own Dirichlet
path, whose ghost values the reference restores after the solve).
"""
import os

import numpy as np
import pytest

import ref_cases
from oracle.oracle import Oracle, U

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fixture(name):
    return np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))


def test_every_case_has_a_fixture():
    for name in ref_cases.CASES:
        assert os.path.exists(os.path.join(GOLDEN, f"ref_{name}.npz")), name


@pytest.mark.parametrize("name", list(ref_cases.CASES))
def test_oracle_matches_reference_solver(name):
    fx = fixture(name)
    build, prm, bc, _ = ref_cases.CASES[name]
    p = build()
    if isinstance(bc, str):  # "faces": coefficients varying along the boundary
        o = Oracle(p, params=prm, bc_faces=ref_cases.all_face_coefs(p))
    else:
        o = Oracle(p, params=prm, bc=bc)
    ok, its, res, hist = o.solve()
    assert its == int(fx["iterations"][0])
    assert ok == bool(fx["converged"][0])
    assert res == fx["residual"][0]
    assert np.array_equal(hist[1:its + 1], fx["hist"])
    for ln in range(p.nlev):
        u = o.get(U, ln)
        m = ref_cases.interior_mask(p, ln)
        assert np.array_equal(ref_cases.digest(u[m]), fx[f"u{ln}_sha_interior"]), ln
        if bc is None:
            assert np.array_equal(ref_cases.digest(u), fx[f"u{ln}_sha_all"]), ln
