"""The constant-null-space fixture (tests/golden/null_space.*, recorded from
the compiled reference's NativeCartesianMgPlan with MgNullSpace::constant by
tests/golden/make_golden.py --null-space): the generator still builds the
recorded pure-Neumann system, its rhs is consistent (zero sum), and, where
the reference is built, the reference reproduces the recorded MG
applications bit for bit."""
import os
import sys

import numpy as np
import pytest

import golden_cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_fixture_system_is_pure_neumann_and_consistent():
    s = golden_cases.null_space_system()
    assert golden_cases.digest(s) == golden_cases.null_space_index()["digest"]
    assert all(b == 1 for b in s.boundary)
    assert abs(float(np.sum(s.rhs))) <= 1e-12 * float(np.abs(s.rhs).sum())
    # the operator annihilates constants on the fluid cells
    fluid = s.active.reshape(-1) != 0 if s.active is not None else np.ones(s.cells, bool)
    d = s.diagonal.reshape(-1)
    assert np.all(d[fluid] > 0.0)


def test_reference_reproduces_fixture():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_oracle
    if not ref_oracle.available():
        pytest.skip("compiled reference (oracle/_ref) not built")
    s = golden_cases.null_space_system()
    fx = dict(np.load(os.path.join(golden_cases.GOLDEN, "null_space.npz")))
    v = golden_cases.probe(s)
    for tag, pol in ((t, e["policy"]) for t, e in golden_cases.null_space_index().items()
                     if isinstance(e, dict) and "policy" in e):
        ref = ref_oracle.RefSession(s, ref_oracle.MgPolicy(**pol), algorithm="pcg",
                                    null_space="constant")
        assert np.array_equal(ref.apply_mg(v), fx[f"{tag}_mg"])
        ref.close()
