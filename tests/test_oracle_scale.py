"""The C restatement at benchmark scale against the recorded reference
outputs (tests/golden/wrinkled128.*): the 128^3 y-stretched wrinkled flame,
whose hierarchy relaxes y-lines and semicoarsens x and z over 7 levels.

In the reference's lexicographic line order the restatement's PCG solve
(unit-scaled production MG plan, src/solver_krylov.cpp:1299-1555) takes the
reference's iteration count and reproduces the recorded sample of its
solution bit for bit; the hierarchy has the reference's level shapes.
"""
import numpy as np
import pytest

import golden_cases
import scale_cases


def test_scale_inputs_match_the_fixture():
    sys_ = scale_cases.system("wrinkled128")
    assert golden_cases.digest(sys_) == scale_cases.entry("wrinkled128")["digest"]


@pytest.mark.usefixtures("oracle_built")
def test_restatement_pcg_at_128_matches_reference():
    import c_oracle
    import ref_oracle
    name = "wrinkled128"
    entry = scale_cases.entry(name)
    ref = scale_cases.arrays(name)
    sys_ = scale_cases.system(name)
    o = c_oracle.OracleSession(sys_, ref_oracle.MgPolicy.production(), line_order=0)
    assert [list(l) for l in o.levels()] == entry["levels"]
    x, info = o.solve(sys_.rhs, rtol=1e-13, maxit=400)
    assert info["iterations"] == entry["pcg_step0_1e13"]["iterations"]
    assert np.array_equal(x.reshape(-1)[ref["cells"]], ref["pcg_step0_1e13"])
