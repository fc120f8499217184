"""The library's own time finite element algebra (dealii-stfem_b200/csrc/
time_fe.cc, reached through stmg_time_weights and stmg_time_transfer) against
the oracle's, which tests/test_oracle_golden.py pins to the reference's
printed matrices (tests/tp_02.output, tests/transfer_02.output).

The two are separate restatements of tests/include/fe_time.h (weights
292-412, wave condensation 98-246, projection 567-623, prolongation
625-669); the library's copy is what the GPU solver uses. Host code only:
the library loads without a GPU.
"""
import numpy as np
import pytest

import oracle_py as orc
import stmg

TYPES = [(orc.DG, r) for r in range(0, 6)] + [(orc.CGP, r) for r in range(1, 6)]


def _close(a, b, tol=1e-13):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape
    scale = max(np.abs(b).max(), 1e-300)
    assert np.abs(a - b).max() <= tol * scale, np.abs(a - b).max() / scale


@pytest.mark.parametrize("ttype,r", TYPES, ids=lambda v: str(v))
@pytest.mark.parametrize("steps", [1, 2, 3, 4])
@pytest.mark.parametrize("problem", [orc.HEAT, orc.WAVE])
def test_time_weights_match_oracle(ttype, r, steps, problem):
    if problem == orc.WAVE and ttype == orc.DG and r == 0:
        pytest.skip("the wave condensation needs r >= 1 (fe_time.h:98-246)")
    tau = 0.37
    mine = stmg.time_weights(ttype, r, tau, steps, problem)
    ref = orc.time_weights(ttype, r, tau, steps, problem)
    names = ("Alpha", "Beta", "rK", "rM", "rV")
    for name, a, b in zip(names, mine, ref):
        if name == "rV" and problem == orc.HEAT:
            continue
        if np.abs(b).max() == 0.0:
            assert np.abs(a).max() == 0.0, name
        else:
            _close(a, b)


@pytest.mark.parametrize("ttype,r", [(orc.DG, r) for r in range(1, 6)] + [(orc.CGP, r) for r in range(2, 6)],
                         ids=lambda v: str(v))
@pytest.mark.parametrize("steps", [1, 2, 4])
def test_k_projection_matches_oracle(ttype, r, steps):
    _close(stmg.time_transfer(ttype, 0, r, steps), orc.time_prolongation(ttype, 0, r, steps))


@pytest.mark.parametrize("ttype,r", TYPES, ids=lambda v: str(v))
@pytest.mark.parametrize("steps", [2, 4])
def test_tau_prolongation_matches_oracle(ttype, r, steps):
    _close(stmg.time_transfer(ttype, 1, r, steps), orc.time_prolongation(ttype, 1, r, steps))


def test_time_transfer_rejects_bad_arguments():
    with pytest.raises(stmg.StmgError):
        stmg.time_transfer(orc.DG, 1, 2, 3)  # odd step count
    with pytest.raises(stmg.StmgError):
        stmg.time_transfer(orc.CGP, 0, 1, 1)  # no cGP(0)
