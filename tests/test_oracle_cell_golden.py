"""Pins the oracle's restatement of CHarm's cell (block-mean) synthesis and
analysis (oracle/orc.c cell_lumped / cell_contract, oracle/orc.py shs_cell /
sha_cell) against the golden vectors of tests/check_shs_cell.c and
tests/check_sha_cell.c, with the tolerances CHarm applies there."""
import numpy as np
import pytest

import golden_data as gd
from oracle import orc


def oracle_cell(case):
    ctype = orc.CELL_GRID if case.ctype == gd.CELL_GRID else orc.CELL_SCATTERED
    return orc.Cell(ctype, *case.cell)


def coeffs():
    nmax, mu, r, c, s = gd.test_coefficients()
    return orc.Shc(nmax, mu, r, c, s)


@pytest.mark.parametrize("subset", ["fft0", "fft1", "sctr"])
def test_oracle_shs_cell_golden(subset):
    G = gd.golden("double")
    shc = coeffs()
    cases = [c for c in gd.shs_cell_cases() if subset in c.name]
    assert cases
    bad = 0
    for case in cases:
        f = orc.shs_cell(oracle_cell(case), shc, case.nmax)
        bad += gd.mismatches(f, G[case.golden_names[0]], case.eps)
    assert bad == 0


def test_oracle_sha_cell_golden():
    G = gd.golden("double")
    shc = coeffs()
    cases = gd.sha_cell_cases()
    assert len(cases) == 28
    bad = 0
    for case in cases:
        cl = oracle_cell(case)
        f = orc.shs_cell(cl, shc, case.nmax)
        out = orc.sha_cell(cl, f, case.nmax, shc.mu, shc.r)
        bad += gd.mismatches(out.c, G[case.golden_names[0]], case.eps)
        bad += gd.mismatches(out.s, G[case.golden_names[1]], case.eps)
    assert bad == 0


def test_oracle_cell_zero_cells():
    """Zero cells are a valid input (check_shs_cell.c:40-48,
    check_sha_cell.c:163-176)."""
    shc = coeffs()
    cl = orc.Cell(orc.CELL_SCATTERED, [], [], [], [], [])
    assert orc.shs_cell(cl, shc, 4).size == 0
    cl = orc.Cell(orc.CELL_GRID, [], [], [], [], [])
    out = orc.sha_cell(cl, np.zeros(0), shc.nmax, shc.mu, shc.r)
    assert not np.any(out.c) and not np.any(out.s)
