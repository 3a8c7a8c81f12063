"""Pins the oracle's restatement of CHarm's global spectral gravity forward
modelling (oracle/orc.py gfm_global, after src/gfm/gfm_sgfm.c) against the
golden degree amplitudes of tests/check_gfm_sgfm_all.c.in: the lunar shape
and densities of degree 10 (tests/parameters.h:298-356), topography powers
1..4, potential to degree 10, tolerance threshold2."""
import os

import numpy as np
import pytest

import golden_data as gd
from oracle import orc

MOON_RREF = 1728000.0
GRAV_CONST = 6.67430e-11
MOON_MASS = 7.346e22
DENSITY_CONST = 2550.0


def moon():
    z = np.load(os.path.join(gd.GOLDEN, "moon_gfm_inputs.npz"))
    shc = {k: orc.Shc(int(z[k + "_nmax"]), float(z[k + "_mu"]),
                      float(z[k + "_r"]), z[k + "_c"], z[k + "_s"])
           for k in ("shape", "rho0", "rho1")}
    return shc


@pytest.mark.parametrize("density", [0, 1, 2])
def test_oracle_gfm_global_golden(density):
    G = gd.golden("double")
    m = moon()
    if density == 0:
        pot = orc.gfm_global(m["shape"], 10, MOON_RREF, [m["rho0"], m["rho1"]],
                             [10, 10], GRAV_CONST, MOON_MASS, 1, 4, 10)
    elif density == 1:
        pot = orc.gfm_global(m["shape"], 10, MOON_RREF, [m["rho0"]], [10],
                             GRAV_CONST, MOON_MASS, 1, 4, 10)
    else:
        pot = orc.gfm_global(m["shape"], 10, MOON_RREF, None, None,
                             GRAV_CONST, MOON_MASS, 1, 4, 10,
                             const_density=DENSITY_CONST)
    da = orc.shc_da(pot, 10)
    ref = G["gfm_sgfm_g_d%d_nx10" % density]
    assert gd.mismatches(da, ref, gd.THRESHOLD2) == 0
