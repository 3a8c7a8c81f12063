"""Global spectral gravity forward modelling on the GPU
(charm_gfm_global_density_3d / _lateral / _const): the shape-density
functions synthesised, multiplied and analysed on Gauss--Legendre grids by
the library's transforms.  Against CHarm's golden degree amplitudes
(tests/check_gfm_sgfm_all.c.in, threshold2), against the oracle's
restatement (oracle/orc.py gfm_global) coefficient by coefficient at
higher degrees, and the exported partial potentials against the sum."""
import ctypes as ct
import os

import numpy as np
import pytest

import golden_data as gd
from charm_b200.workloads import coef_rel_rms
from oracle import orc

pytestmark = pytest.mark.gpu

MOON_RREF = 1728000.0
GRAV_CONST = 6.67430e-11
MOON_MASS = 7.346e22
DENSITY_CONST = 2550.0


@pytest.fixture(scope="module")
def cb():
    import charm_b200
    return charm_b200


def moon_inputs(cb):
    z = np.load(os.path.join(gd.GOLDEN, "moon_gfm_inputs.npz"))
    out = {}
    for k in ("shape", "rho0", "rho1"):
        args = (int(z[k + "_nmax"]), float(z[k + "_mu"]), float(z[k + "_r"]),
                z[k + "_c"], z[k + "_s"])
        out[k] = (cb.Shc(*args), orc.Shc(*args))
    return out


@pytest.mark.parametrize("density", [0, 1, 2])
def test_gfm_global_golden(cb, density):
    G = gd.golden("double")
    m = moon_inputs(cb)
    shape = m["shape"][0]
    if density == 0:
        pot = cb.gfm_global_density_3d(shape, 10, MOON_RREF,
                                       [m["rho0"][0], m["rho1"][0]], [10, 10],
                                       1, GRAV_CONST, MOON_MASS, 1, 4, 10)
    elif density == 1:
        pot = cb.gfm_global_density_lateral(shape, 10, MOON_RREF,
                                            m["rho0"][0], 10, GRAV_CONST,
                                            MOON_MASS, 1, 4, 10)
    else:
        pot = cb.gfm_global_density_const(shape, 10, MOON_RREF, DENSITY_CONST,
                                          GRAV_CONST, MOON_MASS, 1, 4, 10)
    assert pot.mu == GRAV_CONST * MOON_MASS and pot.r == MOON_RREF
    da = orc.shc_da(orc.Shc(10, pot.mu, pot.r, pot.c, pot.s), 10)
    assert gd.mismatches(da, G["gfm_sgfm_g_d%d_nx10" % density],
                         gd.THRESHOLD2) == 0


def random_body(nmax, seed, R, relief):
    """A shape of radius R + relief-scaled Kaula topography and two
    density coefficient sets (mu = r = 1)."""
    rng = np.random.default_rng(seed)
    T = (nmax + 1) * (nmax + 2) // 2
    n = np.concatenate([np.arange(m, nmax + 1) for m in range(nmax + 1)])
    sig = relief / (1.0 + n) ** 2
    c = rng.standard_normal(T) * sig
    s = rng.standard_normal(T) * sig
    s[:nmax + 1] = 0.0
    c[0] = R + 1000.0
    return c, s


def test_gfm_global_vs_oracle_and_exports(cb, tmp_path):
    """Shape of degree 40, densities of degree 20 and 15, powers 1..5,
    potential to degree 150 (grids up to nmax 220): the GPU potential
    against the oracle's, and the exported partial potentials (one binary
    file per power and density order) summing to it."""
    R = 1728000.0
    c, s = random_body(40, 5, R, 4000.0)
    shape = (cb.Shc(40, 1.0, 1.0, c, s), orc.Shc(40, 1.0, 1.0, c, s))
    dens = []
    for k, nm in enumerate((20, 15)):
        dc, ds = random_body(nm, 10 + k, 0.0, 100.0)
        dc[0] = 2500.0 if k == 0 else -1e-4
        dens.append((cb.Shc(nm, 1.0, 1.0, dc, ds), orc.Shc(nm, 1.0, 1.0, dc, ds)))
    prefix = str(tmp_path / "pot")
    pot = cb.gfm_global_density_3d(shape[0], 40, R, [d[0] for d in dens],
                                   [20, 15], 1, GRAV_CONST, MOON_MASS, 1, 5,
                                   150, potential_shcs_path=prefix,
                                   shcs_file_format="bin")
    ref = orc.gfm_global(shape[1], 40, R, [d[1] for d in dens], [20, 15],
                         GRAV_CONST, MOON_MASS, 1, 5, 150)
    assert coef_rel_rms(pot.c, pot.s, ref.c, ref.s) <= 1e-12
    # the exports: files pot-p<p>-i<i>.shcs, p = 1..5, i = 0..1
    from charm_b200._lib import _libcharm as L
    L.charm_shc_read_bin.restype = ct.c_ulong
    L.charm_shc_read_bin.argtypes = [ct.c_char_p, ct.c_ulong, ct.c_void_p,
                                     ct.c_void_p]
    acc = cb.Shc(150, 1.0, 1.0)
    total_c = np.zeros_like(pot.c)
    total_s = np.zeros_like(pot.s)
    files = sorted(os.listdir(tmp_path))
    assert files == ["pot-p%d-i%d.shcs" % (p, i) for p in range(1, 6)
                     for i in range(2)]
    for name in files:
        # the contribution of power p is analysed to degree
        # min(p shape_nmax + density_nmax, potential degree), and written
        # at that degree (gfm_sgfm.c export_shcs_powers writes shcs->nmax)
        p = int(name.split("-p")[1].split("-")[0])
        d = min(40 * p + 20, 150)
        part = cb.Shc(d, 1.0, 1.0)
        err = L.charm_err_init()
        n = L.charm_shc_read_bin(str(tmp_path / name).encode(), d,
                                 ct.cast(part._Shc, ct.c_void_p),
                                 ct.cast(err, ct.c_void_p))
        assert L.charm_err_isempty(err) and n == d
        L.charm_err_free(err)
        assert part.mu == pot.mu and part.r == pot.r
        for m in range(d + 1):
            a0 = m * (d + 1) - m * (m - 1) // 2
            b0 = m * 151 - m * (m - 1) // 2
            total_c[b0:b0 + d + 1 - m] += part.c[a0:a0 + d + 1 - m]
            total_s[b0:b0 + d + 1 - m] += part.s[a0:a0 + d + 1 - m]
    assert coef_rel_rms(total_c, total_s, pot.c, pot.s) <= 1e-14
    del acc


def test_gfm_batched_synthesis_matches_per_set(cb, monkeypatch):
    """The shape and the densities of a power synthesised in one batched
    launch against one synthesis per set (the batching budget set to 0):
    the same potential to rounding."""
    R = 1728000.0
    c, s = random_body(30, 7, R, 3000.0)
    shape = cb.Shc(30, 1.0, 1.0, c, s)
    dens = []
    for k, nm in enumerate((25, 12, 8)):
        dc, ds = random_body(nm, 20 + k, 0.0, 50.0)
        dc[0] = (2600.0, -2e-4, 1e-10)[k]
        dens.append(cb.Shc(nm, 1.0, 1.0, dc, ds))
    args = (shape, 30, R, dens, [25, 12, 8], 2, GRAV_CONST, MOON_MASS, 1, 4,
            120)
    monkeypatch.delenv("CHARM_B200_GFM_BATCH_BYTES", raising=False)
    batched = cb.gfm_global_density_3d(*args)
    monkeypatch.setenv("CHARM_B200_GFM_BATCH_BYTES", "0")
    single = cb.gfm_global_density_3d(*args)
    assert coef_rel_rms(batched.c, batched.s, single.c, single.s) <= 1e-14
    ref = orc.gfm_global(orc.Shc(30, 1.0, 1.0, c, s), 30, R,
                         [orc.Shc(d.nmax, 1.0, 1.0, d.c, d.s) for d in dens],
                         [25, 12, 8], GRAV_CONST, MOON_MASS, 1, 4, 120)
    assert coef_rel_rms(batched.c, batched.s, ref.c, ref.s) <= 1e-12


def test_gfm_argument_errors(cb):
    m = moon_inputs(cb)
    with pytest.raises(cb.CHarmError, match="shape_nmax"):
        cb.gfm_global_density_const(m["shape"][0], 11, MOON_RREF, 1.0,
                                    GRAV_CONST, MOON_MASS, 1, 2, 10)
    with pytest.raises(cb.CHarmError, match="Topography power must be"):
        cb.gfm_global_density_const(m["shape"][0], 10, MOON_RREF, 1.0,
                                    GRAV_CONST, MOON_MASS, 0, 2, 10)
    with pytest.raises(cb.CHarmError, match="cannot be larger than"):
        cb.gfm_global_density_const(m["shape"][0], 10, MOON_RREF, 1.0,
                                    GRAV_CONST, MOON_MASS, 3, 2, 10)
    with pytest.raises(cb.CHarmError, match="mass"):
        cb.gfm_global_density_const(m["shape"][0], 10, MOON_RREF, 1.0,
                                    GRAV_CONST, 0.0, 1, 2, 10)
    with pytest.raises(cb.CHarmError, match="shcs_file_format"):
        cb.gfm_global_density_const(m["shape"][0], 10, MOON_RREF, 1.0,
                                    GRAV_CONST, MOON_MASS, 1, 2, 10,
                                    potential_shcs_path="/tmp/x",
                                    shcs_file_format="xyz")
