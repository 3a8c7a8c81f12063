"""The synthesis autotuner: the first call of a problem shape times every
candidate tile (latitude pairs per lane) and keeps the fastest; later calls
of that shape reuse it, and the result does not depend on the choice (each
latitude pair's sums are formed the same way whatever the tile).  The
parity tests at nmax >= 256 (test_gpu_parity.py) run with tuned tiles."""
import ctypes as ct

import numpy as np
import pytest

from charm_b200.workloads import GM, R_EARTH, kaula

pytestmark = pytest.mark.gpu


def report(L):
    L.charm_b200_autotune_report.restype = ct.c_size_t
    L.charm_b200_autotune_report.argtypes = [ct.c_char_p, ct.c_size_t]
    buf = ct.create_string_buffer(16384)
    L.charm_b200_autotune_report(buf, 16384)
    return buf.value.decode().splitlines()


def test_tuned_once_per_shape_and_same_result():
    import charm_b200 as cb
    from charm_b200._lib import _libcharm as L
    N = 301
    p = cb.PointGridGL(N, R_EARTH)
    c, s = kaula(N, 990)
    shc = cb.Shc(N, GM, R_EARTH, c, s)
    f1 = cb.shs_point(p, shc, N)
    lines = [x for x in report(L) if ("nmax=%d " % N) in x and "kgrad=0" in x]
    assert len(lines) == 1, report(L)
    assert " K=" in lines[0] and "ms:" in lines[0]
    # candidates 1, 2 and 4 were measured
    for k in (1, 2, 4):
        assert (" %d:" % k) in lines[0]
    f2 = cb.shs_point(p, shc, N)
    assert np.array_equal(f1, f2)
    assert len([x for x in report(L) if ("nmax=%d " % N) in x
                and "kgrad=0" in x]) == 1


def test_result_independent_of_the_tile(tmp_path):
    """The tuned synthesis equals, bit for bit, the synthesis with the
    built-in tile (autotuner off, in a separate process)."""
    import os
    import subprocess
    import sys
    import charm_b200 as cb
    N = 420
    p = cb.PointGridDH2(N, R_EARTH + 5e3)
    c, s = kaula(N, 991)
    f_tuned = cb.shs_point(p, cb.Shc(N, GM, R_EARTH, c, s), N)
    out = tmp_path / "f.npy"
    code = (
        "import numpy as np, charm_b200 as cb\n"
        "from charm_b200.workloads import GM, R_EARTH, kaula\n"
        "N = %d\n"
        "p = cb.PointGridDH2(N, R_EARTH + 5e3)\n"
        "c, s = kaula(N, 991)\n"
        "np.save(%r, cb.shs_point(p, cb.Shc(N, GM, R_EARTH, c, s), N))\n"
        % (N, str(out)))
    env = dict(os.environ, CHARM_B200_AUTOTUNE="0")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    subprocess.run([sys.executable, "-c", code], check=True, env=env,
                   cwd=root, timeout=600)
    assert np.array_equal(f_tuned, np.load(out))
