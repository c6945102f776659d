"""klft's legacy measurement API on the device: get_W_loop_mu_nu
(GaugeVector.hpp:237-262) and stapleField (Gauge_Util.hpp:27-97), through the
Python binding and through the C++ names of include/klft/klft.hpp."""
import os
import subprocess

import numpy as np
import pytest

from klft_b200 import GaugeField, KlftError
from oracle.oracle import Lat

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("L,nc", [([4, 6, 4, 6], 3), ([6, 4, 8], 2), ([8, 6], 1)])
@pytest.mark.parametrize("precision,rtol,atol", [("fp64", 1e-12, 1e-14), ("mixed", 0.0, 2e-6)])
def test_get_w_loop_matches_legacy_oracle(oracle, L, nc, precision, rtol, atol):
    lat = Lat(nc, L)
    U = oracle.init(lat, True, 31)
    g = GaugeField(L, nc, precision)
    g.upload(U)
    nd = len(L)
    V = int(np.prod(L))
    for mu, nu, Lmu, Lnu in [(0, nd - 1, 2, 3), (nd - 1, 0, 1, 5), (1, 0, 3, 1), (0, 1, 7, 2)]:
        ref = oracle.wilson_legacy(lat, U, mu, nu, Lmu, Lnu)
        np.testing.assert_allclose(g.wilson_loop(mu, nu, Lmu, Lnu), ref, rtol=rtol, atol=atol)
        raw = oracle.wilson_legacy(lat, U, mu, nu, Lmu, Lnu, normalize=False)
        np.testing.assert_allclose(g.wilson_loop(mu, nu, Lmu, Lnu, normalize=False), raw, rtol=rtol,
                                   atol=atol * V * nc)
    with pytest.raises(KlftError, match="EINVAL"):
        g.wilson_loop(1, 1, 2, 2)


@pytest.mark.parametrize("nc,L,precision", [(3, [4, 4, 6, 4], 0), (2, [6, 4, 4, 0], 1), (1, [8, 6, 0, 0], 0)])
def test_cxx_names(tmp_path, nc, L, precision):
    """get_W_loop_mu_nu, GaugePlaquette and stapleField from C++ agree with the
    Python binding on the same hot start."""
    exe = str(tmp_path / "legacy_api")
    lib = os.path.join(ROOT, "klft_b200")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cxx", "legacy_api.cpp"), "-o", exe, "-L", lib, "-lklft_b200",
                    "-Wl,-rpath," + lib], check=True)
    nd = sum(1 for x in L if x > 0)
    mu, nu, Lmu, Lnu = nd - 1, 0, 2, 3
    out = subprocess.run([exe, str(nc)] + [str(x) for x in L] + ["99", str(precision), str(mu), str(nu), str(Lmu),
                                                                 str(Lnu)],
                         check=True, capture_output=True, text=True).stdout.split("\n")
    g = GaugeField(L[:nd], nc, "fp64" if precision == 0 else "mixed", "hot", 99)
    assert float(out[0]) == g.plaquette()
    assert float(out[1]) == g.wilson_loop(mu, nu, Lmu, Lnu)
    assert float(out[2]) == g.wilson_loop(mu, nu, Lmu, Lnu, normalize=False)
    st = np.array(out[3].split(), dtype=np.float64)
    st = (st[0::2] + 1j * st[1::2]).reshape(g.shape())
    np.testing.assert_array_equal(st, g.staple_field())
