"""Lattice transfers of the mixed form: only the stored FP32 reals cross PCIe
and the host rounds (upload) or completes (download) each link.  Rows stored on
the device come back as their FP32 values exactly; the rebuilt rows are the
unit-determinant completion of those values in FP64.  Sizes span one and
several 32 MB staging chunks."""
import numpy as np
import pytest

from klft_b200 import GaugeField
from oracle.oracle import Lat

pytestmark = pytest.mark.gpu


def completion(U):
    """Row 2 of SU(3) from rows 0 and 1 (conj of the cross product), in FP64."""
    r0, r1 = U[..., 0, :], U[..., 1, :]
    return np.conj(np.cross(r0, r1))


@pytest.mark.parametrize("nc,L", [(3, [4, 6, 4, 2]), (3, [24, 24, 24, 24]), (2, [8, 8, 8, 8]),
                                  (2, [32, 32, 24, 24]), (1, [6, 4, 8]), (1, [128, 128, 96])])
def test_mixed_transfers_round_and_complete(oracle, nc, L):
    lat = Lat(nc, L)
    U = oracle.init(lat, True, 7 + nc)
    g = GaugeField(L, nc, "mixed")
    g.upload(U)
    D = g.download()
    stored = U.astype(np.complex64).astype(np.complex128)
    if nc == 3:
        np.testing.assert_array_equal(D[..., :2, :], stored[..., :2, :])
        np.testing.assert_allclose(D[..., 2, :], completion(stored), rtol=0, atol=1e-15)
        np.testing.assert_allclose(D, U, rtol=0, atol=3e-7)
    elif nc == 2:
        np.testing.assert_array_equal(D[..., 0, :], stored[..., 0, :])
        np.testing.assert_array_equal(D[..., 1, 0], -np.conj(stored[..., 0, 1]))
        np.testing.assert_array_equal(D[..., 1, 1], np.conj(stored[..., 0, 0]))
    else:
        np.testing.assert_array_equal(D, stored)
    # a second round trip changes nothing
    g.upload(D)
    np.testing.assert_array_equal(g.download(), D)
    g.close()


def test_mixed_download_of_open_boundary_and_device_work(oracle):
    """Zeroed boundary links come back zero; a configuration updated on the
    device downloads to the same values as the FP64 form evaluates it with."""
    L = [4, 4, 4, 6]
    g = GaugeField(L, 3, "mixed", "hot", 3)
    g.set_stream(3, 0)
    g.set_open_boundary(3)
    g.metropolis(6.0, 0.0, 4, 2, "exp", 0.3)
    D = g.download()
    last = D.reshape(L[::-1] + [4, 3, 3])[L[3] - 1, :, :, :, 3]
    assert np.all(last == 0)
    h = GaugeField(L, 3, "fp64")
    h.upload(D)
    h.set_open_boundary(3)
    assert abs(h.plaquette() - g.plaquette()) < 1e-7
    g.close()
    h.close()
