"""klft_metropolis_sweeps_noalloc: the sweep entry point for callers that cannot
let the library allocate (device memory already given to their own pool, or a
latency-critical loop that must not pay cudaMalloc's device-wide
synchronisation).  It must give exactly what klft_metropolis_sweeps gives.

This file is collected last on purpose: it exercises the per-device static
counter array, which is set up on the first call in the process, and it must
pass both alone in a fresh process and after every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_SWEEPS = 1024  # KLFT_NOALLOC_MAX_SWEEPS in include/klft_b200.h

CASES = [
    # (nc, L, precision, proposal, beta, delta, eps, nhits, nsweeps, links atol)
    (3, [8, 8, 8, 8], "fp64", "exp", 6.0, 0.0, 0.3, 10, 3, 1e-11),
    (3, [8, 8, 8, 8], "mixed", "exp", 6.0, 0.0, 0.3, 10, 3, 2e-6),
    (2, [6, 4, 6, 4], "fp64", "reference", 2.3, 0.25, 0.0, 5, 4, 1e-11),
    (1, [8, 6], "mixed", "reference", 2.0, 0.3, 0.0, 4, 5, 2e-6),
]


def noalloc(g, beta, delta, nhits, proposal, eps, nsweeps):
    import klft_b200
    from klft_b200._lib import check, lib
    acc = np.zeros(max(nsweeps, 1))
    check(lib().klft_metropolis_sweeps_noalloc(g.handle, beta, delta, nhits, klft_b200.PROPOSAL[proposal], eps,
                                               nsweeps, acc.ctypes.data_as(C.POINTER(C.c_double))))
    return acc[:nsweeps]


@pytest.mark.parametrize("case", CASES, ids=[f"nc{c[0]}-{c[2]}-{c[3]}" for c in CASES])
def test_noalloc_matches_allocating_entry_point(case):
    import klft_b200
    nc, L, precision, proposal, beta, delta, eps, nhits, nsweeps, atol = case
    ga = klft_b200.GaugeField(L, nc, precision, "hot", 99)
    gb = klft_b200.GaugeField(L, nc, precision, "hot", 99)
    ga.set_stream(4711, 2)
    gb.set_stream(4711, 2)
    for _ in range(2):  # two calls in a row on the same handles
        acc_a = ga.metropolis(beta, delta, nhits, nsweeps, proposal=proposal, eps=eps)
        acc_b = noalloc(gb, beta, delta, nhits, proposal, eps, nsweeps)
        np.testing.assert_array_equal(acc_b, acc_a)
        np.testing.assert_allclose(gb.download(), ga.download(), rtol=0, atol=atol)
        assert gb.counters() == ga.counters()
    ga.close()
    gb.close()


def test_noalloc_rejects_more_sweeps_than_the_static_array_holds():
    import klft_b200
    g = klft_b200.GaugeField([4, 4, 4, 4], 2, "fp64", "hot", 1)
    before = g.download()
    with pytest.raises(klft_b200.KlftError) as e:
        noalloc(g, 2.0, 0.2, 2, "reference", 0.0, MAX_SWEEPS + 1)
    assert "KLFT_EINVAL" in str(e.value) and str(MAX_SWEEPS) in str(e.value)
    np.testing.assert_array_equal(g.download(), before)
    assert g.counters() == (0, 0)
    g.close()
