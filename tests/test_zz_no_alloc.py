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


def noalloc(g, beta, delta, nhits, proposal, eps, nsweeps, want_acc=True):
    import klft_b200
    from klft_b200._lib import check, lib
    acc = np.zeros(max(nsweeps, 1))
    out = acc.ctypes.data_as(C.POINTER(C.c_double)) if want_acc else None
    check(lib().klft_metropolis_sweeps_noalloc(g.handle, beta, delta, nhits, klft_b200.PROPOSAL[proposal], eps,
                                               nsweeps, out))
    return acc[:nsweeps]


def pool_usage():
    """Bytes used and reserved in the current device's default memory pool,
    where the library's stream-ordered scratch comes from, read through the
    CUDA runtime that libklft_b200.so itself loaded."""
    from klft_b200._lib import lib
    lib()
    rt = C.CDLL("libcudart.so.12")
    dev, pool = C.c_int(), C.c_void_p()
    assert rt.cudaGetDevice(C.byref(dev)) == 0
    assert rt.cudaDeviceGetDefaultMemPool(C.byref(pool), dev) == 0
    out = []
    for attr in (0x7, 0x5):  # cudaMemPoolAttrUsedMemCurrent, cudaMemPoolAttrReservedMemCurrent
        v = C.c_uint64()
        assert rt.cudaMemPoolGetAttribute(pool, attr, C.byref(v)) == 0
        out.append(v.value)
    return tuple(out)


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


def test_noalloc_allocates_nothing_after_a_warm_up_call():
    """The contract itself: after one warm-up call (which sets up the array's
    address and lets the driver load the kernels), calls on a fresh handle leave
    the device pool's used and reserved bytes unchanged, where the allocating
    entry point grows them by its counter scratch."""
    import klft_b200
    g = klft_b200.GaugeField([8, 8, 8, 8], 3, "mixed", "hot", 5)
    noalloc(g, 6.0, 0.0, 4, "exp", 0.3, 2)
    fresh = klft_b200.GaugeField([8, 8, 8, 8], 3, "mixed", "hot", 6)
    before = pool_usage()
    noalloc(fresh, 6.0, 0.0, 4, "exp", 0.3, 3)
    noalloc(fresh, 6.0, 0.0, 4, "exp", 0.3, 3, want_acc=False)
    assert pool_usage() == before
    fresh.metropolis(6.0, 0.0, 4, 3, proposal="exp", eps=0.3)
    assert pool_usage()[0] > before[0]
    g.close()
    fresh.close()


def test_noalloc_without_acceptance_output_and_with_zero_hits():
    """acc_out = NULL only waits for the stream; nhits = 0 leaves the links
    unchanged and reports zero acceptance, as the allocating entry point does."""
    import klft_b200
    ga = klft_b200.GaugeField([6, 4, 6, 4], 2, "fp64", "hot", 3)
    gb = klft_b200.GaugeField([6, 4, 6, 4], 2, "fp64", "hot", 3)
    for g in (ga, gb):
        g.set_stream(17, 1)
    ga.metropolis(2.3, 0.25, 5, 2)
    noalloc(gb, 2.3, 0.25, 5, "reference", 0.0, 2, want_acc=False)
    np.testing.assert_array_equal(gb.download(), ga.download())
    assert gb.counters() == ga.counters()
    before = gb.download()
    acc0 = noalloc(gb, 2.3, 0.25, 0, "reference", 0.0, 2)
    np.testing.assert_array_equal(acc0, ga.metropolis(2.3, 0.25, 0, 2))
    np.testing.assert_array_equal(acc0, 0.0)
    np.testing.assert_array_equal(gb.download(), before)
    ga.close()
    gb.close()


def test_noalloc_with_the_tuner_on_matches_the_tuned_entry_point(tmp_path):
    """With KLFT_TUNING on and nothing cached, the allocating entry point times
    block sizes and keeps one, while the no-alloc entry point starts no tuning
    and uses the default block: the chains agree because no random number
    depends on the launch shape."""
    import klft_b200
    from klft_b200._lib import lib
    try:
        lib().klft_tuner_clear()
        lib().klft_tuner_configure(1, 0)
        ga = klft_b200.GaugeField([8, 4, 8, 4], 3, "fp64", "hot", 21)
        gb = klft_b200.GaugeField([8, 4, 8, 4], 3, "fp64", "hot", 21)
        for g in (ga, gb):
            g.set_stream(8, 0)
        for _ in range(2):
            acc_a = ga.metropolis(6.0, 0.0, 5, 2, proposal="exp", eps=0.3)
            acc_b = noalloc(gb, 6.0, 0.0, 5, "exp", 0.3, 2)
            np.testing.assert_array_equal(acc_b, acc_a)
            np.testing.assert_array_equal(gb.download(), ga.download())
        ga.close()
        gb.close()
    finally:
        lib().klft_tuner_configure(0, 0)
        lib().klft_tuner_clear()


def test_noalloc_from_two_threads_on_one_device():
    """Two handles on one device swept from two threads at once share the
    static counters; the per-device lock keeps each call's counters its own, so
    both chains equal serial runs of the allocating entry point."""
    import threading

    import klft_b200
    specs = [(3, [8, 8, 4, 4], "exp", 6.0, 0.0, 0.3, 31), (2, [8, 8, 8, 8], "reference", 2.3, 0.25, 0.0, 32)]
    fields, refs, results = [], [], [None, None]
    for nc, L, prop, beta, delta, eps, seed in specs:
        gt = klft_b200.GaugeField(L, nc, "mixed", "hot", seed)
        gr = klft_b200.GaugeField(L, nc, "mixed", "hot", seed)
        for g in (gt, gr):
            g.set_stream(seed, 0)
        fields.append(gt)
        refs.append(gr)

    def work(k):
        nc, L, prop, beta, delta, eps, seed = specs[k]
        results[k] = [noalloc(fields[k], beta, delta, 4, prop, eps, 3) for _ in range(5)]

    threads = [threading.Thread(target=work, args=(k,)) for k in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for k, (nc, L, prop, beta, delta, eps, seed) in enumerate(specs):
        for r in results[k]:
            np.testing.assert_array_equal(r, refs[k].metropolis(beta, delta, 4, 3, proposal=prop, eps=eps))
        np.testing.assert_array_equal(fields[k].download(), refs[k].download())
        fields[k].close()
        refs[k].close()
