"""Batches: many chains of uneven groups and extents (and PTBC replicas)
advanced in one captured graph per cycle must give exactly what each chain gives
alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make(L, nc, precision, seed, chain):
    import klft_b200
    g = klft_b200.GaugeField(L, nc, precision, "hot", seed)
    g.set_stream(seed, chain)
    return g


CHAINS = [
    # (L, nc, precision, beta, delta, nhits, proposal, eps)
    ([4, 4, 4, 4], 3, "mixed", 6.0, 0.0, 4, "exp", 0.3),
    ([6, 4, 4, 8], 2, "mixed", 2.3, 0.3, 3, "reference", 0.0),
    ([8, 8, 4, 4], 2, "mixed", 2.5, 0.3, 3, "reference", 0.0),
    ([4, 4, 6], 1, "fp64", 1.5, 0.4, 5, "reference", 0.0),
    ([4, 6, 4, 4], 3, "fp64", 5.5, 0.0, 3, "exp", 0.25),
    ([8, 6], 3, "mixed", 4.0, 0.2, 2, "reference", 0.0),
]


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_equals_chains_alone(use_graph):
    import klft_b200
    b = klft_b200.Batch()
    batch_fields, solo_fields = [], []
    for k, (L, nc, prec, beta, delta, nh, prop, eps) in enumerate(CHAINS):
        gb = make(L, nc, prec, 100 + k, k)
        gs = make(L, nc, prec, 100 + k, k)
        b.add(gb, beta, delta, nh, prop, eps)
        batch_fields.append(gb)
        solo_fields.append(gs)
    ncyc = 3
    acc, plaq, _, ms = b.run(ncyc, True, use_graph)
    assert ms > 0
    for k, (L, nc, prec, beta, delta, nh, prop, eps) in enumerate(CHAINS):
        for c in range(ncyc):
            a = solo_fields[k].metropolis(beta, delta, nh, 1, prop, eps)[0]
            assert acc[c, k] == a
            assert plaq[c, k] == solo_fields[k].plaquette()  # the single-lattice partials and order
        np.testing.assert_array_equal(batch_fields[k].download(), solo_fields[k].download())
        assert batch_fields[k].counters() == solo_fields[k].counters()
    # a second run continues every chain
    acc2, _, _, _ = b.run(2, False, use_graph)
    for k, (L, nc, prec, beta, delta, nh, prop, eps) in enumerate(CHAINS):
        np.testing.assert_array_equal(acc2[:, k], solo_fields[k].metropolis(beta, delta, nh, 2, prop, eps))
    b.close()


def test_batch_ptbc_replicas_match_host_swaps():
    import klft_b200
    nrep = 4
    c = np.linspace(1.0, 0.0, nrep)
    L = [4, 4, 4, 4]
    beta = 5.8
    b = klft_b200.Batch()
    reps_b, reps_s = [], []
    ids = []
    for r in range(nrep):
        gb = make(L, 3, "mixed", 300 + r, r)
        gs = make(L, 3, "mixed", 300 + r, r)
        for g in (gb, gs):
            g.set_defect(2, (1, 0, 2), c[r])
        ids.append(b.add(gb, beta, 0.0, 3, "exp", 0.3))
        reps_b.append(gb)
        reps_s.append(gs)
    extra = make([6, 4, 4, 4], 2, "mixed", 999, 9)  # an ordinary chain in the same batch
    b.add(extra, 2.3, 0.3, 2)
    b.set_ptbc(ids, c, beta, 4242)
    ncyc = 4
    acc, plaq, labels, _ = b.run(ncyc, True, True)
    lab = np.arange(nrep)
    for cyc in range(ncyc):
        for r in range(nrep):
            a = reps_s[r].metropolis(beta, 0.0, 3, 1, "exp", 0.3)[0]
            assert acc[cyc, r] == a
        lab, _ = klft_b200.ptbc_swap(reps_s, c, lab, beta, 4242, cyc)
        np.testing.assert_array_equal(labels[cyc], lab)
    for r in range(nrep):
        np.testing.assert_array_equal(reps_b[r].download(), reps_s[r].download())
    b.close()


def test_batch_tuning_changes_nothing(tmp_path):
    """KLFT_TUNING's batch block-size search times candidates on the chains'
    own links (backed up and restored) and caches a key per batch composition;
    the chains end exactly where an untuned batch takes them."""
    import klft_b200
    from klft_b200._lib import lib
    cache = str(tmp_path / "tune.txt")
    runs = {}
    try:
        for tuned in (True, False):
            lib().klft_tuner_clear()
            lib().klft_tuner_configure(int(tuned), 0)
            b = klft_b200.Batch()
            fields = []
            for k, (L, nc, prec, beta, delta, nh, prop, eps) in enumerate(CHAINS):
                g = make(L, nc, prec, 700 + k, k)
                b.add(g, beta, delta, nh, prop, eps)
                fields.append(g)
            acc, plaq, _, _ = b.run(3, True, True)
            acc2, _, _, _ = b.run(2, False, False)
            if tuned:
                assert lib().klft_tuner_write_cache(cache.encode()) == 0
            runs[tuned] = (acc, plaq, acc2, [g.download() for g in fields], [g.counters() for g in fields])
            b.close()
    finally:
        lib().klft_tuner_configure(0, 0)
        lib().klft_tuner_clear()
    assert "sweep_Metropolis_batch_" in open(cache).read()
    a, u = runs[True], runs[False]
    for x, y in zip(a[:3], u[:3]):
        np.testing.assert_array_equal(x, y)
    for x, y in zip(a[3], u[3]):
        np.testing.assert_array_equal(x, y)
    assert a[4] == u[4]
