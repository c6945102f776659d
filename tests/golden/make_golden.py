"""Generate the golden fixtures in this directory from klft's own code.

The reference headers (compiled unchanged against the project's Kokkos-API host
shim into oracle/_ref/libklft_ref.so, `make -C oracle ref`) are run on seeded
hot-start configurations; inputs are regenerated by the oracle's hot start
(pinned separately by the Philox known-answer vectors), outputs are stored.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import Lat, Oracle, RefShim, build  # noqa: E402

CASES = [
    # (nd, nc, L, seed, beta, delta, nhits)
    (2, 1, [8, 6], 101, 2.0, 0.3, 4),
    (2, 2, [6, 4], 102, 2.2, 0.3, 4),
    (2, 3, [4, 6], 103, 5.0, 0.3, 3),
    (3, 1, [4, 4, 6], 104, 1.5, 0.3, 4),
    (3, 2, [4, 6, 4], 105, 2.0, 0.25, 4),
    (3, 3, [4, 4, 4], 106, 5.5, 0.2, 3),
    (4, 1, [4, 4, 4, 4], 107, 2.0, 0.1, 10),
    (4, 2, [4, 2, 4, 2], 108, 2.3, 0.25, 5),
    (4, 3, [4, 4, 2, 4], 109, 6.0, 0.2, 4),
    (4, 3, [4, 4, 4, 4], 32091, 6.0, 0.15, 10),
]
PAIRS = [(1, 1), (2, 2), (1, 2), (2, 1), (3, 2), (2, 3), (1, 3)]
MUNU = [(0, 1), (1, 0), (1, 2), (2, 0)]


def main():
    build()
    o, r = Oracle(), RefShim()
    r.set_threads(1)
    for nd, nc, L, seed, beta, delta, nhits in CASES:
        lat = Lat(nc, L)
        U = o.init(lat, True, seed)
        out = {"nd": nd, "nc": nc, "L": np.array(L), "seed": seed, "beta": beta, "delta": delta, "nhits": nhits}
        out["plaquette"] = r.plaquette(lat, U)
        out["pairs"] = np.array(PAIRS)
        out["W_temp"] = r.wilson_temporal(lat, U, PAIRS)
        munu = [(m, n) for m, n in MUNU if m < nd and n < nd]
        out["munu"] = np.array(munu)
        out["W_mu_nu"] = np.array([r.wilson_mu_nu(lat, U, m, n, PAIRS) for m, n in munu])
        if nd == 4:
            st = r.staple_field(lat, U)
            out["staple_sum"] = st.sum(axis=(2, 3))          # (V, Nd) complex trace-free checksum
            out["staple_first"] = st[:4]
        U2 = U.copy()
        out["acc"] = r.metropolis(lat, U2, beta, delta, nhits, 3, seed)
        out["plaquette_after"] = r.plaquette(lat, U2)
        out["links_after_sum"] = U2.sum(axis=(2, 3))
        out["links_after_first"] = U2[:8]
        name = f"ref_{nd}d_nc{nc}_" + "x".join(map(str, L)) + ".npz"
        np.savez_compressed(os.path.join(HERE, name), **out)
        print(name, out["plaquette"], out["acc"])


if __name__ == "__main__":
    main()
