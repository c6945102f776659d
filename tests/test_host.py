"""The C++ host layer: the `metropolis` and `hmc` binaries, YAML input, output
files (GaugeObservable.hpp formats), environment variables and the tuner cache.

CPU tests cover the CLI and parsing (which happen before any device call); GPU
tests run the binaries end to end and compare with the Python path."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "klft_b200", "bin")

README_INPUT = """\
# input.yaml
MetropolisParams:    # parameters for the Metropolis algorithm
  Ndims: 4    # number of dimensions [2,3,4]
  Nd: 4       # number of link dimensions (this must be strictly same as Ndims)
  Nc: 1       # number of colors (defines SU(Nc)) [1,2,3]
  L0: 8       # lattice extent in 0 direction
  L1: 8
  L2: 8
  L3: 8
  nHits: 10       # number of hits per sweep
  nSweep: {nsweep}      # number of sweeps
  seed: 32091     # random seed
  beta: 2.0       # inverse coupling constant
  delta: 0.1      # step size for the Metropolis algorithm

GaugeObservableParams:
  measurement_interval: 10               # interval for measurements
  measure_plaquette: true                # measure the plaquette
  measure_wilson_loop_temporal: true    # measure the temporal Wilson loop
  measure_wilson_loop_mu_nu: true       # measure the spatial Wilson loop
  W_temp_L_T_pairs:      # pairs of (L, T) values for the temporal Wilson loop
    - [2, 2]
    - [3, 4]             # keep a non-decreasing order (as much as possible)
    - [4, 3]             # for maximum efficiency
    - [4, 4]
  W_mu_nu_pairs:      # pairs of (mu, nu) values for the planar Wilson loop
    - [0, 1]
    - [1, 2]
    - [3, 2]
  W_Lmu_Lnu_pairs:      # pairs of (Lmu, Lnu) values for the lengths of the
    - [2, 2]            # planar Wilson loop in the mu and nu directions
    - [3, 3]            # again, keep a non-decreasing order (as much as possible)
    - [4, 3]
  plaquette_filename: "plaquette.out"  # filename to output the plaquette
  W_temp_filename: "W_temp.out"        # filename to output the temporal Wilson loop
  W_mu_nu_filename: "W_mu_nu.out"      # filename to output the planar Wilson loop
  write_to_file: true                  # write the measurements to file
"""


def run(args, cwd, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run(args, cwd=cwd, env=e, capture_output=True, text=True, timeout=600)


def test_metropolis_help_and_missing_block(tmp_path):
    r = run([os.path.join(BIN, "metropolis"), "-h"], tmp_path)
    assert r.returncode == 0 and "--filename" in r.stdout and "Metropolis for SU(N) gauge fields" in r.stdout
    (tmp_path / "bad.yaml").write_text("GaugeObservableParams:\n  measurement_interval: 1\n")
    r = run([os.path.join(BIN, "metropolis"), "-f", "bad.yaml"], tmp_path)
    assert r.returncode != 0
    assert "Error: MetropolisParams not found in input file" in r.stdout


def test_metropolis_parses_reference_example(tmp_path):
    (tmp_path / "input.yaml").write_text(README_INPUT.format(nsweep=1000))
    r = run([os.path.join(BIN, "metropolis")], tmp_path, {"KLFT_VERBOSITY": "1"})
    # the parameter dump of Metropolis_Params.hpp:80-97 comes before any device call
    for line in ["Ndims: 4", "L0: 8", "nHits: 10", "nSweep: 1000", "seed: 32091", "Nd: 4", "Nc: 1",
                 "beta: 2.0000", "delta: 0.1000"]:
        assert line in r.stdout


def test_hmc_help():
    r = run([os.path.join(BIN, "hmc"), "--help"], ROOT)
    assert r.returncode == 0 and "--gauge-group" in r.stdout and "--outfilename" in r.stdout


@pytest.mark.gpu
def test_metropolis_binary_end_to_end(tmp_path):
    import klft_b200
    (tmp_path / "input.yaml").write_text(README_INPUT.format(nsweep=30))
    r = run([os.path.join(BIN, "metropolis"), "-f", "input.yaml"], tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    plaq = (tmp_path / "plaquette.out").read_text().splitlines()
    assert plaq[0] == "# step, plaquette" and len(plaq) == 3  # steps 10, 20
    wt = (tmp_path / "W_temp.out").read_text().splitlines()
    assert wt[0] == "# step, L, T, W_temp" and len(wt) == 1 + 2 * 4
    assert wt[1].startswith("10, 2, 2, ")
    wm = (tmp_path / "W_mu_nu.out").read_text().splitlines()
    assert wm[0] == "# step, mu, nu, Lmu, Lnu, W_mu_nu" and len(wm) == 1 + 2 * 9
    # the same chain through the Python mirror (cold start, seed 32091, chain 0)
    g = klft_b200.GaugeField([8, 8, 8, 8], 1, "fp64", "cold", 32091)
    g.set_stream(32091, 0)
    ps = []
    for step in range(30):
        g.metropolis(2.0, 0.1, 10, 1)
        if step in (10, 20):
            ps.append(g.plaquette())
    got = [float(l.split(",")[1]) for l in plaq[1:]]
    np.testing.assert_allclose(got, ps, rtol=1e-5)  # 6 significant digits in the file
    # appending: a second run adds another block
    r = run([os.path.join(BIN, "metropolis"), "-f", "input.yaml"], tmp_path)
    assert len((tmp_path / "plaquette.out").read_text().splitlines()) == 6


@pytest.mark.gpu
def test_tuning_changes_nothing_but_writes_cache(tmp_path):
    (tmp_path / "input.yaml").write_text(README_INPUT.format(nsweep=12))
    r0 = run([os.path.join(BIN, "metropolis"), "-f", "input.yaml"], tmp_path)
    assert r0.returncode == 0
    base = (tmp_path / "plaquette.out").read_text()
    os.remove(tmp_path / "plaquette.out")
    cache = tmp_path / "tune.cache"
    r1 = run([os.path.join(BIN, "metropolis"), "-f", "input.yaml"], tmp_path,
             {"KLFT_TUNING": "1", "KLFT_CACHE_FILE": str(cache)})
    assert r1.returncode == 0, r1.stdout + r1.stderr
    assert (tmp_path / "plaquette.out").read_text() == base
    lines = cache.read_text().splitlines()
    assert any(l.startswith("4 sweep_Metropolis_GaugeField_nc1_fp64_ref_rank_4_start_0_0_0_0_end_4_4_4_4_ ")
               for l in lines), lines
    # a second run reads the cache back
    r2 = run([os.path.join(BIN, "metropolis"), "-f", "input.yaml"], tmp_path,
             {"KLFT_TUNING": "1", "KLFT_CACHE_FILE": str(cache), "KLFT_VERBOSITY": "1"})
    assert "Reading cache file" in r2.stdout


@pytest.mark.gpu
def test_hmc_binary(tmp_path):
    r = run([os.path.join(BIN, "hmc"), "--gauge-group", "SU2", "--ndim", "4", "--LX", "4", "--LY", "4", "--LZ", "4",
             "--LT", "4", "--n-traj", "3", "--n-steps", "10", "--beta", "2.3", "--outfilename", "hmc.csv"], tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    rows = (tmp_path / "hmc.csv").read_text().splitlines()
    assert rows[0] == "traj, accept, plaquette, time, acceptance rate" and len(rows) == 4
    assert "Traj: 2 Accept:" in r.stdout
    r = run([os.path.join(BIN, "hmc"), "--gauge-group", "SU3", "--ndim", "3", "--LX", "4", "--LY", "4", "--LT", "4",
             "--n-traj", "2", "--n-steps", "8", "--beta", "5.0", "--integrator", "omelyan", "--precision", "mixed"],
            tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
