"""Instance generators (anechoic_b200.gen) against the reference's own gen_ising: the fixtures in tests/golden/gen
were written by it (tests/golden/make_gen_golden.py). Couplings, biases, edge lists and metadata text must match
byte for byte. Also: the encodings' ground states, found by brute force, are the problems' optima; and on the GPU
the engines anneal these bias workloads bit-exactly with the golden model, and reach the optimum."""
import os
import subprocess

import numpy as np
import pytest

import anechoic_b200 as A
from anechoic_b200 import gen as G
from anechoic_b200 import instances as I
from tests.golden.make_gen_golden import CASES

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "gen")
REF_GEN = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "gen_ising")


def _same_files(a, b):
    for ext in (".jint8", ".bias", ".json", ".edges"):
        if os.path.exists(a + ext):
            with open(a + ext, "rb") as f, open(b + ext, "rb") as g:
                assert f.read() == g.read(), f"{os.path.basename(a)}{ext} differs"


@pytest.mark.parametrize("name,args", CASES, ids=[c[0] for c in CASES])
def test_matches_reference_fixtures(tmp_path, name, args):
    out = str(tmp_path / name)
    assert G.main(args + ["--out", out]) == 0
    _same_files(os.path.join(FIX, name), out)


LIVE = [
    ["gp", "--n", "2000", "--deg", "3", "--k", "700", "--A", "1", "--B", "2", "--seed", "9"],
    ["gp", "--n", "300", "--deg", "5", "--k", "37", "--A", "4", "--B", "3", "--seed", "21"],
    ["tsp", "--n", "46", "--wmax", "3", "--A", "4", "--B", "1", "--seed", "5"],
    ["random", "--n", "777", "--kbits", "8", "--pzero", "0.9", "--bmax", "32767", "--pbig", "0.5", "--bsmall", "1",
     "--seed", "3"],
]


@pytest.mark.skipif(not os.path.exists(REF_GEN), reason="oracle/_ref/gen_ising not built (needs the reference tree)")
@pytest.mark.parametrize("args", LIVE, ids=["gp2000", "gp300", "tsp46", "rnd777"])
def test_matches_reference_live(tmp_path, args):
    """Larger cases, against the reference generator run here."""
    r, o = str(tmp_path / "ref"), str(tmp_path / "ours")
    subprocess.run([REF_GEN, *args, "--out", r], check=True, stdout=subprocess.DEVNULL)
    assert G.main(args + ["--out", o]) == 0
    _same_files(r, o)


def test_ground_states_are_optima():
    """gp: every Ising ground state is a K-subset with the minimum cut; tsp: every ground state is an optimal tour,
    and H = sigma f + C holds on random states (checked inside the generators)."""
    inst, meta, edges = G.graph_partitioning(18, 6, deg=3, A=3, B=1, seed=5, brute=True)
    assert meta["brute"]["consistent"] and meta["brute"]["ising_emin"] == meta["brute"]["emin_expected"]
    t, tm = G.tsp(5, wmax=7, A=25, B=1, seed=8, brute=True)
    assert tm["brute"]["consistent"]
    emin, count, gs = G.brute_force(t.dense, t.bias)
    W = np.array(tm["W"])
    assert emin == tm["brute"]["ising_emin"] and all(G.tour_length(g, W) == tm["brute"]["direct_min_length"]
                                                     for g in gs)


def test_bad_arguments_fail(tmp_path, capsys):
    out = str(tmp_path / "x")
    assert G.main(["gp", "--n", "15", "--deg", "3", "--k", "4", "--out", out]) == 1        # n * deg odd
    assert G.main(["tsp", "--n", "47", "--out", out]) == 1                                 # 46^2 spins > 2048
    assert G.main(["random", "--n", "10", "--kbits", "9", "--out", out]) == 1
    assert G.main(["gp", "--n", "20", "--k", "4", "--bogus", "1"]) == 1
    assert "FAIL" in capsys.readouterr().err


@pytest.mark.gpu
def test_engines_anneal_generated_problems(cuda, oracle):
    """GP (couplings of at most 7, dense planes, bias) and TSP (couplings up to 49, CSR rows, bias) anneal bit-exactly
    with the golden model, and the best anneal reaches the brute-force ground-state energy."""
    cases = [(I.read_jint8(os.path.join(FIX, "gp20_brute.jint8")), "gp20_brute", dict(t0=30.0, t1=0.5, q=30.0)),
             (I.read_jint8(os.path.join(FIX, "tsp5_brute.jint8")), "tsp5_brute", dict(t0=400.0, t1=2.0, q=40.0))]
    for inst, name, sched in cases:
        inst.bias = I.read_bias(os.path.join(FIX, name + ".bias"), inst.n)
        emin, _, _ = G.brute_force(inst.dense, inst.bias)
        # the antiferromagnetic encodings need a large self-coupling q against period-2 oscillation of the
        # synchronous update; dense planes hold |J| <= 7, larger couplings (the TSP penalties) run on the CSR path
        dev = A.DeviceInstance(inst, sparse=inst.stats()["maxabs"] > 7)
        sc = dict(S=400, lam=0.5, ramp=True, **sched)
        r = A.run(dev, A.Tables.from_schedule(A.Schedule(**sc)), 17, 0, 256, trace=True)
        ref = oracle.run_batch(inst.n, oracle.tables(**sc), 17, 0, 256, dense=inst.dense, bias=inst.bias)
        assert np.array_equal(r.spins, ref["spins"]) and np.array_equal(r.trace, ref["nlin"]), name
        e = np.array([inst.energy(r.spins[c]) for c in range(256)])
        assert np.array_equal(e, r.energies()), name
        assert e.min() == emin, (name, int(e.min()), emin)
