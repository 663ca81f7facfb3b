"""GPU: the command-line drop-in writes the reference's run files (trials.jsonl, spins.bin, trace.bin, batches.jsonl,
summary.json); replaying every trial of those files with the golden-model restatement gives the same spins, n_lin
trace, flips and cut (the check_ref replay), and the estimators read them."""
import json
import os

import numpy as np
import pytest

from anechoic_b200 import analyze, cli
from anechoic_b200 import instances as I

pytestmark = pytest.mark.gpu


def _trials(prefix):
    with open(prefix + ".trials.jsonl") as f:
        return [json.loads(line) for line in f]


def test_graph_run_replays_against_oracle(cuda, oracle, tmp_path):
    inst = I.complete_pm1(2000, 20261004)
    g = str(tmp_path / "k.bin")
    I.write_snowgpu1(inst, g)
    prefix = str(tmp_path / "run")
    rc = cli.main(["--graph", g, "--output", prefix, "--chains", "48", "--batches", "2", "--steps", "150",
                   "--lambda", "1.05", "--ramp", "--trace", "1", "--seed", "11", "--offset", "1000",
                   "--target", "32000", "--cs", "8"])
    assert rc == 0
    tr = _trials(prefix)
    assert len(tr) == 96 and [t["trial_id"] for t in tr] == list(range(1000, 1096))
    W = 32
    spins = np.fromfile(prefix + ".spins.bin", np.uint64).reshape(96, W)
    trace = np.fromfile(prefix + ".trace.bin", np.int32).reshape(96, 150)
    ref = oracle.run_batch(2000, oracle.tables(S=150, lam=1.05, ramp=True), 11, 1000, 96, dense=inst.dense)
    assert np.array_equal(spins, ref["spins"]) and np.array_equal(trace, ref["nlin"])
    for c, t in enumerate(tr):
        assert t["flips"] == int(ref["flips"][c]) and t["cut"] == t["device_cut"] == inst.cut(spins[c])
        assert t["success"] == (t["cut"] >= 32000)
    e = analyze.estimate(prefix)
    s = json.load(open(prefix + ".summary.json"))
    assert s["cut_mismatches"] == 0 and s["geometry"] == {"cs": "8"}
    assert e["successes"] == s["successes"] == sum(t["success"] for t in tr)


def test_bias_run_with_field_check(cuda, oracle, tmp_path):
    inst = I.random_kbit(600, 4, 5, pzero=0.3, bmax=9)
    jp, bp = str(tmp_path / "j.bin"), str(tmp_path / "b.bin")
    I.write_jint8(inst, jp)
    I.write_bias(inst.bias, bp)
    prefix = str(tmp_path / "bias")
    rc = cli.main(["--jint8", jp, "--bias", bp, "--kbits", "4", "--output", prefix, "--chains", "12",
                   "--batches", "1", "--steps", "80", "--t0", "40", "--t1", "1", "--q", "2", "--tecT", "2",
                   "--ramp", "--target-energy", "-100000", "--check-fields", "1"])
    assert rc == 0
    tr = _trials(prefix)
    assert all("cut" not in t and t["field_mismatches"] == 0 for t in tr)
    spins = np.fromfile(prefix + ".spins.bin", np.uint64).reshape(12, -1)
    ref = oracle.run_batch(600, oracle.tables(S=80, t0=40.0, t1=1.0, q=2.0, kappa=2.0, ramp=True), 20261004, 0, 12,
                           dense=inst.dense, bias=inst.bias)
    for c, t in enumerate(tr):
        assert np.array_equal(spins[c], ref["spins"][c])
        assert t["energy"] == t["device_energy"] == inst.energy(spins[c])
        assert t["sum_sh"] == int(ref["sum_sh"][c]) and t["sum_bs"] == int(ref["sum_bs"][c])


def test_cli_errors_exit_1(cuda, tmp_path, capsys):
    assert cli.main(["--output", str(tmp_path / "x")]) == 1
    assert "FAIL:" in capsys.readouterr().err
