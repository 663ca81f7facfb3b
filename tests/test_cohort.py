"""Cohort driver (anechoic_b200.cohort): the reference protocol's phases on the engines. CPU: the pilot grid, the
selection rule, phase ordering and refusal to overwrite. GPU: a scaled-down protocol V -> K -> M -> P -> H end to
end on the N = 2000 +-1 instance (validation passes: host rescoring and byte-identical spins across engines)."""
import json
import os

import pytest

import anechoic_b200 as A
from anechoic_b200 import cohort as CO
from anechoic_b200 import instances as I


def test_pilot_grid_is_the_reference_grid():
    cells = list(CO.pilot_cells())
    assert len(cells) == 5 * 2 * 2 * 6 and cells[0] == (0, "--tecT 1.5 --ramp --q 6 --t0 12 --steps 80")
    assert cells[-1] == (119, "--lambda 1.05 --ramp --q 8 --t0 15 --steps 280")


def test_selection_uses_wilson_lower_bound():
    """A cell with a lower point estimate but few batches loses to one whose lower confidence bound is better."""
    def cell(name, kb, nb, k, ntr, t):
        from anechoic_b200 import analyze as AN
        return dict(prefix=name, B=ntr // nb, batches=nb, P_batch=kb / nb, P_batch_wilson95=list(AN.wilson(kb, nb)),
                    p=k / ntr, p_wilson95=list(AN.wilson(k, ntr)), t_batch_ms=t,
                    tts_primary_ms=AN.tts99(kb / nb, t), tts_secondary_ms=AN.tts99_secondary(k / ntr, ntr // nb, t))
    few = cell("few", 2, 2, 30, 480, 1.0)      # P_batch = 1 on 2 batches
    many = cell("many", 31, 32, 400, 7680, 1.0)
    best = CO.select_pilot([few, many])
    assert best["primary"]["prefix"] == "many"


def test_phase_order_and_overwrite(tmp_path):
    g = str(tmp_path / "g.bin")
    I.write_snowgpu1(I.complete_pm1(64, 1), g)
    ctx = CO.Ctx(g, str(tmp_path / "res"), 100, 1, 1.0, [1])
    with pytest.raises(RuntimeError, match="validation"):
        CO.phase_K(ctx)
    os.makedirs(tmp_path / "res" / "V")
    (tmp_path / "res" / "V" / "x.summary.json").write_text("{}")
    with pytest.raises(FileExistsError):
        ctx.run("V/x", 1, 1, 0, CO.VSCHED["plain"])
    assert CO.main(["Z"]) == 1 and CO.main(["V", "--bogus", "1"]) == 1


@pytest.mark.gpu
def test_scaled_protocol_end_to_end(cuda, tmp_path):
    g = str(tmp_path / "k.bin")
    I.write_snowgpu1(I.complete_pm1(2000, 20261004), g)
    res = str(tmp_path / "res")
    ctx = CO.Ctx(g, res, 32300, 20261004, 1 / 64, [1, 16], log=lambda *_: None)
    CO.phase_V(ctx)
    with open(os.path.join(res, "V", "validation_summary.json")) as f:
        v = json.load(f)
    assert v["verdict"] == "PASS" and set(v["engines"]) == {"plain", "cluster", "tensor"}
    CO.phase_K(ctx)
    with open(os.path.join(res, "K", "selected_engines.json")) as f:
        sel = json.load(f)
    assert set(sel) == {"1", "16"}
    CO.phase_M(ctx)
    assert len([p for p in os.listdir(os.path.join(res, "M")) if p.endswith(".summary.json")]) == 7 * 2
    grid = [(0, "--tecT 1.75 --ramp --q 8 --t0 15 --steps 280"), (1, "--lambda 1.05 --ramp --q 8 --t0 12 --steps 400")]
    CO.phase_P(ctx, grid=grid)
    for w in ("primary", "secondary"):
        with open(os.path.join(res, "P", f"selected_{w}.json")) as f:
            assert json.load(f)["prefix"].startswith("p00")
    CO.phase_H(ctx)
    assert os.path.exists(os.path.join(res, "H", "primary_b1.summary.json"))
