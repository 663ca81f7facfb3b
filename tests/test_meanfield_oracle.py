"""CPU checks of the mean-field relaxation's FP64 oracle and schedule mapping (no GPU): autograd of the oracle
against central finite differences in the five schedule parameters, and the exact-engine tables of a schedule
against the reference's own table builder."""
import math

import numpy as np
import pytest
import torch

from anechoic_b200 import instances as I
from anechoic_b200.meanfield import SoftSchedule, initial_magnetisations
from oracle.meanfield_ref import relax64, soft_cut64


def _setup(n=40, S=21, R=3, mode="counted", seed=3):
    inst = I.random_kbit(n, 2, seed, pzero=0.3, bmax=2)
    J = torch.as_tensor(inst.dense, dtype=torch.float64)
    b = torch.as_tensor(inst.bias, dtype=torch.float64)
    m0 = initial_magnetisations(n, R, seed).double()
    mprev = torch.ones_like(m0)
    sch = SoftSchedule(S=S, mode=mode)
    sumw = inst.stats()["sumw"]

    def loss(theta):
        beta, q, u, w = sch.vectors(theta)
        return soft_cut64(J, sumw, relax64(J, b, beta, q, u, w, m0, mprev)).mean()
    return loss


@pytest.mark.parametrize("mode", ["counted", "tecT"])
def test_oracle_gradient_vs_central_differences(mode):
    loss = _setup(mode=mode)
    theta = torch.tensor([6.0, math.log(5.0), 0.8, 0.4, 1.05 if mode == "counted" else 2.0], dtype=torch.float64,
                         requires_grad=True)
    loss(theta).backward()
    g = theta.grad.clone()
    for k in range(5):
        h = 1e-6 * max(1.0, abs(float(theta[k])))
        tp, tm = theta.detach().clone(), theta.detach().clone()
        tp[k] += h
        tm[k] -= h
        fd = (loss(tp) - loss(tm)).item() / (2 * h)
        assert abs(fd - g[k].item()) <= 1e-6 * max(1.0, abs(fd)), (mode, k, fd, g[k].item())


def test_tables_match_reference_builder(oracle):
    """theta = (t0, ln(t0/t1), q, 0, lambda or kappa) gives the reference's own integer tables (tables.hpp:14-40)."""
    for mode, kw in (("counted", dict(lam=1.05)), ("tecT", dict(kappa=2.0))):
        S = 1000
        sch = SoftSchedule(S=S, mode=mode, ramp=True)
        gain = kw.get("lam", kw.get("kappa"))
        tb = sch.table_arrays([30.0, math.log(30.0 / 5.0), 4.0, 0.0, gain])
        ref = oracle.tables(S=S, t0=30.0, t1=5.0, q=4.0, ramp=True, **kw)
        for k in ("fourT", "q", "kcorr", "kconst"):
            assert np.array_equal(np.asarray(tb[k]), np.asarray(ref[k])), (mode, k)
