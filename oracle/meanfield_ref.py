"""FP64 oracle of the mean-field relaxation (test infrastructure only: the checker of anechoic_b200.meanfield, never
shipped or measured).

The same recurrence as the sm_100a kernels, in torch float64 on any device, differentiated by torch autograd:

    P_t = J m_t + b + q_t m_t - gamma_t m_{t-1},  gamma_t = u_t sum_{i<n} (1 - m_t,i^2) + w_t,  m_{t+1} = tanh(beta_t P_t)

It is the tanh form of the reference's effective process (research/dmft_sca_20261004/dmft_torch.py:38-57; the
reference solves it stochastically and does not differentiate it) with the golden model's correction conventions
(sca_ref.hpp:118-131, tables.hpp:14-40: no correction at t = 0, counted gain lambda_t / (2 T_{t-1}), temperature-
scaled kappa T_{t-1}). The reference has no differentiable path to pin this restatement against; it is pinned by
torch autograd against central finite differences (tests/test_meanfield_oracle.py).
"""
from __future__ import annotations

import torch


def relax64(J: torch.Tensor, b: torch.Tensor, beta, q, u, w, m0: torch.Tensor, mprev: torch.Tensor) -> torch.Tensor:
    """J [n, n], b [n], per-step beta, q, u, w [S], m0 / mprev [R, n] (all float64) -> m_S [R, n]."""
    m, mp = m0, mprev
    for t in range(beta.shape[0]):
        gamma = u[t] * (1.0 - m * m).sum(dim=1) + w[t]
        P = m @ J.T + b + q[t] * m - gamma[:, None] * mp
        m, mp = torch.tanh(beta[t] * P), m
    return m


def soft_cut64(J: torch.Tensor, sumw: float, m: torch.Tensor) -> torch.Tensor:
    return (sumw + 0.5 * ((m @ J) * m).sum(dim=1)) / 2.0
