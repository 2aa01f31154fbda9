"""The reference's Lomb-Scargle expression (rust/src/ls.rs:253-275,
periodfind/cuda/ls.cu:107-134) written with torch operations, so that FP64
autograd gives reference derivatives with respect to the angular frequency
and the magnitudes.  Test infrastructure only."""

import math

import torch


def ls_power_tau(t: torch.Tensor, y: torch.Tensor, omega: torch.Tensor) -> torch.Tensor:
    """P(omega) for one curve; t, y 1-D, omega a scalar tensor (any dtype)."""
    th = omega * t
    s, c = torch.sin(th), torch.cos(th)
    mc = (y * c).sum()
    ms = (y * s).sum()
    cc = (c * c).sum()
    cs = (c * s).sum()
    ss = t.shape[0] - cc
    tau = 0.5 * torch.atan2(2.0 * cs, cc - ss)
    st, ct = torch.sin(tau), torch.cos(tau)
    a = ct * mc + st * ms
    b = ct * ms - st * mc
    dl = ct * ct * cc + 2.0 * ct * st * cs + st * st * ss
    dr = ct * ct * ss - 2.0 * ct * st * cs + st * st * cc
    return 0.5 * (a * a / dl + b * b / dr)


def two_pi_over(periods):
    return [2.0 * math.pi / float(p) for p in periods]
