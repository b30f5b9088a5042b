"""Seeded workload generators (CPU): the near-equilibrium cells of the
batched workload are chemical equilibria of the mechanism (every reaction's
net rate vanishes up to rounding) with the elements of their pool state."""
import numpy as np

from openhurricane_b200 import synth, workloads
from oracle import port


def test_equilibrium_tp_is_a_fixed_point_of_the_kinetics(small):
    t = small["tables"]
    base = synth.dirichlet_cells(t.nsp, 64, seed=31)
    T = np.random.default_rng(5).uniform(1500.0, 2800.0, 64)
    Yeq = workloads.equilibrium_tp(t, T, base.p, base.Y)
    A = t.elem_matrix / t.W[None, :]
    assert np.abs(A @ Yeq - A @ base.Y).max() < 1e-14
    assert np.all(Yeq >= 0.0) and np.abs(Yeq.sum(axis=0) - 1.0).max() < 1e-14
    rho = synth.mixture_density(t.W, synth.Cells(T, base.p, Yeq))
    c = rho[None, :] * Yeq / t.W[:, None]
    f, _ = port.rhs_jac(port.MechDesc(t), c, T)
    # net production is rounding left over from forward and reverse rates of
    # up to ~1e8 per second: it moves no species by more than 1e-4 of itself
    # over a 1e-5 s flow step
    assert (np.abs(f[:, :t.nsp]).T / np.maximum(c, 1e-30)).max() * 1e-5 < 1e-4
    assert np.abs(f[:, -1]).max() < 1.0          # dT/dt in K/s


def test_batched_workload_shape_and_mix(small):
    wl = workloads.make_batched(2048, seed=7, pool=256)
    assert wl.T.shape == (2048,) and wl.Y.shape == (9, 2048)
    assert np.abs(wl.Y.sum(axis=0) - 1.0).max() < 1e-12
    ign = (wl.T >= 1100.0) & (wl.T <= 1300.0)
    assert 0.15 < ign.mean() < 0.35      # 20 % ignition cells (+ near-equilibrium ones in range)
    assert wl.dt == 1e-5
