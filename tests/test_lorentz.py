"""The Lorentz-as-critical-point mapping of gsvit_copy_b200.plan.lorentz_as_cp,
checked numerically: one ADE polarisation pole with the planner's
coefficients (calculate_ade_bp, plan.c:2745-2752, in ade_material) is driven
by a broadband E pulse through GSvit's recursion

    P^{n+1} = bp0 P^{n-1} + bp1 P^n + bp2 E^{n-1} + bp3 E^n + bp4 E^{n+1}

(yee.c:914-1108), and the susceptibility recovered as DFT(P) / (eps0 DFT(E))
is compared with the Lorentz model eps_inf + (eps_s - eps_inf) w0^2 /
(w0^2 - w^2 - 2 i delta w) it stands for (time dependence e^{-i w t}).  The
batched workload's Lorentz substrate (eps_s 5, eps_inf 2, w0 4e15 rad/s,
delta 1e14 1/s) at the time step of 5 nm cells."""
import math

import numpy as np
import pytest

from gsvit_copy_b200 import plan

EPS0 = 8.854187817620389850e-12
EPS_S, EPS_INF, W0, DELTA = 5.0, 2.0, 4e15, 1e14


def lorentz_chi(w):
    return (EPS_S - EPS_INF) * W0 * W0 / (W0 * W0 - w * w - 2j * DELTA * w)


def driven_pole(dt, nsteps):
    pole = plan.lorentz_as_cp(EPS_S, EPS_INF, W0, DELTA)
    m = plan.ade_material(EPS_INF, 0.0, 0.0, 0.0, [pole, (0.0, 0.0, 0.0, 0.0)], dt)
    bp = [m.ade_bp0[0], m.ade_bp1[0], m.ade_bp2[0], m.ade_bp3[0], m.ade_bp4[0]]
    t = np.arange(nsteps) * dt
    t0, tw = 400 * dt, 60 * dt     # a short pulse: flat spectrum well past 2 w0
    e = np.exp(-((t - t0) / tw) ** 2)
    p = np.zeros(nsteps)
    for n in range(1, nsteps - 1):
        p[n + 1] = bp[0] * p[n - 1] + bp[1] * p[n] + bp[2] * e[n - 1] + bp[3] * e[n] + bp[4] * e[n + 1]
    return t, e, p


@pytest.fixture(scope="module")
def response():
    dt = plan.plan_dt(5e-9, 5e-9, 5e-9, 0.5)
    nsteps = int(30 / DELTA / dt)      # the pole's ringing decays by e^-30
    return dt, driven_pole(dt, nsteps)


@pytest.mark.parametrize("frac", [0.0, 0.25, 0.5, 0.75, 0.9, 1.1, 1.3, 1.6, 2.0])
def test_lorentz_pole_recovers_the_lorentz_susceptibility(response, frac):
    dt, (t, e, p) = response
    w = frac * W0
    ker = np.exp(1j * w * t)
    chi = (p @ ker) / (EPS0 * (e @ ker))
    want = lorentz_chi(w)
    # second-order time discretisation: relative error grows like (w dt)^2
    # (w dt <= 0.04 here; largest error 4.2e-4, next to the resonance)
    assert abs(chi - want) / abs(want) < 1e-3, (frac, chi, want)


def test_lorentz_pole_at_resonance(response):
    dt, (t, e, p) = response
    ker = np.exp(1j * W0 * t)
    chi = (p @ ker) / (EPS0 * (e @ ker))
    want = lorentz_chi(W0)   # = i (eps_s - eps_inf) w0 / (2 delta), purely imaginary
    assert abs(chi - want) / abs(want) < 5e-3, (chi, want)   # 1.2e-3
    assert abs(chi.real) < 0.05 * abs(chi.imag)


def test_static_limit_and_mapping_parameters():
    a, phi, big_omega, gamma = plan.lorentz_as_cp(EPS_S, EPS_INF, W0, DELTA)
    assert phi == 0.0 and gamma == DELTA
    assert math.isclose(big_omega * big_omega + gamma * gamma, W0 * W0, rel_tol=1e-15)
    # chi_cp(0) = 2 A Omega^2 / (Omega^2 + Gamma^2) = eps_s - eps_inf
    assert math.isclose(2 * a * big_omega ** 2 / (big_omega ** 2 + gamma ** 2), EPS_S - EPS_INF, rel_tol=1e-14)
