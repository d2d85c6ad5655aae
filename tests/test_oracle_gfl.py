"""Known-answer checks of the GFL restatement (oracle/gfl_oracle.cpp), the
checker of the device Taylor-Galerkin step: still water stays still (to
rounding), a lake
at rest over a bump stays at rest, a layer on a slope under Manning friction
reaches its normal-flow velocity, and the set-up's slopes are exact on a
plane."""
import numpy as np
import pytest

import workloads

G = 9.8


def mesh(nx, ny, d):
    intmat, coord = workloads.p1_mesh(nx, ny, d)
    return intmat, coord


def test_still_water_stays_still(oracle_mod):
    intmat, coord = mesh(21, 11, 10.0)
    u = np.zeros((coord.shape[0], 3))
    u[:, 0] = 2.0
    z = np.zeros(coord.shape[0])
    out, t, _, _ = oracle_mod.gfl_run(coord, intmat, z, {1: G, 2: 1000.0, 10: 0.01}, u, 20, 0.5)
    # the boundary integral and the element integrals of the pressure cancel
    # to single-precision rounding at the corners
    assert np.abs(out[:, 0] - 2.0).max() < 1e-6 and np.abs(out[:, 1:]).max() < 1e-5
    assert t == pytest.approx(10.0)


def test_lake_at_rest_over_a_bump(oracle_mod):
    """ntype 2: the free surface Z + h = swl over a Gaussian bump stays flat
    and still (the pressure of h^2 - HH^2 and the slope source balance)."""
    intmat, coord = mesh(31, 31, 10.0)
    r2 = ((coord - 150.0) ** 2).sum(1)
    z = 2.0 * np.exp(-r2 / 2500.0)
    swl = 5.0
    u = np.zeros((coord.shape[0], 3))
    u[:, 0] = swl - z
    out, _, _, _ = oracle_mod.gfl_run(coord, intmat, z, {1: G, 2: 1000.0, 10: 0.01}, u, 50, 0.2, ntype=2, swl=swl)
    assert np.abs(out[:, 1:]).max() < 1e-4
    assert np.abs(out[:, 0] - u[:, 0]).max() < 1e-5


def test_manning_normal_flow_on_a_slope(oracle_mod):
    """A 1 m layer on a 1% slope under Manning n = 0.03 (ntype 2, nfric 1)
    accelerates to the normal-flow velocity h^(2/3) S^(1/2) / n = 3.33 m/s
    in the middle of a long channel, before the waves from its closed ends
    arrive."""
    nx, ny, d = 201, 3, 10.0
    intmat, coord = mesh(nx, ny, d)
    S, n, h = 0.01, 0.03, 1.0
    z = 100.0 - S * coord[:, 0]
    u = np.zeros((coord.shape[0], 3))
    u[:, 0] = h
    out, _, _, _ = oracle_mod.gfl_run(coord, intmat, z, {1: G, 2: 1000.0, 3: n, 5: 1, 10: 0.01}, u, 240, 0.5, ntype=2,
                                      swl=200.0)
    mid = np.abs(coord[:, 0] - 1000.0) < 1.0
    v = out[mid, 1] / out[mid, 0]
    vn = h ** (2.0 / 3.0) * np.sqrt(S) / n
    assert np.allclose(v, vn, rtol=0.02), (v, vn)
    assert np.abs(out[mid, 2]).max() < 5e-3 * vn  # the diagonals of the triangulation skew it slightly


def test_setup_slopes_are_exact_on_a_plane(oracle_mod):
    """Get_Topol's lumped-mass projection of the element slopes returns the
    plane's slopes at every node and zero curvature."""
    intmat, coord = mesh(12, 9, 5.0)
    z = 3.0 + 0.2 * coord[:, 0] - 0.1 * coord[:, 1]
    u = np.zeros((coord.shape[0], 3))
    _, _, topol, topel = oracle_mod.gfl_run(coord, intmat, z, {1: G, 2: 1000.0, 10: 0.01}, u, 0, 0.1)
    assert np.allclose(topol[:, 1], 0.2, atol=1e-5) and np.allclose(topol[:, 2], -0.1, atol=1e-5)
    assert np.allclose(topol[:, 3], 1.04, atol=1e-5) and np.allclose(topol[:, 5], 1.01, atol=1e-5)
    assert np.abs(topol[:, 6:9]).max() < 1e-4
    assert np.allclose(topel[:, 1], 0.2, atol=1e-5)
