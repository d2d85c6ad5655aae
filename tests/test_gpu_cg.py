"""The device CG (solvegc2 semantics) against the oracle's restatement and a
dense solve, through the C ABI."""
import numpy as np
import pytest

import gfsph
import workloads

pytestmark = pytest.mark.gpu


def mass_system(nx, ny, d=5.0, seed=4):
    intmat, coords = workloads.p1_mesh(nx, ny, d)
    g = workloads.p1_mass_matrices(intmat, coords)
    b = np.random.default_rng(seed).normal(size=coords.shape[0])
    return intmat, coords, g, b


def test_cg_matches_oracle_and_dense_solve(gfsph_lib, oracle_mod):
    intmat, coords, g, b = mass_system(31, 23)
    n = coords.shape[0]
    K = np.zeros((n, n))
    for e in range(intmat.shape[0]):
        idx = intmat[e] - 1
        K[np.ix_(idx, idx)] += g[e]
    b32 = b.astype(np.float32)
    cg = gfsph.CG(intmat, g.astype(np.float32))
    x, r, fix, it = cg.solve(b32, tol=1e-20)
    xo, ro, fo, ito = oracle_mod.solvegc2(2, intmat, g.astype(np.float32).astype(np.float64), b32.astype(np.float64),
                                         tol=1e-20)
    assert abs(it - ito) <= 1
    assert np.allclose(x, xo, rtol=1e-6, atol=1e-6)
    dense = np.linalg.solve(K, b32.astype(np.float64))
    assert np.allclose(x, dense, rtol=1e-5, atol=1e-6)
    # second solve on the same handle, with prescribed boundary dofs
    iffix = np.zeros(n, np.int32)
    bnd = (coords[:, 0] == 0) | (coords[:, 1] == coords[:, 1].max())
    iffix[bnd] = 1
    fixed = np.where(bnd, -1.5, 0.0).astype(np.float32)
    x2, _, fix2, it2 = cg.solve(b32, iffix=iffix, fixed=fixed, tol=1e-20)
    xo2, _, _, ito2 = oracle_mod.solvegc2(2, intmat, g.astype(np.float32).astype(np.float64), b32.astype(np.float64),
                                         iffix=iffix, fixed=fixed.astype(np.float64), tol=1e-20)
    assert np.all(x2[bnd] == -1.5)
    assert np.allclose(x2, xo2, rtol=1e-6, atol=1e-6) and abs(it2 - ito2) <= 1
    assert np.array_equal(fix2, iffix)
    cg.close()


def test_cg_large_mesh_converges(gfsph_lib):
    """500x500 DEM window: 500k triangles, 251k dofs, tolerance 1e-10 on the
    squared residual ratio; the residual of the returned solution is checked
    with an independent sparse product."""
    intmat, coords, g, b = mass_system(501, 501, d=2.0)
    cg = gfsph.CG(intmat, g.astype(np.float32))
    x, r, fix, it = cg.solve(b.astype(np.float32), tol=1e-10)
    n = coords.shape[0]
    ax = np.zeros(n)
    xe = x.astype(np.float64)[intmat - 1]                   # (nelem, 3)
    contrib = np.einsum("eab,eb->ea", g, xe)
    np.add.at(ax, (intmat - 1).reshape(-1), contrib.reshape(-1))
    res = b.astype(np.float32).astype(np.float64) - ax
    rel = np.dot(res, res) / np.dot(b, b)
    assert rel < 1e-9
    assert 5 < it < 200
    cg.close()


def test_solvegc2_one_shot_matches_handle(gfsph_lib):
    import ctypes as C
    intmat, coords, g, b = mass_system(17, 19)
    n = coords.shape[0]
    cg = gfsph.CG(intmat, g.astype(np.float32))
    x, r, _, it = cg.solve(b.astype(np.float32), tol=1e-16)
    cg.close()
    gf = np.ascontiguousarray(np.transpose(g.astype(np.float32), (0, 2, 1)))
    im = np.ascontiguousarray(intmat, np.int32)
    fix = np.zeros(n, np.int32)
    fixed = np.zeros(n, np.float32)
    rr = b.astype(np.float32).copy()
    xx = np.zeros(n, np.float32)
    its = C.c_int()
    L = gfsph.lib()
    st = L.gfsph_solvegc2(n, im.shape[0], 3, 1, gfsph._ip(im), gfsph._ip(fix), gfsph._fp(fixed), gfsph._fp(gf),
                          gfsph._fp(rr), gfsph._fp(xx), 1e-16, C.byref(its))
    assert st == 0 and its.value == it
    assert np.array_equal(xx, x) and np.array_equal(rr, r)


def test_persistent_cg_residual_determinism_and_launches(gfsph_lib, oracle_mod):
    """Every iteration runs inside one cooperative launch (four kernels per
    solve: set-up, preconditioner and residual, the iterations, results); the
    returned residual is solvegc2's (the one before the last update), and two
    solves are bit-identical."""
    intmat, coords, g, b = mass_system(41, 37)
    b32 = b.astype(np.float32)
    cg = gfsph.CG(intmat, g.astype(np.float32))
    l0 = cg.launch_count()
    x, r, fix, it = cg.solve(b32, tol=1e-8)
    assert cg.launch_count() - l0 == 4
    assert cg.device_ms() > 0.0
    xo, ro, fo, ito = oracle_mod.solvegc2(2, intmat, g.astype(np.float32).astype(np.float64),
                                         b32.astype(np.float64), tol=1e-8)
    assert it == ito
    assert np.allclose(x, xo, rtol=1e-6, atol=1e-6)
    assert np.allclose(r, ro, rtol=1e-5, atol=1e-6 * np.abs(ro).max())
    x2, r2, _, it2 = cg.solve(b32, tol=1e-8)
    assert it2 == it and np.array_equal(x2, x) and np.array_equal(r2, r)
    cg.close()


def test_cg_zero_system_is_not_iterated(gfsph_lib):
    """rnormX below the tolerance (:93-103): the solution is 0, no iteration."""
    intmat, coords, g, b = mass_system(9, 7)
    cg = gfsph.CG(intmat, g.astype(np.float32))
    x, r, fix, it = cg.solve(np.zeros(coords.shape[0], np.float32), tol=1e-10)
    assert it == 0 and np.all(x == 0.0) and np.all(r == 0.0)
    cg.close()
