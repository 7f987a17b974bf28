"""GPU tests of the matrix-free KKT adjoint (cuOptSolutionAdjointBatch: LSQR on the GPU, one
thread block per active-set system), the torch layer over it, and the vertex crossover (the same
LSQR solves).

References: the constructed optimum of generators.vertex_lp (unique and non-degenerate, with a
known basis), the exact derivatives of that vertex computed from a sparse LU of its basis (SciPy,
independent of the library), and central finite differences of the library's own solution map
(perturbed LPs re-solved in one batched call with crossover, so every solution is an exact
vertex).

Tolerances: crossover reproduces the constructed vertex to 1e-9 (relative to the vector's scale);
adjoint gradients match the basis derivatives to 1e-7 relative to their largest magnitude (1e-5
when they are taken at the PDLP solution without crossover), and the
finite differences (h = 1e-6; round-off of the vertices bounds their error near 1e-6) to 1e-5
relative plus 1e-5 absolute.
"""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.linalg import splu

from cuopt_b200 import generators as gen
from cuopt_b200 import linear_programming as lpm
from tests.helpers import datamodel_from_lp, settings

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _settings(tol=1e-8, crossover=True):
    s = settings(tol=tol)
    s.set_parameter(lpm.CUOPT_CROSSOVER, bool(crossover))
    return s


def _basis_derivatives(lp, w, v):
    """dL/dc, dL/db, dL/dA of L = w.x* + v.y* at the constructed vertex."""
    A = sp.csr_matrix((lp.val, lp.col_idx, lp.row_off), shape=(lp.m, lp.n))
    B = lp.basic
    lu = splu(A[:, B].tocsc())
    lam = lu.solve(w[B], trans="T")
    mu = np.zeros(lp.n)
    mu[B] = lu.solve(v)
    rows = np.repeat(np.arange(lp.m), np.diff(lp.row_off))
    dval = -lam[rows] * lp.x_star[lp.col_idx] - mu[lp.col_idx] * lp.y_star[rows]
    return mu, lam, dval


def _tensors(lp, dev="cuda"):
    f = lambda a: torch.tensor(np.asarray(a, dtype=np.float64), device=dev)
    i = lambda a: torch.tensor(np.asarray(a, dtype=np.int32), device=dev)
    return dict(c=f(lp.c).requires_grad_(), con_lo=f(lp.con_lo).requires_grad_(),
                con_up=f(lp.con_up).requires_grad_(), values=f(lp.val).requires_grad_(),
                row_offsets=i(lp.row_off), column_indices=i(lp.col_idx), var_lo=f(lp.var_lo),
                var_up=f(lp.var_up))


def _close(got, want, rtol):
    scale = max(1.0, float(np.abs(want).max()))
    assert np.abs(got - want).max() <= rtol * scale, (np.abs(got - want).max(), scale)


@pytest.fixture(scope="module")
def vlp():
    return gen.vertex_lp(400, 900, 8, seed=21)


def test_crossover_recovers_constructed_vertex(vlp):
    sol = lpm.Solve(datamodel_from_lp(vlp), _settings(tol=1e-6))
    assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert sol.stats["crossover"] == 1
    _close(sol.get_primal_solution(), vlp.x_star, 1e-9)
    _close(sol.get_dual_solution(), vlp.y_star, 1e-9)
    _close(sol.get_reduced_cost(), vlp.s_star, 1e-9)
    assert abs(sol.get_primal_objective() - vlp.optimal_objective) <= 1e-9 * abs(vlp.optimal_objective)


@pytest.mark.parametrize("crossover", [True, False])
def test_adjoint_matches_basis_derivatives(vlp, crossover):
    from cuopt_b200.torch_layer import lp_solve
    rng = np.random.default_rng(5)
    w, v = rng.standard_normal(vlp.n), rng.standard_normal(vlp.m)
    t = _tensors(vlp)
    x, y = lp_solve(**t, settings=_settings(tol=1e-9, crossover=crossover))
    loss = (torch.tensor(w, device="cuda") * x).sum() + (torch.tensor(v, device="cuda") * y).sum()
    loss.backward()
    dc, db, dval = _basis_derivatives(vlp, w, v)
    # Without crossover the A-gradient uses PDLP's x and y, accurate to the 1e-9 tolerance.
    rtol = 1e-7 if crossover else 1e-5
    _close(t["c"].grad.cpu().numpy(), dc, rtol)
    _close((t["con_lo"].grad + t["con_up"].grad).cpu().numpy(), db, rtol)
    _close(t["values"].grad.cpu().numpy(), dval, rtol)


def test_finite_differences_through_the_solver(vlp):
    """Central differences of L = w.x* + v.y* on 4 coordinates each of c, b and the A values,
    the 24 perturbed LPs solved in one batched call."""
    from cuopt_b200.torch_layer import LPInstance, lp_solve, lp_solve_batch
    rng = np.random.default_rng(9)
    w, v = rng.standard_normal(vlp.n), rng.standard_normal(vlp.m)
    h = 1e-6
    t = _tensors(vlp)
    x, y = lp_solve(**t, settings=_settings())
    wt, vt = torch.tensor(w, device="cuda"), torch.tensor(v, device="cuda")
    ((wt * x).sum() + (vt * y).sum()).backward()
    grads = {"c": t["c"].grad.cpu().numpy(), "b": t["con_lo"].grad.cpu().numpy(),
             "values": t["values"].grad.cpu().numpy()}
    picks = {"c": rng.choice(vlp.n, 4, replace=False), "b": rng.choice(vlp.m, 4, replace=False),
             "values": rng.choice(vlp.nnz, 4, replace=False)}
    insts, keys = [], []
    for kind, idx in picks.items():
        for k in idx:
            for sign in (1.0, -1.0):
                c, lo, up, val = (vlp.c.copy(), vlp.con_lo.copy(), vlp.con_up.copy(),
                                  vlp.val.copy())
                if kind == "c":
                    c[k] += sign * h
                elif kind == "b":
                    lo[k] += sign * h
                    up[k] += sign * h
                else:
                    val[k] += sign * h
                f = lambda a: torch.tensor(a, device="cuda", dtype=torch.float64)
                insts.append(LPInstance(f(c), f(lo), f(up), f(val), t["row_offsets"],
                                        t["column_indices"], t["var_lo"], t["var_up"]))
                keys.append((kind, k, sign))
    outs = lp_solve_batch(insts, _settings())
    loss = {}
    for (kind, k, sign), (xs, ys) in zip(keys, outs):
        loss[(kind, k, sign)] = float((xs.detach().cpu().numpy() @ w) + (ys.detach().cpu().numpy() @ v))
    for kind, idx in picks.items():
        for k in idx:
            fd = (loss[(kind, k, 1.0)] - loss[(kind, k, -1.0)]) / (2 * h)
            g = grads[kind][k]
            assert abs(fd - g) <= 1e-5 * abs(g) + 1e-5, (kind, k, fd, g)


def test_adjoint_on_a_degenerate_optimum_is_finite():
    """constructed_lp has a dual-degenerate optimum (more free variables than rows): the
    adjoint falls back to the least-squares response and stays finite."""
    from cuopt_b200.torch_layer import lp_solve
    lp = gen.constructed_lp(200, 500, 8, seed=11)
    t = _tensors(lp)
    x, y = lp_solve(**t, settings=_settings(tol=1e-8, crossover=False))
    x.sum().backward()
    for k in ("c", "con_lo", "values"):
        assert torch.isfinite(t[k].grad).all()


def test_adjoint_requires_an_optimal_solution(vlp):
    from cuopt_b200.torch_layer import lp_solve
    s = settings(tol=1e-12, iteration_limit=20)
    t = _tensors(vlp)
    x, _ = lp_solve(**t, settings=s)
    with pytest.raises(lpm.CuOptError):
        x.sum().backward()


def test_batched_backward_equals_single_backwards():
    """lp_solve_batch back-propagates through one cuOptSolutionAdjointBatch call (every active-set
    system in one launch); the gradients equal those of the instances solved and differentiated one
    at a time (each system's LSQR runs alone in its thread block, so the batch does not change it)."""
    from cuopt_b200.torch_layer import LPInstance, lp_solve, lp_solve_batch
    lps = [gen.vertex_lp(150 + 50 * i, 300 + 100 * i, 6, seed=70 + i) for i in range(3)]
    rng = np.random.default_rng(12)
    ws = [rng.standard_normal(lp.n) for lp in lps]
    batch_t = [_tensors(lp) for lp in lps]
    outs = lp_solve_batch([LPInstance(**t) for t in batch_t], _settings())
    sum((torch.tensor(w, device="cuda") * x).sum() for w, (x, _) in zip(ws, outs)).backward()
    for lp, w, tb in zip(lps, ws, batch_t):
        ts = _tensors(lp)
        x, _ = lp_solve(**ts, settings=_settings())
        (torch.tensor(w, device="cuda") * x).sum().backward()
        for k in ("c", "con_lo", "con_up", "values"):
            _close(tb[k].grad.cpu().numpy(), ts[k].grad.cpu().numpy(), 1e-9)


def test_c4_shape_adjoint_against_vertex_map():
    """Four 5000 x 10000 vertex LPs (the 64-LP adjoint workload's shape) through the bench's own
    check: batched forward with crossover, the batched matrix-free backward of L = w.x*, then
    (a) the crossover vertex equals each LP's constructed vertex to 1e-9, (b) the gradients equal
    the exact derivatives of the vertex to 1e-7 (relative to their largest magnitude), and
    (c) central differences (h = 1e-6) of the vertex map on 32 coordinates of each of c, b and the
    A values per instance agree to 1e-4 (|fd - g| / (1 + |g|)), as do differences through the full
    solver on one instance."""
    import argparse
    from cuopt_b200.profile import run_adjoint
    r = run_adjoint(argparse.Namespace(count=4, tol=1e-6, fd_coords=32, fd_solver=1))
    assert r["crossover_vertex_max_rel_error"] <= 1e-9
    assert max(r["grad_vs_exact_max_rel_error"].values()) <= 1e-7
    assert r["fd_checked"] == 4 * 3 * 32
    assert r["fd_max_rel_error"] <= 1e-4, r["fd_worst"]
    assert r["fd_through_solver_checked"] == 12
    assert r["fd_through_solver_max_rel_error"] <= 1e-4
