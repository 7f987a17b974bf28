"""Differentiable LP layer for PyTorch over libcuopt_b200.

    x, y = lp_solve(c, con_lo, con_up, values, row_offsets, column_indices, var_lo, var_up)

solves  min c.x  s.t.  con_lo <= A x <= con_up,  var_lo <= x <= var_up  (A in CSR: values,
column_indices, row_offsets; int32 indices) with the library's PDLP and returns the primal and
dual solutions as float64 tensors on the device of `c`.  Backward is the KKT adjoint of the
optimal solution (cuOptSolutionAdjointBatch: matrix-free LSQR solves with the active-set matrix
on the GPU, one thread block per system): gradients flow to c, con_lo, con_up and values; the CSR
structure and the variable bounds are constants.  At a non-degenerate vertex these are the exact
derivatives of the solution map; elsewhere they are those of its minimum-norm response.

`lp_solve_batch` solves a list of such LPs with one batched call (cuOptBatchSolve) and returns
one differentiable (x, y) pair per LP.

The layer needs a CUDA device: the forward pass runs on the GPU, as does the adjoint's linear
solve.  Tensors may live on the CPU or on the GPU (the C interface accepts both).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import torch

from cuopt_b200 import linear_programming as lpm
from cuopt_b200._lib import handle_t, lib

__all__ = ["LPInstance", "lp_solve", "lp_solve_batch"]


@dataclass
class LPInstance:
    """One LP of a batch: the tensors of lp_solve's signature."""
    c: torch.Tensor
    con_lo: torch.Tensor
    con_up: torch.Tensor
    values: torch.Tensor
    row_offsets: torch.Tensor
    column_indices: torch.Tensor
    var_lo: torch.Tensor
    var_up: torch.Tensor


def _contig(t: torch.Tensor, dtype) -> torch.Tensor:
    return t.detach().to(dtype=dtype).contiguous()


def _ptr(t: torch.Tensor) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


class _Solved:
    """Owns the C problem and solution handles of one forward pass (kept for backward)."""

    def __init__(self, inst: LPInstance):
        L = lib()
        self.m = int(inst.row_offsets.numel()) - 1
        self.n = int(inst.c.numel())
        self.nnz = int(inst.values.numel())
        self.device = inst.c.device
        # Kept alive while the C layer copies them.
        self._arrays = [_contig(inst.c, torch.float64), _contig(inst.row_offsets, torch.int32),
                        _contig(inst.column_indices, torch.int32),
                        _contig(inst.values, torch.float64), _contig(inst.con_lo, torch.float64),
                        _contig(inst.con_up, torch.float64), _contig(inst.var_lo, torch.float64),
                        _contig(inst.var_up, torch.float64)]
        self.problem = handle_t()
        self.solution = handle_t()
        rc = L.cuOptCreateRangedProblem(self.m, self.n, 1, 0.0,
                                        *[_ptr(a) for a in self._arrays], b"C" * max(self.n, 1),
                                        C.byref(self.problem))
        if rc != 0:
            raise lpm.CuOptError(rc, "cuOptCreateRangedProblem")

    def outputs(self):
        L = lib()
        x = torch.empty(self.n, dtype=torch.float64, device=self.device)
        y = torch.empty(self.m, dtype=torch.float64, device=self.device)
        for f, t in ((L.cuOptGetPrimalSolution, x), (L.cuOptGetDualSolution, y)):
            rc = f(self.solution, _ptr(t))
            if rc != 0:
                raise lpm.CuOptError(rc, f.__name__)
        status = C.c_int32()
        L.cuOptGetTerminationStatus(self.solution, C.byref(status))
        self.status = status.value
        return x, y

    def __del__(self):
        try:
            L = lib()
            if self.solution:
                L.cuOptDestroySolution(C.byref(self.solution))
            if self.problem:
                L.cuOptDestroyProblem(C.byref(self.problem))
        except Exception:
            pass


def _settings(settings: Optional[lpm.SolverSettings]) -> lpm.SolverSettings:
    if settings is not None:
        return settings
    s = lpm.SolverSettings()
    s.set_optimality_tolerance(1e-8)
    s.set_parameter(lpm.CUOPT_METHOD, int(lpm.SolverMethod.PDLP))
    s.set_parameter(lpm.CUOPT_LOG_TO_CONSOLE, False)
    return s


def _adjoint_batch(solved, pairs):
    """cuOptSolutionAdjointBatch over the solutions with a gradient: all their active-set solves in
    one launch.  Returns one (dc, dlo, dup, dval) tuple per solution (None without a gradient)."""
    L = lib()
    jobs = [i for i, (gx, gy) in enumerate(pairs) if gx is not None or gy is not None]
    results = [None] * len(solved)
    if not jobs:
        return results
    keep, ptrs = [], {k: [] for k in ("gx", "gy", "dc", "dlo", "dup", "dval")}
    for i in jobs:
        sv, (gx, gy) = solved[i], pairs[i]
        dev = sv.device
        gx = (torch.zeros(sv.n, dtype=torch.float64, device=dev) if gx is None
              else _contig(gx, torch.float64))
        gy = None if gy is None else _contig(gy, torch.float64)
        outs = (torch.empty(sv.n, dtype=torch.float64, device=dev),
                torch.empty(sv.m, dtype=torch.float64, device=dev),
                torch.empty(sv.m, dtype=torch.float64, device=dev),
                torch.empty(sv.nnz, dtype=torch.float64, device=dev))
        keep.append((gx, gy))
        results[i] = outs
        ptrs["gx"].append(gx.data_ptr())
        ptrs["gy"].append(gy.data_ptr() if gy is not None else None)
        for k, t in zip(("dc", "dlo", "dup", "dval"), outs):
            ptrs[k].append(t.data_ptr())
    arr = lambda vals: (C.c_void_p * len(vals))(*vals)
    probs = (handle_t * len(jobs))(*[solved[i].problem.value for i in jobs])
    sols = (handle_t * len(jobs))(*[solved[i].solution.value for i in jobs])
    if any(t is not None and t.is_cuda for t, _ in keep):
        torch.cuda.synchronize()  # the gradients are complete before the library reads them
    rc = L.cuOptSolutionAdjointBatch(len(jobs), probs, sols, arr(ptrs["gx"]), arr(ptrs["gy"]),
                                     arr(ptrs["dc"]), arr(ptrs["dlo"]), arr(ptrs["dup"]),
                                     arr(ptrs["dval"]))
    if rc != 0:
        raise lpm.CuOptError(rc, "cuOptSolutionAdjointBatch (every solution must be Optimal)")
    return results


class _AttachBatch(torch.autograd.Function):
    """Returns already computed solutions and routes their gradients through the KKT adjoint; the
    adjoints of a batch are one cuOptSolutionAdjointBatch call."""

    @staticmethod
    def forward(ctx, solved, *tensors):
        ctx.solved = solved
        ctx.set_materialize_grads(False)  # an unused output passes no gradient (NULL to the C API)
        out = []
        for sv in solved:
            out.extend(sv.outputs())
        return tuple(out)

    @staticmethod
    def backward(ctx, *grads):
        pairs = [(grads[2 * i], grads[2 * i + 1]) for i in range(len(ctx.solved))]
        results = _adjoint_batch(ctx.solved, pairs)
        flat = [None]
        for r in results:
            flat.extend(r if r is not None else (None, None, None, None))
        return tuple(flat)


def lp_solve(c, con_lo, con_up, values, row_offsets, column_indices, var_lo, var_up,
             settings: Optional[lpm.SolverSettings] = None):
    """Solves one LP; returns differentiable (x, y)."""
    return lp_solve_batch([LPInstance(c, con_lo, con_up, values, row_offsets, column_indices,
                                      var_lo, var_up)], settings)[0]


def lp_solve_batch(instances: Sequence[LPInstance],
                   settings: Optional[lpm.SolverSettings] = None):
    """Solves the LPs with one cuOptBatchSolve call; returns a list of differentiable (x, y)."""
    L = lib()
    solved = [_Solved(inst) for inst in instances]
    s = _settings(settings)._create()
    try:
        probs = (handle_t * len(solved))(*[sv.problem.value for sv in solved])
        sols = (handle_t * len(solved))()
        rc = L.cuOptBatchSolve(probs, len(solved), s, sols)
        for sv, h in zip(solved, sols):
            sv.solution = handle_t(h)
        if rc != 0:
            raise lpm.CuOptError(rc, "cuOptBatchSolve")
    finally:
        L.cuOptDestroySolverSettings(C.byref(s))
    tensors = [t for inst in instances for t in (inst.c, inst.con_lo, inst.con_up, inst.values)]
    out = _AttachBatch.apply(solved, *tensors)
    return [(out[2 * i], out[2 * i + 1]) for i in range(len(instances))]
