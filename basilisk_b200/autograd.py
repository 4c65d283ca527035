"""The differentiable Poisson--Helmholtz solve.

``solve(problem, b, alpha, lam)`` returns ``a`` with ``L(alpha, lambda) a = b``
(the operator whose residual is Basilisk's poisson.h:373-389) as a
``torch.autograd.Function`` over the C-ABI of ``libbmg.so``: the forward is
the GPU multigrid solve, and the hand-written backward is one more solve of
the same (symmetric) operator for the adjoint ``mu`` from ``dl/da`` with the
homogeneous boundary conditions, followed by the fused adjoint kernel of the
library (``bmg_adjoint_gradients``):

    dl/db      = mu
    dl/dalpha  = grad(mu) . grad(a) on every face (boundary faces: the
                 interior cell's term only)
    dl/dlambda = -mu a

On a singular problem (no Dirichlet side and no lambda: periodic or Neumann
walls, pure Poisson) the solution is defined up to a constant.  The forward
pass then solves for the zero-mean projection of b (the compatibility
condition) and returns the zero-mean solution; the backward pass projects
dl/da to zero mean before the adjoint solve and returns the zero-mean
adjoint, so the gradients are those of that well-defined map.  A solve that
does not reach the tolerance raises ``BMGError`` (status ENOTCONV) instead of
returning an unconverged field.

The function keeps only the forward solution for the backward pass.
``chain`` runs time-stepped sequences of solves with a checkpoint every k
steps (the solutions inside a segment are recomputed in the backward pass).

Tensors are CUDA float64, shape (n,)*dim or (B,)+(n,)*dim for a batch of
independent instances; face component d has n+1 entries along d.
"""
import ctypes

import torch

from . import _lib
from .grid import Grid


class _Lane:
    """One grid of a Problem, with the fields of one instance's solve and its
    own CUDA stream (each grid owns one)."""

    def __init__(self, pb, L0, origin, relax, precision, alpha, lam):
        self.pb = pb
        self.grid = Grid(pb.dim, pb.depth, L0=L0, origin=origin, relax=relax, precision=precision)
        g = self.grid
        for d in pb.periodic:
            g.periodic(2 * d)
        self.a, self.b, self.mu, self.rhs = g.scalar(), g.scalar(), g.scalar(), g.scalar()
        for side, (kind, val) in pb.bc.items():
            self.a.bc(side, kind, val)
            self.mu.bc(side, kind, 0.0)          # the homogeneous twin
        self.alpha = g.face_vector() if alpha else None
        self.lam = g.scalar() if lam else None

    def _set_coefficients(self, alpha, lam):
        if self.alpha is not None:
            for c, v in zip(self.alpha.components, alpha):
                c.set(v)
        if self.lam is not None:
            self.lam.set(lam)

    def _solve(self, a, b, out):
        pb = self.pb
        a.set(torch.zeros_like(out))
        st = self.grid.poisson(a, b, alpha=self.alpha, lambda_=self.lam,
                               tolerance=pb.tolerance, nrelax=pb.nrelax)
        pb.stats.append(st)
        if st["status"] != _lib.OK:
            raise _lib.BMGError(st["status"], "differentiable solve (residual %g after %d "
                                "V-cycles, tolerance %g)" % (st["resa"], st["i"], pb.tolerance))
        a.get(out=out)
        if pb.singular:
            out -= out.mean()
        return st

    def forward_one(self, b, alpha, lam, out):
        self._set_coefficients(alpha, lam)
        self.b.set(self.pb._compatible(b))
        return self._solve(self.a, self.b, out)

    def backward_one(self, a_sol, grad_a, alpha, lam, grad_b, grad_alpha, grad_lam):
        """mu from dl/da, then the coefficient gradients; grad_b receives mu."""
        self._set_coefficients(alpha, lam)
        self.rhs.set(self.pb._compatible(grad_a))
        self._solve(self.mu, self.rhs, grad_b)
        # a with the ghosts of its boundary conditions, for the face kernel
        self.a.set(a_sol)
        L = _lib.load()
        ptrs = (ctypes.c_void_p * 3)()
        for d in range(3):
            ptrs[d] = grad_alpha[d].data_ptr() if grad_alpha is not None and d < self.pb.dim else None
        torch.cuda.current_stream().synchronize()
        _lib.check(L.bmg_adjoint_gradients(
            self.grid.ptr, self.mu.scalar, self.a.scalar,
            ptrs if grad_alpha is not None else None,
            grad_lam.data_ptr() if grad_lam is not None else None, _lib.DEVICE),
            "bmg_adjoint_gradients")


class Problem:
    """The fixed part of a family of solves: grid, boundary conditions of a
    (``bc = {side: (kind, value)}``, sides in the reference's order right,
    left, top, bottom, front, back), periodic directions, tolerance,
    precision ("fp64" or "mixed") and smoother.

    ``lanes`` > 1 gives the problem that many independent grids, each on its
    own CUDA stream: the instances of a batch are dealt out to them and
    solved concurrently, one host thread per lane (a solve is a sequence of
    V-cycles whose residual is read back after each, so a single thread runs
    one solve at a time; ctypes releases the interpreter lock during the
    library's calls).  The results are those of one lane, instance by
    instance."""

    def __init__(self, dim, depth, periodic=(), bc=None, tolerance=1e-10, precision="fp64",
                 relax="rbgs", nrelax=4, L0=1.0, origin=(0.0, 0.0, 0.0), alpha=True,
                 lam=False, lanes=1):
        self.dim, self.depth, self.n = dim, depth, 1 << depth
        self.tolerance, self.nrelax = tolerance, nrelax
        self.periodic = tuple(periodic)
        self.bc = dict(bc or {})
        # no Dirichlet side and no lambda: L has the constants as its null space
        self.singular = not lam and not any(kind == "dirichlet" for kind, _ in self.bc.values())
        self.stats = []
        self.lanes = [_Lane(self, L0, origin, relax, precision, alpha, lam)
                      for _ in range(max(1, int(lanes)))]
        first = self.lanes[0]
        self.grid, self.a, self.b, self.mu, self.rhs = first.grid, first.a, first.b, first.mu, first.rhs
        self.alpha, self.lam = first.alpha, first.lam
        self._pool = None

    def close(self):
        if self._pool is not None:
            self._pool.shutdown()
            self._pool = None
        for lane in self.lanes:
            lane.grid.close()

    def _compatible(self, rhs):
        """the right-hand side of a solve: its zero-mean projection on a
        singular problem (in FP64, before the solve)"""
        return rhs - rhs.mean() if self.singular else rhs

    # -- one instance on the first lane (the single-lane interface) -----
    def forward_one(self, b, alpha, lam, out):
        return self.lanes[0].forward_one(b, alpha, lam, out)

    def backward_one(self, *args):
        return self.lanes[0].backward_one(*args)

    def _each(self, count, work):
        """work (lane, k) for k < count: instance k on lane k mod lanes, the
        lanes concurrently"""
        nl = len(self.lanes)
        if nl == 1 or count == 1:
            for k in range(count):
                work(self.lanes[0], k)
            return
        from concurrent.futures import ThreadPoolExecutor
        if self._pool is None:
            self._pool = ThreadPoolExecutor(max_workers=nl)
        torch.cuda.current_stream().synchronize()

        def lane_job(j):
            for k in range(j, count, nl):
                work(self.lanes[j], k)
            # this thread's own torch work (zero-mean projections) is done
            # before the caller reads the results on its stream
            torch.cuda.current_stream().synchronize()
        for f in [self._pool.submit(lane_job, j) for j in range(min(nl, count))]:
            f.result()


class _Solve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, problem, b, lam, *alpha):
        batched = b.dim() == problem.dim + 1
        bb = b if batched else b.unsqueeze(0)
        out = torch.empty_like(bb)
        def one(lane, k):
            al = [x[k] if batched else x for x in alpha]
            lm = None if lam is None else (lam[k] if batched else lam)
            lane.forward_one(bb[k].contiguous(), al, lm, out[k])
        problem._each(bb.shape[0], one)
        a = out if batched else out[0]
        ctx.problem, ctx.batched = problem, batched
        ctx.has_lam, ctx.nalpha = lam is not None, len(alpha)
        ctx.save_for_backward(a, *((lam,) if lam is not None else ()), *alpha)
        return a

    @staticmethod
    def backward(ctx, grad_a):
        problem, batched = ctx.problem, ctx.batched
        saved = ctx.saved_tensors
        a = saved[0]
        lam = saved[1] if ctx.has_lam else None
        alpha = saved[1 + ctx.has_lam:]
        A = a if batched else a.unsqueeze(0)
        G = (grad_a if batched else grad_a.unsqueeze(0)).contiguous()
        grad_b = torch.empty_like(A)
        grad_alpha = [torch.empty((A.shape[0],) + tuple(x.shape[-problem.dim:]),
                                  dtype=torch.float64, device=A.device) for x in alpha]
        grad_lam = torch.empty_like(A) if lam is not None else None
        def one(lane, k):
            al = [x[k] if batched else x for x in alpha]
            lm = None if lam is None else (lam[k] if batched else lam)
            lane.backward_one(A[k].contiguous(), G[k], al, lm, grad_b[k],
                              [ga[k] for ga in grad_alpha] if alpha else None,
                              grad_lam[k] if lam is not None else None)
        problem._each(A.shape[0], one)
        if not batched:
            grad_b = grad_b[0]
            grad_alpha = [x[0] for x in grad_alpha]
            grad_lam = grad_lam[0] if grad_lam is not None else None
        return (None, grad_b, grad_lam, *grad_alpha)


def solve(problem, b, alpha=None, lam=None):
    """a = L(alpha, lam)^{-1} b on ``problem``'s grid (differentiable in b,
    alpha and lam).  alpha: a list of dim face tensors (None: alpha = 1);
    lam: a cell tensor (None: lambda = 0)."""
    if (alpha is None) != (problem.alpha is None):
        raise ValueError("alpha must match the Problem (alpha=True/False)")
    if (lam is None) != (problem.lam is None):
        raise ValueError("lam must match the Problem (lam=True/False)")
    alpha = tuple(alpha) if alpha is not None else ()
    return _Solve.apply(problem, b, lam, *alpha)


def chain(step, x, nsteps, every=1):
    """x_{k+1} = step(x_k), nsteps times, with a checkpoint every ``every``
    steps: only the segment boundaries are kept for the backward pass; the
    solves inside a segment are run again when the gradient reaches it."""
    from torch.utils.checkpoint import checkpoint

    def segment(x, m):
        for _ in range(m):
            x = step(x)
        return x

    done = 0
    while done < nsteps:
        m = min(every, nsteps - done)
        if every > 1 and x.requires_grad:
            x = checkpoint(segment, x, m, use_reentrant=False)
        else:
            x = segment(x, m)
        done += m
    return x
