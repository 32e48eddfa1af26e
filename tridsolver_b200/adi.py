"""ADI heat diffusion on the GPU over the C ABI (tridXadiSteps / tridXadiSolve).

The reference app (apps/adi/src/adi_orig.c:147-240) advances
    u <- u + Z^{-1} Y^{-1} X^{-1} (lambda * L u)
with L the interior-masked 7-point Laplacian and X, Y, Z tridiagonal along
x, y, z: interior rows (a, b, c), face rows identity.  Two coefficient sets:
    "reference": a = c = -lambda/2, b = 1 + lambda   (the reference app)
    "plain":     a = c = -lambda,   b = 1 + 2*lambda   (the plain implicit step)
("baseline" is accepted as another name of "plain").
Tensors are (nz, ny, nx) contiguous CUDA tensors (x fastest).

ADI.run(u, n, graph=True) captures one step in a CUDA graph and replays it;
ADI.grad_final_norm(u0, n, every) differentiates ||u_n||_2 with respect to
u0 and lambda by the adjoint of each step, recomputing the forward states of
each segment from checkpoints stored every `every` steps.
"""

import ctypes

import torch

from ._lib import TridError, c_int, lib, register, vp
from .scalar import _bind_stream, _ptr

c_dbl = ctypes.c_double
c_flt = ctypes.c_float
register({
    "tridDadiSteps": (c_int, [vp, vp, c_int, c_int, c_int, c_int, c_dbl, c_dbl, c_dbl, c_dbl]),
    "tridSadiSteps": (c_int, [vp, vp, c_int, c_int, c_int, c_int, c_flt, c_flt, c_flt, c_flt]),
    "tridDadiSolve": (c_int, [vp, vp, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_dbl, c_dbl,
                              c_dbl, c_dbl]),
    "tridSadiSolve": (c_int, [vp, vp, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_flt, c_flt,
                              c_flt, c_flt]),
    "tridDadiLaplacianT": (c_int, [vp, vp, c_int, c_int, c_int, c_dbl]),
    "tridDadiStepVjp": (c_int, [vp, vp, vp, vp, vp, vp, vp, vp, c_int, c_int, c_int, c_dbl, c_dbl,
                                c_dbl, c_dbl, vp]),
})

COEFFS = {
    "reference": (lambda lam: (-0.5 * lam, 1.0 + lam, -0.5 * lam), (-0.5, 1.0, -0.5)),
    "plain": (lambda lam: (-lam, 1.0 + 2.0 * lam, -lam), (-1.0, 2.0, -1.0)),
}
COEFFS["baseline"] = COEFFS["plain"]


def _check(st, what):
    if st != 0:
        raise TridError(st, what)


class ADI:
    def __init__(self, shape, lam, coeffs="plain", dtype=torch.float64, device="cuda"):
        self.nz, self.ny, self.nx = (int(v) for v in shape)
        self.lam = float(lam)
        self.kind = coeffs
        self.a, self.b, self.c = COEFFS[coeffs][0](self.lam)
        self.da, self.db, self.dc = COEFFS[coeffs][1]
        if dtype not in (torch.float32, torch.float64):
            raise TypeError("ADI runs in float32 or float64")
        self.dtype = dtype
        self.work = torch.empty((2,) + tuple(shape), dtype=dtype, device=device)
        self._graph = None
        self._graph_u = None

    # ------------------------------------------------------------ forward --
    def step(self, u, nsteps=1):
        if u.dtype != self.dtype:
            raise TypeError(f"u is {u.dtype}, this ADI runs in {self.dtype}")
        L = lib()
        _bind_stream(L)
        fn = L.tridDadiSteps if self.dtype == torch.float64 else L.tridSadiSteps
        _check(fn(_ptr(u), _ptr(self.work), self.nx, self.ny, self.nz, int(nsteps), self.lam,
                  self.a, self.b, self.c), "tridXadiSteps")
        return u

    def run(self, u, nsteps, graph=True):
        """nsteps steps in place; with graph=True one step is captured in a
        CUDA graph (three kernels) and replayed."""
        if not graph:
            return self.step(u, nsteps)
        if self._graph is None or self._graph_u is not u:
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                self.step(u)  # warm-up outside the capture
            torch.cuda.current_stream().wait_stream(s)
            torch.cuda.synchronize()
            with torch.cuda.graph(g):
                self.step(u)
            self._graph, self._graph_u = g, u
            nsteps -= 1  # the warm-up step counted
        for _ in range(nsteps):
            self._graph.replay()
        return u

    def _solve(self, rhs, out, axis, stencil=0, transpose=0, inc=0):
        if rhs.dtype != self.dtype or out.dtype != self.dtype:
            raise TypeError(f"arrays must be {self.dtype}")
        L = lib()
        _bind_stream(L)
        fn = L.tridDadiSolve if self.dtype == torch.float64 else L.tridSadiSolve
        _check(fn(_ptr(rhs), _ptr(out), self.nx, self.ny, self.nz, axis, stencil, transpose, inc,
                  self.lam, self.a, self.b, self.c), "tridXadiSolve")
        return out

    def parts(self, u):
        """du1 = X^-1 (lam L u), du2 = Y^-1 du1, du3 = Z^-1 du2."""
        du1 = self._solve(u, torch.empty_like(u), 0, stencil=1)
        du2 = self._solve(du1, torch.empty_like(u), 1)
        du3 = self._solve(du2, torch.empty_like(u), 2)
        return du1, du2, du3

    # ------------------------------------------------------------ adjoint --
    def _step_vjp_into(self, u, ubar, lbar):
        """One step's adjoint: ubar (the cotangent of the step's output) is
        replaced by the cotangent of its input u and the lambda cotangent is
        added into the device scalar lbar.  Six solves (the step's three
        parts, then the three transposed solves) and one fused pass
        (tridDadiStepVjp)."""
        if self.dtype != torch.float64:
            raise TypeError("the ADI adjoint runs in float64")
        du1, du2, du3 = self.parts(u)
        g3 = self._solve(ubar, torch.empty_like(u), 2, transpose=1)
        g2 = self._solve(g3, torch.empty_like(u), 1, transpose=1)
        g1 = self._solve(g2, torch.empty_like(u), 0, transpose=1)
        L = lib()
        _bind_stream(L)
        _check(L.tridDadiStepVjp(_ptr(u), _ptr(du1), _ptr(du2), _ptr(du3), _ptr(g1), _ptr(g2),
                                 _ptr(g3), _ptr(ubar), self.nx, self.ny, self.nz, self.lam,
                                 self.da, self.db, self.dc, _ptr(lbar)), "tridDadiStepVjp")
        return ubar

    def step_vjp(self, u, ubar):
        """Cotangents of (u, lambda) for one step u' = u + du3, given ubar = dL/du'."""
        lbar = torch.zeros((), dtype=u.dtype, device=u.device)
        uprev = self._step_vjp_into(u, ubar.clone(), lbar)
        return uprev, lbar

    def grad_final_norm(self, u0, nsteps, every=20):
        """loss = ||u_n||_2 after nsteps; returns (loss, dloss/du0, dloss/dlambda).
        Checkpoints every `every` steps; each backward segment recomputes its
        states from its checkpoint."""
        ckpts = []
        u = u0.clone()
        for t in range(nsteps):
            if t % every == 0:
                ckpts.append(u.clone())
            self.step(u)
        loss = torch.linalg.vector_norm(u)
        ubar = u / loss
        lbar = torch.zeros((), dtype=u.dtype, device=u.device)
        for seg in reversed(range(len(ckpts))):
            t0 = seg * every
            t1 = min(nsteps, t0 + every)
            states = [ckpts[seg].clone()]
            for _ in range(t0, t1 - 1):
                nxt = states[-1].clone()
                self.step(nxt)
                states.append(nxt)
            for t in reversed(range(t1 - t0)):
                self._step_vjp_into(states[t], ubar, lbar)
        return loss, ubar, lbar
