"""torch.autograd bridge: the listener samples of a Solver as a differentiable function of the
per-triangle surface accelerations.

    sig, token = listener_signal(solver, acc)            # acc: (nsteps, nt) CUDA tensor
    sig2, token = listener_signal(solver, acc2, token)   # a later chunk of the same run
    loss(sig, sig2).backward()                           # acc.grad, acc2.grad

Forward runs pppm_step on the accelerations and returns the new listener samples (nsteps,
nlisteners) in the solver's precision; backward runs pppm_adjoint, the transposed step
backwards in time.  The samples are linear in the accelerations with the geometry held fixed,
so backward needs no stored forward state.  Chunks of one run are chained through the token:
each chunk's backward continues the reverse sweep the later chunk left, so the gradient of an
early chunk includes its effect on every later chunk.  The geometry must not change between
the forward calls and the backward pass (update_mesh invalidates the sweep), and no other
steps may be taken on the solver between chained chunks.
"""
import torch

__all__ = ["listener_signal"]


def _solver_stream(solver, device):
    return torch.cuda.ExternalStream(solver.stream, device=device) if solver.stream else None


class _ListenerSignal(torch.autograd.Function):
    @staticmethod
    def forward(ctx, acc, token, solver):
        if not acc.is_cuda or acc.dim() != 2 or acc.shape[1] != solver.nt:
            raise ValueError("acc must be a (nsteps, %d) CUDA tensor" % solver.nt)
        dev = acc.device
        a = acc.detach().to(torch.float32).contiguous()
        n = a.shape[0]
        first = solver.series_count
        t0 = solver.t
        ext = _solver_stream(solver, dev)
        cur = torch.cuda.current_stream(dev)
        if ext is not None:
            ext.wait_stream(cur)  # the accelerations are ready before the solver reads them
        solver.step(a)
        dtype = torch.float64 if solver.precision == "fp64" else torch.float32
        out = torch.empty((n, solver.n_listeners), dtype=dtype, device=dev)
        solver.series(first, n, out=out)
        if ext is not None:
            # later work on the caller's stream (including reuse of a's and out's memory) comes
            # after the solver's; no record_stream: the solver's stream may be destroyed first
            cur.wait_stream(ext)
        ctx.solver = solver
        ctx.span = (t0 + 1, t0 + 1 + n)  # forward time indices of the chunk's steps
        ctx.set_materialize_grads(False)
        return out, torch.zeros((), device=dev)

    @staticmethod
    def backward(ctx, g_sig, g_token):
        solver = ctx.solver
        a, b = ctx.span
        # the chunk whose token nobody consumed is the latest: it starts the reverse sweep
        fresh = g_token is None
        pos = getattr(solver, "_adjoint_pos", None)
        if not fresh and pos != b:
            raise RuntimeError("chained chunks must be differentiated latest first, with no other steps in between")
        n = b - a
        dtype = torch.float64 if solver.precision == "fp64" else torch.float32
        if g_sig is None:
            g_sig = torch.zeros((n, solver.n_listeners), dtype=dtype, device="cuda")
        dev = g_sig.device
        g = g_sig.to(dtype).contiguous()
        ext = _solver_stream(solver, dev)
        cur = torch.cuda.current_stream(dev)
        if ext is not None:
            ext.wait_stream(cur)
        grad = solver.adjoint(g, fresh=fresh)
        if ext is not None:
            cur.wait_stream(ext)
        solver._adjoint_pos = a
        return grad.to(torch.float32), torch.zeros((), device=dev), None


def listener_signal(solver, acc, token=None):
    """(samples, token): the listener samples of the next acc.shape[0] steps of `solver`, and a
    token that chains a later chunk of the same run to this one."""
    if token is None:
        token = torch.zeros((), device=acc.device)
    return _ListenerSignal.apply(acc, token, solver)
