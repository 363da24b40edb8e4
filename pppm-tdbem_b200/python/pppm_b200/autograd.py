"""torch.autograd bridge: the listener samples of a Solver as a differentiable function of the
per-triangle surface accelerations.

    sig, token = listener_signal(solver, acc)            # acc: (nsteps, nt) CUDA tensor
    sig2, token = listener_signal(solver, acc2, token)   # a later chunk of the same run
    loss(sig, sig2).backward()                           # acc.grad, acc2.grad

Forward runs pppm_step on the accelerations and returns the new listener samples (nsteps,
nlisteners) in the solver's precision; backward runs pppm_adjoint, the transposed step
backwards in time (the gradient comes back in acc's dtype; the step itself reads the
accelerations as float32).  The samples are linear in the accelerations with the geometry held fixed,
so backward needs no stored forward state.  Chunks of one run are chained through the token:
each chunk's backward continues the reverse sweep the later chunk left, so the gradient of an
early chunk includes its effect on every later chunk.  The geometry must not change between
the forward calls and the backward pass, and no other steps may be taken on the solver between
chained chunks.

    sig = moving_listener_signal(solver, acc, frames, checkpoint_steps=200)

differentiates a moving run: frames = [(first_step, vertices), ...], motion frame f covering
steps [first_f, first_{f+1}).  Its tables depend on the whole motion (the caches refresh only
what moved), so the forward takes a motion checkpoint of the caches at the start of every
segment of about checkpoint_steps steps, and the backward differentiates the frames latest
first, each with its own tables rebuilt from its segment's checkpoint (rewind, then the
segment's update_mesh calls up to that frame) - checkpointing with recomputation on the
geometry side.  The step is linear in the accelerations, so the reverse sweep itself needs no
stored field state.
"""
import numpy as np
import torch

__all__ = ["listener_signal", "moving_listener_signal"]


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
        ctx.solver, ctx.acc_dtype = solver, acc.dtype
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
        return grad.to(ctx.acc_dtype), torch.zeros((), device=dev), None


def listener_signal(solver, acc, token=None):
    """(samples, token): the listener samples of the next acc.shape[0] steps of `solver`, and a
    token that chains a later chunk of the same run to this one."""
    if token is None:
        token = torch.zeros((), device=acc.device)
    return _ListenerSignal.apply(acc, token, solver)


def _segments(bounds, k):
    """start frames of the checkpoint segments: a new segment when at least k steps passed"""
    starts, last = [0], bounds[0]
    for f in range(1, len(bounds) - 1):
        if bounds[f] - last >= k:
            starts.append(f)
            last = bounds[f]
    return starts


class _MovingSignal(torch.autograd.Function):
    @staticmethod
    def forward(ctx, acc, solver, frames, k):
        if not acc.is_cuda or acc.dim() != 2 or acc.shape[1] != solver.nt:
            raise ValueError("acc must be a (nsteps, %d) CUDA tensor" % solver.nt)
        if not frames or frames[0][0] != 0 or any(b[0] <= a[0] for a, b in zip(frames, frames[1:])):
            raise ValueError("frames must start at step 0 with increasing first steps")
        dev = acc.device
        a = acc.detach().to(torch.float32).contiguous()
        n = a.shape[0]
        bounds = [f[0] for f in frames] + [n]
        if bounds[-2] >= n:
            raise ValueError("the last frame starts after the last step")
        starts = _segments(bounds, k)
        first = solver.series_count
        ext = _solver_stream(solver, dev)
        cur = torch.cuda.current_stream(dev)
        if ext is not None:
            ext.wait_stream(cur)
        solver.checkpoint_clear()
        ids = {}
        for f in range(len(frames)):
            if f:
                solver.update_mesh(frames[f][1])
            if f in starts:
                ids[f] = solver.checkpoint_push()
            solver.step(a[bounds[f]: bounds[f + 1]])
        dtype = torch.float64 if solver.precision == "fp64" else torch.float32
        out = torch.empty((n, solver.n_listeners), dtype=dtype, device=dev)
        solver.series(first, n, out=out)
        if ext is not None:
            cur.wait_stream(ext)
        ctx.solver, ctx.frames, ctx.bounds, ctx.starts, ctx.ids = solver, frames, bounds, starts, ids
        ctx.acc_dtype = acc.dtype
        ctx.set_materialize_grads(False)
        return out

    @staticmethod
    def backward(ctx, g_sig):
        solver, frames, bounds, starts = ctx.solver, ctx.frames, ctx.bounds, ctx.starts
        n = bounds[-1]
        dtype = torch.float64 if solver.precision == "fp64" else torch.float32
        if g_sig is None:
            g_sig = torch.zeros((n, solver.n_listeners), dtype=dtype, device="cuda")
        dev = g_sig.device
        g = g_sig.to(dtype).contiguous()
        grad = torch.empty((n, solver.nt), dtype=dtype, device=dev)
        ext = _solver_stream(solver, dev)
        cur = torch.cuda.current_stream(dev)
        if ext is not None:
            ext.wait_stream(cur)
        fresh = True
        ends = starts[1:] + [len(frames)]
        for s0, s1 in reversed(list(zip(starts, ends))):
            for f in range(s1 - 1, s0 - 1, -1):
                # frame f's tables: the segment's checkpoint, then its meshes up to frame f
                solver.checkpoint_rewind(ctx.ids[s0])
                for ff in range(s0, f + 1):
                    solver.update_mesh(frames[ff][1])
                a, b = bounds[f], bounds[f + 1]
                solver.adjoint(g[a:b], fresh=fresh, out=grad[a:b])
                fresh = False
        solver.checkpoint_clear()
        if ext is not None:
            cur.wait_stream(ext)
        return grad.to(ctx.acc_dtype), None, None, None


def moving_listener_signal(solver, acc, frames, checkpoint_steps=200):
    """The listener samples (nsteps, nlisteners) of a moving run of `solver` over the rows of
    `acc`, differentiable with respect to acc (one backward pass).  frames: [(first_step,
    vertices), ...] with first_step 0 first (its vertices are those the solver's mesh holds now).
    The motion checkpoints (pppm_checkpoint_*) stay in device memory until the backward ends,
    their arena until solver.checkpoint_clear(release=True) (a training loop reuses it); the
    solver's own checkpoints are replaced.  After backward the solver's caches are those of
    frame 0 and its fields those of the reverse sweep, not of the run's end."""
    return _MovingSignal.apply(acc, solver, list(frames), int(checkpoint_steps))
