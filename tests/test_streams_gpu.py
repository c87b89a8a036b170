"""The split form's stream handling: the solve runs on a highest-priority stream
forked from the caller's (or on the caller's own when its priority is already above
the lowest), and the recovery's digit kernel on a lowest-priority side stream forked
when the Newton steps start.  Whatever the caller's stream, and with several caller
streams in flight at once, the results are bit-identical and ordered on the caller's
stream."""
from __future__ import annotations

import pytest
import torch

from oracle import ssn_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sp():
    import symplectic_projection as sp
    sp.initialize_kernels()
    return sp


def _same(a, b):
    return (torch.equal(a.X, b.X) and torch.equal(a.omega, b.omega) and torch.equal(a.iterations, b.iterations)
            and torch.equal(a.status, b.status))


@pytest.mark.parametrize("n,k,batch", [(512, 16, 6), (4096, 48, 3)])
def test_split_solve_is_the_same_on_every_caller_stream(sp, n, k, batch):
    from symplectic_projection.dual_recommended_hvp import solve_ex
    T = O.make_inputs(n, k, 1, batch)[0].cuda()
    ref = solve_ex(T, precision="split")
    torch.cuda.synchronize()
    highest = torch.cuda.Stream.priority_range()[1]     # (least, greatest)
    for priority in (0, highest):
        s = torch.cuda.Stream(priority=priority)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            out = solve_ex(T, precision="split")
            # ordered on the caller's stream: a copy enqueued after the call sees the result
            Xc = out.X.clone()
        s.synchronize()
        assert _same(out, ref), f"priority {priority}"
        assert torch.equal(Xc, ref.X)
    assert ref.status.cpu().tolist() == [0] * batch


def test_split_solves_on_concurrent_streams(sp):
    """Four caller streams with solves in flight at once (each forks its own
    highest-priority stream; they share the thread's side stream)."""
    from symplectic_projection.dual_recommended_hvp import solve_ex
    inputs = [O.make_inputs(1024, 24, c, 4)[0].cuda() for c in range(4)]
    refs = [solve_ex(T, precision="split") for T in inputs]
    torch.cuda.synchronize()
    streams = [torch.cuda.Stream() for _ in inputs]
    outs = []
    for s, T in zip(streams, inputs):
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            outs.append(solve_ex(T, precision="split"))
    for s in streams:
        s.synchronize()
    for out, ref in zip(outs, refs):
        assert _same(out, ref)
        assert ref.status.cpu().tolist() == [0] * 4
