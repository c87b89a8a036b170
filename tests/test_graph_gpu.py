"""The solve pipeline captured in a CUDA graph and replayed.

ssn_solve enqueues its kernels (and, in the split form, the fork and join of
its side stream) without host synchronisation or resource creation, so it can
be captured once and replayed on new inputs copied into the captured buffers.
Replays must give bit-identical results to direct calls.
"""
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


@pytest.mark.parametrize("precision", ["fp64", "split"])
@pytest.mark.parametrize("n,k,batch", [(512, 16, 8), (4096, 48, 2)])
def test_solve_replays_from_a_cuda_graph(sp, precision, n, k, batch):
    from symplectic_projection.dual_recommended_hvp import solve_ex
    inputs = [O.make_inputs(n, k, c, batch)[0].cuda() for c in range(3)]
    static_T = inputs[0].clone()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):                       # warm-up on the capture stream
        solve_ex(static_T, precision=precision)
    torch.cuda.current_stream().wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        out = solve_ex(static_T, precision=precision)
    for T in inputs[1:] + inputs[:1]:
        static_T.copy_(T)
        graph.replay()
        ref = solve_ex(T, precision=precision)
        torch.cuda.synchronize()
        assert out.status.cpu().tolist() == [0] * batch
        assert torch.equal(out.X, ref.X)
        assert torch.equal(out.omega, ref.omega)
        assert torch.equal(out.iterations, ref.iterations)
