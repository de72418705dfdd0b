"""The hot-path calls allocate nothing and never synchronise with the host, so they can be
captured in a CUDA graph: the chain getrf -> getrs -> getri, matinv, geqrf and gels are captured
once and replayed on fresh inputs; every replay equals the eager calls bit for bit."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


def test_chain_and_extensions_replay_from_a_cuda_graph(ob):
    import torch

    n, batch, nrhs = 32, 4096, 4
    s = torch.cuda.Stream()
    h = ob.Handle(stream=s)
    g = torch.Generator(device="cuda").manual_seed(21)
    src = [torch.randn((batch, n, n), device="cuda", generator=g) for _ in range(2)]
    rhs = [torch.randn((batch, nrhs, n), device="cuda", generator=g) for _ in range(2)]
    A, B = torch.empty_like(src[0]), torch.empty_like(rhs[0])
    Ci, Mi, Q, Ls, Cs = (torch.empty_like(src[0]) for _ in range(5))
    Cg = torch.empty((batch, 2, n), device="cuda")
    piv = torch.empty((batch, n), dtype=torch.int32, device="cuda")
    info, rinfo, minfo, ginfo = (torch.empty(batch, dtype=torch.int32, device="cuda") for _ in range(4))
    tau = torch.empty((batch, n), device="cuda")
    ptr = {k: ob.ptr_array(v) for k, v in dict(A=A, B=B, Ci=Ci, Mi=Mi, Q=Q, Ls=Ls, Cg=Cg, tau=tau, Src=src[0]).items()}
    staging = src[0]  # the captured calls read their inputs from here

    def body():
        A.copy_(staging)
        B.copy_(rhs[0])
        h.getrf(A, n, n, piv=piv, info=info, aptr=ptr["A"])
        h.getrs("N", A, n, n, piv, B, nrhs, n, aptr=ptr["A"], bptr=ptr["B"])
        h.getri(A, n, n, piv, Ci, n, info=rinfo, aptr=ptr["A"], cptr=ptr["Ci"])
        h.matinv(staging, n, n, Mi, n, info=minfo, aptr=ptr["Src"], cptr=ptr["Mi"])
        Q.copy_(staging)
        h.geqrf(Q, n, n, n, tau=tau, aptr=ptr["Q"], tptr=ptr["tau"])
        Ls.copy_(staging)
        Cg.copy_(rhs[0][:, :2, :])
        h.gels("N", Ls, n, 16, 2, n, Cg, n, info=ginfo, aptr=ptr["Ls"], cptr=ptr["Cg"])

    def snapshot():
        return [t.clone() for t in (A, B, Ci, Mi, Q, tau, Ls, Cg, piv, info, rinfo, minfo, ginfo)]

    with torch.cuda.stream(s):
        body()  # warm-up outside the capture (kernel attributes, lazy loading)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        body()
    for i in (0, 1):
        staging.copy_(src[i])
        if i == 1:
            rhs[0].copy_(rhs[1])  # new right-hand sides where the captured copies read them
        graph.replay()
        torch.cuda.synchronize()
        got = snapshot()
        with torch.cuda.stream(s):
            body()
        torch.cuda.synchronize()
        want = snapshot()
        for x, y in zip(got, want):
            assert torch.equal(x.view(torch.int32), y.view(torch.int32))
    h.close()
