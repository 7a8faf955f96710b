"""GPU test of sbp_mdl_device_noalloc, the allocation-free MDL entry point.

Callers that cannot allocate GPU memory (a fixed device-memory budget, or code that must not
call cudaMalloc/cudaFree because those synchronize the device while work is in flight) pass
their own device buffers; the entry point's only scratch is a static device array.  This test
owns every buffer (allocated here with torch, as such a caller would), calls the entry point
through the C ABI twice in a row and checks each result against sbp_mdl, the allocating entry
point, and against the CPU oracle's MDL, within the MDL tolerance of the other GPU tests.  It is
collected last so that a run that stops at the first failure has already run everything else,
and it also passes alone.
"""
import numpy as np
import pytest

from conftest import random_assignment, random_graph

pytestmark = pytest.mark.gpu
RTOL_MDL = 1e-9


def device_inputs(S, torch, bm):
    M = torch.from_numpy(np.ascontiguousarray(bm.blockmatrix())).cuda()
    do, di, _ = bm.degrees_all()
    return M, torch.from_numpy(do).cuda(), torch.from_numpy(di).cuda()


def call(S, torch, M, do, di, V, E, out):
    stream = torch.cuda.current_stream()
    S.mdl_device_noalloc(M.data_ptr(), M.shape[0], M.shape[1], do.data_ptr(), di.data_ptr(), V, E, out.data_ptr(),
                         stream.cuda_stream)
    stream.synchronize()
    return float(out.item())


def test_noalloc_mdl_matches_allocating_mdl_twice(S, O):
    import torch
    V, s, d, _ = random_graph(2000, 8, 91)
    g, og = S.Graph(V, s, d), O.Graph(V, s, d)
    cases = []
    for B, seed in ((300, 1), (40, 2)):
        a = random_assignment(V, B, seed)
        bm = S.Blockmodel(g, B, a)
        ref = S.entropy.mdl(bm)
        assert ref == pytest.approx(O.Blockmodel(og, B, a).mdl(), rel=RTOL_MDL)
        cases.append((bm, ref))
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    # two calls in a row on the same inputs, then a different B, then the first again: the
    # shared scratch array keeps the previous call's contents, which must not leak
    bm0, ref0 = cases[0]
    M, do, di = device_inputs(S, torch, bm0)
    first = call(S, torch, M, do, di, V, g.E, out)
    second = call(S, torch, M, do, di, V, g.E, out)
    assert first == pytest.approx(ref0, rel=RTOL_MDL)
    assert second == pytest.approx(ref0, rel=RTOL_MDL)
    bm1, ref1 = cases[1]
    M1, do1, di1 = device_inputs(S, torch, bm1)
    assert call(S, torch, M1, do1, di1, V, g.E, out) == pytest.approx(ref1, rel=RTOL_MDL)
    assert call(S, torch, M, do, di, V, g.E, out) == pytest.approx(ref0, rel=RTOL_MDL)


def test_noalloc_mdl_rejects_sizes_beyond_its_limit(S):
    import torch
    M = torch.zeros((1, 1), dtype=torch.int32, device="cuda")
    deg = torch.zeros((1,), dtype=torch.int32, device="cuda")
    out = torch.zeros((1,), dtype=torch.float64, device="cuda")
    with pytest.raises(S.SbpError) as e:
        S.mdl_device_noalloc(M.data_ptr(), 32769, 32769, deg.data_ptr(), deg.data_ptr(), 10, 10, out.data_ptr(), None)
    assert e.value.code == 3
    assert "32768-block limit" in S.last_error()
    assert "32768-block limit" in str(e.value)
