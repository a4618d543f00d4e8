"""ostc_residual_noalloc: the residual norms for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc (a host whose device memory is pre-planned and owned by its own
pool, loops that must not pay an allocation's implicit synchronisation, code running during another
thread's global-mode graph capture).  For them the library offers one entry point whose scratch is a
static device array: this test calls it through the C ABI on device copies of two states and checks
it against the context's allocating ostc_residual, on two calls in a row (the second call reuses
the static scratch left by the first), checks that a call leaves the device's free memory unchanged,
and runs it on a non-blocking stream (the kind a caller beside another thread's graph capture must
use).  It runs alone or after every other test.
"""
import numpy as np
import pytest

import ostc
import ostc_cases as oc

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def test_residual_noalloc_matches_residual(built, tmp_path):
    import torch

    case = oc.mixing_layer_3d(mx=40, my=24, mz=20)
    d = oc.write_case(case, tmp_path / "noalloc")
    s = ostc.Solver(str(d))
    s.set_state(case.bv)
    n = case.nodes
    for call in range(2):
        s.store_residual_reference()
        _, b0 = s.get_state()
        s.step(2 + call)
        _, b1 = s.get_state()
        ref = s.residual()
        d_new = torch.from_numpy(np.ascontiguousarray(b1)).cuda()
        d_old = torch.from_numpy(np.ascontiguousarray(b0)).cuda()
        torch.cuda.synchronize()
        got = ostc.residual_noalloc(d_new.data_ptr(), d_old.data_ptr(), n)
        assert np.all(ref > 0), ref
        assert np.allclose(got, ref, rtol=RTOL, atol=0), (call, got, ref)


def test_residual_noalloc_allocates_nothing_on_a_nonblocking_stream(built, tmp_path):
    import torch

    case = oc.mixing_layer_3d(mx=32, my=20, mz=16)
    d = oc.write_case(case, tmp_path / "noalloc_stream")
    s = ostc.Solver(str(d))
    s.set_state(case.bv)
    s.store_residual_reference()
    _, b0 = s.get_state()
    s.step(3)
    _, b1 = s.get_state()
    ref = s.residual()
    d_new = torch.from_numpy(np.ascontiguousarray(b1)).cuda()
    d_old = torch.from_numpy(np.ascontiguousarray(b0)).cuda()
    stream = torch.cuda.Stream()  # cudaStreamNonBlocking
    torch.cuda.synchronize()
    ostc.residual_noalloc(d_new.data_ptr(), d_old.data_ptr(), case.nodes, stream.cuda_stream)  # warm-up
    free0, _ = torch.cuda.mem_get_info()
    got = ostc.residual_noalloc(d_new.data_ptr(), d_old.data_ptr(), case.nodes, stream.cuda_stream)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert np.allclose(got, ref, rtol=RTOL, atol=0), (got, ref)


def test_residual_noalloc_rejects_oversize(built):
    with pytest.raises(ostc.OstcError, match="outside 1.."):
        ostc.residual_noalloc(1, 1, 256 * 64 * 4096 + 1)
