"""The context-free shift solve (isa_solve_shifts_static).

It serves hosts that cannot allocate device memory at the point where they
align tiles; its row tables live in a static device array of the library
instead of an isa_ctx. Its results must equal those of the context-owning
entry point isa_solve_shifts on the same inputs, within the tolerance of the
solver parity tests (2e-5 on shifts, exact status), for two calls in a row
with different burst sizes and strategies, so that nothing left in the
shared array by the first call leaks into the second.
"""
import ctypes

import numpy as np
import pytest

from imagestackalignator_b200 import isa, params as P

pytestmark = pytest.mark.gpu


def _case(rng, n, ref, strategy, block, tcx, tcy):
    A = P.shift_matrix(n, ref, strategy, block)
    m = A.shape[0]
    truth = rng.uniform(-4, 4, (tcx * tcy, n - 1, 2))
    meas = (np.einsum("mk,tkc->tmc", A, truth) + rng.normal(0, 0.05, (tcx * tcy, m, 2))).astype(np.float32)
    meas[::2, rng.integers(0, m), :] += 6.0
    meas[1::3, rng.integers(0, m), 1] -= 9.0
    return np.ascontiguousarray(meas.transpose(1, 0, 2).reshape(m, tcy, tcx, 2))


def _solve(fn, grids_host, n, ref, strategy, block, tcx, tcy, ctx=None):
    import torch
    grids = torch.from_numpy(grids_host.copy()).cuda()
    x = torch.zeros((tcx * tcy, n - 1, 2), dtype=torch.float32, device="cuda")
    st = torch.zeros(tcx * tcy, dtype=torch.int32, device="cuda")
    args = [n, ref, strategy, block, isa.vp(grids), ctypes.c_size_t(tcx * 8), ctypes.c_size_t(tcx * tcy * 8), tcx, tcy, isa.vp(x), isa.vp(st),
            None]
    if ctx is not None:
        args = [ctx] + args
    isa.check(fn(*args))
    torch.cuda.synchronize()
    return grids.cpu().numpy(), x.cpu().numpy(), st.cpu().numpy()


@pytest.mark.parametrize("order", ["large_first", "small_first"])
def test_static_solve_matches_context_solve(cuda, order):
    lib = isa.lib()
    rng = np.random.default_rng(99)
    cases = [(20, 0, P.FULL, 5, 23, 15), (7, 3, P.ON_REFERENCE_BLOCK, 3, 9, 6)]
    if order == "small_first":
        cases = cases[::-1]
    merger = isa.Merger(512, 512, 20)  # owns the scratch of the context entry point
    for n, ref, strategy, block, tcx, tcy in cases:  # two calls in a row on the shared static array
        g = _case(rng, n, ref, strategy, block, tcx, tcy)
        want = _solve(lib.isa_solve_shifts, g, n, ref, strategy, block, tcx, tcy, ctx=merger.ctx)
        got = _solve(lib.isa_solve_shifts_static, g, n, ref, strategy, block, tcx, tcy)
        np.testing.assert_array_equal(got[2], want[2])
        np.testing.assert_allclose(got[1], want[1], rtol=0, atol=2e-5)
        np.testing.assert_allclose(got[0], want[0], rtol=0, atol=2e-5)
    merger.close()


def test_static_solve_allocates_nothing_after_set_up(cuda):
    """After the set-up call on the device, a call leaves the device's free
    memory unchanged (every buffer of the call is made beforehand)."""
    import torch
    lib = isa.lib()
    rng = np.random.default_rng(5)
    n, ref, strategy, block, tcx, tcy = 12, 0, P.FULL, 5, 31, 23
    g = _case(rng, n, ref, strategy, block, tcx, tcy)
    grids = torch.from_numpy(g).cuda()
    x = torch.zeros((tcx * tcy, n - 1, 2), dtype=torch.float32, device="cuda")
    st = torch.zeros(tcx * tcy, dtype=torch.int32, device="cuda")
    args = [n, ref, strategy, block, isa.vp(grids), ctypes.c_size_t(tcx * 8), ctypes.c_size_t(tcx * tcy * 8), tcx, tcy, isa.vp(x), isa.vp(st),
            None]
    isa.check(lib.isa_solve_shifts_static(*args))  # set-up on this device
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    isa.check(lib.isa_solve_shifts_static(*args))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_static_solve_rejects_sizes_beyond_its_limit(cuda):
    import torch
    lib = isa.lib()
    grids = torch.zeros(16, device="cuda")
    x = torch.zeros(16, device="cuda")
    st = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc = lib.isa_solve_shifts_static(70, 0, P.FULL, 5, isa.vp(grids), ctypes.c_size_t(8), ctypes.c_size_t(8), 1, 1, isa.vp(x), isa.vp(st), None)
    assert rc == isa.ISA_EINVAL
    assert b"static limit" in lib.isa_last_error()
    # 65 frames are within the frame limit, but Full tracking makes 2080 pairs (> 2048)
    rc = lib.isa_solve_shifts_static(65, 0, P.FULL, 5, isa.vp(grids), ctypes.c_size_t(8), ctypes.c_size_t(8), 1, 1, isa.vp(x), isa.vp(st), None)
    assert rc == isa.ISA_EINVAL
    assert b"frame pairs exceed the static limit" in lib.isa_last_error()
