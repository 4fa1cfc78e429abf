"""The static-scratch entry point, for callers that cannot allocate device
memory (open stream captures, host callbacks, programs whose device memory
belongs to another allocator): called through the C ABI on device buffers,
twice in a row, it must give the same field as the context entry point
(vpm_fmm2d_field_device) within the FP64 tolerance of the other tests."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _static_call(lib, bufs, n, prm, ex, ey, stream):
    msg = C.create_string_buffer(256)
    st = lib.vpm_fmm2d_field_device_static(*[C.c_void_p(b.data_ptr()) for b in bufs], n, C.byref(prm),
                                           C.c_void_p(ex.data_ptr()), C.c_void_p(ey.data_ptr()),
                                           C.c_void_p(stream), msg, len(msg))
    return st, msg.value.decode()


def test_static_entry_matches_context_entry():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from lsmps_vpm_v2_b200 import Context, default_params, lib, workloads
    from lsmps_vpm_v2_b200.workloads import rel_l2

    L = lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream().cuda_stream
    ctx = Context(0)
    ctx.set_stream(stream)
    prm = default_params()
    cases = [workloads.lamb_oseen_2d(n_side=64, seed=1), workloads.lamb_oseen_2d(n_side=88, seed=2)]
    try:
        for d in cases:  # two calls in a row, different inputs
            bufs = [torch.from_numpy(np.ascontiguousarray(d[k])).to(dev) for k in ("x", "y", "q", "active")]
            n = bufs[0].numel()
            ex_s = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
            ey_s = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
            st, msg = _static_call(L, bufs, n, prm, ex_s, ey_s, stream)
            assert st == 0, msg
            ex_c = torch.empty(n, dtype=torch.float64, device=dev)
            ey_c = torch.empty(n, dtype=torch.float64, device=dev)
            ctx.field2d_device(*bufs, ex_c, ey_c, prm)
            ctx.sync()
            assert rel_l2((ex_s.cpu().numpy(), ey_s.cpu().numpy()), (ex_c.cpu().numpy(), ey_c.cpu().numpy())) <= TOL
        # beyond the stated maximum: rejected with a clear error
        big = torch.zeros(8193, dtype=torch.float64, device=dev)
        st, msg = _static_call(L, [big, big, big, torch.zeros(8193, dtype=torch.uint8, device=dev)], 8193, prm,
                               big, big, stream)
        assert st == 22 and "8192" in msg
    finally:
        ctx.set_stream(None)
        ctx.close()
