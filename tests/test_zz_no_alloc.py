"""The static-scratch entry point, for callers that cannot allocate device
memory (programs whose device memory belongs to another allocator, and step
loops that must not stall on an allocation): called through the C ABI on
device buffers, twice in a row, it must give the same field as the context
entry point (vpm_fmm2d_field_device) within the tolerance the other tests use
for each form, reject sizes beyond its maximum, and report a tree that
outgrows its array as VPM_EOVERFLOW."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL_FP64 = 1e-10    # FP64 form against FP64 form
TOL_MIXED = 1e-5    # FP32 near field against the same form with a different FP64 M2L
VPM_EINVAL, VPM_EOVERFLOW = 22, 75
VPM_PREC_MIXED, VPM_PREC_MIXED_FP64_M2L = 1, 2


def _static_call(lib, bufs, n, prm, ex, ey, stream):
    msg = C.create_string_buffer(256)
    st = lib.vpm_fmm2d_field_device_static(*[C.c_void_p(b.data_ptr()) for b in bufs], n, C.byref(prm),
                                           C.c_void_p(ex.data_ptr()), C.c_void_p(ey.data_ptr()),
                                           C.c_void_p(stream), msg, len(msg))
    return st, msg.value.decode()


@pytest.fixture(scope="module")
def env():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from lsmps_vpm_v2_b200 import Context, lib
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream().cuda_stream
    ctx = Context(0)
    ctx.set_stream(stream)
    yield torch, lib(), dev, stream, ctx
    ctx.set_stream(None)
    ctx.close()


def _compare(env, d, prm_static, prm_ctx, tol):
    from lsmps_vpm_v2_b200.workloads import rel_l2
    torch, L, dev, stream, ctx = env
    bufs = [torch.from_numpy(np.ascontiguousarray(d[k])).to(dev) for k in ("x", "y", "q", "active")]
    n = bufs[0].numel()
    ex_s = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
    ey_s = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
    st, msg = _static_call(L, bufs, n, prm_static, ex_s, ey_s, stream)
    assert st == 0, msg
    ex_c = torch.empty(n, dtype=torch.float64, device=dev)
    ey_c = torch.empty(n, dtype=torch.float64, device=dev)
    ctx.field2d_device(*bufs, ex_c, ey_c, prm_ctx)
    ctx.sync()
    err = rel_l2((ex_s.cpu().numpy(), ey_s.cpu().numpy()), (ex_c.cpu().numpy(), ey_c.cpu().numpy()))
    assert err <= tol, err


def test_static_entry_matches_context_entry(env):
    from lsmps_vpm_v2_b200 import default_params, workloads
    prm = default_params()
    # two calls in a row, different inputs
    for d in (workloads.lamb_oseen_2d(n_side=64, seed=1), workloads.lamb_oseen_2d(n_side=88, seed=2)):
        _compare(env, d, prm, prm, TOL_FP64)


def test_static_entry_mixed(env):
    """Both mixed settings run the FP32 near field with the FP64 M2L; the context
    entry point's VPM_PREC_MIXED_FP64_M2L is the same form."""
    from lsmps_vpm_v2_b200 import default_params, workloads
    ref = default_params(precision=VPM_PREC_MIXED_FP64_M2L, binom=1)
    for prec, seed in ((VPM_PREC_MIXED, 3), (VPM_PREC_MIXED_FP64_M2L, 4)):
        prm = default_params(precision=prec, binom=1)
        _compare(env, workloads.lamb_oseen_2d(n_side=80, seed=seed), prm, ref, TOL_MIXED)


def test_static_entry_limits(env):
    torch, L, dev, stream, ctx = env
    from lsmps_vpm_v2_b200 import default_params, workloads
    prm = default_params()
    # beyond the stated maximum: rejected with a clear error
    big = torch.zeros(8193, dtype=torch.float64, device=dev)
    st, msg = _static_call(L, [big, big, big, torch.zeros(8193, dtype=torch.uint8, device=dev)], 8193, prm,
                           big, big, stream)
    assert st == VPM_EINVAL and "8192" in msg
    # within the particle limit, but one particle per leaf needs more than 8192 cells
    d = workloads.lamb_oseen_2d(n_side=88, seed=5)
    bufs = [torch.from_numpy(np.ascontiguousarray(d[k])).to(dev) for k in ("x", "y", "q", "active")]
    n = bufs[0].numel()
    out = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(2)]
    st, msg = _static_call(L, bufs, n, default_params(max_src=1, max_par=1), *out, stream)
    assert st == VPM_EOVERFLOW and "outgrew" in msg, (st, msg)
    # the array is usable again after the overflow
    _compare(env, workloads.lamb_oseen_2d(n_side=64, seed=6), prm, prm, TOL_FP64)
