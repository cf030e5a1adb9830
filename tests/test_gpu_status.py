"""Device status word: a bounded wait that runs out is reported on the host.

Every wait of the pipelined kernels (mbarriers, the radix sort's look-back) gives up
after a bounded spin and records a status bit instead of hanging.  Here one block waits
on a barrier that nothing completes (a flag nothing sets); the wait ends after about
0.1 s, the kernel returns, and gvc_sync_status reports GVC_ERR_TIMEOUT once, then the
word is clear and the context keeps working."""
import ctypes

import numpy as np
import pytest
import torch

import gvc_native

pytestmark = pytest.mark.gpu


def test_bounded_wait_timeout_is_reported(cuda):
    ctx = gvc_native.Context()
    stream = torch.cuda.current_stream().cuda_stream
    ctx.sync_status(stream)  # clear
    ctx.call("gvc_debug_wait_timeout", ctypes.c_void_p(stream))
    with pytest.raises(gvc_native.GvcError) as ei:
        ctx.sync_status(stream)
    assert ei.value.code == gvc_native.GVC_ERR_TIMEOUT
    assert "bounded device-side wait" in str(ei.value)
    # the report cleared the word, and the device context still runs kernels
    ctx.sync_status(stream)
    A = torch.ones(128, 16, dtype=torch.bfloat16, device=cuda)
    B = torch.ones(32, 16, dtype=torch.bfloat16, device=cuda)
    D = torch.empty(128 * 32, device=cuda)
    ctx.call("gvc_debug_tc_gemm", gvc_native.ptr(A), gvc_native.ptr(B), 32, gvc_native.ptr(D),
             ctypes.c_void_p(stream))
    ctx.sync_status(stream)
    np.testing.assert_array_equal(D.cpu().numpy(), np.full(128 * 32, 16.0, np.float32))
