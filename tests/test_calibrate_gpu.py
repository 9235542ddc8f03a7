"""The L2 atomic-add calibration kernel behind the scatter's roofline.

``fis_red_rate`` adds 1 at pseudo-random words of a buffer; every add must
land inside the buffer, so the buffer's sum is the number of adds, and its
argument checks refuse sizes it cannot address.
"""

import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu


def test_red_rate_adds_every_unit_inside_the_buffer():
    import fis._lib as L

    lib = L.load()
    words, iters, ctas = 1 << 20, 64, 37
    buf = torch.zeros(words + 64, dtype=torch.int32, device="cuda")  # 64 guard words
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.fis_red_rate(ctypes.c_void_p(buf.data_ptr()), words, iters, ctas, st) == 0
    torch.cuda.synchronize()
    assert int(buf[:words].sum()) == ctas * 256 * iters
    assert int(buf[words:].abs().sum()) == 0
    assert int((buf[:words] > 0).sum()) > ctas * 256 * iters // 2  # spread over the buffer
    for bad in ((0, iters, ctas), (words, 12, ctas), (words, iters, 0)):
        assert lib.fis_red_rate(ctypes.c_void_p(buf.data_ptr()), *bad, st) == -1
