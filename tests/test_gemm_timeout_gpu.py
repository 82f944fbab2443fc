"""The tensor-core GEMM's bounded waits: a wait that runs out is reported as
GTP_ETIMEOUT and leaves the device usable.

gtp_bf16_gemm_checked takes the pipeline's wait limit and a test hook that
makes the first CTA's TMA producer skip one K block's loads: the bytes the
MMA issuer waits for never arrive (a barrier nothing completes), its wait
gives up after the short limit, the kernel lets its other copies and MMAs
finish, frees its TMEM and returns with the error bit set. The same process
then runs the GEMM again, correctly. The skipped block is the last K block
of the first CTA's only tile, so no copy is issued after it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# about 10 ms at the B200's SM clock: far above any healthy wait here
SHORT_LIMIT = 20_000_000


def _gemm(a, b, skip=-1, limit=SHORT_LIMIT):
    import ctypes as C
    import torch
    from gtpower_b200 import _abi
    m, k = a.shape
    n = b.shape[0]
    c = torch.full((m, n), float("nan"), dtype=torch.float32, device=a.device)
    err = torch.zeros(1, dtype=torch.int32, device=a.device)
    st = _abi.lib().gtp_bf16_gemm_checked(a.data_ptr(), k, b.data_ptr(), k, m, n, k, None, 0,
                                          c.data_ptr(), n, limit, skip, err.data_ptr(), None)
    return st, c, int(err.item())


def test_gemm_wait_runs_out_then_next_call_is_correct():
    import torch
    from gtpower_b200 import _abi
    g = torch.Generator(device="cuda").manual_seed(5)
    # 2 row tiles x 1 column tile: two CTAs, one tile each; K = 256 is four
    # K blocks, and CTA 0 skips its last (index 3)
    a = torch.randn(256, 256, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(128, 256, device="cuda", generator=g).to(torch.bfloat16)
    ref = a.float() @ b.float().T
    st, _, err = _gemm(a, b, skip=3)
    assert st == _abi.GTP_ETIMEOUT
    assert err != 0
    for _ in range(2):
        st, c, err = _gemm(a, b)
        assert st == _abi.GTP_OK and err == 0
        diff = (c - ref).abs().max().item()
        assert diff <= 1e-4 * ref.abs().max().item() + 1e-6, diff


def test_gemm_short_limit_does_not_fire_on_healthy_pipeline():
    import torch
    from gtpower_b200 import _abi
    g = torch.Generator(device="cuda").manual_seed(6)
    a = torch.randn(4096, 512, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(512, 512, device="cuda", generator=g).to(torch.bfloat16)
    st, c, err = _gemm(a, b)
    assert st == _abi.GTP_OK and err == 0
    ref = a.float() @ b.float().T
    assert (c - ref).abs().max().item() <= 1e-4 * ref.abs().max().item() + 1e-6


def test_gemm_checked_rejects_bad_arguments():
    import torch
    from gtpower_b200 import _abi
    a = torch.zeros(128, 64, dtype=torch.bfloat16, device="cuda")
    b = torch.zeros(128, 64, dtype=torch.bfloat16, device="cuda")
    st, _, _ = _gemm(a, b, skip=-2)
    assert st == _abi.GTP_EINVAL
