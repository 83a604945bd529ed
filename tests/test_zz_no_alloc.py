"""sg_ntt_noalloc: the NTT entry point for callers that must not have this
library allocate device memory (its buffers come from file-scope static
device arrays). Checked through the C ABI against sg_ntt, the allocating entry
point, on two calls in a row -- the second call reuses the static scratch the
first one left behind -- and against the oracle's transform in both directions.
Results are exact field elements, so the tolerance is zero. This file is named
to be collected last."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P = 0xFFFFFFFF00000001


def _rand(torch, cols, log_n, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return torch.randint(0, 1 << 62, (cols, 1 << log_n), dtype=torch.int64, device="cuda", generator=g)


@pytest.mark.parametrize("cols,log_n", [(1, 13), (4, 16), (1, 20), (16, 16), (3, 10), (2, 1), (1, 12)])
@pytest.mark.parametrize("inverse", [0, 1])
def test_noalloc_ntt_matches_allocating_entry_point(sgpu, ctx, cols, log_n, inverse):
    torch = pytest.importorskip("torch")
    L = sgpu.lib()
    x = _rand(torch, cols, log_n, 1000 * cols + log_n)
    want = torch.empty_like(x)
    ctx.ntt(x, log_n, bool(inverse), out=want)  # sg_ntt (allocates its scratch from the pool)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        out = torch.full_like(x, -1)
        rc = L.sg_ntt_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), cols, log_n, inverse,
                              ctypes.c_void_p(stream))
        assert rc == sgpu.SG_OK, rc
        torch.cuda.synchronize()
        assert torch.equal(out, want), f"call {call}"


@pytest.mark.parametrize("cols,log_n", [(2, 16), (1, 20), (3, 11)])
@pytest.mark.parametrize("inverse", [0, 1])
def test_noalloc_ntt_matches_oracle(sgpu, cols, log_n, inverse):
    # each column against the oracle's transform (ark-poly radix-2 domain semantics)
    import oracle_lib as O
    torch = pytest.importorskip("torch")
    L = sgpu.lib()
    x = _rand(torch, cols, log_n, 77 + 10 * cols + log_n)
    out = torch.full_like(x, -1)
    rc = L.sg_ntt_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), cols, log_n, inverse,
                          ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == sgpu.SG_OK, rc
    torch.cuda.synchronize()
    xh = x.cpu().numpy().view(np.uint64)
    got = out.cpu().numpy().view(np.uint64)
    for c in range(cols):
        assert np.array_equal(got[c], O.ntt(xh[c], bool(inverse))), c


def test_noalloc_ntt_in_place_round_trip(sgpu):
    torch = pytest.importorskip("torch")
    L = sgpu.lib()
    x = _rand(torch, 2, 18, 7)
    y = x.clone()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.sg_ntt_noalloc(ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(y.data_ptr()), 2, 18, 0, stream) == 0
    assert L.sg_ntt_noalloc(ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(y.data_ptr()), 2, 18, 1, stream) == 0
    torch.cuda.synchronize()
    assert torch.equal(x, y)


def test_noalloc_ntt_rejects_oversize_and_host_buffers(sgpu):
    torch = pytest.importorskip("torch")
    L = sgpu.lib()
    # the buffer holds 2^21 elements, so the shapes below stay in bounds even
    # though the entry point must refuse them before launching anything
    x = _rand(torch, 1, 21, 3)
    ptr = ctypes.c_void_p(x.data_ptr())
    # 2^21 elements on a two-pass transform: larger than the static scratch
    assert L.sg_ntt_noalloc(ptr, ptr, 1, 21, 0, None) == sgpu.SG_ELIMIT
    assert L.sg_ntt_noalloc(ptr, ptr, 256, 13, 0, None) == sgpu.SG_ELIMIT
    host = np.zeros(1 << 13, dtype=np.uint64)
    hp = ctypes.c_void_p(host.ctypes.data)
    assert L.sg_ntt_noalloc(hp, hp, 1, 13, 0, None) == sgpu.SG_EINVAL
    assert L.sg_ntt_noalloc(ptr, ptr, 0, 13, 0, None) == sgpu.SG_EINVAL
    # 2^25 is a valid transform size but needs more scratch than the static buffer;
    # 2^29 is beyond the largest supported domain (2^28)
    assert L.sg_ntt_noalloc(ptr, ptr, 1, 25, 0, None) == sgpu.SG_ELIMIT
    assert L.sg_ntt_noalloc(ptr, ptr, 1, 29, 0, None) == sgpu.SG_EINVAL


@pytest.mark.parametrize("cols,log_n", [(3, 14), (1, 9)])
def test_noalloc_python_wrapper_matches_context_and_oracle(sgpu, ctx, cols, log_n):
    # the package's wrapper on a (cols, 2^log_n) tensor: it derives n_cols from the
    # tensor, and its result equals the context's sg_ntt and the oracle's transform
    torch = pytest.importorskip("torch")
    import oracle_lib as O
    rng = np.random.default_rng(50 + log_n)
    host = rng.integers(0, P, size=(cols, 1 << log_n), dtype=np.uint64)
    x = torch.from_numpy(host.view(np.int64)).cuda()
    want = torch.empty_like(x)
    ctx.ntt(x, log_n, False, out=want)
    for call in range(2):
        out = torch.full_like(x, -1)
        assert sgpu.ntt_noalloc(x, out, log_n) == sgpu.SG_OK
        torch.cuda.synchronize()
        assert torch.equal(out, want), f"call {call}"
    got = out.cpu().numpy().view(np.uint64)
    for c in range(cols):
        assert np.array_equal(got[c], O.ntt(host[c])), c
    # raw device pointers with an explicit column count
    out2 = torch.full_like(x, -1)
    assert sgpu.ntt_noalloc(x.data_ptr(), out2.data_ptr(), log_n, n_cols=cols) == sgpu.SG_OK
    torch.cuda.synchronize()
    assert torch.equal(out2, want)
