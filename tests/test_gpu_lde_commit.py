"""sg_lde_commit: the LDE of a trace and the Merkle commitment to its rows in one
call, against the oracle (root bytes and kept LDE columns, bit-exact).

For w a multiple of 16 the forward transform's last pass (a 2^7-point DFT)
hashes the rows itself and the LDE is never stored: domains of 2^9 .. 2^19 take
the two-pass form, larger ones the three-pass form. Other widths take the
materialised path (LDE, then the leaf kernel)."""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu
P = O.P


def arities_for(n0, a=16):
    ar, n = [], n0
    while n > 1:
        ar.append(a)
        n = (n + a - 1) // a
    return ar


@pytest.mark.parametrize("w,log_n,blowup,shift,label", [
    (16, 6, 8, 1, 0), (32, 10, 8, 7, 3), (64, 9, 8, 7, 0), (16, 12, 4, 5, 9), (16, 16, 16, 7, 0),
    (48, 13, 8, 1, 1),
    # widths the fused pass does not take: materialised LDE, then the leaf kernel
    (5, 8, 8, 7, 0), (64, 3, 8, 1, 2),
])
def test_lde_commit_matches_oracle(ctx, w, log_n, blowup, shift, label):
    rng = np.random.default_rng(w * 100 + log_n)
    tr = rng.integers(0, P, size=(w, 1 << log_n), dtype=np.uint64)
    n0 = (1 << log_n) * blowup
    ar = arities_for(n0, 16 if n0 >= 256 else 2)
    lde = O.lde(tr, blowup, shift)
    want = O.merkle_root(np.ascontiguousarray(lde.T), ar, label)
    assert ctx.lde_commit(tr, blowup, shift, ar, label) == want
    root, cols = ctx.lde_commit(tr, blowup, shift, ar, label, keep_cols=min(w, 3))
    assert root == want
    assert np.array_equal(cols, lde[:min(w, 3)])


def test_lde_commit_device_input_and_opening(sgpu, ctx):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(77)
    tr = rng.integers(0, P, size=(32, 1 << 11), dtype=np.uint64)
    ar = [16, 16, 16, 16]
    d_tr = torch.from_numpy(tr.view(np.int64)).cuda()
    d_col = torch.empty((1, 1 << 14), dtype=torch.int64, device="cuda")
    root, _, tree = ctx.lde_commit(d_tr, 8, 7, ar, 5, keep_cols=1, out=d_col, keep=True)
    torch.cuda.synchronize()
    lde = O.lde(tr, 8, 7)
    assert root == O.merkle_root(np.ascontiguousarray(lde.T), ar, 5)
    assert np.array_equal(d_col.cpu().numpy().view(np.uint64)[0], lde[0])
    root2, tree2 = ctx.merkle_commit(lde, ar, 5, keep=True)
    for idx in (0, 1, 12345, (1 << 14) - 1):
        assert tree.open(idx) == tree2.open(idx)
    tree.free()
    tree2.free()
