"""The P-256 ECDSA double-chain oracle against the properties the reference's
tests assert (deep_ali/src/p256_ecdsa_double_multirow_air.rs tests
double_multirow_k4_all_zero and double_multirow_wrong_rproj_violates_boundary,
p256_field_air.rs / p256_group_air.rs gadget tests), plus an algebraic check
that the gadget programs compute the group law: each chain ends at
(2^K + u) times its base point."""
import hashlib
import random

import numpy as np

import oracle_p256 as E

Q2 = E._affine_add(E.G, E.G)


def _nonzero(lay, tr, rows=None):
    n = tr.shape[1]
    total = 0
    for r in (range(n) if rows is None else rows):
        total += int(np.count_nonzero(E.eval_row(lay, tr[:, r], tr[:, (r + 1) % n], r, n)))
    return total


def _affine(xyz):
    x, y, z = xyz
    zi = pow(z, -1, E.P)
    return x * zi % E.P, y * zi % E.P


def test_layout_counts():
    lay = E.Layout()
    assert lay.width == 151334 and lay.n_constraints == 155774
    assert lay.table.shape == (260, 8)
    # 75,637 cells per chain (p256_ecdsa_double_multirow_air.rs:14) plus the r_proj columns
    assert lay.r_proj[0] == 2 * 75637
    kinds, counts = np.unique(lay.table[:, 0], return_counts=True)
    assert dict(zip(kinds.tolist(), counts.tolist())) == {1: 54, 2: 70, 3: 30, 4: 100, 5: 6}


def test_k4_all_zero():
    lay = E.Layout()
    tr, _ = E.trace(E.G, [1, 0, 1, 0], Q2, [0, 1, 1, 0], lay=lay)
    assert _nonzero(lay, tr) == 0


def test_wrong_rproj_violates_boundary():
    lay = E.Layout()
    a_bits, b_bits = [1, 0, 1, 0], [0, 1, 1, 0]
    ra, rb = E.chain_outputs((E.GX, E.GY, 1), a_bits, (Q2[0], Q2[1], 1), b_bits)
    bogus = list(ra) + list(rb)
    bogus[0] = (bogus[0] + 1) % E.P
    tr, _ = E.trace(E.G, a_bits, Q2, b_bits, r_proj=bogus, lay=lay)
    cv = E.eval_row(lay, tr[:, 3], tr[:, 0], 3, 4)
    assert np.count_nonzero(cv[-180:-120]) >= 1
    assert _nonzero(lay, tr, rows=[0, 1, 2]) == 0


def test_chains_compute_the_group_law():
    rng = random.Random(7)
    for k in (4, 8):
        a_bits = [rng.randrange(2) for _ in range(k)]
        b_bits = [rng.randrange(2) for _ in range(k)]
        ra, rb = E.chain_outputs((E.GX, E.GY, 1), a_bits, (Q2[0], Q2[1], 1), b_bits)
        ua = int("".join(map(str, a_bits)), 2)
        ub = int("".join(map(str, b_bits)), 2)
        assert _affine(ra) == E.scalar_mul((1 << k) + ua, E.G)
        assert _affine(rb) == E.scalar_mul((1 << k) + ub, Q2)


def test_tampered_mul_output_violates():
    lay = E.Layout()
    tr, _ = E.trace(E.G, [1, 1, 0, 1], Q2, [0, 0, 1, 1], lay=lay)
    c = int(lay.table[0, 3])  # first mul gadget's c limb 0
    tr[c, 2] = (int(tr[c, 2]) + 1) % (2 ** 64 - 2 ** 32 + 1)
    assert _nonzero(lay, tr, rows=[2]) > 0


def test_ecdsa_scalars_verify():
    d, q = E.keypair(0xC0FFEE)
    digest = hashlib.sha256(b"DNSSEC-RRSIG-V0|example.com.|A|192.0.2.1").digest()
    r, s = E.sign(digest, d, 0x1234567)
    u1, u2 = E.u_bits(digest, r, s)
    a = int("".join(map(str, u1)), 2)
    b = int("".join(map(str, u2)), 2)
    R = E._affine_add(E.scalar_mul(a, E.G), E.scalar_mul(b, q))
    assert R[0] % E.N == r
