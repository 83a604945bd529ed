"""P-256 ECDSA double-chain part of the CPU oracle (test infrastructure only).

The layout (a gadget program) and the trace are restated here with Python
integers; the constraint evaluation, merge and proof go through the C++ oracle
(oracle/p256_air.hpp, oracle/oracle.cpp).

Follows (stark-stir-swarm paths, crates/deep_ali/src/):
  p256_field.rs:6-36            10 limbs of 26 bits, P in tight limbs
  p256_field_air.rs:344-398     fill_add_gadget: limb-wise carry chain, carries 0/1
  p256_field_air.rs:570-610     fill_sub_gadget: a + P - b, carries -1/0/1 as pos/neg bits
  p256_field_air.rs:953-1040    fill_mul_gadget: c = a b mod p (canonical), q = (ab - c)/p,
                                18 carries biased by 2^35 in 36 bits
  p256_field_air.rs:1229-1241   fill_select_gadget
  p256_field_air.rs:1374-1447   fill_freeze_gadget: a - P chain, c = a if it borrowed else a - P
  p256_group_air.rs:302-447,705-869  group double / add programs (cell allocation order)
  p256_scalar_mul_air.rs:74-160  step = double, add (of the base), select on the bit
  p256_ecdsa_double_multirow_air.rs:63-112,134-234  two chains per row, r_proj columns
  p256_group.rs:227-256          the generator G (FIPS 186-4 D.1.2.3)
"""
import ctypes
import hashlib

import numpy as np

import oracle_lib as O

NL, LB = 10, 26
P = 0xFFFFFFFF00000001000000000000000000000000FFFFFFFFFFFFFFFFFFFFFFFF
N = 0xFFFFFFFF00000000FFFFFFFFFFFFFFFFBCE6FAADA7179E84F3B9CAC2FC632551
B = 0x5AC635D8AA3A93E7B3EBBD55769886BC651D06B0CC53B0F63BCE3C3E27D2604B
GX = 0x6B17D1F2E12C4247F8BCE6E563A440F277037D812DEB33A0F4A13945D898C296
GY = 0x4FE342E2FE1A7F9B8EE7EB4A7C0F9E162BCE33576B315ECECBB6406837BF51F5
P_TIGHT = [0x3FFFFFF, 0x3FFFFFF, 0x3FFFFFF, 0x003FFFF, 0, 0, 0, 0x0000400, 0x3FF0000, 0x03FFFFF]
assert sum(l << (LB * i) for i, l in enumerate(P_TIGHT)) == P
ELEM = NL + NL * LB            # 270
MUL_CB, MUL_CP, MUL_SP = 36, 18, 19
MUL_OWNED = 2 * ELEM + MUL_CP * MUL_CB
ADD_OWNED = ELEM + NL
SUB_OWNED = ELEM + 2 * NL
FREEZE_OWNED = 2 * ELEM + 2 * NL
G_MUL, G_ADD, G_SUB, G_FREEZE, G_SELECT = 1, 2, 3, 4, 5
CONSTRAINTS = {G_MUL: 2 * ELEM + MUL_SP + MUL_CP * MUL_CB, G_ADD: ELEM + 2 * NL,
               G_SUB: ELEM + NL + 2 * NL + NL + 1, G_FREEZE: 2 * ELEM + NL + 2 * NL + NL + 1 + NL,
               G_SELECT: ELEM + NL + 1}
BLOWUP = 32


def limbs(x):
    assert 0 <= x < 1 << (NL * LB)
    return [(x >> (LB * i)) & ((1 << LB) - 1) for i in range(NL)]


class Group:
    """One group gadget (double or add): its program in fill order and its
    gadget records grouped in emission order (muls, adds, subs, freezes after
    adds, freezes after subs)."""

    def __init__(self, cursor):
        self.cursor = cursor
        self.b_base = cursor
        self.cursor += ELEM
        self.prog, self.muls, self.adds, self.subs, self.fz_adds, self.fz_subs = [], [], [], [], [], []

    def _take(self, n):
        base = self.cursor
        self.cursor += n
        return base

    def _freeze(self, a):
        d = self._take(FREEZE_OWNED)
        rec = (G_FREEZE, a, d, d + NL, d + ELEM, d + ELEM + NL, d + 2 * ELEM, d + 2 * ELEM + NL)
        return rec

    def mul(self, a, b):
        c = self._take(MUL_OWNED)
        rec = (G_MUL, a, b, c, c + NL, c + ELEM, c + ELEM + NL, c + 2 * ELEM)
        self.muls.append(rec)
        self.prog.append(("mul", rec))
        return c

    def addf(self, a, b):
        c = self._take(ADD_OWNED)
        rec = (G_ADD, a, b, c, c + NL, c + ELEM, 0, 0)
        fz = self._freeze(c)
        self.adds.append(rec)
        self.fz_adds.append(fz)
        self.prog.append(("add", rec, fz))
        return fz[4]

    def subf(self, a, b):
        c = self._take(SUB_OWNED)
        rec = (G_SUB, a, b, c, c + NL, c + ELEM, c + ELEM + NL, 0)
        fz = self._freeze(c)
        self.subs.append(rec)
        self.fz_subs.append(fz)
        self.prog.append(("sub", rec, fz))
        return fz[4]

    def table(self):
        return self.muls + self.adds + self.subs + self.fz_adds + self.fz_subs


def group_double(cursor, x, y, z):
    g = Group(cursor)
    b = g.b_base
    t0 = g.mul(x, x); t1 = g.mul(y, y); t2 = g.mul(z, z); t3 = g.mul(x, y)
    t3 = g.addf(t3, t3)
    z3 = g.mul(x, z); z3 = g.addf(z3, z3)
    y3 = g.mul(b, t2); y3 = g.subf(y3, z3)
    x3 = g.addf(y3, y3); y3 = g.addf(x3, y3)
    x3 = g.subf(t1, y3); y3 = g.addf(t1, y3)
    y3 = g.mul(x3, y3); x3 = g.mul(x3, t3)
    t3 = g.addf(t2, t2); t2 = g.addf(t2, t3)
    z3 = g.mul(b, z3); z3 = g.subf(z3, t2); z3 = g.subf(z3, t0)
    t3 = g.addf(z3, z3); z3 = g.addf(z3, t3)
    t3 = g.addf(t0, t0); t0 = g.addf(t3, t0); t0 = g.subf(t0, t2)
    t0 = g.mul(t0, z3)
    ry = g.addf(y3, t0)
    t0 = g.mul(y, z); t0 = g.addf(t0, t0)
    z3 = g.mul(t0, z3)
    rx = g.subf(x3, z3)
    z3 = g.mul(t0, t1); z3 = g.addf(z3, z3)
    rz = g.addf(z3, z3)
    g.result = (rx, ry, rz)
    return g


def group_add(cursor, px, py, pz, qx, qy, qz):
    g = Group(cursor)
    b = g.b_base
    t0 = g.mul(px, qx); t1 = g.mul(py, qy); t2 = g.mul(pz, qz)
    t3 = g.addf(px, py); t4 = g.addf(qx, qy)
    t3 = g.mul(t3, t4)
    t4 = g.addf(t0, t1); t3 = g.subf(t3, t4)
    t4 = g.addf(py, pz); x3 = g.addf(qy, qz)
    t4 = g.mul(t4, x3)
    x3 = g.addf(t1, t2); t4 = g.subf(t4, x3)
    x3 = g.addf(px, pz); y3 = g.addf(qx, qz)
    x3 = g.mul(x3, y3)
    y3 = g.addf(t0, t2); y3 = g.subf(x3, y3)
    z3 = g.mul(b, t2)
    x3 = g.subf(y3, z3); z3 = g.addf(x3, x3); x3 = g.addf(x3, z3)
    z3 = g.subf(t1, x3); x3 = g.addf(t1, x3)
    y3 = g.mul(b, y3)
    t1 = g.addf(t2, t2); t2 = g.addf(t1, t2)
    y3 = g.subf(y3, t2); y3 = g.subf(y3, t0)
    t1 = g.addf(y3, y3); y3 = g.addf(t1, y3)
    t1 = g.addf(t0, t0); t0 = g.addf(t1, t0); t0 = g.subf(t0, t2)
    t1 = g.mul(t4, y3); t2 = g.mul(t0, y3)
    y3 = g.mul(x3, z3)
    ry = g.addf(y3, t2)
    x3 = g.mul(t3, x3)
    rx = g.subf(x3, t1)
    z3 = g.mul(t4, z3); t1 = g.mul(t3, t0)
    rz = g.addf(z3, t1)
    g.result = (rx, ry, rz)
    return g


class Step:
    def __init__(self, cursor, acc, base, bit):
        self.acc, self.base, self.bit = acc, base, bit
        self.double = group_double(cursor, *acc)
        self.add = group_add(self.double.cursor, *self.double.result, *base)
        c = self.add.cursor
        self.select = []
        for k in range(3):
            self.select.append((G_SELECT, self.add.result[k], self.double.result[k], c, c + NL, bit, 0, 0))
            c += ELEM
        self.cursor = c
        self.out = tuple(s[3] for s in self.select)

    def table(self):
        return self.double.table() + self.add.table() + self.select


class Layout:
    """build_ecdsa_double_multirow_layout(0)."""

    def __init__(self):
        cur = 0
        self.steps = []
        for _ in range(2):
            acc = (cur, cur + NL, cur + 2 * NL)
            base = (cur + 3 * NL, cur + 4 * NL, cur + 5 * NL)
            bit = cur + 6 * NL
            st = Step(bit + 1, acc, base, bit)
            self.steps.append(st)
            cur = st.cursor
        self.r_proj = [cur + NL * k for k in range(6)]
        self.width = cur + 6 * NL
        rows = [r for st in self.steps for r in st.table()]
        self.table = np.array(rows, dtype=np.uint64).reshape(-1, 8)
        tail = []
        for st in self.steps:
            tail += list(st.acc) + list(st.out)
        self.tail = np.array(tail + self.r_proj, dtype=np.uint64)
        self.n_constraints = sum(CONSTRAINTS[int(k)] for k in self.table[:, 0]) + 180


# ---------------------------------------------------------------- trace fill
def _put_limbs(row, base, ls):
    row[base:base + NL] = ls


def _put_elem(row, lb, bb, ls):
    row[lb:lb + NL] = ls
    a = np.array(ls, dtype=np.uint64)
    row[bb:bb + NL * LB] = ((a[:, None] >> np.arange(LB, dtype=np.uint64)) & 1).reshape(-1)


def _fill_mul(row, rec, a, b):
    _, _, _, c_b, cb_b, q_b, qb_b, cy_b = rec
    prod = a * b
    c, q = prod % P, prod // P
    al, bl, cl, ql = limbs(a), limbs(b), limbs(c), limbs(q)
    carries = []
    prev = 0
    for k in range(MUL_SP):
        lo, hi = max(0, k - (NL - 1)), min(NL - 1, k)
        pab = sum(al[i] * bl[k - i] for i in range(lo, hi + 1))
        pqp = sum(ql[i] * P_TIGHT[k - i] for i in range(lo, hi + 1))
        lhs = pab - pqp - (cl[k] if k < NL else 0) + prev
        if k < MUL_SP - 1:
            assert lhs % (1 << LB) == 0
            prev = lhs >> LB
            assert abs(prev) < 1 << (MUL_CB - 1)
            carries.append(prev)
        else:
            assert lhs == 0
    _put_elem(row, c_b, cb_b, cl)
    _put_elem(row, q_b, qb_b, ql)
    biased = np.array([x + (1 << (MUL_CB - 1)) for x in carries], dtype=np.uint64)
    row[cy_b:cy_b + MUL_CP * MUL_CB] = ((biased[:, None] >> np.arange(MUL_CB, dtype=np.uint64)) & 1).reshape(-1)
    return c


def _fill_chain(row, lb, bb, al, bl, sign_p, rbase_or_carries):
    """limb chain of a + sign_p * P (+ or -) - ... : shared by add (b added), sub, freeze."""
    raise NotImplementedError


def _fill_add(row, rec, a, b):
    _, _, _, c_b, cb_b, cr_b, _, _ = rec
    al, bl = limbs(a), limbs(b)
    cl, carries, prev = [], [], 0
    for k in range(NL):
        s = al[k] + bl[k] + prev
        cl.append(s & ((1 << LB) - 1))
        prev = s >> LB
        assert prev in (0, 1)
        carries.append(prev)
    assert carries[-1] == 0
    _put_elem(row, c_b, cb_b, cl)
    row[cr_b:cr_b + NL] = carries
    return a + b


def _signed_chain(al, bl, sign):
    """a + sign * P_TIGHT - b, limb by limb with floor division (rem_euclid / div_euclid)."""
    out, carries, prev = [], [], 0
    for k in range(NL):
        lhs = al[k] + sign * P_TIGHT[k] - bl[k] + prev
        out.append(lhs % (1 << LB))
        prev = lhs // (1 << LB)
        assert abs(prev) <= 1
        carries.append(prev)
    return out, carries


def _put_posneg(row, pos_b, neg_b, carries):
    row[pos_b:pos_b + NL] = [1 if c == 1 else 0 for c in carries]
    row[neg_b:neg_b + NL] = [1 if c == -1 else 0 for c in carries]


def _fill_sub(row, rec, a, b):
    _, _, _, c_b, cb_b, pos_b, neg_b, _ = rec
    cl, carries = _signed_chain(limbs(a), limbs(b), 1)
    assert carries[-1] == 0
    _put_elem(row, c_b, cb_b, cl)
    _put_posneg(row, pos_b, neg_b, carries)
    return a + P - b


def _fill_freeze(row, rec, raw):
    _, _, d_b, db_b, c_b, cb_b, pos_b, neg_b = rec
    al = limbs(raw)
    dl, carries = _signed_chain(al, [0] * NL, -1)
    assert carries[-1] in (0, -1)
    cl = al if carries[-1] == -1 else dl
    _put_elem(row, d_b, db_b, dl)
    _put_elem(row, c_b, cb_b, cl)
    _put_posneg(row, pos_b, neg_b, carries)
    out = sum(l << (LB * i) for i, l in enumerate(cl))
    assert out < P
    return out


def _run_group(row, g, vals):
    """Fill a group gadget: vals maps cell base -> canonical value of its inputs."""
    _put_elem(row, g.b_base, g.b_base + NL, limbs(B))
    vals[g.b_base] = B
    for op in g.prog:
        if op[0] == "mul":
            rec = op[1]
            vals[rec[3]] = _fill_mul(row, rec, vals[rec[1]], vals[rec[2]])
        else:
            rec, fz = op[1], op[2]
            f = _fill_add if op[0] == "add" else _fill_sub
            raw = f(row, rec, vals[rec[1]], vals[rec[2]])
            vals[fz[4]] = _fill_freeze(row, fz, raw)


def _run_step(row, st, acc, base, bit):
    vals = {}
    for k in range(3):
        _put_limbs(row, st.acc[k], limbs(acc[k]))
        _put_limbs(row, st.base[k], limbs(base[k]))
        vals[st.acc[k]] = acc[k]
        vals[st.base[k]] = base[k]
    row[st.bit] = int(bit)
    _run_group(row, st.double, vals)
    _run_group(row, st.add, vals)
    out = []
    for rec in st.select:
        chosen = vals[rec[1]] if bit else vals[rec[2]]
        _put_elem(row, rec[3], rec[4], limbs(chosen))
        out.append(chosen)
    return tuple(out)


def chain_outputs(a_base, a_bits, b_base, b_bits):
    """The two chains' final projective points (the r_proj values), by running them."""
    lay = Layout()
    row = np.zeros(lay.width, dtype=np.uint64)
    acc_a, acc_b = a_base, b_base
    for r in range(len(a_bits)):
        acc_a = _run_step(row, lay.steps[0], acc_a, a_base, a_bits[r])
        acc_b = _run_step(row, lay.steps[1], acc_b, b_base, b_bits[r])
    return acc_a, acc_b


def trace(a_point, a_bits, b_point, b_bits, r_proj=None, lay=None):
    """fill_ecdsa_double_multirow with chains starting at (x, y, 1) of the two affine
    points, one bit per row (n_trace = len(bits)); r_proj defaults to the chains'
    outputs. Returns ((width, n_trace) uint64, layout)."""
    lay = lay or Layout()
    n_trace = len(a_bits)
    assert len(b_bits) == n_trace and n_trace & (n_trace - 1) == 0
    a_base = (a_point[0], a_point[1], 1)
    b_base = (b_point[0], b_point[1], 1)
    if r_proj is None:
        ra, rb = chain_outputs(a_base, a_bits, b_base, b_bits)
        r_proj = list(ra) + list(rb)
    tr = np.zeros((lay.width, n_trace), dtype=np.uint64)
    acc_a, acc_b = a_base, b_base
    row = np.zeros(lay.width, dtype=np.uint64)
    for r in range(n_trace):
        row[:] = 0
        acc_a = _run_step(row, lay.steps[0], acc_a, a_base, a_bits[r])
        acc_b = _run_step(row, lay.steps[1], acc_b, b_base, b_bits[r])
        for k in range(6):
            _put_limbs(row, lay.r_proj[k], limbs(r_proj[k]))
        tr[:, r] = row
    return tr, lay


# ---------------------------------------------------------------- ECDSA
def _affine_add(p1, p2):
    if p1 is None:
        return p2
    if p2 is None:
        return p1
    (x1, y1), (x2, y2) = p1, p2
    if x1 == x2 and (y1 + y2) % P == 0:
        return None
    if p1 == p2:
        lam = (3 * x1 * x1 - 3) * pow(2 * y1, -1, P) % P
    else:
        lam = (y2 - y1) * pow(x2 - x1, -1, P) % P
    x3 = (lam * lam - x1 - x2) % P
    return x3, (lam * (x1 - x3) - y1) % P


def scalar_mul(k, pt):
    acc = None
    for bit in bin(k)[2:]:
        acc = _affine_add(acc, acc)
        if bit == "1":
            acc = _affine_add(acc, pt)
    return acc


G = (GX, GY)


def keypair(d):
    return d, scalar_mul(d, G)


def sign(digest: bytes, d: int, k: int):
    e = int.from_bytes(digest, "big") % N
    r = scalar_mul(k, G)[0] % N
    s = pow(k, -1, N) * (e + r * d) % N
    assert r and s
    return r, s


def u_bits(digest: bytes, r: int, s: int):
    """u1 = e s^-1, u2 = r s^-1 mod n as MSB-first 256-bit lists (prove_ecdsa_record_v1.rs:97-118)."""
    e = int.from_bytes(digest, "big") % N
    w = pow(s, -1, N)
    u1, u2 = e * w % N, r * w % N
    return [(u1 >> (255 - i)) & 1 for i in range(256)], [(u2 >> (255 - i)) & 1 for i in range(256)]


def pi_hash(qx, qy, r, s, digest: bytes) -> bytes:
    """prove_ecdsa_record_v1.rs:213-222: SHA3("ECDSA-V1-PI-PRE" || qx || qy || r || s || digest)."""
    h = hashlib.sha3_256(b"ECDSA-V1-PI-PRE")
    for v in (qx, qy, r, s):
        h.update(v.to_bytes(32, "big"))
    h.update(digest)
    return h.digest()


# ---------------------------------------------------------------- C++ oracle
def _lib():
    L = O.lib()
    if not getattr(L, "_p256_bound", False):
        sz = ctypes.c_size_t
        L.orc_p256_eval.argtypes = [O.U64P, O.U64P, sz, sz, O.U64P, sz, O.U64P, O.U64P]
        L.orc_merge_p256.argtypes = [O.U64P, sz, O.U64P, sz, O.U64P, sz, sz, O.U64P]
        L.orc_prove_p256.argtypes = [O.U64P, sz, O.U64P, sz, O.U64P, sz, ctypes.c_char_p, sz, ctypes.c_char_p, sz,
                                     ctypes.POINTER(sz)]
        L._p256_bound = True
    return L


def eval_row(lay, cur, nxt, row, n_trace):
    cur = np.ascontiguousarray(cur, dtype=np.uint64)
    nxt = np.ascontiguousarray(nxt, dtype=np.uint64)
    out = np.zeros(lay.n_constraints, dtype=np.uint64)
    tab = np.ascontiguousarray(lay.table)
    n = _lib().orc_p256_eval(O._ptr(cur), O._ptr(nxt), row, n_trace, O._ptr(tab), tab.shape[0],
                             O._ptr(lay.tail), O._ptr(out))
    assert n == lay.n_constraints, n
    return out


def merge(lay, lde_cols, n_trace, blowup=BLOWUP):
    lde_cols = np.ascontiguousarray(lde_cols, dtype=np.uint64)
    out = np.zeros(n_trace * blowup, dtype=np.uint64)
    tab = np.ascontiguousarray(lay.table)
    rc = _lib().orc_merge_p256(O._ptr(lde_cols), lay.width, O._ptr(tab), tab.shape[0], O._ptr(lay.tail), n_trace,
                               blowup, O._ptr(out))
    assert rc == 0, rc
    return out


def prove(lay, tr, pi: bytes, blowup: int = BLOWUP) -> bytes:
    tr = np.ascontiguousarray(tr, dtype=np.uint64)
    tab = np.ascontiguousarray(lay.table)
    cap = 1 << 24
    buf = ctypes.create_string_buffer(cap)
    ln = ctypes.c_size_t()
    rc = _lib().orc_prove_p256(O._ptr(tr), lay.width, O._ptr(tab), tab.shape[0], O._ptr(lay.tail), tr.shape[1], pi,
                               blowup, buf, cap, ctypes.byref(ln))
    assert rc == 0, rc
    return buf.raw[:ln.value]
