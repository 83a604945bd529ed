"""Ed25519 verify AIR (v16) part of the CPU oracle (test infrastructure only).

The layout, the constraint program (the blocks of the constraint vector in the
reference's emission order, each with its row gate) and the trace are restated
here with Python integers; the constraint evaluation, merge and proof go
through the C++ oracle (oracle/ed25519_air.hpp, oracle/oracle.cpp). Signing
(RFC 8032 section 5.1.6) is here only to make test inputs.

Follows (stark-stir-swarm paths, crates/deep_ali/src/):
  ed25519_field.rs:103-116        10 limbs, widths 26/25, offsets
  ed25519_field_air.rs:330-418    fill_add_gadget: carries 0/1, carry_in[0] = 19 carry[9]
  ed25519_field_air.rs:584-668    fill_sub_gadget: signed carries as pos/neg cells
  ed25519_field_air.rs:847-996    fill_mul_gadget: 19-folded schoolbook, carries biased by 2^35
  ed25519_field_air.rs:1441-1455  fill_select_gadget
  ed25519_group.rs:101-165        HWCD add and double (the native values the trace holds)
  ed25519_group.rs:204-232        decompress; ed25519_field.rs:527-557 sqrt_ratio_i
  ed25519_group_air.rs:202-321    point-add cell allocation and fill
  ed25519_group_air.rs:476-546    point-double allocation and fill
  ed25519_group_air.rs:662-752    conditional add (point add + 4 selects)
  ed25519_group_air.rs:887-1029   point-decompress allocation and fill
  ed25519_scalar_air.rs:99-372    scalar reduction mod L: q, r, slack, 33 biased carries
  ed25519_scalar_mult_air.rs:93-171  ladder row layout and fill
  ed25519_verify_air.rs:162-4960  the v0..v16 compositions: rows, cells and constraint blocks
  swarm-dns/src/prover.rs:829-839,856-951  s_bits_for_ladder, prove_zsk_ksk_binding_v2
"""
import ctypes
import hashlib

import numpy as np

import oracle_lib as O

P = 2 ** 255 - 19
L_ORDER = 2 ** 252 + 27742317777372353535851937790883648493
D_INT = (-121665 * pow(121666, P - 2, P)) % P
SQRT_M1 = pow(2, (P - 1) // 4, P)
NL = 10
LW = [26, 25] * 5
LOFF = [0, 26, 51, 77, 102, 128, 153, 179, 204, 230]
MUL_CB = 36
RED_LIMBS_IN, RED_R, RED_Q, RED_LB, RED_CB = 32, 16, 17, 16, 24
RED_PROD = RED_Q + RED_R
SHA512_WIDTH, SHA512_K, SHA512_H0_LO = O.SHA512_WIDTH, O.SHA512_K, O.SHA512_H0_LO
BLOWUP = 32

ELEM = NL + 255
ADD_OWNED, SUB_OWNED, MUL_OWNED = ELEM + NL, ELEM + 2 * NL, ELEM + MUL_CB * NL
ADD_K, SUB_K, MUL_K, SEL_K, RANGE_K = ELEM + 2 * NL, ELEM + 4 * NL, ELEM + NL + MUL_CB * NL, 1 + NL, ELEM
PA_K = NL + 4 * SUB_K + 5 * ADD_K + 9 * MUL_K          # 8370
DBL_K = 8 * MUL_K + 4 * ADD_K + 2 * SUB_K              # 6830
DECOMP_K = NL + ELEM + 4 * MUL_K + 3 * SUB_K + NL + 2  # 3742
REDUCE_K = (RED_Q * RED_LB + RED_Q + 2 * (RED_R * RED_LB + RED_R) + RED_R + RED_PROD + RED_PROD * RED_CB)
FORMAT_K = 512 + 16 + 32

# C++ oracle record kinds (oracle/ed25519_air.hpp)
GATE_ALWAYS, GATE_EQ, GATE_RANGE, GATE_SET = 0, 1, 2, 3
B_SHA512, B_REDUCE, B_FORMAT, B_MUL, B_ADD, B_SUB, B_SEL, B_RANGE, B_SIGN, B_PAIRS = range(1, 11)
REC = 16
SRC_CUR, SRC_NXT, SRC_CONST = 0, 1, 2
NONE = (1 << 64) - 1


# ---------------------------------------------------------------- field and curve
def limbs(x):
    """tight 26/25-bit limbs of x in [0, 2^255)"""
    assert 0 <= x < 1 << 255
    return [(x >> LOFF[i]) & ((1 << LW[i]) - 1) for i in range(NL)]


def value(ls):
    return sum(int(l) << LOFF[i] for i, l in enumerate(ls))


D_LIMBS = limbs(D_INT)
D2_LOOSE = [2 * l for l in D_LIMBS]  # ed25519_field.rs:609: D2 = D.add(&D), limb-wise, never reduced
ONE_LIMBS = limbs(1)


def inv(x):
    return pow(x, P - 2, P)


def pt_add(p1, p2):
    """EdwardsPoint::add (ed25519_group.rs:101-126), values mod p"""
    X1, Y1, Z1, T1 = p1
    X2, Y2, Z2, T2 = p2
    a = (Y1 - X1) * (Y2 - X2) % P
    b = (Y1 + X1) * (Y2 + X2) % P
    c = T1 * T2 % P * (2 * D_INT) % P
    d = 2 * Z1 * Z2 % P
    e, f, g, h = (b - a) % P, (d - c) % P, (d + c) % P, (b + a) % P
    return (e * f % P, g * h % P, f * g % P, e * h % P)


def pt_double(p1):
    """EdwardsPoint::double (ed25519_group.rs:147-165)"""
    X1, Y1, Z1, _ = p1
    a, b = X1 * X1 % P, Y1 * Y1 % P
    c = 2 * Z1 * Z1 % P
    h = (a + b) % P
    e = (h - (X1 + Y1) ** 2) % P
    g = (a - b) % P
    f = (c + g) % P
    return (e * f % P, g * h % P, f * g % P, e * h % P)


IDENTITY = (0, 1, 1, 0)


def pt_neg(p1):
    return ((-p1[0]) % P, p1[1], p1[2], (-p1[3]) % P)


def ladder(base, bits):
    """MSB-first double-and-add from the identity (ed25519_verify_air.rs:4830-4836)"""
    acc = IDENTITY
    for b in bits:
        acc = pt_double(acc)
        if b:
            acc = pt_add(acc, base)
    return acc


def affine(p1):
    zi = inv(p1[2])
    return p1[0] * zi % P, p1[1] * zi % P


def split_compressed(b32: bytes):
    """(y, sign) of a 32-byte encoding (ed25519_verify_air.rs:642-648); y keeps the non-canonical case"""
    sign = b32[31] >> 7
    y = int.from_bytes(b32, "little") & ((1 << 255) - 1)
    return y, sign


def decompress(b32: bytes):
    """EdwardsPoint::decompress: x^2 = (y^2 - 1)/(d y^2 + 1), the root whose parity is the sign bit;
    None when (y^2 - 1)/(d y^2 + 1) is not a square. Non-canonical y (>= p) is refused here."""
    y, sign = split_compressed(b32)
    if y >= P:
        return None
    u = (y * y - 1) % P
    v = (D_INT * y * y + 1) % P
    x2 = u * inv(v) % P
    x = pow(x2, (P + 3) // 8, P)
    if x * x % P != x2:
        x = x * SQRT_M1 % P
    if x * x % P != x2:
        return None
    if x & 1 != sign:
        x = (-x) % P
    return (x, y, 1, x * y % P)


def compress(p1) -> bytes:
    x, y = affine(p1)
    return (y | ((x & 1) << 255)).to_bytes(32, "little")


BASE_COMPRESSED = bytes([0x58] + [0x66] * 31)
BASEPOINT = decompress(BASE_COMPRESSED)


def _scalar_mul_int(k, pt):
    acc = IDENTITY
    for i in range(k.bit_length() - 1, -1, -1):
        acc = pt_double(acc)
        if (k >> i) & 1:
            acc = pt_add(acc, pt)
    return acc


def keypair(seed: bytes):
    """RFC 8032 section 5.1.5: (secret scalar a, prefix, 32-byte public key)"""
    h = hashlib.sha512(seed).digest()
    a = int.from_bytes(h[:32], "little")
    a &= (1 << 254) - 8
    a |= 1 << 254
    return a, h[32:], compress(_scalar_mul_int(a, BASEPOINT))


def sign(seed: bytes, msg: bytes) -> bytes:
    """RFC 8032 section 5.1.6"""
    a, prefix, pub = keypair(seed)
    r = int.from_bytes(hashlib.sha512(prefix + msg).digest(), "little") % L_ORDER
    R = compress(_scalar_mul_int(r, BASEPOINT))
    k = int.from_bytes(hashlib.sha512(R + pub + msg).digest(), "little") % L_ORDER
    s = (r + k * a) % L_ORDER
    return R + s.to_bytes(32, "little")


def verify(pub: bytes, sig: bytes, msg: bytes) -> bool:
    """RFC 8032 section 5.1.7, cofactored (ed25519_verify.rs:54-117)"""
    R, A = decompress(sig[:32]), decompress(pub)
    s = int.from_bytes(sig[32:], "little")
    if R is None or A is None or s >= L_ORDER:
        return False
    k = int.from_bytes(hashlib.sha512(sig[:32] + pub + msg).digest(), "little") % L_ORDER
    res = pt_add(pt_add(_scalar_mul_int(s, BASEPOINT), pt_neg(R)), pt_neg(_scalar_mul_int(k, A)))
    for _ in range(3):
        res = pt_double(res)
    return res[0] == 0 and res[1] == res[2]


def ladder_bits(scalar32: bytes, k: int):
    """s_bits_for_ladder / r_thread_bits_for_kA: the k low bits, most significant first"""
    v = int.from_bytes(scalar32, "little")
    return [(v >> (k - 1 - i)) & 1 for i in range(k)]


def k_scalar_bytes(sig: bytes, pub: bytes, msg: bytes) -> bytes:
    return (int.from_bytes(hashlib.sha512(sig[:32] + pub + msg).digest(), "little") % L_ORDER).to_bytes(32, "little")


def pi_hash(pub: bytes, sig: bytes, msg: bytes, fs_binding: bytes, merkle_root: bytes, root_f0: bytes) -> bytes:
    """zsk_ksk_pi_hash_v2_stark (swarm-dns/src/prover.rs:763-780)"""
    h = hashlib.sha3_256()
    for part in (b"ZSK-KSK-PIHASH-V2-ST", pub, sig, len(msg).to_bytes(8, "little"), msg, fs_binding, merkle_root,
                 root_f0):
        h.update(part)
    return h.digest()


# ---------------------------------------------------------------- layout
class Gad:
    """one field gadget's cells: a, b inputs by reference; the rest owned"""

    def __init__(self, kind, **kw):
        self.kind = kind
        self.__dict__.update(kw)


class Alloc:
    def __init__(self, start):
        self.next = start

    def take(self, n):
        r = self.next
        self.next += n
        return r

    def sub(self, a, b):
        c = self.take(NL)
        return Gad("sub", a=a, b=b, c=c, bits=self.take(255), pos=self.take(NL), neg=self.take(NL))

    def add(self, a, b):
        c = self.take(NL)
        return Gad("add", a=a, b=b, c=c, bits=self.take(255), carries=self.take(NL))

    def mul(self, a, b):
        c = self.take(NL)
        return Gad("mul", a=a, b=b, c=c, bits=self.take(255), carry=self.take(MUL_CB * NL))


def point_add_layout(base, p1, p2):
    """point_add_layout_at (ed25519_group_air.rs:202-249); p1, p2 = (x, y, z, t) limb bases"""
    al = Alloc(base)
    g = Gad("pa", p1=p1, p2=p2, d2=al.take(NL))
    g.sub_ym1 = al.sub(p1[1], p1[0])
    g.sub_ym2 = al.sub(p2[1], p2[0])
    g.add_yp1 = al.add(p1[1], p1[0])
    g.add_yp2 = al.add(p2[1], p2[0])
    g.mul_A = al.mul(g.sub_ym1.c, g.sub_ym2.c)
    g.mul_B = al.mul(g.add_yp1.c, g.add_yp2.c)
    g.mul_tt = al.mul(p1[3], p2[3])
    g.mul_C = al.mul(g.mul_tt.c, g.d2)
    g.mul_zz = al.mul(p1[2], p2[2])
    g.add_D = al.add(g.mul_zz.c, g.mul_zz.c)
    g.sub_E = al.sub(g.mul_B.c, g.mul_A.c)
    g.sub_F = al.sub(g.add_D.c, g.mul_C.c)
    g.add_G = al.add(g.add_D.c, g.mul_C.c)
    g.add_H = al.add(g.mul_B.c, g.mul_A.c)
    g.mul_X3 = al.mul(g.sub_E.c, g.sub_F.c)
    g.mul_Y3 = al.mul(g.add_G.c, g.add_H.c)
    g.mul_T3 = al.mul(g.sub_E.c, g.add_H.c)
    g.mul_Z3 = al.mul(g.sub_F.c, g.add_G.c)
    g.end = al.next
    g.out = (g.mul_X3.c, g.mul_Y3.c, g.mul_Z3.c, g.mul_T3.c)
    return g


def point_double_layout(base, x, y, z):
    """point_double_layout_at (ed25519_group_air.rs:476-505)"""
    al = Alloc(base)
    g = Gad("dbl", p1=(x, y, z))
    g.sq_A = al.mul(x, x)
    g.sq_B = al.mul(y, y)
    g.sq_zz = al.mul(z, z)
    g.add_C = al.add(g.sq_zz.c, g.sq_zz.c)
    g.add_H = al.add(g.sq_A.c, g.sq_B.c)
    g.add_xy = al.add(x, y)
    g.sq_xy = al.mul(g.add_xy.c, g.add_xy.c)
    g.sub_E = al.sub(g.add_H.c, g.sq_xy.c)
    g.sub_G = al.sub(g.sq_A.c, g.sq_B.c)
    g.add_F = al.add(g.add_C.c, g.sub_G.c)
    g.mul_X3 = al.mul(g.sub_E.c, g.add_F.c)
    g.mul_Y3 = al.mul(g.sub_G.c, g.add_H.c)
    g.mul_T3 = al.mul(g.sub_E.c, g.add_H.c)
    g.mul_Z3 = al.mul(g.add_F.c, g.sub_G.c)
    g.end = al.next
    g.out = (g.mul_X3.c, g.mul_Y3.c, g.mul_Z3.c, g.mul_T3.c)
    return g


def cond_add_layout(base, acc, bp):
    """cond_add_layout_at (ed25519_group_air.rs:662-719)"""
    al = Alloc(base)
    g = Gad("cadd", bit=al.take(1))
    g.out = (al.take(NL), al.take(NL), al.take(NL), al.take(NL))
    g.add = point_add_layout(al.next, acc, bp)
    al.next = g.add.end
    g.sel = [Gad("sel", a=acc[q], b=g.add.out[q], bit=g.bit, c=g.out[q]) for q in range(4)]
    g.end = al.next
    return g


def decompress_layout(base, y_limbs, sign_bit):
    """point_decompress_layout_at (ed25519_group_air.rs:887-955)"""
    al = Alloc(base)
    g = Gad("decomp", y=y_limbs, sign=sign_bit, d=al.take(NL))
    g.x = al.take(NL)
    g.x_bits = al.take(255)
    g.sq_x = al.mul(g.x, g.x)
    g.sq_y = al.mul(y_limbs, y_limbs)
    g.mul_dx2 = al.mul(g.d, g.sq_x.c)
    g.mul_dxy = al.mul(g.mul_dx2.c, g.sq_y.c)
    g.one = al.take(NL)
    g.sub_y2m1 = al.sub(g.sq_y.c, g.one)
    g.sub_lhs = al.sub(g.sub_y2m1.c, g.sq_x.c)
    g.sub_eq = al.sub(g.sub_lhs.c, g.mul_dxy.c)
    g.sign_match = al.take(1)
    g.end = al.next
    return g


class Layout:
    """VerifyAirLayoutV16 (ed25519_verify_air.rs:4670-4814) for a message of msg_len bytes
    (the SHA-512 input R || A || M) and k_scalar ladder rows."""

    def __init__(self, msg_len, k_scalar):
        K = self.k = k_scalar
        assert 2 <= K <= 256
        self.n_blocks = (msg_len + 1 + 16 + 127) // 128
        kh = 128
        while kh < 128 * self.n_blocks:
            kh *= 2
        self.k_hash = kh
        self.reduce_row, self.decomp_R_row, self.decomp_A_row = kh, kh + 1, kh + 2
        self.sB_first = kh + 3
        self.kA_first = self.sB_first + K
        self.sB_last, self.kA_last = self.sB_first + K - 1, self.kA_first + K - 1
        self.residual_row = self.kA_last + 1
        self.dbl_rows = (self.kA_last + 2, self.kA_last + 3, self.kA_last + 4)
        self.result_row = self.kA_last + 5
        # scalar reduction at columns 0.. of its row (v0)
        nx = RED_LIMBS_IN
        self.red = {"input": 0}
        for name, n in (("q", RED_Q), ("q_bits", RED_Q * RED_LB), ("r", RED_R), ("r_bits", RED_R * RED_LB),
                        ("slack", RED_R), ("slack_bits", RED_R * RED_LB), ("carry_bits", RED_PROD * RED_CB)):
            self.red[name] = nx
            nx += n
        self.digest_bits = SHA512_WIDTH  # v1
        self.decomp = decompress_layout(NL + 1, 0, NL)  # v2: y at 0, sign at 10
        # ladder row (ed25519_scalar_mult_air.rs:93-131)
        self.base = tuple(q * NL for q in range(4))
        self.acc = tuple(40 + q * NL for q in range(4))
        self.mdbl = point_double_layout(80, *self.acc[:3])
        self.cadd = cond_add_layout(self.mdbl.end, self.mdbl.out, self.base)
        assert self.cadd.end == 14941
        w = 14941
        self.sblock_sB, self.sblock_kA = w, w + K  # v6
        self.r_thread = w + 2 * K  # v7
        nx = w + 3 * K
        self.result = tuple(nx + q * NL for q in range(4))  # v10
        nx += 4 * NL
        self.zero_const = nx
        nx += NL
        al = Alloc(nx)
        self.sub_X = al.sub(self.result[0], self.zero_const)
        self.sub_T = al.sub(self.result[3], self.zero_const)
        self.sub_YZ = al.sub(self.result[1], self.result[2])
        self.dbl_in = (al.take(NL), al.take(NL), al.take(NL))
        self.dbl = point_double_layout(al.next, *self.dbl_in)
        nx = self.dbl.end
        self.thr_sB = tuple(nx + q * NL for q in range(4))  # v11
        nx += 4 * NL
        self.thr_kA = tuple(nx + q * NL for q in range(4))  # v12
        nx += 4 * NL
        self.thr_R = tuple(nx + q * NL for q in range(4))  # v13
        nx += 4 * NL
        self.one_R = nx
        nx += NL
        al = Alloc(nx)
        self.mul_RT = al.mul(self.thr_R[0], self.thr_R[1])
        self.zero_R1 = al.take(NL)  # v14
        self.sub_negR_X = al.sub(self.zero_R1, self.thr_R[0])
        self.sub_negR_T = al.sub(self.zero_R1, self.thr_R[3])
        self.pa_R1 = point_add_layout(al.next, self.thr_sB,
                                      (self.sub_negR_X.c, self.thr_R[1], self.thr_R[2], self.sub_negR_T.c))
        al = Alloc(self.pa_R1.end)  # v15
        self.sub_negkA_X = al.sub(self.zero_R1, self.thr_kA[0])
        self.sub_negkA_T = al.sub(self.zero_R1, self.thr_kA[3])
        self.pa_R2 = point_add_layout(al.next, self.pa_R1.out,
                                      (self.sub_negkA_X.c, self.thr_kA[1], self.thr_kA[2], self.sub_negkA_T.c))
        self.width = self.pa_R2.end
        h = 1
        while h < self.sB_first + 2 * K:
            h *= 2
        need = self.result_row + 1
        if h < need + 1:
            h = 1
            while h < need:
                h *= 2
        self.height = h


# ---------------------------------------------------------------- constraint program
class Program:
    """The constraint vector as blocks with row gates, in emission order; `records()` and
    `pairs` are what the C++ oracle evaluates."""

    def __init__(self):
        self.blocks = []  # (gate, kind, params, count)
        self.pairs = []   # (a_ref, b_ref), ref = src << 62 | cell_or_const
        self.n = 0

    def _blk(self, gate, kind, params, count):
        self.blocks.append((gate, kind, tuple(params), count))
        self.n += count

    def sha512(self, gate, n_blocks):
        self._blk(gate, B_SHA512, [n_blocks], SHA512_K)

    def reduce(self, gate, r):
        self._blk(gate, B_REDUCE, [r[k] for k in ("input", "q", "q_bits", "r", "r_bits", "slack", "slack_bits",
                                                   "carry_bits")], REDUCE_K)

    def format(self, gate, digest_bits, input_base):
        self._blk(gate, B_FORMAT, [digest_bits, input_base, SHA512_H0_LO], FORMAT_K)

    def gadget(self, gate, g):
        if g.kind == "mul":
            self._blk(gate, B_MUL, [g.a, g.b, g.c, g.bits, g.carry], MUL_K)
        elif g.kind == "add":
            self._blk(gate, B_ADD, [g.a, g.b, g.c, g.bits, g.carries], ADD_K)
        elif g.kind == "sub":
            self._blk(gate, B_SUB, [g.a, g.b, g.c, g.bits, g.pos, g.neg], SUB_K)
        elif g.kind == "sel":
            self._blk(gate, B_SEL, [g.a, g.b, g.bit, g.c], SEL_K)
        else:
            raise ValueError(g.kind)

    def range_check(self, gate, limbs_base, bits_base):
        self._blk(gate, B_RANGE, [limbs_base, bits_base], RANGE_K)

    def sign(self, gate, sign_bit, x_bits):
        self._blk(gate, B_SIGN, [sign_bit, x_bits], 2)

    def diff(self, gate, items):
        """items: ((src, cell), (src, cell_or_const)) pairs, each one constraint A - B"""
        off = len(self.pairs)
        for (sa, a), (sb, b) in items:
            assert 0 <= a < 1 << 62 and 0 <= b < 1 << 62
            self.pairs.append(((sa << 62) | a, (sb << 62) | b))
        self._blk(gate, B_PAIRS, [off, len(items)], len(items))

    def records(self):
        out = np.full((len(self.blocks), REC), NONE, dtype=np.uint64)
        for i, (gate, kind, params, _count) in enumerate(self.blocks):
            out[i, 0] = gate[0]
            for j, g in enumerate(gate[1:]):
                out[i, 1 + j] = g
            out[i, 4] = kind
            for j, p in enumerate(params):
                out[i, 5 + j] = p
        return out

    def pair_array(self):
        return np.array(self.pairs, dtype=np.uint64).reshape(-1, 2) if self.pairs else np.zeros((0, 2), np.uint64)


def cur(c):
    return (SRC_CUR, c)


def nxt(c):
    return (SRC_NXT, c)


def const(v):
    return (SRC_CONST, v)


def _pa_blocks(pr, gate, g):
    """eval_point_add_gadget (ed25519_group_air.rs:334-380)"""
    pr.diff(gate, [(cur(g.d2 + k), const(D2_LOOSE[k])) for k in range(NL)])
    for name in ("sub_ym1", "sub_ym2", "add_yp1", "add_yp2", "mul_A", "mul_B", "mul_tt", "mul_C", "mul_zz",
                 "add_D", "sub_E", "sub_F", "add_G", "add_H", "mul_X3", "mul_Y3", "mul_T3", "mul_Z3"):
        pr.gadget(gate, getattr(g, name))


def _dbl_blocks(pr, gate, g):
    """eval_point_double_gadget (ed25519_group_air.rs:548-573)"""
    for name in ("sq_A", "sq_B", "sq_zz", "add_C", "add_H", "add_xy", "sq_xy", "sub_E", "sub_G", "add_F",
                 "mul_X3", "mul_Y3", "mul_T3", "mul_Z3"):
        pr.gadget(gate, getattr(g, name))


def _decomp_blocks(pr, gate, g):
    """eval_point_decompress_gadget (ed25519_group_air.rs:1031-1090)"""
    pr.diff(gate, [(cur(g.d + k), const(D_LIMBS[k])) for k in range(NL)])
    pr.range_check(gate, g.x, g.x_bits)
    for gg in (g.sq_x, g.sq_y, g.mul_dx2, g.mul_dxy, g.sub_y2m1, g.sub_lhs, g.sub_eq):
        pr.gadget(gate, gg)
    pr.diff(gate, [(cur(g.sub_eq.c + k), const(0)) for k in range(NL)])
    pr.sign(gate, g.sign, g.x_bits)


def _ladder_blocks(pr, lay, first, last):
    """v3 phase E/F (ed25519_verify_air.rs:1137-1175): per row, transition, initial acc"""
    rows = (GATE_RANGE, first, last + 1)
    _dbl_blocks(pr, rows, lay.mdbl)
    _pa_blocks(pr, rows, lay.cadd.add)
    for s in lay.cadd.sel:
        pr.gadget(rows, s)
    items = []
    for k in range(NL):  # eval_scalar_mult_transition (ed25519_scalar_mult_air.rs:208-236)
        for q in range(4):
            items.append((nxt(lay.base[q] + k), cur(lay.base[q] + k)))
    for k in range(NL):
        for q in range(4):
            items.append((nxt(lay.acc[q] + k), cur(lay.cadd.out[q] + k)))
    pr.diff((GATE_RANGE, first, last), items)
    ident = [limbs(c) for c in IDENTITY]  # eval_scalar_mult_initial_acc (:239-256)
    pr.diff((GATE_EQ, first), [(cur(lay.acc[q] + k), const(ident[q][k])) for k in range(NL) for q in range(4)])


def _copy4(dst, src, src_dst=SRC_CUR):
    return [((src_dst, dst[q] + i), cur(src[q] + i)) for q in range(4) for i in range(NL)]


def program(lay, s_bits, k_bits, r_y, r_sign, a_y, a_sign, a_point):
    """eval_verify_air_v16_per_row (ed25519_verify_air.rs:4870-4960) as blocks, through the v15 .. v0
    evaluators it delegates to; the constant pins come from the public inputs"""
    K = lay.k
    pr = Program()
    # v3 (v0 .. v2 inside)
    pr.sha512((GATE_RANGE, 0, lay.k_hash - 1), lay.n_blocks)
    pr.reduce((GATE_EQ, lay.reduce_row), lay.red)
    pr.format((GATE_EQ, lay.k_hash - 1), lay.digest_bits, lay.red["input"])
    _decomp_blocks(pr, (GATE_EQ, lay.decomp_R_row), lay.decomp)
    _decomp_blocks(pr, (GATE_EQ, lay.decomp_A_row), lay.decomp)
    _ladder_blocks(pr, lay, lay.sB_first, lay.sB_last)
    _ladder_blocks(pr, lay, lay.kA_first, lay.kA_last)
    # v4: ladder bases
    bp = [limbs(c) for c in BASEPOINT]
    pr.diff((GATE_EQ, lay.sB_first), [(cur(lay.base[q] + k), const(bp[q][k])) for q in range(4) for k in range(NL)])
    ap = [limbs(c) for c in a_point]
    pr.diff((GATE_EQ, lay.kA_first), [(cur(lay.base[q] + k), const(ap[q][k])) for q in range(4) for k in range(NL)])
    # v5: decompression inputs
    for row, y, s in ((lay.decomp_R_row, r_y, r_sign), (lay.decomp_A_row, a_y, a_sign)):
        yl = limbs(y)
        pr.diff((GATE_EQ, row), [(cur(lay.decomp.y + k), const(yl[k])) for k in range(NL)] +
                [(cur(lay.decomp.sign), const(s))])
    # v6: scalar shift chains
    for first, last, base, bits in ((lay.sB_first, lay.sB_last, lay.sblock_sB, s_bits),
                                    (lay.kA_first, lay.kA_last, lay.sblock_kA, k_bits)):
        pr.diff((GATE_EQ, first), [(cur(base + i), const(bits[i])) for i in range(K)])
        pr.diff((GATE_RANGE, first, last + 1), [(cur(lay.cadd.bit), cur(base))])
        pr.diff((GATE_RANGE, first, last), [(nxt(base + i), cur(base + i + 1)) for i in range(K - 1)])
    # v7: r thread
    pr.diff((GATE_EQ, lay.reduce_row), [(cur(lay.r_thread + i), cur(lay.red["r_bits"] + K - 1 - i)) for i in range(K)])
    pr.diff((GATE_ALWAYS,), [(nxt(lay.r_thread + i), cur(lay.r_thread + i)) for i in range(K)])
    pr.diff((GATE_EQ, lay.kA_first), [(cur(lay.sblock_kA + i), cur(lay.r_thread + i)) for i in range(K)])
    # v10: verdict, doubling chain, result binding
    res = (GATE_EQ, lay.result_row)
    pr.diff(res, [(cur(lay.zero_const + i), const(0)) for i in range(NL)])
    for g in (lay.sub_X, lay.sub_T, lay.sub_YZ):
        pr.gadget(res, g)
    pr.diff(res, [(cur(g.c + i), const(0)) for g in (lay.sub_X, lay.sub_T, lay.sub_YZ) for i in range(NL)])
    d1, d2, d3 = lay.dbl_rows
    _dbl_blocks(pr, (GATE_SET, d1, d2, d3), lay.dbl)
    pr.diff((GATE_SET, d1, d2, NONE), [(nxt(lay.dbl_in[q] + i), cur(lay.dbl.out[q] + i)) for q in range(3)
                                       for i in range(NL)])
    pr.diff((GATE_EQ, d3), [(nxt(lay.result[q] + i), cur(lay.dbl.out[q] + i)) for q in range(4) for i in range(NL)])
    # v11, v12: output threads of the two ladders
    for last, thr in ((lay.sB_last, lay.thr_sB), (lay.kA_last, lay.thr_kA)):
        pr.diff((GATE_EQ, last), [(cur(thr[q] + i), cur(lay.cadd.out[q] + i)) for q in range(4) for i in range(NL)])
        pr.diff((GATE_ALWAYS,), [(nxt(thr[q] + i), cur(thr[q] + i)) for q in range(4) for i in range(NL)])
    # v13: R thread with T = X Y
    rr = (GATE_EQ, lay.decomp_R_row)
    src = (lay.decomp.x, lay.decomp.y, lay.one_R, lay.mul_RT.c)
    pr.diff(rr, [(cur(lay.thr_R[q] + i), cur(src[q] + i)) for q in range(4) for i in range(NL)])
    pr.diff(rr, [(cur(lay.one_R + i), const(ONE_LIMBS[i])) for i in range(NL)])
    pr.gadget(rr, lay.mul_RT)
    pr.diff((GATE_ALWAYS,), [(nxt(lay.thr_R[q] + i), cur(lay.thr_R[q] + i)) for q in range(4) for i in range(NL)])
    # v14, v15: the residual row
    rs = (GATE_EQ, lay.residual_row)
    pr.diff(rs, [(cur(lay.zero_R1 + i), const(0)) for i in range(NL)])
    pr.gadget(rs, lay.sub_negR_X)
    pr.gadget(rs, lay.sub_negR_T)
    _pa_blocks(pr, rs, lay.pa_R1)
    pr.gadget(rs, lay.sub_negkA_X)
    pr.gadget(rs, lay.sub_negkA_T)
    _pa_blocks(pr, rs, lay.pa_R2)
    # v16: residual_2 into the doubling chain
    pr.diff(rs, [(nxt(lay.dbl_in[q] + i), cur(lay.pa_R2.out[q] + i)) for q in range(3) for i in range(NL)])
    return pr


def n_constraints(k_scalar):
    """verify_v16_per_row_constraints"""
    fixed = (SHA512_K + REDUCE_K + FORMAT_K + 2 * DECOMP_K + 2 * (DBL_K + PA_K + 4 * SEL_K + 80 + 40) + 80 + 22 +
             2 + 955 + DBL_K + 30 + 40 + 4 * 40 + 40 + 10 + MUL_K + 40 + (NL + 2 * SUB_K + PA_K) +
             (2 * SUB_K + PA_K) + 30)
    return fixed + 7 * k_scalar - 2


# ---------------------------------------------------------------- trace
class Trace:
    def __init__(self, width, height):
        self.t = np.zeros((width, height), dtype=np.uint64)

    def limbs(self, row, base, ls):
        for i, l in enumerate(ls):
            self.t[base + i, row] = l

    def elem(self, row, c, bits, x):
        ls = limbs(x)
        self.limbs(row, c, ls)
        off = 0
        for i in range(NL):
            for b in range(LW[i]):
                self.t[bits + off + b, row] = (ls[i] >> b) & 1
            off += LW[i]

    # -- field gadgets; a, b are limb lists as the cells hold them
    def add(self, row, g, a, b):
        c = (value(a) + value(b)) % P
        self.elem(row, g.c, g.bits, c)
        cl = limbs(c)
        top = 1 if value(a) + value(b) >= P else 0
        prev = 19 * top
        for k in range(NL):
            d = a[k] + b[k] + prev - cl[k]
            cy = d >> LW[k]
            assert cy in (0, 1) and cy << LW[k] == d
            self.t[g.carries + k, row] = cy
            prev = cy
        assert prev == top
        return c

    def sub(self, row, g, a, b):
        c = (value(a) - value(b)) % P
        self.elem(row, g.c, g.bits, c)
        cl = limbs(c)
        top = 1 if value(a) < value(b) else 0  # c = a - b + net[9] p
        prev = 19 * top
        for k in range(NL):
            v = a[k] - b[k] - prev
            net = (cl[k] - v) >> LW[k]
            assert net in (-1, 0, 1) and cl[k] - v == net << LW[k]
            self.t[g.pos + k, row] = 1 if net == 1 else 0
            self.t[g.neg + k, row] = 1 if net == -1 else 0
            prev = net
        assert prev == top
        return c

    def mul(self, row, g, a, b):
        c = value(a) * value(b) % P
        self.elem(row, g.c, g.bits, c)
        cl = limbs(c)
        t = [0] * NL
        for i in range(NL):
            for j in range(NL):
                f = 2 if (i & 1 and j & 1) else 1
                s = i + j
                if s >= NL:
                    s, f = s - NL, 19 * f
                t[s] += f * a[i] * b[j]
        tot = sum(t[k] << LOFF[k] for k in range(NL)) - c
        assert tot % P == 0
        top = tot // P
        prev = 19 * top
        half = 1 << (MUL_CB - 1)
        for k in range(NL):
            d = t[k] + prev - cl[k]
            cy = d >> LW[k]
            assert cy << LW[k] == d and -half <= cy < half
            biased = cy + half
            for bb in range(MUL_CB):
                self.t[g.carry + k * MUL_CB + bb, row] = (biased >> bb) & 1
            prev = cy
        assert prev == top
        return c

    def sel(self, row, g, a, b, bit):
        self.t[g.bit, row] = bit
        self.limbs(row, g.c, b if bit else a)

    # -- group gadgets; points are canonical ints mod p
    def point_add(self, row, g, p1, p2):
        """fill_point_add_gadget (ed25519_group_air.rs:251-321)"""
        self.limbs(row, g.d2, D2_LOOSE)
        X1, Y1, Z1, T1 = [limbs(v) for v in p1]
        X2, Y2, Z2, T2 = [limbs(v) for v in p2]
        ym1 = self.sub(row, g.sub_ym1, Y1, X1)
        ym2 = self.sub(row, g.sub_ym2, Y2, X2)
        yp1 = self.add(row, g.add_yp1, Y1, X1)
        yp2 = self.add(row, g.add_yp2, Y2, X2)
        A = self.mul(row, g.mul_A, limbs(ym1), limbs(ym2))
        B = self.mul(row, g.mul_B, limbs(yp1), limbs(yp2))
        tt = self.mul(row, g.mul_tt, T1, T2)
        C = self.mul(row, g.mul_C, limbs(tt), D2_LOOSE)
        zz = self.mul(row, g.mul_zz, Z1, Z2)
        D_ = self.add(row, g.add_D, limbs(zz), limbs(zz))
        E = self.sub(row, g.sub_E, limbs(B), limbs(A))
        F_ = self.sub(row, g.sub_F, limbs(D_), limbs(C))
        G = self.add(row, g.add_G, limbs(D_), limbs(C))
        H = self.add(row, g.add_H, limbs(B), limbs(A))
        X3 = self.mul(row, g.mul_X3, limbs(E), limbs(F_))
        Y3 = self.mul(row, g.mul_Y3, limbs(G), limbs(H))
        T3 = self.mul(row, g.mul_T3, limbs(E), limbs(H))
        Z3 = self.mul(row, g.mul_Z3, limbs(F_), limbs(G))
        return (X3, Y3, Z3, T3)

    def point_double(self, row, g, p1):
        """fill_point_double_gadget (ed25519_group_air.rs:507-546)"""
        X1, Y1, Z1 = [limbs(v) for v in p1[:3]]
        A = self.mul(row, g.sq_A, X1, X1)
        B = self.mul(row, g.sq_B, Y1, Y1)
        zz = self.mul(row, g.sq_zz, Z1, Z1)
        C = self.add(row, g.add_C, limbs(zz), limbs(zz))
        H = self.add(row, g.add_H, limbs(A), limbs(B))
        xy = self.add(row, g.add_xy, X1, Y1)
        xy_sq = self.mul(row, g.sq_xy, limbs(xy), limbs(xy))
        E = self.sub(row, g.sub_E, limbs(H), limbs(xy_sq))
        G = self.sub(row, g.sub_G, limbs(A), limbs(B))
        F_ = self.add(row, g.add_F, limbs(C), limbs(G))
        X3 = self.mul(row, g.mul_X3, limbs(E), limbs(F_))
        Y3 = self.mul(row, g.mul_Y3, limbs(G), limbs(H))
        T3 = self.mul(row, g.mul_T3, limbs(E), limbs(H))
        Z3 = self.mul(row, g.mul_Z3, limbs(F_), limbs(G))
        return (X3, Y3, Z3, T3)

    def decompress(self, row, g, y, sign):
        """v2 phase C/D (ed25519_verify_air.rs:700-724) and fill_point_decompress_gadget (:957-1029)"""
        self.limbs(row, g.y, limbs(y))
        self.t[g.sign, row] = sign
        self.limbs(row, g.d, D_LIMBS)
        self.limbs(row, g.one, ONE_LIMBS)
        pt = decompress((y | (sign << 255)).to_bytes(32, "little"))
        assert pt is not None
        x = pt[0]
        self.elem(row, g.x, g.x_bits, x)
        x_sq = self.mul(row, g.sq_x, limbs(x), limbs(x))
        y_sq = self.mul(row, g.sq_y, limbs(y), limbs(y))
        dx2 = self.mul(row, g.mul_dx2, D_LIMBS, limbs(x_sq))
        dxy = self.mul(row, g.mul_dxy, limbs(dx2), limbs(y_sq))
        y2m1 = self.sub(row, g.sub_y2m1, limbs(y_sq), ONE_LIMBS)
        lhs = self.sub(row, g.sub_lhs, limbs(y2m1), limbs(x_sq))
        self.sub(row, g.sub_eq, limbs(lhs), limbs(dxy))
        return pt

    def reduce(self, row, r, digest: bytes):
        """v0 input limbs and fill_scalar_reduce_gadget (ed25519_scalar_air.rs:168-372)"""
        inp = [digest[2 * i] | (digest[2 * i + 1] << 8) for i in range(RED_LIMBS_IN)]
        self.limbs(row, r["input"], inp)
        d = int.from_bytes(digest, "little")
        rv = d % L_ORDER
        q = (d - rv) // L_ORDER
        slack = L_ORDER - 1 - rv
        l16 = [(L_ORDER >> (16 * j)) & 0xFFFF for j in range(RED_R)]
        parts = {"q": [(q >> (16 * i)) & 0xFFFF for i in range(RED_Q)],
                 "r": [(rv >> (16 * i)) & 0xFFFF for i in range(RED_R)],
                 "slack": [(slack >> (16 * i)) & 0xFFFF for i in range(RED_R)]}
        assert q >> (16 * RED_Q) == 0
        for name, ls in parts.items():
            self.limbs(row, r[name], ls)
            for i, l in enumerate(ls):
                for b in range(RED_LB):
                    self.t[r[name + "_bits"] + i * RED_LB + b, row] = (l >> b) & 1
        prev = 0
        half = 1 << (RED_CB - 1)
        for k in range(RED_PROD):
            prod = sum(parts["q"][i] * l16[k - i] for i in range(RED_Q) if 0 <= k - i < RED_R)
            resid = (inp[k] if k < RED_LIMBS_IN else 0) - prod - (parts["r"][k] if k < RED_R else 0)
            tot = resid + prev
            assert tot % (1 << RED_LB) == 0
            cy = tot >> RED_LB
            biased = cy + half
            for b in range(RED_CB):
                self.t[r["carry_bits"] + k * RED_CB + b, row] = (biased >> b) & 1
            prev = cy
        assert prev == 0
        return rv

    def ladder(self, first, lay, base, bits):
        """fill_scalar_mult_trace (ed25519_scalar_mult_air.rs:133-171) at rows first .."""
        acc = IDENTITY
        for j, bit in enumerate(bits):
            row = first + j
            for q in range(4):
                self.limbs(row, lay.base[q], limbs(base[q]))
                self.limbs(row, lay.acc[q], limbs(acc[q]))
            self.point_double(row, lay.mdbl, acc)
            dbl = pt_double(acc)
            tmp = self.point_add(row, lay.cadd.add, dbl, base)
            assert tmp == pt_add(dbl, base)
            for q in range(4):
                self.sel(row, lay.cadd.sel[q], limbs(dbl[q]), limbs(tmp[q]), bit)
            acc = tmp if bit else dbl
        return acc


def public_constants(sig: bytes, pub: bytes):
    """(r_y, r_sign, a_y, a_sign, A) of the v4/v5 pins; None for an invalid encoding"""
    r_y, r_sign = split_compressed(sig[:32])
    a_y, a_sign = split_compressed(pub)
    A = decompress(pub)
    if A is None or decompress(sig[:32]) is None:
        return None
    return r_y, r_sign, a_y, a_sign, A


def layout_program(pub: bytes, sig: bytes, msg: bytes, k_scalar: int = 256):
    """verify_air_layout_v16 and the constraint program for prove_zsk_ksk_binding_v2's inputs"""
    lay = Layout(32 + 32 + len(msg), k_scalar)
    s_bits = ladder_bits(sig[32:], k_scalar)
    k_bits = ladder_bits(k_scalar_bytes(sig, pub, msg), k_scalar)
    pc = public_constants(sig, pub)
    assert pc is not None, "R or A does not decode"
    r_y, r_sign, a_y, a_sign, A = pc
    return lay, program(lay, s_bits, k_bits, r_y, r_sign, a_y, a_sign, A), s_bits, k_bits


def build(pub: bytes, sig: bytes, msg: bytes, k_scalar: int = 256):
    """fill_verify_air_v16 for prove_zsk_ksk_binding_v2's inputs -> (layout, program, trace (width, height))"""
    sha_in = sig[:32] + pub + msg
    K = k_scalar
    lay, pr, s_bits, k_bits = layout_program(pub, sig, msg, K)
    digest = hashlib.sha512(sha_in).digest()
    r_y, r_sign, a_y, a_sign, A = public_constants(sig, pub)
    R = decompress(sig[:32])
    tr = Trace(lay.width, lay.height)
    # v0/v1: SHA-512 rows, digest bits, the reduction row
    sha, nb = O.sha512_trace(sha_in)
    assert nb == lay.n_blocks and sha.shape[1] == lay.k_hash
    tr.t[:SHA512_WIDTH, :lay.k_hash] = sha
    for k in range(8):
        h = int.from_bytes(digest[8 * k:8 * k + 8], "big")
        for i in range(64):
            tr.t[lay.digest_bits + 64 * k + i, lay.k_hash - 1] = (h >> i) & 1
    tr.reduce(lay.reduce_row, lay.red, digest)
    # v2: decompressions
    tr.decompress(lay.decomp_R_row, lay.decomp, r_y, r_sign)
    tr.decompress(lay.decomp_A_row, lay.decomp, a_y, a_sign)
    # v3: ladders
    sB = tr.ladder(lay.sB_first, lay, BASEPOINT, s_bits)
    kA = tr.ladder(lay.kA_first, lay, A, k_bits)
    assert sB == ladder(BASEPOINT, s_bits) and kA == ladder(A, k_bits)
    # v6: scalar shift chains
    for first, base, bits in ((lay.sB_first, lay.sblock_sB, s_bits), (lay.kA_first, lay.sblock_kA, k_bits)):
        for j in range(K):
            for i in range(K):
                tr.t[base + i, first + j] = bits[j + i] if j + i < K else 0
    # v7, v11-v13: threads at every row
    for i in range(K):
        tr.t[lay.r_thread + i, :] = k_bits[i]
    R_thread = (R[0], R[1], 1, R[0] * R[1] % P)
    for thr, pt in ((lay.thr_sB, sB), (lay.thr_kA, kA), (lay.thr_R, R_thread)):
        for q in range(4):
            for i, l in enumerate(limbs(pt[q])):
                tr.t[thr[q] + i, :] = l
    # v13: one constant and T = X Y at the R decompression row
    tr.limbs(lay.decomp_R_row, lay.one_R, ONE_LIMBS)
    tr.mul(lay.decomp_R_row, lay.mul_RT, limbs(R_thread[0]), limbs(R_thread[1]))
    # v14, v15: the residual row
    rs = lay.residual_row
    zero = limbs(0)
    tr.sub(rs, lay.sub_negR_X, zero, limbs(R_thread[0]))
    tr.sub(rs, lay.sub_negR_T, zero, limbs(R_thread[3]))
    res1 = tr.point_add(rs, lay.pa_R1, sB, pt_neg(R_thread))
    tr.sub(rs, lay.sub_negkA_X, zero, limbs(kA[0]))
    tr.sub(rs, lay.sub_negkA_T, zero, limbs(kA[3]))
    res2 = tr.point_add(rs, lay.pa_R2, res1, pt_neg(kA))
    assert res1 == pt_add(sB, pt_neg(R_thread)) and res2 == pt_add(res1, pt_neg(kA))
    # v9/v10 cells at the v14 rows: the cofactor doublings and the verdict
    p = res2
    for row in lay.dbl_rows:
        for q in range(3):
            tr.limbs(row, lay.dbl_in[q], limbs(p[q]))
        tr.point_double(row, lay.dbl, p)
        p = pt_double(p)
    row = lay.result_row
    for q in range(4):
        tr.limbs(row, lay.result[q], limbs(p[q]))
    tr.sub(row, lay.sub_X, limbs(p[0]), zero)
    tr.sub(row, lay.sub_T, limbs(p[3]), zero)
    tr.sub(row, lay.sub_YZ, limbs(p[1]), limbs(p[2]))
    return lay, pr, tr.t


# ---------------------------------------------------------------- C++ oracle
def _lib():
    L = O.lib()
    if not getattr(L, "_ed25519_bound", False):
        sz = ctypes.c_size_t
        L.orc_ed25519_eval.argtypes = [O.U64P, O.U64P, sz, O.U64P, sz, O.U64P, sz, O.U64P]
        L.orc_merge_ed25519.argtypes = [O.U64P, sz, O.U64P, sz, O.U64P, sz, sz, sz, sz, O.U64P]
        L.orc_prove_ed25519.argtypes = [O.U64P, sz, O.U64P, sz, O.U64P, sz, sz, sz, ctypes.c_char_p, sz,
                                        ctypes.c_char_p, sz, ctypes.POINTER(sz)]
        L._ed25519_bound = True
    return L


def eval_row(pr, cur_row, nxt_row, row):
    cur_row = np.ascontiguousarray(cur_row, dtype=np.uint64)
    nxt_row = np.ascontiguousarray(nxt_row, dtype=np.uint64)
    out = np.zeros(pr.n, dtype=np.uint64)
    rec, pairs = pr.records(), pr.pair_array()
    n = _lib().orc_ed25519_eval(O._ptr(cur_row), O._ptr(nxt_row), row, O._ptr(rec), rec.shape[0],
                                O._ptr(pairs), pairs.shape[0], O._ptr(out))
    assert n == pr.n, (n, pr.n)
    return out


def merge(lay, pr, lde_cols, n_trace, blowup=BLOWUP):
    lde_cols = np.ascontiguousarray(lde_cols, dtype=np.uint64)
    out = np.zeros(n_trace * blowup, dtype=np.uint64)
    rec, pairs = pr.records(), pr.pair_array()
    rc = _lib().orc_merge_ed25519(O._ptr(lde_cols), lay.width, O._ptr(rec), rec.shape[0], O._ptr(pairs),
                                  pairs.shape[0], pr.n, n_trace, blowup, O._ptr(out))
    assert rc == 0, rc
    return out


def prove(lay, pr, tr, fs_binding: bytes, blowup: int = BLOWUP) -> bytes:
    tr = np.ascontiguousarray(tr, dtype=np.uint64)
    rec, pairs = pr.records(), pr.pair_array()
    cap = 1 << 24
    buf = ctypes.create_string_buffer(cap)
    ln = ctypes.c_size_t()
    rc = _lib().orc_prove_ed25519(O._ptr(tr), lay.width, O._ptr(rec), rec.shape[0], O._ptr(pairs), pairs.shape[0],
                                  pr.n, tr.shape[1], fs_binding, blowup, buf, cap, ctypes.byref(ln))
    assert rc == 0, rc
    return buf.raw[:ln.value]
