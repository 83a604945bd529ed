// protocol.hpp — host-side Fiat-Shamir, query derivation and proof encoding.
//
// The transcript is a few dozen absorbs per proof and stays on the host; the
// byte layout must match the reference exactly:
//   transcript/src/lib.rs:13-17,158-213  SHA3-256 running hash with FSv1 tags;
//                                        challenges clone the state (non-mutating)
//   deep_ali/src/fri.rs:73-85            safe_field_challenge (7-byte chunks from the end)
//   deep_ali/src/fri.rs:1372-1392        challenge_ext ("tag/c{i}") / absorb_ext
//   deep_ali/src/fri.rs:1105-1129        statement binding
//   deep_ali/src/fri.rs:1044-1058        query index: ChaCha12 StdRng seeded by le8(seed)||0^24
//   deep_ali/src/fri.rs:1235-1300        DeepFriProof field order, ark-serialize Compress::Yes
//   merkle/src/lib.rs:135-140            MerkleOpening
#pragma once
#include <array>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "gl.cuh"
#include "keccak.cuh"
#include "stark_gpu.h"

namespace sg {

using Digest = std::array<uint8_t, kc::kHashBytes>;  // the build's hash profile

struct HostTranscript {
  kc::Sha3Sel h;  // new_matching_hash (transcript/src/lib.rs:338-344)
  explicit HostTranscript(const char* label) {
    static const char kInit[] = "FSv1-TRANSCRIPT-INIT";
    h.update(kInit, sizeof kInit - 1);
    h.update(label, strlen(label));
  }
  void absorb_bytes(const void* b, size_t n) {
    static const char kAbs[] = "FSv1-ABSORB-BYTES";
    h.update(kAbs, sizeof kAbs - 1);
    h.update(b, n);
  }
  void absorb_str(const char* s) { absorb_bytes(s, strlen(s)); }
  void absorb_field(uint64_t canonical) {
    uint8_t le[8];
    memcpy(le, &canonical, 8);
    absorb_bytes(le, 8);
  }
  void absorb_u64(uint64_t x) { absorb_field(x % gl::P); }
  void absorb_ext(const gl::Fp6& e) {
    for (int i = 0; i < 6; ++i) absorb_field(e.c[i]);
  }
  void challenge_bytes(const std::string& label, uint8_t out[kc::kHashBytes]) const {
    static const char kCh[] = "FSv1-CHALLENGE";
    kc::Sha3Sel c = h;
    c.update(kCh, sizeof kCh - 1);
    c.update(label.data(), label.size());
    c.finalize(out);
  }
  uint64_t challenge_field(const std::string& label) const {
    uint8_t d[kc::kHashBytes];
    challenge_bytes(label, d);
    uint64_t acc = 0;
    for (int end = kc::kHashBytes; end > 0;) {
      int start = end >= 7 ? end - 7 : 0, len = end - start;
      uint64_t v = 0;
      for (int i = 0; i < len; ++i) v |= (uint64_t)d[start + i] << (8 * i);
      acc = gl::add(gl::mul(acc, 1ull << (8 * len)), v % gl::P);
      end = start;
    }
    return acc;
  }
  gl::Fp6 challenge_ext(const std::string& tag) const {
    gl::Fp6 e;
    for (int i = 0; i < 6; ++i) e.c[i] = challenge_field(tag + "/c" + std::to_string(i));
    return e;
  }
};

inline void bind_statement(HostTranscript& tr, const sg_fri_params& p, uint64_t n0) {
  if (p.has_pi) {
    tr.absorb_str("CAIRO-PUBLIC-INPUTS-V1");
    tr.absorb_bytes(p.pi_hash, 32);
  }
  tr.absorb_str("DEEP-FRI-STATEMENT-V2");
  tr.absorb_u64(n0);
  tr.absorb_u64(p.schedule_len);
  for (uint64_t i = 0; i < p.schedule_len; ++i) tr.absorb_u64(p.schedule[i]);
  tr.absorb_u64(p.seed_z);
  tr.absorb_u64(6);  // E::DEGREE of the sextic extension
  tr.absorb_u64(p.coeff_commit_final ? 1 : 0);
  tr.absorb_u64(p.stir ? 1 : 0);
}

// ChaCha with 12 rounds, key = seed, 64-bit block counter 0, stream 0; first u64 of output.
inline uint64_t chacha12_first_u64(const uint8_t seed[32]) {
  uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u};
  for (int i = 0; i < 8; ++i) memcpy(&s[4 + i], seed + 4 * i, 4);
  for (int i = 12; i < 16; ++i) s[i] = 0;
  uint32_t x[16];
  memcpy(x, s, sizeof x);
  auto rl = [](uint32_t v, int r) { return (v << r) | (v >> (32 - r)); };
  auto qr = [&](int a, int b, int c, int d) {
    x[a] += x[b]; x[d] = rl(x[d] ^ x[a], 16);
    x[c] += x[d]; x[b] = rl(x[b] ^ x[c], 12);
    x[a] += x[b]; x[d] = rl(x[d] ^ x[a], 8);
    x[c] += x[d]; x[b] = rl(x[b] ^ x[c], 7);
  };
  for (int r = 0; r < 12; r += 2) {
    qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15);
    qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14);
  }
  return (uint64_t)(x[0] + s[0]) | ((uint64_t)(x[1] + s[1]) << 32);
}

// index_seed(query_seed, 0, q) -> index_from_seed(., n0_pow2) % n0
inline uint64_t query_index(uint64_t query_seed, uint64_t q, uint64_t n0) {
  HostTranscript tr("FRI/FS");
  tr.absorb_str("FRI/index");
  tr.absorb_field(query_seed);
  tr.absorb_field(0);
  tr.absorb_u64(q);
  uint64_t seed = tr.challenge_field("out");
  uint8_t sb[32] = {0};
  memcpy(sb, &seed, 8);
  uint64_t np2 = 1;
  while (np2 < n0) np2 <<= 1;
  return (chacha12_first_u64(sb) & (np2 - 1)) % n0;
}

inline uint64_t pick_arity_for_layer(uint64_t n, uint64_t m) {
  const uint64_t c[] = {128, 64, 32, 16, 8, 4};
  for (uint64_t a : c)
    if (m >= a && n % a == 0) return a;
  return n % 2 == 0 ? 2 : 1;
}
inline uint64_t merkle_depth(uint64_t leaves, uint64_t arity) {
  uint64_t d = 1, cur = leaves;
  while (cur > arity) {
    cur = (cur + arity - 1) / arity;
    ++d;
  }
  return d;
}
// MerkleChannelCfg used for STIR layer l (arity from (n, m)) and for the packed
// f0 / coefficient trees (requested arity 16), fri.rs:863,1071-1082,1508.
inline std::vector<uint32_t> layer_arities(uint64_t n, uint64_t m) {
  uint64_t a = pick_arity_for_layer(n, m);
  if (a < 2) a = 2;
  return std::vector<uint32_t>(merkle_depth(n, a), (uint32_t)a);
}

struct Opening {
  Digest leaf;
  std::vector<std::vector<Digest>> path;
  uint64_t index = 0;
};

struct ProxQuery {
  uint64_t base = 0, raw = 0;
  std::vector<uint64_t> fib_idx, fib_vals;
  Opening f0_open;
  gl::Fp6 f_next = gl::e_zero();
  bool has_l1 = false;
  Opening l1_open;
};

// classic FRI query (fri.rs:1236-1263): per-layer refs (i, child_pos,
// parent_index, parent_pos), payloads (f, s, q), the f0 opening, final index
struct ClassicQuery {
  std::vector<std::array<uint64_t, 4>> refs;
  std::vector<std::array<gl::Fp6, 3>> pay;
  Opening f0_open;
  uint64_t final_index = 0;
};

// DeepFriProof (fri.rs:1286-1300). `stir` selects which optional payload is
// present: STIR coset evaluations + proximity queries, or the classic layer
// openings, f0 openings and fold queries.
struct StirProof {
  bool stir = true;
  std::vector<std::vector<Opening>> layer_open;
  std::vector<Opening> f0_openings;
  std::vector<ClassicQuery> queries;
  Digest root_f0{};
  std::vector<Digest> roots;
  std::vector<gl::Fp6> fz;
  std::vector<gl::Fp6> final_coeffs;
  uint64_t n0 = 0;
  uint64_t omega0 = 0;
  bool has_ct = false;
  std::vector<std::vector<gl::Fp6>> coeff_tuples;
  bool has_croot = false;
  Digest coeff_root{};
  std::vector<std::vector<gl::Fp6>> coset_evals;
  std::vector<ProxQuery> prox;
};

struct ByteWriter {
  std::vector<uint8_t> b;
  void u8(uint8_t x) { b.push_back(x); }
  void u64(uint64_t x) {
    for (int i = 0; i < 8; ++i) b.push_back((uint8_t)(x >> (8 * i)));
  }
  void dig(const Digest& d) { b.insert(b.end(), d.begin(), d.end()); }
  void ext(const gl::Fp6& e) {
    for (int i = 0; i < 6; ++i) u64(e.c[i]);
  }
  void opening(const Opening& o) {
    dig(o.leaf);
    u64(o.path.size());
    for (auto& lv : o.path) {
      u64(lv.size());
      for (auto& d : lv) dig(d);
    }
    u64(o.index);
  }
};

inline std::vector<uint8_t> encode_proof(const StirProof& pr) {
  ByteWriter w;
  w.dig(pr.root_f0);
  w.u64(pr.roots.size());
  for (auto& r : pr.roots) w.dig(r);
  w.u64(pr.layer_open.size());  // layer_proofs.layers (classic FRI)
  for (auto& lo : pr.layer_open) {
    w.u64(lo.size());
    for (auto& o : lo) w.opening(o);
  }
  w.u64(pr.f0_openings.size());
  for (auto& o : pr.f0_openings) w.opening(o);
  w.u64(pr.queries.size());
  for (auto& q : pr.queries) {
    w.u64(q.refs.size());
    for (auto& r : q.refs)
      for (int k = 0; k < 4; ++k) w.u64(r[k]);
    w.u64(q.pay.size());
    for (auto& pl : q.pay)
      for (int k = 0; k < 3; ++k) w.ext(pl[k]);
    w.opening(q.f0_open);
    w.u64(q.final_index);
  }
  w.u64(pr.fz.size());
  for (auto& e : pr.fz) w.ext(e);
  w.u64(pr.final_coeffs.size());
  for (auto& e : pr.final_coeffs) w.ext(e);
  w.u64(pr.n0);
  w.u64(pr.omega0);
  w.u8(pr.has_ct);
  if (pr.has_ct) {
    w.u64(pr.coeff_tuples.size());
    for (auto& t : pr.coeff_tuples) {
      w.u64(t.size());
      for (auto& e : t) w.ext(e);
    }
  }
  w.u8(pr.has_croot);
  if (pr.has_croot) w.dig(pr.coeff_root);
  w.u8(pr.stir);  // stir_coset_evals: Some only for STIR
  if (!pr.stir) {
    w.u8(0);  // stir_proximity_queries: None
    return w.b;
  }
  w.u64(pr.coset_evals.size());
  for (auto& v : pr.coset_evals) {
    w.u64(v.size());
    for (auto& e : v) w.ext(e);
  }
  w.u8(1);
  w.u64(pr.prox.size());
  for (auto& q : pr.prox) {
    w.u64(q.base);
    w.u64(q.raw);
    w.u64(q.fib_idx.size());
    for (auto i : q.fib_idx) w.u64(i);
    w.u64(q.fib_vals.size());
    for (auto v : q.fib_vals) w.u64(v);
    w.opening(q.f0_open);
    w.ext(q.f_next);
    w.u8(q.has_l1);
    if (q.has_l1) w.opening(q.l1_open);
  }
  return w.b;
}

struct ByteReader {
  const uint8_t* p;
  size_t n, o = 0;
  ByteReader(const uint8_t* pp, size_t nn) : p(pp), n(nn) {}
  void need(size_t k) {
    if (k > n - o) throw std::runtime_error("proof truncated");
  }
  uint8_t u8() {
    need(1);
    return p[o++];
  }
  uint64_t u64() {
    need(8);
    uint64_t x;
    memcpy(&x, p + o, 8);
    o += 8;
    return x;
  }
  uint64_t len() {
    uint64_t x = u64();
    if (x > n) throw std::runtime_error("implausible length");
    return x;
  }
  Digest dig() {
    need(kc::kHashBytes);
    Digest d;
    memcpy(d.data(), p + o, kc::kHashBytes);
    o += kc::kHashBytes;
    return d;
  }
  uint64_t fe() {
    uint64_t x = u64();
    if (x >= gl::P) throw std::runtime_error("non-canonical field element");
    return x;
  }
  gl::Fp6 ext() {
    gl::Fp6 e;
    for (int i = 0; i < 6; ++i) e.c[i] = fe();
    return e;
  }
  bool flag() {
    uint8_t f = u8();
    if (f > 1) throw std::runtime_error("bad option flag");
    return f == 1;
  }
  Opening opening() {
    Opening op;
    op.leaf = dig();
    uint64_t nl = len();
    for (uint64_t i = 0; i < nl; ++i) {
      uint64_t ns = len();
      std::vector<Digest> v(ns);
      for (auto& d : v) d = dig();
      op.path.push_back(std::move(v));
    }
    op.index = u64();
    return op;
  }
};

inline StirProof decode_proof(const uint8_t* b, size_t n) {
  ByteReader r(b, n);
  StirProof pr;
  pr.root_f0 = r.dig();
  uint64_t k = r.len();
  for (uint64_t i = 0; i < k; ++i) pr.roots.push_back(r.dig());
  k = r.len();
  for (uint64_t i = 0; i < k; ++i) {
    uint64_t m = r.len();
    std::vector<Opening> lo;
    for (uint64_t j = 0; j < m; ++j) lo.push_back(r.opening());
    pr.layer_open.push_back(std::move(lo));
  }
  k = r.len();
  for (uint64_t i = 0; i < k; ++i) pr.f0_openings.push_back(r.opening());
  k = r.len();
  for (uint64_t i = 0; i < k; ++i) {
    ClassicQuery q;
    uint64_t m = r.len();
    for (uint64_t j = 0; j < m; ++j) {
      std::array<uint64_t, 4> ref;
      for (auto& x : ref) x = r.u64();
      q.refs.push_back(ref);
    }
    m = r.len();
    for (uint64_t j = 0; j < m; ++j) {
      std::array<gl::Fp6, 3> pl;
      for (auto& e : pl) e = r.ext();
      q.pay.push_back(pl);
    }
    q.f0_open = r.opening();
    q.final_index = r.u64();
    pr.queries.push_back(std::move(q));
  }
  k = r.len();
  for (uint64_t i = 0; i < k; ++i) pr.fz.push_back(r.ext());
  k = r.len();
  for (uint64_t i = 0; i < k; ++i) pr.final_coeffs.push_back(r.ext());
  pr.n0 = r.u64();
  pr.omega0 = r.fe();
  pr.has_ct = r.flag();
  if (pr.has_ct) {
    k = r.len();
    for (uint64_t i = 0; i < k; ++i) {
      uint64_t m = r.len();
      std::vector<gl::Fp6> t(m);
      for (auto& e : t) e = r.ext();
      pr.coeff_tuples.push_back(std::move(t));
    }
  }
  pr.has_croot = r.flag();
  if (pr.has_croot) pr.coeff_root = r.dig();
  pr.stir = r.flag();
  if (!pr.stir) {
    if (r.flag()) throw std::runtime_error("proximity queries without coset evaluations");
    if (r.o != n) throw std::runtime_error("trailing bytes");
    return pr;
  }
  k = r.len();
  for (uint64_t i = 0; i < k; ++i) {
    uint64_t m = r.len();
    std::vector<gl::Fp6> v(m);
    for (auto& e : v) e = r.ext();
    pr.coset_evals.push_back(std::move(v));
  }
  if (!r.flag()) throw std::runtime_error("missing stir_proximity_queries");
  k = r.len();
  for (uint64_t i = 0; i < k; ++i) {
    ProxQuery q;
    q.base = r.u64();
    q.raw = r.u64();
    uint64_t m = r.len();
    q.fib_idx.resize(m);
    for (auto& x : q.fib_idx) x = r.u64();
    m = r.len();
    q.fib_vals.resize(m);
    for (auto& x : q.fib_vals) x = r.fe();
    q.f0_open = r.opening();
    q.f_next = r.ext();
    q.has_l1 = r.flag();
    if (q.has_l1) q.l1_open = r.opening();
    pr.prox.push_back(std::move(q));
  }
  if (r.o != n) throw std::runtime_error("trailing bytes");
  return pr;
}

}  // namespace sg
