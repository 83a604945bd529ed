// oracle/transcript.hpp — CPU restatement of the SHA3-256 Fiat-Shamir transcript.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle; never linked into the product).
//
// Follows:
//   transcript/src/lib.rs:13-17     domain tags FSv1-TRANSCRIPT-INIT / -ABSORB-BYTES / -CHALLENGE
//   transcript/src/lib.rs:158-213   SHA3 backend: one running hash; absorb = update(tag||bytes);
//                                   challenge_bytes = clone, update(tag||label), finalize (non-mutating)
//   transcript/src/lib.rs:338-344   new_matching_hash -> SHA3-256 for HASH_BYTES=32
//   deep_ali/src/fri.rs:73-85       safe_field_challenge (rchunks(7) fold)
//   deep_ali/src/fri.rs:123-130     tr_hash_fields_tagged
//   deep_ali/src/fri.rs:1372-1392   challenge_ext / absorb_ext
#pragma once
#include <string>
#include "gl.hpp"
#include "keccak.hpp"

namespace orc {

struct Transcript {
  SelectedHasher h;
  explicit Transcript(const char* label) {
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
  void absorb_field(Fp x) {
    uint8_t le[8];
    memcpy(le, &x.v, 8);
    absorb_bytes(le, 8);
  }
  void absorb_u64(uint64_t x) { absorb_field(Fp(x)); }
  void absorb_ext(const Fp6& e) {
    for (int i = 0; i < 6; ++i) absorb_field(e.comp(i));
  }
  void challenge_bytes(const void* label, size_t n, uint8_t out[HASH_BYTES]) const {
    static const char kCh[] = "FSv1-CHALLENGE";
    SelectedHasher c = h;
    c.update(kCh, sizeof kCh - 1);
    c.update(label, n);
    c.finalize(out);
  }
  // safe_field_challenge: fold the digest's 7-byte chunks taken from the END.
  Fp challenge_field(const std::string& label) const {
    uint8_t d[HASH_BYTES];
    challenge_bytes(label.data(), label.size(), d);
    Fp acc;
    int end = HASH_BYTES;
    while (end > 0) {
      int start = end >= 7 ? end - 7 : 0;
      int len = end - start;
      uint64_t val = 0;
      for (int i = 0; i < len; ++i) val |= (uint64_t)d[start + i] << (8 * i);
      acc = acc * Fp::raw(1ull << (8 * len)) + Fp(val);
      end = start;
    }
    return acc;
  }
  Fp6 challenge_ext(const std::string& tag) const {
    Fp6 e;
    for (int i = 0; i < 6; ++i) e.set_comp(i, challenge_field(tag + "/c" + std::to_string(i)));
    return e;
  }
};

inline Fp hash_fields_tagged(const char* tag, const Fp* fields, size_t n) {
  Transcript tr("FRI/FS");
  tr.absorb_str(tag);
  for (size_t i = 0; i < n; ++i) tr.absorb_field(fields[i]);
  return tr.challenge_field("out");
}

}  // namespace orc
