// ed25519_prover.hpp — Ed25519 verify AIR pipeline entry points used by the C ABI.
#pragma once
#include <cstdint>
#include <vector>

#include "context.hpp"
#include "ed25519.hpp"
#include "prover.hpp"

namespace sg {

// The width x height trace of a witness, expanded on the device.
void ed25519_trace_device(sg_ctx* c, const ed25519::Witness& w, uint64_t* d_trace);
// The LDE values the merge reads (make_lde_plan): the transform of the dense
// columns, then the constant and sparse columns filled where they are read; the
// other cells of d_lde (width x height*blowup) are left unwritten.
void ed25519_lde_device(sg_ctx* c, const ed25519::Witness& w, const uint64_t* d_trace, uint64_t blowup,
                        uint64_t* d_lde);
// Phi + quotient on a materialised (width x height*blowup) LDE.
void ed25519_merge_device(sg_ctx* c, const ed25519::Witness& w, const uint64_t* d_lde, uint64_t blowup,
                          uint64_t* d_c);
// The same without the LDE: coset by coset from the trace (the reference's
// deep_ali_merge_ed25519_verify_streaming, lib.rs:854-974).
void ed25519_merge_cosets(sg_ctx* c, const ed25519::Witness& w, const uint64_t* d_trace, uint64_t blowup,
                          uint64_t* d_c);
// prove_zsk_ksk_binding_v2 (swarm-dns/src/prover.rs:856-951) up to c_eval: witness,
// trace, LDE x blowup, merge; params = build_params(height * blowup, fs_binding).
CEval ed25519_ceval(sg_ctx* c, const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, uint64_t len,
                    const uint8_t fs_binding[32], uint32_t k_scalar, uint64_t blowup = 32);
std::vector<uint8_t> prove_ed25519(sg_ctx* c, const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg,
                                   uint64_t len, const uint8_t fs_binding[32], uint32_t k_scalar, bool self_verify,
                                   uint64_t blowup = 32);

}  // namespace sg
