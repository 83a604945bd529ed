/* oracle/oracle.h — C API of the CPU oracle (ctypes-callable).
 *
 * TEST INFRASTRUCTURE ONLY. The oracle is a CPU restatement of the
 * stark-stir-swarm prover path (LDE -> DEEP-ALI merge -> STIR) used to check
 * the GPU library. Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it. All element buffers are canonical u64 Goldilocks
 * values; trace/LDE buffers are column-major (column c at c*n).
 * Return codes: 0 ok, negative on error.
 */
#ifndef STARK_ORACLE_H
#define STARK_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_SCHEDULE 64

/* Mirrors DeepFriParams (deep_ali/src/fri.rs:1303-1314). */
typedef struct {
  uint64_t schedule[ORC_MAX_SCHEDULE];
  uint64_t schedule_len;
  uint64_t r;
  uint64_t s0;
  uint64_t seed_z;
  uint64_t d_final;
  int32_t coeff_commit_final;
  int32_t stir;
  int32_t has_pi;
  uint8_t pi_hash[32];
} orc_fri_params;

/* Φ gating, deep_ali/src/lib.rs:20-33,372-397:
 * 0 = reference built with feature "parallel" on >1 rayon thread: Φ computed only if n >= 4096
 * 1 = Φ always computed (build without "parallel")
 * 2 = Φ never computed (feature "parallel" with one rayon thread) */
#define ORC_PHI_PARALLEL_GATE 0
#define ORC_PHI_ALWAYS 1
#define ORC_PHI_NEVER 2

#define ORC_AIR_HASH_ROLLUP 4
#define ORC_AIR_SHA256 6

/* field / extension / primitive checks (known-answer tests) */
uint64_t orc_fp_add(uint64_t a, uint64_t b);
uint64_t orc_fp_sub(uint64_t a, uint64_t b);
uint64_t orc_fp_mul(uint64_t a, uint64_t b);
uint64_t orc_fp_pow(uint64_t a, uint64_t e);
uint64_t orc_fp_inv(uint64_t a);
void orc_fp6_mul(const uint64_t a[6], const uint64_t b[6], uint64_t out[6]);
int orc_fp6_inv(const uint64_t a[6], uint64_t out[6]);
void orc_chacha_block(const uint8_t key[32], uint64_t counter, uint64_t stream, int rounds, uint32_t out[16]);

void orc_set_threads(int n);
int orc_get_threads(void);
int orc_ntt(uint64_t* a, size_t n, int inverse);
int orc_lde(const uint64_t* trace, size_t w, size_t n_trace, size_t blowup, uint64_t shift, uint64_t* out);
void orc_sha3_256(const uint8_t* msg, size_t len, uint8_t out[32]);
uint64_t orc_stdrng_first_u64(const uint8_t seed[32]);
uint64_t orc_root_of_unity(unsigned log_n);
/* Digest bytes of this build's hash profile (32, 48 or 64: SHA3-256/384/512). */
int orc_hash_bytes(void);
/* SHA3 of this build's profile; out: orc_hash_bytes() bytes. */
void orc_sha3_selected(const uint8_t* msg, size_t len, uint8_t* out);
/* root: orc_hash_bytes() bytes */
int orc_merkle_root(const uint64_t* rows, size_t n_leaves, size_t width, const uint64_t* arities, size_t depth,
                    uint64_t label, uint8_t* root);
int orc_hash_rollup_trace(const uint64_t* leaves, size_t n_leaves, size_t n_trace, uint64_t* trace);
int orc_merge(int air, const uint64_t* lde, size_t w, size_t n_trace, size_t blowup, const uint64_t* lambdas,
              size_t k, int phi_mode, uint64_t* c_eval);
int orc_poly_div_zh(const uint64_t* coeffs, size_t n, size_t m, uint64_t* q);
int orc_merge_sha256(const uint64_t* lde, size_t n_trace, size_t blowup, const uint64_t* lambdas, size_t n_blocks,
                     int phi_mode, uint64_t* c_eval);
int orc_sha256_trace(const uint8_t* msg, size_t len, uint64_t* out, size_t cap_elems, size_t* height,
                     size_t* n_blocks);
int orc_sha256_eval(const uint64_t* cur, const uint64_t* nxt, size_t row, size_t n_blocks, uint64_t* out);
int orc_merge_sha512(const uint64_t* lde, size_t n_trace, size_t blowup, const uint64_t* lambdas, size_t n_blocks,
                     int phi_mode, uint64_t* c_eval);
int orc_sha512_trace(const uint8_t* msg, size_t len, uint64_t* out, size_t cap_elems, size_t* height,
                     size_t* n_blocks);
int orc_sha512_eval(const uint64_t* cur, const uint64_t* nxt, size_t row, size_t n_blocks, uint64_t* out);
/* The SHA-256 / SHA-512 AIR proofs at LDE blowup `blowup` (32 in the reference's
 * prove_ds_ksk_binding; any power of two >= 2). */
int orc_prove_sha512(const uint8_t* msg, size_t len, const uint8_t fs_binding[32], int phi_mode, size_t blowup,
                     uint8_t* out, size_t cap, size_t* out_len, uint8_t digest[64]);
int orc_prove_sha256(const uint8_t* msg, size_t len, const uint8_t fs_binding[32], int phi_mode, size_t blowup,
                     uint8_t* out, size_t cap, size_t* out_len, uint8_t digest[32]);
/* RSA-2048 exponentiation AIR (rsa2048_exp_air.rs), n_records records side by side
 * (rsa2048_stacked_air.rs): 11041 cells and 11280 constraints per record. */
int orc_rsa_eval(const uint64_t* cur, const uint64_t* nxt, size_t row, size_t n_trace, size_t n_records,
                 uint64_t* out);
int orc_merge_rsa(const uint64_t* lde, size_t n_records, size_t n_trace, size_t blowup, uint64_t* c_eval);
int orc_prove_rsa(const uint64_t* trace, size_t n_records, size_t n_trace, const uint8_t pi[32], size_t blowup,
                  uint8_t* out, size_t cap, size_t* out_len);
/* P-256 ECDSA double-chain AIR (p256_ecdsa_double_multirow_air.rs): the row is a
 * gadget table (8 u64 per gadget, constraint order) plus an 18-entry tail of chain
 * bases. orc_p256_eval returns the number of constraint values written. */
int orc_p256_eval(const uint64_t* cur, const uint64_t* nxt, size_t row, size_t n_trace, const uint64_t* table,
                  size_t n_gadgets, const uint64_t* tail, uint64_t* out);
int orc_merge_p256(const uint64_t* lde, size_t width, const uint64_t* table, size_t n_gadgets,
                   const uint64_t* tail, size_t n_trace, size_t blowup, uint64_t* c_eval);
int orc_prove_p256(const uint64_t* trace, size_t width, const uint64_t* table, size_t n_gadgets,
                   const uint64_t* tail, size_t n_trace, const uint8_t pi[32], size_t blowup, uint8_t* out,
                   size_t cap, size_t* out_len);
/* Ed25519 verify AIR v16 (ed25519_verify_air.rs): the row's constraint vector is a
 * program of 16-u64 block records (row gate, kind, cell bases) plus a table of
 * A - B pairs (see ed25519_air.hpp); n_constraints is its length. */
int orc_ed25519_eval(const uint64_t* cur, const uint64_t* nxt, size_t row, const uint64_t* recs, size_t n_recs,
                     const uint64_t* pairs, size_t n_pairs, uint64_t* out);
int orc_merge_ed25519(const uint64_t* lde, size_t width, const uint64_t* recs, size_t n_recs, const uint64_t* pairs,
                      size_t n_pairs, size_t n_constraints, size_t n_trace, size_t blowup, uint64_t* c_eval);
int orc_prove_ed25519(const uint64_t* trace, size_t width, const uint64_t* recs, size_t n_recs,
                      const uint64_t* pairs, size_t n_pairs, size_t n_constraints, size_t n_trace,
                      const uint8_t fs_binding[32], size_t blowup, uint8_t* out, size_t cap, size_t* out_len);
void orc_build_params(size_t n0, const uint8_t pi[32], int stir, orc_fri_params* out);
int orc_stir_prove(const uint64_t* f0, size_t n0, const orc_fri_params* p, uint8_t* out, size_t cap, size_t* len);
int orc_stir_verify(const uint8_t* proof, size_t len, const orc_fri_params* p);
/* prove_inner_shard / prove_outer_rollup core: HashRollup trace over `leaves`
 * -> LDE(blowup 32) -> merge -> STIR, params = build_params(n0, pi, stir). */
int orc_prove_hash_rollup(const uint64_t* leaves, size_t n_leaves, const uint8_t pi[32], int phi_mode,
                          uint8_t* out, size_t cap, size_t* len);

#ifdef __cplusplus
}
#endif
#endif
