/* stark_gpu.h — C ABI of the B200 (sm_100a) STARK prover path of stark-stir-swarm.
 *
 * Drop-in boundary for the reference prover core (paths relative to
 * stark-stir-swarm/crates/): trace LDE -> DEEP-ALI merge -> STIR prove, plus
 * the SHA3-256 Merkle channel and the STIR verifier. A Rust caller binds these
 * with `extern "C"` and converts its 16-byte Montgomery `Goldilocks` values to
 * canonical u64 (into_bigint().0[0]) at the boundary.
 *
 * Conventions
 *  - Field elements are canonical little-endian u64 in [0, p), p = 2^64 - 2^32 + 1.
 *  - Column-major matrices: column c occupies [c*n, (c+1)*n).
 *  - Element buffers may live in host memory or in device memory of the
 *    context's GPU; the library detects which (cudaPointerGetAttributes).
 *    Host buffers are staged through the device inside the call.
 *  - Every call is ordered on the context's stream and returns when its
 *    results are available to the caller (host results are written back).
 *  - Return 0 on success, a negative SG_E* code on error; nothing aborts.
 *    sg_last_error() gives a human-readable reason for the last failure.
 *  - A context is not thread-safe; use one context per host thread/stream.
 */
#ifndef STARK_GPU_H
#define STARK_GPU_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SG_OK 0
#define SG_EINVAL -1    /* bad argument (shape, power-of-two, schedule ...) */
#define SG_ECUDA -2     /* CUDA runtime error */
#define SG_ENOMEM -3    /* device allocation failed */
#define SG_ESPACE -4    /* output buffer too small; *len holds the needed size */
#define SG_EVERIFY -5   /* self-verification of a produced proof failed */
#define SG_ELIMIT -6    /* request exceeds the fixed scratch of sg_ntt_noalloc */
#define SG_ETIMEDOUT -7 /* sg_server_wait_for: the job did not finish within the time limit */
#define SG_ECANCELED -8 /* the job was cancelled (sg_server_cancel) */

#define SG_MAX_SCHEDULE 64

/* Mirrors DeepFriParams (deep_ali/src/fri.rs:1303-1314). */
typedef struct {
  uint64_t schedule[SG_MAX_SCHEDULE];
  uint64_t schedule_len;
  uint64_t r;                 /* classic-FRI query count (unused by STIR) */
  uint64_t s0;                /* STIR proximity queries */
  uint64_t seed_z;
  uint64_t d_final;
  int32_t coeff_commit_final; /* bool */
  int32_t stir;               /* bool: STIR (1) or classic DEEP-FRI (0) */
  int32_t has_pi;             /* bool: public_inputs_hash is Some */
  uint8_t pi_hash[32];
} sg_fri_params;

/* Phi gating of the reference merges (deep_ali/src/lib.rs:20-33, 372-397). */
#define SG_PHI_PARALLEL_GATE 0 /* feature "parallel", >1 rayon thread: Phi = 0 unless n >= 4096 */
#define SG_PHI_ALWAYS 1        /* built without "parallel": Phi always computed */
#define SG_PHI_NEVER 2         /* feature "parallel" with one rayon thread: Phi = 0 */

/* AIR ids follow deep_ali::air_workloads::AirType's declaration order. */
#define SG_AIR_HASH_ROLLUP 4
#define SG_AIR_SHA256 6 /* Sha256DsKsk: 756 columns, 766 constraints */

typedef struct sg_ctx sg_ctx;
typedef struct sg_tree sg_tree;

/* Context: one CUDA device + stream + twiddle tables + a stream-ordered pool. */
int sg_ctx_create(int device, sg_ctx** out);
void sg_ctx_destroy(sg_ctx* ctx);
/* Use an existing cudaStream_t (passed as void*) for all later calls; NULL = the context's own stream. */
int sg_ctx_set_stream(sg_ctx* ctx, void* cuda_stream);
const char* sg_last_error(const sg_ctx* ctx);
/* Context options.
 * SG_OPT_WIDE_MERGE selects how sg_prove_sha256 / sg_prove_sha512 / sg_prove_p256_ecdsa (and the
 * server's jobs of those kinds) evaluate their AIR over the LDE:
 *   SG_WIDE_MERGE_LDE     materialise the 756- (1510-, 151,334-) column LDE, then evaluate (fewest launches);
 *   SG_WIDE_MERGE_COSETS  never store the LDE: for each of the `blowup` cosets r, evaluate
 *                         all columns on r*<w_n0^blowup> (coefficients twisted by w_n0^{rk},
 *                         one n_trace-point NTT per column) and fold the constraints of that
 *                         coset straight into Phi (row i+blowup of the LDE is the next point
 *                         of the same coset) -- memory 3 x trace instead of blowup x trace;
 *   SG_WIDE_MERGE_AUTO    (default) cosets once the LDE would exceed 2 GiB; for
 *                         sg_prove_ed25519 always the LDE, of which only the
 *                         columns read on most rows are transformed.
 * Both give bit-identical results. */
#define SG_OPT_WIDE_MERGE 1
/* SG_OPT_STIR_GROUP (1 .. 64, default 1): servers (and sg_prove_batch) created
 * from this context let a worker take up to this many queued jobs whose proofs
 * have the same domain n0 (any kinds except HashRollup) and prove their STIR
 * phase in lockstep (sg_stir_prove_group: one launch per stage for the group, one
 * host round trip per fold layer). Each job's trace, LDE and constraint merge
 * still run on their own; every proof's bytes are unchanged. */
#define SG_OPT_STIR_GROUP 2
#define SG_WIDE_MERGE_AUTO 0
#define SG_WIDE_MERGE_LDE 1
#define SG_WIDE_MERGE_COSETS 2
int sg_ctx_set_option(sg_ctx* ctx, int option, int64_t value);

/* Grow the device's stream-ordered memory pool (which keeps freed memory) to at
 * least `bytes`, capped at the device's free memory less 2 GiB, with one
 * allocation freed at once; later proofs sub-allocate from it instead of growing
 * the pool while other streams' kernels run, which stalls them. Best effort:
 * SG_OK also when the cap leaves nothing to reserve. sg_server_create calls it
 * with the server's HBM budget. */
int sg_pool_reserve(sg_ctx* ctx, uint64_t bytes);

/* Number of kernels this library has launched in this process (instrumentation). */
uint64_t sg_kernel_launches(const sg_ctx* ctx);

/* Per-kernel-family timing (instrumentation, no reference counterpart): while
 * enabled, every launch is bracketed by a CUDA event pair on its own stream.
 * sg_profile_read waits for the pending events and reports, per family, the
 * number of launches and the summed device time since the last reset. */
typedef struct {
  char name[48];
  uint64_t launches;
  double total_ms;
} sg_profile_entry;
int sg_profile_enable(int on);
int sg_profile_read(sg_profile_entry* out, size_t cap, size_t* n);
void sg_profile_reset(void);

/* Batched NTT with ark-poly Radix2EvaluationDomain semantics: forward = evaluations
 * at w^0..w^{n-1} (natural order), inverse includes 1/n; w = 7^((p-1)/2^32)
 * squared (32 - log_n) times. n_cols columns of 2^log_n, log_n <= 28.
 * Replaces the domain.fft / domain.ifft calls of trace_import.rs:276-279 and
 * lib.rs:402-410. in == out allowed. */
int sg_ntt(sg_ctx* ctx, const uint64_t* in, uint64_t* out, size_t n_cols, size_t log_n, int inverse);

/* sg_ntt for callers that must not have this library allocate device memory
 * (no counterpart in the reference, which allocates freely on the host): for
 * example a serving process that has already split all of HBM between its
 * jobs, a host framework whose own allocator owns every device buffer, or a
 * latency-critical loop that cannot afford cudaMalloc's device-wide sync.
 * Same transform and results as sg_ntt, but no context and no allocation:
 * the buffer between the two passes of a transform longer than 2^12 and the
 * twiddle table are static device arrays (8 MiB + 576 KiB, held by every GPU
 * that loads the library until exit).
 *  - in/out: device pointers on the current device (in == out allowed);
 *    host pointers and memory of another GPU are rejected with SG_EINVAL.
 *    The library cannot see a buffer's length: in and out must each hold
 *    n_cols * 2^log_n elements.
 *  - limit: for log_n > 12, n_cols * 2^log_n must be <= 2^20, else SG_ELIMIT;
 *    log_n <= 12 needs no scratch and has no limit.
 *  - the first call on a device sets it up (cudaGetSymbolAddress of the static
 *    arrays and a synchronous copy of the twiddle table), so make that first
 *    call before any stream capture. Every call resolves the arrays' addresses
 *    again and compares the current context's id with the one it set up in:
 *    after cudaDeviceReset the next call repeats the set-up (and its copy).
 *  - every call shares the one static buffer: calls whose kernels can overlap
 *    on the GPU (different streams, no ordering between them) race; order
 *    them on one stream or synchronize between them.
 *  - cuda_stream: a cudaStream_t as void*, NULL for the legacy default stream.
 *    The call returns after enqueueing; results are ordered on that stream. */
int sg_ntt_noalloc(const uint64_t* in, uint64_t* out, size_t n_cols, size_t log_n, int inverse, void* cuda_stream);

/* Replaces lde_trace_columns (deep_ali/src/trace_import.rs:251-281): each of the
 * w columns (n_trace rows, column-major) -> iFFT, zero-pad to n_trace*blowup,
 * FFT. shift = 1 reproduces the reference (plain subgroup); another shift
 * evaluates on the coset shift*<w>. out: w x (n_trace*blowup). */
int sg_lde(sg_ctx* ctx, const uint64_t* trace, size_t w, size_t n_trace, size_t blowup, uint64_t shift,
           uint64_t* out);

/* Replaces deep_ali_merge_general (deep_ali/src/lib.rs:343-437) for the AIRs
 * listed above: Phi_i = sum_j lambda_j C_j(row i, row (i+blowup) mod n),
 * c = FFT_n(iFFT_n(Phi) / (X^n_trace - 1)), remainder dropped as in release
 * builds (lib.rs:190-228). lde: w x n (n = n_trace*blowup); c_eval: n values. */
int sg_merge(sg_ctx* ctx, int air, const uint64_t* lde, size_t w, size_t n_trace, size_t blowup,
             const uint64_t* lambdas, size_t k, int phi_mode, uint64_t* c_eval);

/* Replaces deep_ali_merge_sha256 (deep_ali/src/lib.rs:453-545): the SHA-256 AIR
 * (eval_sha256_constraints, sha256_air.rs:956-1294) with an explicit block count
 * gating its phases. lde: 756 x (n_trace*blowup); lambdas: 766 values (host). */
int sg_merge_sha256(sg_ctx* ctx, const uint64_t* lde, size_t n_trace, size_t blowup, const uint64_t* lambdas,
                    size_t n_blocks, int phi_mode, uint64_t* c_eval);

/* Replaces build_sha256_trace_multi (deep_ali/src/sha256_air.rs:429-472), host only:
 * FIPS 180-4 padding, 128 rows per block, height = next power of two, last useful
 * row replicated. Writes 756 x height column-major into `trace` (cap in elements),
 * the block count, and the 32-byte digest carried in the H-state. */
int sg_sha256_trace(const uint8_t* msg, size_t len, uint64_t* trace, size_t cap, size_t* height, size_t* n_blocks,
                    uint8_t digest[32]);

/* The same trace (build_sha256_trace_multi, sha256_air.rs:429-472) with the
 * column expansion on the device: the host runs only the compressions and ships
 * one 2368-byte witness per block; `trace` (756 x height elements, host or device)
 * receives the cells. SG_ESPACE (height, n_blocks, digest still set) when cap is
 * too small. */
int sg_sha256_trace_gpu(sg_ctx* ctx, const uint8_t* msg, size_t len, uint64_t* trace, size_t cap, size_t* height,
                        size_t* n_blocks, uint8_t digest[32]);

/* Core of prove_ds_ksk_binding (swarm-dns/src/prover.rs:512-585): SHA-256 AIR trace
 * of `msg` -> LDE x32 -> merge (lambda_j = j+1) -> STIR with
 * build_params(n0, fs_binding). Self-verified before return; `digest` receives the
 * asserted SHA-256 digest read from the trace's H-state. */
int sg_prove_sha256(sg_ctx* ctx, const uint8_t* msg, size_t len, const uint8_t fs_binding[32], int phi_mode,
                    uint8_t* proof, size_t cap, size_t* len_out, uint8_t digest[32]);

/* Replaces deep_ali_merge_sha512 (deep_ali/src/lib.rs:561-641): the SHA-512 AIR
 * (eval_sha512_constraints, sha512_air.rs:909-1270; 64-bit words as 32-bit limb
 * pairs) with an explicit block count. lde: 1510 x (n_trace*blowup); lambdas:
 * 1526 values (host). */
int sg_merge_sha512(sg_ctx* ctx, const uint64_t* lde, size_t n_trace, size_t blowup, const uint64_t* lambdas,
                    size_t n_blocks, int phi_mode, uint64_t* c_eval);

/* Replaces build_sha512_trace_multi (deep_ali/src/sha512_air.rs:551-578), host
 * only: FIPS 180-4 §5.1.2 padding, 128 rows per block (80 rounds, post-state,
 * finalisation, idle), height = next power of two, last useful row replicated.
 * Writes 1510 x height column-major into `trace` (cap in elements), the block
 * count, and the 64-byte digest carried in the H-state. */
int sg_sha512_trace(const uint8_t* msg, size_t len, uint64_t* trace, size_t cap, size_t* height, size_t* n_blocks,
                    uint8_t digest[64]);
/* The same trace with the column expansion on the device (one 5888-byte witness
 * per block crosses PCIe); `trace` is host or device memory. */
int sg_sha512_trace_gpu(sg_ctx* ctx, const uint8_t* msg, size_t len, uint64_t* trace, size_t cap, size_t* height,
                        size_t* n_blocks, uint8_t digest[64]);

/* SHA-512 AIR proof of `msg`: trace -> LDE x32 -> merge_sha512 (lambda_j = j+1)
 * -> STIR with build_params(n0, fs_binding), self-verified. The reference has
 * the AIR and its merge but no SHA-512 prover yet (sha512_air.rs:16-19); this
 * uses the SHA-256 binding's parameters (swarm-dns/src/prover.rs:512-585).
 * `digest` receives the 64-byte digest read from the trace's H-state. */
int sg_prove_sha512(sg_ctx* ctx, const uint8_t* msg, size_t len, const uint8_t fs_binding[32], int phi_mode,
                    uint8_t* proof, size_t cap, size_t* len_out, uint8_t digest[64]);

/* Autotuner for the NTT's four-step split (sizes 2^13 .. 2^24, done in two passes
 * N = N1 * N2 with N1, N2 <= 2^12): times every split on a scratch transform of
 * min(n_cols, 2^26 / 2^log_n) columns (input zero-padded beyond n_valid, as in an
 * LDE, when n_valid < 2^log_n; 0 = none) and keeps the fastest for that size and
 * padding, for every later transform in the process (all splits give the same
 * output). best_log_n1 (optional) receives log N1 of the chosen split. Call it
 * before the timed or latency-sensitive work, like cuDNN's benchmark mode. */
int sg_ntt_autotune(sg_ctx* ctx, size_t n_cols, size_t log_n, int inverse, size_t n_valid, int* best_log_n1);
/* Set the split directly (a saved sg_ntt_autotune result; 0 = the default log N / 2):
 * SG_EINVAL unless 13 <= log_n <= 24 and max(1, log_n - 12) <= log_n1 <= min(12, log_n - 1). */
int sg_ntt_set_split(size_t log_n, int padded, int log_n1);

/* Hash profile of this build, the counterpart of the reference's compile-time hash
 * feature (hash/src/selected.rs:8-48): digest bytes of every Merkle node and of the
 * Fiat-Shamir transcript, so of every root in a proof. libstarkgpu.so is the
 * sha3-256 build (32), libstarkgpu_sha3_384.so 48, libstarkgpu_sha3_512.so 64.
 * Record hashing and the pi_hash recipes are SHA3-256 in every build, and the
 * swarm-dns shard entries (which bind 32-byte roots) need the sha3-256 build. */
int sg_hash_bytes(void);

/* Merkle commitment over the rows of a column-major matrix (leaf i = the
 * `width` values of row i), with the reference channel's framing
 * (merkle/src/lib.rs:95-238, 391-476): per-level arities, tree label, last-node
 * padding. root: sg_hash_bytes() bytes. `keep` (optional) receives a
 * device-resident tree for sg_merkle_open. */
int sg_merkle_commit(sg_ctx* ctx, const uint64_t* cols, size_t n_leaves, size_t width, size_t col_stride,
                     const uint64_t* arities, size_t depth, uint64_t tree_label, uint8_t* root, sg_tree** keep);
/* Serialized MerkleOpening (ark-serialize compressed: leaf[HASH_BYTES], path
 * Vec<Vec<[u8; HASH_BYTES]>>, index u64) for leaf `index` (merkle/src/lib.rs:478-512). */
int sg_merkle_open(sg_ctx* ctx, const sg_tree* tree, size_t index, uint8_t* out, size_t cap, size_t* len);
void sg_merkle_free(sg_tree* tree);

/* lde_trace_columns (deep_ali/src/trace_import.rs:251-281, with sg_lde's coset
 * shift) followed by the MerkleTreeChannel commitment to the rows of the LDE
 * (merkle/src/lib.rs:391-476; leaf i = row i of the w LDE columns), in one call:
 * the same root as sg_merkle_commit over sg_lde's output. With w a multiple of
 * 16 and a domain of at least 2^9, the forward transform's
 * last pass hashes the rows as it produces them and the LDE is never stored;
 * otherwise it is materialised on the device first. `out` receives the LDE's
 * first keep_cols columns (column stride n_trace * blowup; NULL when keep_cols is
 * 0), e.g. the column a STIR proof takes next. root: sg_hash_bytes() bytes;
 * `keep` (optional) receives the device-resident tree for sg_merkle_open. */
int sg_lde_commit(sg_ctx* ctx, const uint64_t* trace, size_t w, size_t n_trace, size_t blowup, uint64_t shift,
                  const uint64_t* arities, size_t depth, uint64_t tree_label, uint8_t* root, uint64_t* out,
                  size_t keep_cols, sg_tree** keep);

/* make_schedule + build_params (swarm-dns/src/prover.rs:53-98): schedule of 8s plus
 * a remainder for STIR (2s for FRI), r = s0 = 54, seed_z = 0xDEEF_BAAD,
 * coeff_commit_final, d_final = 1, public_inputs_hash = pi (NULL = None). */
void sg_build_params(size_t n0, const uint8_t* pi32, int stir, sg_fri_params* out);

/* Replaces deep_fri_prove::<SexticExt> (deep_ali/src/fri.rs:1900-2055) in both
 * branches, selected by params->stir: STIR (s0 proximity queries against the
 * coset-packed f0 tree) or classic DEEP-FRI (fri.rs:1724-1807: per-layer DEEP
 * quotients, r fold queries through every layer). Writes the exact ark-serialize
 * (Compress::Yes) bytes of the DeepFriProof. f0: n0 values. */
int sg_stir_prove(sg_ctx* ctx, const uint64_t* f0, size_t n0, const sg_fri_params* params, uint8_t* proof,
                  size_t cap, size_t* len);

/* n_proofs STIR proofs of one shape in lockstep (the reference proves one per
 * call; its swarm runs many shards side by side): the same n0 and parameters
 * except public_inputs_hash, f0 of proof g at f0 + g * n0. Every device stage is
 * one launch over all the proofs and each fold layer has one host round trip for
 * all of their transcripts. Proof g (the bytes of sg_stir_prove on its f0 and
 * params[g]) goes to proofs + g * cap_per_proof, its length to lens[g]. */
int sg_stir_prove_group(sg_ctx* ctx, const uint64_t* f0, size_t n0, size_t n_proofs, const sg_fri_params* params,
                        uint8_t* proofs, size_t cap_per_proof, size_t* lens);

/* Replaces deep_fri_verify::<SexticExt> (deep_ali/src/fri.rs:2136-2707), both
 * branches, on serialized proof bytes. Returns 1 accept, 0 reject. Host only. */
int sg_stir_verify(const uint8_t* proof, size_t len, const sg_fri_params* params);

/* Core of prove_inner_shard / prove_outer_rollup (swarm-dns/src/prover.rs:148-304):
 * HashRollup trace over `leaves` (n_trace = next_pow2(n_leaves) >= 8) -> LDE x32 ->
 * merge (lambda = 1,2,3) -> STIR with build_params(n0, pi). The proof is
 * self-verified before return (SG_EVERIFY on failure), like the reference worker. */
int sg_prove_hash_rollup(sg_ctx* ctx, const uint64_t* leaves, size_t n_leaves, const uint8_t pi[32], int phi_mode,
                         uint8_t* proof, size_t cap, size_t* len);

/* ---------------------------------------------------------------- RSA-2048 signature checks
 * RSASSA-PKCS1-v1_5 / SHA-256 (DNSSEC algorithm 8) proved as the e = 65537
 * exponentiation chain AIR (deep_ali/src/rsa2048_exp_air.rs): 32 rows of 11041
 * cells, each row one witness-quotient multiply modulo n
 * (rsa2048_field_air.rs), 16 squarings then the multiply by s on row 16, whose
 * output is bound to the encoded message EM; 11280 constraints per row. Several
 * records stack side by side in one trace (rsa2048_stacked_air.rs). All integers
 * are 256-byte big-endian (n, s = signature, em); arrays of records are
 * contiguous, 256 bytes per record. */

/* EMSA-PKCS1-v1_5 encoding of SHA-256(msg) for a 256-byte modulus
 * (deep_ali/src/rsa2048.rs:71-90, emsa_pkcs1_v1_5_encode_sha256). */
int sg_rsa2048_em(const uint8_t* msg, size_t len, uint8_t em[256]);
/* Native check s^65537 mod n == em with 0 < s < n (rsa2048.rs:92-127, verify).
 * Returns 1 valid, 0 invalid. */
int sg_rsa2048_verify(const uint8_t n_be[256], const uint8_t s_be[256], const uint8_t em[256]);
/* pi_hash of one record: SHA3-256("RSA2048-V2-PI-PRE" || n || s || msg || em)
 * (swarm-dns/examples/prove_rsa2048_record_v1.rs:178-187). */
int sg_rsa2048_pi_record(const uint8_t n_be[256], const uint8_t s_be[256], const uint8_t* msg, size_t len,
                         const uint8_t em[256], uint8_t out[32]);
/* pi_hash of a stacked zone under one key: SHA3-256("RSA2048-STACKED-ZONE" || n ||
 * le64(n_records) || em_0 || ... ) (swarm-dns/examples/stacked_rsa_zone_prover.rs:158-165). */
int sg_rsa2048_pi_stacked(const uint8_t n_be[256], size_t n_records, const uint8_t* ems, uint8_t out[32]);
/* fill_rsa_exp_multirow / fill_rsa_stacked (rsa2048_exp_air.rs:126-204,
 * rsa2048_stacked_air.rs:40-54) on the host: (n_records * 11041) x 32
 * column-major into `trace` (cap in elements). SG_EINVAL unless 1 < n and s < n. */
int sg_rsa2048_trace(const uint8_t* n_be, const uint8_t* s_be, const uint8_t* em_be, size_t n_records,
                     uint64_t* trace, size_t cap);
/* The same trace with the cells expanded on the device from per-row witnesses
 * (limbs, quotient, biased carries; 2.5 KB a row); `trace` is host or device memory. */
int sg_rsa2048_trace_gpu(sg_ctx* ctx, const uint8_t* n_be, const uint8_t* s_be, const uint8_t* em_be,
                         size_t n_records, uint64_t* trace, size_t cap);
/* deep_ali_merge_rsa_exp_multirow(_streaming) / deep_ali_merge_rsa_stacked_streaming
 * (deep_ali/src/lib.rs:1694-2070): Phi_i = sum_j (j + 1) C_j over the concatenated
 * constraints at every LDE point (always evaluated: this merge has no
 * parallel-build gate), then iFFT, poly_div_zh, FFT -> c_eval (n_trace * blowup
 * values). lde: (n_records * 11041) columns of n_trace * blowup, host or device. */
int sg_merge_rsa2048(sg_ctx* ctx, const uint64_t* lde, size_t n_records, size_t n_trace, size_t blowup,
                     uint64_t* c_eval);
/* RSA-2048 proof: witnesses (host) -> trace (device) -> LDE x32 -> RSA merge ->
 * STIR with build_params(1024, pi) (schedule [8,8,8,2]), self-verified. One
 * record is prove_rsa2048_record_v1.rs; several are stacked_rsa_zone_prover.rs.
 * The proof binds em only through the constraints: pass EM from sg_rsa2048_em
 * and check the signature with sg_rsa2048_verify first, as the reference does. */
int sg_prove_rsa2048(sg_ctx* ctx, const uint8_t* n_be, const uint8_t* s_be, const uint8_t* em_be, size_t n_records,
                     const uint8_t pi[32], uint8_t* proof, size_t cap, size_t* len);

/* ---------------------------------------------------------------- P-256 ECDSA signature checks
 * ECDSA-P256 (DNSSEC algorithm 13) proved as the double-chain scalar
 * multiplication AIR of deep_ali/src/p256_ecdsa_double_multirow_air.rs: each row
 * carries one step of chain A (u1·G) and one of chain B (u2·Q), a step being a
 * group double, an add of the chain's base point and a select on the row's bit
 * (p256_scalar_mul_air.rs, p256_group_air.rs), all written as field gadgets over
 * 10 limbs of 26 bits (p256_field_air.rs). 151,334 cells and 155,774 constraints
 * per row; the last row binds each chain's output to constant r_proj columns.
 * Coordinates, scalars and digests are 32-byte big-endian; bits are bytes 0/1. */

/* The row layout as a gadget table in constraint order (8 u32 per gadget:
 * kind 1 mul, 2 add, 3 sub, 4 freeze, 5 select, then its cell bases), and the 18
 * tail bases (chain A accumulator x,y,z, A output x,y,z, the same for B, r_proj
 * A x,y,z and B x,y,z). table may be NULL; cap is in gadgets. */
int sg_p256_layout(uint32_t* width, uint32_t* n_gadgets, uint32_t* n_constraints, uint32_t* table, size_t cap,
                   uint32_t tail[18]);
/* u1 = e s^-1, u2 = r s^-1 mod n (e = digest mod n) as MSB-first bits, the
 * chains' inputs (prove_ecdsa_record_v1.rs:97-118). SG_EINVAL unless 1 <= r, s < n. */
int sg_p256_u_bits(const uint8_t digest[32], const uint8_t r[32], const uint8_t s[32], uint8_t u1[256],
                   uint8_t u2[256]);
/* pi_hash SHA3-256("ECDSA-V1-PI-PRE" || qx || qy || r || s || digest)
 * (prove_ecdsa_record_v1.rs:213-222). */
int sg_p256_ecdsa_pi(const uint8_t qx[32], const uint8_t qy[32], const uint8_t r[32], const uint8_t s[32],
                     const uint8_t digest[32], uint8_t out[32]);
/* fill_ecdsa_double_multirow (p256_ecdsa_double_multirow_air.rs:134-234) on the
 * host: chain A starts at (ax, ay, 1) and takes a_bits, chain B at (bx, by, 1)
 * with b_bits, one bit per row, k rows (a power of 2, 2..65536); the r_proj
 * columns hold the chains' final points. width x k column-major into `trace`
 * (cap in elements). SG_EINVAL for a coordinate >= p or a point off the curve. */
int sg_p256_chain_trace(const uint8_t ax[32], const uint8_t ay[32], const uint8_t* a_bits, const uint8_t bx[32],
                        const uint8_t by[32], const uint8_t* b_bits, size_t k, uint64_t* trace, size_t cap);
/* The same trace with the cells expanded on the device from per-row gadget
 * witnesses (15 MB for k = 256 instead of the 310 MB trace); host or device output. */
int sg_p256_chain_trace_gpu(sg_ctx* ctx, const uint8_t ax[32], const uint8_t ay[32], const uint8_t* a_bits,
                            const uint8_t bx[32], const uint8_t by[32], const uint8_t* b_bits, size_t k,
                            uint64_t* trace, size_t cap);
/* deep_ali_merge_ecdsa_double_multirow_streaming: Phi_i = sum_j (j + 1) C_j at every
 * point of a (151,334 x n_trace*blowup) LDE (always evaluated), then iFFT,
 * poly_div_zh, FFT -> c_eval. lde: host or device. */
int sg_merge_p256_ecdsa(sg_ctx* ctx, const uint64_t* lde, size_t n_trace, size_t blowup, uint64_t* c_eval);
/* Proof of two chains of k rows: trace -> LDE x32 -> merge -> STIR with
 * build_params(32 k, pi), self-verified. */
int sg_prove_p256_chains(sg_ctx* ctx, const uint8_t ax[32], const uint8_t ay[32], const uint8_t* a_bits,
                         const uint8_t bx[32], const uint8_t by[32], const uint8_t* b_bits, size_t k,
                         const uint8_t pi[32], uint8_t* proof, size_t cap, size_t* len);
/* prove_ecdsa_record_v1.rs:97-240: u1/u2 from (digest, r, s), chain A = u1 bits
 * from G, chain B = u2 bits from the public key Q, K = 256 rows, blowup 32
 * (n0 = 8192, 9.9 GB LDE on the device), STIR with build_params(8192, pi),
 * self-verified. The reference checks the signature natively before proving
 * and finishes the verification (R = chain outputs combined, x(R) = r mod n)
 * natively; the caller does both here. */
int sg_prove_p256_ecdsa(sg_ctx* ctx, const uint8_t qx[32], const uint8_t qy[32], const uint8_t r[32],
                        const uint8_t s[32], const uint8_t digest[32], const uint8_t pi[32], uint8_t* proof,
                        size_t cap, size_t* len);

/* ---------------------------------------------------------------- Ed25519 signature checks
 * Ed25519 (RFC 8032) verification proved as the v16 verify AIR of
 * deep_ali/src/ed25519_verify_air.rs: the SHA-512 rows of R || A || M, the
 * reduction k = digest mod L, the decompressions of R and A, the [s]B and [k]A
 * ladders (k_scalar rows each), the residual [s]B - R - [k]A as two point
 * additions, three doublings and the identity verdict on [8] residual. Field
 * elements of 2^255 - 19 are 10 limbs of 26/25 bits with range bits and carries
 * (ed25519_field_air.rs). For k_scalar = 256 and a 32-byte message: 1024 rows,
 * 41,519 cells and 70,606 constraints per row; the proof's domain is 1024 x 32.
 * pub is the 32-byte public key A, sig the 64-byte signature R || S, msg the
 * signed data (the SHA-512 input is R || A || msg). Every entry refuses, with
 * SG_EINVAL, an R or A that does not decode (y >= p, off the curve, or x = 0 with
 * the sign bit set) and k_scalar outside [2, 256]. */

/* verify_air_layout_v16 (ed25519_verify_air.rs:4741-4814) for a msg_len-byte
 * message: trace width and height, constraints per row, and the rows of its
 * phases (k_hash, reduction, decompress R, decompress A, first [s]B row, first
 * [k]A row, residual, doubling 1, 2, 3, verdict). */
int sg_ed25519_layout(uint32_t k_scalar, size_t msg_len, uint32_t* width, uint32_t* height, uint32_t* n_constraints,
                      uint32_t rows[11]);
/* The row's constraint vector as a program (eval_verify_air_v16_per_row,
 * ed25519_verify_air.rs:4870-4960, through the v15 .. v0 evaluators): per block 16
 * u64 (row gate kind 0 every row / 1 row == g0 / 2 g0 <= row < g1 / 3 row in {g0,
 * g1, g2}; g0..g2; block kind 1 SHA-512, 2 scalar reduction, 3 digest format,
 * 4 mul, 5 add, 6 sub, 7 select, 8 range check, 9 sign bit, 10 A - B pairs; its
 * cell bases; ~0 in unused slots) and the pairs (2 u64 each: src << 62 | cell, src
 * 0 this row, 1 next row, 2 a constant). The public inputs fix the pinned
 * constants. recs / pairs may be NULL to read the counts (caps in records / pairs). */
int sg_ed25519_program(const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, size_t msg_len,
                       uint32_t k_scalar, uint64_t* recs, size_t cap_recs, size_t* n_recs, uint64_t* pairs,
                       size_t cap_pairs, size_t* n_pairs);
/* fill_verify_air_v16 (ed25519_verify_air.rs:4820-4868) for the signature on the
 * host: width x height column-major into `trace` (cap in elements). */
int sg_ed25519_trace(const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, size_t msg_len,
                     uint32_t k_scalar, uint64_t* trace, size_t cap);
/* The same trace with the cells expanded on the device from per-row words (about
 * 4 MB for k_scalar = 256 instead of the 340 MB trace); host or device output. */
int sg_ed25519_trace_gpu(sg_ctx* ctx, const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg,
                         size_t msg_len, uint32_t k_scalar, uint64_t* trace, size_t cap);
/* deep_ali_merge_ed25519_verify (lib.rs:707-838): Phi_i = sum_j (j + 1) C_j at every
 * point of a (width x height*blowup) LDE, each point evaluating the blocks its row
 * opens, then iFFT, poly_div_zh, FFT -> c_eval. The signature fixes the program's
 * constants. lde: host or device. */
int sg_merge_ed25519(sg_ctx* ctx, const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, size_t msg_len,
                     uint32_t k_scalar, const uint64_t* lde, size_t blowup, uint64_t* c_eval);
/* Proof: witness (host) -> trace (device) -> LDE x blowup of the columns the merge
 * reads (the others are filled only at the points that read them) -> merge ->
 * STIR with build_params(height * blowup, fs_binding), self-verified
 * (prove_zsk_ksk_binding_v2, swarm-dns/src/prover.rs:856-951, with blowup 32 and
 * k_scalar 256). The LDE buffer is width x height*blowup (10.9 GB for k_scalar
 * 256); SG_OPT_WIDE_MERGE = SG_WIDE_MERGE_COSETS streams the merge coset by coset
 * instead (about 1 GB, twice the time). */
int sg_prove_ed25519(sg_ctx* ctx, const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, size_t msg_len,
                     const uint8_t fs_binding[32], uint32_t k_scalar, size_t blowup, uint8_t* proof, size_t cap,
                     size_t* len);
/* RFC 8032 §5.1.7 cofactored verification (ed25519_verify.rs:54-117): 1 valid, 0 not,
 * a negative error code (SG_EINVAL, SG_ENOMEM) on a bad argument or failed allocation. */
int sg_ed25519_verify(const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, size_t msg_len);
/* zsk_ksk_pi_hash_v2_stark (swarm-dns/src/prover.rs:763-780): SHA3-256 of
 * "ZSK-KSK-PIHASH-V2-ST" || pub || sig || le64(msg_len) || msg || fs_binding ||
 * merkle_root || root_f0. */
int sg_ed25519_pi_hash(const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, size_t msg_len,
                       const uint8_t fs_binding[32], const uint8_t merkle_root[32], const uint8_t root_f0[32],
                       uint8_t out[32]);
/* prove_zsk_ksk_binding_v2 (swarm-dns/src/prover.rs:856-951): the signature is
 * checked natively first (SG_EVERIFY when it does not verify, before any proving),
 * then proved with k_scalar rows per ladder at blowup 32 and self-verified; pi_hash
 * binds the proof's root_f0. SHA3-256 hash profile only (the bundle holds 32-byte
 * roots), SG_EINVAL otherwise. */
int sg_prove_zsk_ksk_binding_v2(sg_ctx* ctx, const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg,
                                size_t msg_len, const uint8_t fs_binding[32], const uint8_t merkle_root[32],
                                uint32_t k_scalar, uint8_t* proof, size_t cap, size_t* len, uint8_t pi_hash[32]);

/* ---------------------------------------------------------------- DNS shards
 * The steps either side of the prover in swarm-dns. Records are passed in
 * canonical form (DnsRecord::canonical_bytes, swarm-dns/src/dns.rs:43-54):
 * record i is canon[offsets[i] .. offsets[i+1]), offsets has n+1 entries. */

/* DnsRecord::leaf_hash (dns.rs:56-79): SHA3("DNS-LEAF-DOUBLE-V1" || salt ||
 * SHA3("DNS-LEAF-V1" || salt || canonical)); out: n x 32 bytes. Host. */
int sg_dns_record_leaves(const uint8_t* canon, const size_t* offsets, size_t n, const uint8_t salt[16],
                         uint8_t* out);
/* merkle_build + merkle_root (dns.rs:85-102): binary SHA3 tree, parent =
 * SHA3("DNS-NODE-V1" || left || right), an odd last node paired with itself. Host. */
int sg_dns_merkle_root(const uint8_t* leaves, size_t n, uint8_t root[32]);
/* merkle_path (dns.rs:104-114): one 32-byte sibling per level; *depth receives
 * the level count (SG_ESPACE when cap < 32 * depth). Host. */
int sg_dns_merkle_path(const uint8_t* leaves, size_t n, size_t index, uint8_t* path, size_t cap, size_t* depth);
/* merkle_verify (dns.rs:116-131): 1 if the path leads from leaf to root. Host. */
int sg_dns_merkle_verify(const uint8_t leaf[32], size_t index, const uint8_t* path, size_t depth,
                         const uint8_t root[32]);
/* pi_hash of an inner shard (swarm-dns/src/prover.rs:207-214):
 * SHA3("DNS-SHARD-PIHASH-V1" || salt || le64(count) || merkle_root || root_f0 || fs_binding). Host. */
void sg_shard_pi_hash(const uint8_t salt[16], uint64_t record_count, const uint8_t merkle_root[32],
                      const uint8_t root_f0[32], const uint8_t fs_binding[32], uint8_t out[32]);
/* prove_inner_shard (swarm-dns/src/prover.rs:148-225): record leaves -> DNS Merkle
 * root -> leaves packed as 4 x le64 (pack_hash_to_leaves) -> HashRollup proof
 * (stir = 1: STIR, 0: classic DEEP-FRI; fs_binding as public_inputs_hash),
 * self-verified -> pi_hash. Outputs the proof bytes, pi_hash and merkle_root. */
int sg_prove_inner_shard(sg_ctx* ctx, const uint8_t* canon, const size_t* offsets, size_t n_records,
                         const uint8_t salt[16], const uint8_t fs_binding[32], int stir, uint8_t* proof, size_t cap,
                         size_t* len, uint8_t pi_hash[32], uint8_t merkle_root[32]);
/* prove_outer_rollup (swarm-dns/src/prover.rs:250-304): the inner pi_hashes
 * (n x 32 bytes) packed as rollup leaves, HashRollup proof under pk_hash. */
int sg_prove_outer_rollup(sg_ctx* ctx, const uint8_t* pi_hashes, size_t n, const uint8_t pk_hash[32], int stir,
                          uint8_t* proof, size_t cap, size_t* len);

/* ---------------------------------------------------------------- batched / served proving
 * No single reference function: the reference scales by running one proof per
 * worker process (swarm-worker/src/main.rs:341-355, driven by swarm-ctrl). Here
 * many proofs share one GPU: N worker threads, each with its own stream, take
 * jobs FIFO as soon as they are free (continuous batching); a job starts only
 * while the estimated device footprint of the running jobs plus its own fits
 * the HBM budget (0 = unlimited; a job larger than the budget runs alone).
 * Every proof is self-verified and byte-identical to the single-proof call. */
#define SG_JOB_SHA256 1      /* input = message bytes, input_len = bytes (sg_prove_sha256) */
#define SG_JOB_HASH_ROLLUP 2 /* input = u64 rollup leaves, input_len = count (sg_prove_hash_rollup) */
#define SG_JOB_SHA512 3      /* input = message bytes, input_len = bytes (sg_prove_sha512) */
#define SG_JOB_RSA2048 4     /* input = records of n || s || em (256 bytes each, big-endian), input_len =
                                768 * records (sg_prove_rsa2048; pi = public_inputs_hash) */
#define SG_JOB_P256_ECDSA 5  /* input = qx || qy || r || s || digest (32 bytes each), input_len = 160
                                (sg_prove_p256_ecdsa; pi = public_inputs_hash) */
#define SG_JOB_ED25519 6     /* input = pub (32) || sig (64) || msg, input_len = 96 + message bytes
                                (sg_prove_ed25519 with k_scalar 256; pi = fs_binding); the signature
                                is verified natively first (SG_EVERIFY when it does not verify) */

typedef struct {
  int32_t kind;
  int32_t phi_mode;
  const void* input;
  size_t input_len;
  uint8_t pi[32]; /* fs_binding / public_inputs_hash */
  /* LDE blowup of the proof: 0 = the reference prover's own (32); otherwise a
   * power of two in [2, 1024] (n0 = n_trace * blowup, STIR schedule
   * make_schedule(n0)). HashRollup jobs always use 32. */
  uint32_t blowup;
  /* SG_JOB_FAULT_* bits: host-side fault injection for tests of the serving
   * loop's failure handling (0 in production). No GPU work is made to fail:
   * the fault is raised on the host where the named call would have failed. */
  uint32_t flags;
} sg_job;
#define SG_JOB_FAULT_ALLOC 1u  /* the job's first attempt fails as if its device allocation had (SG_ENOMEM) */
#define SG_JOB_FAULT_VERIFY 2u /* one byte of the proof is flipped before self-verification (SG_EVERIFY) */

typedef struct {
  int32_t status; /* SG_OK or an SG_E* code */
  uint32_t reserved;
  size_t proof_len;
  uint8_t digest[64]; /* SHA-256 jobs: the asserted digest (32 bytes); SHA-512 jobs: 64 bytes; others: zero */
  double queue_ms;    /* submit -> start */
  double run_ms;      /* start -> proof ready */
  double latency_ms;  /* submit -> proof ready */
} sg_job_result;

typedef struct sg_server sg_server;
int sg_server_create(sg_ctx* ctx, int n_streams, uint64_t hbm_budget_bytes, sg_server** out);
void sg_server_destroy(sg_server* srv); /* waits for running jobs; queued jobs are dropped */
int sg_server_submit(sg_server* srv, const sg_job* job, uint64_t* ticket); /* copies the input */
int sg_server_poll(sg_server* srv, uint64_t ticket);                       /* 1 done, 0 pending */
/* Blocks until the job is done; copies the proof (cap bytes available) and releases
 * the ticket, except on SG_ESPACE, which keeps it so the caller can retry. */
int sg_server_wait(sg_server* srv, uint64_t ticket, sg_job_result* res, uint8_t* proof, size_t cap);
/* sg_server_wait with a time limit, the per-shard deadline of the reference's
 * controller (swarm-ctrl/src/main.rs:94-99): returns SG_ETIMEDOUT, keeping the
 * ticket, if the job is not done within timeout_ms (0 = poll once). */
int sg_server_wait_for(sg_server* srv, uint64_t ticket, int64_t timeout_ms, sg_job_result* res, uint8_t* proof,
                       size_t cap);
/* Cancels a job: a queued job is dropped before it starts (returns SG_OK); a
 * running one finishes on the GPU but its result is discarded (returns 1).
 * Either way its wait returns SG_ECANCELED. A job that had already finished
 * keeps its result (returns 2). Unknown tickets: SG_EINVAL. */
int sg_server_cancel(sg_server* srv, uint64_t ticket);
/* Re-queue a job whose attempt failed with a transient error (SG_ENOMEM or
 * SG_ECUDA) up to max_retries times, as the reference's controller reopens a
 * failed shard (swarm-ctrl/src/main.rs:1085). Default 0. A proof that fails
 * self-verification (SG_EVERIFY) is deterministic and is never retried. */
int sg_server_set_retries(sg_server* srv, int max_retries);
/* Proves n jobs with n_streams proofs in flight; proof i goes to proofs + i*cap_per_job. */
int sg_prove_batch(sg_ctx* ctx, const sg_job* jobs, size_t n, int n_streams, uint64_t hbm_budget_bytes,
                   uint8_t* proofs, size_t cap_per_job, sg_job_result* results);

#ifdef __cplusplus
}
#endif
#endif /* STARK_GPU_H */
