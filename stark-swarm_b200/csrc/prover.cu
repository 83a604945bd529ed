// prover.cu — device-resident prover pipeline: LDE, merge, STIR prove.
//
// Data stays in HBM from the trace to the last fold. The host only drives the
// Fiat-Shamir transcript: per STIR layer it reads back the m coset
// evaluations and the layer root (a few hundred bytes), derives the next
// challenges, and finally gathers the s0 query openings in one copy.
#include <algorithm>
#include <thread>
#include <vector>

#include "context.hpp"
#include "fri_classic.cuh"
#include "gl.cuh"
#include "merge.cuh"
#include "merkle.cuh"
#include "rsa_air.cuh"
#include "prover.hpp"
#include "hash_air.hpp"
#include "sha256_air.cuh"
#include "stir.cuh"
#include "verifier.hpp"

namespace sg {

bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

static unsigned log2_exact(uint64_t n) {
  unsigned l = 0;
  while ((1ull << l) < n) ++l;
  return l;
}
static bool pow2(uint64_t n) { return n && !(n & (n - 1)); }

static void ntt(sg_ctx* c, const uint64_t* in, uint64_t* out, uint32_t cols, uint64_t in_stride, uint64_t out_stride,
                unsigned log_n, bool inverse, uint64_t n_valid, uint64_t* scratch, const PowSpec* pre = nullptr) {
  cuda_check(ntt_batch(c->tw, in, out, cols, in_stride, out_stride, (int)log_n, inverse, n_valid, scratch, c->stream,
                       pre),
             "ntt");
}

// ------------------------------------------------------------------ LDE
namespace {

void lde_check(uint64_t w, uint64_t n_trace, uint64_t blowup, uint64_t shift) {
  require(w > 0 && w < (1u << 31), "lde: bad column count");
  require(pow2(n_trace), "lde: trace_len must be a power of 2");
  require(pow2(blowup) && blowup >= 2, "lde: blowup must be a power of 2 >= 2");
  require(log2_exact(n_trace * blowup) <= kMaxLogN, "lde: domain larger than 2^28");
  require(shift % gl::P != 0, "lde: shift must be nonzero");
}

// Powers of the coset shift for the forward transform's first pass (none for
// shift 1). The tables stay on the device in the context, so an LDE with the same
// shift as the previous one uploads nothing; a new shift is copied in stream
// order, after every earlier use of the old tables on this context.
struct ShiftTables {
  PowSpec spec;
  bool active = false;
  ShiftTables(sg_ctx* c, uint64_t shift, cudaStream_t s) {
    shift %= gl::P;
    if (shift == 1) return;
    if (!c->shift_tab) cuda_check(cudaMalloc(&c->shift_tab, 2 * kTwEntries * 8), "shift tables");
    if (c->shift_key != shift) {
      cuda_check(cudaStreamSynchronize(s), "sync");  // the host copy below is reused across calls
      c->shift_host.resize(2 * kTwEntries);
      pow_tables_host(shift, 1, c->shift_host.data());
      cuda_check(cudaMemcpyAsync(c->shift_tab, c->shift_host.data(), 2 * kTwEntries * 8, cudaMemcpyHostToDevice, s),
                 "h2d");
      c->shift_key = shift;
    }
    spec.lo = c->shift_tab;
    spec.hi = c->shift_tab + kTwEntries;
    active = true;
  }
};

// A domain above one pass (2^12) from a trace of at most 2^12 rows is evaluated
// coset by coset in one pass (ntt_coset_eval): no scratch round trip, and no
// scratch buffer the size of the LDE.
bool lde_by_cosets(uint64_t n_trace, uint64_t blowup) {
  const int lm = (int)log2_exact(n_trace), lb = (int)log2_exact(blowup);
  return lm + lb > 12 && ntt_coset_eval_ok(lm, lb);
}

// iNTT of w columns into coef, then the zero-padded forward transform into d_out,
// coefficient k times shift^k (applied as the forward transform loads it).
void lde_core(sg_ctx* c, const uint64_t* d_trace, uint64_t w, uint64_t n_trace, uint64_t blowup,
              const ShiftTables& sh, uint64_t* coef, uint64_t* scratch, uint64_t* d_out) {
  const uint64_t n0 = n_trace * blowup;
  ntt(c, d_trace, coef, (uint32_t)w, n_trace, n_trace, log2_exact(n_trace), true, n_trace, scratch);
  if (lde_by_cosets(n_trace, blowup)) {
    cuda_check(ntt_coset_eval(c->tw, coef, d_out, (uint32_t)w, (int)log2_exact(n_trace), (int)log2_exact(blowup),
                              c->stream, sh.active ? &sh.spec : nullptr),
               "coset evaluation");
    return;
  }
  ntt(c, coef, d_out, (uint32_t)w, n_trace, n0, log2_exact(n0), false, n_trace, scratch,
      sh.active ? &sh.spec : nullptr);
}

uint64_t lde_scratch_elems(uint64_t w, uint64_t n_trace, uint64_t blowup) {
  const uint64_t inv = ntt_scratch_elems(w, log2_exact(n_trace));
  if (lde_by_cosets(n_trace, blowup)) return inv;
  return std::max(ntt_scratch_elems(w, log2_exact(n_trace * blowup)), inv);
}

}  // namespace

void lde_device(sg_ctx* c, const uint64_t* d_trace, uint64_t w, uint64_t n_trace, uint64_t blowup, uint64_t shift,
                uint64_t* d_out) {
  lde_check(w, n_trace, blowup, shift);
  cudaStream_t s = c->stream;
  ShiftTables sh(c, shift, s);
  DBuf coef(w * n_trace, s), scratch(lde_scratch_elems(w, n_trace, blowup), s);
  lde_core(c, d_trace, w, n_trace, blowup, sh, coef.p, scratch.p, d_out);
}

// The same LDE from a host trace: column chunks of ~64 MB are copied on the
// context's copy stream while earlier chunks are transformed on its compute
// stream, so only the first chunk's copy is exposed (with pinned host memory;
// a pageable buffer is staged by the driver and overlaps less).
void lde_from_host(sg_ctx* c, const uint64_t* h_trace, uint64_t w, uint64_t n_trace, uint64_t blowup, uint64_t shift,
                   uint64_t* d_out) {
  lde_check(w, n_trace, blowup, shift);
  cudaStream_t s = c->stream;
  const uint64_t chunk = std::min<uint64_t>(w, std::max<uint64_t>(1, (uint64_t(8) << 20) / n_trace));
  const uint64_t n_chunks = (w + chunk - 1) / chunk;
  ShiftTables sh(c, shift, s);  // before the chunk copies take the copy engine
  DBuf d_in(w * n_trace, s);
  if (n_chunks == 1) {
    cuda_check(cudaMemcpyAsync(d_in.p, h_trace, w * n_trace * 8, cudaMemcpyHostToDevice, s), "h2d");
    lde_device(c, d_in.p, w, n_trace, blowup, shift, d_out);
    cuda_check(cudaStreamSynchronize(s), "sync");
    return;
  }
  if (!c->copy_stream) cuda_check(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking), "copy stream");
  std::vector<cudaEvent_t> ev(n_chunks + 1, nullptr);
  for (auto& e : ev) cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
  // the copy stream may only write d_in once its stream-ordered allocation exists
  cuda_check(cudaEventRecord(ev[n_chunks], s), "event");
  cuda_check(cudaStreamWaitEvent(c->copy_stream, ev[n_chunks], 0), "wait");
  for (uint64_t k = 0; k < n_chunks; ++k) {
    const uint64_t c0 = k * chunk, wk = std::min(chunk, w - c0);
    cuda_check(cudaMemcpyAsync(d_in.p + c0 * n_trace, h_trace + c0 * n_trace, wk * n_trace * 8,
                               cudaMemcpyHostToDevice, c->copy_stream),
               "h2d");
    cuda_check(cudaEventRecord(ev[k], c->copy_stream), "event");
  }
  DBuf coef(chunk * n_trace, s), scratch(lde_scratch_elems(chunk, n_trace, blowup), s);
  for (uint64_t k = 0; k < n_chunks; ++k) {
    const uint64_t c0 = k * chunk, wk = std::min(chunk, w - c0);
    cuda_check(cudaStreamWaitEvent(s, ev[k], 0), "wait");
    lde_core(c, d_in.p + c0 * n_trace, wk, n_trace, blowup, sh, coef.p, scratch.p, d_out + c0 * n_trace * blowup);
  }
  cuda_check(cudaStreamSynchronize(s), "sync");  // d_in's copies and the transforms are done
  for (auto& e : ev) cudaEventDestroy(e);
}

// LDE of w columns (lde_trace_columns, trace_import.rs:251-281) and the Merkle
// commitment to its rows (MerkleTreeChannel::push_leaves_parallel + finalize,
// merkle/src/lib.rs:391-476) in one pipeline. When lde_leaf_ok, the forward
// transform's last pass hashes the rows as it produces them, so the LDE is never
// written (only its first keep_cols columns, into d_keep); otherwise the LDE is
// materialised and hashed by the leaf kernel. A host trace is copied in column
// chunks overlapped with their inverse transforms, as lde_from_host does.
void lde_commit(sg_ctx* c, const uint64_t* trace, bool host_trace, uint64_t w, uint64_t n_trace, uint64_t blowup,
                uint64_t shift, const DevTree& tree, uint64_t* d_keep, uint64_t keep_cols) {
  lde_check(w, n_trace, blowup, shift);
  require(keep_cols <= w && (keep_cols == 0 || d_keep), "lde_commit: bad kept columns");
  require(tree.len[0] == n_trace * blowup, "lde_commit: the tree does not have one leaf per LDE row");
  cudaStream_t s = c->stream;
  const uint64_t n0 = n_trace * blowup;
  const int ln = (int)log2_exact(n0), lt = (int)log2_exact(n_trace);
  if (!lde_leaf_ok((uint32_t)w, ln)) {
    DBuf lde(keep_cols == w ? 0 : w * n0, s);
    uint64_t* dst = keep_cols == w ? d_keep : lde.p;
    if (host_trace)
      lde_from_host(c, trace, w, n_trace, blowup, shift, dst);
    else
      lde_device(c, trace, w, n_trace, blowup, shift, dst);
    cuda_check(tree_hash_leaves(tree, dst, (uint32_t)w, n0, 0, s), "leaves");
    if (keep_cols && dst != d_keep)
      cuda_check(cudaMemcpyAsync(d_keep, dst, keep_cols * n0 * 8, cudaMemcpyDeviceToDevice, s), "copy");
    return;
  }
  ShiftTables sh(c, shift, s);
  const PowSpec* pre = sh.active ? &sh.spec : nullptr;
  DBuf coef(w * n_trace, s), fscratch(lde_leaf_scratch_elems((uint32_t)w, ln), s);
  {
    DBuf scratch(ntt_scratch_elems(w, lt), s);
    if (!host_trace) {
      ntt(c, trace, coef.p, (uint32_t)w, n_trace, n_trace, lt, true, n_trace, scratch.p);
      cuda_check(lde_leaf_prepasses(c->tw, coef.p, n_trace, (uint32_t)w, 0, (uint32_t)w, ln, n_trace, pre,
                                    fscratch.p, s),
                 "LDE passes");
    } else {
      // column chunks of ~64 MB: chunk k's copy overlaps chunk k-1's inverse
      // transform and the passes before the fused one
      const uint64_t chunk = std::min<uint64_t>(w, std::max<uint64_t>(1, (uint64_t(8) << 20) / n_trace));
      const uint64_t n_chunks = (w + chunk - 1) / chunk;
      if (!c->copy_stream)
        cuda_check(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking), "copy stream");
      DBuf d_in(w * n_trace, s);
      std::vector<cudaEvent_t> ev(n_chunks + 1, nullptr);
      for (auto& e : ev) cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
      cuda_check(cudaEventRecord(ev[n_chunks], s), "event");
      cuda_check(cudaStreamWaitEvent(c->copy_stream, ev[n_chunks], 0), "wait");
      for (uint64_t k = 0; k < n_chunks; ++k) {
        const uint64_t c0 = k * chunk, wk = std::min(chunk, w - c0);
        cuda_check(cudaMemcpyAsync(d_in.p + c0 * n_trace, trace + c0 * n_trace, wk * n_trace * 8,
                                   cudaMemcpyHostToDevice, c->copy_stream),
                   "h2d");
        cuda_check(cudaEventRecord(ev[k], c->copy_stream), "event");
      }
      for (uint64_t k = 0; k < n_chunks; ++k) {
        const uint64_t c0 = k * chunk, wk = std::min(chunk, w - c0);
        cuda_check(cudaStreamWaitEvent(s, ev[k], 0), "wait");
        ntt(c, d_in.p + c0 * n_trace, coef.p + c0 * n_trace, (uint32_t)wk, n_trace, n_trace, lt, true, n_trace,
            scratch.p);
        cuda_check(lde_leaf_prepasses(c->tw, coef.p, n_trace, (uint32_t)w, (uint32_t)c0, (uint32_t)wk, ln, n_trace,
                                      pre, fscratch.p, s),
                   "LDE passes");
      }
      cuda_check(cudaStreamSynchronize(s), "sync");  // the copies and transforms are done before d_in is freed
      for (auto& e : ev) cudaEventDestroy(e);
    }
  }
  coef = DBuf();
  cuda_check(lde_leaf_final(c->tw, (uint32_t)w, ln, fscratch.p, tree.arity0, tree.label, tree.d, d_keep,
                            (uint32_t)keep_cols, s),
             "fused LDE and leaf hashing");
}

// ------------------------------------------------------------------ merge
static bool phi_live(int mode, uint64_t n) {
  if (mode == SG_PHI_ALWAYS) return true;
  if (mode == SG_PHI_NEVER) return false;
  return n >= 4096;
}

void merge_device(sg_ctx* c, int air, const uint64_t* d_lde, uint64_t w, uint64_t n_trace, uint64_t blowup,
                  const uint64_t* lambdas, uint64_t k, int phi_mode, uint64_t* d_c, uint64_t n_blocks) {
  require(air == SG_AIR_HASH_ROLLUP || air == SG_AIR_SHA256, "merge: unsupported AIR id");
  if (air == SG_AIR_HASH_ROLLUP) require(w == 4 && k == 3, "merge: HashRollup has 4 columns and 3 constraints");
  if (air == SG_AIR_SHA256)
    require(w == sha::WIDTH && k == sha::NUM_CONSTRAINTS, "merge: the SHA-256 AIR has 756 columns and 766 constraints");
  require(pow2(n_trace) && pow2(blowup), "merge: sizes must be powers of 2");
  require(phi_mode >= 0 && phi_mode <= 2, "merge: bad phi mode");
  const uint64_t n = n_trace * blowup;
  require(log2_exact(n) <= kMaxLogN, "merge: domain larger than 2^28");
  cudaStream_t s = c->stream;
  if (!phi_live(phi_mode, n)) {
    cuda_check(cudaMemsetAsync(d_c, 0, n * 8, s), "memset");
    return;
  }
  if (air == SG_AIR_SHA256) {
    merge_hash_device(c, sha256_hash_air(), d_lde, n_trace, blowup, lambdas, phi_mode, d_c, n_blocks);
    return;
  }
  DBuf phi(n, s);
  DBuf scratch(ntt_scratch_elems(1, log2_exact(n)), s);
  cuda_check(hash_rollup_phi(d_lde, n, blowup, lambdas, phi.p, s), "phi");
  ntt(c, phi.p, phi.p, 1, n, n, log2_exact(n), true, n, scratch.p);
  cuda_check(quotient_zh(phi.p, n, n_trace, d_c, s), "quotient");
  ntt(c, d_c, d_c, 1, n, n, log2_exact(n), false, n > n_trace ? n - n_trace : n, scratch.p);
}

// ------------------------------------------------------------------ STIR
namespace {

constexpr int DL = kc::kDigestLanes;  // u64 lanes per digest of the build's hash profile
constexpr int HB = kc::kHashBytes;

struct Tree {
  DevTree t;
  DBuf buf;
  void make(uint64_t n, const std::vector<uint32_t>& ar, uint64_t label, cudaStream_t s) {
    require(tree_plan(&t, n, ar, label), "merkle: arity schedule does not reach the root");
    buf.alloc(t.total_digests * DL, s);
    t.d = buf.p;
  }
};

template <class T>
void d2h(std::vector<T>* v, const uint64_t* src, size_t elems, cudaStream_t s) {
  v->resize(elems * 8 / sizeof(T));
  cuda_check(cudaMemcpyAsync(v->data(), src, elems * 8, cudaMemcpyDeviceToHost, s), "d2h");
}

Digest digest_at(const std::vector<uint64_t>& h, size_t lane0) {
  Digest d;
  memcpy(d.data(), h.data() + lane0, HB);
  return d;
}

}  // namespace

// fri.rs:1900-2055 deep_fri_prove, classic branch (stir = false): fri.rs:1398-1718
// fri_build_transcript and fri.rs:1724-1807 fri_prove_queries. Per layer the
// DEEP quotient q = (f - f(z)) / (x - z) and s (the folded next layer, broadcast
// over its fibres) are committed with f as 18-component leaves; r fold queries
// open every layer at i, i mod n_1, ... .
std::vector<uint8_t> classic_prove_device(sg_ctx* c, const uint64_t* d_f0, uint64_t n0, const sg_fri_params& p,
                                          const std::vector<uint64_t>& sizes) {
  cudaStream_t s = c->stream;
  const uint64_t L = p.schedule_len;
  const bool use_cc = p.coeff_commit_final != 0;
  StirProof pr;
  pr.stir = false;
  pr.n0 = n0;
  pr.omega0 = gl::root_of_unity(log2_exact(n0));
  HostTranscript tr("FRI/FS");
  bind_statement(tr, p, n0);

  // f0 tree (fri.rs:1060-1076): one value per leaf, arity pick(n0, 16), label 0xFF
  Tree f0t;
  f0t.make(n0, layer_arities(n0, 16), 0xFF, s);
  cuda_check(tree_hash_leaves(f0t.t, d_f0, 1, n0, 0, s), "f0 leaves");
  cuda_check(tree_hash_levels(f0t.t, s), "f0 levels");
  std::vector<uint64_t> h;
  d2h(&h, f0t.t.d + DL * f0t.t.off.back(), DL, s);
  cuda_check(cudaStreamSynchronize(s), "sync");
  pr.root_f0 = digest_at(h, 0);
  tr.absorb_bytes(pr.root_f0.data(), HB);
  const gl::Fp6 z = tr.challenge_ext("z_fp3");

  const uint64_t work = std::max<uint64_t>(n0, 6 * sizes[1]);
  uint64_t scratch_len = ntt_scratch_elems(1, log2_exact(n0));
  for (uint64_t i = 1; i <= L; ++i) scratch_len = std::max(scratch_len, ntt_scratch_elems(6, log2_exact(sizes[i])));
  DBuf coef(work, s), scratch(scratch_len, s), partials(ood_partials_len(n0, 2), s), evals(2 * 6, s);
  std::vector<DBuf> planes(L + 1), mats(L);
  std::vector<Tree> trees(L);
  DBuf tuples;
  Tree ctree;
  std::vector<gl::Fp6> alphas;

  const uint64_t* cur = d_f0;
  bool base = true;
  for (uint64_t ell = 0; ell < L; ++ell) {
    const uint64_t m = p.schedule[ell], n = sizes[ell], nn = n / m;
    const unsigned lg = log2_exact(n);
    const bool last_cc = use_cc && ell == L - 1;
    gl::Fp6 alpha = gl::e_zero();
    if (!last_cc) alpha = tr.challenge_ext("alpha");
    // f(z): component iNTT, then the first of the two OOD points z, -z
    ntt(c, cur, coef.p, base ? 1 : 6, n, n, lg, true, n, scratch.p);
    cuda_check(ood_evaluate(coef.p, base, n, 2, z, partials.p, evals.p, s), "f(z)");
    std::vector<uint64_t> fzh;
    d2h(&fzh, evals.p, 6, s);
    cuda_check(cudaStreamSynchronize(s), "sync");
    gl::Fp6 fz;
    for (int k = 0; k < 6; ++k) fz.c[k] = fzh[k];
    pr.fz.push_back(fz);
    // leaf matrix rows 12..17: the DEEP quotient
    mats[ell].alloc(18 * n, s);
    cuda_check(deep_quotient(cur, base, n, (int)lg, c->tw.d_fwd_lo, c->tw.d_fwd_hi, z, fz, mats[ell].p + 12 * n, s),
               "deep quotient");
    // coset coefficients -> next layer (or the committed tuples of the last layer)
    FoldArgs fa{};
    fa.f = cur;
    fa.base = base;
    fa.n = n;
    fa.log_n = (int)lg;
    fa.m = (int)m;
    fa.alpha = alpha;
    fa.tw_inv_lo = c->tw.d_inv_lo;
    fa.tw_inv_hi = c->tw.d_inv_hi;
    if (!last_cc) {
      planes[ell + 1].alloc(6 * nn, s);
      fa.next = planes[ell + 1].p;
    } else {
      tuples.alloc(6 * m * nn, s);
      fa.tuples = tuples.p;
    }
    cuda_check(stir_fold(fa, s), "fold");
    cuda_check(fill_leaf_rows(cur, base, last_cc ? nullptr : planes[ell + 1].p, nn, n, mats[ell].p, s), "leaf rows");
    trees[ell].make(n, layer_arities(n, m), ell, s);
    cuda_check(tree_hash_leaves(trees[ell].t, mats[ell].p, 18, n, 0, s), "layer leaves");
    cuda_check(tree_hash_levels(trees[ell].t, s), "layer levels");
    if (last_cc) {
      ctree.make(nn, layer_arities(nn, 16), 0xFE, s);
      cuda_check(tree_hash_leaves(ctree.t, tuples.p, (uint32_t)(6 * m), nn, 0, s), "coeff leaves");
      cuda_check(tree_hash_levels(ctree.t, s), "coeff levels");
    }
    std::vector<uint64_t> root, croot, tup;
    d2h(&root, trees[ell].t.d + DL * trees[ell].t.off.back(), DL, s);
    if (last_cc) {
      d2h(&croot, ctree.t.d + DL * ctree.t.off.back(), DL, s);
      d2h(&tup, tuples.p, 6 * m * nn, s);
    }
    cuda_check(cudaStreamSynchronize(s), "sync");
    pr.roots.push_back(digest_at(root, 0));
    tr.absorb_ext(fz);
    tr.absorb_bytes(pr.roots.back().data(), HB);
    if (last_cc) {
      pr.has_ct = pr.has_croot = true;
      pr.coeff_root = digest_at(croot, 0);
      tr.absorb_bytes(pr.coeff_root.data(), HB);
      alpha = tr.challenge_ext("alpha");
      (void)tr.challenge_ext("beta_deg");
      pr.coeff_tuples.assign(nn, std::vector<gl::Fp6>(m));
      for (uint64_t b = 0; b < nn; ++b)
        for (uint64_t k = 0; k < m; ++k)
          for (int q = 0; q < 6; ++q) pr.coeff_tuples[b][k].c[q] = tup[(k * 6 + q) * nn + b];
      planes[ell + 1].alloc(6 * nn, s);
      cuda_check(fold_tuples(tuples.p, nn, (int)m, alpha, planes[ell + 1].p, s), "final fold");
    }
    alphas.push_back(alpha);
    cur = planes[ell + 1].p;
    base = false;
  }

  // final polynomial coefficients (fri.rs:1915-1935) and the query seed
  const uint64_t nf = sizes[L];
  if (nf > 1) {
    ntt(c, cur, coef.p, 6, nf, nf, log2_exact(nf), true, nf, scratch.p);
  } else {
    cuda_check(cudaMemcpyAsync(coef.p, cur, 6 * 8, cudaMemcpyDeviceToDevice, s), "copy");
  }
  std::vector<uint64_t> fc;
  d2h(&fc, coef.p, 6 * nf, s);
  cuda_check(cudaStreamSynchronize(s), "sync");
  for (uint64_t k = 0; k < std::min<uint64_t>(p.d_final, nf); ++k) {
    gl::Fp6 e;
    for (int q = 0; q < 6; ++q) e.c[q] = fc[q * nf + k];
    pr.final_coeffs.push_back(e);
    tr.absorb_ext(e);
  }
  const uint64_t query_seed = tr.challenge_field("query_seed");

  // fri_prove_queries (fri.rs:1724-1807): index chains on the host, one gather per
  // buffer for the payload values and the opening digests
  std::vector<std::vector<uint64_t>> chain(p.r);
  for (uint64_t q = 0; q < p.r; ++q) {
    uint64_t i = query_index(query_seed, q, n0);
    for (uint64_t ell = 0; ell < L; ++ell) {
      chain[q].push_back(i);
      i %= sizes[ell] / p.schedule[ell];
    }
    chain[q].push_back(i);  // final index
  }
  auto gather_openings = [&](const DevTree& t, const std::vector<uint64_t>& idx) {
    std::vector<uint64_t> di;
    for (uint64_t i : idx) opening_indices(t, i, &di);
    DBuf d_i(di.size(), s), d_o(DL * di.size(), s);
    std::vector<uint64_t> got;
    if (!di.empty()) {
      cuda_check(cudaMemcpyAsync(d_i.p, di.data(), di.size() * 8, cudaMemcpyHostToDevice, s), "h2d");
      cuda_check(gather_digests(t.d, d_i.p, di.size(), d_o.p, s), "gather paths");
      d2h(&got, d_o.p, DL * di.size(), s);
    }
    cuda_check(cudaStreamSynchronize(s), "sync");
    std::vector<Opening> out;
    size_t pos = 0;
    for (uint64_t i : idx) {
      Opening o;
      o.index = i;
      o.leaf = digest_at(got, pos);
      pos += DL;
      for (size_t l = 0; l + 1 < t.len.size(); ++l) {
        std::vector<Digest> sib(t.arity[l] - 1);
        for (auto& d : sib) {
          d = digest_at(got, pos);
          pos += DL;
        }
        o.path.push_back(std::move(sib));
      }
      out.push_back(std::move(o));
    }
    return out;
  };
  auto gather_values = [&](const uint64_t* src, const std::vector<uint64_t>& idx) {
    DBuf d_i(idx.size(), s), d_o(idx.size(), s);
    std::vector<uint64_t> got;
    if (!idx.empty()) {
      cuda_check(cudaMemcpyAsync(d_i.p, idx.data(), idx.size() * 8, cudaMemcpyHostToDevice, s), "h2d");
      cuda_check(gather_u64(src, d_i.p, idx.size(), d_o.p, s), "gather values");
      d2h(&got, d_o.p, idx.size(), s);
    }
    cuda_check(cudaStreamSynchronize(s), "sync");
    return got;
  };
  std::vector<uint64_t> i0s(p.r);
  for (uint64_t q = 0; q < p.r; ++q) i0s[q] = chain[q][0];
  const std::vector<Opening> f0_open = gather_openings(f0t.t, i0s);
  pr.queries.resize(p.r);
  pr.layer_open.resize(L);
  for (uint64_t ell = 0; ell < L; ++ell) {
    const uint64_t n = sizes[ell], m = p.schedule[ell], nn = n / m;
    std::vector<uint64_t> idx(p.r), vidx;
    for (uint64_t q = 0; q < p.r; ++q) {
      idx[q] = chain[q][ell];
      for (uint64_t k = 0; k < 18; ++k) vidx.push_back(k * n + idx[q]);
    }
    pr.layer_open[ell] = gather_openings(trees[ell].t, idx);
    const std::vector<uint64_t> v = gather_values(mats[ell].p, vidx);
    for (uint64_t q = 0; q < p.r; ++q) {
      const uint64_t i = idx[q];
      pr.queries[q].refs.push_back({i, i % m, i % nn, 0});
      std::array<gl::Fp6, 3> pl;
      for (int t = 0; t < 3; ++t)
        for (int k = 0; k < 6; ++k) pl[t].c[k] = v[q * 18 + t * 6 + k];
      pr.queries[q].pay.push_back(pl);
    }
  }
  for (uint64_t q = 0; q < p.r; ++q) {
    pr.queries[q].f0_open = f0_open[q];
    pr.queries[q].final_index = chain[q][L];
    pr.f0_openings.push_back(f0_open[q]);
  }
  return encode_proof(pr);
}

namespace {

std::vector<uint8_t> stir_prove_on_stream(sg_ctx* c, const uint64_t* d_f0, uint64_t n0, const sg_fri_params& p) {
  cudaStream_t s = c->stream;
  const uint64_t L = p.schedule_len;
  require(L >= 1 && L <= SG_MAX_SCHEDULE, "stir_prove: empty or oversized schedule");
  require(pow2(n0) && n0 >= 2 && log2_exact(n0) <= kMaxLogN, "stir_prove: n0 must be a power of 2 in [2, 2^28]");
  require(p.s0 <= (1u << 20) && p.r <= (1u << 20), "stir_prove: too many queries");
  std::vector<uint64_t> sizes{n0};
  for (uint64_t i = 0; i < L; ++i) {
    const uint64_t m = p.schedule[i];
    require(m == 2 || m == 4 || m == 8 || m == 16, "stir_prove: fold arities must be 2, 4, 8 or 16");
    require(sizes.back() % m == 0, "stir_prove: schedule does not divide the domain");
    sizes.push_back(sizes.back() / m);
  }
  if (!p.stir) return classic_prove_device(c, d_f0, n0, p, sizes);
  const bool use_cc = p.coeff_commit_final != 0;

  StirProof pr;
  pr.n0 = n0;
  pr.omega0 = gl::root_of_unity(log2_exact(n0));
  HostTranscript tr("FRI/FS");
  bind_statement(tr, p, n0);

  // packed f0 tree: leaf b = {f0[b + j n0/m0]}_j (fri.rs:1420-1431), label 0xFF
  const uint64_t m0 = p.schedule[0], nn0 = n0 / m0;
  Tree f0t;
  f0t.make(nn0, layer_arities(nn0, 16), 0xFF, s);
  cuda_check(tree_hash_leaves(f0t.t, d_f0, (uint32_t)m0, nn0, 0, s), "f0 leaves");
  cuda_check(tree_hash_levels(f0t.t, s), "f0 levels");
  std::vector<uint64_t> h;
  d2h(&h, f0t.t.d + DL * f0t.t.off.back(), DL, s);
  cuda_check(cudaStreamSynchronize(s), "sync");
  pr.root_f0 = digest_at(h, 0);
  tr.absorb_bytes(pr.root_f0.data(), HB);
  const gl::Fp6 z = tr.challenge_ext("z_fp3");

  const uint64_t work = std::max<uint64_t>(n0, 6 * sizes[1]);
  uint64_t scratch_len = ntt_scratch_elems(1, log2_exact(n0));
  for (uint64_t i = 1; i <= L; ++i) scratch_len = std::max(scratch_len, ntt_scratch_elems(6, log2_exact(sizes[i])));
  DBuf coef(work, s), scratch(scratch_len, s);
  uint64_t part_len = 0;
  for (uint64_t i = 0; i < L; ++i) part_len = std::max<uint64_t>(part_len, ood_partials_len(sizes[i], (int)p.schedule[i]));
  DBuf partials(part_len, s);
  DBuf evals(16 * 6, s);
  std::vector<DBuf> planes(L + 1);
  std::vector<Tree> trees(L);
  DBuf tuples;
  Tree ctree;

  const uint64_t* cur = d_f0;
  bool base = true;
  gl::Fp6 zc = z;
  for (uint64_t ell = 0; ell < L; ++ell) {
    const uint64_t m = p.schedule[ell], n = sizes[ell], nn = n / m;
    const unsigned lg = log2_exact(n);
    const bool last_cc = use_cc && ell == L - 1;
    gl::Fp6 alpha = gl::e_zero();
    if (!last_cc) alpha = tr.challenge_ext("alpha");

    // layer tree (label ell) over the 6 components of f_ell; for ell >= 1 the
    // previous fold already wrote its leaves
    if (ell == 0) {
      trees[0].make(n, layer_arities(n, m), 0, s);
      cuda_check(tree_hash_leaves(trees[0].t, d_f0, 1, n, 5, s), "layer-0 leaves");
    }
    cuda_check(tree_hash_levels(trees[ell].t, s), "layer levels");

    // out-of-domain coset evaluation
    const uint32_t cols = base ? 1 : 6;
    ntt(c, cur, coef.p, cols, n, n, lg, true, n, scratch.p);
    cuda_check(ood_evaluate(coef.p, base, n, (int)m, zc, partials.p, evals.p, s), "ood");

    FoldArgs fa{};
    fa.f = cur;
    fa.base = base;
    fa.n = n;
    fa.log_n = (int)lg;
    fa.m = (int)m;
    fa.alpha = alpha;
    fa.tw_inv_lo = c->tw.d_inv_lo;
    fa.tw_inv_hi = c->tw.d_inv_hi;
    if (!last_cc) {
      planes[ell + 1].alloc(6 * nn, s);
      fa.next = planes[ell + 1].p;
      if (ell + 1 < L) {
        trees[ell + 1].make(nn, layer_arities(nn, p.schedule[ell + 1]), ell + 1, s);
        fa.leaves = trees[ell + 1].t.d;
        fa.leaf_label = ell + 1;
        fa.leaf_arity0 = trees[ell + 1].t.arity0;
      }
      cuda_check(stir_fold(fa, s), "fold");
    } else {
      tuples.alloc(6 * m * nn, s);
      fa.tuples = tuples.p;
      cuda_check(stir_fold(fa, s), "coefficient tuples");
      ctree.make(nn, layer_arities(nn, 16), 0xFE, s);
      cuda_check(tree_hash_leaves(ctree.t, tuples.p, (uint32_t)(6 * m), nn, 0, s), "coeff leaves");
      cuda_check(tree_hash_levels(ctree.t, s), "coeff levels");
    }

    std::vector<uint64_t> ev, root, croot, tup;
    d2h(&ev, evals.p, m * 6, s);
    d2h(&root, trees[ell].t.d + DL * trees[ell].t.off.back(), DL, s);
    if (last_cc) {
      d2h(&croot, ctree.t.d + DL * ctree.t.off.back(), DL, s);
      d2h(&tup, tuples.p, 6 * m * nn, s);
    }
    cuda_check(cudaStreamSynchronize(s), "sync");
    std::vector<gl::Fp6> evs(m);
    for (uint64_t j = 0; j < m; ++j)
      for (int q = 0; q < 6; ++q) evs[j].c[q] = ev[j * 6 + q];
    pr.fz.push_back(evs[0]);
    for (auto& e : evs) tr.absorb_ext(e);
    pr.coset_evals.push_back(std::move(evs));
    pr.roots.push_back(digest_at(root, 0));
    tr.absorb_bytes(pr.roots.back().data(), HB);
    zc = gl::e_pow(zc, m);
    if (last_cc) {
      pr.has_ct = pr.has_croot = true;
      pr.coeff_root = digest_at(croot, 0);
      tr.absorb_bytes(pr.coeff_root.data(), HB);
      alpha = tr.challenge_ext("alpha");
      (void)tr.challenge_ext("beta_deg");
      pr.coeff_tuples.assign(nn, std::vector<gl::Fp6>(m));
      for (uint64_t b = 0; b < nn; ++b)
        for (uint64_t k = 0; k < m; ++k)
          for (int q = 0; q < 6; ++q) pr.coeff_tuples[b][k].c[q] = tup[(k * 6 + q) * nn + b];
      planes[ell + 1].alloc(6 * nn, s);
      cuda_check(fold_tuples(tuples.p, nn, (int)m, alpha, planes[ell + 1].p, s), "final fold");
    }
    cur = planes[ell + 1].p;
    base = false;
  }

  // final polynomial coefficients (fri.rs:1915-1935)
  const uint64_t nf = sizes[L];
  const unsigned lgf = log2_exact(nf);
  if (nf > 1) {
    ntt(c, cur, coef.p, 6, nf, nf, lgf, true, nf, scratch.p);
  } else {
    cuda_check(cudaMemcpyAsync(coef.p, cur, 6 * 8, cudaMemcpyDeviceToDevice, s), "copy");
  }
  std::vector<uint64_t> fc;
  d2h(&fc, coef.p, 6 * nf, s);
  cuda_check(cudaStreamSynchronize(s), "sync");
  const uint64_t d_final = std::min<uint64_t>(p.d_final, nf);
  for (uint64_t k = 0; k < d_final; ++k) {
    gl::Fp6 e;
    for (int q = 0; q < 6; ++q) e.c[q] = fc[q * nf + k];
    pr.final_coeffs.push_back(e);
    tr.absorb_ext(e);
  }
  const uint64_t query_seed = tr.challenge_field("query_seed");

  // proximity queries (fri.rs:1813-1893): indices on the host, one gather each way
  std::vector<uint64_t> val_idx, dig_idx0, dig_idx1;
  std::vector<ProxQuery> qs(p.s0);
  for (uint64_t q = 0; q < p.s0; ++q) {
    qs[q].raw = query_index(query_seed, q, n0);
    qs[q].base = qs[q].raw % nn0;
    for (uint64_t j = 0; j < m0; ++j) {
      qs[q].fib_idx.push_back(qs[q].base + j * nn0);
      val_idx.push_back(qs[q].base + j * nn0);
    }
    opening_indices(f0t.t, qs[q].base, &dig_idx0);
    if (L >= 2) opening_indices(trees[1].t, qs[q].base, &dig_idx1);
  }
  const size_t nv = val_idx.size(), nd0 = dig_idx0.size(), nd1 = dig_idx1.size();
  const size_t n_next = L >= 2 ? 6 * p.s0 : 0;
  std::vector<uint64_t> idx_all;
  idx_all.insert(idx_all.end(), val_idx.begin(), val_idx.end());
  idx_all.insert(idx_all.end(), dig_idx0.begin(), dig_idx0.end());
  idx_all.insert(idx_all.end(), dig_idx1.begin(), dig_idx1.end());
  for (uint64_t q = 0; q < (L >= 2 ? p.s0 : 0); ++q)
    for (int k = 0; k < 6; ++k) idx_all.push_back((uint64_t)k * sizes[1] + qs[q].base);
  DBuf d_idx(idx_all.size(), s), d_out(nv + DL * (nd0 + nd1) + n_next, s);
  if (!idx_all.empty()) {
    cuda_check(cudaMemcpyAsync(d_idx.p, idx_all.data(), idx_all.size() * 8, cudaMemcpyHostToDevice, s), "h2d");
    cuda_check(gather_u64(d_f0, d_idx.p, nv, d_out.p, s), "gather values");
    cuda_check(gather_digests(f0t.t.d, d_idx.p + nv, nd0, d_out.p + nv, s), "gather f0 paths");
    if (L >= 2) {
      cuda_check(gather_digests(trees[1].t.d, d_idx.p + nv + nd0, nd1, d_out.p + nv + DL * nd0, s), "gather l1");
      cuda_check(gather_u64(planes[1].p, d_idx.p + nv + nd0 + nd1, n_next, d_out.p + nv + DL * (nd0 + nd1), s),
                 "gather f1");
    }
  }
  std::vector<uint64_t> got;
  d2h(&got, d_out.p, d_out.n, s);
  cuda_check(cudaStreamSynchronize(s), "sync");

  size_t pv = 0, p0 = nv, p1 = nv + DL * nd0, pn = nv + DL * (nd0 + nd1);
  auto take_opening = [&](const DevTree& t, uint64_t index, size_t* pos) {
    Opening o;
    o.index = index;
    o.leaf = digest_at(got, *pos);
    *pos += DL;
    for (size_t l = 0; l + 1 < t.len.size(); ++l) {
      std::vector<Digest> sib(t.arity[l] - 1);
      for (auto& d : sib) {
        d = digest_at(got, *pos);
        *pos += DL;
      }
      o.path.push_back(std::move(sib));
    }
    return o;
  };
  for (uint64_t q = 0; q < p.s0; ++q) {
    for (uint64_t j = 0; j < m0; ++j) qs[q].fib_vals.push_back(got[pv++]);
    qs[q].f0_open = take_opening(f0t.t, qs[q].base, &p0);
    qs[q].has_l1 = L >= 2;
    if (L >= 2) {
      qs[q].l1_open = take_opening(trees[1].t, qs[q].base, &p1);
      for (int k = 0; k < 6; ++k) qs[q].f_next.c[k] = got[pn++];
    }
  }
  pr.prox = std::move(qs);
  return encode_proof(pr);
}

// Trees of one shape, one per proof of a group, side by side in one buffer.
struct GroupTree {
  DevTree t;
  DBuf buf;
  uint64_t stride = 0;  // u64 between two trees' digests
  void make(uint64_t n, const std::vector<uint32_t>& ar, uint64_t label, uint32_t G, cudaStream_t s) {
    require(tree_plan(&t, n, ar, label), "merkle: arity schedule does not reach the root");
    stride = t.total_digests * DL;
    buf.alloc(stride * G, s);
    t.d = buf.p;
  }
  // the G roots (DL lanes each, one after another) into h
  void roots(std::vector<uint64_t>* h, uint32_t G, cudaStream_t s) const {
    h->resize((size_t)G * DL);
    cuda_check(cudaMemcpy2DAsync(h->data(), DL * 8, t.d + DL * t.off.back(), stride * 8, DL * 8, G,
                                 cudaMemcpyDeviceToHost, s),
               "d2h roots");
  }
};

// G STIR proofs of one shape in lockstep (fri.rs:1398-1718, 1813-1893, 1900-2055,
// as stir_prove_on_stream): the same n0 and parameters except the public-input
// hash, proof g's f0 at d_f0 + g * g_f0. Every device stage is one launch over
// all G proofs (trees side by side, transforms over 6G columns, grid.y = proof
// for the OOD and fold kernels), and each layer's one host synchronisation serves
// all G transcripts. The bytes of proof g are those of stir_prove_on_stream.
std::vector<std::vector<uint8_t>> stir_prove_group_on_stream(sg_ctx* c, const uint64_t* d_f0, uint64_t g_f0,
                                                             uint64_t n0, const std::vector<sg_fri_params>& ps) {
  cudaStream_t s = c->stream;
  const uint32_t G = (uint32_t)ps.size();
  require(G >= 1 && G <= 4096, "stir_prove_group: 1 to 4096 proofs");
  const sg_fri_params& p = ps[0];
  for (const auto& q : ps)
    require(q.schedule_len == p.schedule_len && q.s0 == p.s0 && q.r == p.r && q.seed_z == p.seed_z &&
                q.d_final == p.d_final && q.coeff_commit_final == p.coeff_commit_final && q.stir == p.stir &&
                !memcmp(q.schedule, p.schedule, sizeof p.schedule[0] * p.schedule_len),
            "stir_prove_group: the proofs differ in more than their public-input hash");
  const uint64_t L = p.schedule_len;
  require(p.stir, "stir_prove_group: STIR parameters only");
  require(L >= 1 && L <= SG_MAX_SCHEDULE, "stir_prove: empty or oversized schedule");
  require(pow2(n0) && n0 >= 2 && log2_exact(n0) <= kMaxLogN, "stir_prove: n0 must be a power of 2 in [2, 2^28]");
  require(p.s0 <= (1u << 20), "stir_prove: too many queries");
  require(g_f0 >= n0, "stir_prove_group: f0 stride below n0");
  std::vector<uint64_t> sizes{n0};
  for (uint64_t i = 0; i < L; ++i) {
    const uint64_t m = p.schedule[i];
    require(m == 2 || m == 4 || m == 8 || m == 16, "stir_prove: fold arities must be 2, 4, 8 or 16");
    require(sizes.back() % m == 0, "stir_prove: schedule does not divide the domain");
    sizes.push_back(sizes.back() / m);
  }
  const bool use_cc = p.coeff_commit_final != 0;
  std::vector<StirProof> pr(G);
  std::vector<HostTranscript> tr;
  tr.reserve(G);
  for (uint32_t g = 0; g < G; ++g) {
    pr[g].n0 = n0;
    pr[g].omega0 = gl::root_of_unity(log2_exact(n0));
    tr.emplace_back("FRI/FS");
    bind_statement(tr[g], ps[g], n0);
  }

  const uint64_t m0 = p.schedule[0], nn0 = n0 / m0;
  GroupTree f0t;
  f0t.make(nn0, layer_arities(nn0, 16), 0xFF, G, s);
  cuda_check(tree_hash_leaves_group(f0t.t, d_f0, (uint32_t)m0, nn0, 0, g_f0, f0t.stride, G, s), "f0 leaves");
  cuda_check(tree_hash_levels_group(f0t.t, f0t.stride, G, s), "f0 levels");
  std::vector<uint64_t> h;
  f0t.roots(&h, G, s);
  cuda_check(cudaStreamSynchronize(s), "sync");
  std::vector<gl::Fp6> zc(G);
  for (uint32_t g = 0; g < G; ++g) {
    pr[g].root_f0 = digest_at(h, (size_t)g * DL);
    tr[g].absorb_bytes(pr[g].root_f0.data(), HB);
    zc[g] = tr[g].challenge_ext("z_fp3");
  }

  const uint64_t work = std::max<uint64_t>(n0, 6 * sizes[1]);
  uint64_t scratch_len = ntt_scratch_elems(G, log2_exact(n0));
  for (uint64_t i = 1; i <= L; ++i)
    scratch_len = std::max(scratch_len, ntt_scratch_elems(6ull * G, log2_exact(sizes[i])));
  DBuf coef(work * G, s), scratch(scratch_len, s);
  uint64_t part_len = 0;
  for (uint64_t i = 0; i < L; ++i) part_len = std::max<uint64_t>(part_len, ood_partials_len(sizes[i], (int)p.schedule[i]));
  DBuf partials(part_len * G, s), evals(16 * 6 * (uint64_t)G, s);
  // per-proof OOD scalars and fold challenges, uploaded before each layer's launches
  const size_t sc_words = sizeof(OodScalars) / 8, al_words = sizeof(gl::Fp6) / 8;
  DBuf d_sc(sc_words * G, s), d_al(al_words * G, s);
  std::vector<OodScalars> h_sc(G);
  std::vector<gl::Fp6> h_al(G);
  std::vector<DBuf> planes(L + 1);
  std::vector<GroupTree> trees(L);
  DBuf tuples;
  GroupTree ctree;

  const uint64_t* cur = d_f0;
  uint64_t g_cur = g_f0;
  bool base = true;
  for (uint64_t ell = 0; ell < L; ++ell) {
    const uint64_t m = p.schedule[ell], n = sizes[ell], nn = n / m;
    const unsigned lg = log2_exact(n);
    const bool last_cc = use_cc && ell == L - 1;
    for (uint32_t g = 0; g < G; ++g) h_al[g] = last_cc ? gl::e_zero() : tr[g].challenge_ext("alpha");
    if (ell == 0) {
      trees[0].make(n, layer_arities(n, m), 0, G, s);
      cuda_check(tree_hash_leaves_group(trees[0].t, d_f0, 1, n, 5, g_f0, trees[0].stride, G, s), "layer-0 leaves");
    }
    cuda_check(tree_hash_levels_group(trees[ell].t, trees[ell].stride, G, s), "layer levels");

    const uint32_t cols = base ? 1 : 6;
    // proof g's component c at cur + g g_cur + c n; coefficients at coef + (g cols + c) n
    if (base)
      ntt(c, cur, coef.p, G, g_cur, n, lg, true, n, scratch.p);
    else
      ntt(c, cur, coef.p, 6 * G, n, n, lg, true, n, scratch.p);
    for (uint32_t g = 0; g < G; ++g) h_sc[g] = ood_scalars(zc[g], n, (int)m);
    cuda_check(cudaMemcpyAsync(d_sc.p, h_sc.data(), G * sizeof(OodScalars), cudaMemcpyHostToDevice, s), "h2d");
    cuda_check(cudaMemcpyAsync(d_al.p, h_al.data(), G * sizeof(gl::Fp6), cudaMemcpyHostToDevice, s), "h2d");
    cuda_check(ood_evaluate_group(coef.p, (uint64_t)cols * n, base, n, (int)m, (const OodScalars*)d_sc.p, partials.p,
                                  evals.p, 16 * 6, G, s),
               "ood");

    FoldArgs fa{};
    fa.f = cur;
    fa.base = base;
    fa.n = n;
    fa.log_n = (int)lg;
    fa.m = (int)m;
    fa.alpha = gl::e_zero();
    fa.tw_inv_lo = c->tw.d_inv_lo;
    fa.tw_inv_hi = c->tw.d_inv_hi;
    fa.n_proofs = G;
    fa.g_f = g_cur;
    fa.alphas = (const gl::Fp6*)d_al.p;
    if (!last_cc) {
      planes[ell + 1].alloc(6 * nn * G, s);
      fa.next = planes[ell + 1].p;
      fa.g_next = 6 * nn;
      if (ell + 1 < L) {
        trees[ell + 1].make(nn, layer_arities(nn, p.schedule[ell + 1]), ell + 1, G, s);
        fa.leaves = trees[ell + 1].t.d;
        fa.g_leaves = trees[ell + 1].stride;
        fa.leaf_label = ell + 1;
        fa.leaf_arity0 = trees[ell + 1].t.arity0;
      }
      cuda_check(stir_fold(fa, s), "fold");
    } else {
      tuples.alloc(6 * m * nn * G, s);
      fa.tuples = tuples.p;
      fa.g_tuples = 6 * m * nn;
      cuda_check(stir_fold(fa, s), "coefficient tuples");
      ctree.make(nn, layer_arities(nn, 16), 0xFE, G, s);
      cuda_check(tree_hash_leaves_group(ctree.t, tuples.p, (uint32_t)(6 * m), nn, 0, 6 * m * nn, ctree.stride, G, s),
                 "coeff leaves");
      cuda_check(tree_hash_levels_group(ctree.t, ctree.stride, G, s), "coeff levels");
    }

    std::vector<uint64_t> ev, root, croot, tup;
    d2h(&ev, evals.p, 16 * 6 * (uint64_t)G, s);
    trees[ell].roots(&root, G, s);
    if (last_cc) {
      ctree.roots(&croot, G, s);
      d2h(&tup, tuples.p, 6 * m * nn * G, s);
    }
    cuda_check(cudaStreamSynchronize(s), "sync");
    for (uint32_t g = 0; g < G; ++g) {
      std::vector<gl::Fp6> evs(m);
      for (uint64_t j = 0; j < m; ++j)
        for (int q = 0; q < 6; ++q) evs[j].c[q] = ev[(uint64_t)g * 96 + j * 6 + q];
      pr[g].fz.push_back(evs[0]);
      for (auto& e : evs) tr[g].absorb_ext(e);
      pr[g].coset_evals.push_back(std::move(evs));
      pr[g].roots.push_back(digest_at(root, (size_t)g * DL));
      tr[g].absorb_bytes(pr[g].roots.back().data(), HB);
      zc[g] = gl::e_pow(zc[g], m);
      if (last_cc) {
        pr[g].has_ct = pr[g].has_croot = true;
        pr[g].coeff_root = digest_at(croot, (size_t)g * DL);
        tr[g].absorb_bytes(pr[g].coeff_root.data(), HB);
        h_al[g] = tr[g].challenge_ext("alpha");
        (void)tr[g].challenge_ext("beta_deg");
        const uint64_t* tg = tup.data() + (uint64_t)g * 6 * m * nn;
        pr[g].coeff_tuples.assign(nn, std::vector<gl::Fp6>(m));
        for (uint64_t b = 0; b < nn; ++b)
          for (uint64_t k = 0; k < m; ++k)
            for (int q = 0; q < 6; ++q) pr[g].coeff_tuples[b][k].c[q] = tg[(k * 6 + q) * nn + b];
      }
    }
    if (last_cc) {
      planes[ell + 1].alloc(6 * nn * G, s);
      cuda_check(cudaMemcpyAsync(d_al.p, h_al.data(), G * sizeof(gl::Fp6), cudaMemcpyHostToDevice, s), "h2d");
      cuda_check(fold_tuples_group(tuples.p, 6 * m * nn, nn, (int)m, (const gl::Fp6*)d_al.p, planes[ell + 1].p,
                                   6 * nn, G, s),
                 "final fold");
    }
    cur = planes[ell + 1].p;
    g_cur = 6 * nn;
    base = false;
  }

  // final polynomial coefficients (fri.rs:1915-1935), proof g's at coef + 6 g nf
  const uint64_t nf = sizes[L];
  const unsigned lgf = log2_exact(nf);
  if (nf > 1) {
    ntt(c, cur, coef.p, 6 * G, nf, nf, lgf, true, nf, scratch.p);
  } else {
    cuda_check(cudaMemcpyAsync(coef.p, cur, 6 * 8 * (uint64_t)G, cudaMemcpyDeviceToDevice, s), "copy");
  }
  std::vector<uint64_t> fc;
  d2h(&fc, coef.p, 6 * nf * G, s);
  cuda_check(cudaStreamSynchronize(s), "sync");
  const uint64_t d_final = std::min<uint64_t>(p.d_final, nf);
  std::vector<uint64_t> query_seed(G);
  for (uint32_t g = 0; g < G; ++g) {
    for (uint64_t k = 0; k < d_final; ++k) {
      gl::Fp6 e;
      for (int q = 0; q < 6; ++q) e.c[q] = fc[(uint64_t)g * 6 * nf + q * nf + k];
      pr[g].final_coeffs.push_back(e);
      tr[g].absorb_ext(e);
    }
    query_seed[g] = tr[g].challenge_field("query_seed");
  }

  // proximity queries of every proof: one gather per kind of value
  std::vector<uint64_t> val_idx, dig_idx0, dig_idx1, next_idx;
  std::vector<std::vector<ProxQuery>> qs(G, std::vector<ProxQuery>(p.s0));
  const uint64_t td0 = f0t.t.total_digests, td1 = L >= 2 ? trees[1].t.total_digests : 0;
  for (uint32_t g = 0; g < G; ++g) {
    for (uint64_t q = 0; q < p.s0; ++q) {
      ProxQuery& x = qs[g][q];
      x.raw = query_index(query_seed[g], q, n0);
      x.base = x.raw % nn0;
      for (uint64_t j = 0; j < m0; ++j) {
        x.fib_idx.push_back(x.base + j * nn0);
        val_idx.push_back((uint64_t)g * g_f0 + x.base + j * nn0);
      }
      const size_t a0 = dig_idx0.size();
      opening_indices(f0t.t, x.base, &dig_idx0);
      for (size_t i = a0; i < dig_idx0.size(); ++i) dig_idx0[i] += (uint64_t)g * td0;
      if (L >= 2) {
        const size_t a1 = dig_idx1.size();
        opening_indices(trees[1].t, x.base, &dig_idx1);
        for (size_t i = a1; i < dig_idx1.size(); ++i) dig_idx1[i] += (uint64_t)g * td1;
        for (int k = 0; k < 6; ++k) next_idx.push_back((uint64_t)g * 6 * sizes[1] + (uint64_t)k * sizes[1] + x.base);
      }
    }
  }
  const size_t nv = val_idx.size(), nd0 = dig_idx0.size(), nd1 = dig_idx1.size(), nx = next_idx.size();
  std::vector<uint64_t> idx_all;
  idx_all.insert(idx_all.end(), val_idx.begin(), val_idx.end());
  idx_all.insert(idx_all.end(), dig_idx0.begin(), dig_idx0.end());
  idx_all.insert(idx_all.end(), dig_idx1.begin(), dig_idx1.end());
  idx_all.insert(idx_all.end(), next_idx.begin(), next_idx.end());
  DBuf d_idx(idx_all.size(), s), d_out(nv + DL * (nd0 + nd1) + nx, s);
  if (!idx_all.empty()) {
    cuda_check(cudaMemcpyAsync(d_idx.p, idx_all.data(), idx_all.size() * 8, cudaMemcpyHostToDevice, s), "h2d");
    cuda_check(gather_u64(d_f0, d_idx.p, nv, d_out.p, s), "gather values");
    cuda_check(gather_digests(f0t.t.d, d_idx.p + nv, nd0, d_out.p + nv, s), "gather f0 paths");
    if (L >= 2) {
      cuda_check(gather_digests(trees[1].t.d, d_idx.p + nv + nd0, nd1, d_out.p + nv + DL * nd0, s), "gather l1");
      cuda_check(gather_u64(planes[1].p, d_idx.p + nv + nd0 + nd1, nx, d_out.p + nv + DL * (nd0 + nd1), s),
                 "gather f1");
    }
  }
  std::vector<uint64_t> got;
  d2h(&got, d_out.p, d_out.n, s);
  cuda_check(cudaStreamSynchronize(s), "sync");

  size_t pv = 0, p0 = nv, p1 = nv + DL * nd0, pn = nv + DL * (nd0 + nd1);
  auto take_opening = [&](const DevTree& t, uint64_t index, size_t* pos) {
    Opening o;
    o.index = index;
    o.leaf = digest_at(got, *pos);
    *pos += DL;
    for (size_t l = 0; l + 1 < t.len.size(); ++l) {
      std::vector<Digest> sib(t.arity[l] - 1);
      for (auto& d : sib) {
        d = digest_at(got, *pos);
        *pos += DL;
      }
      o.path.push_back(std::move(sib));
    }
    return o;
  };
  std::vector<std::vector<uint8_t>> out(G);
  for (uint32_t g = 0; g < G; ++g) {
    for (uint64_t q = 0; q < p.s0; ++q) {
      ProxQuery& x = qs[g][q];
      for (uint64_t j = 0; j < m0; ++j) x.fib_vals.push_back(got[pv++]);
      x.f0_open = take_opening(f0t.t, x.base, &p0);
      x.has_l1 = L >= 2;
      if (L >= 2) {
        x.l1_open = take_opening(trees[1].t, x.base, &p1);
        for (int k = 0; k < 6; ++k) x.f_next.c[k] = got[pn++];
      }
    }
    pr[g].prox = std::move(qs[g]);
    out[g] = encode_proof(pr[g]);
  }
  return out;
}

// For the STIR phase, a context with a stir_stream (a server worker) moves to it:
// the stream waits for everything queued so far, and `stream` waits for the STIR
// work before the caller queues more (its buffers are freed in stream order).
struct StirStreamScope {
  sg_ctx* c;
  cudaStream_t saved;
  explicit StirStreamScope(sg_ctx* ctx) : c(ctx), saved(ctx->stream) {
    cuda_check(cudaEventRecord(c->stir_in, saved), "event");
    cuda_check(cudaStreamWaitEvent(c->stir_stream, c->stir_in, 0), "wait");
    c->stream = c->stir_stream;
  }
  ~StirStreamScope() {
    c->stream = saved;
    if (cudaEventRecord(c->stir_out, c->stir_stream) == cudaSuccess) cudaStreamWaitEvent(saved, c->stir_out, 0);
  }
};

}  // namespace

std::vector<uint8_t> stir_prove_device(sg_ctx* c, const uint64_t* d_f0, uint64_t n0, const sg_fri_params& p) {
  if (!c->stir_stream) return stir_prove_on_stream(c, d_f0, n0, p);
  StirStreamScope scope(c);
  return stir_prove_on_stream(c, d_f0, n0, p);
}

std::vector<std::vector<uint8_t>> stir_prove_group(sg_ctx* c, const uint64_t* d_f0, uint64_t g_f0, uint64_t n0,
                                                   const std::vector<sg_fri_params>& ps) {
  if (!c->stir_stream) return stir_prove_group_on_stream(c, d_f0, g_f0, n0, ps);
  StirStreamScope scope(c);
  return stir_prove_group_on_stream(c, d_f0, g_f0, n0, ps);
}

// ------------------------------------------------------------------ HashRollup pipeline
std::vector<uint8_t> prove_hash_rollup_host_leaves(sg_ctx* c, const uint64_t* leaves, uint64_t n_leaves,
                                                   const uint8_t pi[32], int phi_mode, bool self_verify, bool stir) {
  uint64_t n_trace = 8;
  while (n_trace < n_leaves) n_trace <<= 1;
  const uint64_t blowup = 32, n0 = n_trace * blowup;
  require(log2_exact(n0) <= kMaxLogN, "prove_hash_rollup: too many leaves");
  // build_hash_rollup_trace (air_workloads.rs:571-589): a sequential recurrence, built on the host
  std::vector<uint64_t> trace(4 * n_trace);
  uint64_t st = 0;
  for (uint64_t i = 0; i < n_trace; ++i) {
    const uint64_t leaf = i < n_leaves ? leaves[i] % gl::P : 0;
    const uint64_t sq = gl::mul(st, st);
    trace[i] = i % gl::P;
    trace[n_trace + i] = leaf;
    trace[2 * n_trace + i] = st;
    trace[3 * n_trace + i] = sq;
    st = gl::add(sq, leaf);
  }
  cudaStream_t s = c->stream;
  DBuf d_trace(4 * n_trace, s), d_lde(4 * n0, s), d_c(n0, s);
  cuda_check(cudaMemcpyAsync(d_trace.p, trace.data(), trace.size() * 8, cudaMemcpyHostToDevice, s), "h2d");
  lde_device(c, d_trace.p, 4, n_trace, blowup, 1, d_lde.p);
  const uint64_t lam[3] = {1, 2, 3};  // comb_coeffs (prover.rs:100-102)
  merge_device(c, SG_AIR_HASH_ROLLUP, d_lde.p, 4, n_trace, blowup, lam, 3, phi_mode, d_c.p);
  sg_fri_params p;
  sg_build_params(n0, pi, stir ? 1 : 0, &p);
  std::vector<uint8_t> proof = stir_prove_device(c, d_c.p, n0, p);
  if (self_verify && !stir_verify(decode_proof(proof.data(), proof.size()), p))
    throw SgError{SG_EVERIFY, "self-verification of the produced proof failed"};
  return proof;
}

// ------------------------------------------------------------------ hash-AIR pipeline
// Phi of a hash AIR on a materialised LDE (deep_ali_merge_sha256, lib.rs:453-545;
// deep_ali_merge_sha512, lib.rs:561-641): point i reads rows i and i + blowup.
void merge_hash_device(sg_ctx* c, const HashAir& air, const uint64_t* d_lde, uint64_t n_trace, uint64_t blowup,
                       const uint64_t* lambdas, int phi_mode, uint64_t* d_c, uint64_t n_blocks) {
  require(pow2(n_trace) && pow2(blowup), "merge: sizes must be powers of 2");
  require(phi_mode >= 0 && phi_mode <= 2, "merge: bad phi mode");
  const uint64_t n = n_trace * blowup;
  const unsigned ln = log2_exact(n);
  require(ln <= kMaxLogN, "merge: domain larger than 2^28");
  cudaStream_t s = c->stream;
  if (!phi_live(phi_mode, n)) {
    cuda_check(cudaMemsetAsync(d_c, 0, n * 8, s), "memset");
    return;
  }
  std::vector<uint64_t> lam(lambdas, lambdas + air.num_constraints);
  for (auto& x : lam) x %= gl::P;
  DBuf phi(n, s), d_lam(lam.size(), s), scratch(ntt_scratch_elems(1, ln), s);
  cuda_check(cudaMemcpyAsync(d_lam.p, lam.data(), lam.size() * 8, cudaMemcpyHostToDevice, s), "h2d");
  cuda_check(air.phi_points(d_lde, n, blowup, blowup, n_blocks, d_lam.p, phi.p, 1, 0, s), "phi");
  ntt(c, phi.p, phi.p, 1, n, n, ln, true, n, scratch.p);
  cuda_check(quotient_zh(phi.p, n, n_trace, d_c, s), "quotient");
  ntt(c, d_c, d_c, 1, n, n, ln, false, n > n_trace ? n - n_trace : n, scratch.p);
  cuda_check(cudaStreamSynchronize(s), "sync");  // lam (host) must outlive the copy
}

// The same merge without materialising the LDE: LDE point i = r + blowup a lies
// on coset r, whose evaluations are NTT_{n_trace}(c_k w_n0^{rk}), and point
// i + blowup is point a + 1 of the same coset. Each coset is produced, folded
// into Phi[r + blowup a] by the constraint kernel, and dropped.
void merge_hash_cosets(sg_ctx* c, const HashAir& air, const uint64_t* d_trace, uint64_t n_trace, uint64_t blowup,
                       uint64_t n_blocks, const uint64_t* lambdas, int phi_mode, uint64_t* d_c) {
  const uint64_t W = air.width, n = n_trace * blowup;
  const unsigned lt = log2_exact(n_trace), ln = log2_exact(n);
  require(pow2(n_trace) && pow2(blowup) && ln <= kMaxLogN, "merge: bad sizes");
  cudaStream_t s = c->stream;
  if (!phi_live(phi_mode, n)) {
    cuda_check(cudaMemsetAsync(d_c, 0, n * 8, s), "memset");
    return;
  }
  std::vector<uint64_t> lam(lambdas, lambdas + air.num_constraints);
  for (auto& x : lam) x %= gl::P;
  DBuf d_lam(lam.size(), s), phi(n, s), coef(W * n_trace, s), ev(W * n_trace, s);
  DBuf scratch(std::max(ntt_scratch_elems(W, lt), ntt_scratch_elems(1, ln)), s);
  cuda_check(cudaMemcpyAsync(d_lam.p, lam.data(), lam.size() * 8, cudaMemcpyHostToDevice, s), "h2d");
  ntt(c, d_trace, coef.p, (uint32_t)W, n_trace, n_trace, lt, true, n_trace, scratch.p);
  DBuf twist_tab(n_trace, s);
  for (uint64_t r = 0; r < blowup; ++r) {
    const uint64_t* evals = d_trace;  // coset 0 holds the trace values themselves
    if (r > 0) {
      // coefficient k times w_n^(r k), applied as the transform loads it, from a
      // table of the coset's n_trace powers (one load instead of two and a product)
      cuda_check(pow_table_device(c->tw, r, (int)ln, n_trace, twist_tab.p, s), "twist table");
      PowSpec twist;
      twist.tab = twist_tab.p;
      ntt(c, coef.p, ev.p, (uint32_t)W, n_trace, n_trace, lt, false, n_trace, scratch.p, &twist);
      evals = ev.p;
    }
    cuda_check(air.phi_points(evals, n_trace, 1, 1, n_blocks, d_lam.p, phi.p, blowup, r, s), "coset phi");
  }
  ntt(c, phi.p, phi.p, 1, n, n, ln, true, n, scratch.p);
  cuda_check(quotient_zh(phi.p, n, n_trace, d_c, s), "quotient");
  ntt(c, d_c, d_c, 1, n, n, ln, false, n > n_trace ? n - n_trace : n, scratch.p);
  cuda_check(cudaStreamSynchronize(s), "sync");  // lam (host) must outlive the copy
}

// prove_ds_ksk_binding (swarm-dns/src/prover.rs:512-585) for SHA-256, and the
// same pipeline for SHA-512 (whose reference prover is not written yet,
// sha512_air.rs:16-19): the host runs the compressions, the trace columns are
// expanded on the device, then LDE x32 -> merge with lambda_j = j + 1
// (prover.rs:100-102) -> STIR with build_params(n0, fs_binding).
void check_blowup(uint64_t blowup) {
  require(blowup >= 2 && blowup <= 1024 && pow2(blowup), "prove: blowup must be a power of 2 in [2, 1024]");
}

CEval hash_message_ceval(sg_ctx* c, const HashAir& air, const uint8_t* msg, uint64_t len,
                         const uint8_t fs_binding[32], int phi_mode, uint8_t* digest, uint64_t blowup) {
  check_blowup(blowup);
  std::vector<uint8_t> wit;
  uint64_t n_blocks = 0;
  const uint64_t n_trace = air.witness(msg, len, &wit, &n_blocks, digest);
  const uint64_t n0 = n_trace * blowup;
  require(log2_exact(n0) <= kMaxLogN, "prove: message too long for a 2^28 domain");
  cudaStream_t s = c->stream;
  const uint64_t lde_bytes = (uint64_t)air.width * n0 * 8;
  const bool cosets = c->wide_merge == SG_WIDE_MERGE_COSETS ||
                      (c->wide_merge == SG_WIDE_MERGE_AUTO && lde_bytes > (2ull << 30));
  DBuf d_trace((uint64_t)air.width * n_trace, s), d_c(n0, s);
  {
    DBuf d_wit((wit.size() + 7) / 8, s);
    cuda_check(cudaMemcpyAsync(d_wit.p, wit.data(), wit.size(), cudaMemcpyHostToDevice, s), "h2d");
    cuda_check(air.expand(d_wit.p, n_blocks, n_trace, d_trace.p, s), "trace expand");
    cuda_check(cudaStreamSynchronize(s), "sync");  // wit (host) must outlive its copy
  }
  std::vector<uint64_t> lam(air.num_constraints);
  for (uint64_t j = 0; j < lam.size(); ++j) lam[j] = j + 1;
  if (cosets) {
    merge_hash_cosets(c, air, d_trace.p, n_trace, blowup, n_blocks, lam.data(), phi_mode, d_c.p);
  } else {
    DBuf d_lde((uint64_t)air.width * n0, s);
    lde_device(c, d_trace.p, air.width, n_trace, blowup, 1, d_lde.p);
    merge_hash_device(c, air, d_lde.p, n_trace, blowup, lam.data(), phi_mode, d_c.p, n_blocks);
  }
  cuda_check(cudaStreamSynchronize(s), "sync");
  CEval r;
  r.d_c = std::move(d_c);
  r.n0 = n0;
  sg_build_params(n0, fs_binding, 1, &r.params);
  return r;
}

std::vector<uint8_t> prove_from_ceval(sg_ctx* c, const CEval& ce, bool self_verify) {
  std::vector<uint8_t> proof = stir_prove_device(c, ce.d_c.p, ce.n0, ce.params);
  if (self_verify && !stir_verify(decode_proof(proof.data(), proof.size()), ce.params))
    throw SgError{SG_EVERIFY, "self-verification of the produced proof failed"};
  return proof;
}

std::vector<uint8_t> prove_hash_message(sg_ctx* c, const HashAir& air, const uint8_t* msg, uint64_t len,
                                        const uint8_t fs_binding[32], int phi_mode, bool self_verify,
                                        uint8_t* digest, uint64_t blowup) {
  return prove_from_ceval(c, hash_message_ceval(c, air, msg, len, fs_binding, phi_mode, digest, blowup),
                          self_verify);
}

// ------------------------------------------------------------------ RSA-2048 pipeline
void rsa_witnesses(const uint8_t* n_be, const uint8_t* s_be, const uint8_t* em_be, uint64_t n_records,
                   std::vector<rsa::RecordW>* recs, std::vector<rsa::RowW>* rows) {
  recs->resize(n_records);
  rows->resize(n_records * rsa::N_TRACE);
  const uint64_t hw = std::max(1u, std::thread::hardware_concurrency());
  const uint64_t nt = std::min<uint64_t>(n_records, std::min<uint64_t>(hw, 32));
  std::vector<SgError> errs(nt);
  std::vector<char> failed(nt, 0);
  auto work = [&](uint64_t w) {
    try {
      for (uint64_t r = w; r < n_records; r += nt)
        rsa::witness(n_be + 256 * r, s_be + 256 * r, em_be + 256 * r, &(*recs)[r], &(*rows)[r * rsa::N_TRACE]);
    } catch (const SgError& e) {
      errs[w] = e;
      failed[w] = 1;
    }
  };
  if (nt <= 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    for (uint64_t w = 0; w < nt; ++w) th.emplace_back(work, w);
    for (auto& t : th) t.join();
  }
  for (uint64_t w = 0; w < nt; ++w)
    if (failed[w]) throw errs[w];
}

CEval rsa2048_ceval(sg_ctx* c, const uint8_t* n_be, const uint8_t* s_be, const uint8_t* em_be, uint64_t n_records,
                    const uint8_t pi[32], uint64_t blowup) {
  require(n_records >= 1 && n_records <= 65535, "prove_rsa2048: 1 to 65535 records");
  check_blowup(blowup);
  std::vector<rsa::RecordW> recs;
  std::vector<rsa::RowW> rows;
  rsa_witnesses(n_be, s_be, em_be, n_records, &recs, &rows);
  const uint64_t n_trace = rsa::N_TRACE, n0 = n_trace * blowup;
  const uint64_t W = n_records * rsa::WIDTH;
  const unsigned ln = log2_exact(n0);
  cudaStream_t s = c->stream;
  const uint64_t rec_bytes = recs.size() * sizeof(rsa::RecordW), row_bytes = rows.size() * sizeof(rsa::RowW);
  DBuf d_trace(W * n_trace, s), d_c(n0, s);
  {
    DBuf d_wit((rec_bytes + row_bytes + 7) / 8, s);
    uint8_t* base = (uint8_t*)d_wit.p;
    static_assert(sizeof(rsa::RecordW) % 8 == 0, "witness alignment");
    cuda_check(cudaMemcpyAsync(base, recs.data(), rec_bytes, cudaMemcpyHostToDevice, s), "h2d");
    cuda_check(cudaMemcpyAsync(base + rec_bytes, rows.data(), row_bytes, cudaMemcpyHostToDevice, s), "h2d");
    cuda_check(rsa_expand((const rsa::RecordW*)base, (const rsa::RowW*)(base + rec_bytes), n_records, d_trace.p, s),
               "rsa trace expand");
    cuda_check(cudaStreamSynchronize(s), "sync");  // the host witnesses must outlive their copies
  }
  {
    DBuf d_lde(W * n0, s), phi(n0, s), part(n_records > 1 ? n_records * n0 : 0, s);
    DBuf scratch(ntt_scratch_elems(1, ln), s);
    lde_device(c, d_trace.p, W, n_trace, blowup, 1, d_lde.p);
    cuda_check(rsa_phi(d_lde.p, n_records, n_trace, blowup, part.p, phi.p, s), "rsa phi");
    ntt(c, phi.p, phi.p, 1, n0, n0, ln, true, n0, scratch.p);
    cuda_check(quotient_zh(phi.p, n0, n_trace, d_c.p, s), "quotient");
    ntt(c, d_c.p, d_c.p, 1, n0, n0, ln, false, n0 - n_trace, scratch.p);
  }
  CEval r;
  r.d_c = std::move(d_c);
  r.n0 = n0;
  sg_build_params(n0, pi, 1, &r.params);
  return r;
}

std::vector<uint8_t> prove_rsa2048(sg_ctx* c, const uint8_t* n_be, const uint8_t* s_be, const uint8_t* em_be,
                                   uint64_t n_records, const uint8_t pi[32], bool self_verify, uint64_t blowup) {
  return prove_from_ceval(c, rsa2048_ceval(c, n_be, s_be, em_be, n_records, pi, blowup), self_verify);
}

std::vector<uint8_t> prove_sha256_message(sg_ctx* c, const uint8_t* msg, uint64_t len, const uint8_t fs_binding[32],
                                          int phi_mode, bool self_verify, uint8_t digest[32], uint64_t blowup) {
  return prove_hash_message(c, sha256_hash_air(), msg, len, fs_binding, phi_mode, self_verify, digest, blowup);
}

}  // namespace sg
