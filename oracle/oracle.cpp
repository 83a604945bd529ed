// oracle/oracle.cpp — CPU restatement of the stark-stir-swarm prover hot path.
//
// TEST INFRASTRUCTURE ONLY: the checker for the GPU library, never shipped or
// called by it. Restates, in plain C++ (OpenMP for the multi-threaded CPU
// baseline), the reference functions cited beside each routine below (paths
// relative to stark-stir-swarm/crates/). Pinned by the reference's golden
// proofs primary-state/proofs/{outer-rollup,inner-shard-000[123]}.bin.
#include "oracle.h"

#include <omp.h>

#include <algorithm>
#include <array>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "air.hpp"
#include "ed25519_air.hpp"
#include "p256_air.hpp"
#include "rsa2048_air.hpp"
#include "chacha.hpp"
#include "gl.hpp"
#include "keccak.hpp"
#include "merkle.hpp"
#include "ntt.hpp"
#include "transcript.hpp"

using namespace orc;

namespace {

// ------------------------------------------------------------------ LDE
// trace_import.rs:251-281 lde_trace_columns: per column iFFT_{n}, zero-pad to
// n*blowup, FFT. `shift` != 1 evaluates on the coset shift*<w> instead
// (coefficient k scaled by shift^k); the reference path always uses 1.
void lde_column(const Fp* col, size_t n, size_t n0, Fp shift, Fp* out) {
  std::vector<Fp> c(col, col + n);
  ifft(c.data(), n);
  for (size_t i = 0; i < n0; ++i) out[i] = Fp();
  Fp s = Fp::raw(1);
  for (size_t k = 0; k < n; ++k) {
    out[k] = c[k] * s;
    s = s * shift;
  }
  fft(out, n0);
}

// ------------------------------------------------------------------ quotient
// lib.rs:190-228 poly_div_zh: q[k-m] = d[k] + q[k] for k = n-1 .. m; the
// remainder (coefficients below m) is dropped as in release builds.
std::vector<Fp> poly_div_zh(const std::vector<Fp>& d, size_t m) {
  size_t n = d.size();
  if (n <= m) return std::vector<Fp>(1);
  size_t ql = n - m;
  std::vector<Fp> q(ql);
  for (size_t k = n; k-- > m;) {
    Fp qk = k < ql ? q[k] : Fp();
    q[k - m] = d[k] + qk;
  }
  return q;
}

bool phi_live(int mode, size_t n) {
  if (mode == ORC_PHI_ALWAYS) return true;
  if (mode == ORC_PHI_NEVER) return false;
  return n >= 4096;  // enable_parallel (lib.rs:20-33) with >1 rayon thread
}

// lib.rs:343-437 deep_ali_merge_general and :453-545 deep_ali_merge_sha256.
// Constraint j at LDE point i uses cur = row i, nxt = row (i+blowup) mod n and
// trace_row = i / blowup (lib.rs:270-319).
std::vector<Fp> merge(int air, const Fp* lde, size_t w, size_t n_trace, size_t blowup, const Fp* lambdas,
                      size_t k, int phi_mode, size_t n_blocks) {
  size_t n = n_trace * blowup;
  std::vector<Fp> phi(n);
  if (phi_live(phi_mode, n)) {
#pragma omp parallel
    {
      std::vector<Fp> cur(w), nxt(w), cv(k);
#pragma omp for schedule(static)
      for (long i = 0; i < (long)n; ++i) {
        size_t ni = (i + blowup) % n;
        for (size_t c = 0; c < w; ++c) {
          cur[c] = lde[c * n + i];
          nxt[c] = lde[c * n + ni];
        }
        eval_constraints(air, cur.data(), nxt.data(), i / blowup, n_blocks, cv.data());
        Fp acc;
        for (size_t j = 0; j < k; ++j) acc = acc + lambdas[j] * cv[j];
        phi[i] = acc;
      }
    }
  }
  ifft(phi.data(), n);
  std::vector<Fp> q = poly_div_zh(phi, n_trace);
  q.resize(n);
  fft(q.data(), n);
  return q;
}

// ------------------------------------------------------------------ STIR helpers
// fri.rs:404-457 fft_in_place_ext: X[k] = sum_j x[j] root^{jk} with base-field twiddles.
void dft_ext(std::vector<Fp6>& v, Fp root) {
  size_t m = v.size();
  std::vector<Fp6> out(m);
  for (size_t k = 0; k < m; ++k) {
    Fp6 acc = e_zero();
    Fp wk = pow(root, k), w = Fp::raw(1);
    for (size_t j = 0; j < m; ++j) {
      acc = e_add(acc, e_scale(v[j], w));
      w = w * wk;
    }
    out[k] = acc;
  }
  v.swap(out);
}

// fri.rs:468-502 interpolate_stir_coset / :714-752 interpolate_coset_ext:
// d = (1/m) DFT_{zeta^-1}(evals); coeff_k = d_k * shift^-k.
std::vector<Fp6> interp_coset(const std::vector<Fp6>& evals, Fp zeta) {
  std::vector<Fp6> d = evals;
  dft_ext(d, inv(zeta));
  Fp minv = inv(Fp::raw(d.size()));
  for (auto& x : d) x = e_scale(x, minv);
  return d;
}

std::vector<Fp6> interp_stir_coset(const std::vector<Fp6>& evals, const Fp6& z, Fp zeta) {
  std::vector<Fp6> d = interp_coset(evals, zeta);
  Fp6 zi;
  if (!e_inv(z, &zi)) throw std::runtime_error("STIR z_ell must be nonzero");
  Fp6 p = e_one();
  for (auto& x : d) {
    x = e_mul(x, p);
    p = e_mul(p, zi);
  }
  return d;
}

std::vector<Fp6> interp_base_coset(const std::vector<Fp6>& fibre, Fp omega_b, Fp zeta) {
  std::vector<Fp6> d = interp_coset(fibre, zeta);
  Fp obi = omega_b.is_zero() ? Fp::raw(1) : inv(omega_b);
  Fp p = Fp::raw(1);
  for (auto& x : d) {
    x = e_scale(x, p);
    p = p * obi;
  }
  return d;
}

// fri.rs:338-391 evaluate_ood_coset: component iFFTs then Horner at zeta^j * z.
void evaluate_ood_coset(const std::vector<Fp6>& f, const Fp6& z, Fp omega, size_t m, std::vector<Fp6>* evals,
                        std::vector<Fp6>* interp) {
  size_t n = f.size();
  std::vector<std::vector<Fp>> comp(6, std::vector<Fp>(n));
#pragma omp parallel for schedule(static) if (n >= 4096)
  for (long i = 0; i < (long)n; ++i)
    for (int c = 0; c < 6; ++c) comp[c][i] = f[i].comp(c);
#pragma omp parallel for schedule(static, 1)
  for (int c = 0; c < 6; ++c) ifft(comp[c].data(), n);
  Fp zeta = pow(omega, n / m);
  std::vector<Fp6> pts(m);
  Fp zp = Fp::raw(1);
  for (size_t j = 0; j < m; ++j) {
    pts[j] = e_scale(z, zp);
    zp = zp * zeta;
  }
  evals->assign(m, e_zero());
#pragma omp parallel for schedule(static, 1)
  for (long j = 0; j < (long)m; ++j) {
    Fp6 r = e_zero();
    for (size_t k = n; k-- > 0;) {
      Fp6 ck;
      for (int c = 0; c < 6; ++c) ck.set_comp(c, comp[c][k]);
      r = e_add(e_mul(r, pts[j]), ck);
    }
    (*evals)[j] = r;
  }
  *interp = interp_stir_coset(*evals, z, zeta);
}

// fri.rs:670-707 extract_all_coset_coefficients
std::vector<std::vector<Fp6>> extract_coset_coeffs(const std::vector<Fp6>& f, Fp omega, size_t m) {
  size_t n = f.size(), nn = n / m;
  Fp zeta = pow(omega, nn);
  std::vector<std::vector<Fp6>> out(nn);
#pragma omp parallel for schedule(static) if (nn >= 4096)
  for (long b = 0; b < (long)nn; ++b) {
    std::vector<Fp6> fib(m);
    for (size_t j = 0; j < m; ++j) fib[j] = f[b + j * nn];
    out[b] = interp_base_coset(fib, pow(omega, b), zeta);
  }
  return out;
}

// fri.rs:754-771 interpolation_fold_ext
std::vector<Fp6> fold(const std::vector<std::vector<Fp6>>& tuples, const Fp6& alpha) {
  size_t m = tuples.empty() ? 0 : tuples[0].size();
  std::vector<Fp6> ap(m);
  Fp6 a = e_one();
  for (size_t i = 0; i < m; ++i) {
    ap[i] = a;
    a = e_mul(a, alpha);
  }
  std::vector<Fp6> out(tuples.size());
#pragma omp parallel for schedule(static) if (tuples.size() >= 4096)
  for (long b = 0; b < (long)tuples.size(); ++b) {
    Fp6 s = e_zero();
    for (size_t i = 0; i < m; ++i) s = e_add(s, e_mul(tuples[b][i], ap[i]));
    out[b] = s;
  }
  return out;
}

// fri.rs:875-907 ext_evals_to_coeffs
std::vector<Fp6> ext_evals_to_coeffs(const std::vector<Fp6>& ev) {
  size_t n = ev.size();
  if (n <= 1) return ev;
  std::vector<Fp6> out(n);
  for (int c = 0; c < 6; ++c) {
    std::vector<Fp> col(n);
    for (size_t i = 0; i < n; ++i) col[i] = ev[i].comp(c);
    ifft(col.data(), n);
    for (size_t i = 0; i < n; ++i) out[i].set_comp(c, col[i]);
  }
  return out;
}

Fp6 eval_poly_ext(const std::vector<Fp6>& coeffs, const Fp6& x) {
  Fp6 r = e_zero();
  for (size_t i = coeffs.size(); i-- > 0;) r = e_add(e_mul(r, x), coeffs[i]);
  return r;
}

// fri.rs:816-856 batched_degree_check_ext
bool batched_degree_check(const std::vector<std::vector<Fp6>>& tuples, const Fp6& beta, size_t d_final) {
  size_t nf = tuples.size();
  if (nf == 0) return true;
  size_t m = tuples[0].size();
  std::vector<Fp6> g(nf);
  for (size_t b = 0; b < nf; ++b) {
    Fp6 s = e_zero(), bp = e_one();
    for (size_t i = 0; i < m; ++i) {
      s = e_add(s, e_mul(tuples[b][i], bp));
      bp = e_mul(bp, beta);
    }
    g[b] = s;
  }
  std::vector<Fp6> c = ext_evals_to_coeffs(g);
  for (size_t k = d_final; k < nf; ++k)
    if (!c[k].is_zero()) return false;
  return true;
}

// fri.rs:1105-1129 bind_statement_to_transcript (E::DEGREE = 6)
void bind_statement(Transcript& tr, const orc_fri_params& p, size_t n0) {
  if (p.has_pi) {
    tr.absorb_str("CAIRO-PUBLIC-INPUTS-V1");
    tr.absorb_bytes(p.pi_hash, 32);
  }
  tr.absorb_str("DEEP-FRI-STATEMENT-V2");
  tr.absorb_u64(n0);
  tr.absorb_u64(p.schedule_len);
  for (size_t i = 0; i < p.schedule_len; ++i) tr.absorb_u64(p.schedule[i]);
  tr.absorb_u64(p.seed_z);
  tr.absorb_u64(6);
  tr.absorb_u64(p.coeff_commit_final ? 1 : 0);
  tr.absorb_u64(p.stir ? 1 : 0);
}

// fri.rs:1044-1058 index_seed + index_from_seed
size_t query_index(Fp query_seed, size_t q, size_t n0) {
  Fp fields[3] = {query_seed, Fp(0), Fp((uint64_t)q)};
  Fp seed = hash_fields_tagged("FRI/index", fields, 3);
  uint8_t sb[32] = {0};
  memcpy(sb, &seed.v, 8);
  size_t np2 = 1;
  while (np2 < n0) np2 <<= 1;
  return (size_t)(stdrng_first_u64(sb) & (np2 - 1)) % n0;
}

struct TreeCfg {
  std::vector<size_t> ar;
  uint64_t label;
};
TreeCfg layer_cfg(size_t n, size_t m, uint64_t label) {
  size_t a = std::max<size_t>(2, pick_arity_for_layer(n, m));
  return {std::vector<size_t>(merkle_depth(n, a), a), label};
}

struct ProxQuery {
  uint64_t base, raw;
  std::vector<uint64_t> fib_idx;
  std::vector<Fp> fib_vals;
  MerkleOpening f0_open;
  Fp6 f_next;
  bool has_l1;
  MerkleOpening l1_open;
};

// classic FRI query (fri.rs:1236-1263): per-layer refs (i, child_pos,
// parent_index, parent_pos), payloads (f, s, q), the f0 opening, final index
struct ClassicQuery {
  std::vector<std::array<uint64_t, 4>> refs;
  std::vector<std::array<Fp6, 3>> pay;
  MerkleOpening f0_open;
  uint64_t final_index = 0;
};

struct StirProof {
  bool stir = true;
  std::vector<std::vector<MerkleOpening>> layer_open;  // classic: layer_proofs.layers[ell].openings
  std::vector<MerkleOpening> f0_openings;               // classic
  std::vector<ClassicQuery> queries;                    // classic
  Digest root_f0;
  std::vector<Digest> roots;
  std::vector<Fp6> fz;
  std::vector<Fp6> final_coeffs;
  uint64_t n0;
  Fp omega0;
  bool has_ct;
  std::vector<std::vector<Fp6>> coeff_tuples;
  bool has_croot;
  Digest coeff_root;
  std::vector<std::vector<Fp6>> coset_evals;
  std::vector<ProxQuery> prox;
};

// ------------------------------------------------------------------ classic FRI
// fri.rs:255-336 compute_q_layer_ext_on_ext: f(z) from the component iFFTs and
// Horner, then q_i = (f_i - f(z)) / (w^i - z).
void q_layer(const std::vector<Fp6>& f, const Fp6& z, Fp omega, std::vector<Fp6>* q, Fp6* fz) {
  const size_t n = f.size();
  std::vector<std::vector<Fp>> comp(6, std::vector<Fp>(n));
  for (size_t i = 0; i < n; ++i)
    for (int c = 0; c < 6; ++c) comp[c][i] = f[i].comp(c);
  for (int c = 0; c < 6; ++c) ifft(comp[c].data(), n);
  Fp6 r = e_zero();
  for (size_t k = n; k-- > 0;) {
    Fp6 ck;
    for (int c = 0; c < 6; ++c) ck.set_comp(c, comp[c][k]);
    r = e_add(e_mul(r, z), ck);
  }
  *fz = r;
  q->assign(n, e_zero());
#pragma omp parallel for schedule(static) if (n >= 1024)
  for (long i = 0; i < (long)n; ++i) {
    Fp6 d = e_sub(e_from(pow(omega, (uint64_t)i)), z), di;
    if (!e_inv(d, &di)) throw std::runtime_error("DEEP point on the domain");
    (*q)[i] = e_mul(e_sub(f[i], r), di);
  }
}

// fri.rs:1356-1362 ext_leaf_fields: the 18 components of (f, s, q)
std::vector<Fp> ext_leaf_rows(const std::vector<Fp6>& f, const std::vector<Fp6>& s, const std::vector<Fp6>& q) {
  std::vector<Fp> rows(f.size() * 18);
  for (size_t i = 0; i < f.size(); ++i)
    for (int k = 0; k < 6; ++k) {
      rows[i * 18 + k] = f[i].comp(k);
      rows[i * 18 + 6 + k] = s[i].comp(k);
      rows[i * 18 + 12 + k] = q[i].comp(k);
    }
  return rows;
}

// fri.rs:1900-2055 deep_fri_prove, classic branch: fri.rs:1398-1718
// fri_build_transcript (stir = false) and fri.rs:1724-1807 fri_prove_queries.
StirProof classic_prove(const std::vector<Fp>& f0, const orc_fri_params& p) {
  const size_t n0 = f0.size(), L = p.schedule_len;
  const bool use_cc = p.coeff_commit_final && L > 0;
  const size_t normal = use_cc ? L - 1 : L;
  StirProof pr;
  pr.stir = false;
  pr.n0 = n0;
  pr.omega0 = root_of_unity(log2_exact(n0));
  Transcript tr("FRI/FS");
  bind_statement(tr, p, n0);
  // f0 tree (fri.rs:1060-1076): one value per leaf, arity pick(n0, 16), label 0xFF
  TreeCfg f0cfg = layer_cfg(n0, 16, 0xFF);
  MerkleTree f0tree(f0cfg.ar, f0cfg.label);
  f0tree.build(f0, 1);
  pr.root_f0 = f0tree.root();
  tr.absorb_bytes(pr.root_f0.data(), HASH_BYTES);
  const Fp6 z = tr.challenge_ext("z_fp3");

  std::vector<std::vector<Fp6>> layers, s_layers, q_layers;
  layers.emplace_back(n0);
  for (size_t i = 0; i < n0; ++i) layers[0][i] = e_from(f0[i]);
  std::vector<MerkleTree> trees;
  size_t cur = n0;
  auto commit = [&](size_t ell, size_t m) {
    TreeCfg c = layer_cfg(cur, m, ell);
    MerkleTree t(c.ar, c.label);
    t.build(ext_leaf_rows(layers[ell], s_layers[ell], q_layers[ell]), 18);
    pr.roots.push_back(t.root());
    trees.push_back(std::move(t));
  };
  for (size_t ell = 0; ell < normal; ++ell) {
    const size_t m = p.schedule[ell], nn = cur / m;
    const Fp6 alpha = tr.challenge_ext("alpha");
    const Fp omega = root_of_unity(log2_exact(cur));
    std::vector<Fp6> q;
    Fp6 fz;
    q_layer(layers[ell], z, omega, &q, &fz);
    pr.fz.push_back(fz);
    auto tuples = extract_coset_coeffs(layers[ell], omega, m);
    std::vector<Fp6> next = fold(tuples, alpha);
    std::vector<Fp6> sl(cur);  // compute_s_layer_from_coeffs (fri.rs:773-789)
    for (size_t i = 0; i < cur; ++i) sl[i] = next[i % nn];
    s_layers.push_back(std::move(sl));
    q_layers.push_back(std::move(q));
    commit(ell, m);
    tr.absorb_ext(fz);
    tr.absorb_bytes(pr.roots.back().data(), HASH_BYTES);
    layers.push_back(std::move(next));
    cur = nn;
  }
  pr.has_ct = pr.has_croot = false;
  if (use_cc) {
    const size_t ell = L - 1, m = p.schedule[ell], nf = cur / m;
    const Fp omega = root_of_unity(log2_exact(cur));
    std::vector<Fp6> q;
    Fp6 fz;
    q_layer(layers[ell], z, omega, &q, &fz);
    pr.fz.push_back(fz);
    s_layers.emplace_back(cur, e_zero());
    q_layers.push_back(std::move(q));
    commit(ell, m);
    tr.absorb_ext(fz);
    tr.absorb_bytes(pr.roots.back().data(), HASH_BYTES);
    auto tuples = extract_coset_coeffs(layers[ell], omega, m);
    TreeCfg cc = layer_cfg(nf, 16, 0xFE);
    MerkleTree ct(cc.ar, cc.label);
    std::vector<Fp> rows(nf * m * 6);
    for (size_t b = 0; b < nf; ++b)
      for (size_t i = 0; i < m; ++i)
        for (int k = 0; k < 6; ++k) rows[(b * m + i) * 6 + k] = tuples[b][i].comp(k);
    ct.build(rows, m * 6);
    pr.coeff_root = ct.root();
    tr.absorb_bytes(pr.coeff_root.data(), HASH_BYTES);
    const Fp6 alpha = tr.challenge_ext("alpha");
    (void)tr.challenge_ext("beta_deg");
    layers.push_back(fold(tuples, alpha));
    pr.coeff_tuples = std::move(tuples);
    pr.has_ct = pr.has_croot = true;
    cur = nf;
  }
  auto all = ext_evals_to_coeffs(layers[L]);
  const size_t d_final = std::min<size_t>(p.d_final, all.size());
  pr.final_coeffs.assign(all.begin(), all.begin() + d_final);
  for (auto& c : pr.final_coeffs) tr.absorb_ext(c);
  const Fp query_seed = tr.challenge_field("query_seed");

  pr.layer_open.resize(L);
  for (size_t qi = 0; qi < p.r; ++qi) {
    ClassicQuery cq;
    size_t i = query_index(query_seed, qi, n0), n = n0;
    for (size_t ell = 0; ell < L; ++ell) {
      const size_t m = p.schedule[ell], nn = n / m;
      cq.refs.push_back({(uint64_t)i, (uint64_t)(i % m), (uint64_t)(i % nn), 0});
      cq.pay.push_back({layers[ell][i], s_layers[ell][i], q_layers[ell][i]});
      pr.layer_open[ell].push_back(trees[ell].open(i));
      i %= nn;
      n = nn;
    }
    cq.final_index = i;
    cq.f0_open = f0tree.open(cq.refs[0][0]);
    pr.f0_openings.push_back(cq.f0_open);
    pr.queries.push_back(std::move(cq));
  }
  return pr;
}

// ------------------------------------------------------------------ prover
// fri.rs:1900-2055 deep_fri_prove (STIR branch) with fri.rs:1398-1718
// fri_build_transcript and fri.rs:1813-1893 stir_prove_proximity_queries.
StirProof stir_prove(const std::vector<Fp>& f0, const orc_fri_params& p) {
  size_t n0 = f0.size();
  size_t L = p.schedule_len;
  if (L == 0) throw std::runtime_error("empty folding schedule");
  if (!p.stir) return classic_prove(f0, p);
  bool use_cc = p.coeff_commit_final && L > 0;
  size_t normal = use_cc ? L - 1 : L;
  StirProof pr;
  pr.n0 = n0;
  pr.omega0 = root_of_unity(log2_exact(n0));

  Transcript tr("FRI/FS");
  bind_statement(tr, p, n0);

  // packed f0 tree: leaf b = {f0[b + j*n0/m0]}_j, label 0xFF
  size_t m0 = p.schedule[0], nn0 = n0 / m0;
  TreeCfg f0cfg = layer_cfg(nn0, 16, 0xFF);
  MerkleTree f0tree(f0cfg.ar, f0cfg.label);
  {
    std::vector<Fp> rows(n0);
    for (size_t b = 0; b < nn0; ++b)
      for (size_t j = 0; j < m0; ++j) rows[b * m0 + j] = f0[b + j * nn0];
    f0tree.build(rows, m0);
  }
  pr.root_f0 = f0tree.root();
  tr.absorb_bytes(pr.root_f0.data(), HASH_BYTES);
  Fp6 z = tr.challenge_ext("z_fp3");

  std::vector<std::vector<Fp6>> layers;
  layers.emplace_back(n0);
  for (size_t i = 0; i < n0; ++i) layers[0][i] = e_from(f0[i]);
  std::vector<Fp6> alphas;
  Fp6 zc = z;
  size_t cur = n0;
  std::vector<MerkleTree> trees;

  auto commit_layer = [&](size_t ell, size_t m) {
    const auto& f = layers[ell];
    TreeCfg c = layer_cfg(cur, m, ell);
    MerkleTree t(c.ar, c.label);
    std::vector<Fp> rows(cur * 6);
    for (size_t i = 0; i < cur; ++i)
      for (int k = 0; k < 6; ++k) rows[i * 6 + k] = f[i].comp(k);
    t.build(rows, 6);
    pr.roots.push_back(t.root());
    trees.push_back(std::move(t));
  };

  for (size_t ell = 0; ell < normal; ++ell) {
    size_t m = p.schedule[ell];
    Fp6 alpha = tr.challenge_ext("alpha");
    alphas.push_back(alpha);
    Fp omega = root_of_unity(log2_exact(cur));
    std::vector<Fp6> ev, ip;
    evaluate_ood_coset(layers[ell], zc, omega, m, &ev, &ip);
    pr.fz.push_back(ev[0]);
    zc = e_pow(zc, m);
    auto tuples = extract_coset_coeffs(layers[ell], omega, m);
    commit_layer(ell, m);
    for (auto& e : ev) tr.absorb_ext(e);
    tr.absorb_bytes(pr.roots.back().data(), HASH_BYTES);
    pr.coset_evals.push_back(ev);
    layers.push_back(fold(tuples, alpha));
    cur /= m;
  }
  pr.has_ct = pr.has_croot = false;
  if (use_cc) {
    size_t ell = L - 1, m = p.schedule[ell];
    Fp omega = root_of_unity(log2_exact(cur));
    std::vector<Fp6> ev, ip;
    evaluate_ood_coset(layers[ell], zc, omega, m, &ev, &ip);
    pr.fz.push_back(ev[0]);
    zc = e_pow(zc, m);
    commit_layer(ell, m);
    for (auto& e : ev) tr.absorb_ext(e);
    tr.absorb_bytes(pr.roots.back().data(), HASH_BYTES);
    pr.coset_evals.push_back(ev);
    auto tuples = extract_coset_coeffs(layers[ell], omega, m);
    size_t nf = cur / m;
    TreeCfg cc = layer_cfg(nf, 16, 0xFE);
    MerkleTree ct(cc.ar, cc.label);
    std::vector<Fp> rows(nf * m * 6);
    for (size_t b = 0; b < nf; ++b)
      for (size_t i = 0; i < m; ++i)
        for (int k = 0; k < 6; ++k) rows[(b * m + i) * 6 + k] = tuples[b][i].comp(k);
    ct.build(rows, m * 6);
    pr.coeff_root = ct.root();
    tr.absorb_bytes(pr.coeff_root.data(), HASH_BYTES);
    Fp6 alpha = tr.challenge_ext("alpha");
    alphas.push_back(alpha);
    (void)tr.challenge_ext("beta_deg");
    layers.push_back(fold(tuples, alpha));
    pr.coeff_tuples = std::move(tuples);
    pr.has_ct = pr.has_croot = true;
    cur = nf;
  }
  auto all = ext_evals_to_coeffs(layers[L]);
  size_t d_final = std::min<size_t>(p.d_final, all.size());
  pr.final_coeffs.assign(all.begin(), all.begin() + d_final);
  for (auto& c : pr.final_coeffs) tr.absorb_ext(c);
  Fp query_seed = tr.challenge_field("query_seed");

  for (size_t q = 0; q < p.s0; ++q) {
    ProxQuery pq;
    pq.raw = query_index(query_seed, q, n0);
    pq.base = pq.raw % nn0;
    for (size_t j = 0; j < m0; ++j) {
      pq.fib_idx.push_back(pq.base + j * nn0);
      pq.fib_vals.push_back(f0[pq.base + j * nn0]);
    }
    pq.f0_open = f0tree.open(pq.base);
    pq.has_l1 = L >= 2;
    if (pq.has_l1) {
      pq.f_next = layers[1][pq.base];
      pq.l1_open = trees[1].open(pq.base);
    } else {
      pq.f_next = e_zero();
    }
    pr.prox.push_back(std::move(pq));
  }
  return pr;
}

// ------------------------------------------------------------------ serializer
// ark-serialize 0.4.2 Compress::Yes on DeepFriProof (fri.rs:1235-1300) and
// MerkleOpening (merkle/src/lib.rs:135-140): [u8; HASH_BYTES] raw, usize/len as le64,
// F as le64 canonical, Fp6 as 6 components, Option as one flag byte + payload.
struct Writer {
  std::vector<uint8_t> b;
  void u8(uint8_t x) { b.push_back(x); }
  void u64(uint64_t x) { for (int i = 0; i < 8; ++i) b.push_back((uint8_t)(x >> (8 * i))); }
  void dig(const Digest& d) { b.insert(b.end(), d.begin(), d.end()); }
  void ext(const Fp6& e) { for (int i = 0; i < 6; ++i) u64(e.comp(i).v); }
  void opening(const MerkleOpening& o) {
    dig(o.leaf);
    u64(o.path.size());
    for (auto& lv : o.path) {
      u64(lv.size());
      for (auto& d : lv) dig(d);
    }
    u64(o.index);
  }
};

std::vector<uint8_t> serialize(const StirProof& pr) {
  Writer w;
  w.dig(pr.root_f0);
  w.u64(pr.roots.size());
  for (auto& r : pr.roots) w.dig(r);
  w.u64(pr.layer_open.size());  // layer_proofs.layers (classic FRI only)
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
  w.u64(pr.omega0.v);
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
  w.u8(pr.stir);
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
    for (auto v : q.fib_vals) w.u64(v.v);
    w.opening(q.f0_open);
    w.ext(q.f_next);
    w.u8(q.has_l1);
    if (q.has_l1) w.opening(q.l1_open);
  }
  return w.b;
}

struct Reader {
  const uint8_t* p;
  size_t n, o = 0;
  Reader(const uint8_t* pp, size_t nn) : p(pp), n(nn) {}
  void need(size_t k) {
    if (o + k > n) throw std::runtime_error("proof truncated");
  }
  uint8_t u8() { need(1); return p[o++]; }
  uint64_t u64() {
    need(8);
    uint64_t x = 0;
    for (int i = 0; i < 8; ++i) x |= (uint64_t)p[o + i] << (8 * i);
    o += 8;
    return x;
  }
  uint64_t len() {
    uint64_t x = u64();
    if (x > n) throw std::runtime_error("implausible length");
    return x;
  }
  Digest dig() { need(HASH_BYTES); Digest d; memcpy(d.data(), p + o, HASH_BYTES); o += HASH_BYTES; return d; }
  Fp fe() {
    uint64_t x = u64();
    if (x >= P) throw std::runtime_error("non-canonical field element");
    return Fp::raw(x);
  }
  Fp6 ext() { Fp6 e; for (int i = 0; i < 6; ++i) e.set_comp(i, fe()); return e; }
  bool flag() {
    uint8_t f = u8();
    if (f > 1) throw std::runtime_error("bad option flag");
    return f;
  }
  MerkleOpening opening() {
    MerkleOpening o2;
    o2.leaf = dig();
    uint64_t nl = len();
    for (uint64_t i = 0; i < nl; ++i) {
      uint64_t ns = len();
      std::vector<Digest> v;
      for (uint64_t j = 0; j < ns; ++j) v.push_back(dig());
      o2.path.push_back(v);
    }
    o2.index = u64();
    return o2;
  }
};

StirProof deserialize(const uint8_t* b, size_t n) {
  Reader r(b, n);
  StirProof pr;
  pr.root_f0 = r.dig();
  uint64_t k = r.len();
  for (uint64_t i = 0; i < k; ++i) pr.roots.push_back(r.dig());
  k = r.len();
  for (uint64_t i = 0; i < k; ++i) {
    uint64_t m = r.len();
    std::vector<MerkleOpening> lo;
    for (uint64_t j = 0; j < m; ++j) lo.push_back(r.opening());
    pr.layer_open.push_back(std::move(lo));
  }
  k = r.len();
  for (uint64_t i = 0; i < k; ++i) pr.f0_openings.push_back(r.opening());
  k = r.len();
  for (uint64_t i = 0; i < k; ++i) {
    ClassicQuery q;
    uint64_t m = r.len();
    for (uint64_t j = 0; j < m; ++j) q.refs.push_back({r.u64(), r.u64(), r.u64(), r.u64()});
    m = r.len();
    for (uint64_t j = 0; j < m; ++j) q.pay.push_back({r.ext(), r.ext(), r.ext()});
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
      std::vector<Fp6> t;
      for (uint64_t j = 0; j < m; ++j) t.push_back(r.ext());
      pr.coeff_tuples.push_back(t);
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
    std::vector<Fp6> v;
    for (uint64_t j = 0; j < m; ++j) v.push_back(r.ext());
    pr.coset_evals.push_back(v);
  }
  if (!r.flag()) throw std::runtime_error("missing stir_proximity_queries");
  k = r.len();
  for (uint64_t i = 0; i < k; ++i) {
    ProxQuery q;
    q.base = r.u64();
    q.raw = r.u64();
    uint64_t m = r.len();
    for (uint64_t j = 0; j < m; ++j) q.fib_idx.push_back(r.u64());
    m = r.len();
    for (uint64_t j = 0; j < m; ++j) q.fib_vals.push_back(r.fe());
    q.f0_open = r.opening();
    q.f_next = r.ext();
    q.has_l1 = r.flag();
    if (q.has_l1) q.l1_open = r.opening();
    pr.prox.push_back(std::move(q));
  }
  if (r.o != n) throw std::runtime_error("trailing bytes");
  return pr;
}

// ------------------------------------------------------------------ verifier
// coeff-commit checks shared by both branches (fri.rs:2275-2322): tuple shapes,
// the recomputed coefficient root, and the batched degree check.
bool coeff_commit_ok(const StirProof& pr, const orc_fri_params& p, const std::vector<size_t>& sizes,
                     const Fp6& beta) {
  const size_t L = p.schedule_len;
  if (!pr.has_ct) return false;
  const size_t nf = sizes[L], mf = p.schedule[L - 1];
  if (pr.coeff_tuples.size() != nf) return false;
  for (auto& t : pr.coeff_tuples)
    if (t.size() != mf) return false;
  TreeCfg cc = layer_cfg(nf, 16, 0xFE);
  MerkleTree ct(cc.ar, cc.label);
  std::vector<Fp> rows;
  for (auto& t : pr.coeff_tuples)
    for (auto& e : t)
      for (int k = 0; k < 6; ++k) rows.push_back(e.comp(k));
  ct.build(rows, mf * 6);
  if (ct.root() != pr.coeff_root) return false;
  return batched_degree_check(pr.coeff_tuples, beta, p.d_final);
}

// fri.rs:2136-2258 + 2517-2707 deep_fri_verify, classic branch.
bool classic_verify(const StirProof& pr, const orc_fri_params& p) {
  const size_t L = p.schedule_len;
  if (L == 0 || pr.stir) return false;
  std::vector<size_t> sizes{(size_t)pr.n0};
  for (size_t i = 0; i < L; ++i) {
    if (p.schedule[i] == 0 || sizes.back() % p.schedule[i]) return false;
    sizes.push_back(sizes.back() / p.schedule[i]);
  }
  const bool use_cc = p.coeff_commit_final && L > 0;
  if (pr.roots.size() < L || pr.fz.size() < L) return false;
  Transcript tr("FRI/FS");
  bind_statement(tr, p, pr.n0);
  tr.absorb_bytes(pr.root_f0.data(), HASH_BYTES);
  const Fp6 z = tr.challenge_ext("z_fp3");
  std::vector<Fp6> alphas;
  Fp6 beta;
  for (size_t ell = 0; ell < L; ++ell) {
    const bool last_cc = use_cc && ell == L - 1;
    if (!last_cc) alphas.push_back(tr.challenge_ext("alpha"));
    tr.absorb_ext(pr.fz[ell]);
    tr.absorb_bytes(pr.roots[ell].data(), HASH_BYTES);
    if (last_cc) {
      if (!pr.has_croot) return false;
      tr.absorb_bytes(pr.coeff_root.data(), HASH_BYTES);
      alphas.push_back(tr.challenge_ext("alpha"));
      beta = tr.challenge_ext("beta_deg");
    }
  }
  for (auto& c : pr.final_coeffs) tr.absorb_ext(c);
  const Fp query_seed = tr.challenge_field("query_seed");
  if (pr.final_coeffs.size() != p.d_final) return false;
  if (use_cc && !coeff_commit_ok(pr, p, sizes, beta)) return false;
  const Fp omega_final = sizes[L] >= 2 ? root_of_unity(log2_exact(sizes[L])) : Fp::raw(1);
  if (pr.queries.size() < p.r || pr.layer_open.size() < L) return false;
  TreeCfg f0cfg = layer_cfg(pr.n0, 16, 0xFF);
  for (size_t qi = 0; qi < p.r; ++qi) {
    const ClassicQuery& q = pr.queries[qi];
    if (q.refs.size() < L || q.pay.size() < L) return false;
    const size_t i0 = query_index(query_seed, qi, pr.n0);
    size_t ei = i0;
    for (size_t ell = 0; ell < L; ++ell) {
      if (q.refs[ell][0] != ei) return false;
      ei %= sizes[ell] / p.schedule[ell];
    }
    if (q.final_index != ei) return false;
    if (!verify_opening(f0cfg.ar, f0cfg.label, pr.root_f0, q.f0_open)) return false;
    for (int k = 1; k < 6; ++k)
      if (!q.pay[0][0].comp(k).is_zero()) return false;  // layer 0 is in the base field
    const Fp f0v = q.pay[0][0].comp(0);
    if (leaf_hash(f0cfg.ar[0], f0cfg.label, q.f0_open.index, &f0v, 1) != q.f0_open.leaf) return false;
    if (q.f0_open.index != i0) return false;
    for (size_t ell = 0; ell < L; ++ell) {
      if (pr.layer_open[ell].size() <= qi) return false;
      const MerkleOpening& o = pr.layer_open[ell][qi];
      const auto& pl = q.pay[ell];
      const size_t i = q.refs[ell][0];
      TreeCfg cfg = layer_cfg(sizes[ell], p.schedule[ell], ell);
      if (!verify_opening(cfg.ar, cfg.label, pr.roots[ell], o)) return false;
      if (o.index != i) return false;
      Fp vals[18];
      for (int t = 0; t < 3; ++t)
        for (int k = 0; k < 6; ++k) vals[t * 6 + k] = pl[t].comp(k);
      if (leaf_hash(cfg.ar[0], cfg.label, o.index, vals, 18) != o.leaf) return false;
      const Fp omega = root_of_unity(log2_exact(sizes[ell]));
      const Fp xi = pow(omega, i);
      // DEEP check: q (x_i - z) = f - f(z)
      if (e_mul(pl[2], e_sub(e_from(xi), z)) != e_sub(pl[0], pr.fz[ell])) return false;
      const Fp6 x_final = e_from(pow(omega_final, q.final_index));
      if (ell == L - 1 && use_cc) {
        const size_t m = p.schedule[ell];
        if (q.final_index >= pr.coeff_tuples.size()) return false;
        const auto& t = pr.coeff_tuples[q.final_index];
        Fp6 h = e_zero(), fv = e_zero(), ap = e_one();
        Fp xp = Fp::raw(1);
        for (size_t k = 0; k < m; ++k) {
          h = e_add(h, e_scale(t[k], xp));
          xp = xp * xi;
          fv = e_add(fv, e_mul(t[k], ap));
          ap = e_mul(ap, alphas[L - 1]);
        }
        if (pl[0] != h) return false;
        if (fv != eval_poly_ext(pr.final_coeffs, x_final)) return false;
      } else {
        const Fp6 f_next = ell + 1 < L ? q.pay[ell + 1][0] : eval_poly_ext(pr.final_coeffs, x_final);
        if (pl[1] != f_next) return false;
      }
    }
  }
  return true;
}

// fri.rs:2136-2521 deep_fri_verify, STIR branch.
bool stir_verify(const StirProof& pr, const orc_fri_params& p) {
  size_t L = p.schedule_len;
  if (!p.stir) return classic_verify(pr, p);
  if (L == 0 || !pr.stir) return false;
  std::vector<size_t> sizes{(size_t)pr.n0};
  for (size_t i = 0; i < L; ++i) {
    if (sizes.back() % p.schedule[i]) return false;
    sizes.push_back(sizes.back() / p.schedule[i]);
  }
  bool use_cc = p.coeff_commit_final && L > 0;
  size_t normal = use_cc ? L - 1 : L;
  if (pr.roots.size() < L || pr.coset_evals.size() < L) return false;
  Transcript tr("FRI/FS");
  bind_statement(tr, p, pr.n0);
  tr.absorb_bytes(pr.root_f0.data(), HASH_BYTES);
  Fp6 z = tr.challenge_ext("z_fp3");
  Fp6 zc = z;
  std::vector<std::vector<Fp6>> interps;
  std::vector<Fp6> alphas;
  Fp6 beta;
  for (size_t ell = 0; ell < L; ++ell) {
    size_t m = p.schedule[ell];
    bool last_cc = use_cc && ell == L - 1;
    if (!last_cc) alphas.push_back(tr.challenge_ext("alpha"));
    const auto& ev = pr.coset_evals[ell];
    if (ev.size() != m) return false;
    Fp zeta = pow(root_of_unity(log2_exact(sizes[ell])), sizes[ell] / m);
    interps.push_back(interp_stir_coset(ev, zc, zeta));
    zc = e_pow(zc, m);
    for (auto& e : ev) tr.absorb_ext(e);
    tr.absorb_bytes(pr.roots[ell].data(), HASH_BYTES);
    if (last_cc) {
      if (!pr.has_croot) return false;
      tr.absorb_bytes(pr.coeff_root.data(), HASH_BYTES);
      alphas.push_back(tr.challenge_ext("alpha"));
      beta = tr.challenge_ext("beta_deg");
    }
  }
  (void)normal;
  for (auto& c : pr.final_coeffs) tr.absorb_ext(c);
  Fp query_seed = tr.challenge_field("query_seed");
  if (pr.final_coeffs.size() != p.d_final) return false;
  for (size_t ell = 0; ell < L; ++ell) {
    size_t m = p.schedule[ell];
    Fp6 acc = e_zero(), ap = e_one();
    for (size_t k = 0; k < m; ++k) {
      acc = e_add(acc, e_mul(interps[ell][k], ap));
      ap = e_mul(ap, alphas[ell]);
    }
    Fp6 expect;
    if (ell + 1 < L) {
      expect = pr.coset_evals[ell + 1][0];
    } else {
      Fp6 zf = z;
      for (size_t i = 0; i < L; ++i) zf = e_pow(zf, p.schedule[i]);
      expect = eval_poly_ext(pr.final_coeffs, zf);
    }
    if (acc != expect) return false;
  }
  if (use_cc) {
    if (!pr.has_ct) return false;
    size_t nf = sizes[L], mf = p.schedule[L - 1];
    if (pr.coeff_tuples.size() != nf) return false;
    for (auto& t : pr.coeff_tuples)
      if (t.size() != mf) return false;
    TreeCfg cc = layer_cfg(nf, 16, 0xFE);
    MerkleTree ct(cc.ar, cc.label);
    std::vector<Fp> rows;
    for (auto& t : pr.coeff_tuples)
      for (auto& e : t)
        for (int k = 0; k < 6; ++k) rows.push_back(e.comp(k));
    ct.build(rows, mf * 6);
    if (ct.root() != pr.coeff_root) return false;
    if (!batched_degree_check(pr.coeff_tuples, beta, p.d_final)) return false;
  }
  Fp omega_final = sizes[L] >= 2 ? root_of_unity(log2_exact(sizes[L])) : Fp::raw(1);
  if (pr.prox.size() != p.s0) return false;
  size_t n0 = pr.n0, m0 = p.schedule[0], nn = sizes[0] / m0;
  Fp omega0 = root_of_unity(log2_exact(sizes[0]));
  Fp zeta0 = pow(omega0, nn);
  TreeCfg f0cfg = layer_cfg(nn, 16, 0xFF);
  TreeCfg l1cfg = L >= 2 ? layer_cfg(sizes[1], p.schedule[1], 1) : TreeCfg{};
  std::vector<Fp6> ap0(m0);
  {
    Fp6 a = e_one();
    for (size_t k = 0; k < m0; ++k) { ap0[k] = a; a = e_mul(a, alphas[0]); }
  }
  for (size_t qi = 0; qi < pr.prox.size(); ++qi) {
    const auto& q = pr.prox[qi];
    size_t raw = query_index(query_seed, qi, n0);
    if (q.raw != raw || q.base != raw % nn) return false;
    if (q.fib_idx.size() != m0 || q.fib_vals.size() != m0) return false;
    for (size_t j = 0; j < m0; ++j)
      if (q.fib_idx[j] != q.base + j * nn) return false;
    if (!verify_opening(f0cfg.ar, f0cfg.label, pr.root_f0, q.f0_open)) return false;
    if (q.f0_open.index != q.base) return false;
    if (leaf_hash(f0cfg.ar[0], f0cfg.label, q.f0_open.index, q.fib_vals.data(), m0) != q.f0_open.leaf) return false;
    std::vector<Fp6> fib(m0);
    for (size_t j = 0; j < m0; ++j) fib[j] = e_from(q.fib_vals[j]);
    auto ct = interp_base_coset(fib, pow(omega0, q.base), zeta0);
    Fp6 fv = e_zero();
    for (size_t k = 0; k < m0; ++k) fv = e_add(fv, e_mul(ct[k], ap0[k]));
    if (L >= 2) {
      if (!q.has_l1) return false;
      if (!verify_opening(l1cfg.ar, l1cfg.label, pr.roots[1], q.l1_open)) return false;
      if (q.l1_open.index != q.base) return false;
      Fp vals[6];
      for (int k = 0; k < 6; ++k) vals[k] = q.f_next.comp(k);
      if (leaf_hash(l1cfg.ar[0], l1cfg.label, q.l1_open.index, vals, 6) != q.l1_open.leaf) return false;
      if (fv != q.f_next) return false;
    } else {
      Fp6 xf = e_from(pow(omega_final, q.base));
      if (fv != eval_poly_ext(pr.final_coeffs, xf)) return false;
    }
  }
  return true;
}

}  // namespace

// ================================================================== C API
extern "C" {

uint64_t orc_fp_add(uint64_t a, uint64_t b) { return (Fp(a) + Fp(b)).v; }
uint64_t orc_fp_sub(uint64_t a, uint64_t b) { return (Fp(a) - Fp(b)).v; }
uint64_t orc_fp_mul(uint64_t a, uint64_t b) { return (Fp(a) * Fp(b)).v; }
uint64_t orc_fp_pow(uint64_t a, uint64_t e) { return pow(Fp(a), e).v; }
uint64_t orc_fp_inv(uint64_t a) { return inv(Fp(a)).v; }
static Fp6 load6(const uint64_t* a) {
  Fp6 e;
  for (int i = 0; i < 6; ++i) e.set_comp(i, Fp(a[i]));
  return e;
}
static void store6(const Fp6& e, uint64_t* o) {
  for (int i = 0; i < 6; ++i) o[i] = e.comp(i).v;
}
void orc_fp6_mul(const uint64_t a[6], const uint64_t b[6], uint64_t out[6]) { store6(e_mul(load6(a), load6(b)), out); }
int orc_fp6_inv(const uint64_t a[6], uint64_t out[6]) {
  Fp6 r;
  if (!e_inv(load6(a), &r)) return -1;
  store6(r, out);
  return 0;
}
void orc_chacha_block(const uint8_t key[32], uint64_t counter, uint64_t stream, int rounds, uint32_t out[16]) {
  uint32_t k[8];
  memcpy(k, key, 32);
  chacha_block(k, counter, stream, rounds, out);
}

void orc_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int orc_get_threads(void) { return omp_get_max_threads(); }

int orc_ntt(uint64_t* a, size_t n, int inverse) {
  if (n == 0 || (n & (n - 1))) return -1;
  for (size_t i = 0; i < n; ++i)
    if (a[i] >= P) return -2;
  if (inverse) ifft((Fp*)a, n); else fft((Fp*)a, n);
  return 0;
}

int orc_lde(const uint64_t* trace, size_t w, size_t n_trace, size_t blowup, uint64_t shift, uint64_t* out) {
  if (w == 0) return -1;
  if (n_trace == 0 || (n_trace & (n_trace - 1))) return -2;
  if (blowup < 2 || (blowup & (blowup - 1))) return -3;
  size_t n0 = n_trace * blowup;
#pragma omp parallel for schedule(dynamic, 1)
  for (long c = 0; c < (long)w; ++c)
    lde_column((const Fp*)trace + c * n_trace, n_trace, n0, Fp(shift), (Fp*)out + c * n0);
  return 0;
}

void orc_sha3_256(const uint8_t* msg, size_t len, uint8_t out[32]) { sha3_256(msg, len, out); }
uint64_t orc_stdrng_first_u64(const uint8_t seed[32]) { return stdrng_first_u64(seed); }
uint64_t orc_root_of_unity(unsigned log_n) { return root_of_unity(log_n).v; }

int orc_hash_bytes(void) { return HASH_BYTES; }
void orc_sha3_selected(const uint8_t* msg, size_t len, uint8_t* out) {
  SelectedHasher h;
  h.update(msg, len);
  h.finalize(out);
}

int orc_merkle_root(const uint64_t* rows, size_t n_leaves, size_t width, const uint64_t* arities, size_t depth,
                    uint64_t label, uint8_t* root) {
  if (n_leaves == 0 || depth == 0) return -1;
  std::vector<size_t> ar(arities, arities + depth);
  MerkleTree t(ar, label);
  std::vector<Fp> v((const Fp*)rows, (const Fp*)rows + n_leaves * width);
  try {
    t.build(v, width);
  } catch (...) {
    return -2;
  }
  memcpy(root, t.root().data(), HASH_BYTES);
  return 0;
}

int orc_hash_rollup_trace(const uint64_t* leaves, size_t n_leaves, size_t n_trace, uint64_t* trace) {
  build_hash_rollup_trace(leaves, n_leaves, n_trace, (Fp*)trace);
  return 0;
}

int orc_merge(int air, const uint64_t* lde, size_t w, size_t n_trace, size_t blowup, const uint64_t* lambdas,
              size_t k, int phi_mode, uint64_t* c_eval) {
  if (air_width(air) != w || air_num_constraints(air) != k) return -1;
  if (n_trace == 0 || (n_trace & (n_trace - 1)) || blowup == 0 || (blowup & (blowup - 1))) return -2;
  auto c = merge(air, (const Fp*)lde, w, n_trace, blowup, (const Fp*)lambdas, k, phi_mode, 1);
  memcpy(c_eval, c.data(), c.size() * 8);
  return 0;
}

// deep_ali_merge_sha256 (lib.rs:453-545): the SHA-256 AIR with an explicit block count.
int orc_merge_sha256(const uint64_t* lde, size_t n_trace, size_t blowup, const uint64_t* lambdas, size_t n_blocks,
                     int phi_mode, uint64_t* c_eval) {
  if (n_trace == 0 || (n_trace & (n_trace - 1)) || blowup == 0 || (blowup & (blowup - 1))) return -2;
  auto c = merge(ORC_AIR_SHA256, (const Fp*)lde, sha::WIDTH, n_trace, blowup, (const Fp*)lambdas,
                 sha::NUM_CONSTRAINTS, phi_mode, n_blocks);
  memcpy(c_eval, c.data(), c.size() * 8);
  return 0;
}

// build_sha256_trace_multi (sha256_air.rs:429-472): WIDTH x height column-major.
int orc_sha256_trace(const uint8_t* msg, size_t len, uint64_t* out, size_t cap_elems, size_t* height,
                     size_t* n_blocks) {
  std::vector<Fp> tr;
  *height = sha::build_trace_multi(msg, len, &tr, n_blocks);
  if (tr.size() > cap_elems) return -3;
  memcpy(out, tr.data(), tr.size() * 8);
  return 0;
}

// eval_sha256_constraints at one row (for known-answer / tamper tests).
int orc_sha256_eval(const uint64_t* cur, const uint64_t* nxt, size_t row, size_t n_blocks, uint64_t* out) {
  sha::eval((const Fp*)cur, (const Fp*)nxt, row, n_blocks, (Fp*)out);
  return 0;
}

// prove_ds_ksk_binding core (swarm-dns/src/prover.rs:512-585): multi-block trace ->
// LDE x32 -> merge_sha256 (lambda_j = j+1) -> STIR with build_params(n0, fs_binding).
// digest receives the asserted SHA-256 digest read from the H-state.
int orc_prove_sha256(const uint8_t* msg, size_t len, const uint8_t fs_binding[32], int phi_mode, size_t blowup,
                     uint8_t* out, size_t cap, size_t* out_len, uint8_t digest[32]) {
  if (blowup < 2 || (blowup & (blowup - 1))) return -2;
  std::vector<Fp> tr;
  size_t n_blocks = 0;
  const size_t n_trace = sha::build_trace_multi(msg, len, &tr, &n_blocks);
  const size_t digest_row = sha::ROWS_PER_BLOCK * (n_blocks - 1) + 65;
  for (int k = 0; k < 8; ++k) {
    uint32_t wd = (uint32_t)tr[(sha::H0 + k) * n_trace + digest_row].v;
    for (int b = 0; b < 4; ++b) digest[4 * k + b] = (uint8_t)(wd >> (24 - 8 * b));
  }
  const size_t n0 = n_trace * blowup;
  std::vector<uint64_t> lde(sha::WIDTH * n0), c(n0);
  orc_lde((const uint64_t*)tr.data(), sha::WIDTH, n_trace, blowup, 1, lde.data());
  std::vector<uint64_t> lam(sha::NUM_CONSTRAINTS);
  for (size_t j = 0; j < lam.size(); ++j) lam[j] = j + 1;
  orc_merge_sha256(lde.data(), n_trace, blowup, lam.data(), n_blocks, phi_mode, c.data());
  orc_fri_params p;
  orc_build_params(n0, fs_binding, 1, &p);
  return orc_stir_prove(c.data(), n0, &p, out, cap, out_len);
}

// deep_ali_merge_sha512 (lib.rs:561-641): the SHA-512 AIR with an explicit block count.
int orc_merge_sha512(const uint64_t* lde, size_t n_trace, size_t blowup, const uint64_t* lambdas, size_t n_blocks,
                     int phi_mode, uint64_t* c_eval) {
  if (n_trace == 0 || (n_trace & (n_trace - 1)) || blowup == 0 || (blowup & (blowup - 1))) return -2;
  auto c = merge(AIR_SHA512, (const Fp*)lde, sha512::WIDTH, n_trace, blowup, (const Fp*)lambdas,
                 sha512::NUM_CONSTRAINTS, phi_mode, n_blocks);
  memcpy(c_eval, c.data(), c.size() * 8);
  return 0;
}

// build_sha512_trace_multi (sha512_air.rs:551-578): WIDTH x height column-major.
int orc_sha512_trace(const uint8_t* msg, size_t len, uint64_t* out, size_t cap_elems, size_t* height,
                     size_t* n_blocks) {
  std::vector<Fp> tr;
  *height = sha512::build_trace_multi(msg, len, &tr, n_blocks);
  if (tr.size() > cap_elems) return -3;
  memcpy(out, tr.data(), tr.size() * 8);
  return 0;
}

// eval_sha512_constraints at one row (for known-answer / tamper tests).
int orc_sha512_eval(const uint64_t* cur, const uint64_t* nxt, size_t row, size_t n_blocks, uint64_t* out) {
  sha512::eval((const Fp*)cur, (const Fp*)nxt, row, n_blocks, (Fp*)out);
  return 0;
}

// SHA-512 proof with the SHA-256 binding's parameters (the reference has no
// SHA-512 prover yet, sha512_air.rs:16-19): trace -> LDE x32 -> merge_sha512
// (lambda_j = j+1) -> STIR with build_params(n0, fs_binding). digest receives the
// 64-byte digest read from the H-state (row 128 (n_blocks - 1) + 81).
int orc_prove_sha512(const uint8_t* msg, size_t len, const uint8_t fs_binding[32], int phi_mode, size_t blowup,
                     uint8_t* out, size_t cap, size_t* out_len, uint8_t digest[64]) {
  if (blowup < 2 || (blowup & (blowup - 1))) return -2;
  std::vector<Fp> tr;
  size_t n_blocks = 0;
  const size_t n_trace = sha512::build_trace_multi(msg, len, &tr, &n_blocks);
  const size_t digest_row = sha512::ROWS_PER_BLOCK * (n_blocks - 1) + 81;
  for (int k = 0; k < 8; ++k) {
    const uint64_t lo = tr[(sha512::H0_LO + 2 * k) * n_trace + digest_row].v;
    const uint64_t hi = tr[(sha512::H0_LO + 2 * k + 1) * n_trace + digest_row].v;
    const uint64_t wd = lo | hi << 32;
    for (int b = 0; b < 8; ++b) digest[8 * k + b] = (uint8_t)(wd >> (56 - 8 * b));
  }
  const size_t n0 = n_trace * blowup;
  std::vector<uint64_t> lde(sha512::WIDTH * n0), c(n0);
  orc_lde((const uint64_t*)tr.data(), sha512::WIDTH, n_trace, blowup, 1, lde.data());
  std::vector<uint64_t> lam(sha512::NUM_CONSTRAINTS);
  for (size_t j = 0; j < lam.size(); ++j) lam[j] = j + 1;
  orc_merge_sha512(lde.data(), n_trace, blowup, lam.data(), n_blocks, phi_mode, c.data());
  orc_fri_params p;
  orc_build_params(n0, fs_binding, 1, &p);
  return orc_stir_prove(c.data(), n0, &p, out, cap, out_len);
}

// ------------------------------------------------------------------ RSA-2048
// eval_rsa_stacked_per_row (rsa2048_stacked_air.rs:56-70): n_records records of
// rsa2048_exp_air.rs side by side; cur/nxt hold n_records * 11041 cells.
int orc_rsa_eval(const uint64_t* cur, const uint64_t* nxt, size_t row, size_t n_trace, size_t n_records,
                 uint64_t* out) {
  for (size_t r = 0; r < n_records; ++r)
    rsa::eval_record((const Fp*)cur + r * rsa::WIDTH, (const Fp*)nxt + r * rsa::WIDTH, row, n_trace,
                     (Fp*)out + r * rsa::CONSTRAINTS);
  return 0;
}

// deep_ali_merge_rsa_exp_multirow(_streaming) / deep_ali_merge_rsa_stacked_streaming
// (lib.rs:1694-1823, 1827-1945, 1949-2070): Phi is always evaluated (no
// parallel-build gate), lambda_j = j + 1 over the concatenated constraints,
// point i reads rows i and i + blowup, then iFFT, poly_div_zh, FFT.
int orc_merge_rsa(const uint64_t* lde, size_t n_records, size_t n_trace, size_t blowup, uint64_t* c_eval) {
  if (n_trace == 0 || (n_trace & (n_trace - 1)) || blowup == 0 || (blowup & (blowup - 1)) || n_records == 0)
    return -2;
  const size_t n = n_trace * blowup, w = n_records * rsa::WIDTH, k = n_records * rsa::CONSTRAINTS;
  const Fp* L = (const Fp*)lde;
  std::vector<Fp> phi(n);
#pragma omp parallel
  {
    std::vector<Fp> cur(w), nxt(w), cv(k);
#pragma omp for schedule(static)
    for (long i = 0; i < (long)n; ++i) {
      const size_t ni = (i + blowup) % n;
      for (size_t c = 0; c < w; ++c) {
        cur[c] = L[c * n + i];
        nxt[c] = L[c * n + ni];
      }
      orc_rsa_eval((const uint64_t*)cur.data(), (const uint64_t*)nxt.data(), i / blowup, n_trace, n_records,
                   (uint64_t*)cv.data());
      Fp acc;
      for (size_t j = 0; j < k; ++j) acc = acc + Fp(j + 1) * cv[j];
      phi[i] = acc;
    }
  }
  ifft(phi.data(), n);
  std::vector<Fp> q = poly_div_zh(phi, n_trace);
  q.resize(n);
  fft(q.data(), n);
  memcpy(c_eval, q.data(), n * 8);
  return 0;
}

// prove_rsa2048_record_v1.rs:150-205 (one record) and stacked_rsa_zone_prover.rs:
// 120-175 (n_records): trace (n_records * 11041 x n_trace, column-major) -> LDE x32
// (shift 1) -> RSA merge -> STIR with build_params(n0, pi) (schedule [8,8,8,2] at n0 1024).
int orc_prove_rsa(const uint64_t* trace, size_t n_records, size_t n_trace, const uint8_t pi[32], size_t blowup,
                  uint8_t* out, size_t cap, size_t* out_len) {
  if (blowup < 2 || (blowup & (blowup - 1))) return -2;
  const size_t n0 = n_trace * blowup, w = n_records * rsa::WIDTH;
  std::vector<uint64_t> lde(w * n0), c(n0);
  if (orc_lde(trace, w, n_trace, blowup, 1, lde.data()) != 0) return -2;
  if (orc_merge_rsa(lde.data(), n_records, n_trace, blowup, c.data()) != 0) return -2;
  orc_fri_params p;
  orc_build_params(n0, pi, 1, &p);
  return orc_stir_prove(c.data(), n0, &p, out, cap, out_len);
}

// ------------------------------------------------------------------ P-256 ECDSA double chain
// The row is described by a gadget table (8 u64 per gadget, in constraint order)
// and an 18-entry tail of chain bases (see p256_air.hpp).
size_t p256_constraints(const uint64_t* table, size_t n_gadgets) {
  size_t k = 180;
  for (size_t g = 0; g < n_gadgets; ++g) k += p256::gadget_constraints(table[g * p256::REC]);
  return k;
}

int orc_p256_eval(const uint64_t* cur, const uint64_t* nxt, size_t row, size_t n_trace, const uint64_t* table,
                  size_t n_gadgets, const uint64_t* tail, uint64_t* out) {
  Fp* o = (Fp*)out;
  for (size_t g = 0; g < n_gadgets; ++g) p256::eval_gadget((const Fp*)cur, table + g * p256::REC, o);
  p256::eval_tail((const Fp*)cur, (const Fp*)nxt, tail, row, n_trace, o);
  return (int)(o - (Fp*)out);
}

// deep_ali_merge_ecdsa_double_multirow_streaming: lambda_j = j + 1 over the row's
// constraints, Phi always evaluated, then iFFT, poly_div_zh, FFT.
int orc_merge_p256(const uint64_t* lde, size_t width, const uint64_t* table, size_t n_gadgets,
                   const uint64_t* tail, size_t n_trace, size_t blowup, uint64_t* c_eval) {
  if (n_trace == 0 || (n_trace & (n_trace - 1)) || blowup == 0 || (blowup & (blowup - 1))) return -2;
  const size_t n = n_trace * blowup, k = p256_constraints(table, n_gadgets);
  const Fp* L = (const Fp*)lde;
  std::vector<Fp> phi(n);
#pragma omp parallel
  {
    std::vector<Fp> cur(width), nxt(width), cv(k);
#pragma omp for schedule(dynamic, 4)
    for (long i = 0; i < (long)n; ++i) {
      const size_t ni = (i + blowup) % n;
      for (size_t c = 0; c < width; ++c) {
        cur[c] = L[c * n + i];
        nxt[c] = L[c * n + ni];
      }
      orc_p256_eval((const uint64_t*)cur.data(), (const uint64_t*)nxt.data(), i / blowup, n_trace, table, n_gadgets,
                    tail, (uint64_t*)cv.data());
      Fp acc;
      for (size_t j = 0; j < k; ++j) acc = acc + Fp(j + 1) * cv[j];
      phi[i] = acc;
    }
  }
  ifft(phi.data(), n);
  std::vector<Fp> q = poly_div_zh(phi, n_trace);
  q.resize(n);
  fft(q.data(), n);
  memcpy(c_eval, q.data(), n * 8);
  return 0;
}

// prove_ecdsa_record_v1.rs:193-240: trace -> LDE x32 (shift 1) -> merge -> STIR with
// build_params(n0, pi).
int orc_prove_p256(const uint64_t* trace, size_t width, const uint64_t* table, size_t n_gadgets,
                   const uint64_t* tail, size_t n_trace, const uint8_t pi[32], size_t blowup, uint8_t* out,
                   size_t cap, size_t* out_len) {
  if (blowup < 2 || (blowup & (blowup - 1))) return -2;
  const size_t n0 = n_trace * blowup;
  std::vector<uint64_t> lde(width * n0), c(n0);
  if (orc_lde(trace, width, n_trace, blowup, 1, lde.data()) != 0) return -2;
  if (orc_merge_p256(lde.data(), width, table, n_gadgets, tail, n_trace, blowup, c.data()) != 0) return -2;
  orc_fri_params p;
  orc_build_params(n0, pi, 1, &p);
  return orc_stir_prove(c.data(), n0, &p, out, cap, out_len);
}

// ------------------------------------------------------------------ Ed25519 verify AIR v16
int orc_ed25519_eval(const uint64_t* cur, const uint64_t* nxt, size_t row, const uint64_t* recs, size_t n_recs,
                     const uint64_t* pairs, size_t n_pairs, uint64_t* out) {
  (void)n_pairs;
  return (int)ed25519::eval_row((const Fp*)cur, (const Fp*)nxt, row, recs, n_recs, pairs, (Fp*)out);
}

// deep_ali_merge_ed25519_verify(_streaming) (lib.rs:707-974): trace row i / blowup,
// next row (i + blowup) mod n, lambda_j = j + 1, then iFFT, poly_div_zh, FFT.
int orc_merge_ed25519(const uint64_t* lde, size_t width, const uint64_t* recs, size_t n_recs, const uint64_t* pairs,
                      size_t n_pairs, size_t n_constraints, size_t n_trace, size_t blowup, uint64_t* c_eval) {
  if (n_trace == 0 || (n_trace & (n_trace - 1)) || blowup == 0 || (blowup & (blowup - 1))) return -2;
  const size_t n = n_trace * blowup, k = n_constraints;
  const Fp* L = (const Fp*)lde;
  std::vector<Fp> phi(n);
  int bad = 0;
#pragma omp parallel
  {
    std::vector<Fp> cur(width), nxt(width), cv(k);
#pragma omp for schedule(dynamic, 4)
    for (long i = 0; i < (long)n; ++i) {
      const size_t ni = (i + blowup) % n;
      for (size_t c = 0; c < width; ++c) {
        cur[c] = L[c * n + i];
        nxt[c] = L[c * n + ni];
      }
      if (orc_ed25519_eval((const uint64_t*)cur.data(), (const uint64_t*)nxt.data(), i / blowup, recs, n_recs, pairs,
                           n_pairs, (uint64_t*)cv.data()) != (int)k) {
#pragma omp atomic write
        bad = 1;
      }
      Fp acc;
      for (size_t j = 0; j < k; ++j)
        if (!cv[j].is_zero()) acc = acc + Fp(j + 1) * cv[j];
      phi[i] = acc;
    }
  }
  if (bad) return -3;
  ifft(phi.data(), n);
  std::vector<Fp> q = poly_div_zh(phi, n_trace);
  q.resize(n);
  fft(q.data(), n);
  memcpy(c_eval, q.data(), n * 8);
  return 0;
}

// prove_zsk_ksk_binding_v2 (swarm-dns/src/prover.rs:856-951): trace -> LDE (shift 1)
// -> merge -> STIR with build_params(n0, fs_binding).
int orc_prove_ed25519(const uint64_t* trace, size_t width, const uint64_t* recs, size_t n_recs,
                      const uint64_t* pairs, size_t n_pairs, size_t n_constraints, size_t n_trace,
                      const uint8_t fs_binding[32], size_t blowup, uint8_t* out, size_t cap, size_t* out_len) {
  if (blowup < 2 || (blowup & (blowup - 1))) return -2;
  const size_t n0 = n_trace * blowup;
  std::vector<uint64_t> lde(width * n0), c(n0);
  if (orc_lde(trace, width, n_trace, blowup, 1, lde.data()) != 0) return -2;
  const int rc = orc_merge_ed25519(lde.data(), width, recs, n_recs, pairs, n_pairs, n_constraints, n_trace, blowup,
                                   c.data());
  if (rc != 0) return rc;
  std::vector<uint64_t>().swap(lde);
  orc_fri_params p;
  orc_build_params(n0, fs_binding, 1, &p);
  return orc_stir_prove(c.data(), n0, &p, out, cap, out_len);
}

int orc_poly_div_zh(const uint64_t* coeffs, size_t n, size_t m, uint64_t* q) {
  std::vector<Fp> d((const Fp*)coeffs, (const Fp*)coeffs + n);
  auto r = poly_div_zh(d, m);
  memcpy(q, r.data(), r.size() * 8);
  return (int)r.size();
}

// swarm-dns/src/prover.rs:53-98 make_schedule + build_params
void orc_build_params(size_t n0, const uint8_t pi[32], int stir, orc_fri_params* out) {
  memset(out, 0, sizeof *out);
  unsigned lg = log2_exact(n0);
  if (stir) {
    for (unsigned i = 0; i < lg / 3; ++i) out->schedule[out->schedule_len++] = 8;
    if (lg % 3) out->schedule[out->schedule_len++] = 1u << (lg % 3);
  } else {
    for (unsigned i = 0; i < lg; ++i) out->schedule[out->schedule_len++] = 2;
  }
  out->r = out->s0 = 54;
  out->seed_z = 0xDEEFBAADull;
  out->coeff_commit_final = 1;
  out->d_final = 1;
  out->stir = stir;
  if (pi) {
    out->has_pi = 1;
    memcpy(out->pi_hash, pi, 32);
  }
}

int orc_stir_prove(const uint64_t* f0, size_t n0, const orc_fri_params* p, uint8_t* out, size_t cap, size_t* len) {
  try {
    std::vector<Fp> f((const Fp*)f0, (const Fp*)f0 + n0);
    auto b = serialize(stir_prove(f, *p));
    *len = b.size();
    if (b.size() > cap) return -3;
    memcpy(out, b.data(), b.size());
    return 0;
  } catch (...) {
    return -1;
  }
}

int orc_stir_verify(const uint8_t* proof, size_t len, const orc_fri_params* p) {
  try {
    return stir_verify(deserialize(proof, len), *p) ? 1 : 0;
  } catch (...) {
    return 0;
  }
}

int orc_prove_hash_rollup(const uint64_t* leaves, size_t n_leaves, const uint8_t pi[32], int phi_mode, uint8_t* out,
                          size_t cap, size_t* len) {
  size_t n_trace = 8;
  while (n_trace < n_leaves) n_trace <<= 1;
  const size_t blowup = 32;
  size_t n0 = n_trace * blowup;
  std::vector<uint64_t> trace(4 * n_trace), lde(4 * n0);
  build_hash_rollup_trace(leaves, n_leaves, n_trace, (Fp*)trace.data());
  orc_lde(trace.data(), 4, n_trace, blowup, 1, lde.data());
  uint64_t lam[3] = {1, 2, 3};  // comb_coeffs, prover.rs:100-102
  std::vector<uint64_t> c(n0);
  orc_merge(ORC_AIR_HASH_ROLLUP, lde.data(), 4, n_trace, blowup, lam, 3, phi_mode, c.data());
  orc_fri_params p;
  orc_build_params(n0, pi, 1, &p);
  return orc_stir_prove(c.data(), n0, &p, out, cap, len);
}

}  // extern "C"
