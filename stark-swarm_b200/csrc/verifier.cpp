// verifier.cpp — host DEEP-FRI verifier (deep_ali/src/fri.rs:2136-2707), STIR and
// classic branches.
//
// Used for the self-verification the reference worker performs before it
// reports a proof (swarm-dns/src/prover.rs:189-192) and exported as
// sg_stir_verify. Verification is a few hundred hashes and small
// interpolations, so it runs on the host.
#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "protocol.hpp"
#include "verifier.hpp"

namespace sg {
namespace {

using gl::Fp6;

// In-place DFT with root w (n a power of two), host.
void host_dft(std::vector<uint64_t>& a, uint64_t w) {
  size_t n = a.size();
  if (n <= 1) return;
  unsigned lg = 0;
  while ((size_t(1) << lg) < n) ++lg;
  for (size_t i = 0; i < n; ++i) {
    size_t j = 0;
    for (unsigned b = 0; b < lg; ++b)
      if (i >> b & 1) j |= size_t(1) << (lg - 1 - b);
    if (i < j) std::swap(a[i], a[j]);
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    uint64_t wl = gl::pow(w, n / len);
    for (size_t s = 0; s < n; s += len) {
      uint64_t t = 1;
      for (size_t j = 0; j < len / 2; ++j) {
        uint64_t u = a[s + j], v = gl::mul(a[s + j + len / 2], t);
        a[s + j] = gl::add(u, v);
        a[s + j + len / 2] = gl::sub(u, v);
        t = gl::mul(t, wl);
      }
    }
  }
}

unsigned log2u(uint64_t n) {
  unsigned l = 0;
  while ((1ull << l) < n) ++l;
  return l;
}

// d = (1/m) DFT_{zeta^-1}(evals) per component
std::vector<Fp6> coset_dft(const std::vector<Fp6>& ev, uint64_t zeta) {
  size_t m = ev.size();
  std::vector<Fp6> d(m);
  uint64_t zi = gl::inv(zeta), minv = gl::inv(m);
  for (int c = 0; c < 6; ++c) {
    std::vector<uint64_t> col(m);
    for (size_t j = 0; j < m; ++j) col[j] = ev[j].c[c];
    host_dft(col, zi);
    for (size_t k = 0; k < m; ++k) d[k].c[c] = gl::mul(col[k], minv);
  }
  return d;
}

// interpolate_stir_coset (fri.rs:468-502)
bool interp_stir(const std::vector<Fp6>& ev, const Fp6& z, uint64_t zeta, std::vector<Fp6>* out) {
  *out = coset_dft(ev, zeta);
  Fp6 zi;
  if (!gl::e_inv(z, &zi)) return false;
  Fp6 p = gl::e_one();
  for (auto& x : *out) {
    x = gl::e_mul(x, p);
    p = gl::e_mul(p, zi);
  }
  return true;
}

// interpolate_coset_ext (fri.rs:714-752)
std::vector<Fp6> interp_base(const std::vector<Fp6>& fib, uint64_t omega_b, uint64_t zeta) {
  std::vector<Fp6> d = coset_dft(fib, zeta);
  uint64_t obi = omega_b == 0 ? 1 : gl::inv(omega_b), p = 1;
  for (auto& x : d) {
    x = gl::e_scale(x, p);
    p = gl::mul(p, obi);
  }
  return d;
}

Fp6 eval_poly(const std::vector<Fp6>& c, const Fp6& x) {
  Fp6 r = gl::e_zero();
  for (size_t i = c.size(); i-- > 0;) r = gl::e_add(gl::e_mul(r, x), c[i]);
  return r;
}

Digest leaf_hash(uint64_t arity0, uint64_t label, uint64_t pos, const uint64_t* v, size_t n) {
  kc::Sha3Sel h;
  uint64_t ds[4] = {arity0, 0xFFFFFFFFull, pos, label};
  h.update(ds, 32);
  h.update(v, 8 * n);
  Digest d;
  h.finalize(d.data());
  return d;
}

bool verify_opening(const std::vector<uint32_t>& ar, uint64_t label, const Digest& root, const Opening& o) {
  Digest cur = o.leaf;
  uint64_t idx = o.index;
  for (size_t lv = 0; lv < o.path.size(); ++lv) {
    if (lv >= ar.size()) return false;
    uint64_t a = ar[lv], pos = idx % a;
    kc::Sha3Sel h;
    uint64_t ds[4] = {a, lv + 1, idx / a, label};
    h.update(ds, 32);
    size_t k = 0;
    for (uint64_t i = 0; i < a; ++i) {
      if (i == pos) {
        h.update(cur.data(), kc::kHashBytes);
      } else {
        if (k >= o.path[lv].size()) return false;
        h.update(o.path[lv][k++].data(), kc::kHashBytes);
      }
    }
    h.finalize(cur.data());
    idx /= a;
  }
  return cur == root;
}

Digest tree_root_host(const std::vector<std::vector<uint64_t>>& leaves, const std::vector<uint32_t>& ar,
                      uint64_t label) {
  std::vector<Digest> lv(leaves.size());
  for (size_t i = 0; i < leaves.size(); ++i) lv[i] = leaf_hash(ar[0], label, i, leaves[i].data(), leaves[i].size());
  size_t level = 0;
  while (lv.size() > 1) {
    uint64_t a = ar.at(level);
    while (lv.size() % a) lv.push_back(lv.back());
    std::vector<Digest> par(lv.size() / a);
    for (size_t p = 0; p < par.size(); ++p) {
      kc::Sha3Sel h;
      uint64_t ds[4] = {a, level + 1, p, label};
      h.update(ds, 32);
      for (uint64_t k = 0; k < a; ++k) h.update(lv[p * a + k].data(), kc::kHashBytes);
      h.finalize(par[p].data());
    }
    lv.swap(par);
    ++level;
  }
  return lv[0];
}

// coefficient commitment + batched degree check (fri.rs:816-856, 2275-2322)
bool coeff_commit_ok(const StirProof& pr, const sg_fri_params& p, const std::vector<uint64_t>& sizes,
                     const Fp6& beta) {
  const uint64_t L = p.schedule_len;
  if (!pr.has_ct) return false;
  const uint64_t nf = sizes[L], mf = p.schedule[L - 1];
  if (pr.coeff_tuples.size() != nf) return false;
  std::vector<std::vector<uint64_t>> leaves;
  for (auto& t : pr.coeff_tuples) {
    if (t.size() != mf) return false;
    std::vector<uint64_t> row;
    for (auto& e : t)
      for (int c = 0; c < 6; ++c) row.push_back(e.c[c]);
    leaves.push_back(std::move(row));
  }
  if (tree_root_host(leaves, layer_arities(nf, 16), 0xFE) != pr.coeff_root) return false;
  std::vector<Fp6> g(nf);
  for (uint64_t b = 0; b < nf; ++b) {
    Fp6 s = gl::e_zero(), bp = gl::e_one();
    for (uint64_t i = 0; i < mf; ++i) {
      s = gl::e_add(s, gl::e_mul(pr.coeff_tuples[b][i], bp));
      bp = gl::e_mul(bp, beta);
    }
    g[b] = s;
  }
  if (nf > 1) {
    uint64_t wi = gl::inv(gl::root_of_unity(log2u(nf))), ninv = gl::inv(nf);
    for (int c = 0; c < 6; ++c) {
      std::vector<uint64_t> col(nf);
      for (uint64_t i = 0; i < nf; ++i) col[i] = g[i].c[c];
      host_dft(col, wi);
      for (uint64_t k = p.d_final; k < nf; ++k)
        if (gl::mul(col[k], ninv) != 0) return false;
    }
  }
  return true;
}

// fri.rs:2136-2258 + 2517-2707 deep_fri_verify, classic branch: fold queries
// through every layer tree, the DEEP identity q (x - z) = f - f(z) at each
// opened point, s against the next layer, and the final coefficient tuple.
bool classic_verify(const StirProof& pr, const sg_fri_params& p, const std::vector<uint64_t>& sizes) {
  const uint64_t L = p.schedule_len;
  const bool use_cc = p.coeff_commit_final && L > 0;
  if (pr.stir || pr.roots.size() < L || pr.fz.size() < L) return false;
  HostTranscript tr("FRI/FS");
  bind_statement(tr, p, pr.n0);
  tr.absorb_bytes(pr.root_f0.data(), kc::kHashBytes);
  const Fp6 z = tr.challenge_ext("z_fp3");
  Fp6 beta = gl::e_zero();
  std::vector<Fp6> alphas;
  for (uint64_t ell = 0; ell < L; ++ell) {
    const bool last_cc = use_cc && ell == L - 1;
    if (!last_cc) alphas.push_back(tr.challenge_ext("alpha"));
    tr.absorb_ext(pr.fz[ell]);
    tr.absorb_bytes(pr.roots[ell].data(), kc::kHashBytes);
    if (last_cc) {
      if (!pr.has_croot) return false;
      tr.absorb_bytes(pr.coeff_root.data(), kc::kHashBytes);
      alphas.push_back(tr.challenge_ext("alpha"));
      beta = tr.challenge_ext("beta_deg");
    }
  }
  for (auto& c : pr.final_coeffs) tr.absorb_ext(c);
  const uint64_t query_seed = tr.challenge_field("query_seed");
  if (pr.final_coeffs.size() != p.d_final) return false;
  if (use_cc && !coeff_commit_ok(pr, p, sizes, beta)) return false;
  const uint64_t omega_final = sizes[L] >= 2 ? gl::root_of_unity(log2u(sizes[L])) : 1;
  if (pr.queries.size() < p.r || pr.layer_open.size() < L) return false;
  const auto f0_ar = layer_arities(pr.n0, 16);
  for (uint64_t qi = 0; qi < p.r; ++qi) {
    const ClassicQuery& q = pr.queries[qi];
    if (q.refs.size() < L || q.pay.size() < L) return false;
    const uint64_t i0 = query_index(query_seed, qi, pr.n0);
    uint64_t ei = i0;
    for (uint64_t ell = 0; ell < L; ++ell) {
      if (q.refs[ell][0] != ei) return false;
      ei %= sizes[ell] / p.schedule[ell];
    }
    if (q.final_index != ei) return false;
    if (!verify_opening(f0_ar, 0xFF, pr.root_f0, q.f0_open) || q.f0_open.index != i0) return false;
    for (int k = 1; k < 6; ++k)
      if (q.pay[0][0].c[k] != 0) return false;  // layer 0 is in the base field
    if (leaf_hash(f0_ar[0], 0xFF, q.f0_open.index, q.pay[0][0].c, 1) != q.f0_open.leaf) return false;
    const Fp6 x_final = gl::e_from(gl::pow(omega_final, q.final_index));
    for (uint64_t ell = 0; ell < L; ++ell) {
      if (pr.layer_open[ell].size() <= qi) return false;
      const Opening& o = pr.layer_open[ell][qi];
      const auto& pl = q.pay[ell];
      const uint64_t i = q.refs[ell][0];
      const auto ar = layer_arities(sizes[ell], p.schedule[ell]);
      if (!verify_opening(ar, ell, pr.roots[ell], o) || o.index != i) return false;
      uint64_t vals[18];
      for (int t = 0; t < 3; ++t)
        for (int k = 0; k < 6; ++k) vals[t * 6 + k] = pl[t].c[k];
      if (leaf_hash(ar[0], ell, o.index, vals, 18) != o.leaf) return false;
      const uint64_t xi = gl::pow(gl::root_of_unity(log2u(sizes[ell])), i);
      if (!gl::e_eq(gl::e_mul(pl[2], gl::e_sub(gl::e_from(xi), z)), gl::e_sub(pl[0], pr.fz[ell]))) return false;
      if (ell == L - 1 && use_cc) {
        const uint64_t m = p.schedule[ell];
        if (q.final_index >= pr.coeff_tuples.size()) return false;
        const auto& t = pr.coeff_tuples[q.final_index];
        Fp6 h = gl::e_zero(), fv = gl::e_zero(), ap = gl::e_one();
        uint64_t xp = 1;
        for (uint64_t k = 0; k < m; ++k) {
          h = gl::e_add(h, gl::e_scale(t[k], xp));
          xp = gl::mul(xp, xi);
          fv = gl::e_add(fv, gl::e_mul(t[k], ap));
          ap = gl::e_mul(ap, alphas[L - 1]);
        }
        if (!gl::e_eq(pl[0], h) || !gl::e_eq(fv, eval_poly(pr.final_coeffs, x_final))) return false;
      } else {
        const Fp6 f_next = ell + 1 < L ? q.pay[ell + 1][0] : eval_poly(pr.final_coeffs, x_final);
        if (!gl::e_eq(pl[1], f_next)) return false;
      }
    }
  }
  return true;
}

}  // namespace

bool stir_verify(const StirProof& pr, const sg_fri_params& p) {
  const uint64_t L = p.schedule_len;
  if (L == 0 || L > SG_MAX_SCHEDULE) return false;
  if (pr.n0 == 0 || (pr.n0 & (pr.n0 - 1)) || pr.n0 > (1ull << 32)) return false;
  std::vector<uint64_t> sizes{pr.n0};
  for (uint64_t i = 0; i < L; ++i) {
    if (p.schedule[i] < 2 || sizes.back() % p.schedule[i]) return false;
    sizes.push_back(sizes.back() / p.schedule[i]);
  }
  if (!p.stir) return classic_verify(pr, p, sizes);
  const bool use_cc = p.coeff_commit_final && L > 0;
  if (!pr.stir || pr.roots.size() < L || pr.coset_evals.size() < L) return false;
  HostTranscript tr("FRI/FS");
  bind_statement(tr, p, pr.n0);
  tr.absorb_bytes(pr.root_f0.data(), kc::kHashBytes);
  const Fp6 z = tr.challenge_ext("z_fp3");
  Fp6 zc = z, beta = gl::e_zero();
  std::vector<std::vector<Fp6>> interps;
  std::vector<Fp6> alphas;
  for (uint64_t ell = 0; ell < L; ++ell) {
    const uint64_t m = p.schedule[ell];
    const bool last_cc = use_cc && ell == L - 1;
    if (!last_cc) alphas.push_back(tr.challenge_ext("alpha"));
    const auto& ev = pr.coset_evals[ell];
    if (ev.size() != m) return false;
    const uint64_t zeta = gl::pow(gl::root_of_unity(log2u(sizes[ell])), sizes[ell] / m);
    std::vector<Fp6> ip;
    if (!interp_stir(ev, zc, zeta, &ip)) return false;
    interps.push_back(std::move(ip));
    zc = gl::e_pow(zc, m);
    for (auto& e : ev) tr.absorb_ext(e);
    tr.absorb_bytes(pr.roots[ell].data(), kc::kHashBytes);
    if (last_cc) {
      if (!pr.has_croot) return false;
      tr.absorb_bytes(pr.coeff_root.data(), kc::kHashBytes);
      alphas.push_back(tr.challenge_ext("alpha"));
      beta = tr.challenge_ext("beta_deg");
    }
  }
  for (auto& c : pr.final_coeffs) tr.absorb_ext(c);
  const uint64_t query_seed = tr.challenge_field("query_seed");
  if (pr.final_coeffs.size() != p.d_final) return false;

  // per-layer OOD fold consistency
  for (uint64_t ell = 0; ell < L; ++ell) {
    const uint64_t m = p.schedule[ell];
    Fp6 acc = gl::e_zero(), ap = gl::e_one();
    for (uint64_t k = 0; k < m; ++k) {
      acc = gl::e_add(acc, gl::e_mul(interps[ell][k], ap));
      ap = gl::e_mul(ap, alphas[ell]);
    }
    Fp6 expect;
    if (ell + 1 < L) {
      expect = pr.coset_evals[ell + 1][0];
    } else {
      Fp6 zf = z;
      for (uint64_t i = 0; i < L; ++i) zf = gl::e_pow(zf, p.schedule[i]);
      expect = eval_poly(pr.final_coeffs, zf);
    }
    if (!gl::e_eq(acc, expect)) return false;
  }

  if (use_cc && !coeff_commit_ok(pr, p, sizes, beta)) return false;

  // s0 proximity queries against the packed f0 tree and the layer-1 tree
  if (pr.prox.size() != p.s0) return false;
  const uint64_t n0 = pr.n0, m0 = p.schedule[0], nn = sizes[0] / m0;
  const uint64_t omega0 = gl::root_of_unity(log2u(sizes[0]));
  const uint64_t zeta0 = gl::pow(omega0, nn);
  const uint64_t omega_final = sizes[L] >= 2 ? gl::root_of_unity(log2u(sizes[L])) : 1;
  const auto f0_ar = layer_arities(nn, 16);
  const auto l1_ar = L >= 2 ? layer_arities(sizes[1], p.schedule[1]) : std::vector<uint32_t>{};
  std::vector<Fp6> ap0(m0);
  {
    Fp6 a = gl::e_one();
    for (uint64_t k = 0; k < m0; ++k) {
      ap0[k] = a;
      a = gl::e_mul(a, alphas[0]);
    }
  }
  // Each query reads only the proof: they are checked on up to 8 threads, a strided
  // share each (about 20 us a query, mostly its two Merkle openings).
  auto query_ok = [&](uint64_t qi) -> bool {
    const ProxQuery& q = pr.prox[qi];
    const uint64_t raw = query_index(query_seed, qi, n0);
    if (q.raw != raw || q.base != raw % nn) return false;
    if (q.fib_idx.size() != m0 || q.fib_vals.size() != m0) return false;
    for (uint64_t j = 0; j < m0; ++j)
      if (q.fib_idx[j] != q.base + j * nn) return false;
    if (!verify_opening(f0_ar, 0xFF, pr.root_f0, q.f0_open) || q.f0_open.index != q.base) return false;
    if (leaf_hash(f0_ar[0], 0xFF, q.f0_open.index, q.fib_vals.data(), m0) != q.f0_open.leaf) return false;
    std::vector<Fp6> fib(m0);
    for (uint64_t j = 0; j < m0; ++j) fib[j] = gl::e_from(q.fib_vals[j]);
    const auto ct = interp_base(fib, gl::pow(omega0, q.base), zeta0);
    Fp6 fv = gl::e_zero();
    for (uint64_t k = 0; k < m0; ++k) fv = gl::e_add(fv, gl::e_mul(ct[k], ap0[k]));
    if (L >= 2) {
      if (!q.has_l1) return false;
      if (!verify_opening(l1_ar, 1, pr.roots[1], q.l1_open) || q.l1_open.index != q.base) return false;
      if (leaf_hash(l1_ar[0], 1, q.l1_open.index, q.f_next.c, 6) != q.l1_open.leaf) return false;
      return gl::e_eq(fv, q.f_next);
    }
    return gl::e_eq(fv, eval_poly(pr.final_coeffs, gl::e_from(gl::pow(omega_final, q.base))));
  };
  const uint64_t nq = pr.prox.size();
  const unsigned nt = (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>({8, std::max(1u, std::thread::hardware_concurrency()), nq / 8}));
  std::atomic<bool> ok{true};
  auto share = [&](unsigned t) {
    for (uint64_t qi = t; qi < nq && ok.load(std::memory_order_relaxed); qi += nt)
      if (!query_ok(qi)) ok = false;
  };
  std::vector<std::thread> th;
  for (unsigned t = 1; t < nt; ++t) th.emplace_back(share, t);
  share(0);
  for (auto& x : th) x.join();
  return ok.load();
}

}  // namespace sg
