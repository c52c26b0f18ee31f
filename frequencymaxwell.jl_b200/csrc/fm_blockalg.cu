// libfmcuda: host algebra of s-step (block) GMRES for one right-hand side (see fm_blockalg.h).
//
// Block step at column m (K = m + 1 stored vectors, X = V Rf with Rf block upper triangular):
//   Y_0 = V_m,  Y_t = (M^{-1}A - theta_t) Y_{t-1}           (device)
//   D = X^H Y_{1..S}                                         (device, FP64 tensor cores)
//   C = Rf^{-H} D (V coordinates),  E = Rf^{-1} C            (here)
//   Y' = Y - X E,  G = Y'^H Y' = Rb^H Rb                     (device; Cholesky here)
//   raw storage:           X_{m+1..m+S} = Y', Rf block = Rb
//   orthonormalised storage: X_{m+1..m+S} = Y' Rb^{-1}, Rf block = I
//   next shifts: Ritz values of this block's S x S diagonal Hessenberg block
// and the Hessenberg columns m..m+S-1 follow from the relations
//   (M^{-1}A) V W_{0:S-1} = V (W_{1:S} + W_{0:S-1} diag(theta)),
// where W holds the V coordinates of Y_0..Y_S (block CA-GMRES change of basis).  Givens rotations and the
// stopping test then run column by column, as in GMRES, so the iteration at which a right-hand side stops and
// the iterate it returns are those of full GMRES (in exact arithmetic).
#include "fm_blockalg.h"

#include <cmath>

// Givens rotation of Krylov.jl's gmres (fm_gmres.cu)
void sym_givens(std::complex<double> a, double b, double& c, std::complex<double>& s, std::complex<double>& rho);

namespace fm {

using cd = cdb;

bool hess_eigs(int n, std::vector<cd> A, std::vector<cd>& ev) {
  ev.clear();
  auto a = [&](int i, int j) -> cd& { return A[i + (size_t)j * n]; };
  int hi = n - 1, iter = 0;
  while (hi >= 0) {
    if (hi == 0) {
      ev.push_back(a(0, 0));
      break;
    }
    int l = hi;
    while (l > 0 && std::abs(a(l, l - 1)) > 1e-15 * (std::abs(a(l, l)) + std::abs(a(l - 1, l - 1)))) --l;
    if (l == hi) {
      ev.push_back(a(hi, hi));
      --hi;
      iter = 0;
      continue;
    }
    if (++iter > 100 * n) return false;
    // Wilkinson shift from the trailing 2x2 block of the window [l, hi]
    const cd p = a(hi - 1, hi - 1), q = a(hi - 1, hi), r = a(hi, hi - 1), t = a(hi, hi);
    const cd tr = p + t, det = p * t - q * r, disc = std::sqrt(tr * tr / 4.0 - det);
    const cd m1 = tr / 2.0 + disc, m2 = tr / 2.0 - disc;
    cd mu = std::abs(m1 - t) < std::abs(m2 - t) ? m1 : m2;
    if (iter % 11 == 10) mu += std::abs(a(hi, hi - 1));  // exceptional shift
    std::vector<double> cs(hi - l);
    std::vector<cd> sn(hi - l);
    for (int k = l; k <= hi; ++k) a(k, k) -= mu;
    for (int k = l; k < hi; ++k) {  // A - mu I = Q R, Givens G_k zeroes a(k+1, k)
      const cd x = a(k, k), y = a(k + 1, k);
      const double nr = std::sqrt(std::norm(x) + std::norm(y));
      double c = 1.0;
      cd sg = 0.0;
      if (nr > 0) {
        c = std::abs(x) / nr;
        sg = (std::abs(x) > 0 ? x / std::abs(x) : cd(1.0, 0.0)) * std::conj(y) / nr;
      }
      for (int j = k; j <= hi; ++j) {
        const cd t1 = a(k, j), t2 = a(k + 1, j);
        a(k, j) = c * t1 + sg * t2;
        a(k + 1, j) = -std::conj(sg) * t1 + c * t2;
      }
      cs[k - l] = c;
      sn[k - l] = sg;
    }
    for (int k = l; k < hi; ++k) {  // R Q = R G_l^H ... G_{hi-1}^H
      const double c = cs[k - l];
      const cd sg = sn[k - l];
      for (int i = l; i <= k + 1; ++i) {
        const cd t1 = a(i, k), t2 = a(i, k + 1);
        a(i, k) = c * t1 + std::conj(sg) * t2;
        a(i, k + 1) = -sg * t1 + c * t2;
      }
    }
    for (int k = l; k <= hi; ++k) a(k, k) += mu;
  }
  return true;
}

void leja_order(std::vector<cd>& z) {
  std::vector<cd> out;
  std::vector<bool> used(z.size(), false);
  for (size_t n = 0; n < z.size(); ++n) {
    int best = -1;
    double bv = -1.0;
    for (size_t i = 0; i < z.size(); ++i) {
      if (used[i]) continue;
      double v = 1.0;
      if (out.empty()) v = std::abs(z[i]);
      else
        for (const cd& o : out) v *= std::abs(z[i] - o);
      if (v > bv) {
        bv = v;
        best = (int)i;
      }
    }
    used[best] = true;
    out.push_back(z[best]);
  }
  z = out;
}

bool chol_upper(int n, const std::vector<cd>& G, std::vector<cd>& R) {
  R.assign((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) {
    cd d = G[j + (size_t)j * n];
    for (int k = 0; k < j; ++k) d -= std::conj(R[k + (size_t)j * n]) * R[k + (size_t)j * n];
    if (!(d.real() > 0.0) || !std::isfinite(d.real())) return false;
    const double rd = std::sqrt(d.real());
    R[j + (size_t)j * n] = rd;
    for (int i = j + 1; i < n; ++i) {
      cd v = G[j + (size_t)i * n];
      for (int k = 0; k < j; ++k) v -= std::conj(R[k + (size_t)j * n]) * R[k + (size_t)i * n];
      R[j + (size_t)i * n] = v / rd;
    }
  }
  return true;
}

void rf_solve(const BlkState& st, int K, const cd* c, cd* d) {
  for (int k = K - 1; k >= 0;) {
    const int a0 = st.b0[k];
    for (int i = k; i >= a0; --i) {
      cd v = c[i];
      for (int j = i + 1; j <= k; ++j) v -= st.Rf[i + (size_t)j * st.ld] * d[j];
      d[i] = v / st.Rf[i + (size_t)i * st.ld];
    }
    k = a0 - 1;
  }
}

void rf_solve_h(const BlkState& st, int K, const cd* c, cd* d) {
  for (int k0 = 0; k0 < K;) {
    int k1 = k0;
    while (k1 + 1 < K && st.b0[k1 + 1] == k0) ++k1;
    for (int i = k0; i <= k1; ++i) {
      cd v = c[i];
      for (int j = k0; j < i; ++j) v -= std::conj(st.Rf[j + (size_t)i * st.ld]) * d[j];
      d[i] = v / std::conj(st.Rf[i + (size_t)i * st.ld]);
    }
    k0 = k1 + 1;
  }
}

static const double kBtol = std::pow(2.220446049250313e-16, 0.75);

bool blk_init(BlkState& r, int ld, double beta, double abstol, double reltol) {
  r = BlkState();
  r.ld = ld;
  r.H.assign((size_t)ld * ld, 0.0);
  r.Rf.assign((size_t)ld * ld, 0.0);
  r.b0.assign(ld, 0);
  r.beta = beta;
  r.rnorm = beta;
  r.eps = abstol + reltol * beta;
  r.Rf[0] = beta;
  r.b0[0] = 0;
  r.nvec = 1;
  r.z.assign(1, cd(beta, 0.0));
  if (beta == 0.0 || r.rnorm <= r.eps) {
    r.active = false;
    r.solved = true;
    return true;
  }
  return false;
}

void blk_restart(BlkState& r, int ld, double beta, double eps) {
  blk_init(r, ld, beta, 0.0, 0.0);
  r.active = true;
  r.solved = false;
  r.eps = eps;
}

bool blk_givens_col(BlkState& r, int j, int itmax) {
  const int ld = r.ld;
  const int K = j + 1;
  std::vector<cd> col(K);
  for (int i = 0; i < K; ++i) col[i] = r.H[i + (size_t)j * ld];
  const double hb = r.H[(j + 1) + (size_t)j * ld].real();
  for (int i = 0; i < K - 1; ++i) {
    cd t = r.c[i] * col[i] + r.s[i] * col[i + 1];
    col[i + 1] = std::conj(r.s[i]) * col[i] - r.c[i] * col[i + 1];
    col[i] = t;
  }
  double c;
  cd sn, rho;
  sym_givens(col[K - 1], hb, c, sn, rho);
  col[K - 1] = rho;
  r.c.push_back(c);
  r.s.push_back(sn);
  r.Rg.push_back(col);
  const cd zk1 = std::conj(sn) * r.z[K - 1];
  r.z[K - 1] = c * r.z[K - 1];
  r.rnorm = std::abs(zk1);
  r.iters = K;
  r.solved = (r.rnorm <= r.eps) || (r.rnorm + 1.0 <= 1.0);
  if (r.solved || hb <= kBtol || K >= itmax) return true;
  r.z.push_back(zk1);
  return false;
}

void blk_cgs_coefs(BlkState& r, int m, const double2* hr, double2* cf) {
  const int ld = r.ld, K = m + 1;
  for (int k = 0; k < K; ++k) {
    const double rk = r.Rf[k + (size_t)k * ld].real();
    const cd h = cd(hr[k].x, hr[k].y) / rk;
    r.H[k + (size_t)m * ld] = h;
    const cd e = h / rk;
    cf[k] = make_double2(e.real(), e.imag());
  }
}

bool blk_cgs_close(BlkState& r, int m, double hb, int itmax) {
  const int ld = r.ld;
  r.H[(m + 1) + (size_t)m * ld] = hb;
  r.Rf[(m + 1) + (size_t)(m + 1) * ld] = hb;
  r.b0[m + 1] = m + 1;
  r.nvec = m + 2;
  return blk_givens_col(r, m, itmax);
}

void blk_shifts(BlkState& r, int j0, int S) {
  if ((int)r.theta.size() != S) r.theta.assign(S, 0.0);
  std::vector<cd> Hs((size_t)S * S), ev;
  for (int j = 0; j < S; ++j)
    for (int i = 0; i < S; ++i) Hs[i + (size_t)j * S] = r.H[(j0 + i) + (size_t)(j0 + j) * r.ld];
  if (hess_eigs(S, Hs, ev) && (int)ev.size() == S) {
    leja_order(ev);
    r.theta = ev;
  }
}

int blk_start(const BlkState& r, int m, double2* cc) {
  const int K = m + 1, k0 = r.b0[m];
  std::vector<cd> em(K, 0.0), d(K, 0.0);
  em[m] = 1.0;
  rf_solve(r, K, em.data(), d.data());
  for (int a = 0; a < m - k0 + 1; ++a) cc[a] = make_double2(d[k0 + a].real(), d[k0 + a].imag());
  return k0;
}

void blk_project(const BlkState& r, int m, int S, const double2* D, std::vector<cd>& Cv, double2* cf) {
  const int K = m + 1;
  Cv.assign((size_t)K * S, 0.0);
  std::vector<cd> dcol(K), ccol(K), ecol(K);
  for (int t = 0; t < S; ++t) {
    for (int k = 0; k < K; ++k) {
      const double2 v = D[(size_t)k * S + t];
      dcol[k] = cd(v.x, v.y);
    }
    rf_solve_h(r, K, dcol.data(), ccol.data());
    rf_solve(r, K, ccol.data(), ecol.data());
    for (int k = 0; k < K; ++k) {
      Cv[k + (size_t)t * K] = ccol[k];
      cf[(size_t)k * S + t] = make_double2(ecol[k].real(), ecol[k].imag());
    }
  }
}

bool blk_absorb(BlkState& r, int m, int S, bool ortho_store, const double2* Gt, const std::vector<cd>& Cv,
                double2* rbi, int itmax) {
  const int ld = r.ld, K = m + 1;
  std::vector<cd> G((size_t)S * S), Rb;
  int gi = 0;
  for (int t = 0; t < S; ++t)
    for (int u = t; u < S; ++u, ++gi) {
      const size_t at = S <= 8 ? (size_t)gi : (size_t)t * S + u;
      const cd v(Gt[at].x, Gt[at].y);
      G[t + (size_t)u * S] = v;
      G[u + (size_t)t * S] = std::conj(v);
    }
  if (!chol_upper(S, G, Rb)) {  // the block lost rank: Krylov breakdown, keep the columns so far
    r.active = false;
    return true;
  }
  if (ortho_store) {
    // stored columns V = Y' Rb^{-1} are orthonormal: identity diagonal blocks of Rf
    for (int t = 0; t < S; ++t) {
      std::vector<cd> col(S, 0.0);
      col[t] = 1.0;
      for (int i = t; i >= 0; --i) {
        cd v = col[i];
        for (int q = i + 1; q <= t; ++q) v -= Rb[i + (size_t)q * S] * col[q];
        col[i] = v / Rb[i + (size_t)i * S];
      }
      for (int u = 0; u <= t; ++u) rbi[(size_t)u * S + t] = make_double2(col[u].real(), col[u].imag());
    }
    for (int u = 0; u < S; ++u) {
      for (int a = 0; a <= u; ++a) r.Rf[(K + a) + (size_t)(K + u) * ld] = (a == u) ? cd(1.0, 0.0) : cd(0.0, 0.0);
      r.b0[K + u] = K + u;
    }
  } else {
    for (int u = 0; u < S; ++u) {
      for (int a = 0; a <= u; ++a) r.Rf[(K + a) + (size_t)(K + u) * ld] = Rb[a + (size_t)u * S];
      r.b0[K + u] = K;
    }
  }
  r.nvec = K + S;
  // W: V coordinates of Y_0..Y_S, n x (S+1)
  const int n = K + S;
  std::vector<cd> W((size_t)n * (S + 1), 0.0);
  W[m] = 1.0;  // Y_0 = V_m
  for (int t = 0; t < S; ++t) {
    for (int i = 0; i < K; ++i) W[i + (size_t)(t + 1) * n] = Cv[i + (size_t)t * K];
    for (int a = 0; a < S; ++a) W[K + a + (size_t)(t + 1) * n] = Rb[a + (size_t)t * S];
  }
  // Rh = W[:,1:S] + W[:,0:S-1] diag(theta) - [H_{0:m,0:m-1} W_{0:m-1,0:S-1}; 0]
  std::vector<cd> Rh((size_t)n * S), Hn((size_t)n * S);
  for (int c = 0; c < S; ++c) {
    for (int i = 0; i < n; ++i) Rh[i + (size_t)c * n] = W[i + (size_t)(c + 1) * n] + r.theta[c] * W[i + (size_t)c * n];
    for (int j = 0; j < m; ++j) {
      const cd w = W[j + (size_t)c * n];
      if (w == cd(0.0, 0.0)) continue;
      for (int i = 0; i <= j + 1; ++i) Rh[i + (size_t)c * n] -= r.H[i + (size_t)j * ld] * w;
    }
  }
  // Hn = Rh T^{-1}, T = W[m..m+S-1, 0..S-1] upper triangular
  for (int c = 0; c < S; ++c)
    for (int i = 0; i < n; ++i) {
      cd v = Rh[i + (size_t)c * n];
      for (int a = 0; a < c; ++a) v -= Hn[i + (size_t)a * n] * W[m + a + (size_t)c * n];
      Hn[i + (size_t)c * n] = v / W[m + c + (size_t)c * n];
    }
  for (int c = 0; c < S; ++c)
    for (int i = 0; i < n; ++i) r.H[i + (size_t)(m + c) * ld] = (i <= m + c + 1) ? Hn[i + (size_t)c * n] : cd(0.0, 0.0);
  // Newton shifts of the next block: Ritz values of this block's S x S diagonal Hessenberg block, Leja ordered.
  // Shifts kept from the first S steps only let the basis of a later block lose conditioning; refreshed ones
  // keep it near that of s = 4 up to s = 16 (a numpy restatement with FP32-rounded basis vectors on the CBS
  // operator: 4.6e-6 -> 6e-8 at s = 8).
  blk_shifts(r, m, S);
  for (int c = 0; c < S; ++c)
    if (blk_givens_col(r, m + c, itmax)) {
      r.active = false;
      return true;
    }
  return false;
}

int blk_solution(const BlkState& r, double2* dout) {
  const int n_in = r.iters;
  if (n_in == 0) return 0;
  std::vector<cd> y(r.z.begin(), r.z.begin() + n_in);
  for (int i = n_in - 1; i >= 0; --i) {
    for (int jj = n_in - 1; jj > i; --jj) y[i] -= r.Rg[jj][i] * y[jj];
    if (std::abs(r.Rg[i][i]) <= kBtol) {
      for (int q = 0; q <= i; ++q) y[q] = 0.0;
      break;
    }
    y[i] /= r.Rg[i][i];
  }
  std::vector<cd> yv(r.nvec, 0.0), d(r.nvec, 0.0);
  for (int i = 0; i < n_in; ++i) yv[i] = y[i];
  rf_solve(r, r.nvec, yv.data(), d.data());
  for (int i = 0; i < r.nvec; ++i) dout[i] = make_double2(d[i].real(), d[i].imag());
  return r.nvec;
}

}  // namespace fm
