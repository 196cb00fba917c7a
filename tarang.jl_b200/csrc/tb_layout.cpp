// Host-side plan compiler: per-class banded layout of the RBC tau system and
// the Chebyshev transform matrices.  Runs once per plan.
//
// Operator content follows the reference's per-mode assembly
// (src/core/operators/matrices/matrices_subproblem_operators.jl:19-330 and
// matrices_subproblem_helpers.jl:101-166) for the equations of
// test/test_subproblem_rk.jl:50-57:
//   trace(grad_u) + tau_p = 0
//   dt(b) - kappa div(grad_b) + lift(tau_b2) = -u.grad(b),  grad_b = grad(b) + ez lift(tau_b1)
//   dt(u) - nu div(grad_u) + grad(p) - b ez + lift(tau_u2) = -u.grad(u), grad_u = grad(u) + ez lift(tau_u1)
//   b(z=0) = b_bottom, u(z=0) = 0, b(z=Lz) = b_top, u(z=Lz) = 0, integ(p) = 0
// with lift(., -1) = unit column e_{N-1} in the T basis (:218-260), and the
// valid-mode filtering that removes integ(p) and tau_p at kx != 0
// (subproblem_matrix_build.jl:102-168).  Here integ(p) is replaced at kx != 0
// by the pin tau_p = 0, which leaves every other unknown unchanged.
#include <algorithm>
#include <cmath>
#include <tuple>

#include "tb_internal.h"

namespace tb {

namespace {

// T -> C^(2) conversion S = S1 S0, only the three nonzero diagonals.
inline double S_at(int N, int k, int j) {
  if (k < 0 || j < 0 || k >= N || j >= N) return 0.0;
  if (j == k) return (k == 0 ? 1.0 : 0.5) / (k + 1.0);
  if (j == k + 2) return -0.5 * (1.0 / (k + 1.0) + 1.0 / (k + 3.0));
  if (j == k + 4) return 0.5 / (k + 3.0);
  return 0.0;
}
// S1 D1 (first derivative T -> C^(2)), scaled by s = 2/Lz.
inline double SD_at(int N, int k, int j, double s) {
  if (k < 0 || j < 0 || k >= N || j >= N) return 0.0;
  if (j == k + 1) return s;
  if (j == k + 3) return -s;
  return 0.0;
}
// D2 (second derivative T -> C^(2)), scaled by s^2.
inline double D2_at(int N, int k, int j, double s) {
  if (k < 0 || j < 0 || k >= N || j >= N) return 0.0;
  if (j == k + 2) return 2.0 * (k + 2.0) * s * s;
  return 0.0;
}

struct Key {
  double a;
  int b;
  bool operator<(const Key& o) const { return a < o.a || (a == o.a && b < o.b); }
};

}  // namespace

TauLayout build_rbc_layout(int N, double Lx, double Lz, double kappa, double nu, double Nx_scale,
                           double b_bottom, double b_top) {
  TauLayout out;
  out.Nz = N;
  const double s = 2.0 / Lz;
  // field pivot order inside a Chebyshev block: p, b, uz, vx (minimises 2 kl + ku)
  auto forder = [](int unk) {
    switch (unk) {
      case UK_P: return 0;
      case UK_B: return 1;
      case UK_UZ: return 2;
      default: return 3;  // UK_UX
    }
  };
  auto eq_field = [](int e) {
    switch (e) {
      case EQ_B: return (int)UK_B;
      case EQ_MZ: return (int)UK_UZ;
      case EQ_MX: return (int)UK_UX;
      default: return (int)UK_P;
    }
  };
  const int tau_class[7] = {1, N % 2, (N - 1) % 2, (N - 1) % 2, N % 2, N % 2, (N - 1) % 2};
  //                       tau_p tau_b1 tau_b2   tau_u1x     tau_u1z tau_u2x tau_u2z

  for (int sg = 0; sg < 2; ++sg) {
    ClassLayout& L = out.cls[sg];
    auto upar = [&](int unk) { return (unk == UK_B || unk == UK_UZ) ? sg : 1 - sg; };
    auto epar = [&](int e) { return (e == EQ_B || e == EQ_MZ) ? sg : 1 - sg; };

    // ---- unknowns ----
    std::vector<std::pair<int, int>> left;
    if (sg == 0)
      left = {{UK_B, 0}, {UK_UZ, 0}, {UK_UX, 1}};
    else
      left = {{UK_P, 0}, {UK_B, 1}, {UK_UZ, 1}, {UK_UX, 0}};
    std::vector<std::tuple<Key, int, int>> cols;
    for (int unk : {UK_P, UK_B, UK_UZ, UK_UX})
      for (int j = 0; j < N; ++j) {
        if (j % 2 != upar(unk)) continue;
        if (std::find(left.begin(), left.end(), std::make_pair(unk, j)) != left.end()) continue;
        cols.push_back({Key{(double)j, forder(unk)}, unk, j});
      }
    for (int t = 0; t < 7; ++t) {
      if (tau_class[t] != sg) continue;
      if (t == 0)
        cols.push_back({Key{2.0, -1}, UK_TAU0 + t, 0});
      else
        cols.push_back({Key{N + 0.5, t}, UK_TAU0 + t, 0});
    }
    std::sort(cols.begin(), cols.end(),
              [](const auto& a, const auto& b) { return std::get<0>(a) < std::get<0>(b); });
    // ---- rows ----
    std::vector<std::tuple<Key, int, int>> rows;
    for (int e : {EQ_CONT, EQ_B, EQ_MX, EQ_MZ})
      for (int k = 0; k < N; ++k) {
        if (k % 2 != epar(e)) continue;
        rows.push_back({Key{k + 2.0, forder(eq_field(e))}, e, k});
      }
    std::sort(rows.begin(), rows.end(),
              [](const auto& a, const auto& b) { return std::get<0>(a) < std::get<0>(b); });
    TB_REQUIRE(rows.size() == cols.size(), TB_EINVAL, "tau layout: bulk rows != band columns");
    const int n = (int)rows.size();
    const int nb = (int)left.size();
    L.n = n;
    L.nb = nb;
    for (auto& r : rows) {
      L.row_eq.push_back(std::get<1>(r));
      L.row_k.push_back(std::get<2>(r));
    }
    for (auto& c : cols) {
      L.col_unk.push_back(std::get<1>(c));
      L.col_k.push_back(std::get<2>(c));
    }
    for (auto& l : left) {
      L.left_unk.push_back(l.first);
      L.left_k.push_back(l.second);
    }

    // position lookup: unknown -> band column or border index
    auto col_of = [&](int unk, int j) -> int {
      for (int c = 0; c < n; ++c)
        if (L.col_unk[c] == unk && L.col_k[c] == j) return c;
      return -1;
    };
    auto left_of = [&](int unk, int j) -> int {
      for (int b = 0; b < nb; ++b)
        if (L.left_unk[b] == unk && L.left_k[b] == j) return b;
      return -1;
    };

    // dense entry tables for this class
    std::vector<Coef> dense((size_t)n * n, Coef{0, 0, 0, 0});
    std::vector<Coef> bordd((size_t)n * nb, Coef{0, 0, 0, 0});
    auto add = [&](int r, int unk, int j, Coef c) {
      if (c.m == 0 && c.l0 == 0 && c.l1 == 0 && c.l2 == 0) return;
      int col = col_of(unk, j);
      if (col >= 0) {
        Coef& d = dense[(size_t)r * n + col];
        d.m += c.m; d.l0 += c.l0; d.l1 += c.l1; d.l2 += c.l2;
        return;
      }
      int b = left_of(unk, j);
      TB_REQUIRE(b >= 0, TB_EINVAL, "tau layout: entry outside its parity class");
      Coef& d = bordd[(size_t)r * nb + b];
      d.m += c.m; d.l0 += c.l0; d.l1 += c.l1; d.l2 += c.l2;
    };
    const int TP = UK_TAU0 + 0, TB1 = UK_TAU0 + 1, TB2 = UK_TAU0 + 2, TU1X = UK_TAU0 + 3,
              TU1Z = UK_TAU0 + 4, TU2X = UK_TAU0 + 5, TU2Z = UK_TAU0 + 6;
    for (int r = 0; r < n; ++r) {
      const int e = L.row_eq[r], k = L.row_k[r];
      for (int j = k; j < std::min(N, k + 5); ++j) {
        const double Sv = S_at(N, k, j), SDv = SD_at(N, k, j, s), D2v = D2_at(N, k, j, s);
        switch (e) {
          case EQ_CONT:
            add(r, UK_UX, j, Coef{0, 0, -Sv, 0});
            add(r, UK_UZ, j, Coef{0, SDv, 0, 0});
            break;
          case EQ_B:
            add(r, UK_B, j, Coef{Sv, -kappa * D2v, 0, kappa * Sv});
            break;
          case EQ_MX:
            add(r, UK_UX, j, Coef{Sv, -nu * D2v, 0, nu * Sv});
            add(r, UK_P, j, Coef{0, 0, Sv, 0});
            break;
          case EQ_MZ:
            add(r, UK_UZ, j, Coef{Sv, -nu * D2v, 0, nu * Sv});
            add(r, UK_P, j, Coef{0, SDv, 0, 0});
            add(r, UK_B, j, Coef{0, -Sv, 0, 0});
            break;
        }
      }
      const double SeN = S_at(N, k, N - 1), SDeN = SD_at(N, k, N - 1, s);
      switch (e) {
        case EQ_CONT:
          if (SeN != 0) add(r, TU1Z, 0, Coef{0, SeN, 0, 0});
          if (k == 0) add(r, TP, 0, Coef{0, S_at(N, 0, 0), 0, 0});
          break;
        case EQ_B:
          if (SDeN != 0) add(r, TB1, 0, Coef{0, -kappa * SDeN, 0, 0});
          if (SeN != 0) add(r, TB2, 0, Coef{0, SeN, 0, 0});
          break;
        case EQ_MX:
          if (SDeN != 0) add(r, TU1X, 0, Coef{0, -nu * SDeN, 0, 0});
          if (SeN != 0) add(r, TU2X, 0, Coef{0, SeN, 0, 0});
          break;
        case EQ_MZ:
          if (SDeN != 0) add(r, TU1Z, 0, Coef{0, -nu * SDeN, 0, 0});
          if (SeN != 0) add(r, TU2Z, 0, Coef{0, SeN, 0, 0});
          break;
      }
    }
    // bandwidths
    int kl = 0, ku = 0;
    for (int r = 0; r < n; ++r)
      for (int c = 0; c < n; ++c) {
        const Coef& d = dense[(size_t)r * n + c];
        if (d.m == 0 && d.l0 == 0 && d.l1 == 0 && d.l2 == 0) continue;
        kl = std::max(kl, r - c);
        ku = std::max(ku, c - r);
      }
    L.kl = kl;
    L.ku = ku;
    const int w = kl + ku + 1;
    L.band.assign((size_t)n * w, Coef{0, 0, 0, 0});
    for (int r = 0; r < n; ++r)
      for (int c = std::max(0, r - kl); c <= std::min(n - 1, r + ku); ++c)
        L.band[(size_t)r * w + (c - r + kl)] = dense[(size_t)r * n + c];
    L.bord = bordd;

    // ---- boundary rows (even/odd recombination of the z=0 / z=Lz rows) ----
    L.c2_z.assign((size_t)nb * n, 0.0);
    L.c2_nz.assign((size_t)nb * n, 0.0);
    L.c1_z.assign((size_t)nb * nb, 0.0);
    L.c1_nz.assign((size_t)nb * nb, 0.0);
    L.bc_rhs.assign(nb, 0.0);
    // boundary row list
    std::vector<std::pair<int, int>> bcrows;  // (unknown, parity) ; (-1,-1) integ/pin
    if (sg == 0)
      bcrows = {{UK_B, 0}, {UK_UZ, 0}, {UK_UX, 1}};
    else
      bcrows = {{UK_B, 1}, {UK_UZ, 1}, {UK_UX, 0}, {-1, -1}};
    for (int q = 0; q < nb; ++q) {
      auto put = [&](int unk, int j, double vz, double vnz) {
        int c = col_of(unk, j);
        if (c >= 0) {
          L.c2_z[(size_t)q * n + c] += vz;
          L.c2_nz[(size_t)q * n + c] += vnz;
          return;
        }
        int b = left_of(unk, j);
        TB_REQUIRE(b >= 0, TB_EINVAL, "tau layout: boundary entry outside class");
        L.c1_z[(size_t)q * nb + b] += vz;
        L.c1_nz[(size_t)q * nb + b] += vnz;
      };
      const int unk = bcrows[q].first, par = bcrows[q].second;
      if (unk >= 0) {
        for (int j = par; j < N; j += 2) put(unk, j, 1.0, 1.0);
        if (unk == UK_B)
          L.bc_rhs[q] = (par == 0 ? 0.5 * (b_top + b_bottom) : 0.5 * (b_top - b_bottom)) * Nx_scale;
      } else {
        // integ(p) = Lx * int_0^Lz T_n dz at kx = 0; pin tau_p = 0 otherwise
        for (int j = 0; j < N; j += 2) put(UK_P, j, Lx * Lz / (1.0 - (double)j * j), 0.0);
        put(TP, 0, 0.0, 1.0);
      }
    }
  }
  return out;
}

TauLayout build_helmholtz_layout(int N, double Lz, double nu) {
  // One velocity component decoupled from the pressure (the 3D cross-wavevector
  // component):  dt(u) - nu div(grad_u) + lift(tau_2) = F,
  // grad_u = grad(u) + ez lift(tau_1),  u(z=0) = u(z=Lz) = 0.
  // Unknown codes: UK_B for u, UK_TAU0 + 1 / + 2 for tau_1 / tau_2.  Class sg
  // holds the coefficients and C^(2) rows of parity sg; its lowest coefficient
  // u_sg is the border unknown, so the bulk block is tridiagonal with the
  // dominant S_{k,k+2} / D2 entries on its diagonal.
  TB_REQUIRE(N % 2 == 0, TB_ENOTSUPPORTED, "the 3D plan needs an even Nz");
  TauLayout out;
  out.Nz = N;
  const double s = 2.0 / Lz;
  for (int sg = 0; sg < 2; ++sg) {
    ClassLayout& L = out.cls[sg];
    const int tau = (sg == N % 2) ? UK_TAU0 + 1 : UK_TAU0 + 2;
    for (int k = sg; k < N; k += 2) {
      L.row_eq.push_back(EQ_B);
      L.row_k.push_back(k);
    }
    for (int j = sg + 2; j < N; j += 2) {
      L.col_unk.push_back(UK_B);
      L.col_k.push_back(j);
    }
    L.col_unk.push_back(tau);
    L.col_k.push_back(0);
    L.left_unk.push_back(UK_B);
    L.left_k.push_back(sg);
    const int n = (int)L.row_eq.size();
    TB_REQUIRE((int)L.col_unk.size() == n, TB_EINVAL, "helmholtz layout: rows != columns");
    L.n = n;
    L.nb = 1;
    std::vector<Coef> dense((size_t)n * n, Coef{0, 0, 0, 0});
    L.bord.assign((size_t)n, Coef{0, 0, 0, 0});
    for (int r = 0; r < n; ++r) {
      const int k = L.row_k[r];
      for (int j = k; j < std::min(N, k + 5); ++j) {
        const double Sv = S_at(N, k, j), D2v = D2_at(N, k, j, s);
        const Coef c{Sv, -nu * D2v, 0, nu * Sv};
        if (c.m == 0 && c.l0 == 0 && c.l2 == 0) continue;
        if (j == sg) {
          L.bord[r] = c;
        } else {
          const int col = (j - sg) / 2 - 1;
          dense[(size_t)r * n + col] = c;
        }
      }
      const double lift = (tau == UK_TAU0 + 1) ? -nu * SD_at(N, k, N - 1, s) : S_at(N, k, N - 1);
      if (lift != 0) dense[(size_t)r * n + (n - 1)].l0 += lift;
    }
    int kl = 0, ku = 0;
    for (int r = 0; r < n; ++r)
      for (int c = 0; c < n; ++c) {
        const Coef& d = dense[(size_t)r * n + c];
        if (d.m == 0 && d.l0 == 0 && d.l1 == 0 && d.l2 == 0) continue;
        kl = std::max(kl, r - c);
        ku = std::max(ku, c - r);
      }
    L.kl = kl;
    L.ku = ku;
    const int w = kl + ku + 1;
    L.band.assign((size_t)n * w, Coef{0, 0, 0, 0});
    for (int r = 0; r < n; ++r)
      for (int c = std::max(0, r - kl); c <= std::min(n - 1, r + ku); ++c)
        L.band[(size_t)r * w + (c - r + kl)] = dense[(size_t)r * n + c];
    // wall rows: u(z=Lz) +- u(z=0) = sum of the class's coefficients
    L.c2_z.assign((size_t)n, 0.0);
    L.c1_z.assign(1, 1.0);
    for (int c = 0; c + 1 < n; ++c) L.c2_z[c] = 1.0;
    L.c2_nz = L.c2_z;
    L.c1_nz = L.c1_z;
    L.bc_rhs.assign(1, 0.0);
  }
  return out;
}

ChebMats build_cheb_mats(int N, double Lz) {
  ChebMats m;
  typedef long double ld;
  const ld pi = 3.141592653589793238462643383279502884L;
  std::vector<ld> bwd((size_t)N * N), fwd((size_t)N * N), D((size_t)N * N, 0.0L), S((size_t)N * N, 0.0L);
  const int twoM = 2 * (N - 1);
  for (int j = 0; j < N; ++j)
    for (int n = 0; n < N; ++n) {
      // T_n at x_j = -cos(pi j/(N-1)) equals (-1)^n cos(pi n j/(N-1))
      long long r = ((long long)n * j) % twoM;
      ld c = cosl(pi * (ld)r / (ld)(N - 1));
      bwd[(size_t)j * N + n] = ((n & 1) ? -c : c);
    }
  for (int n = 0; n < N; ++n)
    for (int j = 0; j < N; ++j) {
      long long r = ((long long)n * j) % twoM;
      ld c = cosl(pi * (ld)r / (ld)(N - 1));
      ld wj = (j == 0 || j == N - 1) ? 1.0L : 2.0L;
      ld hn = (n == 0 || n == N - 1) ? 0.5L : 1.0L;
      ld v = ((n & 1) ? -1.0L : 1.0L) * hn * wj * c / (ld)(N - 1);
      fwd[(size_t)n * N + j] = v;
    }
  const ld sc = 2.0L / (ld)Lz;
  for (int k = 0; k + 1 < N; ++k)
    for (int j = k + 1; j < N; ++j)
      if ((j - k) % 2 == 1) D[(size_t)k * N + j] = (k == 0 ? (ld)j : 2.0L * j) * sc;
  for (int k = 0; k < N; ++k)
    for (int j = k; j < std::min(N, k + 5); ++j) S[(size_t)k * N + j] = S_at(N, k, j);
  m.bwd.resize((size_t)N * N);
  m.bwd_d.resize((size_t)N * N);
  m.fwd.resize((size_t)N * N);
  m.sfwd.resize((size_t)N * N);
  for (int j = 0; j < N; ++j)
    for (int n = 0; n < N; ++n) {
      m.bwd[(size_t)j * N + n] = (double)bwd[(size_t)j * N + n];
      ld acc = 0;
      for (int q = 0; q < N; ++q) acc += bwd[(size_t)j * N + q] * D[(size_t)q * N + n];
      m.bwd_d[(size_t)j * N + n] = (double)acc;
      m.fwd[(size_t)j * N + n] = (double)fwd[(size_t)j * N + n];
    }
  for (int k = 0; k < N; ++k)
    for (int j = 0; j < N; ++j) {
      ld acc = 0;
      for (int q = k; q < std::min(N, k + 5); ++q) acc += S[(size_t)k * N + q] * fwd[(size_t)q * N + j];
      m.sfwd[(size_t)k * N + j] = (double)acc;
    }
  m.s3.resize((size_t)N * 3);
  for (int k = 0; k < N; ++k) {
    m.s3[3 * k + 0] = S_at(N, k, k);
    m.s3[3 * k + 1] = S_at(N, k, k + 2);
    m.s3[3 * k + 2] = S_at(N, k, k + 4);
  }
  return m;
}

bool make_fft_plan(int n, FftPlan* out) {
  FftPlan p;
  p.n = n;
  int r = n, ns = 0;
  while (r % 8 == 0 && ns < 16) { p.radix[ns++] = 8; r /= 8; }
  while (r % 4 == 0 && ns < 16) { p.radix[ns++] = 4; r /= 4; }
  while (r % 2 == 0 && ns < 16) { p.radix[ns++] = 2; r /= 2; }
  while (r % 3 == 0 && ns < 16) { p.radix[ns++] = 3; r /= 3; }
  if (r != 1 || n < 2) return false;
  p.nstages = ns;
  *out = p;
  return true;
}

}  // namespace tb
