#include "mpo_builders.h"

#include <cmath>
#include <complex>
#include <functional>
#include <stdexcept>

namespace dmrg2cli {

namespace {
typedef std::complex<double> cd;
typedef std::vector<cd> Op;  // d x d row-major, op[out*d + in]

Op zeros(int d) { return Op((size_t)d * d, 0.0); }
Op eye(int d) {
  Op o = zeros(d);
  for (int i = 0; i < d; ++i) o[(size_t)i * d + i] = 1.0;
  return o;
}
Op scale(cd a, const Op& o) {
  Op r(o.size());
  for (size_t i = 0; i < o.size(); ++i) r[i] = a * o[i];
  return r;
}
Op matmul(const Op& a, const Op& b, int d) {
  Op r = zeros(d);
  for (int i = 0; i < d; ++i)
    for (int k = 0; k < d; ++k)
      for (int j = 0; j < d; ++j) r[(size_t)i * d + j] += a[(size_t)i * d + k] * b[(size_t)k * d + j];
  return r;
}
Op kron(const Op& a, int da, const Op& b, int db) {
  int d = da * db;
  Op r = zeros(d);
  for (int i = 0; i < da; ++i)
    for (int j = 0; j < da; ++j)
      for (int k = 0; k < db; ++k)
        for (int l = 0; l < db; ++l)
          r[(size_t)(i * db + k) * d + (j * db + l)] = a[(size_t)i * da + j] * b[(size_t)k * db + l];
  return r;
}
Op add(const Op& a, const Op& b) {
  Op r(a.size());
  for (size_t i = 0; i < a.size(); ++i) r[i] = a[i] + b[i];
  return r;
}

// bulk tensor with D x D operator-valued entries; boundaries cut to row 0 / column D-1
struct Bulk {
  int D, d;
  std::vector<Op> e;  // D*D entries
  Bulk(int D_, int d_) : D(D_), d(d_), e((size_t)D_ * D_, Op((size_t)d_ * d_, 0.0)) {}
  void put(int wl, int wr, const Op& o) { e[(size_t)wl * D + wr] = o; }
};

Mpo finish(const Bulk& B, int L, bool cplx, const std::string& name) {
  Mpo m;
  m.L = L;
  m.d = B.d;
  m.cplx = cplx;
  m.name = name;
  const int D = B.D, d = B.d, per = cplx ? 2 : 1;
  for (int i = 0; i < L; ++i) {
    int r0 = 0, r1 = D, c0 = 0, c1 = D;
    if (i == 0) r1 = 1;
    if (i == L - 1) c0 = D - 1;
    int a = r1 - r0, b = c1 - c0;
    m.Dl.push_back(a);
    m.Dr.push_back(b);
    std::vector<double> w((size_t)a * b * d * d * per, 0.0);
    for (int wl = 0; wl < a; ++wl)
      for (int wr = 0; wr < b; ++wr) {
        const Op& o = B.e[(size_t)(wl + r0) * D + (wr + c0)];
        for (int s = 0; s < d; ++s)
          for (int t = 0; t < d; ++t) {
            cd v = o[(size_t)t * d + s];  // applied operator O[t][s] stored at W[..][s][t]
            size_t idx = ((((size_t)wl * b + wr) * d + s) * d + t) * per;
            w[idx] = v.real();
            if (cplx) w[idx + 1] = v.imag();
            else if (v.imag() != 0.0) throw std::logic_error("complex entry in a real MPO");
          }
      }
    m.W.push_back(std::move(w));
  }
  return m;
}

const Op SZ = {0.5, 0.0, 0.0, -0.5};
const Op SP = {0.0, 1.0, 0.0, 0.0};  // |up><down|
const Op SM = {0.0, 0.0, 1.0, 0.0};
const Op PX = {0.0, 1.0, 1.0, 0.0};
const Op PZ = {1.0, 0.0, 0.0, -1.0};
}  // namespace

Mpo heisenberg(int L, double J, double delta, double hz) {
  Bulk B(5, 2);
  B.put(0, 0, eye(2));
  B.put(0, 1, SP);
  B.put(0, 2, SM);
  B.put(0, 3, SZ);
  B.put(0, 4, scale(-hz, SZ));
  B.put(1, 4, scale(0.5 * J, SM));
  B.put(2, 4, scale(0.5 * J, SP));
  B.put(3, 4, scale(J * delta, SZ));
  B.put(4, 4, eye(2));
  return finish(B, L, false, "heisenberg");
}

Mpo tfim(int L, double J, double h) {
  Bulk B(3, 2);
  B.put(0, 0, eye(2));
  B.put(0, 1, scale(-J, PZ));
  B.put(0, 2, scale(-h, PX));
  B.put(1, 2, PZ);
  B.put(2, 2, eye(2));
  return finish(B, L, false, "tfim");
}

Mpo josephson(int L, int n_max, double E_J, double E_C, double n_g, double phi,
              const std::string& onsite) {
  const int d = 2 * n_max + 1;
  Op n = zeros(d), R = zeros(d), Lo = zeros(d);
  for (int i = 0; i < d; ++i) n[(size_t)i * d + i] = (double)(i - n_max);
  for (int i = 0; i + 1 < d; ++i) {
    R[(size_t)(i + 1) * d + i] = 1.0;
    Lo[(size_t)i * d + (i + 1)] = 1.0;
  }
  Op U;
  if (onsite == "reference") {
    U = add(scale(E_C, matmul(n, n, d)), scale(-n_g, n));
  } else if (onsite == "shifted") {
    Op m = add(n, scale(-n_g, eye(d)));
    U = scale(E_C, matmul(m, m, d));
  } else {
    throw std::invalid_argument("josephson: onsite must be 'reference' or 'shifted'");
  }
  cd alpha = -0.5 * E_J * std::exp(cd(0.0, phi));
  Bulk B(4, d);
  B.put(0, 0, eye(d));
  B.put(0, 1, scale(alpha, R));
  B.put(0, 2, scale(std::conj(alpha), Lo));
  B.put(0, 3, U);
  B.put(1, 3, Lo);
  B.put(2, 3, R);
  B.put(3, 3, eye(d));
  return finish(B, L, true, "josephson");
}

Mpo longrange(int L, const std::vector<double>& Js) {
  const int Rg = (int)Js.size();
  const int D = 2 + 3 * Rg, done = D - 1;
  Bulk B(D, 2);
  const Op ops[3] = {SP, SM, SZ};
  const Op close[3] = {SM, SP, SZ};
  const double wt[3] = {0.5, 0.5, 1.0};
  auto st = [&](int t, int k) { return 1 + t * Rg + (k - 1); };
  B.put(0, 0, eye(2));
  B.put(done, done, eye(2));
  for (int t = 0; t < 3; ++t) {
    B.put(0, st(t, 1), ops[t]);
    for (int k = 1; k <= Rg; ++k) {
      if (Js[k - 1] != 0.0) B.put(st(t, k), done, scale(wt[t] * Js[k - 1], close[t]));
      if (k < Rg) B.put(st(t, k), st(t, k + 1), eye(2));
    }
  }
  return finish(B, L, false, Rg == 2 ? "j1j2" : "j1j2j3");
}

Mpo ladder(int L_rungs, double J_leg, double J_rung) {
  const Op I2 = eye(2);
  Op leg1[3] = {kron(SP, 2, I2, 2), kron(SM, 2, I2, 2), kron(SZ, 2, I2, 2)};
  Op leg2[3] = {kron(I2, 2, SP, 2), kron(I2, 2, SM, 2), kron(I2, 2, SZ, 2)};
  Op rung = scale(J_rung, add(add(scale(0.5, matmul(leg1[0], leg2[1], 4)),
                                  scale(0.5, matmul(leg1[1], leg2[0], 4))),
                              matmul(leg1[2], leg2[2], 4)));
  const int close[3] = {1, 0, 2};
  const double wt[3] = {0.5, 0.5, 1.0};
  Bulk B(8, 4);
  B.put(0, 0, eye(4));
  B.put(0, 7, rung);
  B.put(7, 7, eye(4));
  for (int t = 0; t < 3; ++t) {
    B.put(0, 1 + t, leg1[t]);
    B.put(0, 4 + t, leg2[t]);
    B.put(1 + t, 7, scale(wt[t] * J_leg, leg1[close[t]]));
    B.put(4 + t, 7, scale(wt[t] * J_leg, leg2[close[t]]));
  }
  return finish(B, L_rungs, false, "ladder");
}

}  // namespace dmrg2cli
