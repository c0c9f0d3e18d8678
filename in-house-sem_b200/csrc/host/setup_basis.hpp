// One-dimensional collocation rules and Lagrange interpolation for the native
// case setup.
//
// The setup must hand the kernels the same double-precision nodes and weights
// the reference computes (cpp/src/basis/quadrature.cpp,
// cpp/src/basis/lagrange.cpp): every mass entry, metric term and constraint
// weight is derived from them and then rounded to float, so a node one ulp
// off changes arrays.  The published constructions are therefore kept
// operation for operation:
//   - Jacobi polynomials by their three-term recurrence;
//   - roots by Newton's method with deflation, started from Chebyshev points
//     averaged with the previous root (Karniadakis & Sherwin, App. B);
//   - Gauss-Legendre weights 2 / ((1 - x^2) P_n'(x)^2);
//   - Gauss-Lobatto-Jacobi weights from the moment system sum_j w_j P_k(x_j) =
//     int (1-x)^alpha (1+x)^beta P_k(x) dx, solved by Gaussian elimination
//     with partial pivoting;
//   - barycentric Lagrange values and derivatives.
// The code around those operations is this library's own.
#pragma once

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

namespace insem_setup {

struct Rule1D {
  std::vector<double> x;  // ascending nodes on [-1, 1]
  std::vector<double> w;  // weights
  int n() const { return static_cast<int>(x.size()); }
};

// The Jacobi family P_k^{(a, b)} evaluated by recurrence.
struct JacobiFamily {
  double a, b;

  double value(int degree, double x) const {
    if (degree == 0) return 1.0;
    double lower = 1.0;
    double cur = 0.5 * ((a + b + 2.0) * x + (a - b));
    for (int k = 1; k < degree; ++k) {
      const double s = 2.0 * k + a + b;
      const double den = 2.0 * (k + 1) * (k + a + b + 1) * s;
      const double lin = (s + 1) * (a * a - b * b);
      const double slope = (s + 1) * (s + 2) * s;
      const double back = 2.0 * (k + a) * (k + b) * (s + 2);
      const double next = ((lin + slope * x) * cur - back * lower) / den;
      lower = cur;
      cur = next;
    }
    return cur;
  }

  // d/dx P_k^{(a,b)} = (k + a + b + 1) / 2 P_{k-1}^{(a+1,b+1)}
  double slope(int degree, double x) const {
    if (degree == 0) return 0.0;
    return 0.5 * (degree + a + b + 1) * JacobiFamily{a + 1.0, b + 1.0}.value(degree - 1, x);
  }

  // The `count` zeros of P_count^{(a,b)}, ascending.
  std::vector<double> zeros(int count) const {
    constexpr double kPi = 3.14159265358979323846;
    std::vector<double> z;
    z.reserve(count);
    for (int k = 0; k < count; ++k) {
      double r = -std::cos((2.0 * k + 1.0) * kPi / (2.0 * count));
      if (k > 0) r = 0.5 * (r + z.back());
      for (int it = 0; it < 200; ++it) {
        double pull = 0.0;  // deflation of the zeros already found
        for (double found : z) pull += 1.0 / (r - found);
        const double p = value(count, r);
        const double step = -p / (slope(count, r) - pull * p);
        r += step;
        if (std::abs(step) < 1e-16) break;
      }
      z.push_back(r);
    }
    return z;
  }
};

// x^k for the small non-negative integer exponents of the GLJ weight function
// (exact for k = 0 and 1, the values used).
inline double small_power(double v, int k) {
  double out = 1.0;
  for (int i = 0; i < k; ++i) out = i == 0 ? v : out * v;
  return out;
}

inline Rule1D gauss_rule(int n) {
  const JacobiFamily legendre{0.0, 0.0};
  Rule1D r;
  r.x = legendre.zeros(n);
  for (double x : r.x) {
    const double d = legendre.slope(n, x);
    r.w.push_back(2.0 / ((1.0 - x * x) * d * d));
  }
  return r;
}

// Dense solve by Gaussian elimination with partial pivoting, rows addressed
// through a permutation instead of being swapped.
inline std::vector<double> solve_moments(std::vector<double> m, std::vector<double> rhs, int n) {
  std::vector<int> row(n);
  for (int i = 0; i < n; ++i) row[i] = i;
  for (int c = 0; c < n; ++c) {
    int best = c;
    for (int r = c + 1; r < n; ++r)
      if (std::abs(m[row[r] * n + c]) > std::abs(m[row[best] * n + c])) best = r;
    if (m[row[best] * n + c] == 0.0) throw std::runtime_error("collocation weights: the moment matrix is singular");
    std::swap(row[c], row[best]);
    const double* piv = &m[row[c] * n];
    for (int r = c + 1; r < n; ++r) {
      double* dst = &m[row[r] * n];
      const double ratio = dst[c] / piv[c];
      for (int k = c; k < n; ++k) dst[k] -= ratio * piv[k];
      rhs[row[r]] -= ratio * rhs[row[c]];
    }
  }
  std::vector<double> out(n);
  for (int r = n - 1; r >= 0; --r) {
    const double* src = &m[row[r] * n];
    double acc = rhs[row[r]];
    for (int k = r + 1; k < n; ++k) acc -= src[k] * out[k];
    out[r] = acc / src[r];
  }
  return out;
}

// Gauss-Lobatto-Jacobi rule of n >= 2 points for the weight (1-x)^alpha (1+x)^beta.
inline Rule1D lobatto_rule(int n, int alpha, int beta) {
  if (n < 2) throw std::runtime_error("a Lobatto rule has at least two points");
  Rule1D r;
  r.x.push_back(-1.0);
  for (double z : JacobiFamily{alpha + 1.0, beta + 1.0}.zeros(n - 2)) r.x.push_back(z);
  r.x.push_back(1.0);
  const JacobiFamily legendre{0.0, 0.0};
  const Rule1D exact = gauss_rule(n + alpha + beta + 2);
  std::vector<double> moment(n, 0.0);
  for (int q = 0; q < exact.n(); ++q) {
    const double xq = exact.x[q];
    const double wq = exact.w[q] * small_power(1.0 - xq, alpha) * small_power(1.0 + xq, beta);
    for (int k = 0; k < n; ++k) moment[k] += wq * legendre.value(k, xq);
  }
  std::vector<double> vander(static_cast<std::size_t>(n) * n);
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j) vander[k * n + j] = legendre.value(k, r.x[j]);
  r.w = solve_moments(std::move(vander), std::move(moment), n);
  return r;
}

// Gauss-Lobatto-Legendre points (the collocation points) and the GLJ(0,1)
// points of the radial direction of elements touching the symmetry axis.
inline Rule1D gll_rule(int n) { return lobatto_rule(n, 0, 0); }
inline Rule1D glj_rule(int n) { return lobatto_rule(n, 0, 1); }

// Lagrange polynomials through distinct nodes, barycentric form.
class Interpolant {
 public:
  explicit Interpolant(std::vector<double> nodes) : x_(std::move(nodes)), lam_(x_.size(), 1.0) {
    const int n = size();
    for (int j = 0; j < n; ++j)
      for (int k = 0; k < n; ++k)
        if (k != j) lam_[j] /= x_[j] - x_[k];
  }

  int size() const { return static_cast<int>(x_.size()); }
  const std::vector<double>& nodes() const { return x_; }

  // l_j(t) for every j.
  std::vector<double> at(double t) const {
    const int n = size();
    std::vector<double> v(n);
    const int hit = coincident(t);
    if (hit >= 0) {
      v[hit] = 1.0;
      return v;
    }
    double sum = 0.0;
    for (int j = 0; j < n; ++j) {
      v[j] = lam_[j] / (t - x_[j]);
      sum += v[j];
    }
    for (double& e : v) e /= sum;
    return v;
  }

  // l_j'(t) for every j.
  std::vector<double> slope_at(double t) const {
    const int n = size();
    const int hit = coincident(t);
    if (hit >= 0) {
      std::vector<double> d(n);
      double diag = 0.0;
      for (int j = 0; j < n; ++j) {
        if (j == hit) continue;
        d[j] = (lam_[j] / lam_[hit]) / (x_[hit] - x_[j]);
        diag -= d[j];
      }
      d[hit] = diag;
      return d;
    }
    std::vector<double> d = at(t);
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int k = 0; k < n; ++k)
        if (k != j) s += 1.0 / (t - x_[k]);
      d[j] *= s;
    }
    return d;
  }

  // D[i][j] = l_j'(x_i), row-major.
  std::vector<double> derivative_matrix() const {
    std::vector<double> d;
    for (double xi : x_) {
      const auto row = slope_at(xi);
      d.insert(d.end(), row.begin(), row.end());
    }
    return d;
  }

 private:
  int coincident(double t) const {
    for (int j = 0; j < size(); ++j)
      if (std::abs(t - x_[j]) <= 1e-14 * (1.0 + std::abs(x_[j]))) return j;
    return -1;
  }

  std::vector<double> x_;
  std::vector<double> lam_;
};

}  // namespace insem_setup
