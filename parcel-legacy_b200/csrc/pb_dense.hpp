// pb_dense.hpp -- small dense host routines for CA-GMRES (column-major, s <= 64).
//
// The reference calls LAPACK for these (DPOTRF, DTRTRI, DHSEQR, DGEMM:
// src/QRDecomposition.f90:713-828, src/pcagmres.f90:613-742, 879-1052).  They act on
// matrices of order s*t <= 64, so they stay on the host, as in the reference.
#pragma once

#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

namespace pb {
namespace dense {

// Column-major view helper.
struct Mat {
  int m = 0, n = 0;
  std::vector<double> a;
  Mat() = default;
  Mat(int m_, int n_) : m(m_), n(n_), a((size_t)m_ * n_, 0.0) {}
  double& operator()(int i, int j) { return a[(size_t)j * m + i]; }
  double operator()(int i, int j) const { return a[(size_t)j * m + i]; }
};

// C = A * B
inline Mat gemm(const Mat& A, const Mat& B) {
  Mat C(A.m, B.n);
  for (int j = 0; j < B.n; ++j)
    for (int k = 0; k < A.n; ++k) {
      const double b = B(k, j);
      for (int i = 0; i < A.m; ++i) C(i, j) += A(i, k) * b;
    }
  return C;
}

// Upper Cholesky factor R of a symmetric positive definite G (G = R^T R).  Returns false
// if G is not numerically positive definite.
inline bool chol_upper(const Mat& G, Mat& R) {
  const int n = G.n;
  R = Mat(n, n);
  for (int j = 0; j < n; ++j) {
    double d = G(j, j);
    for (int k = 0; k < j; ++k) d -= R(k, j) * R(k, j);
    if (!(d > 0.0)) return false;
    const double rjj = std::sqrt(d);
    R(j, j) = rjj;
    for (int i = j + 1; i < n; ++i) {
      double v = G(j, i);
      for (int k = 0; k < j; ++k) v -= R(k, j) * R(k, i);
      R(j, i) = v / rjj;
    }
  }
  return true;
}

// Inverse of an upper triangular matrix.
inline Mat trinv_upper(const Mat& R) {
  const int n = R.n;
  Mat X(n, n);
  for (int j = 0; j < n; ++j) {
    X(j, j) = 1.0 / R(j, j);
    for (int i = j - 1; i >= 0; --i) {
      double v = 0.0;
      for (int k = i + 1; k <= j; ++k) v += R(i, k) * X(k, j);
      X(i, j) = -v / R(i, i);
    }
  }
  return X;
}

// Eigenvalues of an upper Hessenberg matrix by the Francis double-shift QR iteration
// (Golub & Van Loan, Matrix Computations, section 7.5) with deflation on negligible
// subdiagonal entries and the usual exceptional shifts after 10 and 20 iterations.
// Complex conjugate pairs are returned next to each other, positive imaginary part first.
inline void hessenberg_eigs(Mat H, std::vector<double>& wr, std::vector<double>& wi) {
  const int n = H.n;
  wr.assign(n, 0.0);
  wi.assign(n, 0.0);
  double anorm = 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = std::max(i - 1, 0); j < n; ++j) anorm += std::fabs(H(i, j));
  int nn = n - 1;
  double shift = 0.0;
  while (nn >= 0) {
    int its = 0, l = 0;
    do {
      for (l = nn; l >= 1; --l) {                       // look for a small subdiagonal
        double sc = std::fabs(H(l - 1, l - 1)) + std::fabs(H(l, l));
        if (sc == 0.0) sc = anorm;
        if (std::fabs(H(l, l - 1)) + sc == sc) { H(l, l - 1) = 0.0; break; }
      }
      const double x = H(nn, nn);
      if (l == nn) {                                    // 1x1 block converged
        wr[nn] = x + shift;
        wi[nn] = 0.0;
        --nn;
        continue;
      }
      const double y = H(nn - 1, nn - 1);
      const double w = H(nn, nn - 1) * H(nn - 1, nn);
      if (l == nn - 1) {                                // 2x2 block converged
        const double p = 0.5 * (y - x);
        const double q = p * p + w;
        const double z = std::sqrt(std::fabs(q));
        const double xs = x + shift;
        if (q >= 0.0) {
          const double zz = p + (p >= 0.0 ? z : -z);
          wr[nn - 1] = wr[nn] = xs + zz;
          if (zz != 0.0) wr[nn] = xs - w / zz;
          wi[nn - 1] = wi[nn] = 0.0;
        } else {
          wr[nn - 1] = wr[nn] = xs + p;
          wi[nn - 1] = z;
          wi[nn] = -z;
        }
        nn -= 2;
        continue;
      }
      if (its == 60) {                                  // give up on this block
        for (int i = l; i <= nn; ++i) { wr[i] = H(i, i) + shift; wi[i] = 0.0; }
        nn = l - 1;
        continue;
      }
      double sx = x, sy = y, sw = w;
      if (its == 10 || its == 20) {                     // exceptional shift
        shift += sx;
        for (int i = 0; i <= nn; ++i) H(i, i) -= sx;
        const double sc = std::fabs(H(nn, nn - 1)) + std::fabs(H(nn - 1, nn - 2));
        sx = sy = 0.75 * sc;
        sw = -0.4375 * sc * sc;
      }
      ++its;
      // first column of (H - s1)(H - s2), starting at the lowest row m where the bulge
      // can be introduced
      int m = nn - 2;
      double p = 0.0, q = 0.0, r = 0.0;
      for (; m >= l; --m) {
        const double z = H(m, m);
        const double rr = sx - z, ss = sy - z;
        p = (rr * ss - sw) / H(m + 1, m) + H(m, m + 1);
        q = H(m + 1, m + 1) - z - rr - ss;
        r = H(m + 2, m + 1);
        const double sc = std::fabs(p) + std::fabs(q) + std::fabs(r);
        p /= sc; q /= sc; r /= sc;
        if (m == l) break;
        const double u = std::fabs(H(m, m - 1)) * (std::fabs(q) + std::fabs(r));
        const double v = std::fabs(p) * (std::fabs(H(m - 1, m - 1)) + std::fabs(z) + std::fabs(H(m + 1, m + 1)));
        if (u + v == v) break;
      }
      for (int i = m + 2; i <= nn; ++i) {
        H(i, i - 2) = 0.0;
        if (i != m + 2) H(i, i - 3) = 0.0;
      }
      // chase the bulge with 3x3 Householder reflections
      for (int k = m; k <= nn - 1; ++k) {
        double norm = 1.0;
        if (k != m) {
          p = H(k, k - 1);
          q = H(k + 1, k - 1);
          r = (k != nn - 1) ? H(k + 2, k - 1) : 0.0;
          norm = std::fabs(p) + std::fabs(q) + std::fabs(r);
          if (norm == 0.0) continue;
          p /= norm; q /= norm; r /= norm;
        }
        double s = std::sqrt(p * p + q * q + r * r);
        if (p < 0.0) s = -s;
        if (k == m) {
          if (l != m) H(k, k - 1) = -H(k, k - 1);
        } else {
          H(k, k - 1) = -s * norm;
        }
        p += s;
        const double hx = p / s, hy = q / s, hz = r / s;
        q /= p;
        r /= p;
        for (int j = k; j <= nn; ++j) {                 // rows k..k+2
          double t = H(k, j) + q * H(k + 1, j);
          if (k != nn - 1) { t += r * H(k + 2, j); H(k + 2, j) -= t * hz; }
          H(k + 1, j) -= t * hy;
          H(k, j) -= t * hx;
        }
        const int imax = std::min(nn, k + 3);
        for (int i = l; i <= imax; ++i) {               // columns k..k+2
          double t = hx * H(i, k) + hy * H(i, k + 1);
          if (k != nn - 1) { t += hz * H(i, k + 2); H(i, k + 2) -= t * r; }
          H(i, k + 1) -= t * q;
          H(i, k) -= t;
        }
      }
    } while (l < nn - 1);
  }
}

}  // namespace dense
}  // namespace pb
