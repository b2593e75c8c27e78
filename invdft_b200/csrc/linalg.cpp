#include "linalg.h"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace invdft {

bool cholesky_lower(int n, const std::vector<double> &S, std::vector<double> &L) {
  L.assign((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) {
    double d = S[(size_t)j * n + j];
    for (int k = 0; k < j; ++k) d -= L[(size_t)j * n + k] * L[(size_t)j * n + k];
    if (!(d > 0.0) || !std::isfinite(d)) return false;
    const double ljj = std::sqrt(d);
    L[(size_t)j * n + j] = ljj;
    for (int i = j + 1; i < n; ++i) {
      double s = S[(size_t)i * n + j];
      for (int k = 0; k < j; ++k) s -= L[(size_t)i * n + k] * L[(size_t)j * n + k];
      L[(size_t)i * n + j] = s / ljj;
    }
  }
  return true;
}

void lower_inverse_transpose(int n, const std::vector<double> &L, std::vector<double> &T) {
  // Li = L^{-1} (lower), then T = Li^T.
  std::vector<double> Li((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) {
    Li[(size_t)j * n + j] = 1.0 / L[(size_t)j * n + j];
    for (int i = j + 1; i < n; ++i) {
      double s = 0.0;
      for (int k = j; k < i; ++k) s += L[(size_t)i * n + k] * Li[(size_t)k * n + j];
      Li[(size_t)i * n + j] = -s / L[(size_t)i * n + i];
    }
  }
  T.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) T[(size_t)i * n + j] = Li[(size_t)j * n + i];
}

void jacobi_eigh(int n, const std::vector<double> &Ain, std::vector<double> &w, std::vector<double> &V) {
  std::vector<double> A(Ain);
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
  auto a = [&](int i, int j) -> double & { return A[(size_t)i * n + j]; };
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        tot += a(i, j) * a(i, j);
        if (i != j) off += a(i, j) * a(i, j);
      }
    if (off <= 1e-32 * tot || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a(p, q);
        if (apq == 0.0) continue;
        const double app = a(p, p), aqq = a(q, q);
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          const double akp = a(k, p), akq = a(k, q);
          a(k, p) = c * akp - s * akq;
          a(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = a(p, k), aqk = a(q, k);
          a(p, k) = c * apk - s * aqk;
          a(q, k) = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = V[(size_t)k * n + p], vkq = V[(size_t)k * n + q];
          V[(size_t)k * n + p] = c * vkp - s * vkq;
          V[(size_t)k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return a(x, x) < a(y, y); });
  w.resize(n);
  std::vector<double> Vs((size_t)n * n);
  for (int j = 0; j < n; ++j) {
    const int src = order[j];
    w[j] = a(src, src);
    int imax = 0;
    double vmax = -1.0;
    for (int i = 0; i < n; ++i) {
      const double v = std::fabs(V[(size_t)i * n + src]);
      if (v > vmax) { vmax = v; imax = i; }
    }
    const double sg = V[(size_t)imax * n + src] < 0.0 ? -1.0 : 1.0;
    for (int i = 0; i < n; ++i) Vs[(size_t)i * n + j] = sg * V[(size_t)i * n + src];
  }
  V.swap(Vs);
}

double hash_uniform(uint64_t i, uint64_t salt) {
  uint64_t h = (i * 2654435761ull + salt * 40503ull) & 0xFFFFFFFFull;
  h ^= h >> 15;
  h = (h * 2246822519ull) & 0xFFFFFFFFull;
  h ^= h >> 13;
  return (double)h / 4294967296.0 - 0.5;
}

double partial_occupancy(double eig, double mu, double kT) {
  const double x = (eig - mu) / kT;
  if (x >= 0) return std::exp(-x) / (1.0 + std::exp(-x));
  return 1.0 / (1.0 + std::exp(x));
}

double partial_occupancy_der(double eig, double mu, double kT) {
  const double x = (eig - mu) / kT;
  const double e = std::exp(-std::fabs(x));
  return -e / (kT * (1.0 + e) * (1.0 + e));
}

double fermi_energy(const std::vector<double> &eig, double n_electrons, double kT) {
  double lo = *std::min_element(eig.begin(), eig.end()) - 1.0;
  double hi = *std::max_element(eig.begin(), eig.end()) + 1.0;
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    double n = 0.0;
    for (double e : eig) n += partial_occupancy(e, mid, kT);
    n *= 2.0;
    if (n > n_electrons) hi = mid;
    else lo = mid;
    if (hi - lo < 1e-15 * std::max(1.0, std::fabs(mid))) break;
  }
  return 0.5 * (lo + hi);
}

}  // namespace invdft
