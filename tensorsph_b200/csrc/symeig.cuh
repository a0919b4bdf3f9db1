// Small symmetric eigen-solves used by the renormalised density gradient.
//
// floored_solve<D>(M, g, f): x = V diag(1 / max(l_k, f * trace(M)/D)) V^T g,
// zero when trace(M) <= 0 -- the eigenvalue-floored inverse of the first
// moment matrix (density_diffusion.py:95-142).  2x2 in closed form, 3x3 by
// cyclic Jacobi rotations; both in double.
#pragma once

#include <cuda_runtime.h>

namespace tsph {

__device__ __forceinline__ void eig2(const double m[3][3], double lam[2], double vec[2][2]) {
  const double a = m[0][0], b = m[1][0], c = m[1][1];
  const double half = 0.5 * (a - c);
  const double rad = sqrt(half * half + b * b);
  const double mid = 0.5 * (a + c);
  lam[0] = mid - rad;
  lam[1] = mid + rad;
  if (rad == 0.0) {
    vec[0][0] = 1; vec[0][1] = 0; vec[1][0] = 0; vec[1][1] = 1;
    return;
  }
  // eigenvector of the larger eigenvalue, then its orthogonal complement
  double x, y;
  if (half >= 0) { x = half + rad; y = b; } else { x = b; y = rad - half; }
  const double nrm = sqrt(x * x + y * y);
  x /= nrm; y /= nrm;
  vec[1][0] = x; vec[1][1] = y;
  vec[0][0] = -y; vec[0][1] = x;
}

__device__ __forceinline__ void eig3(const double m_in[3][3], double lam[3], double vec[3][3]) {
  double a[3][3], v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[i][j] = m_in[i][j];
  for (int sweep = 0; sweep < 32; ++sweep) {
    const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    const double diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (off <= 1e-34 * diag || off == 0.0) break;
    for (int p = 0; p < 2; ++p) {
      for (int q = p + 1; q < 3; ++q) {
        const double apq = a[p][q];
        if (apq == 0.0) continue;
        const double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 3; ++k) {
          const double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k) {
          const double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; ++k) {
          const double vkp = v[k][p], vkq = v[k][q];
          v[k][p] = c * vkp - s * vkq;
          v[k][q] = s * vkp + c * vkq;
        }
      }
    }
  }
  for (int k = 0; k < 3; ++k) {
    lam[k] = a[k][k];
    for (int i = 0; i < 3; ++i) vec[k][i] = v[i][k];  // vec[k] = k-th eigenvector
  }
}

template <int D>
__device__ __forceinline__ void floored_solve(const double m[3][3], const double g[3], double floor_frac,
                                              double out[3]) {
  double lam[3] = {0, 0, 0}, vec[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  if (D == 2) {
    double v2[2][2];
    eig2(m, lam, v2);
    for (int k = 0; k < 2; ++k)
      for (int i = 0; i < 2; ++i) vec[k][i] = v2[k][i];
  } else {
    eig3(m, lam, vec);
  }
  double trace = 0;
  for (int k = 0; k < D; ++k) trace += lam[k];
  for (int i = 0; i < 3; ++i) out[i] = 0.0;
  if (!(trace > 0.0)) return;
  double mean = trace / D;
  mean = mean > 1e-30 ? mean : 1e-30;
  const double fl = floor_frac * mean;
  for (int k = 0; k < D; ++k) {
    double proj = 0;
    for (int i = 0; i < D; ++i) proj += vec[k][i] * g[i];
    const double l = lam[k] > fl ? lam[k] : fl;
    for (int i = 0; i < D; ++i) out[i] += vec[k][i] * (proj / l);
  }
}

}  // namespace tsph
