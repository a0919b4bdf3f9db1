// Smoothing kernels evaluated per pair inside the gather loops.
//
// Cubic spline (Monaghan 1992), support 2h, q = r / h:
//   f(q)  = 1 - 1.5 q^2 + 0.75 q^3      (q < 1)
//         = 0.25 (2 - q)^3              (1 <= q < 2)
//   f'(q) = -3 q + 2.25 q^2 | -0.75 (2 - q)^2
//   f''(q)= -3 + 4.5 q      | 1.5 (2 - q)
// W = sigma f(q), grad_i W = delta * sigma f'(q) / (h max(r, eps)),
// 3-D Laplacian = sigma (f'' + 2 f'/q) / h^2 with the q -> 0 limit -6 for
// 2 f'/q (droplet_impact.py:276-371, threed/kernel3.py:48-181).
// Wendland C2: f = (1 - q/2)^4 (2 q + 1), f' = -5 q (1 - q/2)^3
// (droplet_impact.py:320-346).
#pragma once

#include <cuda_runtime.h>

namespace tsph {

template <class T>
struct Cubic {
  T inv_h, h, sigma, eps;
  __device__ __forceinline__ T shape(T q) const {
    if (q < T(1)) return T(1) - T(1.5) * q * q + T(0.75) * q * q * q;
    if (q < T(2)) {
      T t = T(2) - q;
      return T(0.25) * t * t * t;
    }
    return T(0);
  }
  __device__ __forceinline__ T dshape(T q) const {
    if (q < T(1)) return T(-3) * q + T(2.25) * q * q;
    if (q < T(2)) {
      T t = T(2) - q;
      return T(-0.75) * t * t;
    }
    return T(0);
  }
  // W(r)
  __device__ __forceinline__ T w(T r) const {
    T s = shape(r / h);
    return sigma * (s > T(0) ? s : T(0));
  }
  // W(r) and the gradient scale g such that grad_i W = delta * g.
  __device__ __forceinline__ void wg(T r, T& W, T& g) const {
    T q = r / h;
    T s = shape(q);
    W = sigma * (s > T(0) ? s : T(0));
    g = sigma * dshape(q) / (h * (r > eps ? r : eps));
  }
  // 3-D Laplacian of W (threed/kernel3.py:108-124).
  __device__ __forceinline__ T lap3(T r) const {
    T q = r / h;
    if (!(q < T(2))) return T(0);
    T second = q < T(1) ? T(-3) + T(4.5) * q : T(1.5) * (T(2) - q);
    T twice = q > T(1e-10) ? T(2) * dshape(q) / (q > eps ? q : eps) : T(-6);
    return sigma * (second + twice) / (h * h);
  }
};

template <class T>
struct Wendland {
  T h, sigma, eps;
  __device__ __forceinline__ T w(T r) const {
    T q = r / h;
    T t = T(1) - T(0.5) * q;
    t = t > T(0) ? t : T(0);
    T t2 = t * t;
    return sigma * t2 * t2 * (T(2) * q + T(1));
  }
  __device__ __forceinline__ void wg(T r, T& W, T& g) const {
    T q = r / h;
    T t = T(1) - T(0.5) * q;
    t = t > T(0) ? t : T(0);
    T t2 = t * t;
    W = sigma * t2 * t2 * (T(2) * q + T(1));
    g = sigma * (T(-5) * q * t2 * t) / (h * (r > eps ? r : eps));
  }
};

}  // namespace tsph
