// Per-neighbourhood PCA on the device: covariance accumulation and the
// symmetric 3x3 eigensolve (estimate_normals.cpp:84-110, vfuncs.cpp:1241-1293).
//
// The eigensolve is the cyclic Jacobi method (Golub & Van Loan, Matrix
// Computations, 4th ed., Alg. 8.5.2/8.5.3): rotations annihilate the (0,1),
// (0,2), (1,2) entries in turn until the off-diagonal mass is negligible.
// Eigenvalues come out ascending; each eigenvector is signed so that its
// largest-magnitude component is positive.
#pragma once

#include "common.cuh"

namespace pptkg {

template <typename P>
struct Sym3 {
  P a00, a01, a02, a11, a12, a22;
};

template <typename P>
__device__ __forceinline__ void jacobi_rotate(P& app, P& aqq, P& apq, P& arp, P& arq, P* V, int p, int q) {
  if (apq == (P)0) return;
  const P tau = (aqq - app) / ((P)2 * apq);
  const P t = (tau >= (P)0 ? (P)1 : (P)-1) / (fabs(tau) + sqrt((P)1 + tau * tau));
  const P c = (P)1 / sqrt((P)1 + t * t);
  const P s = t * c;
  app = app - t * apq;
  aqq = aqq + t * apq;
  apq = (P)0;
  const P rp = arp, rq = arq;
  arp = c * rp - s * rq;
  arq = s * rp + c * rq;
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const P vp = V[r * 3 + p], vq = V[r * 3 + q];
    V[r * 3 + p] = c * vp - s * vq;
    V[r * 3 + q] = s * vp + c * vq;
  }
}

// w ascending; V[r*3+c] = component r of eigenvector c.
template <typename P>
__device__ void eigh3(Sym3<P> A, P w[3], P V[9]) {
#pragma unroll
  for (int i = 0; i < 9; i++) V[i] = (i % 4 == 0) ? (P)1 : (P)0;
  const P eps = sizeof(P) == 4 ? (P)1.1920929e-7 : (P)2.220446049250313e-16;
  const int max_sweeps = sizeof(P) == 4 ? 12 : 20;
  for (int sweep = 0; sweep < max_sweeps; sweep++) {
    const P off = A.a01 * A.a01 + A.a02 * A.a02 + A.a12 * A.a12;
    const P diag = A.a00 * A.a00 + A.a11 * A.a11 + A.a22 * A.a22;
    if (!(off > eps * eps * (P)1e-4 * diag)) break;
    // (p, q) = (0, 1): the remaining row is 2
    jacobi_rotate(A.a00, A.a11, A.a01, A.a02, A.a12, V, 0, 1);
    // (0, 2): remaining row 1
    jacobi_rotate(A.a00, A.a22, A.a02, A.a01, A.a12, V, 0, 2);
    // (1, 2): remaining row 0
    jacobi_rotate(A.a11, A.a22, A.a12, A.a01, A.a02, V, 1, 2);
  }
  P d[3] = {A.a00, A.a11, A.a22};
  int o0 = 0, o1 = 1, o2 = 2;
  // stable sort of three values
  if (d[o1] < d[o0]) { int t = o0; o0 = o1; o1 = t; }
  if (d[o2] < d[o1]) { int t = o1; o1 = o2; o2 = t; }
  if (d[o1] < d[o0]) { int t = o0; o0 = o1; o1 = t; }
  const int ord[3] = {o0, o1, o2};
  P Vs[9];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const int src = ord[c];
    w[c] = src == 0 ? d[0] : (src == 1 ? d[1] : d[2]);
    P v0 = V[0 * 3 + src], v1 = V[1 * 3 + src], v2 = V[2 * 3 + src];
    int best = 0;
    P bm = fabs(v0);
    if (fabs(v1) > bm) { best = 1; bm = fabs(v1); }
    if (fabs(v2) > bm) { best = 2; }
    const P sel = best == 0 ? v0 : (best == 1 ? v1 : v2);
    const P sg = sel < (P)0 ? (P)-1 : (P)1;
    Vs[0 * 3 + c] = sg * v0;
    Vs[1 * 3 + c] = sg * v1;
    Vs[2 * 3 + c] = sg * v2;
  }
#pragma unroll
  for (int i = 0; i < 9; i++) V[i] = Vs[i];
}

// Neumaier compensated accumulator.
template <typename P>
struct CSum {
  P s = (P)0, c = (P)0;
  __device__ __forceinline__ void add(P x) {
    const P t = s + x;
    if (fabs(s) >= fabs(x))
      c += (s - t) + x;
    else
      c += (x - t) + s;
    s = t;
  }
  __device__ __forceinline__ P value() const { return s + c; }
};

// Relative gap between the two smallest eigenvalues, against the largest.
template <typename P>
__device__ __forceinline__ P rel_gap(const P w[3]) {
  const P tiny = sizeof(P) == 4 ? (P)1e-30 : (P)1e-300;
  return (w[1] - w[0]) / fmax(fabs(w[2]), tiny);
}

}  // namespace pptkg
