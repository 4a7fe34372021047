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
  // order the eigenpairs ascending with compare-exchanges on whole columns
  // (static register indices only)
  P d0 = A.a00, d1 = A.a11, d2 = A.a22;
  P c0[3] = {V[0], V[3], V[6]}, c1[3] = {V[1], V[4], V[7]}, c2[3] = {V[2], V[5], V[8]};
  auto cx = [](P& da, P* ca, P& db, P* cb) {
    if (db < da) {
      P t = da;
      da = db;
      db = t;
#pragma unroll
      for (int r = 0; r < 3; r++) {
        t = ca[r];
        ca[r] = cb[r];
        cb[r] = t;
      }
    }
  };
  cx(d0, c0, d1, c1);
  cx(d1, c1, d2, c2);
  cx(d0, c0, d1, c1);
  auto canon = [](P* c) {
    // largest-magnitude component positive (first on ties)
    P sel = c[0], bm = fabs(c[0]);
    if (fabs(c[1]) > bm) {
      sel = c[1];
      bm = fabs(c[1]);
    }
    if (fabs(c[2]) > bm) sel = c[2];
    if (sel < (P)0) {
      c[0] = -c[0];
      c[1] = -c[1];
      c[2] = -c[2];
    }
  };
  canon(c0);
  canon(c1);
  canon(c2);
  w[0] = d0;
  w[1] = d1;
  w[2] = d2;
#pragma unroll
  for (int r = 0; r < 3; r++) {
    V[r * 3 + 0] = c0[r];
    V[r * 3 + 1] = c1[r];
    V[r * 3 + 2] = c2[r];
  }
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
