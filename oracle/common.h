// Test infrastructure (oracle side): helpers shared by the reference harness
// (ref_harness.cpp) and the CPU restatement (port.cpp).  Nothing here is
// linked into the product library.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>

namespace oracle {

// Element type codes, identical to the product C ABI (include/pptkg.h).
enum DType { F32 = 0, F64 = 1, I8 = 2, I16 = 3, I32 = 4, I64 = 5, U8 = 6, U16 = 7, U32 = 8, U64 = 9 };

template <typename F>
bool dispatch_type(int dtype, F&& f) {
  switch (dtype) {
    case F32: f(float()); return true;
    case F64: f(double()); return true;
    case I8: f(int8_t()); return true;
    case I16: f(int16_t()); return true;
    case I32: f(int32_t()); return true;
    case I64: f(int64_t()); return true;
    case U8: f(uint8_t()); return true;
    case U16: f(uint16_t()); return true;
    case U32: f(uint32_t()); return true;
    case U64: f(uint64_t()); return true;
  }
  return false;
}

// Query element types supported by the oracle: the tree's own type, float32
// or float64.  Other query types only change the order in which equal-distance
// candidates are visited, never a result set.
template <typename T, typename F>
bool dispatch_query(int qdtype, int tdtype, F&& f) {
  if (qdtype == tdtype) {
    f(T());
    return true;
  }
  if (qdtype == F32) {
    f(float());
    return true;
  }
  if (qdtype == F64) {
    f(double());
    return true;
  }
  return false;
}

template <int D>
struct DimTag {
  static const int value = D;
};

template <typename F>
bool dispatch_dim(int dim, F&& f) {
  switch (dim) {
    case 2: f(DimTag<2>()); return true;
    case 3: f(DimTag<3>()); return true;
    case 4: f(DimTag<4>()); return true;
  }
  return false;
}

template <typename F>
bool dispatch(int dtype, int dim, F&& f) {
  bool ok = false;
  dispatch_type(dtype, [&](auto t) {
    dispatch_dim(dim, [&](auto d) {
      f(t, d);
      ok = true;
    });
  });
  return ok;
}

// Eigen-decomposition of a symmetric 3x3 matrix A (row-major) in T by the
// cyclic Jacobi method (Golub & Van Loan, Matrix Computations, 4th ed.,
// Alg. 8.5.2 sym.schur2 and Alg. 8.5.3).  On return w holds the eigenvalues
// ascending and V the eigenvectors as columns (V[r*3+c] = component r of
// eigenvector c); each eigenvector is signed so that its component of
// largest magnitude (the first one on ties) is positive.
template <typename T>
void jacobi3(const T A_in[9], T w[3], T V[9]) {
  T A[9];
  for (int i = 0; i < 9; i++) A[i] = A_in[i];
  for (int i = 0; i < 9; i++) V[i] = (i % 4 == 0) ? (T)1 : (T)0;
  const T eps = std::numeric_limits<T>::epsilon();
  for (int sweep = 0; sweep < 60; sweep++) {
    T off = A[1] * A[1] + A[2] * A[2] + A[5] * A[5];
    T diag = A[0] * A[0] + A[4] * A[4] + A[8] * A[8];
    if (!(off > eps * eps * (T)1e-4 * diag)) break;
    const int P[3] = {0, 0, 1}, Q[3] = {1, 2, 2};
    for (int r = 0; r < 3; r++) {
      int p = P[r], q = Q[r];
      T apq = A[p * 3 + q];
      if (apq == (T)0) continue;
      T app = A[p * 3 + p], aqq = A[q * 3 + q];
      T tau = (aqq - app) / ((T)2 * apq);
      T t = (tau >= (T)0 ? (T)1 : (T)-1) / (std::fabs(tau) + std::sqrt((T)1 + tau * tau));
      T c = (T)1 / std::sqrt((T)1 + t * t);
      T s = t * c;
      for (int k = 0; k < 3; k++) {
        T akp = A[k * 3 + p], akq = A[k * 3 + q];
        A[k * 3 + p] = c * akp - s * akq;
        A[k * 3 + q] = s * akp + c * akq;
      }
      for (int k = 0; k < 3; k++) {
        T apk = A[p * 3 + k], aqk = A[q * 3 + k];
        A[p * 3 + k] = c * apk - s * aqk;
        A[q * 3 + k] = s * apk + c * aqk;
      }
      for (int k = 0; k < 3; k++) {
        T vkp = V[k * 3 + p], vkq = V[k * 3 + q];
        V[k * 3 + p] = c * vkp - s * vkq;
        V[k * 3 + q] = s * vkp + c * vkq;
      }
    }
  }
  int order[3] = {0, 1, 2};
  T d[3] = {A[0], A[4], A[8]};
  std::sort(order, order + 3, [&](int a, int b) { return d[a] < d[b] || (d[a] == d[b] && a < b); });
  T Vs[9];
  for (int c = 0; c < 3; c++) {
    w[c] = d[order[c]];
    int best = 0;
    for (int r = 0; r < 3; r++) {
      Vs[r * 3 + c] = V[r * 3 + order[c]];
      if (std::fabs(Vs[r * 3 + c]) > std::fabs(Vs[best * 3 + c])) best = r;
    }
    if (Vs[best * 3 + c] < (T)0)
      for (int r = 0; r < 3; r++) Vs[r * 3 + c] = -Vs[r * 3 + c];
  }
  for (int i = 0; i < 9; i++) V[i] = Vs[i];
}

}  // namespace oracle
