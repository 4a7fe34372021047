// Covariances of neighbourhood lists: the MEAN / DOT(TRANSPOSE(Y), Y) / n
// chain that pptk's expression layer evaluates per neighbourhood with vfuncs
// (pptk/points/expr.py:27-72, vfuncs.cpp `_mean`, `_dot`, `_transpose`),
// fused into one kernel over a CSR list of neighbourhoods; its output feeds
// the batched 3x3 eigensolve (vfuncs `_eigh`).
#include "common.cuh"
#include "profile.cuh"
#include "query.cuh"
#include "util.cuh"

namespace pptkg {

namespace {

// One thread per neighbourhood: mean, then the centred second moments, both
// accumulated in double (per-element rounding of the float32 expression
// chain is not reproduced; results agree with a float64 evaluation to the
// precision of T).  Index entries outside [0, n), or offsets outside
// [0, total] or decreasing, set *status = 4 and give a NaN matrix.  C (m x 3 x 3, row-major) = Y^T Y / count, Y the centred rows.
template <typename T>
__global__ void k_nbhd_cov(const T* pts, int64_t n, const int64_t* off, const int32_t* idx, int64_t total, int64_t m,
                           T* C, int* status) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int64_t b = off[i], e = off[i + 1];
  T* out = C + i * 9;
  bool bad = b < 0 || e < b || e > total;
  double s0 = 0, s1 = 0, s2 = 0;
  for (int64_t j = b; j < e && !bad; j++) {
    const int64_t p = idx[j];
    if (p < 0 || p >= n) {
      bad = true;
      break;
    }
    s0 += (double)pts[p * 3];
    s1 += (double)pts[p * 3 + 1];
    s2 += (double)pts[p * 3 + 2];
  }
  const double cnt = (double)(e - b);
  if (bad || cnt <= 0) {
    if (bad) atomicExch(status, 4);
    for (int t = 0; t < 9; t++) out[t] = (T)NAN;
    return;
  }
  const double m0 = s0 / cnt, m1 = s1 / cnt, m2 = s2 / cnt;
  double c00 = 0, c01 = 0, c02 = 0, c11 = 0, c12 = 0, c22 = 0;
  for (int64_t j = b; j < e; j++) {
    const int64_t p = idx[j];
    const double a = (double)pts[p * 3] - m0, c = (double)pts[p * 3 + 1] - m1, d = (double)pts[p * 3 + 2] - m2;
    c00 += a * a;
    c01 += a * c;
    c02 += a * d;
    c11 += c * c;
    c12 += c * d;
    c22 += d * d;
  }
  out[0] = (T)(c00 / cnt);
  out[1] = out[3] = (T)(c01 / cnt);
  out[2] = out[6] = (T)(c02 / cnt);
  out[4] = (T)(c11 / cnt);
  out[5] = out[7] = (T)(c12 / cnt);
  out[8] = (T)(c22 / cnt);
}

}  // namespace

template <typename T>
void nbhd_covariance(const T* d_pts, int64_t n, const int64_t* d_off, const int32_t* d_idx, int64_t total, int64_t m,
                     T* d_C, cudaStream_t st) {
  if (m <= 0) return;
  DevBuf<int> status(1, st);
  PPTKG_CUDA(cudaMemsetAsync(status.get(), 0, sizeof(int), st));
  {
    Stage s("nbhd_cov", st);
    k_nbhd_cov<T><<<(unsigned)((m + 255) / 256), 256, 0, st>>>(d_pts, n, d_off, d_idx, total, m, d_C,
                                                                status.get());
    PPTKG_CHECK_LAUNCH();
  }
  int h = 0;
  PPTKG_CUDA(cudaMemcpyAsync(&h, status.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
  PPTKG_CUDA(cudaStreamSynchronize(st));
  if (h) throw Error(E_RANGE, "neighbourhood index outside of [0, n) or decreasing offsets");
}

template void nbhd_covariance<float>(const float*, int64_t, const int64_t*, const int32_t*, int64_t, int64_t,
                                     float*, cudaStream_t);
template void nbhd_covariance<double>(const double*, int64_t, const int64_t*, const int32_t*, int64_t, int64_t,
                                      double*, cudaStream_t);

}  // namespace pptkg
