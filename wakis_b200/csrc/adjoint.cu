// Adjoint of the FIT leap-frog step (reverse mode), sm_100a.
//
// Forward step n (wakis/solverFIT3D.py:482-503, beam and capture fused as in
// the step kernels):
//   H' = H - A E                       (A = dt iDa iDmu C Ds, PEC/PMC masks)
//   E' = E + dt ieps (B0 H' - J),      J = sigma E for n >= 1 (0 at n = 0,
//                                      the beam current on the beam line)
// with B = diag(ieps) B0.  Given the adjoints lE', lH' of (E', H') the
// reverse step is
//   lH = lH' + dt B0^T (ieps lE')                        (wk_adj_h)
//   lE = (1 - dt ieps sigma m) lE' - A^T lH  (+ source)  (wk_adj_e)
// (m = 1 where J = sigma E holds), and the parameter adjoints of step n are
//   d/d ieps_c  += sum_comp lE' dt (B0 H' - J)             (wk_adj_grad)
//   d/d sigma_c += -dt sum_comp ieps lE' E m,
// the increment dt (B0 H' - J) of the design entries being formed in FP64
// by the caller (no cancellation of E' - E in a float state).
// A^T and B0^T are CSR matrices assembled on the host from the same
// coefficient tables the step kernels read (one thread per row; ~4 entries
// per row), in the state dtype.
#include <stdint.h>

#include "../../include/wakis_b200.h"
#include "abi_internal.h"

namespace {

constexpr int kAdjThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kAdjThreads)
k_adj_h(const long long* __restrict__ rowptr, const int* __restrict__ col,
        const T* __restrict__ val, long long nrows, const T* __restrict__ lamE,
        const T* __restrict__ ieps, T dt, const T* lamH_in, T* lamH_out) {
  const long long r = blockIdx.x * (long long)kAdjThreads + threadIdx.x;
  if (r >= nrows) return;
  T acc = T(0);
  for (long long q = rowptr[r]; q < rowptr[r + 1]; q++) {
    const int c = col[q];
    acc += val[q] * (ieps[c] * lamE[c]);
  }
  lamH_out[r] = lamH_in[r] + dt * acc;
}

template <typename T>
__global__ void __launch_bounds__(kAdjThreads)
k_adj_e(const long long* __restrict__ rowptr, const int* __restrict__ col,
        const T* __restrict__ val, long long nrows, const T* __restrict__ lamH,
        const T* lamE_in, const T* __restrict__ decay, T* lamE_out) {
  const long long r = blockIdx.x * (long long)kAdjThreads + threadIdx.x;
  if (r >= nrows) return;
  T acc = T(0);
  for (long long q = rowptr[r]; q < rowptr[r + 1]; q++) acc += val[q] * lamH[col[q]];
  lamE_out[r] = decay[r] * lamE_in[r] - acc;
}

template <typename T>
__global__ void __launch_bounds__(kAdjThreads)
k_adj_grad(const long long* __restrict__ cells, long long ncell, long long N,
           const T* __restrict__ lamE1, const double* __restrict__ inc,
           const T* __restrict__ E0, const T* __restrict__ ieps, const T* __restrict__ smask,
           int use_sigma, double dt, double* gI, double* gS) {
  const long long q = blockIdx.x * (long long)kAdjThreads + threadIdx.x;
  if (q >= ncell) return;
  const long long n = cells[q];
  double gi = 0.0, gs = 0.0;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const long long x = d * N + n;
    const double l = (double)lamE1[x];
    gi += l * inc[d * ncell + q];
    if (use_sigma) gs -= dt * (double)ieps[x] * l * (double)E0[x] * (double)smask[x];
  }
  gI[q] += gi;
  gS[q] += gs;
}

int check_common(int dtype, const void* a, const void* b, long long n, const char* where) {
  if (dtype != WK_F64 && dtype != WK_F32) return wk_fail(WK_E_DTYPE, "%s: dtype", where);
  if (!a || !b) return wk_fail(WK_E_NULL, "%s: NULL pointer", where);
  if (n < 0) return wk_fail(WK_E_SHAPE, "%s: negative size", where);
  return WK_OK;
}

unsigned blocks(long long n) { return (unsigned)((n + kAdjThreads - 1) / kAdjThreads); }

}  // namespace

extern "C" int wk_adj_h(int dtype, const long long* rowptr, const int* col, const void* val,
                        long long nrows, const void* lamE, const void* ieps, double dt,
                        const void* lamH_in, void* lamH_out, void* stream) {
  int rc = check_common(dtype, rowptr, col, nrows, "wk_adj_h");
  if (rc) return rc;
  if (!val || !lamE || !ieps || !lamH_in || !lamH_out)
    return wk_fail(WK_E_NULL, "wk_adj_h: NULL pointer");
  if (nrows == 0) return WK_OK;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == WK_F64)
    k_adj_h<double><<<blocks(nrows), kAdjThreads, 0, st>>>(
        rowptr, col, (const double*)val, nrows, (const double*)lamE, (const double*)ieps, dt,
        (const double*)lamH_in, (double*)lamH_out);
  else
    k_adj_h<float><<<blocks(nrows), kAdjThreads, 0, st>>>(
        rowptr, col, (const float*)val, nrows, (const float*)lamE, (const float*)ieps,
        (float)dt, (const float*)lamH_in, (float*)lamH_out);
  return wk_check_launch("wk_adj_h");
}

extern "C" int wk_adj_e(int dtype, const long long* rowptr, const int* col, const void* val,
                        long long nrows, const void* lamH, const void* lamE_in,
                        const void* decay, void* lamE_out, void* stream) {
  int rc = check_common(dtype, rowptr, col, nrows, "wk_adj_e");
  if (rc) return rc;
  if (!val || !lamH || !lamE_in || !decay || !lamE_out)
    return wk_fail(WK_E_NULL, "wk_adj_e: NULL pointer");
  if (nrows == 0) return WK_OK;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == WK_F64)
    k_adj_e<double><<<blocks(nrows), kAdjThreads, 0, st>>>(
        rowptr, col, (const double*)val, nrows, (const double*)lamH, (const double*)lamE_in,
        (const double*)decay, (double*)lamE_out);
  else
    k_adj_e<float><<<blocks(nrows), kAdjThreads, 0, st>>>(
        rowptr, col, (const float*)val, nrows, (const float*)lamH, (const float*)lamE_in,
        (const float*)decay, (float*)lamE_out);
  return wk_check_launch("wk_adj_e");
}

extern "C" int wk_adj_grad(int dtype, const long long* cells, long long ncell, long long N,
                           const void* lamE1, const double* inc, const void* E0,
                           const void* ieps, const void* smask, int use_sigma, double dt,
                           double* gI, double* gS, void* stream) {
  int rc = check_common(dtype, cells, lamE1, ncell, "wk_adj_grad");
  if (rc) return rc;
  if (!inc || !E0 || !ieps || !smask || !gI || !gS)
    return wk_fail(WK_E_NULL, "wk_adj_grad: NULL pointer");
  if (ncell == 0) return WK_OK;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == WK_F64)
    k_adj_grad<double><<<blocks(ncell), kAdjThreads, 0, st>>>(
        cells, ncell, N, (const double*)lamE1, inc, (const double*)E0, (const double*)ieps,
        (const double*)smask, use_sigma, dt, gI, gS);
  else
    k_adj_grad<float><<<blocks(ncell), kAdjThreads, 0, st>>>(
        cells, ncell, N, (const float*)lamE1, inc, (const float*)E0, (const float*)ieps,
        (const float*)smask, use_sigma, dt, gI, gS);
  return wk_check_launch("wk_adj_grad");
}
