// Frequency-domain field monitor: acc[f][d][n] += E_d[n] * phase_f, the
// running DFT of upstream FieldMonitor.update (wakis/field_monitors.py:60-107),
// one thread per cell reading the three E components once for all
// frequencies.  The complex product of a real E and phase (pr, pi) is formed
// as (E*pr - 0*pi, E*pi + 0*pr) like numpy's complex multiply of E + 0j.
#include <stdint.h>

#include "../../include/wakis_b200.h"
#include "abi_internal.h"

namespace {

constexpr int kMonThreads = 256;
constexpr int kMonMaxFreq = 64;

template <typename T>
__global__ void __launch_bounds__(kMonThreads)
k_monitor(const T* __restrict__ E, long long N, const double* __restrict__ phases, int nf,
          double* __restrict__ acc) {
  __shared__ double ph[2 * kMonMaxFreq];
  for (int q = threadIdx.x; q < 2 * nf; q += kMonThreads) ph[q] = phases[q];
  __syncthreads();
  const long long n = blockIdx.x * (long long)kMonThreads + threadIdx.x;
  if (n >= N) return;
  const double e[3] = {(double)E[n], (double)E[N + n], (double)E[2 * N + n]};
  for (int f = 0; f < nf; f++) {
    const double pr = ph[2 * f], pi = ph[2 * f + 1];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      double* a = acc + 2 * (((long long)f * 3 + d) * N + n);
      const double re = __dsub_rn(__dmul_rn(e[d], pr), __dmul_rn(0.0, pi));
      const double im = __dadd_rn(__dmul_rn(e[d], pi), __dmul_rn(0.0, pr));
      a[0] = __dadd_rn(a[0], re);
      a[1] = __dadd_rn(a[1], im);
    }
  }
}

}  // namespace

extern "C" int wk_field_monitor(const void* E, int dtype, long long N, const double* phases,
                                int nf, double* acc, void* stream) {
  if (!E || !phases || !acc) return wk_fail(WK_E_NULL, "wk_field_monitor: NULL pointer");
  if (dtype != WK_F64 && dtype != WK_F32) return wk_fail(WK_E_DTYPE, "wk_field_monitor: dtype");
  if (N <= 0) return wk_fail(WK_E_SHAPE, "wk_field_monitor: N <= 0");
  if (nf < 0 || nf > kMonMaxFreq)
    return wk_fail(WK_E_RANGE, "wk_field_monitor: 0 <= nf <= %d", kMonMaxFreq);
  if (nf == 0) return WK_OK;
  if ((uintptr_t)acc % 16) return wk_fail(WK_E_ALIGN, "wk_field_monitor: acc not 16-byte aligned");
  cudaStream_t st = (cudaStream_t)stream;
  const unsigned blocks = (unsigned)((N + kMonThreads - 1) / kMonThreads);
  if (dtype == WK_F64)
    k_monitor<double><<<blocks, kMonThreads, 0, st>>>((const double*)E, N, phases, nf, acc);
  else
    k_monitor<float><<<blocks, kMonThreads, 0, st>>>((const float*)E, N, phases, nf, acc);
  return wk_check_launch("wk_field_monitor");
}
