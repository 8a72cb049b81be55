// Hard sources written on the device (emsolve with PlaneWave, WavePacket,
// Dipole, Pulse; upstream wakis/sources.py:142-762).
//
// Upstream's source.update(solver, t) evaluates the source with numpy and
// assigns it to a box of one field component before every step.  Every such
// value has the form (A(t) * P(i, j, k)) * B(t): a per-step factor, a fixed
// profile over the box (1 for point sources and uniform planes) and a second
// per-step factor, multiplied in upstream's order.  The host forms A, B for
// all steps of the run and P once (the same expressions, the same numpy
// broadcasting), uploads them, and this kernel writes the values of step t
// with no per-step host work or transfer.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/wakis_b200.h"
#include "abi_internal.h"
#include "fit_comp.cuh"

namespace wk {
namespace {

template <int DT>
__global__ void k_source_write(void* field, uint16_t* comp, long long N, int Nx, int NxNy, int d,
                               int i0, int j0, int k0, int ni, int nj, int nk,
                               const double* prof, const double* A, const double* B,
                               long long n_steps, const long long* step_dev, long long step) {
  const long long t = step + (step_dev ? *step_dev : 0);
  if (t < 0 || t >= n_steps) return;
  const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long cells = (long long)ni * nj * nk;
  if (m >= cells) return;
  const int a = (int)(m % ni);
  const long long r = m / ni;
  const int b = (int)(r % nj), c = (int)(r / nj);
  const long long n = (long long)d * N + (i0 + a) + (long long)(j0 + b) * Nx +
                      (long long)(k0 + c) * NxNy;
  double v = A[t];
  if (prof) v = __dmul_rn(v, prof[m]);
  if (B) v = __dmul_rn(v, B[t]);
  if (DT == WK_F64) {
    static_cast<double*>(field)[n] = v;
  } else {
    const float f = (float)v;
    static_cast<float*>(field)[n] = f;
    if (DT == WK_F32C) comp[n] = comp_enc((float)(v - (double)f));
  }
}

}  // namespace
}  // namespace wk

using namespace wk;

extern "C" int wk_source_write(void* field, int dtype, void* comp, int Nx, int Ny, int Nz,
                               int component, int i0, int i1, int j0, int j1, int k0, int k1,
                               const double* prof, const double* A, const double* B,
                               long long n_steps, const long long* step_dev, long long step,
                               void* stream) {
  const char* where = "wk_source_write";
  if (!field || !A) return wk_fail(WK_E_NULL, "%s: field or A is NULL", where);
  if (dtype != WK_F64 && dtype != WK_F32 && dtype != WK_F32C)
    return wk_fail(WK_E_DTYPE, "%s: dtype %d", where, dtype);
  if (dtype == WK_F32C && !comp)
    return wk_fail(WK_E_NULL, "%s: WK_F32C needs the compensation words", where);
  if (Nx < 1 || Ny < 1 || Nz < 1 || (long long)Nx * Ny > (1LL << 31))
    return wk_fail(WK_E_SHAPE, "%s: grid %dx%dx%d", where, Nx, Ny, Nz);
  if (component < 0 || component > 2)
    return wk_fail(WK_E_RANGE, "%s: component %d", where, component);
  if (i0 < 0 || j0 < 0 || k0 < 0 || i1 > Nx || j1 > Ny || k1 > Nz || i0 > i1 || j0 > j1 ||
      k0 > k1)
    return wk_fail(WK_E_RANGE, "%s: box [%d,%d)x[%d,%d)x[%d,%d) outside the grid", where, i0,
                   i1, j0, j1, k0, k1);
  if (n_steps < 0) return wk_fail(WK_E_RANGE, "%s: n_steps %lld", where, n_steps);
  if (!step_dev && (step < 0 || step >= n_steps))
    return wk_fail(WK_E_RANGE, "%s: step %lld outside the %lld tabulated steps", where, step,
                   n_steps);
  const long long cells = (long long)(i1 - i0) * (j1 - j0) * (k1 - k0);
  if (cells == 0) return WK_OK;
  const long long N = (long long)Nx * Ny * Nz;
  const unsigned blocks = (unsigned)((cells + 255) / 256);
  cudaStream_t st = (cudaStream_t)stream;
  const int ni = i1 - i0, nj = j1 - j0, nk = k1 - k0;
  const int NxNy = Nx * Ny;
  uint16_t* cw = static_cast<uint16_t*>(comp);
  if (dtype == WK_F64)
    k_source_write<WK_F64><<<blocks, 256, 0, st>>>(field, cw, N, Nx, NxNy, component, i0, j0, k0,
                                                   ni, nj, nk, prof, A, B, n_steps, step_dev,
                                                   step);
  else if (dtype == WK_F32)
    k_source_write<WK_F32><<<blocks, 256, 0, st>>>(field, cw, N, Nx, NxNy, component, i0, j0, k0,
                                                   ni, nj, nk, prof, A, B, n_steps, step_dev,
                                                   step);
  else
    k_source_write<WK_F32C><<<blocks, 256, 0, st>>>(field, cw, N, Nx, NxNy, component, i0, j0,
                                                    k0, ni, nj, nk, prof, A, B, n_steps,
                                                    step_dev, step);
  return wk_check_launch(where);
}
