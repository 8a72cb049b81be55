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
#include "fit_common.cuh"
#include "fit_kernels.cuh"

using namespace wk;

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

// Matrix-free transposes (wk_adj_h_fit / wk_adj_e_fit), one thread per
// cell m and all three components, from the compact coefficient tables the
// step kernels read (T: their type; L: the adjoint state type, the
// arithmetic type).  With B0 row (d, n) factor itA_d(n) pec_d(n), column
// (e, n - off) factor tL_e pmc_e, and A row (d, n) factor
// dt iA_d(n) imu_d(n) pmc_d(n), column (e, n + off) factor L_e pec_e:
//   lamH'[e, m] = lamH[e, m] + dt tL_e(m) pmc_e(m) sum sg u_d(m + off),
//       u_d(n) = itA_d(n) pec_d(n) ieps_d(n) lamE[d, n]            (n < N)
//   lamE'[e, m] = decay[e, m] lamE[e, m] - L_e(m) pec_e(m) sum sg w_d(m - off),
//       w_d(n) = dt iA_d(n) imu_d(n) pmc_d(n) lamH'[d, n]          (n >= 0)
// with the signs and offsets of the curl (x: +1, y: +Nx, z: +Nx*Ny).
template <typename T, typename L>
__device__ __forceinline__ L adj_u(const FitParams<T>& p, const L* lamE, int d, Cell c,
                                   long long n) {
  const int id = load_id(p.mat_id, p.id_bytes, n);
  T f = d == 0 ? p.itAx[c.j + (long long)c.k * p.Ny]
               : (d == 1 ? p.itAy[c.i + (long long)c.k * p.Nx] : p.itAz[c.i + (long long)c.j * p.Nx]);
  if (p.has_pec && !face_val(p.pec_face, d, c.i, c.j, c.k, p.Nx, p.Ny, p.Nz)) f = T(0);
  return (L)f * (L)p.mat[9 * id + d] * lamE[d * p.N + n];
}

template <typename T, typename L>
__device__ __forceinline__ L adj_w(const FitParams<T>& p, const L* lamH, int d, Cell c,
                                   long long n) {
  const int id = load_id(p.mat_id, p.id_bytes, n);
  T f = d == 0 ? p.iAx[c.j + (long long)c.k * p.Ny]
               : (d == 1 ? p.iAy[c.i + (long long)c.k * p.Nx] : p.iAz[c.i + (long long)c.j * p.Nx]);
  if (p.has_pmc && !face_val(p.pmc_face, d, c.i, c.j, c.k, p.Nx, p.Ny, p.Nz)) f = T(0);
  return (L)p.dt * (L)f * (L)p.mat[9 * id + 3 + d] * lamH[d * p.N + n];
}

template <typename T, typename L>
__global__ void __launch_bounds__(kAdjThreads)
k_adj_h_fit(FitParams<T> p, const L* __restrict__ lamE, const L* lamH_in, L* lamH_out) {
  const long long m = blockIdx.x * (long long)kAdjThreads + threadIdx.x;
  if (m >= p.N) return;
  const Cell c = cell_of(m, p.Nx, p.Ny);
  const long long N = p.N;
  const bool vx = m + 1 < N, vy = m + p.Nx < N, vz = m + p.NxNy < N;
  const Cell cx = plus_x(c, p.Nx, p.Ny), cy = plus_y(c, p.Ny);
  Cell cz = c;
  cz.k++;
  const L u0 = adj_u<T, L>(p, lamE, 0, c, m), u1 = adj_u<T, L>(p, lamE, 1, c, m),
          u2 = adj_u<T, L>(p, lamE, 2, c, m);
  const L u0y = vy ? adj_u<T, L>(p, lamE, 0, cy, m + p.Nx) : L(0);
  const L u0z = vz ? adj_u<T, L>(p, lamE, 0, cz, m + p.NxNy) : L(0);
  const L u1x = vx ? adj_u<T, L>(p, lamE, 1, cx, m + 1) : L(0);
  const L u1z = vz ? adj_u<T, L>(p, lamE, 1, cz, m + p.NxNy) : L(0);
  const L u2x = vx ? adj_u<T, L>(p, lamE, 2, cx, m + 1) : L(0);
  const L u2y = vy ? adj_u<T, L>(p, lamE, 2, cy, m + p.Nx) : L(0);
  const L acc[3] = {u1 - u1z + u2y - u2, u0z - u0 - u2x + u2, u0 - u0y + u1x - u1};
  const L dt = (L)p.dt;
#pragma unroll
  for (int e = 0; e < 3; e++)
    lamH_out[e * N + m] = lamH_in[e * N + m] + dt * (L)coltL(p, e, c.i, c.j, c.k) * acc[e];
}

template <typename T, typename L>
__global__ void __launch_bounds__(kAdjThreads)
k_adj_e_fit(FitParams<T> p, const L* __restrict__ lamH, const L* lamE_in,
            const L* __restrict__ decay, L* lamE_out) {
  const long long m = blockIdx.x * (long long)kAdjThreads + threadIdx.x;
  if (m >= p.N) return;
  const Cell c = cell_of(m, p.Nx, p.Ny);
  const long long N = p.N;
  const bool vx = m >= 1, vy = m >= p.Nx, vz = m >= p.NxNy;
  const Cell cx = minus_x(c, p.Nx, p.Ny), cy = minus_y(c, p.Ny);
  Cell cz = c;
  cz.k--;
  const L w0 = adj_w<T, L>(p, lamH, 0, c, m), w1 = adj_w<T, L>(p, lamH, 1, c, m),
          w2 = adj_w<T, L>(p, lamH, 2, c, m);
  const L w0y = vy ? adj_w<T, L>(p, lamH, 0, cy, m - p.Nx) : L(0);
  const L w0z = vz ? adj_w<T, L>(p, lamH, 0, cz, m - p.NxNy) : L(0);
  const L w1x = vx ? adj_w<T, L>(p, lamH, 1, cx, m - 1) : L(0);
  const L w1z = vz ? adj_w<T, L>(p, lamH, 1, cz, m - p.NxNy) : L(0);
  const L w2x = vx ? adj_w<T, L>(p, lamH, 2, cx, m - 1) : L(0);
  const L w2y = vy ? adj_w<T, L>(p, lamH, 2, cy, m - p.Nx) : L(0);
  const L acc[3] = {w1z - w1 + w2 - w2y, w0 - w0z - w2 + w2x, w0y - w0 + w1 - w1x};
#pragma unroll
  for (int e = 0; e < 3; e++) {
    const L dec = decay ? decay[e * N + m] : L(1);
    lamE_out[e * N + m] = dec * lamE_in[e * N + m] - (L)colL(p, e, c.i, c.j, c.k) * acc[e];
  }
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

// ---------------------------------------------------------------------------
// Matrix-free reverse step from the solver descriptor (coefficient tables of
// wk_fit_desc; the state buffers of the descriptor are not touched).
namespace {
template <typename L>
int adj_fit_launch(const wk_fit_desc* d, int which, const void* a, const void* b,
                   const void* decay, void* out, cudaStream_t st) {
  const long long N = (long long)d->Nx * d->Ny * d->Nz;
  const bool coef64 = d->dtype == WK_F64 || d->dtype == WK_F32C;
  if (coef64) {
    FitParams<double> p = make_params<double>(d, d->par);
    if (which == 0)
      k_adj_h_fit<double, L><<<blocks(N), kAdjThreads, 0, st>>>(p, (const L*)a, (const L*)b, (L*)out);
    else
      k_adj_e_fit<double, L><<<blocks(N), kAdjThreads, 0, st>>>(p, (const L*)a, (const L*)b,
                                                                  (const L*)decay, (L*)out);
  } else {
    FitParams<float> p = make_params<float>(d, d->par);
    if (which == 0)
      k_adj_h_fit<float, L><<<blocks(N), kAdjThreads, 0, st>>>(p, (const L*)a, (const L*)b, (L*)out);
    else
      k_adj_e_fit<float, L><<<blocks(N), kAdjThreads, 0, st>>>(p, (const L*)a, (const L*)b,
                                                                 (const L*)decay, (L*)out);
  }
  return WK_OK;
}

int adj_fit(const wk_fit_desc* d, int dtype, int which, const void* a, const void* b,
            const void* decay, void* out, void* stream, const char* where) {
  int rc = wk_validate_fit(d, where);
  if (rc) return rc;
  if (dtype != WK_F64 && dtype != WK_F32) return wk_fail(WK_E_DTYPE, "%s: dtype", where);
  if (!a || !b || !out) return wk_fail(WK_E_NULL, "%s: NULL pointer", where);
  if ((long long)d->Nx * d->Ny * d->Nz >= (1LL << 31))
    return wk_fail(WK_E_SHAPE, "%s: more than 2^31 cells", where);
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == WK_F64) adj_fit_launch<double>(d, which, a, b, decay, out, st);
  else adj_fit_launch<float>(d, which, a, b, decay, out, st);
  return wk_check_launch(where);
}
}  // namespace

extern "C" int wk_adj_h_fit(const wk_fit_desc* d, int dtype, const void* lamE,
                            const void* lamH_in, void* lamH_out, void* stream) {
  return adj_fit(d, dtype, 0, lamE, lamH_in, nullptr, lamH_out, stream, "wk_adj_h_fit");
}

extern "C" int wk_adj_e_fit(const wk_fit_desc* d, int dtype, const void* lamH,
                            const void* lamE_in, const void* decay, void* lamE_out,
                            void* stream) {
  return adj_fit(d, dtype, 1, lamH, lamE_in, decay, lamE_out, stream, "wk_adj_e_fit");
}
