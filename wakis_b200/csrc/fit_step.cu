// FIT leap-frog step kernels (sm_100a) and their C-ABI launchers.
//
// wk_fit_step       fused step: one pass reads E[par], H[par] and writes
//                   E[par^1], H[par^1] (ping-pong, so neighbouring blocks
//                   always read the old state).
// wk_fit_step_split two in-place passes (H, then E), the schedule of
//                   upstream's _one_step (wakis/solverFIT3D.py:482-503).
#include "../../include/wakis_b200.h"
#include "abi_internal.h"
#include "fit_common.cuh"

using namespace wk;

namespace {

constexpr int kThreads = 256;

template <typename T>
__global__ void k_zero_ghosts(FitParams<T> p) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= p.N) return;
  Cell c = cell_of(n, p.Nx, p.Ny);
  T* E = p.E_in; T* H = p.H_in;
  // H tangential components on the high faces (solverFIT3D.py:829-835)
  if (c.i == p.Nx - 1) { H[p.N + n] = T(0); H[2 * p.N + n] = T(0); }
  if (c.j == p.Ny - 1) { H[n] = T(0); H[2 * p.N + n] = T(0); }
  if (c.k == p.Nz - 1) { H[n] = T(0); H[p.N + n] = T(0); }
  // E along each axis in the last cell of that axis (838-840)
  if (c.i == p.Nx - 1) E[n] = T(0);
  if (c.j == p.Ny - 1) E[p.N + n] = T(0);
  if (c.k == p.Nz - 1) E[2 * p.N + n] = T(0);
}

template <typename T>
__device__ __forceinline__ void capture(const FitParams<T>& p, Cell c, long long n,
                                        long long step, T ez) {
  int a = c.i - p.cap_i0, b = c.j - p.cap_j0;
  if (a >= 0 && a < p.cap_ni && b >= 0 && b < p.cap_nj) {
    long long w = (long long)a * p.cap_nj + b;
    p.cap[(w * p.Nz + c.k) * p.cap_nt + (step - p.cap_step0)] = ez;
  }
}

// J value entering the E row of component d at cell n (before the update).
template <typename T>
__device__ __forceinline__ T j_in(const FitParams<T>& p, int d, Cell c, long long n,
                                  long long step, T e_old, T sigma) {
  if (d == 2 && c.i == p.ixs && c.j == p.iys) {
    if (p.line_on) return p.line[(step - p.line_step0) * p.Nz + c.k];
    if (p.beam_on) return beam_j(p, step, c.k);
  }
  if (p.j_mode == WK_J_SIGMA_E) return mul(sigma, e_old);
  if (p.j_mode == WK_J_ARRAY) return p.J[(long long)d * p.N + n];
  return T(0);
}

// ---------------------------------------------------------------- split ---
template <typename T>
__global__ void k_h_split(FitParams<T> p, long long step) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= p.N) return;
  Cell c = cell_of(n, p.Nx, p.Ny);
  int id = load_id(p.mat_id, p.id_bytes, n);
  if (p.cap_on) capture(p, c, n, step, p.E_in[2 * p.N + n]);
  T h[3];
#pragma unroll
  for (int d = 0; d < 3; d++) h[d] = h_row(p, p.E_in, p.H_in[d * p.N + n], d, c, n, id);
#pragma unroll
  for (int d = 0; d < 3; d++) p.H_out[d * p.N + n] = h[d];
}

template <typename T>
__global__ void k_e_split(FitParams<T> p, long long step) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= p.N) return;
  Cell c = cell_of(n, p.Nx, p.Ny);
  int id = load_id(p.mat_id, p.id_bytes, n);
  const T* Hn = p.H_out;
  auto hval = [&](int e, long long m) -> T { return Hn[e * p.N + m]; };
#pragma unroll
  for (int d = 0; d < 3; d++) {
    T ieps = p.mat[9 * id + d];
    T sigma = p.mat[9 * id + 6 + d];
    T eold = p.E_in[d * p.N + n];
    T jv = j_in(p, d, c, n, step, eold, sigma);
    T curl = e_curl(p, d, c, n, ieps, hval);
    T enew = add(eold, mul(p.dt, sub(curl, mul(ieps, jv))));
    p.E_out[d * p.N + n] = enew;
    if (p.j_mode == WK_J_ARRAY && p.use_cond) p.J[d * p.N + n] = mul(sigma, enew);
  }
}

// ---------------------------------------------------------------- fused ---
// One thread per cell: the new H of the cell and of the three backward
// neighbours it needs is computed from the old state, so the pass reads
// only E_in/H_in and writes only E_out/H_out.
template <typename T>
__global__ void k_fused(FitParams<T> p, long long step) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= p.N) return;
  const long long N = p.N;
  Cell c = cell_of(n, p.Nx, p.Ny);
  int id = load_id(p.mat_id, p.id_bytes, n);
  if (p.cap_on) capture(p, c, n, step, p.E_in[2 * N + n]);
  T hn[3];
#pragma unroll
  for (int d = 0; d < 3; d++) hn[d] = h_row(p, p.E_in, p.H_in[d * N + n], d, c, n, id);
  // backward neighbours (flat offsets 1, Nx, Nx*Ny)
  T hm1[3], hmy[3], hmz[3];
  if (n >= 1) {
    Cell cm = minus_x(c, p.Nx, p.Ny); long long m = n - 1;
    int idm = load_id(p.mat_id, p.id_bytes, m);
    hm1[1] = h_row(p, p.E_in, p.H_in[N + m], 1, cm, m, idm);
    hm1[2] = h_row(p, p.E_in, p.H_in[2 * N + m], 2, cm, m, idm);
  } else { hm1[1] = hm1[2] = T(0); }
  hm1[0] = T(0);
  if (n >= p.Nx) {
    Cell cm = minus_y(c, p.Ny); long long m = n - p.Nx;
    int idm = load_id(p.mat_id, p.id_bytes, m);
    hmy[0] = h_row(p, p.E_in, p.H_in[m], 0, cm, m, idm);
    hmy[2] = h_row(p, p.E_in, p.H_in[2 * N + m], 2, cm, m, idm);
  } else { hmy[0] = hmy[2] = T(0); }
  hmy[1] = T(0);
  if (n >= p.NxNy) {
    Cell cm = c; cm.k--; long long m = n - p.NxNy;
    int idm = load_id(p.mat_id, p.id_bytes, m);
    hmz[0] = h_row(p, p.E_in, p.H_in[m], 0, cm, m, idm);
    hmz[1] = h_row(p, p.E_in, p.H_in[N + m], 1, cm, m, idm);
  } else { hmz[0] = hmz[1] = T(0); }
  hmz[2] = T(0);
  auto hval = [&](int e, long long m) -> T {
    if (m == n) return hn[e];
    if (m == n - 1) return hm1[e];
    if (m == n - p.Nx) return hmy[e];
    return hmz[e];
  };
#pragma unroll
  for (int d = 0; d < 3; d++) {
    T ieps = p.mat[9 * id + d];
    T sigma = p.mat[9 * id + 6 + d];
    T eold = p.E_in[d * N + n];
    T jv = j_in(p, d, c, n, step, eold, sigma);
    T curl = e_curl(p, d, c, n, ieps, hval);
    T enew = add(eold, mul(p.dt, sub(curl, mul(ieps, jv))));
    p.E_out[d * N + n] = enew;
    if (p.j_mode == WK_J_ARRAY && p.use_cond) p.J[d * N + n] = mul(sigma, enew);
  }
#pragma unroll
  for (int d = 0; d < 3; d++) p.H_out[d * N + n] = hn[d];
}

template <typename T>
__global__ void k_sigma_e(FitParams<T> p, T* J) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= p.N) return;
  int id = load_id(p.mat_id, p.id_bytes, n);
#pragma unroll
  for (int d = 0; d < 3; d++) J[d * p.N + n] = mul(p.mat[9 * id + 6 + d], p.E_in[d * p.N + n]);
}

template <typename T>
FitParams<T> make_params(const wk_fit_desc* d, int par) {
  FitParams<T> p;
  p.Nx = d->Nx; p.Ny = d->Ny; p.Nz = d->Nz;
  p.NxNy = (long long)d->Nx * d->Ny;
  p.N = p.NxNy * d->Nz;
  p.E_in = (T*)d->E[par]; p.H_in = (T*)d->H[par];
  p.E_out = (T*)d->E[par ^ 1]; p.H_out = (T*)d->H[par ^ 1];
  p.J = (T*)d->J;
  p.j_mode = d->j_mode; p.use_cond = d->use_conductivity;
  p.mat_id = d->mat_id; p.id_bytes = d->id_bytes;
  p.mat = (const T*)d->mat_table;
  p.Lx = (const T*)d->Lx; p.Ly = (const T*)d->Ly; p.Lz = (const T*)d->Lz;
  p.tLx = (const T*)d->tLx; p.tLy = (const T*)d->tLy; p.tLz = (const T*)d->tLz;
  p.iAx = (const T*)d->iAx; p.iAy = (const T*)d->iAy; p.iAz = (const T*)d->iAz;
  p.itAx = (const T*)d->itAx; p.itAy = (const T*)d->itAy; p.itAz = (const T*)d->itAz;
  for (int f = 0; f < 6; f++) { p.pec_face[f] = d->pec_face[f]; p.pmc_face[f] = d->pmc_face[f]; }
  p.has_pec = d->has_pec; p.has_pmc = d->has_pmc; p.h_desc = d->h_sum_desc;
  p.dt = (T)d->dt;
  p.dt64 = d->dt; p.dt32 = (float)d->dt; p.dt_is_f32 = d->dt_is_f32;
  p.beam_on = d->beam_on; p.ixs = d->ixs; p.iys = d->iys;
  p.b_qv = d->b_qv; p.b_v = d->b_v; p.b_v32 = (float)d->b_v; p.b_s0 = d->b_s0;
  p.b_c0 = d->b_c0; p.b_two_sig2 = d->b_two_sig2; p.b_dx = d->b_dx; p.b_dy = d->b_dy;
  p.zc = d->zc;
  p.line_on = d->line_on; p.line_step0 = d->line_step0; p.line_nsteps = d->line_nsteps;
  p.line = (const T*)d->line;
  p.cap_on = d->cap_on; p.cap_i0 = d->cap_i0; p.cap_j0 = d->cap_j0;
  p.cap_ni = d->cap_ni; p.cap_nj = d->cap_nj; p.cap_nt = d->cap_nt; p.cap_step0 = d->cap_step0;
  p.cap = (T*)d->cap;
  p.status = d->status;
  return p;
}

int blocks_for(long long N) { return (int)((N + kThreads - 1) / kThreads); }

template <typename T>
int run_fused(const wk_fit_desc* d, int n_steps, long long step0, cudaStream_t st) {
  int par = d->par;
  for (int s = 0; s < n_steps; s++) {
    FitParams<T> p = make_params<T>(d, par);
    k_fused<T><<<blocks_for(p.N), kThreads, 0, st>>>(p, step0 + s);
    par ^= 1;
  }
  return wk_check_launch("wk_fit_step");
}

template <typename T>
int run_split(const wk_fit_desc* d, int n_steps, long long step0, cudaStream_t st) {
  FitParams<T> p = make_params<T>(d, d->par);
  p.E_out = p.E_in; p.H_out = p.H_in;   // in place
  for (int s = 0; s < n_steps; s++) {
    k_h_split<T><<<blocks_for(p.N), kThreads, 0, st>>>(p, step0 + s);
    k_e_split<T><<<blocks_for(p.N), kThreads, 0, st>>>(p, step0 + s);
  }
  return wk_check_launch("wk_fit_step_split");
}

}  // namespace

extern "C" int wk_zero_ghosts(const wk_fit_desc* d, void* stream) {
  int rc = wk_validate_fit(d, "wk_zero_ghosts");
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  long long N = (long long)d->Nx * d->Ny * d->Nz;
  if (d->dtype == WK_F64)
    k_zero_ghosts<double><<<blocks_for(N), kThreads, 0, st>>>(make_params<double>(d, d->par));
  else
    k_zero_ghosts<float><<<blocks_for(N), kThreads, 0, st>>>(make_params<float>(d, d->par));
  return wk_check_launch("wk_zero_ghosts");
}

// Every step in [step0, step0 + n_steps) must index inside the capture and
// line buffers.
static int check_steps(const wk_fit_desc* d, int n_steps, long long step0, const char* where) {
  if (n_steps < 0) return wk_fail(WK_E_RANGE, "%s: n_steps < 0", where);
  if (n_steps == 0) return WK_OK;
  long long last = step0 + n_steps - 1;
  if (d->cap_on && (step0 < d->cap_step0 || last >= d->cap_step0 + d->cap_nt))
    return wk_fail(WK_E_RANGE, "%s: steps [%lld, %lld] outside the capture buffer", where,
                   step0, last);
  if (d->line_on && (step0 < d->line_step0 || last >= d->line_step0 + d->line_nsteps))
    return wk_fail(WK_E_RANGE, "%s: steps [%lld, %lld] outside the line buffer", where,
                   step0, last);
  return WK_OK;
}

extern "C" int wk_fit_step(const wk_fit_desc* d, int n_steps, long long step0, void* stream) {
  int rc = wk_validate_fit(d, "wk_fit_step");
  if (rc) return rc;
  rc = check_steps(d, n_steps, step0, "wk_fit_step");
  if (rc) return rc;
  if (d->E[0] == d->E[1] || d->H[0] == d->H[1])
    return wk_fail(WK_E_MODE, "wk_fit_step: ping-pong buffers must be distinct");
  cudaStream_t st = (cudaStream_t)stream;
  return d->dtype == WK_F64 ? run_fused<double>(d, n_steps, step0, st)
                            : run_fused<float>(d, n_steps, step0, st);
}

extern "C" int wk_fit_step_split(const wk_fit_desc* d, int n_steps, long long step0,
                                 void* stream) {
  int rc = wk_validate_fit(d, "wk_fit_step_split");
  if (rc) return rc;
  rc = check_steps(d, n_steps, step0, "wk_fit_step_split");
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  return d->dtype == WK_F64 ? run_split<double>(d, n_steps, step0, st)
                            : run_split<float>(d, n_steps, step0, st);
}

extern "C" int wk_sigma_e(const wk_fit_desc* d, void* J, void* stream) {
  int rc = wk_validate_fit(d, "wk_sigma_e");
  if (rc) return rc;
  if (!J) return wk_fail(WK_E_NULL, "wk_sigma_e: J is NULL");
  cudaStream_t st = (cudaStream_t)stream;
  long long N = (long long)d->Nx * d->Ny * d->Nz;
  if (d->dtype == WK_F64)
    k_sigma_e<double><<<blocks_for(N), kThreads, 0, st>>>(make_params<double>(d, d->par), (double*)J);
  else
    k_sigma_e<float><<<blocks_for(N), kThreads, 0, st>>>(make_params<float>(d, d->par), (float*)J);
  return wk_check_launch("wk_sigma_e");
}
