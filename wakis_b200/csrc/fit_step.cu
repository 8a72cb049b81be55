// FIT leap-frog step kernels (sm_100a) and their C-ABI launchers.
//
// wk_fit_step       fused step: one pass reads E[par], H[par] and writes
//                   E[par^1], H[par^1] (ping-pong, so neighbouring blocks
//                   always read the old state).
// wk_fit_step_split two in-place passes (H, then E), the schedule of
//                   upstream's _one_step (wakis/solverFIT3D.py:482-503).
#include <vector>

#include "../../include/wakis_b200.h"
#include "abi_internal.h"
#include "fit_common.cuh"
#include "fit_kernels.cuh"

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
// One thread per cell over the whole grid, general row code only.
template <typename T>
__global__ void k_fused(FitParams<T> p, long long step) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= p.N) return;
  fused_cell_general(p, step, n, cell_of(n, p.Nx, p.Ny));
}

template <typename T>
__global__ void k_sigma_e(FitParams<T> p, T* J) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= p.N) return;
  int id = load_id(p.mat_id, p.id_bytes, n);
#pragma unroll
  for (int d = 0; d < 3; d++) J[d * p.N + n] = mul(p.mat[9 * id + 6 + d], p.E_in[d * p.N + n]);
}

int blocks_for(long long N) { return (int)((N + kThreads - 1) / kThreads); }

template <typename T>
int run_fused(const wk_fit_desc* d, int n_steps, long long step0, cudaStream_t st) {
  int par = d->par;
  const bool big = d->Nx >= 5 && d->Ny >= 5 && d->Nz >= 5 && d->Nz - 4 <= 65535 &&
                   (d->Ny - 4 + 1) / 2 <= 65535;
  bool use_tma = d->kernel == WK_KERNEL_TMA;
  if (d->kernel == WK_KERNEL_TMA || (d->kernel == WK_KERNEL_AUTO && big)) {
    FitParams<T> p0 = make_params<T>(d, par);
    FitParams<T> p1 = make_params<T>(d, par ^ 1);
    const bool ok = tma_supported<T>(p0) && tma_supported<T>(p1);
    if (d->kernel == WK_KERNEL_TMA && !ok)
      return wk_fail(WK_E_SHAPE, "wk_fit_step: TMA kernel needs a 16-byte row pitch, dims >= 5");
    use_tma = ok;
  }
  if (use_tma) {
    int s = 0;
    // two steps per launch where k_tma2 applies; an even number of such
    // launches keeps the result in E[par ^ (n_steps & 1)]
    if (d->steps_per_launch == 2 && !d->step_dev && n_steps >= 4 &&
        tma2_supported<T>(make_params<T>(d, par))) {
      const int pairs = (n_steps / 4) * 2;
      for (int q = 0; q < pairs; q++, s += 2) {
        cudaError_t e = launch_tma2<T>(make_params<T>(d, par), step0 + s, st, d->tile_planes);
        if (e != cudaSuccess) return wk_fail(-(int)e, "wk_fit_step: %s", cudaGetErrorString(e));
        par ^= 1;
      }
    }
    for (; s < n_steps; s++) {
      FitParams<T> p = make_params<T>(d, par);
      cudaError_t e = launch_tma<T>(p, step0 + s, st, d->tile_planes, d->tile_rows);
      if (e != cudaSuccess) return wk_fail(-(int)e, "wk_fit_step: %s", cudaGetErrorString(e));
      par ^= 1;
    }
    return wk_check_launch("wk_fit_step");
  }
  if (d->kernel == WK_KERNEL_TWOPASS && !big)
    return wk_fail(WK_E_SHAPE, "wk_fit_step: two-pass kernels need every dimension >= 5");
  if (d->kernel == WK_KERNEL_TWOPASS || (d->kernel == WK_KERNEL_AUTO && big)) {
    // planes per thread: 1 for FP64, 2 for FP32 (fastest measured on B200)
    const int kb = d->tile_planes > 0 ? d->tile_planes : (sizeof(T) == 8 ? 1 : 2);
    for (int s = 0; s < n_steps; s++) {
      FitParams<T> p = make_params<T>(d, par);
      cudaError_t e = launch_two_pass<T>(p, step0 + s, st, kb);
      if (e != cudaSuccess) return wk_fail(-(int)e, "wk_fit_step: %s", cudaGetErrorString(e));
      par ^= 1;
    }
    return wk_check_launch("wk_fit_step");
  }
  if (d->kernel != WK_KERNEL_AUTO && d->kernel != WK_KERNEL_CELL)
    return wk_fail(WK_E_MODE, "wk_fit_step: unknown kernel %d", d->kernel);
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
  const bool big = d->Nx >= 5 && d->Ny >= 5 && d->Nz >= 5 && d->Nz - 4 <= 65535 &&
                   (d->Ny - 4 + 1) / 2 <= 65535;
  if (big && d->kernel != WK_KERNEL_CELL) {
    for (int s = 0; s < n_steps; s++) {
      cudaError_t e = launch_two_pass<T>(p, step0 + s, st, d->tile_planes > 0 ? d->tile_planes : 2);
      if (e != cudaSuccess)
        return wk_fail(-(int)e, "wk_fit_step_split: %s", cudaGetErrorString(e));
    }
    return wk_check_launch("wk_fit_step_split");
  }
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
  if (d->dtype == WK_F32C) return wk_comp_zero_ghosts(d, st);
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
  if (d->step_dev) {
    // device step counter: the capture / line ranges are checked by the
    // kernels; only the schedules that read the counter take it
    const bool big = d->Nx >= 5 && d->Ny >= 5 && d->Nz >= 5;
    const bool sched = d->dtype == WK_F32C || d->kernel == WK_KERNEL_AUTO ||
                       d->kernel == WK_KERNEL_TMA || d->kernel == WK_KERNEL_TWOPASS;
    if (!big || !sched)
      return wk_fail(WK_E_MODE, "wk_fit_step: step_dev needs the TMA or two-pass schedule "
                                "and every dimension >= 5");
    step0 = 0;
  } else {
    rc = check_steps(d, n_steps, step0, "wk_fit_step");
    if (rc) return rc;
  }
  if (d->E[0] == d->E[1] || d->H[0] == d->H[1])
    return wk_fail(WK_E_MODE, "wk_fit_step: ping-pong buffers must be distinct");
  cudaStream_t st = (cudaStream_t)stream;
  if (d->dtype == WK_F32C) return wk_comp_step(d, n_steps, step0, st);
  return d->dtype == WK_F64 ? run_fused<double>(d, n_steps, step0, st)
                            : run_fused<float>(d, n_steps, step0, st);
}

thread_local KernelTimer* g_kernel_timer = nullptr;

namespace {
__global__ void k_counter_add(long long* ctr, long long inc) { *ctr += inc; }
}  // namespace

extern "C" int wk_counter_add(long long* ctr, long long inc, void* stream) {
  if (!ctr) return wk_fail(WK_E_NULL, "wk_counter_add: NULL counter");
  if ((uintptr_t)ctr % sizeof(long long))
    return wk_fail(WK_E_ALIGN, "wk_counter_add: counter not 8-byte aligned");
  k_counter_add<<<1, 1, 0, (cudaStream_t)stream>>>(ctr, inc);
  return wk_check_launch("wk_counter_add");
}

extern "C" int wk_fit_step_timed(const wk_fit_desc* d, int n_steps, long long step0,
                                 void* stream, float* ms_interior, int* n_launches) {
  if (!ms_interior || !n_launches)
    return wk_fail(WK_E_NULL, "wk_fit_step_timed: NULL result pointer");
  *ms_interior = 0.0f;
  *n_launches = 0;
  if (n_steps < 0 || n_steps > 4096)
    return wk_fail(WK_E_RANGE, "wk_fit_step_timed: n_steps must be in [0, 4096]");
  KernelTimer t;
  std::vector<cudaEvent_t> ev(4 * (size_t)n_steps + 2);
  int made = 0;
  cudaError_t ce = cudaSuccess;
  for (; made < (int)ev.size(); made++)
    if ((ce = cudaEventCreate(&ev[made])) != cudaSuccess) break;
  if (made < (int)ev.size()) {
    for (int q = 0; q < made; q++) cudaEventDestroy(ev[q]);
    return wk_fail(-(int)ce, "wk_fit_step_timed: %s", cudaGetErrorString(ce));
  }
  t.ev = ev.data();
  t.cap = (int)ev.size() / 2;
  g_kernel_timer = &t;
  int rc = wk_fit_step(d, n_steps, step0, stream);
  g_kernel_timer = nullptr;
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (rc == WK_OK && e != cudaSuccess)
    rc = wk_fail(-(int)e, "wk_fit_step_timed: %s", cudaGetErrorString(e));
  if (rc == WK_OK && t.err != cudaSuccess)
    rc = wk_fail(-(int)t.err, "wk_fit_step_timed: %s", cudaGetErrorString(t.err));
  float total = 0.0f;
  for (int q = 0; rc == WK_OK && q < t.n; q++) {
    float ms = 0.0f;
    e = cudaEventElapsedTime(&ms, ev[2 * q], ev[2 * q + 1]);
    if (e != cudaSuccess) rc = wk_fail(-(int)e, "wk_fit_step_timed: %s", cudaGetErrorString(e));
    total += ms;
  }
  for (auto& x : ev) cudaEventDestroy(x);
  if (rc == WK_OK) {
    *ms_interior = total;
    *n_launches = t.n;
  }
  return rc;
}

extern "C" int wk_fit_step_split(const wk_fit_desc* d, int n_steps, long long step0,
                                 void* stream) {
  int rc = wk_validate_fit(d, "wk_fit_step_split");
  if (rc) return rc;
  rc = check_steps(d, n_steps, step0, "wk_fit_step_split");
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if (d->dtype == WK_F32C)
    return wk_fail(WK_E_DTYPE, "wk_fit_step_split: WK_F32C runs through wk_fit_step");
  return d->dtype == WK_F64 ? run_split<double>(d, n_steps, step0, st)
                            : run_split<float>(d, n_steps, step0, st);
}

extern "C" int wk_sigma_e(const wk_fit_desc* d, void* J, void* stream) {
  int rc = wk_validate_fit(d, "wk_sigma_e");
  if (rc) return rc;
  if (!J) return wk_fail(WK_E_NULL, "wk_sigma_e: J is NULL");
  cudaStream_t st = (cudaStream_t)stream;
  if (d->dtype == WK_F32C) return wk_comp_sigma_e(d, J, st);
  long long N = (long long)d->Nx * d->Ny * d->Nz;
  if (d->dtype == WK_F64)
    k_sigma_e<double><<<blocks_for(N), kThreads, 0, st>>>(make_params<double>(d, d->par), (double*)J);
  else
    k_sigma_e<float><<<blocks_for(N), kThreads, 0, st>>>(make_params<float>(d, d->par), (float*)J);
  return wk_check_launch("wk_sigma_e");
}
