// Helpers shared by the step kernels: Ez capture, J source of an E row,
// descriptor -> kernel parameter conversion, and the plane-marching kernel
// declaration.
#pragma once
#include "../../include/wakis_b200.h"
#include "fit_common.cuh"

namespace wk {

constexpr int kMarchThreads = 256;
constexpr int kShellBlock = 256;

// Shell decomposition of the two-pass and TMA schedules.  Blocks of 256 threads
// are decoded once per block (32-bit): planes k in {0,1,Nz-2,Nz-1} row by
// row (256 cells of a row per block), then rows j in {0,1,Ny-2,Ny-1} of the
// inner planes, then the columns i in {0,1,Nx-2,Nx-1} of the inner rows (4
// cells x 64 rows per block).  Cells that meet the single-coefficient
// condition take the lean rows; the rest the general row code.
struct ShellGrid {
  int cx, cy;          // 256-cell chunks per row, 64-row chunks per column
  int nbA, nbB, nbC;   // blocks of the three regions
};

inline ShellGrid shell_grid(int Nx, int Ny, int Nz, bool planes_only = false) {
  ShellGrid g;
  g.cx = (Nx + kShellBlock - 1) / kShellBlock;
  g.cy = (Ny - 4 + 63) / 64;
  g.nbA = 4 * Ny * g.cx;
  g.nbB = planes_only ? 0 : 4 * (Nz - 4) * g.cx;
  g.nbC = planes_only ? 0 : g.cy * (Nz - 4);
  return g;
}

__device__ __forceinline__ bool shell_cell_of(const ShellGrid& g, int b, int tid, int Nx, int Ny,
                                              int Nz, Cell& c) {
  if (b < g.nbA) {
    const int r = b / g.cx, ck = b - r * g.cx;
    const int kk = r / Ny;
    c.j = r - kk * Ny;
    c.k = kk < 2 ? kk : Nz - 4 + kk;
    c.i = ck * kShellBlock + tid;
    return c.i < Nx;
  }
  b -= g.nbA;
  if (b < g.nbB) {
    const int r = b / g.cx, ck = b - r * g.cx;
    const int jj = r & 3;
    c.k = 2 + (r >> 2);
    c.j = jj < 2 ? jj : Ny - 4 + jj;
    c.i = ck * kShellBlock + tid;
    return c.i < Nx;
  }
  b -= g.nbB;
  const int r = b / g.cy, cj = b - r * g.cy;
  const int ii = tid & 3;
  c.k = 2 + r;
  c.i = ii < 2 ? ii : Nx - 4 + ii;
  c.j = 2 + cj * 64 + (tid >> 2);
  return c.j <= Ny - 3;
}


template <typename T>
__device__ __forceinline__ void capture(const FitParams<T>& p, Cell c, long long n,
                                        long long step, T ez) {
  int a = c.i - p.cap_i0, b = c.j - p.cap_j0;
  const long long t = step - p.cap_step0;
  if (a >= 0 && a < p.cap_ni && b >= 0 && b < p.cap_nj && t >= 0 && t < p.cap_nt) {
    long long w = (long long)a * p.cap_nj + b;
    p.cap[(w * p.Nz + c.k) * p.cap_nt + t] = ez;
  }
}

// J value entering the E row of component d at cell n (before the update).
template <typename T>
__device__ __forceinline__ T j_in(const FitParams<T>& p, int d, Cell c, long long n,
                                  long long step, T e_old, T sigma) {
  if (d == 2 && c.i == p.ixs && c.j == p.iys) {
    if (p.line_on) {
      const long long t = step - p.line_step0;
      return (t >= 0 && t < p.line_nsteps) ? p.line[t * p.Nz + c.k] : T(0);
    }
    if (p.beam_on) return beam_j(p, step, c.k);
  }
  if (p.j_mode == WK_J_SIGMA_E) return mul(sigma, e_old);
  if (p.j_mode == WK_J_ARRAY) return p.J[(long long)d * p.N + n];
  return T(0);
}

template <typename T>
inline FitParams<T> make_params(const wk_fit_desc* d, int par) {
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
  p.n_mat = d->n_mat;
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
  fast_div_magic((unsigned)d->Nx, &p.nx_mul, &p.nx_shift);
  p.status = d->status;
  p.step_dev = d->step_dev;
  p.faces_clean = d->faces_clean;
  p.wait_ns = d->wait_ns;
  p.steps_per_launch = d->steps_per_launch;
  return p;
}


// Cell of the idx-th shell cell: planes k in {0,1,Nz-2,Nz-1}, then rows
// j in {0,1,Ny-2,Ny-1} of the inner planes, then columns i in
// {0,1,Nx-2,Nx-1} of the inner rows (needs Nx, Ny, Nz >= 5).
__device__ __forceinline__ Cell shell_cell(long long idx, int Nx, int Ny, int Nz) {
  Cell c;
  const long long NxNy = (long long)Nx * Ny;
  const long long A = 4 * NxNy;
  if (idx < A) {
    const int kk = (int)(idx / NxNy);
    const long long rem = idx - kk * NxNy;
    c.k = kk < 2 ? kk : Nz - 4 + kk;
    c.j = (int)(rem / Nx);
    c.i = (int)(rem - (long long)c.j * Nx);
    return c;
  }
  idx -= A;
  const long long B = 4LL * Nx * (Nz - 4);
  if (idx < B) {
    const long long t = idx / Nx;
    c.i = (int)(idx - t * Nx);
    const int jj = (int)(t % 4);
    c.j = jj < 2 ? jj : Ny - 4 + jj;
    c.k = 2 + (int)(t / 4);
    return c;
  }
  idx -= B;
  const int ii = (int)(idx % 4);
  c.i = ii < 2 ? ii : Nx - 4 + ii;
  const long long t = idx / 4;
  c.j = 2 + (int)(t % (Ny - 4));
  c.k = 2 + (int)(t / (Ny - 4));
  return c;
}

// Fused step of one cell with the general row code: the new H of the cell
// and of the three backward neighbours it needs is computed from the old
// state, then the new E of the cell.
template <typename T>
__device__ __forceinline__ void fused_cell_general(const FitParams<T>& p, long long step,
                                                   long long n, Cell c) {
  const long long N = p.N;
  int id = load_id(p.mat_id, p.id_bytes, n);
  if (p.cap_on) capture(p, c, n, step, p.E_in[2 * N + n]);
  T hn[3];
#pragma unroll
  for (int d = 0; d < 3; d++) hn[d] = h_row(p, p.E_in, p.H_in[d * N + n], d, c, n, id);
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
  auto hv = [&](int e, int kind) -> T {
    if (kind == 0) return hn[e];
    if (kind == 1) return hm1[e];
    if (kind == 2) return hmy[e];
    return hmz[e];
  };
#pragma unroll
  for (int d = 0; d < 3; d++) {
    T ieps = p.mat[9 * id + d];
    T sigma = p.mat[9 * id + 6 + d];
    T eold = p.E_in[d * N + n];
    T jv = j_in(p, d, c, n, step, eold, sigma);
    T curl = e_curl_acc(p, d, c, n, ieps, hv);
    T enew = add(eold, mul(p.dt, sub(curl, mul(ieps, jv))));
    p.E_out[d * N + n] = enew;
    if (p.j_mode == WK_J_ARRAY && p.use_cond) p.J[d * N + n] = mul(sigma, enew);
  }
#pragma unroll
  for (int d = 0; d < 3; d++) p.H_out[d * N + n] = hn[d];
}

// Launch the two-pass schedule (H pass, then E pass; interior lean kernels
// and general shell kernels) of one step (fit_fused.cu); needs Nx, Ny, Nz >= 5.
// kb = planes per thread (1, 2 or 4).
template <typename T>
cudaError_t launch_two_pass(const FitParams<T>& p, long long step, cudaStream_t st, int kb);

// Shell of a step whose interior was stepped by a fused kernel: H of the
// shell cells from the old state, then E of the shell cells from the new H
// (fit_fused.cu); needs Nx, Ny, Nz >= 5 and the interior H_out written.
template <typename T>
cudaError_t launch_shell_pair(const FitParams<T>& p, long long step, cudaStream_t st,
                              bool planes_only = false);

// TMA-staged fused step (fit_tma.cu): interior tiles + shell launches.
template <typename T>
bool tma_supported(const FitParams<T>& p);
template <typename T>
cudaError_t launch_tma(const FitParams<T>& p, long long step, cudaStream_t st, int KC,
                       int rows);

// Two steps per launch (fit_tma2.cu): k_tma2 covers grids whose faces are
// all PEC-masked and clean, with J = 0 or sigma*E.
template <typename T>
bool tma2_supported(const FitParams<T>& p);
template <typename T>
cudaError_t launch_tma2(const FitParams<T>& p, long long step, cudaStream_t st, int KC);

}  // namespace wk
