// Two-pass FIT step without shared memory (sm_100a), and the shell launches.
//
// The two-pass schedule (H pass, then E pass) updates the interior cells
// (2 <= i <= Nx-3, 2 <= j <= Ny-3, 2 <= k <= Nz-3: no flat-offset wrap and
// no face mask reaches any row they need) with single-coefficient rows, and
// the two-cell shell with the general row code (masks, wraps, grid edges).
// It serves grids the TMA kernel cannot take and is the cross-check of the
// TMA schedule.  The shell kernels here also close the TMA step when a face
// is not PEC-masked.
#include "../../include/wakis_b200.h"
#include "abi_internal.h"
#include "fit_common.cuh"
#include "fit_kernels.cuh"

namespace wk {

constexpr int kShellThreads = 256;

// ------------------------------------------------------------ two passes --
// H pass then E pass over the interior (lean rows) and the shell (general
// rows).  The H pass reads E_in, H_in and writes H_out; the E pass reads
// E_in and the new H (H_out) and writes E_out; H_out may alias H_in and
// E_out may alias E_in (each cell reads only its own old value of the field
// it writes).
constexpr int kPassX = 128, kPassY = 2;

// Each thread updates KB consecutive planes of its (i, j) column; all
// loads of the KB cells are issued before any arithmetic, so a thread keeps
// KB times more bytes in flight.  Neighbour offsets are 32-bit (Nx*Ny < 2^31)
// from per-thread base pointers, and the material table is staged in shared
// memory when it is small (mat_smem = its element count, else 0).
// Resident blocks requested per SM (register cap) for KB planes per thread.
constexpr int pass_min_blocks(size_t bytes, int kb) {
  return kb == 1 ? (bytes == 8 ? 5 : 6) : (kb == 2 ? 3 : 2);
}

template <typename T>
__device__ __forceinline__ const T* stage_table(const FitParams<T>& p, int mat_smem, T* sm) {
  if (mat_smem == 0) return p.mat;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  for (int q = tid; q < mat_smem; q += blockDim.x * blockDim.y) sm[q] = p.mat[q];
  __syncthreads();
  return sm;
}

template <typename T, int KB>
__global__ void __launch_bounds__(kPassX * kPassY, pass_min_blocks(sizeof(T), KB))
k_h_pass(FitParams<T> p, int mat_smem) {
  extern __shared__ __align__(16) unsigned char pass_smem[];
  const T* mat = stage_table(p, mat_smem, reinterpret_cast<T*>(pass_smem));
  const int i = 2 + blockIdx.x * kPassX + threadIdx.x;
  const int j = 2 + blockIdx.y * kPassY + threadIdx.y;
  const int k0 = 2 + blockIdx.z * KB;
  if (i > p.Nx - 3 || j > p.Ny - 3) return;
  const int nk = min(KB, p.Nz - 2 - k0);
  const long long N = p.N;
  const int sy = p.Nx, sz = (int)p.NxNy;
  const long long n0 = i + (long long)j * sy + (long long)k0 * sz;
  const T* ex = p.E_in + n0;
  const T* ey = p.E_in + N + n0;
  const T* ez = p.E_in + 2 * N + n0;
  const T* hx = p.H_in + n0;
  const T* hy = p.H_in + N + n0;
  const T* hz = p.H_in + 2 * N + n0;
  T e0[KB][3], ep1[KB][2], epy[KB][2], epz[KB][2], h[KB][3];
  int id[KB];
#pragma unroll
  for (int q = 0; q < KB; q++) {
    if (q < nk) {
      const int o = q * sz;
      id[q] = load_id(p.mat_id, p.id_bytes, n0 + o);
      e0[q][0] = ex[o]; e0[q][1] = ey[o]; e0[q][2] = ez[o];
      ep1[q][0] = ey[o + 1]; ep1[q][1] = ez[o + 1];
      epy[q][0] = ex[o + sy]; epy[q][1] = ez[o + sy];
      epz[q][0] = ex[o + sz]; epz[q][1] = ey[o + sz];
      h[q][0] = hx[o]; h[q][1] = hy[o]; h[q][2] = hz[o];
    }
  }
  const T iAz = p.iAz[i + j * sy];
  const T Lx = p.Lx[i], Ly = p.Ly[j];
  T* hxo = p.H_out + n0;
  T* hyo = p.H_out + N + n0;
  T* hzo = p.H_out + 2 * N + n0;
#pragma unroll
  for (int q = 0; q < KB; q++) {
    if (q < nk) {
      const int k = k0 + q;
      const int o = q * sz;
      const T* m0 = mat + 9 * id[q];
      const T R0 = mul(p.iAx[j + k * p.Ny], m0[3]);
      const T R1 = mul(p.iAy[i + k * sy], m0[4]);
      const T R2 = mul(iAz, m0[5]);
      h_lean(p.dt, p.h_desc != 0, R0, R1, R2, Lx, Ly, p.Lz[k], e0[q][0], e0[q][1], e0[q][2],
             ep1[q][0], ep1[q][1], epy[q][0], epy[q][1], epz[q][0], epz[q][1], h[q][0], h[q][1],
             h[q][2]);
      hxo[o] = h[q][0];
      hyo[o] = h[q][1];
      hzo[o] = h[q][2];
    }
  }
}

template <typename T, int KB>
__global__ void __launch_bounds__(kPassX * kPassY, pass_min_blocks(sizeof(T), KB))
k_e_pass(FitParams<T> p, long long step, int mat_smem) {
  step = step_index(p, step);
  extern __shared__ __align__(16) unsigned char pass_smem[];
  const T* mat = stage_table(p, mat_smem, reinterpret_cast<T*>(pass_smem));
  const int i = 2 + blockIdx.x * kPassX + threadIdx.x;
  const int j = 2 + blockIdx.y * kPassY + threadIdx.y;
  const int k0 = 2 + blockIdx.z * KB;
  if (i > p.Nx - 3 || j > p.Ny - 3) return;
  const int nk = min(KB, p.Nz - 2 - k0);
  const long long N = p.N;
  const int sy = p.Nx, sz = (int)p.NxNy;
  const long long n0 = i + (long long)j * sy + (long long)k0 * sz;
  const T* hx = p.H_out + n0;
  const T* hy = p.H_out + N + n0;
  const T* hz = p.H_out + 2 * N + n0;
  const T* exi = p.E_in + n0;
  T h0[KB][3], hm1[KB][2], hmy[KB][2], hmz[KB][2], eold[KB][3];
  int id[KB];
#pragma unroll
  for (int q = 0; q < KB; q++) {
    if (q < nk) {
      const int o = q * sz;
      id[q] = load_id(p.mat_id, p.id_bytes, n0 + o);
      h0[q][0] = hx[o]; h0[q][1] = hy[o]; h0[q][2] = hz[o];
      hm1[q][0] = hy[o - 1]; hm1[q][1] = hz[o - 1];
      hmy[q][0] = hx[o - sy]; hmy[q][1] = hz[o - sy];
      hmz[q][0] = hx[o - sz]; hmz[q][1] = hy[o - sz];
      eold[q][0] = exi[o]; eold[q][1] = exi[N + o]; eold[q][2] = exi[2 * N + o];
    }
  }
  const T itAz = p.itAz[i + j * sy];
  const T tLx = p.tLx[i], tLy = p.tLy[j];
#pragma unroll
  for (int q = 0; q < KB; q++) {
    if (q < nk) {
      const int k = k0 + q;
      const long long n = n0 + q * (long long)sz;
      const T* m0 = mat + 9 * id[q];
      const T R0 = mul(m0[0], p.itAx[j + k * p.Ny]);
      const T R1 = mul(m0[1], p.itAy[i + k * sy]);
      const T R2 = mul(m0[2], itAz);
      T curl[3];
      e_lean(R0, R1, R2, tLx, tLy, p.tLz[k], h0[q][0], h0[q][1], h0[q][2], hm1[q][0],
             hm1[q][1], hmy[q][0], hmy[q][1], hmz[q][0], hmz[q][1], curl[0], curl[1], curl[2]);
      Cell c;
      c.i = i; c.j = j; c.k = k;
      if (p.cap_on) capture(p, c, n, step, eold[q][2]);
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const T ieps = m0[d], sigma = m0[6 + d];
        const T jv = j_in(p, d, c, n, step, eold[q][d], sigma);
        const T enew = add(eold[q][d], mul(p.dt, sub(curl[d], mul(ieps, jv))));
        p.E_out[d * N + n] = enew;
        if (p.j_mode == WK_J_ARRAY && p.use_cond) p.J[d * N + n] = mul(sigma, enew);
      }
    }
  }
}

// Shell launches of the two-pass and TMA schedules (decomposition in
// fit_kernels.cuh: ShellGrid).
template <typename T>
__global__ void __launch_bounds__(kShellThreads) k_h_shell(FitParams<T> p, ShellGrid g) {
  Cell c;
  if (!shell_cell_of(g, blockIdx.x, threadIdx.x, p.Nx, p.Ny, p.Nz, c)) return;
  const int Nx = p.Nx;
  const long long N = p.N, NxNy = p.NxNy;
  const long long n = c.i + (long long)c.j * Nx + (long long)c.k * NxNy;
  const int id = load_id(p.mat_id, p.id_bytes, n);
  T h[3];
  if (lean_h<T>(c.i, c.j, c.k, Nx, p.Ny, p.Nz)) {
    const T* E = p.E_in;
    const T* m0 = p.mat + 9 * id;
    const T R0 = mul(p.iAx[c.j + (long long)c.k * p.Ny], m0[3]);
    const T R1 = mul(p.iAy[c.i + (long long)c.k * Nx], m0[4]);
    const T R2 = mul(p.iAz[c.i + (long long)c.j * Nx], m0[5]);
    h[0] = p.H_in[n];
    h[1] = p.H_in[N + n];
    h[2] = p.H_in[2 * N + n];
    h_lean(p.dt, p.h_desc != 0, R0, R1, R2, p.Lx[c.i], p.Ly[c.j], p.Lz[c.k], E[n], E[N + n],
           E[2 * N + n], E[N + n + 1], E[2 * N + n + 1], E[n + Nx], E[2 * N + n + Nx],
           E[n + NxNy], E[N + n + NxNy], h[0], h[1], h[2]);
  } else {
#pragma unroll
    for (int d = 0; d < 3; d++) h[d] = h_row(p, p.E_in, p.H_in[d * N + n], d, c, n, id);
  }
#pragma unroll
  for (int d = 0; d < 3; d++) p.H_out[d * N + n] = h[d];
}

template <typename T>
__global__ void __launch_bounds__(kShellThreads) k_e_shell(FitParams<T> p, long long step,
                                                            ShellGrid g) {
  step = step_index(p, step);
  Cell c;
  if (!shell_cell_of(g, blockIdx.x, threadIdx.x, p.Nx, p.Ny, p.Nz, c)) return;
  const int Nx = p.Nx;
  const long long N = p.N, NxNy = p.NxNy;
  const long long n = c.i + (long long)c.j * Nx + (long long)c.k * NxNy;
  const int id = load_id(p.mat_id, p.id_bytes, n);
  const T* Hn = p.H_out;
  if (p.cap_on) capture(p, c, n, step, p.E_in[2 * N + n]);
  T curl[3];
  const bool lean = lean_e<T>(c.i, c.j, c.k, Nx, p.Ny, p.Nz);
  if (lean) {
    const T* m0 = p.mat + 9 * id;
    const T R0 = mul(m0[0], p.itAx[c.j + (long long)c.k * p.Ny]);
    const T R1 = mul(m0[1], p.itAy[c.i + (long long)c.k * Nx]);
    const T R2 = mul(m0[2], p.itAz[c.i + (long long)c.j * Nx]);
    e_lean(R0, R1, R2, p.tLx[c.i], p.tLy[c.j], p.tLz[c.k], Hn[n], Hn[N + n], Hn[2 * N + n],
           Hn[N + n - 1], Hn[2 * N + n - 1], Hn[n - Nx], Hn[2 * N + n - Nx], Hn[n - NxNy],
           Hn[N + n - NxNy], curl[0], curl[1], curl[2]);
  }
  auto hval = [&](int e, long long m) -> T { return Hn[e * N + m]; };
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const T ieps = p.mat[9 * id + d], sigma = p.mat[9 * id + 6 + d];
    const T eold = p.E_in[d * N + n];
    const T jv = j_in(p, d, c, n, step, eold, sigma);
    const T cu = lean ? curl[d] : e_curl(p, d, c, n, ieps, hval);
    const T enew = add(eold, mul(p.dt, sub(cu, mul(ieps, jv))));
    p.E_out[d * N + n] = enew;
    if (p.j_mode == WK_J_ARRAY && p.use_cond) p.J[d * N + n] = mul(sigma, enew);
  }
}

template <typename T, int KB>
void two_pass_kb(const FitParams<T>& p, long long step, cudaStream_t st) {
  const ShellGrid sg = shell_grid(p.Nx, p.Ny, p.Nz);
  const unsigned sb = (unsigned)(sg.nbA + sg.nbB + sg.nbC);
  dim3 blk(kPassX, kPassY);
  dim3 grid((p.Nx - 4 + kPassX - 1) / kPassX, (p.Ny - 4 + kPassY - 1) / kPassY,
            (p.Nz - 4 + KB - 1) / KB);
  const int mat_smem = p.n_mat * 9 <= 1024 ? p.n_mat * 9 : 0;
  const size_t smem = (size_t)mat_smem * sizeof(T);
  timer_begin(st);
  k_h_pass<T, KB><<<grid, blk, smem, st>>>(p, mat_smem);
  timer_end(st);
  k_h_shell<T><<<sb, kShellThreads, 0, st>>>(p, sg);
  timer_begin(st);
  k_e_pass<T, KB><<<grid, blk, smem, st>>>(p, step, mat_smem);
  timer_end(st);
  k_e_shell<T><<<sb, kShellThreads, 0, st>>>(p, step, sg);
}

template <typename T>
cudaError_t launch_two_pass(const FitParams<T>& p, long long step, cudaStream_t st, int kb) {
  if (kb >= 4)
    two_pass_kb<T, 4>(p, step, st);
  else if (kb == 2)
    two_pass_kb<T, 2>(p, step, st);
  else
    two_pass_kb<T, 1>(p, step, st);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_shell_pair(const FitParams<T>& p, long long step, cudaStream_t st,
                              bool planes_only) {
  const ShellGrid sg = shell_grid(p.Nx, p.Ny, p.Nz, planes_only);
  const unsigned sb = (unsigned)(sg.nbA + sg.nbB + sg.nbC);
  k_h_shell<T><<<sb, kShellThreads, 0, st>>>(p, sg);
  k_e_shell<T><<<sb, kShellThreads, 0, st>>>(p, step, sg);
  return cudaGetLastError();
}

template cudaError_t launch_shell_pair<double>(const FitParams<double>&, long long, cudaStream_t,
                                               bool);
template cudaError_t launch_shell_pair<float>(const FitParams<float>&, long long, cudaStream_t,
                                              bool);

template cudaError_t launch_two_pass<double>(const FitParams<double>&, long long, cudaStream_t,
                                             int);
template cudaError_t launch_two_pass<float>(const FitParams<float>&, long long, cudaStream_t,
                                            int);

}  // namespace wk
