// Fused FIT step without shared memory (sm_100a): interior + shell launches.
//
// One thread per cell reads the old state (E_in, H_in) and writes the new
// state (E_out, H_out), so no block depends on another.  The E row of cell
// n needs the new H at n, n-1, n-Nx and n-Nx*Ny; the thread recomputes those
// H rows itself (3 full rows at n, 2 rows at each backward neighbour), with
// the neighbour E values served by L1/L2 (each E value is read from DRAM
// once per step: ~96 B of DRAM traffic per cell for FP64).
//
// The grid is split in two launches so that every warp runs one code path:
// * k_interior: cells with 2 <= i <= Nx-3, 2 <= j <= Ny-3, 2 <= k <= Nz-3,
//   where no flat-offset wrap and no face mask can reach any row the cell
//   needs; each metric coefficient is formed once (h_lean_* / e_lean).
// * k_shell: the remaining cells (a shell two cells thick), enumerated
//   compactly, with the general row code (masks, wraps, grid edges).
#include "../../include/wakis_b200.h"
#include "abi_internal.h"
#include "fit_common.cuh"
#include "fit_kernels.cuh"

namespace wk {

constexpr int kInteriorX = 128, kInteriorY = 2, kShellThreads = 256;
constexpr int kColumnRows = 4;   // warps (rows j) per block of the column kernel

template <typename T>
__global__ void __launch_bounds__(kInteriorX * kInteriorY)
k_interior(FitParams<T> p, long long step) {
  const int i = 2 + blockIdx.x * kInteriorX + threadIdx.x;
  const int j = 2 + blockIdx.y * kInteriorY + threadIdx.y;
  const int k = 2 + blockIdx.z;
  if (i > p.Nx - 3 || j > p.Ny - 3) return;
  const int Nx = p.Nx, Ny = p.Ny;
  const long long N = p.N, sy = Nx, sz = p.NxNy;
  const long long n = i + j * sy + k * sz;
  const T* __restrict__ ex = p.E_in;
  const T* __restrict__ ey = p.E_in + N;
  const T* __restrict__ ez = p.E_in + 2 * N;
  const T* __restrict__ hx = p.H_in;
  const T* __restrict__ hy = p.H_in + N;
  const T* __restrict__ hz = p.H_in + 2 * N;
  const T dt = p.dt;
  const bool desc = p.h_desc != 0;

  const T* m0 = p.mat + 9 * load_id(p.mat_id, p.id_bytes, n);
  const T* m1 = p.mat + 9 * load_id(p.mat_id, p.id_bytes, n - 1);
  const T* m2 = p.mat + 9 * load_id(p.mat_id, p.id_bytes, n - sy);
  const T* m3 = p.mat + 9 * load_id(p.mat_id, p.id_bytes, n - sz);
  const T Lxi = p.Lx[i], Lxm = p.Lx[i - 1];
  const T Lyj = p.Ly[j], Lym = p.Ly[j - 1];
  const T Lzk = p.Lz[k], Lzm = p.Lz[k - 1];

  // E at n and around it
  const T ex0 = ex[n], ey0 = ey[n], ez0 = ez[n];
  // new H at n (three rows)
  T hxn = hx[n], hyn = hy[n], hzn = hz[n];
  {
    const T R0 = mul(p.iAx[j + (long long)k * Ny], m0[3]);
    const T R1 = mul(p.iAy[i + (long long)k * Nx], m0[4]);
    const T R2 = mul(p.iAz[i + (long long)j * Nx], m0[5]);
    h_lean(dt, desc, R0, R1, R2, Lxi, Lyj, Lzk, ex0, ey0, ez0, ey[n + 1], ez[n + 1],
           ex[n + sy], ez[n + sy], ex[n + sz], ey[n + sz], hxn, hyn, hzn);
  }
  // new H at n-1: y and z rows of cell (i-1, j, k)
  const long long a1 = n - 1;
  const T ex_a1 = ex[a1];
  const T hy1 = h_lean_y(dt, desc, mul(p.iAy[i - 1 + (long long)k * Nx], m1[4]), Lxm, Lzk,
                         ex_a1, ex[a1 + sz], ez[a1], ez0, hy[a1]);
  const T hz1 = h_lean_z(dt, desc, mul(p.iAz[i - 1 + (long long)j * Nx], m1[5]), Lxm, Lyj,
                         ex_a1, ex[a1 + sy], ey[a1], ey0, hz[a1]);
  // new H at n-Nx: x and z rows of cell (i, j-1, k)
  const long long a2 = n - sy;
  const T ey_a2 = ey[a2];
  const T hx2 = h_lean_x(dt, desc, mul(p.iAx[j - 1 + (long long)k * Ny], m2[3]), Lym, Lzk,
                         ey_a2, ey[a2 + sz], ez[a2], ez0, hx[a2]);
  const T hz2 = h_lean_z(dt, desc, mul(p.iAz[i + (long long)(j - 1) * Nx], m2[5]), Lxi, Lym,
                         ex[a2], ex0, ey_a2, ey[a2 + 1], hz[a2]);
  // new H at n-Nx*Ny: x and y rows of cell (i, j, k-1)
  const long long a3 = n - sz;
  const T ez_a3 = ez[a3];
  const T hx3 = h_lean_x(dt, desc, mul(p.iAx[j + (long long)(k - 1) * Ny], m3[3]), Lyj, Lzm,
                         ey[a3], ey0, ez_a3, ez[a3 + sy], hx[a3]);
  const T hy3 = h_lean_y(dt, desc, mul(p.iAy[i + (long long)(k - 1) * Nx], m3[4]), Lxi, Lzm,
                         ex[a3], ex0, ez_a3, ez[a3 + 1], hy[a3]);

  // E at n
  T curl[3];
  {
    const T R0 = mul(m0[0], p.itAx[j + (long long)k * Ny]);
    const T R1 = mul(m0[1], p.itAy[i + (long long)k * Nx]);
    const T R2 = mul(m0[2], p.itAz[i + (long long)j * Nx]);
    e_lean(R0, R1, R2, p.tLx[i], p.tLy[j], p.tLz[k], hxn, hyn, hzn, hy1, hz1, hx2, hz2, hx3,
           hy3, curl[0], curl[1], curl[2]);
  }
  Cell c;
  c.i = i; c.j = j; c.k = k;
  const T eold[3] = {ex0, ey0, ez0};
  if (p.cap_on) capture(p, c, n, step, ez0);
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const T ieps = m0[d], sigma = m0[6 + d];
    const T jv = j_in(p, d, c, n, step, eold[d], sigma);
    const T enew = add(eold[d], mul(dt, sub(curl[d], mul(ieps, jv))));
    p.E_out[d * N + n] = enew;
    if (p.j_mode == WK_J_ARRAY && p.use_cond) p.J[d * N + n] = mul(sigma, enew);
  }
  p.H_out[n] = hxn;
  p.H_out[N + n] = hyn;
  p.H_out[2 * N + n] = hzn;
}

// Interior cells, one thread per (i, j) column marching kz planes.  Lane l
// of a warp sits at i = i0 - 1 + l; lanes 1..31 own their cells, lane 0 only
// supplies the new H of (i0-1, j) to lane 1 (shuffle).  Carried from plane
// k-1 to k: E(n) x/y (loaded as E(n+Nx*Ny) one plane earlier), Ey(n-Nx), and
// the new H(n-Nx*Ny) x/y.  The ±1 neighbours come from the adjacent lanes;
// the H rows of (i, j-1) are recomputed.
template <typename T>
__global__ void __launch_bounds__(32 * kColumnRows)
k_column(FitParams<T> p, long long step, int kz) {
  const int lane = threadIdx.x;
  const int i_raw = 2 + blockIdx.x * 31 - 1 + lane;
  const int j = 2 + blockIdx.y * kColumnRows + threadIdx.y;
  const int k0 = 2 + blockIdx.z * kz;
  const int Nx = p.Nx, Ny = p.Ny, Nz = p.Nz;
  if (j > Ny - 3) return;                 // whole warp
  const int k1 = min(k0 + kz, Nz - 2);
  const bool owner = lane >= 1 && i_raw <= Nx - 3;
  const int i = min(i_raw, Nx - 2);       // lanes past the last owner + 1 only feed shuffles
  const long long N = p.N, sy = Nx, sz = p.NxNy;
  const T* __restrict__ ex = p.E_in;
  const T* __restrict__ ey = p.E_in + N;
  const T* __restrict__ ez = p.E_in + 2 * N;
  const T* __restrict__ hx = p.H_in;
  const T* __restrict__ hy = p.H_in + N;
  const T* __restrict__ hz = p.H_in + 2 * N;
  const T dt = p.dt;
  const bool desc = p.h_desc != 0;
  const unsigned FULL = 0xffffffffu;

  // per-column metrics
  const T Lxi = p.Lx[i], Lyj = p.Ly[j], Lym = p.Ly[j - 1];
  const T tLxi = p.tLx[i], tLyj = p.tLy[j];
  const T iAz0 = p.iAz[i + (long long)j * Nx], iAzm = p.iAz[i + (long long)(j - 1) * Nx];
  const T itAz0 = p.itAz[i + (long long)j * Nx];

  // prologue: carried values for plane k0
  long long n = i + j * sy + k0 * sz;
  T exc = ex[n], eyc = ey[n], eymc = ey[n - sy];
  T hxp, hyp;
  {
    const long long a = n - sz;
    const T* m = p.mat + 9 * load_id(p.mat_id, p.id_bytes, a);
    const T ez_a = ez[a];
    hxp = h_lean_x(dt, desc, mul(p.iAx[j + (long long)(k0 - 1) * Ny], m[3]), Lyj,
                   p.Lz[k0 - 1], ey[a], eyc, ez_a, ez[a + sy], hx[a]);
    hyp = h_lean_y(dt, desc, mul(p.iAy[i + (long long)(k0 - 1) * Nx], m[4]), Lxi,
                   p.Lz[k0 - 1], ex[a], exc, ez_a, ez[a + 1], hy[a]);
  }

  for (int k = k0; k < k1; k++, n += sz) {
    const T* m0 = p.mat + 9 * load_id(p.mat_id, p.id_bytes, n);
    const T* m2 = p.mat + 9 * load_id(p.mat_id, p.id_bytes, n - sy);
    const T Lzk = p.Lz[k];
    const T ez0 = ez[n];
    const T ex_pz = ex[n + sz], ey_pz = ey[n + sz];
    const T ex_py = ex[n + sy], ez_py = ez[n + sy];
    const T ex_my = ex[n - sy], ez_my = ez[n - sy];
    const T ey_mypz = ey[n - sy + sz];
    // +1 neighbours from lane + 1 (lane 31 loads its own)
    T ey_p1 = __shfl_down_sync(FULL, eyc, 1);
    T ez_p1 = __shfl_down_sync(FULL, ez0, 1);
    T ey_myp1 = __shfl_down_sync(FULL, eymc, 1);
    if (lane == 31) {
      ey_p1 = ey[n + 1];
      ez_p1 = ez[n + 1];
      ey_myp1 = ey[n - sy + 1];
    }
    // new H at n
    const T hxn = h_lean_x(dt, desc, mul(p.iAx[j + (long long)k * Ny], m0[3]), Lyj, Lzk, eyc,
                           ey_pz, ez0, ez_py, hx[n]);
    const T hyn = h_lean_y(dt, desc, mul(p.iAy[i + (long long)k * Nx], m0[4]), Lxi, Lzk, exc,
                           ex_pz, ez0, ez_p1, hy[n]);
    const T hzn = h_lean_z(dt, desc, mul(iAz0, m0[5]), Lxi, Lyj, exc, ex_py, eyc, ey_p1, hz[n]);
    // new H at n - Nx (cell (i, j-1, k)): x and z rows
    const T hx2 = h_lean_x(dt, desc, mul(p.iAx[j - 1 + (long long)k * Ny], m2[3]), Lym, Lzk,
                           eymc, ey_mypz, ez_my, ez0, hx[n - sy]);
    const T hz2 = h_lean_z(dt, desc, mul(iAzm, m2[5]), Lxi, Lym, ex_my, exc, eymc, ey_myp1,
                           hz[n - sy]);
    // new H at n - 1 from lane - 1
    const T hy1 = __shfl_up_sync(FULL, hyn, 1);
    const T hz1 = __shfl_up_sync(FULL, hzn, 1);
    if (owner) {
      T curl[3];
      const T R0 = mul(m0[0], p.itAx[j + (long long)k * Ny]);
      const T R1 = mul(m0[1], p.itAy[i + (long long)k * Nx]);
      const T R2 = mul(m0[2], itAz0);
      e_lean(R0, R1, R2, tLxi, tLyj, p.tLz[k], hxn, hyn, hzn, hy1, hz1, hx2, hz2, hxp, hyp,
             curl[0], curl[1], curl[2]);
      Cell c;
      c.i = i; c.j = j; c.k = k;
      const T eold[3] = {exc, eyc, ez0};
      if (p.cap_on) capture(p, c, n, step, ez0);
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const T ieps = m0[d], sigma = m0[6 + d];
        const T jv = j_in(p, d, c, n, step, eold[d], sigma);
        const T enew = add(eold[d], mul(dt, sub(curl[d], mul(ieps, jv))));
        p.E_out[d * N + n] = enew;
        if (p.j_mode == WK_J_ARRAY && p.use_cond) p.J[d * N + n] = mul(sigma, enew);
      }
      p.H_out[n] = hxn;
      p.H_out[N + n] = hyn;
      p.H_out[2 * N + n] = hzn;
    }
    exc = ex_pz;
    eyc = ey_pz;
    eymc = ey_mypz;
    hxp = hxn;
    hyp = hyn;
  }
}

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

// ------------------------------------------------------------- z slabs ----
// The two passes run slab by slab along z: H pass of planes [ka, kb), then
// E pass of the same planes, then the next slab.  H(k) needs E_old at k and
// k+1 and E(k) needs H_new at k and k-1, so this order gives the same result
// as two whole-grid passes, while the E pass re-reads the slab's E_in and
// H_out from L2.  One launch per pass per slab: the first blocks are
// interior tiles (single-coefficient rows), the remaining blocks cover the
// slab's shell cells (general rows).
struct SlabInfo {
  int k_int0, n_int;         // interior planes [k_int0, k_int0 + n_int)
  int gx, gy;                // interior tiles per plane (x, y)
  long long nb_int;          // interior blocks
  int F[4], nF;              // full shell planes in the slab
  int lo, n_inner, S_in;     // inner shell planes [lo, lo + n_inner), cells per plane
  long long shell_count;
};

__device__ __forceinline__ Cell slab_shell_cell(long long idx, int Nx, int Ny,
                                                const SlabInfo& s) {
  Cell c;
  const long long NxNy = (long long)Nx * Ny;
  if (idx < s.nF * NxNy) {
    const int f = (int)(idx / NxNy);
    const long long rem = idx - f * NxNy;
    c.k = s.F[f];
    c.j = (int)(rem / Nx);
    c.i = (int)(rem - (long long)c.j * Nx);
    return c;
  }
  idx -= s.nF * NxNy;
  const long long pl = idx / s.S_in;
  int r = (int)(idx - pl * s.S_in);
  c.k = s.lo + (int)pl;
  if (r < 4 * Nx) {
    const int jj = r / Nx;
    c.i = r - jj * Nx;
    c.j = jj < 2 ? jj : Ny - 4 + jj;
    return c;
  }
  r -= 4 * Nx;
  const int ii = r % 4;
  c.i = ii < 2 ? ii : Nx - 4 + ii;
  c.j = 2 + r / 4;
  return c;
}

template <typename T>
__global__ void __launch_bounds__(kPassX * kPassY, pass_min_blocks(sizeof(T), 1))
k_h_slab(FitParams<T> p, SlabInfo s, int mat_smem) {
  extern __shared__ __align__(16) unsigned char pass_smem[];
  const T* mat = stage_table(p, mat_smem, reinterpret_cast<T*>(pass_smem));
  const long long b = blockIdx.x;
  const long long N = p.N;
  if (b < s.nb_int) {
    const int bx = (int)(b % s.gx);
    const long long r = b / s.gx;
    const int by = (int)(r % s.gy);
    const int bz = (int)(r / s.gy);
    const int i = 2 + bx * kPassX + threadIdx.x;
    const int j = 2 + by * kPassY + threadIdx.y;
    const int k = s.k_int0 + bz;
    if (i > p.Nx - 3 || j > p.Ny - 3) return;
    const int sy = p.Nx, sz = (int)p.NxNy;
    const long long n = i + (long long)j * sy + (long long)k * sz;
    const T* ex = p.E_in + n;
    const T* ey = p.E_in + N + n;
    const T* ez = p.E_in + 2 * N + n;
    const T* m0 = mat + 9 * load_id(p.mat_id, p.id_bytes, n);
    T hx = p.H_in[n], hy = p.H_in[N + n], hz = p.H_in[2 * N + n];
    const T R0 = mul(p.iAx[j + k * p.Ny], m0[3]);
    const T R1 = mul(p.iAy[i + k * sy], m0[4]);
    const T R2 = mul(p.iAz[i + j * sy], m0[5]);
    h_lean(p.dt, p.h_desc != 0, R0, R1, R2, p.Lx[i], p.Ly[j], p.Lz[k], ex[0], ey[0], ez[0],
           ey[1], ez[1], ex[sy], ez[sy], ex[sz], ey[sz], hx, hy, hz);
    p.H_out[n] = hx;
    p.H_out[N + n] = hy;
    p.H_out[2 * N + n] = hz;
  } else {
    const long long idx = (b - s.nb_int) * (kPassX * kPassY) + threadIdx.x +
                          threadIdx.y * kPassX;
    if (idx >= s.shell_count) return;
    const Cell c = slab_shell_cell(idx, p.Nx, p.Ny, s);
    const long long n = c.i + (long long)c.j * p.Nx + (long long)c.k * p.NxNy;
    const int id = load_id(p.mat_id, p.id_bytes, n);
    T h[3];
#pragma unroll
    for (int d = 0; d < 3; d++) h[d] = h_row(p, p.E_in, p.H_in[d * N + n], d, c, n, id);
#pragma unroll
    for (int d = 0; d < 3; d++) p.H_out[d * N + n] = h[d];
  }
}

template <typename T>
__global__ void __launch_bounds__(kPassX * kPassY, pass_min_blocks(sizeof(T), 1))
k_e_slab(FitParams<T> p, long long step, SlabInfo s, int mat_smem) {
  extern __shared__ __align__(16) unsigned char pass_smem[];
  const T* mat = stage_table(p, mat_smem, reinterpret_cast<T*>(pass_smem));
  const long long b = blockIdx.x;
  const long long N = p.N;
  if (b < s.nb_int) {
    const int bx = (int)(b % s.gx);
    const long long r = b / s.gx;
    const int by = (int)(r % s.gy);
    const int bz = (int)(r / s.gy);
    const int i = 2 + bx * kPassX + threadIdx.x;
    const int j = 2 + by * kPassY + threadIdx.y;
    const int k = s.k_int0 + bz;
    if (i > p.Nx - 3 || j > p.Ny - 3) return;
    const int sy = p.Nx, sz = (int)p.NxNy;
    const long long n = i + (long long)j * sy + (long long)k * sz;
    const T* hx = p.H_out + n;
    const T* hy = p.H_out + N + n;
    const T* hz = p.H_out + 2 * N + n;
    const T* m0 = mat + 9 * load_id(p.mat_id, p.id_bytes, n);
    const T eold[3] = {p.E_in[n], p.E_in[N + n], p.E_in[2 * N + n]};
    const T R0 = mul(m0[0], p.itAx[j + k * p.Ny]);
    const T R1 = mul(m0[1], p.itAy[i + k * sy]);
    const T R2 = mul(m0[2], p.itAz[i + j * sy]);
    T curl[3];
    e_lean(R0, R1, R2, p.tLx[i], p.tLy[j], p.tLz[k], hx[0], hy[0], hz[0], hy[-1], hz[-1],
           hx[-sy], hz[-sy], hx[-sz], hy[-sz], curl[0], curl[1], curl[2]);
    Cell c;
    c.i = i; c.j = j; c.k = k;
    if (p.cap_on) capture(p, c, n, step, eold[2]);
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const T ieps = m0[d], sigma = m0[6 + d];
      const T jv = j_in(p, d, c, n, step, eold[d], sigma);
      const T enew = add(eold[d], mul(p.dt, sub(curl[d], mul(ieps, jv))));
      p.E_out[d * N + n] = enew;
      if (p.j_mode == WK_J_ARRAY && p.use_cond) p.J[d * N + n] = mul(sigma, enew);
    }
  } else {
    const long long idx = (b - s.nb_int) * (kPassX * kPassY) + threadIdx.x +
                          threadIdx.y * kPassX;
    if (idx >= s.shell_count) return;
    const Cell c = slab_shell_cell(idx, p.Nx, p.Ny, s);
    const long long n = c.i + (long long)c.j * p.Nx + (long long)c.k * p.NxNy;
    const int id = load_id(p.mat_id, p.id_bytes, n);
    const T* Hn = p.H_out;
    auto hval = [&](int e, long long m) -> T { return Hn[e * N + m]; };
    if (p.cap_on) capture(p, c, n, step, p.E_in[2 * N + n]);
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const T ieps = p.mat[9 * id + d], sigma = p.mat[9 * id + 6 + d];
      const T eold = p.E_in[d * N + n];
      const T jv = j_in(p, d, c, n, step, eold, sigma);
      const T curl = e_curl(p, d, c, n, ieps, hval);
      const T enew = add(eold, mul(p.dt, sub(curl, mul(ieps, jv))));
      p.E_out[d * N + n] = enew;
      if (p.j_mode == WK_J_ARRAY && p.use_cond) p.J[d * N + n] = mul(sigma, enew);
    }
  }
}

template <typename T>
cudaError_t launch_slabs(const FitParams<T>& p, long long step, cudaStream_t st, int planes) {
  const int Nx = p.Nx, Ny = p.Ny, Nz = p.Nz;
  const int mat_smem = p.n_mat * 9 <= 1024 ? p.n_mat * 9 : 0;
  const size_t smem = (size_t)mat_smem * sizeof(T);
  const int threads = kPassX * kPassY;
  for (int ka = 0; ka < Nz; ka += planes) {
    const int kb = min(ka + planes, Nz);
    SlabInfo s;
    s.k_int0 = max(ka, 2);
    s.n_int = max(0, min(kb, Nz - 2) - s.k_int0);
    s.gx = (Nx - 4 + kPassX - 1) / kPassX;
    s.gy = (Ny - 4 + kPassY - 1) / kPassY;
    s.nb_int = (long long)s.gx * s.gy * s.n_int;
    s.nF = 0;
    const int full[4] = {0, 1, Nz - 2, Nz - 1};
    for (int f = 0; f < 4; f++)
      if (full[f] >= ka && full[f] < kb) s.F[s.nF++] = full[f];
    s.lo = max(ka, 2);
    s.n_inner = max(0, min(kb, Nz - 2) - s.lo);
    s.S_in = 4 * Nx + 4 * (Ny - 4);
    s.shell_count = (long long)s.nF * Nx * Ny + (long long)s.n_inner * s.S_in;
    const long long blocks = s.nb_int + (s.shell_count + threads - 1) / threads;
    if (blocks == 0) continue;
    dim3 blk(kPassX, kPassY);
    k_h_slab<T><<<(unsigned)blocks, blk, smem, st>>>(p, s, mat_smem);
    k_e_slab<T><<<(unsigned)blocks, blk, smem, st>>>(p, step, s, mat_smem);
  }
  return cudaGetLastError();
}

template cudaError_t launch_slabs<double>(const FitParams<double>&, long long, cudaStream_t,
                                          int);
template cudaError_t launch_slabs<float>(const FitParams<float>&, long long, cudaStream_t, int);

template <typename T>
cudaError_t launch_interior_shell(const FitParams<T>& p, long long step, cudaStream_t st,
                                  int kz) {
  if (kz <= 0) {
    dim3 blk(kInteriorX, kInteriorY);
    dim3 grid((p.Nx - 4 + kInteriorX - 1) / kInteriorX,
              (p.Ny - 4 + kInteriorY - 1) / kInteriorY, p.Nz - 4);
    k_interior<T><<<grid, blk, 0, st>>>(p, step);
  } else {
    dim3 blk(32, kColumnRows);
    dim3 grid((p.Nx - 4 + 30) / 31, (p.Ny - 4 + kColumnRows - 1) / kColumnRows,
              (p.Nz - 4 + kz - 1) / kz);
    k_column<T><<<grid, blk, 0, st>>>(p, step, kz);
  }
  const long long count = p.N - (long long)(p.Nx - 4) * (p.Ny - 4) * (p.Nz - 4);
  k_shell<T><<<(unsigned)((count + kShellThreads - 1) / kShellThreads), kShellThreads, 0, st>>>(
      p, step, count);
  return cudaGetLastError();
}

template cudaError_t launch_interior_shell<double>(const FitParams<double>&, long long,
                                                   cudaStream_t, int);
template cudaError_t launch_interior_shell<float>(const FitParams<float>&, long long,
                                                  cudaStream_t, int);

}  // namespace wk
