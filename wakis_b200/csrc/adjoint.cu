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
// by the caller (no cancellation of E' - E in a float state); E0 holds E of
// the listed entries only (ncell per component, as the increments).
// A^T and B0^T are CSR matrices assembled on the host from the same
// coefficient tables the step kernels read (one thread per row; ~4 entries
// per row), in the state dtype.
#include <stdint.h>

#include "../../include/wakis_b200.h"
#include "abi_internal.h"
#include "fit_common.cuh"
#include "fit_kernels.cuh"
#include "tma_util.cuh"

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
    if (use_sigma) gs -= dt * (double)ieps[x] * l * (double)E0[d * ncell + q] * (double)smask[x];
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
// with the signs and offsets of the curl (x: +1, y: +Nx, z: +Nx*Ny).  The
// products are rounded one by one (no fused multiply-add), so that every
// form of these sums gives the same values.
// the cell factor of u_d (itA_d pec_d ieps_d) and of w_d (dt iA_d imu_d pmc_d)
template <typename T, typename L>
__device__ __forceinline__ L adj_fu(const FitParams<T>& p, int d, Cell c, long long n) {
  const int id = load_id(p.mat_id, p.id_bytes, n);
  T f = d == 0 ? p.itAx[c.j + (long long)c.k * p.Ny]
               : (d == 1 ? p.itAy[c.i + (long long)c.k * p.Nx] : p.itAz[c.i + (long long)c.j * p.Nx]);
  if (p.has_pec && !face_val(p.pec_face, d, c.i, c.j, c.k, p.Nx, p.Ny, p.Nz)) f = T(0);
  return mul((L)f, (L)p.mat[9 * id + d]);
}

template <typename T, typename L>
__device__ __forceinline__ L adj_fw(const FitParams<T>& p, int d, Cell c, long long n) {
  const int id = load_id(p.mat_id, p.id_bytes, n);
  T f = d == 0 ? p.iAx[c.j + (long long)c.k * p.Ny]
               : (d == 1 ? p.iAy[c.i + (long long)c.k * p.Nx] : p.iAz[c.i + (long long)c.j * p.Nx]);
  if (p.has_pmc && !face_val(p.pmc_face, d, c.i, c.j, c.k, p.Nx, p.Ny, p.Nz)) f = T(0);
  return mul(mul((L)p.dt, (L)f), (L)p.mat[9 * id + 3 + d]);
}

template <typename T, typename L>
__device__ __forceinline__ L adj_u(const FitParams<T>& p, const L* lamE, int d, Cell c,
                                   long long n) {
  return mul(adj_fu<T, L>(p, d, c, n), lamE[d * p.N + n]);
}

template <typename T, typename L>
__device__ __forceinline__ L adj_w(const FitParams<T>& p, const L* lamH, int d, Cell c,
                                   long long n) {
  return mul(adj_fw<T, L>(p, d, c, n), lamH[d * p.N + n]);
}

// fu[d N + n] and fw[d N + n] of every cell (either may be NULL)
template <typename T, typename L>
__global__ void __launch_bounds__(kAdjThreads)
k_adj_factors(FitParams<T> p, L* fu, L* fw) {
  const long long m = blockIdx.x * (long long)kAdjThreads + threadIdx.x;
  if (m >= p.N) return;
  const Cell c = cell_of(m, p.Nx, p.Ny);
#pragma unroll
  for (int d = 0; d < 3; d++) {
    if (fu) fu[d * p.N + m] = adj_fu<T, L>(p, d, c, m);
    if (fw) fw[d * p.N + m] = adj_fw<T, L>(p, d, c, m);
  }
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
    lamH_out[e * N + m] = add(lamH_in[e * N + m], mul(mul(dt, (L)coltL(p, e, c.i, c.j, c.k)), acc[e]));
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
    lamE_out[e * N + m] = sub(mul(dec, lamE_in[e * N + m]), mul((L)colL(p, e, c.i, c.j, c.k), acc[e]));
  }
}

// Tiled transposes (wk_adj_h_fit / wk_adj_e_fit with the cell factors of
// wk_adj_factors): block (bx, by, bz) owns the cells i in [i0, i0+32),
// j in [j0, j0+8) of the planes [k0, k0+KC) and marches in z, one thread per
// cell.  The products u = fu lamE (H transpose, DIR > 0) or w = fw lamH (E
// transpose, DIR < 0) of a plane are formed once, for the tile plus the
// one-cell halo the stencil reaches (+x/+y for u, -x/-y for w), into a
// 3-slot ring of shared-memory planes; every output then reads its
// neighbours' products there (u of planes k and k+1, w of planes k and k-1)
// with the same expressions, in the same order, as the one-thread-per-cell
// kernels above, which stay as the cross-check (wk_fit_desc.kernel =
// WK_KERNEL_CELL, or no factors).  The factor and adjoint values of the
// thread's own entry are loaded one plane ahead into registers, so that the
// loads of the next plane are in flight while this one is formed and
// written.  A halo entry one past the grid's last column or row holds the
// product of the cell that the flat-offset operators reach there (the next
// row or plane), as plus_x / plus_y / minus_x / minus_y give it.
constexpr int kAX = 32, kAY = 8, kATh = kAX * kAY;
constexpr int kAW = kAX + 1;                       // entry row width
constexpr int kAEnt = kAW * (kAY + 1);             // entries per plane and component
constexpr int kAHalo = kAX + kAY;                  // halo entries per plane

// Source cell of the entry (i, j) of plane q: the cell itself inside the
// grid; one past the last column / row (DIR > 0) or before the first
// (DIR < 0) the flat-offset neighbour of the grid's edge cell; false where
// no cell (the flat index leaves [0, N)) or the entry is not read.
template <int DIR>
__device__ __forceinline__ bool adj_src(int i, int j, int q, int Nx, int Ny, int Nz, Cell& c) {
  if (q < 0 || q >= Nz + (DIR > 0 ? 1 : 0)) return false;
  if (i >= 0 && i < Nx && j >= 0 && j < Ny) {
    c.i = i; c.j = j; c.k = q;
    return q < Nz;
  }
  Cell e;
  if (DIR > 0) {
    if (i == Nx && j >= 0 && j < Ny) { e.i = Nx - 1; e.j = j; e.k = q; c = plus_x(e, Nx, Ny); }
    else if (j == Ny && i >= 0 && i < Nx) { e.i = i; e.j = Ny - 1; e.k = q; c = plus_y(e, Ny); }
    else return false;
    return c.k < Nz;
  }
  if (i == -1 && j >= 0 && j < Ny) { e.i = 0; e.j = j; e.k = q; c = minus_x(e, Nx, Ny); }
  else if (j == -1 && i >= 0 && i < Nx) { e.i = i; e.j = 0; e.k = q; c = minus_y(e, Ny); }
  else return false;
  return c.k >= 0 && c.k < Nz;
}

// Raw inputs of the entries of one plane (the factor and adjoint value of
// the three components) are staged in shared memory by cp.async two planes
// ahead, in a 3-slot ring [slot][value][entry]: values f0 f1 f2 v0 v1 v2;
// entry tid is the thread's own cell, kATh + tid its halo entry.  Each
// thread stages and reads only its own entries.
constexpr int kAStage = kATh + kAHalo;             // staged entries per plane
constexpr int kASlots = 3;

// stage the entry (i, j) of plane q into dst[0 .. 5 kAStage) (zero-filled
// where adj_src gives no cell)
template <int DIR, typename L>
__device__ __forceinline__ void adj_stage(const L* fac, const L* lam, int i, int j, int q, int Nx,
                                          int Ny, int Nz, long long N, L* dst) {
  Cell c;
  const bool v = adj_src<DIR>(i, j, q, Nx, Ny, Nz, c);
  const long long n = v ? c.i + (long long)c.j * Nx + (long long)c.k * Nx * (long long)Ny : 0;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    cp_async<sizeof(L)>(dst + d * kAStage, v ? fac + d * N + n : fac, v);
    cp_async<sizeof(L)>(dst + (3 + d) * kAStage, v ? lam + d * N + n : lam, v);
  }
}

// products of a staged entry into the plane slot (entry e)
template <typename L>
__device__ __forceinline__ void adj_put(const L* src, L* slot, int e) {
#pragma unroll
  for (int d = 0; d < 3; d++) slot[d * kAEnt + e] = mul(src[d * kAStage], src[(3 + d) * kAStage]);
}

template <typename L>
constexpr int adj_tile_smem() {
  return (kASlots * 3 * kAEnt + kASlots * 6 * kAStage) * (int)sizeof(L);
}

// DIR > 0: xout = xin + dt tL pmc (sum of u), lam = lamE (wk_adj_h_fit);
// DIR < 0: xout = decay xin - L pec (sum of w), lam = lamH (wk_adj_e_fit).
template <typename T, typename L, int DIR>
__global__ void __launch_bounds__(kATh, 3)
k_adj_tile(FitParams<T> p, const L* __restrict__ fac, const L* __restrict__ lam, const L* xin,
           const L* __restrict__ decay, L* xout, int KC) {
  extern __shared__ __align__(16) unsigned char adj_sm[];
  L* S = reinterpret_cast<L*>(adj_sm);             // [kASlots][3][kAEnt] products
  L* R = S + kASlots * 3 * kAEnt;                  // [kASlots][6][kAStage] staged inputs
  constexpr int o = DIR > 0 ? 0 : 1;               // entry of tile cell (0, 0)
  const int Nx = p.Nx, Ny = p.Ny, Nz = p.Nz;
  const long long N = p.N;
  const int i0 = blockIdx.x * kAX, j0 = blockIdx.y * kAY;
  const int k0 = blockIdx.z * KC, k1 = min(k0 + KC, Nz);
  const int tid = threadIdx.x, a = tid & (kAX - 1), b = tid / kAX;
  const int i = i0 + a, j = j0 + b;
  const bool own = i < Nx && j < Ny;
  const int e0 = (b + o) * kAW + a + o;
  // the halo entry of threads tid < kAHalo: kAY of the x halo column, then
  // kAX of the y halo row
  const bool halo = tid < kAHalo;
  const int ha = tid < kAY ? (DIR > 0 ? kAX : -1) : tid - kAY;
  const int hb = tid < kAY ? tid : (DIR > 0 ? kAY : -1);
  const int he = (hb + o) * kAW + ha + o;
  // plane p0 + t is staged as group t into ring slot t % 3 (t = 0 .. n,
  // n = k1 - k0); its products go into plane slot t % 3 at iteration t - 1
  // (slot 0 before the march): u(k0 + t) or w(k0 - 1 + t)
  const int p0 = DIR > 0 ? k0 : k0 - 1;
  const int n = k1 - k0;
  auto stage = [&](int t) {
    if (t <= n) {
      L* dst = R + (t % kASlots) * 6 * kAStage;
      adj_stage<DIR>(fac, lam, i, j, p0 + t, Nx, Ny, Nz, N, dst + tid);
      if (halo) adj_stage<DIR>(fac, lam, i0 + ha, j0 + hb, p0 + t, Nx, Ny, Nz, N, dst + kATh + tid);
    }
    cp_async_commit();   // one group per plane (empty past the last one)
  };
  auto put = [&](int t, L* slot) {
    const L* src = R + (t % kASlots) * 6 * kAStage;
    adj_put(src + tid, slot, e0);
    if (halo) adj_put(src + kATh + tid, slot, he);
  };
  stage(0);
  stage(1);
  stage(2);
  cp_async_wait<2>();                              // group 0 (this thread's entries)
  put(0, S);
  int sa = 0;                                      // plane slot of plane p0 + it
  for (int k = k0; k < k1; k++) {
    const int it = k - k0;
    const int sb = sa == 2 ? 0 : sa + 1;           // plane slot of plane p0 + it + 1
    const long long m = i + (long long)j * Nx + (long long)k * p.NxNy;
    L xi[3], dc[3];
#pragma unroll
    for (int e = 0; e < 3; e++) {
      xi[e] = own ? xin[e * N + m] : L(0);
      dc[e] = (DIR < 0 && own && decay) ? decay[e * N + m] : L(1);
    }
    cp_async_wait<1>();                            // group it + 1
    put(it + 1, S + sb * 3 * kAEnt);
    // the ring slot of group it was read at iteration it - 1, before the
    // barrier that ended it: stage group it + 3 there
    stage(it + 3);
    __syncthreads();
    if (own) {
      if (DIR > 0) {
        const L* uc = S + sa * 3 * kAEnt;          // u(k)
        const L* un = S + sb * 3 * kAEnt;          // u(k+1)
        const L u0 = uc[e0], u1 = uc[kAEnt + e0], u2 = uc[2 * kAEnt + e0];
        const L u0y = uc[e0 + kAW], u2y = uc[2 * kAEnt + e0 + kAW];
        const L u1x = uc[kAEnt + e0 + 1], u2x = uc[2 * kAEnt + e0 + 1];
        const L u0z = un[e0], u1z = un[kAEnt + e0];
        const L acc[3] = {u1 - u1z + u2y - u2, u0z - u0 - u2x + u2, u0 - u0y + u1x - u1};
        const L dt = (L)p.dt;
#pragma unroll
        for (int e = 0; e < 3; e++)
          xout[e * N + m] = add(xi[e], mul(mul(dt, (L)coltL(p, e, i, j, k)), acc[e]));
      } else {
        const L* wc = S + sb * 3 * kAEnt;          // w(k)
        const L* wp = S + sa * 3 * kAEnt;          // w(k-1)
        const L w0 = wc[e0], w1 = wc[kAEnt + e0], w2 = wc[2 * kAEnt + e0];
        const L w0y = wc[e0 - kAW], w2y = wc[2 * kAEnt + e0 - kAW];
        const L w1x = wc[kAEnt + e0 - 1], w2x = wc[2 * kAEnt + e0 - 1];
        const L w0z = wp[e0], w1z = wp[kAEnt + e0];
        const L acc[3] = {w1z - w1 + w2 - w2y, w0 - w0z - w2 + w2x, w0y - w0 + w1 - w1x};
#pragma unroll
        for (int e = 0; e < 3; e++)
          xout[e * N + m] = sub(mul(dc[e], xi[e]), mul((L)colL(p, e, i, j, k), acc[e]));
      }
    }
    sa = sb;
  }
  cp_async_wait<0>();                              // no copy outlives the block
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
// Planes per block of the tiled transposes: enough blocks for about two
// waves of 148 SMs x 3 resident blocks, and at least 8 planes so that the
// plane formed before the march stays a small share.
dim3 adj_tile_grid(const wk_fit_desc* d, int* KC) {
  const int gx = (d->Nx + kAX - 1) / kAX, gy = (d->Ny + kAY - 1) / kAY;
  const long long tiles = (long long)gx * gy;
  const long long want = (2LL * 148 * 3 + tiles - 1) / tiles;
  int kc = (int)((d->Nz + want - 1) / want);
  if (kc < 8) kc = 8;
  if (kc > d->Nz) kc = d->Nz;
  *KC = kc;
  return dim3(gx, gy, (d->Nz + kc - 1) / kc);
}

template <typename T, typename L>
cudaError_t adj_fit_run(const wk_fit_desc* d, const FitParams<T>& p, int which, const void* fac,
                        const void* a, const void* b, const void* decay, void* out,
                        cudaStream_t st) {
  const long long N = (long long)d->Nx * d->Ny * d->Nz;
  if (d->kernel == WK_KERNEL_CELL || !fac) {
    if (which == 0)
      k_adj_h_fit<T, L><<<blocks(N), kAdjThreads, 0, st>>>(p, (const L*)a, (const L*)b, (L*)out);
    else
      k_adj_e_fit<T, L><<<blocks(N), kAdjThreads, 0, st>>>(p, (const L*)a, (const L*)b,
                                                             (const L*)decay, (L*)out);
    return cudaSuccess;
  }
  int KC;
  const dim3 grid = adj_tile_grid(d, &KC);
  constexpr int smem = adj_tile_smem<L>();
  // the dynamic shared memory above 48 KB, once per kernel and device
  static bool attr[2][64];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!attr[which][dev]) {
    e = which == 0
        ? cudaFuncSetAttribute(k_adj_tile<T, L, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               smem)
        : cudaFuncSetAttribute(k_adj_tile<T, L, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               smem);
    if (e != cudaSuccess) return e;
    attr[which][dev] = true;
  }
  if (which == 0)
    k_adj_tile<T, L, 1><<<grid, kATh, smem, st>>>(p, (const L*)fac, (const L*)a, (const L*)b,
                                                  nullptr, (L*)out, KC);
  else
    k_adj_tile<T, L, -1><<<grid, kATh, smem, st>>>(p, (const L*)fac, (const L*)a, (const L*)b,
                                                   (const L*)decay, (L*)out, KC);
  return cudaSuccess;
}

template <typename L>
int adj_fit_launch(const wk_fit_desc* d, int which, const void* fac, const void* a,
                   const void* b, const void* decay, void* out, cudaStream_t st) {
  const bool coef64 = d->dtype == WK_F64 || d->dtype == WK_F32C;
  const cudaError_t e =
      coef64 ? adj_fit_run<double, L>(d, make_params<double>(d, d->par), which, fac, a, b,
                                      decay, out, st)
             : adj_fit_run<float, L>(d, make_params<float>(d, d->par), which, fac, a, b, decay,
                                     out, st);
  return e == cudaSuccess ? WK_OK : -(int)e;
}

int adj_fit(const wk_fit_desc* d, int dtype, int which, const void* fac, const void* a,
            const void* b, const void* decay, void* out, void* stream, const char* where) {
  int rc = wk_validate_fit(d, where);
  if (rc) return rc;
  if (dtype != WK_F64 && dtype != WK_F32) return wk_fail(WK_E_DTYPE, "%s: dtype", where);
  if (!a || !b || !out) return wk_fail(WK_E_NULL, "%s: NULL pointer", where);
  if ((long long)d->Nx * d->Ny * d->Nz >= (1LL << 31))
    return wk_fail(WK_E_SHAPE, "%s: more than 2^31 cells", where);
  cudaStream_t st = (cudaStream_t)stream;
  rc = dtype == WK_F64 ? adj_fit_launch<double>(d, which, fac, a, b, decay, out, st)
                       : adj_fit_launch<float>(d, which, fac, a, b, decay, out, st);
  if (rc) return wk_fail(rc, "%s: %s", where, cudaGetErrorString((cudaError_t)-rc));
  return wk_check_launch(where);
}

template <typename L>
void adj_factors_launch(const wk_fit_desc* d, void* fu, void* fw, cudaStream_t st) {
  const long long N = (long long)d->Nx * d->Ny * d->Nz;
  if (d->dtype == WK_F64 || d->dtype == WK_F32C)
    k_adj_factors<double, L><<<blocks(N), kAdjThreads, 0, st>>>(make_params<double>(d, d->par),
                                                                (L*)fu, (L*)fw);
  else
    k_adj_factors<float, L><<<blocks(N), kAdjThreads, 0, st>>>(make_params<float>(d, d->par),
                                                               (L*)fu, (L*)fw);
}
}  // namespace

extern "C" int wk_adj_factors(const wk_fit_desc* d, int dtype, void* fu, void* fw,
                              void* stream) {
  const char* where = "wk_adj_factors";
  int rc = wk_validate_fit(d, where);
  if (rc) return rc;
  if (dtype != WK_F64 && dtype != WK_F32) return wk_fail(WK_E_DTYPE, "%s: dtype", where);
  if (!fu && !fw) return wk_fail(WK_E_NULL, "%s: fu and fw are NULL", where);
  if ((long long)d->Nx * d->Ny * d->Nz >= (1LL << 31))
    return wk_fail(WK_E_SHAPE, "%s: more than 2^31 cells", where);
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == WK_F64) adj_factors_launch<double>(d, fu, fw, st);
  else adj_factors_launch<float>(d, fu, fw, st);
  return wk_check_launch(where);
}

extern "C" int wk_adj_h_fit(const wk_fit_desc* d, int dtype, const void* fu, const void* lamE,
                            const void* lamH_in, void* lamH_out, void* stream) {
  return adj_fit(d, dtype, 0, fu, lamE, lamH_in, nullptr, lamH_out, stream, "wk_adj_h_fit");
}

extern "C" int wk_adj_e_fit(const wk_fit_desc* d, int dtype, const void* fw, const void* lamH,
                            const void* lamE_in, const void* decay, void* lamE_out,
                            void* stream) {
  return adj_fit(d, dtype, 1, fw, lamH, lamE_in, decay, lamE_out, stream, "wk_adj_e_fit");
}
