// Plane-marching fused FIT step (sm_100a).
//
// Block (seg, chunk) owns rows j0 = seg*TY .. j0+TY-1 of every plane k in
// [chunk*KC, chunk*KC + KC).  Because upstream's difference operators work
// on flat offsets (+1, +Nx, +Nx*Ny), the owned cells of plane k are one
// contiguous flat range S = [s, s+L), L = rows*Nx, and every neighbour the
// step needs is a fixed flat offset from it:
//   H_new on the extended range [s-Nx, s+L) needs E_old on [s-Nx, s+L+Nx)
//   of plane k (offsets 0, +1, +Nx) and on [s-Nx, s+L) of plane k+1;
//   E_new on S needs H_new of plane k on [s-Nx, s+L) (offsets 0, -1, -Nx)
//   and H_new of plane k-1 on S.
// The block stages E_old of planes k and k+1 in shared memory (a ring of two
// planes), computes H_new on the extended range into shared memory (the halo
// row is recomputed, so no block waits for another), writes H_new and E_new
// of the owned range, and keeps H_new of the owned range for plane k+1.  A
// chunk starting at k0 > 0 first recomputes H_new(k0-1) on its owned range.
// Reads come from the *_in buffers and writes go to the *_out buffers, so
// halo reads always see the old state.
#include "../../include/wakis_b200.h"
#include "abi_internal.h"
#include "fit_common.cuh"
#include "fit_kernels.cuh"

using namespace wk;

namespace wk {

template <typename T>
__global__ void __launch_bounds__(kMarchThreads)
k_march(FitParams<T> p, long long step, int TY, int KC) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* smem = reinterpret_cast<T*>(smem_raw);
  const int Nx = p.Nx, Ny = p.Ny, Nz = p.Nz;
  const long long N = p.N, NxNy = p.NxNy;
  const int j0 = blockIdx.x * TY;
  const int rows = min(TY, Ny - j0);
  const int L = rows * Nx;           // owned cells per plane
  const int LE = L + Nx;             // extended range (owned + halo row)
  const int W = L + 2 * Nx;          // staged E range
  const int Wst = TY * Nx + 2 * Nx;  // smem strides (fixed per launch)
  const int LEst = TY * Nx + Nx;
  const int Lst = TY * Nx;
  T* Eb = smem;                      // [2 planes][3 comps][Wst]
  T* Hs = Eb + 6 * Wst;              // [3][LEst]       H_new(k) extended
  T* Hp = Hs + 3 * LEst;             // [2][Lst]        H_new(k-1) x,y owned
  const int k0 = blockIdx.y * KC;
  const int k1 = min(k0 + KC, Nz);
  const int kstart = k0 > 0 ? k0 - 1 : 0;
  const int T_ = blockDim.x;

  auto load_plane = [&](int kk) {
    T* dst = Eb + (kk & 1) * 3 * Wst;
    const long long base = (long long)kk * NxNy + (long long)j0 * Nx - Nx;
    for (int e = threadIdx.x; e < W; e += T_) {
      const long long q = base + e;
      // the range starts one row before plane kk, so for kk = Nz its first
      // row is the last row of the grid: only the flat bounds decide
      const bool ok = q >= 0 && q < N;
#pragma unroll
      for (int d = 0; d < 3; d++) dst[d * Wst + e] = ok ? p.E_in[d * N + q] : T(0);
    }
  };

  for (int o = threadIdx.x; o < L; o += T_) { Hp[o] = T(0); Hp[Lst + o] = T(0); }
  load_plane(kstart);
  for (int k = kstart; k < k1; k++) {
    const bool prologue = k < k0;
    load_plane(k + 1);
    __syncthreads();
    const T* Ek = Eb + (k & 1) * 3 * Wst;
    const T* Ek1 = Eb + ((k + 1) & 1) * 3 * Wst;
    const long long s = (long long)k * NxNy + (long long)j0 * Nx;

    // ---- H_new(k) on the extended range (owned range only in the prologue)
    for (int e = (prologue ? Nx : 0) + threadIdx.x; e < LE; e += T_) {
      const long long m = s - Nx + e;
      if (m < 0) {
#pragma unroll
        for (int d = 0; d < 3; d++) Hs[d * LEst + e] = T(0);
        continue;
      }
      const int r = fast_div(e, p.nx_mul, p.nx_shift);
      Cell c;
      c.i = e - r * Nx;
      c.j = j0 - 1 + r;
      c.k = k;
      if (c.j < 0) { c.j += Ny; c.k -= 1; }
      const int id = load_id(p.mat_id, p.id_bytes, m);
      T hx = p.H_in[m], hy = p.H_in[N + m], hz = p.H_in[2 * N + m];
      const bool lean = lean_h<T>(c.i, c.j, c.k, Nx, Ny, Nz);
      if (__all_sync(__activemask(), lean)) {
        const T* mt = p.mat + 9 * id;
        const T R0 = mul(p.iAx[c.j + (long long)c.k * Ny], mt[3]);
        const T R1 = mul(p.iAy[c.i + (long long)c.k * Nx], mt[4]);
        const T R2 = mul(p.iAz[c.i + (long long)c.j * Nx], mt[5]);
        h_lean(p.dt, p.h_desc != 0, R0, R1, R2, p.Lx[c.i], p.Ly[c.j], p.Lz[c.k],
               Ek[e], Ek[Wst + e], Ek[2 * Wst + e], Ek[Wst + e + 1], Ek[2 * Wst + e + 1],
               Ek[e + Nx], Ek[2 * Wst + e + Nx], Ek1[e], Ek1[Wst + e], hx, hy, hz);
      } else {
        auto ev = [&](int comp, int kind) -> T {
          if (kind == 3) return Ek1[comp * Wst + e];
          return Ek[comp * Wst + e + (kind == 1 ? 1 : (kind == 2 ? Nx : 0))];
        };
        hx = h_row_acc(p, hx, 0, c, m, id, ev);
        hy = h_row_acc(p, hy, 1, c, m, id, ev);
        hz = h_row_acc(p, hz, 2, c, m, id, ev);
      }
      Hs[e] = hx;
      Hs[LEst + e] = hy;
      Hs[2 * LEst + e] = hz;
      if (!prologue && e >= Nx) {
        p.H_out[m] = hx;
        p.H_out[N + m] = hy;
        p.H_out[2 * N + m] = hz;
      }
    }
    __syncthreads();

    // ---- E_new(k) on the owned range
    if (!prologue) {
      for (int o = threadIdx.x; o < L; o += T_) {
        const long long n = s + o;
        const int e = o + Nx;
        const int r = fast_div(o, p.nx_mul, p.nx_shift);
        Cell c;
        c.i = o - r * Nx;
        c.j = j0 + r;
        c.k = k;
        const int id = load_id(p.mat_id, p.id_bytes, n);
        const T* mt = p.mat + 9 * id;
        if (p.cap_on) capture(p, c, n, step, Ek[2 * Wst + e]);
        T curl[3];
        const bool lean = lean_e<T>(c.i, c.j, c.k, Nx, Ny, Nz);
        if (__all_sync(__activemask(), lean)) {
          const T R0 = mul(mt[0], p.itAx[c.j + (long long)c.k * Ny]);
          const T R1 = mul(mt[1], p.itAy[c.i + (long long)c.k * Nx]);
          const T R2 = mul(mt[2], p.itAz[c.i + (long long)c.j * Nx]);
          e_lean(R0, R1, R2, p.tLx[c.i], p.tLy[c.j], p.tLz[c.k], Hs[e], Hs[LEst + e],
                 Hs[2 * LEst + e], Hs[LEst + e - 1], Hs[2 * LEst + e - 1], Hs[e - Nx],
                 Hs[2 * LEst + e - Nx], Hp[o], Hp[Lst + o], curl[0], curl[1], curl[2]);
        } else {
          auto hv = [&](int comp, int kind) -> T {
            if (kind == 0) return Hs[comp * LEst + e];
            if (kind == 1) return Hs[comp * LEst + e - 1];
            if (kind == 2) return Hs[comp * LEst + e - Nx];
            return Hp[comp * Lst + o];   // n - Nx*Ny (comp 0 or 1)
          };
#pragma unroll
          for (int d = 0; d < 3; d++) curl[d] = e_curl_acc(p, d, c, n, mt[d], hv);
        }
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const T ieps = mt[d];
          const T sigma = mt[6 + d];
          const T eold = Ek[d * Wst + e];
          const T jv = j_in(p, d, c, n, step, eold, sigma);
          const T enew = add(eold, mul(p.dt, sub(curl[d], mul(ieps, jv))));
          p.E_out[d * N + n] = enew;
          if (p.j_mode == WK_J_ARRAY && p.use_cond) p.J[d * N + n] = mul(sigma, enew);
        }
      }
    }
    __syncthreads();
    // H_new(k) of the owned range becomes H_new(k-1) of the next plane
    for (int o = threadIdx.x; o < L; o += T_) {
      Hp[o] = Hs[o + Nx];
      Hp[Lst + o] = Hs[LEst + o + Nx];
    }
    // the next iteration's first __syncthreads orders these copies (and the
    // reads of Ek above) before Hs / this E plane are overwritten
  }
}

template <typename T>
cudaError_t launch_march(const FitParams<T>& p, long long step, int TY, int KC, size_t smem,
                         cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(k_march<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((p.Ny + TY - 1) / TY, (p.Nz + KC - 1) / KC);
  k_march<T><<<grid, kMarchThreads, smem, st>>>(p, step, TY, KC);
  return cudaGetLastError();
}

template cudaError_t launch_march<double>(const FitParams<double>&, long long, int, int, size_t,
                                          cudaStream_t);
template cudaError_t launch_march<float>(const FitParams<float>&, long long, int, int, size_t,
                                         cudaStream_t);

}  // namespace wk
