// Two leap-frog steps per launch with TMA-staged plane tiles (sm_100a):
// temporal blocking of the fused FIT step.
//
// k_tma2 reads the state (E0, H0) once and writes the state two steps later
// (E2, H2), so each cell's six values cross HBM twice per two steps instead
// of four times.  It covers grids whose six faces all carry the PEC column
// mask (pec, electric or pml faces; the whole grid is tiled, no shell
// launch) while the tangential E on those faces is +0 (wk_fit_desc.
// faces_clean), with J = 0 (non-conductive) or J = sigma*E (conductive).
//
// Block (bx, by, bz) owns the output tile i in [i0, i0+64), j in [j0, j0+8)
// of planes [k0, k0+KC) and marches in z.  The first step is computed on an
// extended tile so that the second step of the tile needs nothing from
// another block (the halo is recomputed, as in overlapped tiling).  With
// ext coordinates (ea, eb) from (i0-2, j0-2):
//   A  H1 = H0 - dt A E0            ea in [0, 67), eb in [0, 11)
//   B  E1 = E0 + dt (B H1 - ieps J) ea in [1, 67), eb in [1, 11)
//   C  H2 = H1 - dt A E1            ea in [1, 66), eb in [1, 10)
//   D  E2 = E1 + dt (B H2 - ieps J) ea in [2, 66), eb in [2, 10) (the tile)
// In z, iteration q runs A(q) and D(q-2) (phase 1), a block barrier, then
// B(q) and C(q-1) (phase 2), a barrier: two barriers per iteration for two
// steps.  E0 of planes q, q+1 and H0 of plane q come by
// cp.async.bulk.tensor (no multicast) into rings of three E and two H
// slots, each completing on its own mbarrier; H1, E1 (two planes) and H2
// live in shared memory, the z-neighbours a thread needs of its own cells
// in registers.  Each half-step uses the same single-coefficient rows
// (h_lean / e_lean), the same rounding and the same summation order as the
// one-step kernels, so the result equals two launches of k_tma value for
// value.  Every mbarrier wait is bounded (wk_fit_desc.wait_ns); on timeout
// the block records it in the status word, waits for its loads and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include "../../include/wakis_b200.h"
#include "abi_internal.h"
#include "fit_common.cuh"
#include "fit_kernels.cuh"
#include "tma_util.cuh"

namespace wk {

namespace t2 {

constexpr int TX = 64, TY = 8;             // output tile
constexpr int YA = TY + 3;                 // ext (H1) domain: 67 x 11
constexpr int W = 68;                      // row stride of the smem planes
constexpr int CS = YA * W;                 // component stride: 748
constexpr int BX = 72;                     // TMA box width (x from i0-4)
constexpr int EBY = YA + 1, HBY = YA;      // E0 box rows 12, H0 box rows 11
constexpr int NES = 3, NHS = 2;            // ring slots
constexpr int kThreads = 384;              // 12 warps
constexpr int kRow = 160;                  // per-plane metric row entries
constexpr int kRows = 4;                   // row ring: planes q-2 .. q+1
constexpr int kMat = 32;                   // materials staged in smem

// per-plane metric row of plane q, ext coordinates:
//   [0, 11)    iAx(j0-2+eb)    [11, 78)  iAy(i0-2+ea)
//   [78, 89)   itAx(j0-2+eb)   [89, 156) itAy(i0-2+ea)
//   156 Lz     157 tLz
constexpr int R_IAX = 0, R_IAY = 11, R_ITAX = 78, R_ITAY = 89, R_LZ = 156, R_TLZ = 157;

template <typename T>
struct Layout {
  static constexpr int eslot = round128(BX * EBY * (int)sizeof(T));   // per component
  static constexpr int hslot = round128(BX * HBY * (int)sizeof(T));
  static constexpr int plane = round128(3 * CS * (int)sizeof(T));
  static constexpr int e_off = 0;
  static constexpr int h_off = e_off + NES * 3 * eslot;
  static constexpr int h1_off = h_off + NHS * 3 * hslot;
  static constexpr int e1_off = h1_off + plane;                        // two planes
  static constexpr int h2_off = e1_off + 2 * plane;
  static constexpr int row_off = h2_off + plane;
  static constexpr int l_off = row_off + round128(kRows * kRow * (int)sizeof(T));
  static constexpr int mat_off = l_off + round128(4 * W * (int)sizeof(T));
  static constexpr int bar_off = mat_off + round128(9 * kMat * (int)sizeof(T));
  static constexpr int bytes = bar_off + (NES + NHS) * 8 + 128;        // + base alignment
};

struct Maps {
  CUtensorMap e[3];
  CUtensorMap h[3];
};

}  // namespace t2

// Row entry r of plane q (a[q * stride]), nullptr outside the grid.
template <typename T>
struct Row2 {
  const T* a;
  int stride;
};
template <typename T>
__device__ __forceinline__ Row2<T> row2_entry(const FitParams<T>& p, int r, int i0, int j0) {
  using namespace t2;
  int idx;
  if (r < R_IAY) { idx = j0 - 2 + r; return (idx >= 0 && idx < p.Ny) ? Row2<T>{p.iAx + idx, p.Ny} : Row2<T>{nullptr, 0}; }
  if (r < R_ITAX) { idx = i0 - 2 + r - R_IAY; return (idx >= 0 && idx < p.Nx) ? Row2<T>{p.iAy + idx, p.Nx} : Row2<T>{nullptr, 0}; }
  if (r < R_ITAY) { idx = j0 - 2 + r - R_ITAX; return (idx >= 0 && idx < p.Ny) ? Row2<T>{p.itAx + idx, p.Ny} : Row2<T>{nullptr, 0}; }
  if (r < R_LZ) { idx = i0 - 2 + r - R_ITAY; return (idx >= 0 && idx < p.Nx) ? Row2<T>{p.itAy + idx, p.Nx} : Row2<T>{nullptr, 0}; }
  if (r == R_LZ) return {p.Lz, 1};
  if (r == R_TLZ) return {p.tLz, 1};
  return {nullptr, 0};
}

// SM: material table in shared memory (n_mat <= 32, one-byte ids).  JM:
// WK_J_ZERO or WK_J_SIGMA_E for both steps.  DESC: H-row summation order.
template <typename T, bool SM, int JM, bool DESC>
__global__ void __launch_bounds__(t2::kThreads, 1)
k_tma2(FitParams<T> p, const __grid_constant__ t2::Maps maps, long long step, int KC) {
  using namespace t2;
  using L = Layout<T>;
  step = step_index(p, step);
  constexpr int SE = L::eslot / (int)sizeof(T);
  constexpr int SH = L::hslot / (int)sizeof(T);
  constexpr int PL = L::plane / (int)sizeof(T);
  extern __shared__ __align__(128) unsigned char sm_raw[];
  unsigned char* sm = sm_raw + ((128 - (smem_u32(sm_raw) & 127)) & 127);
  T* Eb = reinterpret_cast<T*>(sm + L::e_off);     // [NES][3][SE]   E0 ring
  T* Hb = reinterpret_cast<T*>(sm + L::h_off);     // [NHS][3][SH]   H0 ring
  T* H1s = reinterpret_cast<T*>(sm + L::h1_off);   // [3][CS]        H1 of plane q
  T* E1s = reinterpret_cast<T*>(sm + L::e1_off);   // [2][PL]        E1 of planes q, q-1
  T* H2s = reinterpret_cast<T*>(sm + L::h2_off);   // [3][CS]        H2 of plane q-1
  T* Rw = reinterpret_cast<T*>(sm + L::row_off);   // [kRows][kRow]
  T* sLx = reinterpret_cast<T*>(sm + L::l_off);    // Lx(i0-2+ea), ea < 67
  T* sLy = sLx + W;                                // Ly(j0-2+eb), eb < 11
  T* stLx = sLy + W;                               // tLx(i0-2+ea)
  T* stLy = stLx + W;                              // tLy(j0-2+eb)
  T* smat = reinterpret_cast<T*>(sm + L::mat_off);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + L::bar_off);

  const int Nx = p.Nx, Ny = p.Ny, Nz = p.Nz;
  const long long N = p.N, NxNy = p.NxNy;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int k0 = blockIdx.z * KC, k1 = min(k0 + KC, Nz);
  const int qs = k0 - 2;                       // first plane of the march
  const int xs = i0 - 4, ys = j0 - 2;          // TMA box origin (x stays 16-byte aligned)
  const int tid = threadIdx.x;
  const bool prod = tid == kThreads - 1;       // producer: last lane of warp 11
  const uint32_t e_bytes = (uint32_t)(3 * BX * EBY * sizeof(T));
  const uint32_t h_bytes = (uint32_t)(3 * BX * HBY * sizeof(T));

  if (prod) {
    for (int s = 0; s < NES + NHS; s++) mbar_init(&bar[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  auto issue_e = [&](int q) {
    const int slot = (q - qs) % NES;
    mbar_expect_tx(&bar[slot], e_bytes);
#pragma unroll
    for (int d = 0; d < 3; d++)
      tma_load_3d(Eb + (slot * 3 + d) * SE, &maps.e[d], xs, ys, q, &bar[slot]);
  };
  auto issue_h = [&](int q) {
    const int slot = (q - qs) % NHS;
    mbar_expect_tx(&bar[NES + slot], h_bytes);
#pragma unroll
    for (int d = 0; d < 3; d++)
      tma_load_3d(Hb + (slot * 3 + d) * SH, &maps.h[d], xs, ys, q, &bar[NES + slot]);
  };
  auto wait_e = [&](int q, long long lim) {
    return mbar_wait(&bar[(q - qs) % NES], (uint32_t)(((q - qs) / NES) & 1), lim);
  };
  auto wait_h = [&](int q, long long lim) {
    return mbar_wait(&bar[NES + (q - qs) % NHS], (uint32_t)(((q - qs) / NHS) & 1), lim);
  };
  // E planes qs..k1+1 and H planes qs..k1 are loaded, each exactly once
  int e_hi = qs - 1, h_hi = qs - 1;
  if (prod) {
    for (int q = qs; q <= qs + NES - 1 && q <= k1 + 1; q++) { issue_e(q); e_hi = q; }
    for (int q = qs; q <= qs + NHS - 1 && q <= k1; q++) { issue_h(q); h_hi = q; }
  }

  // owned cells: warps 0-10 row eb = warp, ea = lane and lane + 32; warp 11
  // the columns ea 64..66 (lane l: (64 + l % 3, l / 3)) and lane 0 also (66, 10)
  const int warp = tid >> 5, lane = tid & 31;
  int ea[2], eb[2];
  bool own[2];
  if (warp < 11) {
    ea[0] = lane; eb[0] = warp; ea[1] = lane + 32; eb[1] = warp;
    own[0] = own[1] = true;
  } else {
    ea[0] = 64 + lane % 3; eb[0] = lane / 3; own[0] = true;
    ea[1] = 66; eb[1] = 10; own[1] = lane == 0;
  }
  int ci[2], cj[2];
  bool ing[2], inB[2], inC[2], inD[2], xf[2], yf[2];
  int cell_bits = 0;   // bit r: capture window; bit 2+r: source line (tile cells / B cells)
  T iAz[2], itAz[2];
#pragma unroll
  for (int r = 0; r < 2; r++) {
    ci[r] = i0 - 2 + ea[r];
    cj[r] = j0 - 2 + eb[r];
    ing[r] = own[r] && ci[r] >= 0 && ci[r] < Nx && cj[r] >= 0 && cj[r] < Ny;
    inB[r] = ing[r] && ea[r] >= 1 && eb[r] >= 1;
    inC[r] = inB[r] && ea[r] <= 65 && eb[r] <= 9;
    inD[r] = inC[r] && ea[r] >= 2 && eb[r] >= 2;
    xf[r] = ci[r] == 0 || ci[r] == Nx - 1;
    yf[r] = cj[r] == 0 || cj[r] == Ny - 1;
    if (inD[r] && p.cap_on && ci[r] >= p.cap_i0 && ci[r] < p.cap_i0 + p.cap_ni &&
        cj[r] >= p.cap_j0 && cj[r] < p.cap_j0 + p.cap_nj)
      cell_bits |= 1 << r;
    if (inB[r] && (p.line_on || p.beam_on) && ci[r] == p.ixs && cj[r] == p.iys)
      cell_bits |= 4 << r;
    const long long m = ing[r] ? ci[r] + (long long)cj[r] * Nx : 0;
    iAz[r] = ing[r] ? p.iAz[m] : T(0);
    itAz[r] = ing[r] ? p.itAz[m] : T(0);
  }
  // plane-invariant metrics of the ext domain
  if (tid < W) {
    const int i = i0 - 2 + tid, j = j0 - 2 + tid;
    sLx[tid] = (i >= 0 && i < Nx) ? p.Lx[i] : T(0);
    stLx[tid] = (i >= 0 && i < Nx) ? p.tLx[i] : T(0);
    sLy[tid] = (tid < YA && j >= 0 && j < Ny) ? p.Ly[j] : T(0);
    stLy[tid] = (tid < YA && j >= 0 && j < Ny) ? p.tLy[j] : T(0);
  }
  if (SM)
    for (int q = tid; q < 9 * p.n_mat; q += kThreads) smat[q] = p.mat[q];
  const T* mat = SM ? smat : p.mat;
  // metric rows of plane q into slot (q - qs) & 3 by cp.async; one group
  // per plane and thread
  auto stage_row = [&](int q) {
    if (tid < kRow && q <= k1 + 1) {
      const Row2<T> e = row2_entry(p, tid, i0, j0);
      const bool v = e.a != nullptr && q >= 0 && q < Nz;
      cp_async<sizeof(T)>(Rw + ((q - qs) & 3) * kRow + tid, v ? e.a + (long long)q * e.stride : p.Lz,
                          v);
    }
    cp_async_commit();
  };
  stage_row(qs);
  stage_row(qs + 1);
  // material ids of plane q of the owned cells
  const unsigned char* idp = static_cast<const unsigned char*>(p.mat_id);
  auto id_at = [&](int r, int q) -> int {
    if (!ing[r] || q < 0 || q >= Nz) return 0;
    const long long n = ci[r] + (long long)cj[r] * Nx + (long long)q * NxNy;
    if (SM || p.id_bytes == 1) return idp[n];
    if (p.id_bytes == 2) return reinterpret_cast<const uint16_t*>(idp)[n];
    return (int)reinterpret_cast<const uint32_t*>(idp)[n];
  };
  int id_q[2], id_q1[2], id_q2[2];   // ids of planes q, q-1, q-2
#pragma unroll
  for (int r = 0; r < 2; r++) {
    id_q[r] = id_at(r, qs);
    id_q1[r] = 0;
    id_q2[r] = 0;
  }
  // registers carried along z: H1 of planes q-1 and q, E1 of plane q (x, y),
  // H2 of plane q-3 (x, y)
  T h1p[2][3], h1c[2][3], e1c[2][2], h2p[2][2];
#pragma unroll
  for (int r = 0; r < 2; r++) {
#pragma unroll
    for (int d = 0; d < 3; d++) h1p[r][d] = h1c[r][d] = T(0);
    e1c[r][0] = e1c[r][1] = h2p[r][0] = h2p[r][1] = T(0);
  }
  const bool desc = DESC;
  const T dt = p.dt;
  const long long lim = loop_wait_ns(p.wait_ns);

  bool ok = true;
  int q = qs;
  for (; q <= k1 + 1; q++) {
    cp_async_wait<1>();                          // this thread's row entry of plane q
    bool got = true;
    if (prod && q <= k1) got = wait_e(q, lim) && wait_e(q + 1, lim) && wait_h(q, lim);
    ok = __syncthreads_and(got);
    if (!ok) break;
    if (prod && q > qs && q + 2 <= k1 + 1) {
      // the slot of E0(q-1) is free: every thread finished B(q-1)
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue_e(q + 2);
      e_hi = q + 2;
    }
    int id_n[2] = {0, 0};
    if (q + 1 <= k1) {
#pragma unroll
      for (int r = 0; r < 2; r++) id_n[r] = id_at(r, q + 1);
    }
    const int es = (q - qs) % NES, es1 = (q + 1 - qs) % NES, hs = (q - qs) % NHS;
    const T* E0 = Eb + es * 3 * SE;
    const T* E0n = Eb + es1 * 3 * SE;
    const T* H0 = Hb + hs * 3 * SH;
    const T* Rq = Rw + ((q - qs) & 3) * kRow;
    const T* Rq1 = Rw + ((q - 1 - qs) & 3) * kRow;
    const T* Rq2 = Rw + ((q - 2 - qs) & 3) * kRow;
    T* E1q = E1s + (q & 1) * PL;
    T* E1q1 = E1s + ((q - 1) & 1) * PL;   // also E1 of plane q-2 until B(q) writes it
    const bool vq = q >= 0 && q < Nz;

    // ---------------- phase 1: D(q-2) (second E half-step), A(q) (first H)
    {
      const int pd = q - 2;
      const bool dout = pd >= k0 && pd < k1;
      const bool zf = pd == 0 || pd == Nz - 1;
      const T* E1d = E1q;                    // E1 of plane q-2
#pragma unroll
      for (int r = 0; r < 2; r++) {
        if (!inC[r] || pd < k0 - 1) continue;
        const int e = eb[r] * W + ea[r];
        const T hx0 = H2s[e], hy0 = H2s[CS + e], hz0 = H2s[2 * CS + e];
        if (dout && inD[r]) {
          const T* m0 = mat + 9 * id_q2[r];
          const T R0 = mul(m0[0], Rq2[R_ITAX + eb[r]]);
          const T R1 = mul(m0[1], Rq2[R_ITAY + ea[r]]);
          const T R2 = mul(m0[2], itAz[r]);
          T curl[3];
          e_lean(R0, R1, R2, stLx[ea[r]], stLy[eb[r]], Rq2[R_TLZ], hx0, hy0, hz0, H2s[CS + e - 1],
                 H2s[2 * CS + e - 1], H2s[e - W], H2s[2 * CS + e - W], h2p[r][0], h2p[r][1],
                 curl[0], curl[1], curl[2]);
          if (yf[r] || zf) curl[0] = T(0);
          if (xf[r] || zf) curl[1] = T(0);
          if (xf[r] || yf[r]) curl[2] = T(0);
          const T eold[3] = {E1d[e], E1d[CS + e], E1d[2 * CS + e]};
          const long long n = ci[r] + (long long)cj[r] * Nx + (long long)pd * NxNy;
          Cell cc;
          cc.i = ci[r]; cc.j = cj[r]; cc.k = pd;
          if (cell_bits & (1 << r)) capture(p, cc, n, step + 1, eold[2]);
#pragma unroll
          for (int d = 0; d < 3; d++) {
            const T ieps = m0[d], sigma = m0[6 + d];
            T jv = T(0);
            if (JM == WK_J_SIGMA_E) jv = mul(sigma, eold[d]);
            if (d == 2 && (cell_bits & (4 << r))) jv = j_in(p, d, cc, n, step + 1, eold[d], sigma);
            p.E_out[d * N + n] = add(eold[d], mul(dt, sub(curl[d], mul(ieps, jv))));
          }
        }
        h2p[r][0] = hx0;
        h2p[r][1] = hy0;
      }
    }
    if (q <= k1) {
#pragma unroll
      for (int r = 0; r < 2; r++) {
        if (!own[r]) continue;
        const int e = eb[r] * W + ea[r];
        T hx = T(0), hy = T(0), hz = T(0);
        if (ing[r] && vq) {
          const int bi = eb[r] * BX + ea[r] + 2;
          const T* m0 = mat + 9 * id_q[r];
          const T R0 = mul(Rq[R_IAX + eb[r]], m0[3]);
          const T R1 = mul(Rq[R_IAY + ea[r]], m0[4]);
          const T R2 = mul(iAz[r], m0[5]);
          hx = H0[bi]; hy = H0[SH + bi]; hz = H0[2 * SH + bi];
          h_lean(dt, desc, R0, R1, R2, sLx[ea[r]], sLy[eb[r]], Rq[R_LZ], E0[bi], E0[SE + bi],
                 E0[2 * SE + bi], E0[SE + bi + 1], E0[2 * SE + bi + 1], E0[bi + BX],
                 E0[2 * SE + bi + BX], E0n[bi], E0n[SE + bi], hx, hy, hz);
        }
        H1s[e] = hx;
        H1s[CS + e] = hy;
        H1s[2 * CS + e] = hz;
        h1c[r][0] = hx;
        h1c[r][1] = hy;
        h1c[r][2] = hz;
      }
    }
    __syncthreads();

    // ---------------- phase 2: B(q) (first E half-step), C(q-1) (second H)
    if (prod && q + 2 <= k1) {
      // the slot of H0(q) is free: every thread finished A(q)
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue_h(q + 2);
      h_hi = q + 2;
    }
    stage_row(q + 2);                           // into the slot of plane q-2 (D done)
    if (q <= k1 && q >= k0 - 1) {               // E1(k0-2) is never read
      const bool zf = q == 0 || q == Nz - 1;
#pragma unroll
      for (int r = 0; r < 2; r++) {
        if (!own[r] || ea[r] < 1 || eb[r] < 1) continue;
        const int e = eb[r] * W + ea[r];
        T en[3] = {T(0), T(0), T(0)};
        if (inB[r] && vq) {
          const T* m0 = mat + 9 * id_q[r];
          const T R0 = mul(m0[0], Rq[R_ITAX + eb[r]]);
          const T R1 = mul(m0[1], Rq[R_ITAY + ea[r]]);
          const T R2 = mul(m0[2], itAz[r]);
          T curl[3];
          e_lean(R0, R1, R2, stLx[ea[r]], stLy[eb[r]], Rq[R_TLZ], h1c[r][0], h1c[r][1],
                 h1c[r][2], H1s[CS + e - 1], H1s[2 * CS + e - 1], H1s[e - W],
                 H1s[2 * CS + e - W], h1p[r][0], h1p[r][1], curl[0], curl[1], curl[2]);
          if (yf[r] || zf) curl[0] = T(0);
          if (xf[r] || zf) curl[1] = T(0);
          if (xf[r] || yf[r]) curl[2] = T(0);
          const int bi = eb[r] * BX + ea[r] + 2;
          const T eold[3] = {E0[bi], E0[SE + bi], E0[2 * SE + bi]};
          const long long n = ci[r] + (long long)cj[r] * Nx + (long long)q * NxNy;
          Cell cc;
          cc.i = ci[r]; cc.j = cj[r]; cc.k = q;
          if ((cell_bits & (1 << r)) && q >= k0 && q < k1) capture(p, cc, n, step, eold[2]);
#pragma unroll
          for (int d = 0; d < 3; d++) {
            const T ieps = m0[d], sigma = m0[6 + d];
            T jv = T(0);
            if (JM == WK_J_SIGMA_E) jv = mul(sigma, eold[d]);
            if (d == 2 && (cell_bits & (4 << r))) jv = j_in(p, d, cc, n, step, eold[d], sigma);
            en[d] = add(eold[d], mul(dt, sub(curl[d], mul(ieps, jv))));
          }
        }
        E1q[e] = en[0];
        E1q[CS + e] = en[1];
        E1q[2 * CS + e] = en[2];
        e1c[r][0] = en[0];
        e1c[r][1] = en[1];
      }
      const int pc = q - 1;                     // C(q-1)
      if (pc >= k0 - 1) {
        const bool hout = pc >= k0 && pc < k1;
        const bool vc = pc >= 0 && pc < Nz;
#pragma unroll
        for (int r = 0; r < 2; r++) {
          if (!own[r] || ea[r] < 1 || ea[r] > 65 || eb[r] < 1 || eb[r] > 9) continue;
          const int e = eb[r] * W + ea[r];
          T hx = T(0), hy = T(0), hz = T(0);
          if (inC[r] && vc) {
            const T* m0 = mat + 9 * id_q1[r];
            const T R0 = mul(Rq1[R_IAX + eb[r]], m0[3]);
            const T R1 = mul(Rq1[R_IAY + ea[r]], m0[4]);
            const T R2 = mul(iAz[r], m0[5]);
            hx = h1p[r][0]; hy = h1p[r][1]; hz = h1p[r][2];
            h_lean(dt, desc, R0, R1, R2, sLx[ea[r]], sLy[eb[r]], Rq1[R_LZ], E1q1[e],
                   E1q1[CS + e], E1q1[2 * CS + e], E1q1[CS + e + 1], E1q1[2 * CS + e + 1],
                   E1q1[e + W], E1q1[2 * CS + e + W], e1c[r][0], e1c[r][1], hx, hy, hz);
            if (hout && inD[r]) {
              const long long n = ci[r] + (long long)cj[r] * Nx + (long long)pc * NxNy;
              p.H_out[n] = hx;
              p.H_out[N + n] = hy;
              p.H_out[2 * N + n] = hz;
            }
          }
          H2s[e] = hx;
          H2s[CS + e] = hy;
          H2s[2 * CS + e] = hz;
        }
      }
    }
#pragma unroll
    for (int r = 0; r < 2; r++) {
#pragma unroll
      for (int d = 0; d < 3; d++) h1p[r][d] = h1c[r][d];
      id_q2[r] = id_q1[r];
      id_q1[r] = id_q[r];
      id_q[r] = id_n[r];
    }
    __syncthreads();
  }
  cp_async_wait<0>();
  if (!ok) {
    // a load did not complete in time: record it, wait (bounded) for the
    // loads this block issued, then return
    if (prod) {
      if (p.status) atomicExch(p.status, 1);
      for (int qq = q; qq <= e_hi; qq++) wait_e(qq, kWaitNs);
      for (int qq = q; qq <= h_hi; qq++) wait_h(qq, kWaitNs);
    }
    __syncthreads();
  }
}

// ----------------------------------------------------------------- host --
template <typename T>
static bool encode2(CUtensorMap* map, const T* base, int Nx, int Ny, int Nz, int by) {
  const CUtensorMapDataType dt =
      sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  cuuint64_t gdim[3] = {(cuuint64_t)Nx, (cuuint64_t)Ny, (cuuint64_t)Nz};
  cuuint64_t gstr[2] = {(cuuint64_t)Nx * sizeof(T), (cuuint64_t)Nx * Ny * sizeof(T)};
  cuuint32_t box[3] = {(cuuint32_t)t2::BX, (cuuint32_t)by, 1};
  cuuint32_t est[3] = {1, 1, 1};
  CUresult r = tma_encode_fn()(map, dt, 3, (void*)base, gdim, gstr, box, est,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// True when two steps of these parameters can run as one k_tma2 launch:
// the TMA conditions, every face PEC-masked (no PMC), clean faces, J = 0
// without conductivity or J = sigma*E with it (no stored J); the source
// line (fused beam or line buffer) is applied in both steps.
template <typename T>
bool tma2_supported(const FitParams<T>& p) {
  if (!tma_supported<T>(p)) return false;
  if (!p.has_pec || p.has_pmc) return false;
  for (int f = 0; f < 6; f++)
    if (p.pec_face[f] != 0) return false;
  if (!p.faces_clean) return false;
  const bool jm_ok = (p.j_mode == WK_J_SIGMA_E && p.use_cond) ||
                     (p.j_mode == WK_J_ZERO && !p.use_cond);
  if (!jm_ok) return false;
  if (p.Nx < 8 || p.Ny < 8 || p.Nz < 5) return false;
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
      cudaSuccess)
    return false;
  return t2::Layout<T>::bytes <= optin;
}

struct Tma2Occ { int sms = 0, per_sm = 0; bool attr = false; };
static Tma2Occ g_occ2[2][2][2][2][64];

template <typename T, bool SM, int JM, bool DESC>
static cudaError_t tma2_occupancy(Tma2Occ** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  Tma2Occ& o = g_occ2[sizeof(T) == 8 ? 0 : 1][SM ? 1 : 0][JM == WK_J_SIGMA_E ? 1 : 0]
                     [DESC ? 1 : 0][dev];
  if (!o.attr) {
    const int smem = t2::Layout<T>::bytes;
    e = cudaFuncSetAttribute(k_tma2<T, SM, JM, DESC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&o.sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.per_sm, k_tma2<T, SM, JM, DESC>,
                                                      t2::kThreads, smem);
    if (e != cudaSuccess) return e;
    if (o.per_sm < 1) o.per_sm = 1;
    o.attr = true;
  }
  *out = &o;
  return cudaSuccess;
}

// Planes per block when none is given: KC in [4, 64] minimising (waves of
// blocks) x (KC + 4), the 4 standing for the planes a chunk recomputes below
// and above its own (two for each step) and the pipeline fill.
static int tma2_auto_kc(long long tiles, int planes, long long slots) {
  int best = 16;
  long long best_cost = -1;
  for (int kc = 4; kc <= 64; kc++) {
    const long long gz = (planes + kc - 1) / kc;
    const long long waves = (tiles * gz + slots - 1) / slots;
    const long long cost = waves * (kc + 4);
    if (best_cost < 0 || cost < best_cost) { best_cost = cost; best = kc; }
    if (kc >= planes) break;
  }
  return best;
}

template <typename T, bool SM, int JM, bool DESC>
static cudaError_t launch_tma2_variant(const FitParams<T>& p, long long step, cudaStream_t st,
                                       int KC) {
  t2::Maps maps;
  for (int d = 0; d < 3; d++) {
    if (!encode2<T>(&maps.e[d], p.E_in + d * p.N, p.Nx, p.Ny, p.Nz, t2::EBY) ||
        !encode2<T>(&maps.h[d], p.H_in + d * p.N, p.Nx, p.Ny, p.Nz, t2::HBY))
      return cudaErrorInvalidValue;
  }
  Tma2Occ* occ = nullptr;
  cudaError_t e = tma2_occupancy<T, SM, JM, DESC>(&occ);
  if (e != cudaSuccess) return e;
  const int gx = (p.Nx + t2::TX - 1) / t2::TX, gy = (p.Ny + t2::TY - 1) / t2::TY;
  if (KC <= 0) KC = tma2_auto_kc((long long)gx * gy, p.Nz, (long long)occ->sms * occ->per_sm);
  const int gz = (p.Nz + KC - 1) / KC;
  timer_begin(st);
  k_tma2<T, SM, JM, DESC><<<dim3(gx, gy, gz), t2::kThreads, t2::Layout<T>::bytes, st>>>(
      p, maps, step, KC);
  timer_end(st);
  return cudaGetLastError();
}

// Two steps (step, step + 1) of the state p.E_in, p.H_in into p.E_out,
// p.H_out with one k_tma2 launch; tma2_supported(p) must hold.
template <typename T>
cudaError_t launch_tma2(const FitParams<T>& p, long long step, cudaStream_t st, int KC) {
  const bool sm_table = p.n_mat <= t2::kMat && p.id_bytes == 1;
  const bool cond = p.j_mode == WK_J_SIGMA_E;
  const bool desc = p.h_desc != 0;
#define WK_T2(SMV, JMV, DV) return launch_tma2_variant<T, SMV, JMV, DV>(p, step, st, KC);
  if (sm_table) {
    if (cond) { if (desc) WK_T2(true, WK_J_SIGMA_E, true) WK_T2(true, WK_J_SIGMA_E, false) }
    if (desc) WK_T2(true, WK_J_ZERO, true) WK_T2(true, WK_J_ZERO, false)
  }
  if (cond) { if (desc) WK_T2(false, WK_J_SIGMA_E, true) WK_T2(false, WK_J_SIGMA_E, false) }
  if (desc) WK_T2(false, WK_J_ZERO, true) WK_T2(false, WK_J_ZERO, false)
#undef WK_T2
}

template bool tma2_supported<double>(const FitParams<double>&);
template bool tma2_supported<float>(const FitParams<float>&);
template cudaError_t launch_tma2<double>(const FitParams<double>&, long long, cudaStream_t, int);
template cudaError_t launch_tma2<float>(const FitParams<float>&, long long, cudaStream_t, int);

}  // namespace wk
