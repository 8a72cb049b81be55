// Fused FIT step with TMA-staged plane tiles (sm_100a).
//
// Which cells a launch covers depends on the face mode (MODE, see k_tma): the
// interior (2 <= i, j, k <= N-3, the two-cell shell in separate launches),
// all of x and y for 2 <= k <= Nz-3 (x/y faces PEC-masked), or the whole grid
// (every face PEC-masked).  Block (bx, by, bz) owns the tile
// i in [i0, i0+TX), j in [j0, j0+TY) of planes [k0, k0+KC) and marches in z;
// the tiles are 64x8 (the default) or 32x16 (wk_fit_desc.tile_rows = 16).
// For plane k it needs E_old of planes k and k+1 on a box from (i0-2, j0-1)
// (interior) or (i0-4, j0-1) (full-domain modes; x offsets stay 16-byte
// aligned) and H_old of plane k on a box one row shorter.  An idle lane of
// warp 9 issues the cp.async.bulk.tensor loads of those boxes (one per field
// component, no multicast) into a ring of shared-memory slots, three planes
// of E and two of H, each slot completing on its own mbarrier; at the start
// of plane k the loads of E(k+2) and H(k+1) go out into the slots plane k-1
// released.
//
// Per plane the block computes the new H on the tile plus its low halo row
// and column (single-coefficient rows; the halo is recomputed so that no
// block waits for another), a barrier, then the new E of the tile.  Each
// thread owns the same cells in both phases (warps 0-7, 64x8: row j0+w of
// the tile, cells i0+lane and i0+32+lane; 32x16: rows j0+2w and j0+2w+1,
// column i0+lane; warp 8: the halo row; warp 9: the halo column and the last
// cell of the halo row), so the new Hx, Hy of its tile
// cells stay in registers as H(k-1) of the next plane.  The per-plane metric
// rows (iAx, iAy, itAx, itAy, Lz, tLz) go into a 3-slot ring by cp.async two
// planes ahead, issued by warps 8 and 9 while the tile warps compute E; the
// material ids of plane k+1 are loaded during plane k; the plane-invariant
// metrics (Lx, Ly, iAz, ...) are loaded once.  A chunk starting at k0 first
// forms the new H of plane k0-1 on its tile.  Every mbarrier wait is
// bounded: on timeout the block records the failure in the status word,
// waits (bounded) for its loads in flight and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include "../../include/wakis_b200.h"
#include "abi_internal.h"
#include "fit_common.cuh"
#include "fit_kernels.cuh"
#include "tma_util.cuh"

namespace wk {

constexpr int kES = 3, kHS = 2;                      // ring slots
static_assert(kES == 3 && kHS == 2, "the step loop counts the ring slots for 3 E and 2 H slots");
constexpr int kTmaThreads = 320;
constexpr int kMatSmem = 32;                         // materials staged in smem

// Tile shape: TW columns x 512/TW rows.  Each thread owns two cells: the
// tile warps (0-7) a cell of tile row w and the cell 32 columns on (64x8),
// or cells of tile rows 2w and 2w+1 in the same column (32x16); warp 8 and
// warp 9 own the halo row and column.
template <int TW>
struct TShape {
  static_assert(TW == 64 || TW == 32, "tile widths 64 and 32");
  static constexpr int TX = TW, TY = 512 / TW;
  static constexpr int BX = TX + 4, BY = TY + 2;     // interior E box, E box rows
  static constexpr int HBY = TY + 1;                 // H box rows
  static constexpr int EW = TX + 1;                  // ext tile row width
  static constexpr int Ext = EW * (TY + 1);
  // second cell of a thread: dx columns and dy rows on
  static constexpr int DX = TW == 64 ? 32 : 0, DY = TW == 64 ? 0 : 1;
  // per-plane metric row: [0, TY+1) iAx(j0-1..), [RY, RY+TX+1) iAy(i0-1..),
  // [RTX, RTX+TY) itAx(j0..), [RTY, RTY+TX) itAy(i0..), RL Lz, RL+1 tLz
  static constexpr int RY = TY + 1, RTX = RY + TX + 1, RTY = RTX + TY, RL = RTY + TX;
  static constexpr int Row = RL + 2;
  static constexpr int Lvals = EW + TY + 1 + TX + TY;   // Lx, Ly, tLx, tLy staged once
  static_assert(Row <= 3 * 64 && Lvals <= kTmaThreads, "staging threads");
};

// H box width (interior variant): TX+2 doubles or TX+4 floats (the inner
// box extent must be a multiple of 16 bytes).
template <typename T, int TW>
constexpr int h_box_x() { return sizeof(T) == 8 ? TW + 2 : TW + 4; }

struct TmaMaps {
  CUtensorMap e[3];
  CUtensorMap h[3];
};

// Box geometry.  The interior variant loads E on x in [i0-2, i0+TX+2) and
// H on [i0-2, i0+TX) (i0 = 2 + TX bx); the full-domain variant (FULL, tiles
// from i0 = TX bx) starts both boxes at i0-4 so that the x offset stays
// 16-byte aligned for float and double: E TX+8 wide, H TX+4 wide.
template <typename T, bool FULL, int TW = 64>
struct TmaGeom {
  using S = TShape<TW>;
  static constexpr int ebx = FULL ? S::TX + 8 : S::BX;            // E box width
  static constexpr int hbx = FULL ? S::TX + 4 : h_box_x<T, TW>();  // H box width
  static constexpr int xo = FULL ? 3 : 1;                          // box x of ext column 0
  static constexpr int xs_off = FULL ? 4 : 2;                      // box start = i0 - xs_off
};

template <typename T, bool FULL, int TW = 64>
struct TmaLayout {
  using S = TShape<TW>;
  using G = TmaGeom<T, FULL, TW>;
  static constexpr int eslot = round128(G::ebx * S::BY * (int)sizeof(T));        // per comp
  static constexpr int hslot = round128(G::hbx * S::HBY * (int)sizeof(T));
  static constexpr int e_off = 0;
  static constexpr int h_off = e_off + kES * 3 * eslot;
  static constexpr int hs_off = h_off + kHS * 3 * hslot;
  static constexpr int row_off = hs_off + round128(3 * S::Ext * (int)sizeof(T));
  static constexpr int l_off = row_off + round128(3 * S::Row * (int)sizeof(T));
  static constexpr int mat_off = l_off + round128(S::Lvals * (int)sizeof(T));
  static constexpr int bar_off = mat_off + round128(9 * kMatSmem * (int)sizeof(T));
  static constexpr int bytes = bar_off + (kES + kHS) * 8 + 128;   // + base alignment
};


// Per-plane metric row of plane q (TShape: RY, RTX, RTY, RL).
// Entry r of plane q is a[q * stride] (RowEntry); entries outside the grid
// (index < 0 or beyond the last cell, a == nullptr) and planes outside
// [0, Nz) read as 0.
template <typename T>
struct RowEntry {
  const T* a;
  int stride;
};
template <typename T, int TW>
__device__ __forceinline__ RowEntry<T> row_entry(const FitParams<T>& p, int r, int i0, int j0) {
  using S = TShape<TW>;
  int idx;
  if (r < S::RY) { idx = j0 - 1 + r; if (idx < 0 || idx >= p.Ny) return {nullptr, 0}; return {p.iAx + idx, p.Ny}; }
  if (r < S::RTX) { idx = i0 - 1 - S::RY + r; if (idx < 0 || idx >= p.Nx) return {nullptr, 0}; return {p.iAy + idx, p.Nx}; }
  if (r < S::RTY) { idx = j0 - S::RTX + r; if (idx < 0 || idx >= p.Ny) return {nullptr, 0}; return {p.itAx + idx, p.Ny}; }
  if (r < S::RL) { idx = i0 - S::RTY + r; if (idx < 0 || idx >= p.Nx) return {nullptr, 0}; return {p.itAy + idx, p.Nx}; }
  if (r == S::RL) return {p.Lz, 1};
  if (r == S::RL + 1) return {p.tLz, 1};
  return {nullptr, 0};
}

// SM: the material table fits in shared memory (n_mat <= kMatSmem) and the
// ids are one byte each; the table reads are then shared-memory loads.  JM: the J mode of the launch
// (WK_J_ZERO, WK_J_SIGMA_E or WK_J_ARRAY), fixed at compile time.
// MODE 0: interior cells only (2 <= i, j, k <= N-3), the two-cell shell runs
// in separate launches.  MODE 1: every face of the grid carries the PEC
// column mask (pec, electric or pml on all six faces, no PMC); the tiles
// cover the whole grid and the cells next to a face use the same
// single-coefficient rows with the masked terms set to zero: an E entry
// tangential to a face it lies on enters no H row, and an E row tangential
// to its face gets no curl.  The neighbours that the flat-offset operators
// reach by wrapping (i+1 past Nx-1, j+1 past Ny-1) are tangential to the
// opposite face, so every wrapped term is masked and no shell launch
// follows.  MODE 2: the four x/y faces are PEC-masked and the z faces are
// not (ABC, periodic): the tiles cover all of x and y for the planes
// 2 <= k <= Nz-3 (no z face is involved there), and the shell launches
// cover only the planes k in {0, 1, Nz-2, Nz-1}.  Warps with no cell on or
// next to a face take the unmasked rows.
template <typename T, bool SM, int JM, int MODE, bool DESC, int TW>
__global__ void __launch_bounds__(kTmaThreads, sizeof(T) == 8 ? 2 : 3)
k_tma(FitParams<T> p, const __grid_constant__ TmaMaps maps, long long step, int KC) {
  constexpr bool FULL = MODE != 0;     // tiles cover x and y entirely
  constexpr bool ZFULL = MODE == 1;    // ... and every plane
  step = step_index(p, step);
  using S = TShape<TW>;
  using Lay = TmaLayout<T, (MODE != 0), TW>;
  using G = TmaGeom<T, (MODE != 0), TW>;
  constexpr int HBX = G::hbx;
  constexpr int EBX = G::ebx;
  constexpr int XO = G::xo;
  constexpr int SE = Lay::eslot / (int)sizeof(T);    // elements per E slot
  constexpr int SH = Lay::hslot / (int)sizeof(T);    // elements per H slot
  extern __shared__ __align__(128) unsigned char sm_raw[];
  unsigned char* sm = sm_raw + ((128 - (smem_u32(sm_raw) & 127)) & 127);
  T* Eb = reinterpret_cast<T*>(sm + Lay::e_off);     // [kES][3][SE]
  T* Hb = reinterpret_cast<T*>(sm + Lay::h_off);     // [kHS][3][SH]
  T* Hs = reinterpret_cast<T*>(sm + Lay::hs_off);    // [3][Ext] new H of the plane
  T* Rw = reinterpret_cast<T*>(sm + Lay::row_off);   // [3][Row] per-plane metrics
  T* sLx = reinterpret_cast<T*>(sm + Lay::l_off);    // Lx(i0-1..i0+TX-1)
  T* sLy = sLx + S::EW;                              // Ly(j0-1..j0+TY-1)
  T* stLx = sLy + S::TY + 1;                         // tLx(i0..i0+TX-1)
  T* stLy = stLx + S::TX;                            // tLy(j0..j0+TY-1)
  T* smat = reinterpret_cast<T*>(sm + Lay::mat_off);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + Lay::bar_off);  // E slots, then H slots

  const int Nx = p.Nx, Ny = p.Ny;
  const long long N = p.N, NxNy = p.NxNy;
  const int Nz = p.Nz;
  const int i0 = (FULL ? 0 : 2) + blockIdx.x * S::TX, j0 = (FULL ? 0 : 2) + blockIdx.y * S::TY;
  const int k0 = (ZFULL ? 0 : 2) + blockIdx.z * KC, k1 = min(k0 + KC, ZFULL ? Nz : Nz - 2);
  const int xs = i0 - G::xs_off, ys = j0 - 1;
  const int tid = threadIdx.x;
  // the producer (mbarrier set-up, TMA issue and waits) is the last lane of
  // warp 9, which owns no cell
  const bool prod = tid == kTmaThreads - 1;
  const int pstart = k0 - 1;
  const uint32_t e_bytes = (uint32_t)(3 * EBX * S::BY * sizeof(T));
  const uint32_t h_bytes = (uint32_t)(3 * HBX * S::HBY * sizeof(T));

  if (prod) {
    for (int s = 0; s < kES + kHS; s++) mbar_init(&bar[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  auto issue_e = [&](int q) {
    const int slot = (q - pstart) % kES;
    mbar_expect_tx(&bar[slot], e_bytes);
#pragma unroll
    for (int d = 0; d < 3; d++)
      tma_load_3d(Eb + (slot * 3 + d) * SE, &maps.e[d], xs, ys, q, &bar[slot]);
  };
  auto issue_h = [&](int q) {
    const int slot = (q - pstart) % kHS;
    mbar_expect_tx(&bar[kES + slot], h_bytes);
#pragma unroll
    for (int d = 0; d < 3; d++)
      tma_load_3d(Hb + (slot * 3 + d) * SH, &maps.h[d], xs, ys, q, &bar[kES + slot]);
  };
  auto wait_e = [&](int q, long long lim) {
    return mbar_wait(&bar[(q - pstart) % kES], (uint32_t)(((q - pstart) / kES) & 1), lim);
  };
  auto wait_h = [&](int q, long long lim) {
    return mbar_wait(&bar[kES + (q - pstart) % kHS], (uint32_t)(((q - pstart) / kHS) & 1), lim);
  };
  // E planes pstart..k1 and H planes pstart..k1-1 are loaded, each exactly
  // once; e_hi / h_hi (producer) track the last plane issued
  int e_hi = pstart - 1, h_hi = pstart - 1;
  if (prod) {
    for (int q = pstart; q <= min(pstart + kES - 1, k1); q++) { issue_e(q); e_hi = q; }
    for (int q = pstart; q <= min(pstart + kHS - 1, k1 - 1); q++) { issue_h(q); h_hi = q; }
  }

  // owned cells, in ext-tile coordinates (ea, eb) with the origin at
  // (i0-1, j0-1).  64x8: warps 0-7 the tile cells (lane+1, w+1) and
  // (lane+33, w+1); warp 8 the halo-row cells (lane, 0) and (lane+32, 0).
  // 32x16: warps 0-7 the tile cells (lane+1, 2w+1) and (lane+1, 2w+2); warp
  // 8 the halo-row cell (lane, 0).  Warp 9: lanes 0..TY-1 the halo-column
  // cells (0, lane+1) and lane TY the halo-row cell (TX, 0).  The second cell
  // of a thread is its first one DX columns and DY rows on.
  const int warp = tid >> 5, lane = tid & 31;
  const bool tile = warp < 8;
  const int ea0 = tile ? lane + 1 : (warp == 8 ? lane : (lane < S::TY ? 0 : S::TX));
  const int eb0 = tile ? (TW == 64 ? warp : 2 * warp) + 1
                       : (warp == 8 ? 0 : (lane < S::TY ? lane + 1 : 0));
  const bool owns[2] = {warp < 9 || lane < S::TY + 1, TW == 64 ? warp < 9 : warp < 8};
  const int ext0 = eb0 * S::EW + ea0;
  constexpr int dext = S::DX + S::DY * S::EW;         // ext offset of the second cell
  const int dcell = S::DX + S::DY * Nx;               // flat offset of the second cell
  int ci[2], cj[2];
  bool hval[2], eval[2];
#pragma unroll
  for (int r = 0; r < 2; r++) {
    ci[r] = i0 - 1 + ea0 + S::DX * r;
    cj[r] = j0 - 1 + eb0 + S::DY * r;
    const bool own = owns[r];
    hval[r] = FULL ? (own && ci[r] >= 0 && ci[r] <= Nx - 1 && cj[r] >= 0 && cj[r] <= Ny - 1)
                   : (own && ci[r] <= Nx - 3 && cj[r] <= Ny - 3);
    eval[r] = tile && hval[r];
  }
  // face flags of the owned cells (FULL): at the cell, and of the +x / +y
  // neighbour (a wrapped neighbour counts as on the face)
  bool xf0[2], xf1[2], yf0[2], yf1[2];
  bool nearface = false;
#pragma unroll
  for (int r = 0; r < 2; r++) {
    xf0[r] = ci[r] == 0 || ci[r] == Nx - 1;
    xf1[r] = ci[r] + 1 >= Nx - 1;
    yf0[r] = cj[r] == 0 || cj[r] == Ny - 1;
    yf1[r] = cj[r] + 1 >= Ny - 1;
    if (hval[r]) nearface |= xf0[r] || xf1[r] || yf0[r] || yf1[r];
  }
  const bool warp_face = FULL && __any_sync(0xffffffffu, nearface);
  constexpr bool desc = DESC;   // H-row summation order (wk_fit_desc.h_sum_desc)
  // plane-invariant tests of the owned cells, one bit each: cell r in the
  // Ez capture window (bit r), on the source line (bit 2 + r)
  int cell_bits = 0;
#pragma unroll
  for (int r = 0; r < 2; r++) {
    if (eval[r] && p.cap_on && ci[r] >= p.cap_i0 && ci[r] < p.cap_i0 + p.cap_ni &&
        cj[r] >= p.cap_j0 && cj[r] < p.cap_j0 + p.cap_nj)
      cell_bits |= 1 << r;
    if (eval[r] && (p.line_on || p.beam_on) && ci[r] == p.ixs && cj[r] == p.iys)
      cell_bits |= 4 << r;
  }
  // plane-invariant metrics
  T iAz[2], itAz[2];
#pragma unroll
  for (int r = 0; r < 2; r++) {
    const long long m = ci[r] + (long long)cj[r] * Nx;
    iAz[r] = hval[r] ? p.iAz[m] : T(0);
    itAz[r] = eval[r] ? p.itAz[m] : T(0);
  }
  {
    constexpr int EW = S::EW, TX = S::TX, TY = S::TY;
    if (tid < EW) sLx[tid] = (i0 - 1 + tid >= 0 && i0 - 1 + tid < Nx) ? p.Lx[i0 - 1 + tid] : T(0);
    else if (tid < EW + TY + 1) { const int j = j0 - 1 + tid - EW; sLy[tid - EW] = (j >= 0 && j < Ny) ? p.Ly[j] : T(0); }
    else if (tid < EW + TY + 1 + TX) { const int i = i0 + tid - EW - TY - 1; stLx[tid - EW - TY - 1] = i < Nx ? p.tLx[i] : T(0); }
    else if (tid < EW + TY + 1 + TX + TY) { const int j = j0 + tid - EW - TY - 1 - TX; stLy[tid - EW - TY - 1 - TX] = j < Ny ? p.tLy[j] : T(0); }
  }
  if (SM)
    for (int q = tid; q < 9 * p.n_mat; q += kTmaThreads) smat[q] = p.mat[q];
  const T* mat = SM ? smat : p.mat;
  // The metric row of plane q goes into ring slot (q - pstart) % 3 (passed
  // as `slot`) by cp.async two planes ahead, issued by warps 8 and 9
  // (entries t, t+64, t+128 for t = tid - 256) while the tile warps compute
  // the E of the plane before; one group per plane and thread.
  auto stage_row = [&](int q, int slot) {
    if (tid >= 256 && q < k1) {
#pragma unroll
      for (int u = 0; u < 3; u++) {
        const int r = tid - 256 + 64 * u;
        if (r < S::Row) {
          const RowEntry<T> e = row_entry<T, TW>(p, r, i0, j0);
          const bool v = e.a != nullptr && q >= 0 && q < Nz;
          cp_async<sizeof(T)>(Rw + slot * S::Row + r, v ? e.a + (long long)q * e.stride : p.Lz, v);
        }
      }
    }
    cp_async_commit();
  };
  stage_row(pstart, 0);
  stage_row(pstart + 1, 1);
  // material ids: one byte each with the table in shared memory (SM),
  // else id_bytes wide; the pointer of cell 0 advances one plane per step
  const unsigned char* idp = static_cast<const unsigned char*>(p.mat_id) +
                             (ci[0] + (long long)cj[0] * Nx) * p.id_bytes;
  const long long id_plane = NxNy * p.id_bytes;
  auto id_at = [&](int r, int q) -> int {
    const unsigned char* a = idp + (long long)q * id_plane + dcell * r * (SM ? 1 : p.id_bytes);
    if (SM) return a[0];
    if (p.id_bytes == 1) return a[0];
    if (p.id_bytes == 2) return *reinterpret_cast<const uint16_t*>(a);
    return (int)*reinterpret_cast<const uint32_t*>(a);
  };
  int id[2];
#pragma unroll
  for (int r = 0; r < 2; r++) id[r] = (hval[r] && pstart >= 0) ? id_at(r, pstart) : 0;
  T hxp[2] = {T(0), T(0)}, hyp[2] = {T(0), T(0)};
  // per-plane cursors: the ids of plane pl+1, the outputs of cell 0 of
  // plane pl (the second cell is dcell entries on); ring slots of E(pl), H(pl)
  // and of the metric row of pl, counted instead of taken modulo
  const unsigned char* idq = idp + (long long)(pstart + 1) * id_plane;
  const long long cn0 = ci[0] + (long long)cj[0] * Nx + (long long)pstart * NxNy;
  T* hq = p.H_out + cn0;
  T* eq = p.E_out + cn0;
  int se = 0, sh = 0;

  bool ok = true;
  int pl = pstart;
  const long long lim = loop_wait_ns(p.wait_ns);   // step-loop waits; the drain keeps kWaitNs
  for (; pl < k1; pl++) {
    cp_async_wait<1>();          // this thread's row entry of plane pl
    bool got = true;
    if (prod) got = wait_e(pl, lim) && wait_e(pl + 1, lim) && wait_h(pl, lim);
    ok = __syncthreads_and(got);
    if (!ok) break;
    const bool prologue = pl == pstart;
    if (prod && !prologue) {
      // the slots of E(pl-1) and H(pl-1) are free: every thread finished plane pl-1
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      if (pl + kES - 1 <= k1) { issue_e(pl + kES - 1); e_hi = pl + kES - 1; }
      if (pl + kHS - 1 <= k1 - 1) { issue_h(pl + kHS - 1); h_hi = pl + kHS - 1; }
    }
    // prefetch the ids of plane pl+1
    const bool more = pl + 1 < k1;
    int idn[2] = {0, 0};
    if (more) {
#pragma unroll
      for (int r = 0; r < 2; r++) {
        if (!hval[r]) continue;
        const unsigned char* a = idq + dcell * r * (SM ? 1 : p.id_bytes);
        if (SM || p.id_bytes == 1) idn[r] = a[0];
        else if (p.id_bytes == 2) idn[r] = *reinterpret_cast<const uint16_t*>(a);
        else idn[r] = (int)*reinterpret_cast<const uint32_t*>(a);
      }
    }
    const int se1 = se == kES - 1 ? 0 : se + 1;     // slot of E(pl+1)
    const T* Ek = Eb + se * 3 * SE;
    const T* Ek1 = Eb + se1 * 3 * SE;
    const T* Hk = Hb + sh * 3 * SH;
    const T* R = Rw + se * S::Row;                   // row ring: also 3 slots
    const long long off = (long long)pl * NxNy;
    T* const hq1 = hq + N;
    T* const eq1 = eq + N;

    // plane face flags (MODE 1): at the plane and of the +z neighbour
    const bool zf0 = ZFULL && (pl == 0 || pl == Nz - 1), zf1 = ZFULL && pl + 1 >= Nz - 1;
    const bool masked = FULL && (warp_face || zf0 || zf1);

    // new H of the owned cells (tile cells only in the prologue; FULL: no H
    // below plane 0, the ext cells outside the grid hold 0)
    T hxn[2], hyn[2];
#pragma unroll
    for (int r = 0; r < 2; r++) {
      hxn[r] = hyn[r] = T(0);
      const bool tile_cell = tile;
      const int e = ext0 + dext * r;
      if (FULL && owns[r] && !hval[r]) {
        Hs[e] = T(0);
        Hs[S::Ext + e] = T(0);
        Hs[2 * S::Ext + e] = T(0);
      }
      if (!hval[r] || (prologue && !tile_cell) || (ZFULL && pl < 0)) continue;
      const int ea = ea0 + S::DX * r, eb = eb0 + S::DY * r;
      const int bi = eb * EBX + ea + XO;
      const int hb = eb * HBX + ea + XO;
      const T* m0 = mat + 9 * id[r];
      const T R0 = mul(R[eb], m0[3]);
      const T R1 = mul(R[S::RY + ea], m0[4]);
      const T R2 = mul(iAz[r], m0[5]);
      T hx = Hk[hb], hy = Hk[SH + hb], hz = Hk[2 * SH + hb];
      T ex0 = Ek[bi], ey0 = Ek[SE + bi], ez0 = Ek[2 * SE + bi];
      T ey1 = Ek[SE + bi + 1], ez1 = Ek[2 * SE + bi + 1];
      T ex2 = Ek[bi + EBX], ez2 = Ek[2 * SE + bi + EBX];
      T ex3 = Ek1[bi], ey3 = Ek1[SE + bi];
      if (masked && !p.faces_clean) {
        // E column entries tangential to a face they lie on are masked
        // (with faces_clean those entries are +0 already)
        const T z = T(0);
        ex0 = (yf0[r] || zf0) ? z : ex0;
        ey0 = (xf0[r] || zf0) ? z : ey0;
        ez0 = (xf0[r] || yf0[r]) ? z : ez0;
        ey1 = (xf1[r] || zf0) ? z : ey1;
        ez1 = (xf1[r] || yf0[r]) ? z : ez1;
        ex2 = (yf1[r] || zf0) ? z : ex2;
        ez2 = (xf0[r] || yf1[r]) ? z : ez2;
        ex3 = (yf0[r] || zf1) ? z : ex3;
        ey3 = (xf0[r] || zf1) ? z : ey3;
      }
      h_lean(p.dt, desc, R0, R1, R2, sLx[ea], sLy[eb], R[S::RL], ex0, ey0, ez0, ey1, ez1, ex2,
             ez2, ex3, ey3, hx, hy, hz);
      Hs[e] = hx;
      Hs[S::Ext + e] = hy;
      Hs[2 * S::Ext + e] = hz;
      hxn[r] = hx;
      hyn[r] = hy;
      if (!prologue && tile_cell) {
        hq[dcell * r] = hx;
        hq1[dcell * r] = hy;
        hq1[N + dcell * r] = hz;
      }
    }
    __syncthreads();

    // warps 8 and 9 own no E row: the row slot of plane pl-1 is free (every
    // thread passed the top barrier of plane pl), stage the row of pl+2
    if (warp >= 8) stage_row(pl + 2, se == 0 ? kES - 1 : se - 1);
    if (!prologue) {
      const T tLz = R[S::RL + 1];
#pragma unroll
      for (int r = 0; r < 2; r++) {
        if (!eval[r]) continue;
        const int e = ext0 + dext * r;
        const int a = ea0 + S::DX * r - 1, b = eb0 + S::DY * r - 1;
        const int bi = (b + 1) * EBX + a + 1 + XO;
        const long long n = ci[r] + (long long)cj[r] * Nx + off;
        const T* m0 = mat + 9 * id[r];
        const T R0 = mul(m0[0], R[S::RTX + b]);
        const T R1 = mul(m0[1], R[S::RTY + a]);
        const T R2 = mul(m0[2], itAz[r]);
        T curl[3];
        e_lean(R0, R1, R2, stLx[a], stLy[b], tLz, Hs[e], Hs[S::Ext + e], Hs[2 * S::Ext + e],
               Hs[S::Ext + e - 1], Hs[2 * S::Ext + e - 1], Hs[e - S::EW],
               Hs[2 * S::Ext + e - S::EW],
               hxp[r], hyp[r], curl[0], curl[1], curl[2]);
        if (masked) {
          // E rows tangential to the face the cell lies on get no curl
          if (yf0[r] || zf0) curl[0] = T(0);
          if (xf0[r] || zf0) curl[1] = T(0);
          if (xf0[r] || yf0[r]) curl[2] = T(0);
        }
        const T eold[3] = {Ek[bi], Ek[SE + bi], Ek[2 * SE + bi]};
        Cell cc;
        cc.i = ci[r]; cc.j = cj[r]; cc.k = pl;
        if (cell_bits & (1 << r)) capture(p, cc, n, step, eold[2]);
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const T ieps = m0[d], sigma = m0[6 + d];
          // J entering the row (the j_in rules with the mode fixed)
          T jv = T(0);
          if (JM == WK_J_SIGMA_E) jv = mul(sigma, eold[d]);
          if (JM == WK_J_ARRAY) jv = p.J[d * N + n];
          if (d == 2 && (cell_bits & (4 << r))) jv = j_in(p, d, cc, n, step, eold[d], sigma);
          const T enew = add(eold[d], mul(p.dt, sub(curl[d], mul(ieps, jv))));
          (d == 0 ? eq : (d == 1 ? eq1 : eq1 + N))[dcell * r] = enew;
          if (JM == WK_J_ARRAY && p.use_cond) p.J[d * N + n] = mul(sigma, enew);
        }
      }
    }
#pragma unroll
    for (int r = 0; r < 2; r++) {
      hxp[r] = hxn[r];
      hyp[r] = hyn[r];
      id[r] = idn[r];
    }
    idq += id_plane;
    hq += NxNy;
    eq += NxNy;
    se = se1;
    sh ^= 1;
  }
  cp_async_wait<0>();
  if (!ok) {
    // a load did not complete in time: record it, wait (bounded) for the
    // loads this block issued, then return
    if (prod) {
      if (p.status) atomicExch(p.status, 1);
      for (int q = pl; q <= e_hi; q++) wait_e(q, kWaitNs);
      for (int q = pl; q <= h_hi; q++) wait_h(q, kWaitNs);
    }
    __syncthreads();
  }
}

// ----------------------------------------------------------------- host --
template <typename T>
static bool encode_comp(CUtensorMap* map, const T* base, int Nx, int Ny, int Nz, int bx,
                        int by) {
  const CUtensorMapDataType dt =
      sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  cuuint64_t gdim[3] = {(cuuint64_t)Nx, (cuuint64_t)Ny, (cuuint64_t)Nz};
  cuuint64_t gstr[2] = {(cuuint64_t)Nx * sizeof(T), (cuuint64_t)Nx * Ny * sizeof(T)};
  cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  cuuint32_t est[3] = {1, 1, 1};
  CUresult r = tma_encode_fn()(map, dt, 3, (void*)base, gdim, gstr, box, est,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// True when the TMA kernel can run this grid: 16-byte strides and bases
// (Nx*sizeof(T) multiple of 16 and N even), dims >= 5, fewer than 2^31
// cells, the driver entry point present.
template <typename T>
bool tma_supported(const FitParams<T>& p) {
  if (p.Nx < 5 || p.Ny < 5 || p.Nz < 5) return false;
  if (p.N >= (1LL << 31)) return false;
  if ((p.Nx * sizeof(T)) % 16 != 0 || (p.N * sizeof(T)) % 16 != 0) return false;
  if (((uintptr_t)p.E_in % 16) || ((uintptr_t)p.H_in % 16)) return false;
  return tma_encode_fn() != nullptr;
}

// Launch geometry cache per device: SM count and resident blocks per SM.
struct TmaOcc { int sms = 0, per_sm = 0; bool attr = false; };
static TmaOcc g_occ[2][2][3][3][2][2][64];

template <typename T, bool SM, int JM, int MODE, bool DESC, int TW>
static cudaError_t tma_occupancy(TmaOcc** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  TmaOcc& o = g_occ[sizeof(T) == 8 ? 0 : 1][SM ? 1 : 0][JM][MODE][DESC ? 1 : 0][TW == 32][dev];
  if (!o.attr) {
    const int smem = TmaLayout<T, (MODE != 0), TW>::bytes;
    e = cudaFuncSetAttribute(k_tma<T, SM, JM, MODE, DESC, TW>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&o.sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.per_sm, k_tma<T, SM, JM, MODE, DESC, TW>,
                                                      kTmaThreads, smem);
    if (e != cudaSuccess) return e;
    if (o.per_sm < 1) o.per_sm = 1;
    o.attr = true;
  }
  *out = &o;
  return cudaSuccess;
}

// TMA mode of a grid: 1 when every face carries the PEC column mask, 2
// when the four x/y faces do (z faces free), else 0; never with PMC faces.
template <typename T>
static int tma_mode(const FitParams<T>& p) {
  if (!p.has_pec || p.has_pmc) return 0;
  for (int f = 0; f < 4; f++)
    if (p.pec_face[f] != 0) return 0;
  return (p.pec_face[4] == 0 && p.pec_face[5] == 0) ? 1 : 2;
}

template <typename T, bool SM, int JM, int MODE, bool DESC, int TW>
static cudaError_t launch_tma_variant(const FitParams<T>& p, long long step, cudaStream_t st,
                                      int KC) {
  using S = TShape<TW>;
  using G = TmaGeom<T, (MODE != 0), TW>;
  TmaMaps maps;
  for (int d = 0; d < 3; d++) {
    if (!encode_comp<T>(&maps.e[d], p.E_in + d * p.N, p.Nx, p.Ny, p.Nz, G::ebx, S::BY) ||
        !encode_comp<T>(&maps.h[d], p.H_in + d * p.N, p.Nx, p.Ny, p.Nz, G::hbx, S::HBY))
      return cudaErrorInvalidValue;
  }
  TmaOcc* occ = nullptr;
  cudaError_t e = tma_occupancy<T, SM, JM, MODE, DESC, TW>(&occ);
  if (e != cudaSuccess) return e;
  const int span_x = MODE ? p.Nx : p.Nx - 4, span_y = MODE ? p.Ny : p.Ny - 4;
  const int planes = MODE == 1 ? p.Nz : p.Nz - 4;
  const int gx = (span_x + S::TX - 1) / S::TX, gy = (span_y + S::TY - 1) / S::TY;
  if (KC <= 0)
    KC = tma_auto_kc((long long)gx * gy, planes, (long long)occ->sms * occ->per_sm);
  const int gz = (planes + KC - 1) / KC;
  timer_begin(st);
  k_tma<T, SM, JM, MODE, DESC, TW><<<dim3(gx, gy, gz), kTmaThreads,
                                     TmaLayout<T, (MODE != 0), TW>::bytes, st>>>(p, maps, step,
                                                                                 KC);
  timer_end(st);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (MODE == 1) return cudaSuccess;
  // shell (MODE 2: the four boundary planes only): H from the old state, then
  // E from the new H (the H the shell E rows read is in H_out once k_tma is
  // done)
  return launch_shell_pair<T>(p, step, st, MODE == 2);
}

// One step with the TMA kernel in the mode the faces allow (see k_tma), on
// 64x8 tiles (rows 8 or 0, the faster on B200 at 256x256x512 in FP64 and
// FP32) or 32x16 tiles (rows 16).
template <typename T>
cudaError_t launch_tma(const FitParams<T>& p, long long step, cudaStream_t st, int KC,
                       int rows) {
  const bool sm_table = p.n_mat <= kMatSmem && p.id_bytes == 1;
  const int jm = p.j_mode == WK_J_SIGMA_E ? 1 : (p.j_mode == WK_J_ARRAY ? 2 : 0);
  const int mode = tma_mode(p);
  const bool desc = p.h_desc != 0;
  const bool w32 = rows == 16;
#define WK_TMA_WIDTH(SMV, JMV, MV, DV)                                                \
  {                                                                                   \
    if (w32) return launch_tma_variant<T, SMV, JMV, MV, DV, 32>(p, step, st, KC);     \
    return launch_tma_variant<T, SMV, JMV, MV, DV, 64>(p, step, st, KC);              \
  }
#define WK_TMA_MODES(SMV, JMV, DV)                                                    \
  {                                                                                   \
    if (mode == 1) WK_TMA_WIDTH(SMV, JMV, 1, DV)                                      \
    if (mode == 2) WK_TMA_WIDTH(SMV, JMV, 2, DV)                                      \
    WK_TMA_WIDTH(SMV, JMV, 0, DV)                                                     \
  }
#define WK_TMA_CASE(SMV, JMV)                                                         \
  if (sm_table == SMV && jm == JMV) {                                                 \
    if (desc) WK_TMA_MODES(SMV, JMV, true)                                            \
    WK_TMA_MODES(SMV, JMV, false)                                                     \
  }
  WK_TMA_CASE(true, 0) WK_TMA_CASE(true, 1) WK_TMA_CASE(true, 2)
  WK_TMA_CASE(false, 0) WK_TMA_CASE(false, 1) WK_TMA_CASE(false, 2)
#undef WK_TMA_CASE
#undef WK_TMA_MODES
#undef WK_TMA_WIDTH
  return cudaErrorInvalidValue;
}

// Launches per step of the TMA schedule for these parameters: 1 (every face
// PEC-masked) or 3 (TMA kernel + two shell launches).
template <typename T>
int tma_launches_per_step(const FitParams<T>& p) {
  return tma_mode(p) == 1 ? 1 : 3;
}

template int tma_launches_per_step<double>(const FitParams<double>&);
template int tma_launches_per_step<float>(const FitParams<float>&);
template bool tma_supported<double>(const FitParams<double>&);
template bool tma_supported<float>(const FitParams<float>&);
template cudaError_t launch_tma<double>(const FitParams<double>&, long long, cudaStream_t, int,
                                        int);
template cudaError_t launch_tma<float>(const FitParams<float>&, long long, cudaStream_t, int, int);

}  // namespace wk
