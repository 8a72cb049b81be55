// Device code of the FP32-compensated TMA step (sm_100a), shared by the
// one-grid launch (fit_tma_comp.cu) and the batched persistent launch
// (fit_batch.cu).
//
// State: float E, H plus bf16 compensation words (fit_comp.cuh); every update
// is a Kahan step y = delta + c followed by TwoSum(v, y), so v + c keeps ~32
// significant bits over many steps.  The update factors are formed in FP64
// from the FP64 metric and material tables and rounded once to float
// (dt folded in); the rows then run in float.
//
// The face modes are those of the FP64 kernel (k_tma): the interior with
// shell launches, all of x and y, or the whole grid.  Block (bx, by, bz) owns
// the tile i in [i0, i0+TW), j in [j0, j0+512/TW) of planes [k0, k0+KC)
// (TW = 64, or 32 for batched instances: CShape) and marches in z.  An idle
// lane of warp 9 issues cp.async.bulk.tensor loads (no
// multicast) of E (three planes in a ring), H (two planes) and, with
// Nx % 8 == 0, the bf16 compensation words of plane k with H(k), into shared
// memory, each slot completing on its own mbarrier; the loads of E(k+2) and
// H(k+1) go out at the start of plane k.
//
// Threads work on pairs of cells (i, i+1) with packed f32x2 arithmetic:
// warps 0-7 own the 256 pairs of the tile (64x8: row = warp, pair = lane)
// in both half-steps, warp 8 the pairs of the halo row j0-1, and lanes of
// warp 9 the halo column i0-1 (single cells).  The halo H is recomputed with the
// same compensated update as its owner's, so it is the value the owner
// stores.  The new Hx, Hy of a tile pair stay in registers as H(k-1) of the
// next plane.  The material ids and the FP64 inputs of the per-plane factor
// rows go into a 3-slot ring by cp.async two planes ahead; the float rows of
// plane k+1 are formed at the end of plane k.  Every mbarrier wait is
// bounded: on timeout the block sets the status word, waits (bounded) for
// its loads in flight and returns.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/wakis_b200.h"
#include "fit_comp.cuh"
#include "fit_common.cuh"
#include "fit_kernels.cuh"
#include "tma_util.cuh"

namespace wk {

constexpr int cES = 3, cHS = 2;
static_assert(cES == 3 && cHS == 2, "the step loop counts the ring slots for 3 E and 2 H slots");
constexpr int cThreads = 320;
constexpr int cMat = 64;                  // materials (16 floats each) in smem
constexpr int cMatW = 16;

// Tile shape: TW columns x 512/TW rows.  Warps 0-7 hold the 256 pairs of
// cells of the tile (TW/2 pairs a row, 64/TW rows a warp), warp 8 the TW/2
// pairs of the halo row, warp 9 the 512/TW + 1 cells of the halo column.
// 64x8 is the one-grid kernel's; 32x16 fills the lanes of grids whose x
// extent lies just above a multiple of 64 better (batched instances).
template <int TW>
struct CShape {
  static_assert(TW == 64 || TW == 32, "tile widths 64 and 32");
  static constexpr int TX = TW, TY = 512 / TW;
  static constexpr int PL = TX / 2;           // pairs (lanes) per tile row
  static constexpr int BX = TX + 4;           // E box (interior) and H box width
  static constexpr int BY = TY + 2;           // E box rows, from j0-1
  static constexpr int HBY = TY + 1;          // H and compensation box rows
  static constexpr int EW = TX + 2;           // Hs row: index eb*EW + ea + 1
  static constexpr int Ext = EW * (TY + 1);
  // per-plane factor rows (floats): H x-row (per ext row j, TY+1 entries
  // padded to an even count), H y-row (per ext column i, stored at ea+1 so
  // that pairs are 8-byte aligned), E x-row (per tile row), E y-row (per
  // tile column); dt folded in
  static constexpr int HX = (TY + 2) / 2 * 2;
  static constexpr int R_HXA = 0, R_HXB = HX, R_HYA = 2 * HX, R_HYB = R_HYA + TX + 2,
                       R_EXA = R_HYB + TX + 2, R_EXB = R_EXA + TY, R_EYA = R_EXB + TY,
                       R_EYB = R_EYA + TX, Row = R_EYB + TX;
  static_assert(Row <= cThreads, "one factor-row entry per thread");
};
// the one-grid kernel's shape
constexpr int cTX = CShape<64>::TX, cTY = CShape<64>::TY;
constexpr int cBX = CShape<64>::BX, cBY = CShape<64>::BY, cHBY = CShape<64>::HBY;

struct CompMaps {
  CUtensorMap e[3];
  CUtensorMap h[3];
  CUtensorMap c[6];        // compensation words (CT): Hc x/y/z, then Ec x/y/z
};

// FULL (every face PEC-masked): tiles from i0 = TW bx cover the whole grid
// and both boxes start at i0-4 (16-byte aligned): E TW+8 wide, H TW+4 wide.
// The compensation-word boxes (CT) are TY+1 rows from j0-1 and start at an
// x that is a multiple of 8 (16 bytes of bf16 words): i0-8, TW+16 wide
// (FULL), or i0-2, TW+8 wide.
template <bool FULL, int TW = 64>
struct CGeom {
  using S = CShape<TW>;
  static constexpr int ebx = FULL ? S::TX + 8 : S::BX;     // E box width
  static constexpr int hbx = S::BX;                        // H box width
  static constexpr int xo = FULL ? 3 : 1;                  // box x of ext column 0
  static constexpr int xs_off = FULL ? 4 : 2;              // box start = i0 - xs_off
  static constexpr int cbx = FULL ? S::TX + 16 : S::TX + 8;   // compensation box width
  static constexpr int cxs_off = FULL ? 8 : 2;                // its start = i0 - cxs_off
  static constexpr int cxo = cxs_off - 1;                     // its x of ext column 0
};

template <bool FULL, bool CT, int TW = 64>
struct CLayout {
  using S = CShape<TW>;
  using G = CGeom<FULL, TW>;
  static constexpr int eslot = round128(G::ebx * S::BY * 4);
  static constexpr int hslot = round128(G::hbx * S::HBY * 4);
  static constexpr int cslot = CT ? round128(G::cbx * S::HBY * 2) : 0;
  static constexpr int e_off = 0;
  static constexpr int h_off = e_off + cES * 3 * eslot;
  static constexpr int c_off = h_off + cHS * 3 * hslot;      // [cHS][6][cslot]
  static constexpr int hs_off = c_off + cHS * 6 * cslot;
  static constexpr int row_off = hs_off + round128(3 * S::Ext * 4);
  static constexpr int raw_off = row_off + round128(2 * S::Row * 4);   // [3][Row][2] doubles
  static constexpr int id_off = raw_off + round128(3 * S::Row * 16);   // [3][threads] u64
  static constexpr int mat_off = id_off + round128(3 * cThreads * 8);
  static constexpr int bar_off = mat_off + round128(cMat * cMatW * 4);
  static constexpr int bytes = bar_off + (cES + cHS) * 8 + 128;
};

__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b, one rounding: fma(b, -1, a)
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}
__device__ __forceinline__ float2 ld2(const float* p) {
  return *reinterpret_cast<const float2*>(p);
}
__device__ __forceinline__ void st2(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }
__device__ __forceinline__ float2 bcast(float v) { return make_float2(v, v); }

// two bf16 words (cell i in the low half) <-> float2
__device__ __forceinline__ float2 cdec2(uint32_t w) {
  return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
}
__device__ __forceinline__ uint32_t cenc2(float2 e) {
  uint32_t w;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(w) : "f"(e.y), "f"(e.x));
  return w;
}
// v + c + delta -> (t, c'): Kahan step, then TwoSum
__device__ __forceinline__ float2 cadd2(float2 v, uint32_t& w, float2 delta) {
  const float2 y = add2(delta, cdec2(w));
  const float2 t = add2(v, y);
  const float2 bp = sub2(t, v);
  const float2 ap = sub2(t, bp);
  const float2 e = add2(sub2(v, ap), sub2(y, bp));
  w = cenc2(e);
  return t;
}

// Factor-row entry r of plane q = dt * f[q] * g[q], f an inverse area and g
// a length (FP64, rounded once to float).  RowSrc holds, per thread, where f
// and g of its entry live (element q*fs of f, q*gs of g); the loads of the
// next plane are issued while this plane is computed.
struct RowSrc {
  const double* f;
  const double* g;
  int fs, gs;
};

template <int TW>
__device__ __forceinline__ RowSrc row_src(const FitParams<double>& p, int r, int i0, int j0) {
  using S = CShape<TW>;
  const int Nx = p.Nx, Ny = p.Ny;
  RowSrc s{nullptr, nullptr, 0, 0};
  if (r < S::R_HXB) {
    const int j = j0 - 1 + (r - S::R_HXA);
    if (r - S::R_HXA < S::TY + 1 && j >= 0 && j < Ny) s = RowSrc{p.iAx + j, p.Ly + j, Ny, 0};
  } else if (r < S::R_HYA) {
    const int j = j0 - 1 + (r - S::R_HXB);
    if (r - S::R_HXB < S::TY + 1 && j >= 0 && j < Ny) s = RowSrc{p.iAx + j, p.Lz, Ny, 1};
  } else if (r < S::R_HYB) {
    const int i = i0 - 2 + (r - S::R_HYA);
    if (r > S::R_HYA && i >= 0 && i < Nx) s = RowSrc{p.iAy + i, p.Lx + i, Nx, 0};
  } else if (r < S::R_EXA) {
    const int i = i0 - 2 + (r - S::R_HYB);
    if (r > S::R_HYB && i >= 0 && i < Nx) s = RowSrc{p.iAy + i, p.Lz, Nx, 1};
  } else if (r < S::R_EXB) {
    const int j = j0 + (r - S::R_EXA);
    if (j < Ny) s = RowSrc{p.itAx + j, p.tLy + j, Ny, 0};
  } else if (r < S::R_EYA) {
    const int j = j0 + (r - S::R_EXB);
    if (j < Ny) s = RowSrc{p.itAx + j, p.tLz, Ny, 1};
  } else if (r < S::R_EYB) {
    const int i = i0 + (r - S::R_EYA);
    if (i < Nx) s = RowSrc{p.itAy + i, p.tLx + i, Nx, 0};
  } else if (r < S::Row) {
    const int i = i0 + (r - S::R_EYB);
    if (i < Nx) s = RowSrc{p.itAy + i, p.tLz, Nx, 1};
  }
  return s;
}
// f and g of plane q into two shared-memory doubles by cp.async (zeros
// outside the grid; `any` is a valid address that is then not read)
__device__ __forceinline__ void row_stage(const RowSrc& s, int q, int Nz, const double* any,
                                          double* dst) {
  const bool v = s.f && q >= 0 && q < Nz;
  cp_async<8>(dst, v ? s.f + (long long)q * s.fs : any, v);
  cp_async<8>(dst + 1, v ? s.g + (long long)q * s.gs : any, v);
}
__device__ __forceinline__ float row_value(double dt, double f, double g) {
  return (float)((dt * f) * g);
}

// IdT: material id type; SIG: the J entering a row is sigma * E (the
// conductive J mode) rather than zero; CT: the compensation words of plane k
// arrive by TMA with H(k) (row pitch Nx % 8 == 0) instead of per-thread
// loads issued one plane ahead.  MODE 0: interior cells, the shell
// follows in separate launches.  MODE 1: every face carries the PEC column
// mask (no PMC); the tiles cover the whole grid and the cells on or next to
// a face use the same rows with the masked entries set to zero (E entries
// tangential to a face they lie on enter no H row; E rows tangential to
// their face get no curl; wrapped flat-offset neighbours are always
// masked), so no shell launch follows.  MODE 2: the x/y faces are PEC-masked
// and the z faces are not; the tiles cover all of x and y for the planes
// 2 <= k <= Nz-3 and the shell launches cover only the four boundary planes.
//
// comp_tile is the work of one block of the step: the tile (bx, by) of the
// z chunk bz at step index `step` (already resolved from the device step
// counter), in the dynamic shared memory `sm_raw`.  CTM: 0 = compensation
// words by per-thread loads, 1 = by TMA (CT above), 2 = chosen at run time
// by `ct_run` (the batched kernel; the shared-memory layout then always
// holds the compensation slots).  BATCH: the block runs further tiles after
// this one, so the mbarriers are invalidated at the end.  Returns false when
// a load wait ran out (the status word is then set).
template <typename IdT, bool SIG, int MODE, int CTM, bool BATCH, int TW = 64>
__device__ __forceinline__ bool comp_tile(const FitParams<double>& p, const CompState& cs,
                                          const CompMaps& maps, long long step, int KC,
                                          unsigned bx, unsigned by, unsigned bz, bool ct_run,
                                          unsigned char* sm_raw) {
  constexpr bool FULL = MODE != 0;     // tiles cover x and y entirely
  constexpr bool ZFULL = MODE == 1;    // ... and every plane
  if (!BATCH) step = step_index(p, step);
  const bool CT = CTM == 2 ? ct_run : CTM == 1;
  using S = CShape<TW>;
  using Lay = CLayout<(MODE != 0), (CTM != 0), TW>;
  using G = CGeom<(MODE != 0), TW>;
  constexpr int SE = Lay::eslot / 4, SH = Lay::hslot / 4, SC = Lay::cslot / 2;
  constexpr int EBX = G::ebx, XO = G::xo;
  unsigned char* sm = sm_raw + ((128 - (smem_u32(sm_raw) & 127)) & 127);
  float* Eb = reinterpret_cast<float*>(sm + Lay::e_off);
  float* Hb = reinterpret_cast<float*>(sm + Lay::h_off);
  uint16_t* Cb = reinterpret_cast<uint16_t*>(sm + Lay::c_off);   // [cHS][6][SC]
  float* Hs = reinterpret_cast<float*>(sm + Lay::hs_off);     // [3][Ext]
  float* Rw = reinterpret_cast<float*>(sm + Lay::row_off);    // [2][Row]
  double* Rraw = reinterpret_cast<double*>(sm + Lay::raw_off); // [3][Row][2] f, g
  uint64_t* sidw = reinterpret_cast<uint64_t*>(sm + Lay::id_off);  // [3][threads] id words
  float* mt = reinterpret_cast<float*>(sm + Lay::mat_off);    // [n_mat][16]
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + Lay::bar_off);

  const int Nx = p.Nx, Ny = p.Ny;
  const long long N = p.N, NxNy = p.NxNy;
  const int Nz = p.Nz;
  const int i0 = (FULL ? 0 : 2) + bx * S::TX, j0 = (FULL ? 0 : 2) + by * S::TY;
  const int k0 = (ZFULL ? 0 : 2) + bz * KC, k1 = min(k0 + KC, ZFULL ? Nz : Nz - 2);
  const int xs = i0 - G::xs_off, ys = j0 - 1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // the producer (mbarrier set-up, TMA issue and waits) is the last lane of
  // warp 9, which owns no item
  const bool prod = tid == cThreads - 1;
  const int pstart = k0 - 1;
  const uint32_t e_bytes = 3u * EBX * S::BY * 4u;
  const uint32_t h_bytes = 3u * G::hbx * S::HBY * 4u + (CT ? 6u * G::cbx * S::HBY * 2u : 0u);

  if (prod) {
    for (int s = 0; s < cES + cHS; s++) mbar_init(&bar[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  auto issue_e = [&](int q) {
    const int slot = (q - pstart) % cES;
    mbar_expect_tx(&bar[slot], e_bytes);
#pragma unroll
    for (int d = 0; d < 3; d++)
      tma_load_3d(Eb + (slot * 3 + d) * SE, &maps.e[d], xs, ys, q, &bar[slot]);
  };
  auto issue_h = [&](int q) {
    const int slot = (q - pstart) % cHS;
    mbar_expect_tx(&bar[cES + slot], h_bytes);
#pragma unroll
    for (int d = 0; d < 3; d++)
      tma_load_3d(Hb + (slot * 3 + d) * SH, &maps.h[d], xs, ys, q, &bar[cES + slot]);
    if (CT) {
#pragma unroll
      for (int c = 0; c < 6; c++)
        tma_load_3d(Cb + (slot * 6 + c) * SC, &maps.c[c], i0 - G::cxs_off, ys, q,
                    &bar[cES + slot]);
    }
  };
  auto wait_e = [&](int q, long long lim) {
    return mbar_wait(&bar[(q - pstart) % cES], (uint32_t)(((q - pstart) / cES) & 1), lim);
  };
  auto wait_h = [&](int q, long long lim) {
    return mbar_wait(&bar[cES + (q - pstart) % cHS], (uint32_t)(((q - pstart) / cHS) & 1), lim);
  };
  int e_hi = pstart - 1, h_hi = pstart - 1;
  if (prod) {
    for (int q = pstart; q <= min(pstart + cES - 1, k1); q++) { issue_e(q); e_hi = q; }
    for (int q = pstart; q <= min(pstart + cHS - 1, k1 - 1); q++) { issue_h(q); h_hi = q; }
  }

  // role: 0 tile pair, 1 halo-row pair, 2 halo-column cell, 3 idle
  const int role = warp < 8 ? 0
                 : (warp == 8 ? (lane < S::PL ? 1 : 3) : (lane < S::TY + 1 ? 2 : 3));
  int ea, eb;
  if (role == 0) { ea = 2 * (lane % S::PL) + 1; eb = warp * (32 / S::PL) + lane / S::PL + 1; }
  else if (role == 1) { ea = 2 * lane + 1; eb = 0; }
  else { ea = 0; eb = lane; }
  const int ci = i0 - 1 + ea, cj = j0 - 1 + eb;          // first cell of the item
  const bool pair = role < 2;
  const bool hval = FULL ? (role < 3 && ci >= 0 && ci <= Nx - 1 && cj >= 0 && cj <= Ny - 1)
                         : (role < 3 && ci <= Nx - 3 && cj <= Ny - 3);
  const bool eval = role == 0 && hval;
  const int bi = eb * EBX + ea + XO;                      // E box index
  const int hbi = eb * G::hbx + ea + XO;                  // H box index
  // face flags (FULL) of the item's cells (x per lane) and of the +x / +y
  // neighbours (a wrapped neighbour counts as on the face)
  const bool xf0a = ci == 0 || ci == Nx - 1, xf0b = ci + 1 == Nx - 1;
  const bool xf1a = ci + 1 >= Nx - 1, xf1b = ci + 2 >= Nx - 1;
  const bool yf0 = cj == 0 || cj == Ny - 1, yf1 = cj + 1 >= Ny - 1;
  const bool nearface = hval && (xf0a || xf1a || (pair && (xf0b || xf1b)) || yf0 || yf1);
  const bool warp_face = FULL && __any_sync(0xffffffffu, nearface);
  const int hi = eb * S::EW + ea + 1;                       // Hs index
  const int cix = eb * G::cbx + ea + G::cxo;              // compensation box index
  const long long nb = ci + (long long)cj * Nx;           // flat index at k = 0
  // the item holds a cell of the Ez capture window (plane-invariant test)
  const bool cap_item = eval && p.cap_on && cj >= p.cap_j0 && cj < p.cap_j0 + p.cap_nj &&
                        ci + 1 >= p.cap_i0 && ci < p.cap_i0 + p.cap_ni;

  // plane-invariant z-row factors
  float2 hza = bcast(0.f), hzb = bcast(0.f), eza = bcast(0.f), ezb = bcast(0.f);
  if (hval) {
    const double dt = p.dt;
    float a[2], b[2], c[2], d[2];
    for (int u = 0; u < (pair ? 2 : 1); u++) {
      const int i = ci + u;
      const double iaz = p.iAz[i + (long long)cj * Nx], itaz = p.itAz[i + (long long)cj * Nx];
      a[u] = (float)((dt * iaz) * p.Lx[i]);
      b[u] = (float)((dt * iaz) * p.Ly[cj]);
      c[u] = (float)((dt * itaz) * p.tLx[i]);
      d[u] = (float)((dt * itaz) * p.tLy[cj]);
    }
    hza = make_float2(a[0], pair ? a[1] : 0.f);
    hzb = make_float2(b[0], pair ? b[1] : 0.f);
    eza = make_float2(c[0], pair ? c[1] : 0.f);
    ezb = make_float2(d[0], pair ? d[1] : 0.f);
  }
  // float material table: imu, ieps, dt*ieps, dt*ieps*sigma
  for (int q = tid; q < p.n_mat * 3; q += cThreads) {
    const int m = q / 3, d = q - m * 3;
    const double* m0 = p.mat + 9 * m;
    mt[m * cMatW + d] = (float)m0[3 + d];
    mt[m * cMatW + 4 + d] = (float)m0[d];
    mt[m * cMatW + 8 + d] = (float)(p.dt * m0[d]);
    mt[m * cMatW + 12 + d] = (float)((p.dt * m0[d]) * m0[6 + d]);
  }
  // material ids of the item at plane q, staged by cp.async (with the
  // factor-row inputs, two planes ahead) as the aligned 4-byte word that
  // holds them (8 bytes for a pair of 4-byte ids).  A pair starts at an even
  // cell, so its ids share the word.  With Nx % 4 == 0 the array length in
  // bytes is a multiple of 4 (every word lies inside it) and the position
  // of the ids in their word is the same on every plane.
  const IdT* idp = static_cast<const IdT*>(p.mat_id) + nb;
  const int id_sh = 8 * (int)((nb * (long long)sizeof(IdT)) & 3);
  auto stage_ids = [&](int q, const IdT* a, uint64_t* dst) {
    if (q < 0) *dst = 0ull;
    else if (pair && sizeof(IdT) == 4) cp_async<8>(dst, a, true);
    else cp_async<4>(dst, reinterpret_cast<const void*>((uintptr_t)a & ~(uintptr_t)3), true);
  };
  auto read_ids = [&](const uint64_t* src, int& a0, int& a1) {
    const uint64_t w = *src;
    if constexpr (sizeof(IdT) == 4) {
      a0 = (int)(uint32_t)w;
      a1 = pair ? (int)(uint32_t)(w >> 32) : a0;
    } else {
      constexpr int bits = 8 * (int)sizeof(IdT);
      constexpr uint32_t m = (1u << bits) - 1u;
      const uint32_t x = (uint32_t)w >> id_sh;
      a0 = (int)(x & m);
      a1 = pair ? (int)((x >> bits) & m) : a0;
    }
  };
  auto load_comp = [&](const comp_t* base, int q, uint32_t* w) {
    const long long n = nb + (long long)q * NxNy;
#pragma unroll
    for (int d = 0; d < 3; d++)
      w[d] = pair ? *reinterpret_cast<const uint32_t*>(base + d * N + n)
                  : (uint32_t)base[d * N + n];
  };
  // compensation words from the staged box (CT): components c0..c0+2
  auto read_comp = [&](const uint16_t* Ck, int c0, uint32_t* w) {
#pragma unroll
    for (int d = 0; d < 3; d++)
      w[d] = pair ? *reinterpret_cast<const uint32_t*>(Ck + (c0 + d) * SC + cix)
                  : (uint32_t)Ck[(c0 + d) * SC + cix];
  };
  uint32_t hc[3] = {0, 0, 0}, ec[3] = {0, 0, 0};
  if (!CT && hval && pstart >= 0) load_comp(cs.Hc_in, pstart, hc);
  // The f, g inputs of factor-row entry tid of plane q go into ring slot
  // (q - pstart) % 3 by cp.async two planes ahead (one group per plane and
  // thread); the float row of plane q is formed at the end of plane q-1.
  const RowSrc rsrc = row_src<TW>(p, tid < S::Row ? tid : S::Row, i0, j0);
  // slot = (q - pstart) % 3, ida = the ids of the item at plane q
  auto stage_rows = [&](int q, int slot, const IdT* ida) {
    if (q < k1) {
      if (tid < S::Row) row_stage(rsrc, q, Nz, p.Lz, Rraw + (slot * S::Row + tid) * 2);
      if (hval) stage_ids(q, ida, sidw + slot * cThreads + tid);
    }
    cp_async_commit();
  };
  auto form_row = [&](int q, int slot) {
    if (tid < S::Row) {
      const double* v = Rraw + (slot * S::Row + tid) * 2;
      Rw[(q & 1) * S::Row + tid] = row_value(p.dt, v[0], v[1]);
    }
  };
  stage_rows(pstart, 0, idp + (long long)pstart * NxNy);
  stage_rows(pstart + 1, 1, idp + (long long)(pstart + 1) * NxNy);
  cp_async_wait<1>();
  form_row(pstart, 0);
  // per-plane cursors: the ids of plane pl+2, the outputs of the item at
  // plane pl; ring slots of E(pl), H(pl) and of the staged inputs of pl,
  // counted instead of taken modulo
  const IdT* idq = idp + (long long)(pstart + 2) * NxNy;
  const long long nq = nb + (long long)pstart * NxNy;
  float* hq = cs.H_out + nq;
  float* eq = cs.E_out + nq;
  comp_t* hcq = cs.Hc_out + nq;
  comp_t* ecq = cs.Ec_out + nq;
  int se = 0, sh = 0;

  float2 hxp = bcast(0.f), hyp = bcast(0.f);
  const float2 zero2 = bcast(0.f);

  bool ok = true;
  int pl = pstart;
  const long long lim = loop_wait_ns(p.wait_ns);   // step-loop waits; the drain keeps kWaitNs
  for (; pl < k1; pl++) {
    bool got = true;
    if (prod) got = wait_e(pl, lim) && wait_e(pl + 1, lim) && wait_h(pl, lim);
    ok = __syncthreads_and(got);
    if (!ok) break;
    const bool prologue = pl == pstart;
    if (prod && !prologue) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      if (pl + cES - 1 <= k1) { issue_e(pl + cES - 1); e_hi = pl + cES - 1; }
      if (pl + cHS - 1 <= k1 - 1) { issue_h(pl + cHS - 1); h_hi = pl + cHS - 1; }
    }
    const int se1 = se == cES - 1 ? 0 : se + 1;     // slot of plane pl+1
    const int se2 = se == 0 ? cES - 1 : se - 1;      // slot of plane pl+2
    stage_rows(pl + 2, se2, idq);  // the ring slot of plane pl-1 is free
    int id0 = 0, id1 = 0;
    if (hval) read_ids(sidw + se * cThreads + tid, id0, id1);
    // prefetch the compensation words of plane pl+1 (without CT)
    const bool more = pl + 1 < k1;
    uint32_t nhc[3] = {0, 0, 0}, nec[3] = {0, 0, 0};
    if (!CT && more) {
      if (hval) load_comp(cs.Hc_in, pl + 1, nhc);
      if (eval) load_comp(cs.Ec_in, pl + 1, nec);
    }
    const float* Ek = Eb + se * 3 * SE;
    const float* Ek1 = Eb + se1 * 3 * SE;
    const float* Hk = Hb + sh * 3 * SH;
    const uint16_t* Ck = Cb + sh * 6 * SC;
    const float* R = Rw + (pl & 1) * S::Row;
    const long long n = nb + (long long)pl * NxNy;

    // plane face flags (MODE 1): at the plane and of the +z neighbour
    const bool zf0 = ZFULL && (pl == 0 || pl == Nz - 1), zf1 = ZFULL && pl + 1 >= Nz - 1;
    const bool masked = FULL && (warp_face || zf0 || zf1);

    // ---- new H of the owned item (tile pairs only in the prologue; FULL:
    // no H below plane 0, items outside the grid hold 0)
    float2 hxn = zero2, hyn = zero2;
    if (FULL && role < 3 && !hval) {
      if (pair) {
        st2(Hs + hi, zero2); st2(Hs + S::Ext + hi, zero2); st2(Hs + 2 * S::Ext + hi, zero2);
      } else {
        Hs[hi] = 0.f; Hs[S::Ext + hi] = 0.f; Hs[2 * S::Ext + hi] = 0.f;
      }
    }
    if (hval && (!prologue || role == 0) && !(ZFULL && pl < 0)) {
      const float* m0 = mt + id0 * cMatW;
      const float* m1 = mt + id1 * cMatW;
      float2 ex0, ey0, ez0, ey1, ez1, ex2, ez2, ex3, ey3, hx, hy, hz, ya, yb;
      if (pair) {
        ex0 = ld2(Ek + bi); ey0 = ld2(Ek + SE + bi); ez0 = ld2(Ek + 2 * SE + bi);
        ey1 = make_float2(ey0.y, Ek[SE + bi + 2]);
        ez1 = make_float2(ez0.y, Ek[2 * SE + bi + 2]);
        ex2 = ld2(Ek + bi + EBX); ez2 = ld2(Ek + 2 * SE + bi + EBX);
        ex3 = ld2(Ek1 + bi); ey3 = ld2(Ek1 + SE + bi);
        hx = ld2(Hk + hbi); hy = ld2(Hk + SH + hbi); hz = ld2(Hk + 2 * SH + hbi);
        ya = ld2(R + S::R_HYA + ea + 1); yb = ld2(R + S::R_HYB + ea + 1);
      } else {
        ex0 = bcast(Ek[bi]); ey0 = bcast(Ek[SE + bi]); ez0 = bcast(Ek[2 * SE + bi]);
        ey1 = bcast(Ek[SE + bi + 1]); ez1 = bcast(Ek[2 * SE + bi + 1]);
        ex2 = bcast(Ek[bi + EBX]); ez2 = bcast(Ek[2 * SE + bi + EBX]);
        ex3 = bcast(Ek1[bi]); ey3 = bcast(Ek1[SE + bi]);
        hx = bcast(Hk[hbi]); hy = bcast(Hk[SH + hbi]); hz = bcast(Hk[2 * SH + hbi]);
        ya = bcast(R[S::R_HYA + ea + 1]); yb = bcast(R[S::R_HYB + ea + 1]);
      }
      if (masked && !p.faces_clean) {
        // E column entries tangential to a face they lie on are masked
        // (with faces_clean those entries are +0 already)
        auto m2 = [](float2 v, bool ma, bool mb) {
          return make_float2(ma ? 0.f : v.x, mb ? 0.f : v.y);
        };
        ex0 = m2(ex0, yf0 || zf0, yf0 || zf0);
        ey0 = m2(ey0, xf0a || zf0, xf0b || zf0);
        ez0 = m2(ez0, xf0a || yf0, xf0b || yf0);
        ey1 = m2(ey1, xf1a || zf0, xf1b || zf0);
        ez1 = m2(ez1, xf1a || yf0, xf1b || yf0);
        ex2 = m2(ex2, yf1 || zf0, yf1 || zf0);
        ez2 = m2(ez2, xf0a || yf1, xf0b || yf1);
        ex3 = m2(ex3, yf0 || zf1, yf0 || zf1);
        ey3 = m2(ey3, xf0a || zf1, xf0b || zf1);
      }
      const float4 u0 = *reinterpret_cast<const float4*>(m0);
      const float4 u1 = *reinterpret_cast<const float4*>(m1);
      const float2 mux = make_float2(u0.x, u1.x), muy = make_float2(u0.y, u1.y),
                   muz = make_float2(u0.z, u1.z);
      // S_x = a (ey0 - ey3) + b (ez2 - ez0)   (a = dt iAx Ly imu_x, b = dt iAx Lz imu_x)
      const float2 sx = fma2(mul2(mux, bcast(R[S::R_HXA + eb])), sub2(ey0, ey3),
                             mul2(mul2(mux, bcast(R[S::R_HXB + eb])), sub2(ez2, ez0)));
      // S_y = a (ex3 - ex0) + b (ez0 - ez1)   (a = dt iAy Lx imu_y, b = dt iAy Lz imu_y)
      const float2 sy = fma2(mul2(muy, ya), sub2(ex3, ex0), mul2(mul2(muy, yb), sub2(ez0, ez1)));
      // S_z = a (ex0 - ex2) + b (ey1 - ey0)   (a = dt iAz Lx imu_z, b = dt iAz Ly imu_z)
      const float2 sz = fma2(mul2(muz, hza), sub2(ex0, ex2), mul2(mul2(muz, hzb), sub2(ey1, ey0)));
      const float2 m1v = bcast(-1.0f);
      if (CT) read_comp(Ck, 0, hc);
      hx = cadd2(hx, hc[0], mul2(sx, m1v));
      hy = cadd2(hy, hc[1], mul2(sy, m1v));
      hz = cadd2(hz, hc[2], mul2(sz, m1v));
      if (pair) {
        st2(Hs + hi, hx); st2(Hs + S::Ext + hi, hy); st2(Hs + 2 * S::Ext + hi, hz);
      } else {
        Hs[hi] = hx.x; Hs[S::Ext + hi] = hy.x; Hs[2 * S::Ext + hi] = hz.x;
      }
      hxn = hx;
      hyn = hy;
      if (role == 0 && !prologue) {
        float* const h1 = hq + N;
        comp_t* const hc1 = hcq + N;
        st2(hq, hx); st2(h1, hy); st2(h1 + N, hz);
        *reinterpret_cast<uint32_t*>(hcq) = hc[0];
        *reinterpret_cast<uint32_t*>(hc1) = hc[1];
        *reinterpret_cast<uint32_t*>(hc1 + N) = hc[2];
      }
    }
    __syncthreads();

    // ---- new E of the tile pair
    if (eval && !prologue) {
      const float* m0 = mt + id0 * cMatW;
      const float* m1 = mt + id1 * cMatW;
      const int b = eb - 1, a = ea - 1;
      const float2 hx0 = ld2(Hs + hi), hy0 = ld2(Hs + S::Ext + hi), hz0 = ld2(Hs + 2 * S::Ext + hi);
      const float2 hy1 = make_float2(Hs[S::Ext + hi - 1], hy0.x);
      const float2 hz1 = make_float2(Hs[2 * S::Ext + hi - 1], hz0.x);
      const float2 hx2 = ld2(Hs + hi - S::EW), hz2 = ld2(Hs + 2 * S::Ext + hi - S::EW);
      const float4 w0 = *reinterpret_cast<const float4*>(m0 + 4);
      const float4 w1 = *reinterpret_cast<const float4*>(m1 + 4);
      const float2 iex = make_float2(w0.x, w1.x), iey = make_float2(w0.y, w1.y),
                   iez = make_float2(w0.z, w1.z);
      const float4 s0 = *reinterpret_cast<const float4*>(m0 + 12);
      const float4 s1 = *reinterpret_cast<const float4*>(m1 + 12);
      const float2 sg[3] = {make_float2(s0.x, s1.x), make_float2(s0.y, s1.y),
                            make_float2(s0.z, s1.z)};
      // curl_x = c1 (hy3 - hy0) + c2 (hz0 - hz2)   (c1 = dt ieps_x itAx tLy, c2 = .. tLz)
      float2 cu[3];
      cu[0] = fma2(mul2(iex, bcast(R[S::R_EXA + b])), sub2(hyp, hy0),
                   mul2(mul2(iex, bcast(R[S::R_EXB + b])), sub2(hz0, hz2)));
      // curl_y = c1 (hx0 - hx3) + c2 (hz1 - hz0)   (c1 = dt ieps_y itAy tLx, c2 = .. tLz)
      cu[1] = fma2(mul2(iey, ld2(R + S::R_EYA + a)), sub2(hx0, hxp),
                   mul2(mul2(iey, ld2(R + S::R_EYB + a)), sub2(hz1, hz0)));
      // curl_z = c1 (hx2 - hx0) + c2 (hy0 - hy1)   (c1 = dt ieps_z itAz tLx, c2 = .. tLy)
      cu[2] = fma2(mul2(iez, eza), sub2(hx2, hx0), mul2(mul2(iez, ezb), sub2(hy0, hy1)));
      if (masked) {
        // E rows tangential to the face the cell lies on get no curl
        if (yf0 || zf0) cu[0] = zero2;
        cu[1] = make_float2((xf0a || zf0) ? 0.f : cu[1].x, (xf0b || zf0) ? 0.f : cu[1].y);
        cu[2] = make_float2((xf0a || yf0) ? 0.f : cu[2].x, (xf0b || yf0) ? 0.f : cu[2].y);
      }
      float2 ev[3] = {ld2(Ek + bi), ld2(Ek + SE + bi), ld2(Ek + 2 * SE + bi)};
      if (CT) read_comp(Ck, 3, ec);
      if (cap_item) {
#pragma unroll
        for (int u = 0; u < 2; u++) {
          Cell c;
          c.i = ci + u; c.j = cj; c.k = pl;
          const float v = u ? ev[2].y : ev[2].x;
          const comp_t q = (comp_t)(u ? (ec[2] >> 16) : (ec[2] & 0xffffu));
          capture(p, c, n + u, step, comp_value(v, q));
        }
      }
#pragma unroll
      for (int d = 0; d < 3; d++) {
        float2 jt = zero2;   // dt*ieps*J of the row
        if (SIG)
          jt = mul2(sg[d], ev[d]);
        if (d == 2 && cj == p.iys && (p.ixs == ci || p.ixs == ci + 1) &&
            (p.line_on || p.beam_on)) {
          const long long lt = step - p.line_step0;
          const double jb = p.line_on ? ((lt >= 0 && lt < p.line_nsteps)
                                             ? p.line[lt * p.Nz + pl] : 0.0)
                                      : beam_j(p, step, pl);
          if (p.ixs == ci) jt.x = (float)((double)m0[10] * jb);
          else jt.y = (float)((double)m1[10] * jb);
        }
        ev[d] = cadd2(ev[d], ec[d], sub2(cu[d], jt));
      }
      float* const e1 = eq + N;
      comp_t* const ec1 = ecq + N;
      st2(eq, ev[0]); st2(e1, ev[1]); st2(e1 + N, ev[2]);
      *reinterpret_cast<uint32_t*>(ecq) = ec[0];
      *reinterpret_cast<uint32_t*>(ec1) = ec[1];
      *reinterpret_cast<uint32_t*>(ec1 + N) = ec[2];
    }
    hxp = hxn;
    hyp = hyn;
    if (!CT) {
#pragma unroll
      for (int d = 0; d < 3; d++) {
        hc[d] = nhc[d];
        ec[d] = nec[d];
      }
    }
    if (more) {
      cp_async_wait<1>();        // this thread's row inputs and ids of plane pl+1
      form_row(pl + 1, se1);
    }
    idq += NxNy;
    hq += NxNy;
    eq += NxNy;
    hcq += NxNy;
    ecq += NxNy;
    se = se1;
    sh ^= 1;
  }
  cp_async_wait<0>();
  if (!ok) {
    if (prod) {
      if (p.status) atomicExch(p.status, 1);
      for (int q = pl; q <= e_hi; q++) wait_e(q, kWaitNs);
      for (int q = pl; q <= h_hi; q++) wait_h(q, kWaitNs);
    }
    __syncthreads();
  }
  if constexpr (BATCH) {
    // every wait of the tile has returned: the barriers can be reused
    __syncthreads();
    if (prod)
      for (int s = 0; s < cES + cHS; s++) mbar_inval(&bar[s]);
    __syncthreads();
    return ok;
  } else {
    return true;
  }
}


// 3-D tensor map of an (Nx, Ny, Nz) array of `esize`-byte elements (float
// or raw bf16 words) with a bx x by x 1 box
inline bool encode_3d(CUtensorMap* map, const void* base, int esize, int Nx, int Ny, int Nz, int bx,
               int by) {
  cuuint64_t gdim[3] = {(cuuint64_t)Nx, (cuuint64_t)Ny, (cuuint64_t)Nz};
  cuuint64_t gstr[2] = {(cuuint64_t)Nx * esize, (cuuint64_t)Nx * Ny * esize};
  cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  cuuint32_t est[3] = {1, 1, 1};
  const CUtensorMapDataType dt =
      esize == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16;
  CUresult r = tma_encode_fn()(map, dt, 3, const_cast<void*>(base), gdim, gstr, box, est,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace wk
