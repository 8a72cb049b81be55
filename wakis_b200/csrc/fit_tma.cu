// Fused FIT step with TMA-staged plane tiles (sm_100a).
//
// Interior cells only (2 <= i <= Nx-3, 2 <= j <= Ny-3, 2 <= k <= Nz-3); the
// two-cell shell runs afterwards in an H launch and an E launch.  Block
// (bx, by, bz) owns the tile
// i in [i0, i0+64), j in [j0, j0+8) of planes [k0, k0+KC) and marches in z.
// For plane k it needs E_old of planes k and k+1 on the box
// x in [i0-2, i0+66), y in [j0-1, j0+9) and H_old of plane k on
// x in [i0-2, i0+64), y in [j0-1, j0+8) (the boxes start at an even x, so
// the TMA x offset is 16-byte aligned).  Thread 0 issues cp.async.bulk.tensor
// loads of those boxes (one per field component, no multicast) into a ring of
// shared-memory slots, three planes of E and two of H, each slot completing
// on its own mbarrier; at the start of plane k the loads of E(k+2) and
// H(k+1) go out into the slots plane k-1 released.
//
// Per plane the block computes the new H on the tile plus its low halo row
// and column (single-coefficient rows; the halo is recomputed so that no
// block waits for another), a barrier, then the new E of the tile.  Each
// thread owns the same tile cells in both phases (320 threads: cells t and
// t+320 of the 512-cell tile; threads 192..264 also own one halo cell), so
// the new Hx, Hy of its tile cells stay in registers as H(k-1) of the next
// plane.  Material ids of the owned cells and the per-plane metric rows
// (iAx, iAy, itAx, itAy, Lz, tLz) of plane k+1 are loaded while plane k is
// computed; the plane-invariant metrics (Lx, Ly, iAz, ...) are loaded once.
// A chunk starting at k0 first forms the new H of plane k0-1 on its tile.
// Every mbarrier wait is bounded: on timeout the block records the failure
// in the status word, waits (bounded) for its loads in flight and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include "../../include/wakis_b200.h"
#include "abi_internal.h"
#include "fit_common.cuh"
#include "fit_kernels.cuh"
#include "tma_util.cuh"

namespace wk {

constexpr int kTX = 64, kTY = 8;
constexpr int kBX = kTX + 4, kBY = kTY + 2;          // E box
constexpr int kHBY = kTY + 1;                        // H box rows
constexpr int kES = 3, kHS = 2;                      // ring slots
constexpr int kTmaThreads = 320;
constexpr int kTile = kTX * kTY;                     // 512
constexpr int kEW = kTX + 1;                         // ext tile row width
constexpr int kExt = kEW * (kTY + 1);                // 585
constexpr int kHalo = kEW + kTY;                     // 73
constexpr int kRow = 148;                            // per-plane metric values
constexpr int kMatSmem = 32;                         // materials staged in smem

// H box width: 66 doubles (528 B) or 68 floats (the inner box extent must
// be a multiple of 16 bytes).
template <typename T>
constexpr int h_box_x() { return sizeof(T) == 8 ? kTX + 2 : kTX + 4; }

struct TmaMaps {
  CUtensorMap e[3];
  CUtensorMap h[3];
};

template <typename T>
struct TmaLayout {
  static constexpr int eslot = round128(kBX * kBY * (int)sizeof(T));          // per comp
  static constexpr int hslot = round128(h_box_x<T>() * kHBY * (int)sizeof(T));
  static constexpr int e_off = 0;
  static constexpr int h_off = e_off + kES * 3 * eslot;
  static constexpr int hs_off = h_off + kHS * 3 * hslot;
  static constexpr int row_off = hs_off + round128(3 * kExt * (int)sizeof(T));
  static constexpr int l_off = row_off + round128(2 * kRow * (int)sizeof(T));
  static constexpr int mat_off = l_off + round128((kEW + kTY + 1 + kTX + kTY) * (int)sizeof(T));
  static constexpr int bar_off = mat_off + round128(9 * kMatSmem * (int)sizeof(T));
  static constexpr int bytes = bar_off + (kES + kHS) * 8 + 128;   // + base alignment
};

// Ext-tile index (row width 65, origin at (i0-1, j0-1)) of tile cell o.
__device__ __forceinline__ int ext_of_tile(int o) { return (o / kTX + 1) * kEW + o % kTX + 1; }
// Ext-tile index of halo cell h: row j0-1 (h < 65), then column i0-1.
__device__ __forceinline__ int ext_of_halo(int h) { return h < kEW ? h : (h - kEW + 1) * kEW; }

// Per-plane metric row of plane q: [0,9) iAx(j0-1..j0+7), [9,74) iAy(i0-1..i0+63),
// [74,82) itAx(j0..j0+7), [82,146) itAy(i0..i0+63), 146 Lz, 147 tLz.
template <typename T>
__device__ __forceinline__ T row_value(const FitParams<T>& p, int r, int q, int i0, int j0) {
  int idx;
  const T* a;
  if (r < 9) { idx = j0 - 1 + r; a = p.iAx; if (idx >= p.Ny) return T(0); idx += q * p.Ny; }
  else if (r < 74) { idx = i0 - 10 + r; a = p.iAy; if (idx >= p.Nx) return T(0); idx += q * p.Nx; }
  else if (r < 82) { idx = j0 - 74 + r; a = p.itAx; if (idx >= p.Ny) return T(0); idx += q * p.Ny; }
  else if (r < 146) { idx = i0 - 82 + r; a = p.itAy; if (idx >= p.Nx) return T(0); idx += q * p.Nx; }
  else if (r == 146) return p.Lz[q];
  else return p.tLz[q];
  return a[idx];
}

// SM: the material table fits in shared memory (n_mat <= kMatSmem); the
// table reads are then shared-memory loads.  JM: the J mode of the launch
// (WK_J_ZERO, WK_J_SIGMA_E or WK_J_ARRAY), fixed at compile time.
template <typename T, bool SM, int JM>
__global__ void __launch_bounds__(kTmaThreads, sizeof(T) == 8 ? 2 : 3)
k_tma(FitParams<T> p, const __grid_constant__ TmaMaps maps, long long step, int KC) {
  step = step_index(p, step);
  using Lay = TmaLayout<T>;
  constexpr int HBX = h_box_x<T>();
  constexpr int SE = Lay::eslot / (int)sizeof(T);    // elements per E slot
  constexpr int SH = Lay::hslot / (int)sizeof(T);    // elements per H slot
  extern __shared__ __align__(128) unsigned char sm_raw[];
  unsigned char* sm = sm_raw + ((128 - (smem_u32(sm_raw) & 127)) & 127);
  T* Eb = reinterpret_cast<T*>(sm + Lay::e_off);     // [kES][3][SE]
  T* Hb = reinterpret_cast<T*>(sm + Lay::h_off);     // [kHS][3][SH]
  T* Hs = reinterpret_cast<T*>(sm + Lay::hs_off);    // [3][kExt] new H of the plane
  T* Rw = reinterpret_cast<T*>(sm + Lay::row_off);   // [2][kRow] per-plane metrics
  T* sLx = reinterpret_cast<T*>(sm + Lay::l_off);    // Lx(i0-1..i0+63)
  T* sLy = sLx + kEW;                                // Ly(j0-1..j0+7)
  T* stLx = sLy + kTY + 1;                           // tLx(i0..i0+63)
  T* stLy = stLx + kTX;                              // tLy(j0..j0+7)
  T* smat = reinterpret_cast<T*>(sm + Lay::mat_off);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + Lay::bar_off);  // E slots, then H slots

  const int Nx = p.Nx, Ny = p.Ny;
  const long long N = p.N, NxNy = p.NxNy;
  const int i0 = 2 + blockIdx.x * kTX, j0 = 2 + blockIdx.y * kTY;
  const int k0 = 2 + blockIdx.z * KC, k1 = min(k0 + KC, p.Nz - 2);
  const int xs = i0 - 2, ys = j0 - 1;
  const int tid = threadIdx.x;
  const int pstart = k0 - 1;
  const uint32_t e_bytes = (uint32_t)(3 * kBX * kBY * sizeof(T));
  const uint32_t h_bytes = (uint32_t)(3 * HBX * kHBY * sizeof(T));

  if (tid == 0) {
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
  auto wait_e = [&](int q) {
    return mbar_wait(&bar[(q - pstart) % kES], (uint32_t)(((q - pstart) / kES) & 1));
  };
  auto wait_h = [&](int q) {
    return mbar_wait(&bar[kES + (q - pstart) % kHS], (uint32_t)(((q - pstart) / kHS) & 1));
  };
  // E planes pstart..k1 and H planes pstart..k1-1 are loaded, each exactly
  // once; e_hi / h_hi (thread 0) track the last plane issued
  int e_hi = pstart - 1, h_hi = pstart - 1;
  if (tid == 0) {
    for (int q = pstart; q <= min(pstart + kES - 1, k1); q++) { issue_e(q); e_hi = q; }
    for (int q = pstart; q <= min(pstart + kHS - 1, k1 - 1); q++) { issue_h(q); h_hi = q; }
  }

  // owned cells: tile cells t and t+320 (t < 192); threads 192..264 also
  // compute the H of halo cell t-192
  const bool two = tid < kTile - kTmaThreads;
  const bool halo = !two && tid < kTile - kTmaThreads + kHalo;
  int ext[2], ci[2], cj[2];
  bool hval[2], eval[2];
  ext[0] = ext_of_tile(tid);
  ext[1] = two ? ext_of_tile(tid + kTmaThreads) : (halo ? ext_of_halo(tid - (kTile - kTmaThreads)) : 0);
#pragma unroll
  for (int r = 0; r < 2; r++) {
    ci[r] = i0 - 1 + ext[r] % kEW;
    cj[r] = j0 - 1 + ext[r] / kEW;
    const bool own = r == 0 || two || halo;
    hval[r] = own && ci[r] <= Nx - 3 && cj[r] <= Ny - 3;
    eval[r] = (r == 0 || two) && hval[r];
  }
  const bool desc = p.h_desc != 0;
  // plane-invariant metrics
  T iAz[2], itAz[2];
#pragma unroll
  for (int r = 0; r < 2; r++) {
    const long long m = ci[r] + (long long)cj[r] * Nx;
    iAz[r] = hval[r] ? p.iAz[m] : T(0);
    itAz[r] = eval[r] ? p.itAz[m] : T(0);
  }
  if (tid < kEW) sLx[tid] = i0 - 1 + tid < Nx ? p.Lx[i0 - 1 + tid] : T(0);
  else if (tid < kEW + kTY + 1) { const int j = j0 - 1 + tid - kEW; sLy[tid - kEW] = j < Ny ? p.Ly[j] : T(0); }
  else if (tid < kEW + kTY + 1 + kTX) { const int i = i0 + tid - kEW - kTY - 1; stLx[tid - kEW - kTY - 1] = i < Nx ? p.tLx[i] : T(0); }
  else if (tid < kEW + kTY + 1 + kTX + kTY) { const int j = j0 + tid - kEW - kTY - 1 - kTX; stLy[tid - kEW - kTY - 1 - kTX] = j < Ny ? p.tLy[j] : T(0); }
  if (SM)
    for (int q = tid; q < 9 * p.n_mat; q += kTmaThreads) smat[q] = p.mat[q];
  const T* mat = SM ? smat : p.mat;
  // ids and metric row of the first plane
  int id[2];
#pragma unroll
  for (int r = 0; r < 2; r++)
    id[r] = hval[r] ? load_id(p.mat_id, p.id_bytes, ci[r] + (long long)cj[r] * Nx + (long long)pstart * NxNy) : 0;
  if (tid < kRow) Rw[(pstart & 1) * kRow + tid] = row_value(p, tid, pstart, i0, j0);
  T hxp[2] = {T(0), T(0)}, hyp[2] = {T(0), T(0)};

  bool ok = true;
  int pl = pstart;
  for (; pl < k1; pl++) {
    bool got = true;
    if (tid == 0) got = wait_e(pl) && wait_e(pl + 1) && wait_h(pl);
    ok = __syncthreads_and(got);
    if (!ok) break;
    const bool prologue = pl == pstart;
    if (tid == 0 && !prologue) {
      // the slots of E(pl-1) and H(pl-1) are free: every thread finished plane pl-1
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      if (pl + kES - 1 <= k1) { issue_e(pl + kES - 1); e_hi = pl + kES - 1; }
      if (pl + kHS - 1 <= k1 - 1) { issue_h(pl + kHS - 1); h_hi = pl + kHS - 1; }
    }
    // prefetch the ids and metric row of plane pl+1
    const bool more = pl + 1 < k1;
    int idn[2] = {0, 0};
    T rn = T(0);
    if (more) {
#pragma unroll
      for (int r = 0; r < 2; r++)
        if (hval[r]) idn[r] = load_id(p.mat_id, p.id_bytes, ci[r] + (long long)cj[r] * Nx + (long long)(pl + 1) * NxNy);
      if (tid < kRow) rn = row_value(p, tid, pl + 1, i0, j0);
    }
    const T* Ek = Eb + ((pl - pstart) % kES) * 3 * SE;
    const T* Ek1 = Eb + ((pl + 1 - pstart) % kES) * 3 * SE;
    const T* Hk = Hb + ((pl - pstart) % kHS) * 3 * SH;
    const T* R = Rw + (pl & 1) * kRow;
    const long long off = (long long)pl * NxNy;

    // new H of the owned cells (tile cells only in the prologue)
    T hxn[2], hyn[2];
#pragma unroll
    for (int r = 0; r < 2; r++) {
      hxn[r] = hyn[r] = T(0);
      const bool tile_cell = r == 0 || two;
      if (!hval[r] || (prologue && !tile_cell)) continue;
      const int e = ext[r];
      const int ea = e % kEW, eb = e / kEW;
      const int bi = eb * kBX + ea + 1;
      const int hb = eb * HBX + ea + 1;
      const T* m0 = mat + 9 * id[r];
      const T R0 = mul(R[eb], m0[3]);
      const T R1 = mul(R[9 + ea], m0[4]);
      const T R2 = mul(iAz[r], m0[5]);
      T hx = Hk[hb], hy = Hk[SH + hb], hz = Hk[2 * SH + hb];
      h_lean(p.dt, desc, R0, R1, R2, sLx[ea], sLy[eb], R[146], Ek[bi], Ek[SE + bi],
             Ek[2 * SE + bi], Ek[SE + bi + 1], Ek[2 * SE + bi + 1], Ek[bi + kBX],
             Ek[2 * SE + bi + kBX], Ek1[bi], Ek1[SE + bi], hx, hy, hz);
      Hs[e] = hx;
      Hs[kExt + e] = hy;
      Hs[2 * kExt + e] = hz;
      hxn[r] = hx;
      hyn[r] = hy;
      if (!prologue && tile_cell) {
        const long long n = ci[r] + (long long)cj[r] * Nx + off;
        p.H_out[n] = hx;
        p.H_out[N + n] = hy;
        p.H_out[2 * N + n] = hz;
      }
    }
    __syncthreads();

    if (!prologue) {
      const T tLz = R[147];
#pragma unroll
      for (int r = 0; r < 2; r++) {
        if (!eval[r]) continue;
        const int e = ext[r];
        const int a = e % kEW - 1, b = e / kEW - 1;
        const int bi = (b + 1) * kBX + a + 2;
        const long long n = ci[r] + (long long)cj[r] * Nx + off;
        const T* m0 = mat + 9 * id[r];
        const T R0 = mul(m0[0], R[74 + b]);
        const T R1 = mul(m0[1], R[82 + a]);
        const T R2 = mul(m0[2], itAz[r]);
        T curl[3];
        e_lean(R0, R1, R2, stLx[a], stLy[b], tLz, Hs[e], Hs[kExt + e], Hs[2 * kExt + e],
               Hs[kExt + e - 1], Hs[2 * kExt + e - 1], Hs[e - kEW], Hs[2 * kExt + e - kEW],
               hxp[r], hyp[r], curl[0], curl[1], curl[2]);
        const T eold[3] = {Ek[bi], Ek[SE + bi], Ek[2 * SE + bi]};
        Cell cc;
        cc.i = ci[r]; cc.j = cj[r]; cc.k = pl;
        if (p.cap_on) capture(p, cc, n, step, eold[2]);
        const bool src = (p.line_on || p.beam_on) && cc.i == p.ixs && cc.j == p.iys;
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const T ieps = m0[d], sigma = m0[6 + d];
          // J entering the row (the j_in rules with the mode fixed)
          T jv = T(0);
          if (JM == WK_J_SIGMA_E) jv = mul(sigma, eold[d]);
          if (JM == WK_J_ARRAY) jv = p.J[d * N + n];
          if (d == 2 && src) jv = j_in(p, d, cc, n, step, eold[d], sigma);
          const T enew = add(eold[d], mul(p.dt, sub(curl[d], mul(ieps, jv))));
          p.E_out[d * N + n] = enew;
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
    if (more && tid < kRow) Rw[((pl + 1) & 1) * kRow + tid] = rn;
  }
  if (!ok) {
    // a load did not complete in time: record it, wait (bounded) for the
    // loads this block issued, then return
    if (tid == 0) {
      if (p.status) atomicExch(p.status, 1);
      for (int q = pl; q <= e_hi; q++) wait_e(q);
      for (int q = pl; q <= h_hi; q++) wait_h(q);
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
static TmaOcc g_occ[2][2][3][64];

template <typename T, bool SM, int JM>
static cudaError_t tma_occupancy(TmaOcc** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  TmaOcc& o = g_occ[sizeof(T) == 8 ? 0 : 1][SM ? 1 : 0][JM][dev];
  if (!o.attr) {
    const int smem = TmaLayout<T>::bytes;
    e = cudaFuncSetAttribute(k_tma<T, SM, JM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&o.sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.per_sm, k_tma<T, SM, JM>, kTmaThreads,
                                                      smem);
    if (e != cudaSuccess) return e;
    if (o.per_sm < 1) o.per_sm = 1;
    o.attr = true;
  }
  *out = &o;
  return cudaSuccess;
}

template <typename T>
cudaError_t launch_tma(const FitParams<T>& p, long long step, cudaStream_t st, int KC) {
  TmaMaps maps;
  for (int d = 0; d < 3; d++) {
    if (!encode_comp<T>(&maps.e[d], p.E_in + d * p.N, p.Nx, p.Ny, p.Nz, kBX, kBY) ||
        !encode_comp<T>(&maps.h[d], p.H_in + d * p.N, p.Nx, p.Ny, p.Nz, h_box_x<T>(), kHBY))
      return cudaErrorInvalidValue;
  }
  const bool sm_table = p.n_mat <= kMatSmem;
  const int jm = p.j_mode == WK_J_SIGMA_E ? 1 : (p.j_mode == WK_J_ARRAY ? 2 : 0);
  const int gx = (p.Nx - 4 + kTX - 1) / kTX, gy = (p.Ny - 4 + kTY - 1) / kTY;
  auto go = [&](auto kern, TmaOcc* occ) {
    if (KC <= 0)
      KC = tma_auto_kc((long long)gx * gy, p.Nz - 4, (long long)occ->sms * occ->per_sm);
    const int gz = (p.Nz - 4 + KC - 1) / KC;
    timer_begin(st);
    kern<<<dim3(gx, gy, gz), kTmaThreads, TmaLayout<T>::bytes, st>>>(p, maps, step, KC);
    timer_end(st);
  };
  TmaOcc* occ = nullptr;
  cudaError_t e;
#define WK_TMA_CASE(SMV, JMV)                                          \
  if (sm_table == SMV && jm == JMV) {                                  \
    e = tma_occupancy<T, SMV, JMV>(&occ);                              \
    if (e != cudaSuccess) return e;                                    \
    go(k_tma<T, SMV, JMV>, occ);                                       \
  }
  WK_TMA_CASE(true, 0) WK_TMA_CASE(true, 1) WK_TMA_CASE(true, 2)
  WK_TMA_CASE(false, 0) WK_TMA_CASE(false, 1) WK_TMA_CASE(false, 2)
#undef WK_TMA_CASE
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // shell: H from the old state, then E from the new H (the interior H
  // the shell E rows read is in H_out once k_tma is done)
  return launch_shell_pair<T>(p, step, st);
}

template bool tma_supported<double>(const FitParams<double>&);
template bool tma_supported<float>(const FitParams<float>&);
template cudaError_t launch_tma<double>(const FitParams<double>&, long long, cudaStream_t, int);
template cudaError_t launch_tma<float>(const FitParams<float>&, long long, cudaStream_t, int);

}  // namespace wk
