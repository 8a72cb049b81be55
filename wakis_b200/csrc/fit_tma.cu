// Fused FIT step with TMA-staged plane tiles (sm_100a).
//
// Interior cells only (2 <= i <= Nx-3, 2 <= j <= Ny-3, 2 <= k <= Nz-3); the
// shell runs in the k_shell launch.  Block (bx, by, bz) owns the tile
// i in [i0, i0+64), j in [j0, j0+8) of planes [k0, k0+KC) and marches in z.
// For plane k it needs E_old of planes k and k+1 and H_old of plane k on the
// box x in [i0-2, i0+66), y in [j0-1, j0+9) (one halo column/row on each
// side; the box starts at an even x so the TMA x offset is 16-byte aligned).
// One thread issues cp.async.bulk.tensor loads of those boxes (one per field
// component, no multicast) into a ring of shared-memory slots, three planes
// of E and two of H, completing on an mbarrier per slot; the loads of plane
// k+3 (E) and k+2 (H) go out while plane k is computed.  Per plane the block
// computes the new H on the tile plus its low halo row and column (single-
// coefficient rows, the halo recomputed so no block waits for another), then
// the new E of the tile, and keeps the tile's new Hx, Hy for plane k+1.  A
// chunk starting at k0 first forms the new H of plane k0-1 on its tile.
// Every mbarrier wait is bounded: on timeout the block records the failure
// in the status word, waits (bounded) for its loads in flight and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include "../../include/wakis_b200.h"
#include "abi_internal.h"
#include "fit_common.cuh"
#include "fit_kernels.cuh"

namespace wk {

constexpr int kTX = 64, kTY = 8;
constexpr int kBX = kTX + 4, kBY = kTY + 2;
constexpr int kES = 3, kHS = 2;
constexpr int kTmaThreads = 256;
constexpr int kExt = (kTX + 1) * (kTY + 1);
constexpr long long kWaitLimit = 1LL << 24;

struct TmaMaps {
  CUtensorMap e[3];
  CUtensorMap h[3];
};

template <typename T>
struct TmaLayout {
  static constexpr int box = kBX * kBY;
  static constexpr int slot = ((box * (int)sizeof(T) + 127) / 128) * 128;  // bytes per comp
  static constexpr int e_off = 0;
  static constexpr int h_off = e_off + kES * 3 * slot;
  static constexpr int hs_off = h_off + kHS * 3 * slot;
  static constexpr int hp_off = hs_off + ((3 * kExt * (int)sizeof(T) + 127) / 128) * 128;
  static constexpr int bar_off = hp_off + ((2 * kTX * kTY * (int)sizeof(T) + 127) / 128) * 128;
  static constexpr int bytes = bar_off + (kES + kHS) * 8 + 128;   // + base alignment
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Bounded wait; false when the limit is reached.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (long long it = 0; it < kWaitLimit; it++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y,
                                            int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

template <typename T>
__global__ void __launch_bounds__(kTmaThreads)
k_tma(FitParams<T> p, const __grid_constant__ TmaMaps maps, long long step, int KC) {
  using Lay = TmaLayout<T>;
  extern __shared__ __align__(128) unsigned char sm_raw[];
  unsigned char* sm = sm_raw + ((128 - (smem_u32(sm_raw) & 127)) & 127);
  T* Eb = reinterpret_cast<T*>(sm + Lay::e_off);     // [kES][3][slot]
  T* Hb = reinterpret_cast<T*>(sm + Lay::h_off);     // [kHS][3][slot]
  T* Hs = reinterpret_cast<T*>(sm + Lay::hs_off);    // [3][kExt]
  T* Hp = reinterpret_cast<T*>(sm + Lay::hp_off);    // [2][kTX*kTY]
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + Lay::bar_off);  // E slots, then H slots
  constexpr int SE = Lay::slot / (int)sizeof(T);     // elements per slot

  const int Nx = p.Nx, Ny = p.Ny, Nz = p.Nz;
  const long long N = p.N, NxNy = p.NxNy;
  const int i0 = 2 + blockIdx.x * kTX, j0 = 2 + blockIdx.y * kTY;
  const int k0 = 2 + blockIdx.z * KC, k1 = min(k0 + KC, Nz - 2);
  const int xs = i0 - 2, ys = j0 - 1;
  const int tid = threadIdx.x;
  const int pstart = k0 - 1;
  const uint32_t box_bytes = (uint32_t)(3 * kBX * kBY * sizeof(T));

  if (tid == 0) {
    for (int s = 0; s < kES + kHS; s++) mbar_init(&bar[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  auto issue_e = [&](int q) {
    const int slot = (q - pstart) % kES;
    mbar_expect_tx(&bar[slot], box_bytes);
#pragma unroll
    for (int d = 0; d < 3; d++)
      tma_load_3d(Eb + (slot * 3 + d) * SE, &maps.e[d], xs, ys, q, &bar[slot]);
  };
  auto issue_h = [&](int q) {
    const int slot = (q - pstart) % kHS;
    mbar_expect_tx(&bar[kES + slot], box_bytes);
#pragma unroll
    for (int d = 0; d < 3; d++)
      tma_load_3d(Hb + (slot * 3 + d) * SE, &maps.h[d], xs, ys, q, &bar[kES + slot]);
  };
  // E planes pstart..k1 and H planes pstart..k1-1 are loaded, each exactly
  // once; e_hi / h_hi (thread 0) track the last plane issued
  int e_hi = pstart - 1, h_hi = pstart - 1;
  if (tid == 0) {
    for (int q = pstart; q <= min(pstart + kES - 1, k1); q++) { issue_e(q); e_hi = q; }
    for (int q = pstart; q <= min(pstart + kHS - 1, k1 - 1); q++) { issue_h(q); h_hi = q; }
  }
  auto wait_e = [&](int q) {
    return mbar_wait(&bar[(q - pstart) % kES], (uint32_t)(((q - pstart) / kES) & 1));
  };
  auto wait_h = [&](int q) {
    return mbar_wait(&bar[kES + (q - pstart) % kHS], (uint32_t)(((q - pstart) / kHS) & 1));
  };

  const bool desc = p.h_desc != 0;
  bool ok = true;
  int pl = pstart;
  for (; pl < k1; pl++) {
    ok = __syncthreads_and(wait_e(pl) && wait_e(pl + 1) && wait_h(pl));
    if (!ok) break;
    const bool prologue = pl == pstart;
    const T* Ek = Eb + ((pl - pstart) % kES) * 3 * SE;
    const T* Ek1 = Eb + ((pl + 1 - pstart) % kES) * 3 * SE;
    const T* Hk = Hb + ((pl - pstart) % kHS) * 3 * SE;
    const T Lz = p.Lz[pl];

    // new H on the tile and its low halo (tile only in the prologue)
    for (int c = tid; c < kExt; c += kTmaThreads) {
      const int b = c / (kTX + 1), a = c - b * (kTX + 1);
      const int i = i0 - 1 + a, j = j0 - 1 + b;
      if (i > Nx - 3 || j > Ny - 3) continue;
      if (prologue && (a == 0 || b == 0)) continue;
      const int bi = b * kBX + a + 1;
      const long long n = i + (long long)j * Nx + (long long)pl * NxNy;
      const T* m0 = p.mat + 9 * load_id(p.mat_id, p.id_bytes, n);
      const T R0 = mul(p.iAx[j + (long long)pl * Ny], m0[3]);
      const T R1 = mul(p.iAy[i + (long long)pl * Nx], m0[4]);
      const T R2 = mul(p.iAz[i + (long long)j * Nx], m0[5]);
      T hx = Hk[bi], hy = Hk[SE + bi], hz = Hk[2 * SE + bi];
      h_lean(p.dt, desc, R0, R1, R2, p.Lx[i], p.Ly[j], Lz, Ek[bi], Ek[SE + bi], Ek[2 * SE + bi],
             Ek[SE + bi + 1], Ek[2 * SE + bi + 1], Ek[bi + kBX], Ek[2 * SE + bi + kBX], Ek1[bi],
             Ek1[SE + bi], hx, hy, hz);
      Hs[c] = hx;
      Hs[kExt + c] = hy;
      Hs[2 * kExt + c] = hz;
      if (!prologue && a > 0 && b > 0) {
        p.H_out[n] = hx;
        p.H_out[N + n] = hy;
        p.H_out[2 * N + n] = hz;
      }
    }
    __syncthreads();

    if (!prologue) {
      const T tLz = p.tLz[pl];
      for (int o = tid; o < kTX * kTY; o += kTmaThreads) {
        const int b = o / kTX, a = o - b * kTX;
        const int i = i0 + a, j = j0 + b;
        if (i > Nx - 3 || j > Ny - 3) continue;
        const int e = (b + 1) * (kTX + 1) + a + 1;
        const int bi = (b + 1) * kBX + a + 2;
        const long long n = i + (long long)j * Nx + (long long)pl * NxNy;
        const T* m0 = p.mat + 9 * load_id(p.mat_id, p.id_bytes, n);
        const T R0 = mul(m0[0], p.itAx[j + (long long)pl * Ny]);
        const T R1 = mul(m0[1], p.itAy[i + (long long)pl * Nx]);
        const T R2 = mul(m0[2], p.itAz[i + (long long)j * Nx]);
        T curl[3];
        e_lean(R0, R1, R2, p.tLx[i], p.tLy[j], tLz, Hs[e], Hs[kExt + e], Hs[2 * kExt + e],
               Hs[kExt + e - 1], Hs[2 * kExt + e - 1], Hs[e - kTX - 1],
               Hs[2 * kExt + e - kTX - 1], Hp[o], Hp[kTX * kTY + o], curl[0], curl[1], curl[2]);
        const T eold[3] = {Ek[bi], Ek[SE + bi], Ek[2 * SE + bi]};
        Cell cc;
        cc.i = i; cc.j = j; cc.k = pl;
        if (p.cap_on) capture(p, cc, n, step, eold[2]);
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const T ieps = m0[d], sigma = m0[6 + d];
          const T jv = j_in(p, d, cc, n, step, eold[d], sigma);
          const T enew = add(eold[d], mul(p.dt, sub(curl[d], mul(ieps, jv))));
          p.E_out[d * N + n] = enew;
          if (p.j_mode == WK_J_ARRAY && p.use_cond) p.J[d * N + n] = mul(sigma, enew);
        }
      }
    }
    __syncthreads();
    // the tile's new Hx, Hy are H(n - Nx*Ny) of the next plane
    for (int o = tid; o < kTX * kTY; o += kTmaThreads) {
      const int b = o / kTX, a = o - b * kTX;
      const int e = (b + 1) * (kTX + 1) + a + 1;
      Hp[o] = Hs[e];
      Hp[kTX * kTY + o] = Hs[kExt + e];
    }
    __syncthreads();
    // slots of E(pl) and H(pl) are free: refill them
    if (tid == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      if (pl + kES <= k1) { issue_e(pl + kES); e_hi = pl + kES; }
      if (pl + kHS <= k1 - 1) { issue_h(pl + kHS); h_hi = pl + kHS; }
    }
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
static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

static bool get_encode() {
  if (g_encode) return true;
  cudaDriverEntryPointQueryResult q;
  void* fn = nullptr;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
          cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !fn)
    return false;
  g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  return true;
}

template <typename T>
static bool encode_comp(CUtensorMap* map, const T* base, int Nx, int Ny, int Nz) {
  const CUtensorMapDataType dt =
      sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  cuuint64_t gdim[3] = {(cuuint64_t)Nx, (cuuint64_t)Ny, (cuuint64_t)Nz};
  cuuint64_t gstr[2] = {(cuuint64_t)Nx * sizeof(T), (cuuint64_t)Nx * Ny * sizeof(T)};
  cuuint32_t box[3] = {(cuuint32_t)kBX, (cuuint32_t)kBY, 1};
  cuuint32_t est[3] = {1, 1, 1};
  CUresult r = g_encode(map, dt, 3, (void*)base, gdim, gstr, box, est,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// True when the TMA kernel can run this grid: 16-byte strides and bases
// (Nx*sizeof(T) multiple of 16 and N even), dims >= 5, driver entry point.
template <typename T>
bool tma_supported(const FitParams<T>& p) {
  if (p.Nx < 5 || p.Ny < 5 || p.Nz < 5) return false;
  if ((p.Nx * sizeof(T)) % 16 != 0 || (p.N * sizeof(T)) % 16 != 0) return false;
  if (((uintptr_t)p.E_in % 16) || ((uintptr_t)p.H_in % 16)) return false;
  return get_encode();
}

template <typename T>
cudaError_t launch_tma(const FitParams<T>& p, long long step, cudaStream_t st, int KC) {
  TmaMaps maps;
  for (int d = 0; d < 3; d++) {
    if (!encode_comp<T>(&maps.e[d], p.E_in + d * p.N, p.Nx, p.Ny, p.Nz) ||
        !encode_comp<T>(&maps.h[d], p.H_in + d * p.N, p.Nx, p.Ny, p.Nz))
      return cudaErrorInvalidValue;
  }
  const int gx = (p.Nx - 4 + kTX - 1) / kTX, gy = (p.Ny - 4 + kTY - 1) / kTY;
  if (KC <= 0) {
    long long want = 148LL * 2 * 2;
    long long gz = (want + (long long)gx * gy - 1) / ((long long)gx * gy);
    KC = (int)((p.Nz - 4 + gz - 1) / gz);
    if (KC < 8) KC = 8;
  }
  const int gz = (p.Nz - 4 + KC - 1) / KC;
  const int smem = TmaLayout<T>::bytes;
  cudaError_t e = cudaFuncSetAttribute(k_tma<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  k_tma<T><<<dim3(gx, gy, gz), kTmaThreads, smem, st>>>(p, maps, step, KC);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const long long count = p.N - (long long)(p.Nx - 4) * (p.Ny - 4) * (p.Nz - 4);
  k_shell<T><<<(unsigned)((count + 255) / 256), 256, 0, st>>>(p, step, count);
  return cudaGetLastError();
}

template bool tma_supported<double>(const FitParams<double>&);
template bool tma_supported<float>(const FitParams<float>&);
template cudaError_t launch_tma<double>(const FitParams<double>&, long long, cudaStream_t, int);
template cudaError_t launch_tma<float>(const FitParams<float>&, long long, cudaStream_t, int);

}  // namespace wk
