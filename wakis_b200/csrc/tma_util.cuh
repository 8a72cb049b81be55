// TMA and mbarrier helpers shared by the TMA-staged step kernels (sm_100a):
// shared-memory addresses, mbarrier init / expect-tx / bounded wait, a 3-D
// tiled bulk tensor load (no multicast) and the tensor-map encoder.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace wk {

// Bound of one mbarrier wait: kWaitNs of %globaltimer time (100 ms, far
// above the microseconds a tile load takes), and at most kWaitPolls polls
// in case the timer does not advance.
constexpr long long kWaitNs = 100000000LL;
constexpr long long kWaitPolls = 1LL << 26;

constexpr int round128(int b) { return (b + 127) / 128 * 128; }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
// Invalidate an mbarrier whose phases have all completed, so that its word
// can be initialised again (a block that runs several tiles in turn).
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
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
__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait for the phase of `parity`: true once it completed, false
// when limit_ns nanoseconds (or kWaitPolls polls) passed first.  A negative
// limit_ns gives up without polling (the timeout test of the step kernels).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          long long limit_ns = kWaitNs) {
  if (limit_ns < 0) return false;
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_ns();
  for (long long it = 0; it < kWaitPolls; it++) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((long long)(globaltimer_ns() - t0) > limit_ns) return false;
  }
  return false;
}
// Bound of the waits of a launch's step loop: wk_fit_desc.wait_ns, 0 = the
// default.
__device__ __forceinline__ long long loop_wait_ns(long long wait_ns) {
  return wait_ns == 0 ? kWaitNs : wait_ns;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y,
                                            int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// cp.async (LDGSTS) of one 4- or 8-byte word into shared memory; with
// valid == false nothing is read and the word is zero-filled.  Completion is
// per thread: cp_async_commit() closes a group, cp_async_wait<N>() waits
// until at most N of this thread's groups are still in flight.
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src, bool valid) {
  static_assert(BYTES == 4 || BYTES == 8, "cp.async word size");
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(smem_u32(dst)), "l"(src),
               "n"(BYTES), "r"(valid ? BYTES : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Material id n of an id array of `bytes`-byte entries (1, 2 or 4) held in
// the 4-byte word that contains it: the word's index and the id's position.
__device__ __forceinline__ long long id_word_index(int bytes, long long n) {
  return (n * bytes) >> 2;
}
__device__ __forceinline__ int id_from_word(uint32_t w, int bytes, long long n) {
  if (bytes == 4) return (int)w;
  const int sh = (int)((n * bytes) & 3) * 8;
  return (int)((w >> sh) & (bytes == 1 ? 0xffu : 0xffffu));
}

// cuTensorMapEncodeTiled from the driver, fetched once through the runtime
// (the library links only the CUDA runtime); nullptr when unavailable.
inline PFN_cuTensorMapEncodeTiled_v12000 tma_encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
  if (g_encode) return g_encode;
  cudaDriverEntryPointQueryResult q;
  void* fn = nullptr;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
          cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !fn)
    return nullptr;
  g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  return g_encode;
}

// Planes per block when none is given: the chunk length KC in [4, 64]
// minimising (waves of blocks) x (KC + 2), the 2 standing for the prologue
// plane and the pipeline fill of each block.
inline int tma_auto_kc(long long tiles, int planes, long long slots) {
  int best = 8;
  long long best_cost = -1;
  for (int kc = 4; kc <= 64; kc++) {
    const long long gz = (planes + kc - 1) / kc;
    const long long waves = (tiles * gz + slots - 1) / slots;
    const long long cost = waves * (kc + 2);
    if (best_cost < 0 || cost < best_cost) { best_cost = cost; best = kc; }
    if (kc >= planes) break;
  }
  return best;
}

}  // namespace wk
