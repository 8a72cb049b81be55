// FP32-compensated fused FIT step with TMA-staged float plane tiles
// (sm_100a): the one-grid launch.  The block's work (comp_tile) and the
// staging scheme are described in fit_tma_comp.cuh.
#include "fit_tma_comp.cuh"

#include "abi_internal.h"

namespace wk {

namespace {

template <typename IdT, bool SIG, int MODE, bool CT, int TW>
__global__ void __launch_bounds__(cThreads, 2)
k_tma_comp(FitParams<double> p, CompState cs, const __grid_constant__ CompMaps maps,
           long long step, int KC) {
  extern __shared__ __align__(128) unsigned char sm_raw[];
  comp_tile<IdT, SIG, MODE, CT ? 1 : 0, false, TW>(p, cs, maps, step, KC, blockIdx.x,
                                                   blockIdx.y, blockIdx.z, CT, sm_raw);
}

// id width x J mode x face mode x compensation words by TMA x tile width
constexpr int kCompKernels = 72;
int g_comp_sms[kCompKernels][64], g_comp_per_sm[kCompKernels][64];
bool g_comp_attr[kCompKernels][64];

}  // namespace

int tma_comp_mode(const FitParams<double>& p) {
  if (!p.has_pec || p.has_pmc) return 0;
  for (int f = 0; f < 4; f++)
    if (p.pec_face[f] != 0) return 0;
  return (p.pec_face[4] == 0 && p.pec_face[5] == 0) ? 1 : 2;
}

bool tma_comp_supported(const wk_fit_desc* d, const FitParams<double>& p) {
  if (p.Nx < 5 || p.Ny < 5 || p.Nz < 5) return false;
  if (p.N >= (1LL << 30)) return false;
  if (p.Nx % 4 != 0 || p.n_mat > cMat) return false;
  // ids are copied as aligned 4- or 8-byte words
  if ((uintptr_t)p.mat_id % 8 != 0) return false;
  for (int q = 0; q < 2; q++)
    if (((uintptr_t)d->E[q] % 16) || ((uintptr_t)d->H[q] % 16) || ((uintptr_t)d->Ec[q] % 4) ||
        ((uintptr_t)d->Hc[q] % 4))
      return false;
  return tma_encode_fn() != nullptr;
}

// Box and layout figures of one tile width
struct CompDims {
  int tx, ty, ebx, hbx, cbx, by, hby, smem;
};
template <int TW>
CompDims comp_dims(bool full, bool ct) {
  using S = CShape<TW>;
  CompDims c;
  c.tx = S::TX;
  c.ty = S::TY;
  c.ebx = full ? CGeom<true, TW>::ebx : CGeom<false, TW>::ebx;
  c.hbx = full ? CGeom<true, TW>::hbx : CGeom<false, TW>::hbx;
  c.cbx = full ? CGeom<true, TW>::cbx : CGeom<false, TW>::cbx;
  c.by = S::BY;
  c.hby = S::HBY;
  c.smem = full ? (ct ? CLayout<true, true, TW>::bytes : CLayout<true, false, TW>::bytes)
                : (ct ? CLayout<false, true, TW>::bytes : CLayout<false, false, TW>::bytes);
  return c;
}

cudaError_t launch_tma_comp(const wk_fit_desc* d, const FitParams<double>& p, int par,
                            long long step, cudaStream_t st, int KC) {
  const int mode = tma_comp_mode(p);
  const bool full = mode != 0;
  CompState cs = comp_state(d, par);
  CompMaps maps;
  // compensation words by TMA: 16-byte row pitch and component bases
  const bool ct = p.Nx % 8 == 0 && ((uintptr_t)cs.Hc_in % 16) == 0 &&
                  ((uintptr_t)cs.Ec_in % 16) == 0;
  // tile shape: 32x16 with tile_rows == 16, 64x8 with 8; by default 32x16
  // on planes of 256x256 cells or more (less halo work per tile; the same
  // rows for every cell) and 64x8 below.  Measured on B200 (Gcell-steps/s,
  // 64x8 / 32x16): 128x128x256 47.7 / 45.2, 256x256x512 58.5 / 59.7,
  // 448x448x896 63.7 / 63.8.
  const bool w32 = d->tile_rows == 16 ||
                   (d->tile_rows != 8 && (long long)p.Nx * p.Ny >= 256LL * 256);
  const CompDims cd = w32 ? comp_dims<32>(full, ct) : comp_dims<64>(full, ct);
  for (int c = 0; c < 3; c++) {
    if (!encode_3d(&maps.e[c], cs.E_in + c * p.N, 4, p.Nx, p.Ny, p.Nz, cd.ebx, cd.by) ||
        !encode_3d(&maps.h[c], cs.H_in + c * p.N, 4, p.Nx, p.Ny, p.Nz, cd.hbx, cd.hby))
      return cudaErrorInvalidValue;
    if (ct &&
        (!encode_3d(&maps.c[c], cs.Hc_in + c * p.N, 2, p.Nx, p.Ny, p.Nz, cd.cbx, cd.hby) ||
         !encode_3d(&maps.c[3 + c], cs.Ec_in + c * p.N, 2, p.Nx, p.Ny, p.Nz, cd.cbx, cd.hby)))
      return cudaErrorInvalidValue;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  const int ib = p.id_bytes == 1 ? 0 : (p.id_bytes == 2 ? 1 : 2);
  const bool sig = p.j_mode == WK_J_SIGMA_E;
  const int slot = (w32 ? 36 : 0) + (ct ? 18 : 0) + mode * 6 + ib * 2 + (sig ? 1 : 0);
  using K = void (*)(FitParams<double>, CompState, const CompMaps, long long, int);
#define WK_COMP_KERNS(CT, TW)                                                              \
  k_tma_comp<uint8_t, false, 0, CT, TW>, k_tma_comp<uint8_t, true, 0, CT, TW>,             \
      k_tma_comp<uint16_t, false, 0, CT, TW>, k_tma_comp<uint16_t, true, 0, CT, TW>,       \
      k_tma_comp<uint32_t, false, 0, CT, TW>, k_tma_comp<uint32_t, true, 0, CT, TW>,       \
      k_tma_comp<uint8_t, false, 1, CT, TW>, k_tma_comp<uint8_t, true, 1, CT, TW>,         \
      k_tma_comp<uint16_t, false, 1, CT, TW>, k_tma_comp<uint16_t, true, 1, CT, TW>,       \
      k_tma_comp<uint32_t, false, 1, CT, TW>, k_tma_comp<uint32_t, true, 1, CT, TW>,       \
      k_tma_comp<uint8_t, false, 2, CT, TW>, k_tma_comp<uint8_t, true, 2, CT, TW>,         \
      k_tma_comp<uint16_t, false, 2, CT, TW>, k_tma_comp<uint16_t, true, 2, CT, TW>,       \
      k_tma_comp<uint32_t, false, 2, CT, TW>, k_tma_comp<uint32_t, true, 2, CT, TW>
  const K kerns[kCompKernels] = {WK_COMP_KERNS(false, 64), WK_COMP_KERNS(true, 64),
                                 WK_COMP_KERNS(false, 32), WK_COMP_KERNS(true, 32)};
#undef WK_COMP_KERNS
  const K kern = kerns[slot];
  const int smem = cd.smem;
  if (!g_comp_attr[slot][dev]) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&g_comp_sms[slot][dev], cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_comp_per_sm[slot][dev], kern, cThreads,
                                                      smem);
    if (e != cudaSuccess) return e;
    if (g_comp_per_sm[slot][dev] < 1) g_comp_per_sm[slot][dev] = 1;
    g_comp_attr[slot][dev] = true;
  }
  const int span_x = full ? p.Nx : p.Nx - 4, span_y = full ? p.Ny : p.Ny - 4;
  const int planes = mode == 1 ? p.Nz : p.Nz - 4;
  const int gx = (span_x + cd.tx - 1) / cd.tx, gy = (span_y + cd.ty - 1) / cd.ty;
  if (KC <= 0)
    KC = tma_auto_kc((long long)gx * gy, planes,
                     (long long)g_comp_sms[slot][dev] * g_comp_per_sm[slot][dev]);
  const int gz = (planes + KC - 1) / KC;
  timer_begin(st);
  kern<<<dim3(gx, gy, gz), cThreads, smem, st>>>(p, cs, maps, step, KC);
  timer_end(st);
  return cudaGetLastError();
}

}  // namespace wk
