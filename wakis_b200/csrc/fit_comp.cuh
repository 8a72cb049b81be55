// FP32-compensated state: a float value v plus a bf16 compensation word c
// (the rounding error of the last update), shared by the two-pass and the
// TMA compensated kernels.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/wakis_b200.h"
#include "fit_common.cuh"

namespace wk {

typedef uint16_t comp_t;   // raw bf16 bits

__device__ __forceinline__ float comp_dec(comp_t q) { return __uint_as_float((unsigned)q << 16); }
__device__ __forceinline__ comp_t comp_enc(float e) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(e));
}
__device__ __forceinline__ double comp_value(float v, comp_t q) {
  return (double)v + (double)comp_dec(q);
}
// v + c + delta -> (t, q'): Kahan step y = delta + c, then TwoSum(v, y)
__device__ __forceinline__ void comp_add(float v, comp_t q, float delta, float& t, comp_t& qn) {
  const float c = comp_dec(q);
  const float y = __fadd_rn(delta, c);
  t = __fadd_rn(v, y);
  const float bp = __fsub_rn(t, v);
  const float ap = __fsub_rn(t, bp);
  const float e = __fadd_rn(__fsub_rn(v, ap), __fsub_rn(y, bp));
  qn = comp_enc(e);
}
// double -> (float, q)
__device__ __forceinline__ void comp_split(double x, float& t, comp_t& q) {
  t = (float)x;
  q = comp_enc((float)(x - (double)t));
}

struct CompState {
  const float* E_in; const float* H_in; float* E_out; float* H_out;
  const comp_t* Ec_in; const comp_t* Hc_in; comp_t* Ec_out; comp_t* Hc_out;
};

inline CompState comp_state(const wk_fit_desc* d, int par) {
  CompState s;
  s.E_in = (const float*)d->E[par];
  s.H_in = (const float*)d->H[par];
  s.E_out = (float*)d->E[par ^ 1];
  s.H_out = (float*)d->H[par ^ 1];
  s.Ec_in = (const comp_t*)d->Ec[par];
  s.Hc_in = (const comp_t*)d->Hc[par];
  s.Ec_out = (comp_t*)d->Ec[par ^ 1];
  s.Hc_out = (comp_t*)d->Hc[par ^ 1];
  return s;
}

// TMA-staged compensated step (fit_tma_comp.cu): true when the grid and
// buffers suit it (row pitch Nx % 4 == 0, dims >= 5, <= 64 materials).
bool tma_comp_supported(const wk_fit_desc* d, const FitParams<double>& p);
cudaError_t launch_tma_comp(const wk_fit_desc* d, const FitParams<double>& p, int par,
                            long long step, cudaStream_t st, int KC);
// Mode of the compensated TMA kernel for these faces: 1 when every face
// carries the PEC column mask (whole grid, no shell launch), 2 when the four
// x/y faces do (shell launches over the four z-boundary planes only), else 0
// (interior + full shell); never with PMC faces.
int tma_comp_mode(const FitParams<double>& p);

}  // namespace wk
