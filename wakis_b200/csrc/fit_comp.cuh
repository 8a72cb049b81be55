// FP32-compensated state: a float value v plus a bf16 compensation word c
// (the rounding error of the last update), shared by the two-pass and the
// TMA compensated kernels.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/wakis_b200.h"
#include "fit_common.cuh"
#include "fit_kernels.cuh"

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

// Compensated stencil (wk_fit_desc.comp_stencil): the neighbour values of a
// row are read as the pairs v + c, and the increment is formed in float
// with error-free transformations (double-float arithmetic: Knuth's TwoSum
// and the exact product error of an FMA, as in Dekker 1971 and Ogita, Rump
// and Oishi 2005) on coefficients split into two floats, so the increment
// carries ~44 significant bits instead of the 24 of a float row sum.
// A value is the unevaluated sum hi + lo of two floats.
struct FPair {
  float hi, lo;
};
__device__ __forceinline__ FPair two_sum(float a, float b) {
  const float s = __fadd_rn(a, b);
  const float bp = __fsub_rn(s, a);
  const float ap = __fsub_rn(s, bp);
  return {s, __fadd_rn(__fsub_rn(a, ap), __fsub_rn(b, bp))};
}
// (va + ca) - (vb + cb): the float difference with its exact error, plus
// the difference of the compensation parts
__device__ __forceinline__ FPair pair_diff(float va, float ca, float vb, float cb) {
  FPair d = two_sum(va, -vb);
  d.lo = __fadd_rn(d.lo, __fsub_rn(ca, cb));
  return d;
}
// k * d for k = kh + kl: the product of the high parts with its exact error
// (FMA), plus the first-order cross terms
__device__ __forceinline__ FPair pair_mul(FPair k, FPair d) {
  const float p = __fmul_rn(k.hi, d.hi);
  const float e = __fmaf_rn(k.hi, d.hi, -p);
  return {p, __fmaf_rn(k.hi, d.lo, __fmaf_rn(k.lo, d.hi, e))};
}
__device__ __forceinline__ FPair pair_add(FPair a, FPair b) {
  const FPair s = two_sum(a.hi, b.hi);
  return {s.hi, __fadd_rn(s.lo, __fadd_rn(a.lo, b.lo))};
}
__device__ __forceinline__ FPair pair_sub(FPair a, FPair b) {
  return pair_add(a, FPair{-b.hi, -b.lo});
}
// an FP64 coefficient (or source value) as two floats
__device__ __forceinline__ FPair pair_of(double x) {
  const float h = (float)x;
  return {h, (float)(x - (double)h)};
}
// state v + c plus an increment pair -> (t, q'): t the float nearest the
// sum, q' its remainder as a bf16 word
__device__ __forceinline__ void comp_add_pair(float v, comp_t q, FPair delta, float& t,
                                              comp_t& qn) {
  const FPair s = two_sum(v, delta.hi);
  const float low = __fadd_rn(s.lo, __fadd_rn(delta.lo, comp_dec(q)));
  const FPair r = two_sum(s.hi, low);
  t = r.hi;
  qn = comp_enc(r.lo);
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

// One shell cell of the compensated step: the state is decoded to FP64,
// the cell takes the lean rows where they apply and the general rows
// elsewhere, and the FP64 result is split back into (float, bf16).  H from
// the old state; E from the new H (every H_out entry it reads written).
__device__ __forceinline__ void comp_shell_h(const FitParams<double>& p, const CompState& st,
                                             Cell c) {
  const int Nx = p.Nx;
  const long long N = p.N, NxNy = p.NxNy;
  const long long n = c.i + (long long)c.j * Nx + (long long)c.k * NxNy;
  auto E = [&](int e, long long m) -> double {
    return comp_value(st.E_in[e * N + m], st.Ec_in[e * N + m]);
  };
  const int id = load_id(p.mat_id, p.id_bytes, n);
  double h[3];
#pragma unroll
  for (int d = 0; d < 3; d++) h[d] = comp_value(st.H_in[d * N + n], st.Hc_in[d * N + n]);
  if (lean_h<double>(c.i, c.j, c.k, Nx, p.Ny, p.Nz)) {
    const double* m0 = p.mat + 9 * id;
    const double R0 = p.iAx[c.j + (long long)c.k * p.Ny] * m0[3];
    const double R1 = p.iAy[c.i + (long long)c.k * Nx] * m0[4];
    const double R2 = p.iAz[c.i + (long long)c.j * Nx] * m0[5];
    h_lean(p.dt, p.h_desc != 0, R0, R1, R2, p.Lx[c.i], p.Ly[c.j], p.Lz[c.k], E(0, n), E(1, n),
           E(2, n), E(1, n + 1), E(2, n + 1), E(0, n + Nx), E(2, n + Nx), E(0, n + NxNy),
           E(1, n + NxNy), h[0], h[1], h[2]);
  } else {
    const long long off[4] = {0, 1, (long long)Nx, NxNy};
    auto ev = [&](int e, int kind) -> double { return E(e, n + off[kind]); };
#pragma unroll
    for (int d = 0; d < 3; d++) h[d] = h_row_acc(p, h[d], d, c, n, id, ev);
  }
#pragma unroll
  for (int d = 0; d < 3; d++) {
    float t;
    comp_t q;
    comp_split(h[d], t, q);
    st.H_out[d * N + n] = t;
    st.Hc_out[d * N + n] = q;
  }
}

__device__ __forceinline__ void comp_shell_e(const FitParams<double>& p, const CompState& st,
                                             Cell c, long long step) {
  const int Nx = p.Nx;
  const long long N = p.N, NxNy = p.NxNy;
  const long long n = c.i + (long long)c.j * Nx + (long long)c.k * NxNy;
  auto Hn = [&](int e, long long m) -> double { return (double)st.H_out[e * N + m]; };
  const int id = load_id(p.mat_id, p.id_bytes, n);
  const double ez_old = comp_value(st.E_in[2 * N + n], st.Ec_in[2 * N + n]);
  if (p.cap_on) capture(p, c, n, step, ez_old);
  double curl[3];
  const bool lean = lean_e<double>(c.i, c.j, c.k, Nx, p.Ny, p.Nz);
  if (lean) {
    const double* m0 = p.mat + 9 * id;
    const double R0 = m0[0] * p.itAx[c.j + (long long)c.k * p.Ny];
    const double R1 = m0[1] * p.itAy[c.i + (long long)c.k * Nx];
    const double R2 = m0[2] * p.itAz[c.i + (long long)c.j * Nx];
    e_lean(R0, R1, R2, p.tLx[c.i], p.tLy[c.j], p.tLz[c.k], Hn(0, n), Hn(1, n), Hn(2, n),
           Hn(1, n - 1), Hn(2, n - 1), Hn(0, n - Nx), Hn(2, n - Nx), Hn(0, n - NxNy),
           Hn(1, n - NxNy), curl[0], curl[1], curl[2]);
  }
  const long long off[4] = {0, 1, (long long)Nx, NxNy};
  auto hv = [&](int e, int kind) -> double { return Hn(e, n - off[kind]); };
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double ieps = p.mat[9 * id + d], sigma = p.mat[9 * id + 6 + d];
    const double eold = d == 2 ? ez_old : comp_value(st.E_in[d * N + n], st.Ec_in[d * N + n]);
    const double jv = j_in(p, d, c, n, step, eold, sigma);
    const double cu = lean ? curl[d] : e_curl_acc(p, d, c, n, ieps, hv);
    const double enew = eold + p.dt * (cu - ieps * jv);
    float t;
    comp_t q;
    comp_split(enew, t, q);
    st.E_out[d * N + n] = t;
    st.Ec_out[d * N + n] = q;
  }
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
