// FP32-compensated FIT step (sm_100a).
//
// State: every E and H component is a float v plus an int8 compensation q
// holding the rounding error of the last update, c = q * 2^(E(v)-30) with
// E(v) the exponent of v, so v + c carries ~30 significant bits.  The
// update coefficients are formed in FP64 from the FP64 tables (one rounding
// to float per coefficient, dt folded in), the row sums run in float, and
// the increment is added with a Kahan step (y = delta + c, TwoSum(v, y)).
// The Ez capture stores v + c in FP64, so the wake integration and the
// impedance DFT stay FP64.  Two passes (H, then E) over interior tiles and
// the two-cell shell; shell cells decode the state to FP64 and use the
// general FP64 row code.
#include <stdint.h>

#include "../../include/wakis_b200.h"
#include "abi_internal.h"
#include "fit_common.cuh"
#include "fit_kernels.cuh"

namespace wk {

__device__ __forceinline__ float comp_scale_dec(float v) {  // 2^(E(v)-30)
  const int ex = (__float_as_int(v) >> 23) & 0xff;
  return ex > 30 ? __int_as_float((ex - 30) << 23) : 0.0f;
}
__device__ __forceinline__ float comp_scale_enc(float v) {  // 2^(30-E(v))
  const int ex = (__float_as_int(v) >> 23) & 0xff;
  return (ex > 30 && ex < 255) ? __int_as_float((284 - ex) << 23) : 0.0f;
}
__device__ __forceinline__ int8_t comp_encode(float t, float e) {
  float r = rintf(__fmul_rn(e, comp_scale_enc(t)));
  r = fminf(fmaxf(r, -127.0f), 127.0f);
  return (int8_t)r;
}
__device__ __forceinline__ double comp_value(float v, int8_t q) {
  return (double)v + (double)((float)q * comp_scale_dec(v));
}
// v + c + delta -> (t, q')
__device__ __forceinline__ void comp_add(float v, int8_t q, float delta, float& t, int8_t& qn) {
  const float c = (float)q * comp_scale_dec(v);
  const float y = __fadd_rn(delta, c);
  t = __fadd_rn(v, y);
  const float bp = __fsub_rn(t, v);
  const float ap = __fsub_rn(t, bp);
  const float e = __fadd_rn(__fsub_rn(v, ap), __fsub_rn(y, bp));
  qn = comp_encode(t, e);
}
// double -> (float, q)
__device__ __forceinline__ void comp_split(double x, float& t, int8_t& q) {
  t = (float)x;
  q = comp_encode(t, (float)(x - (double)t));
}

struct CompState {
  const float* E_in; const float* H_in; float* E_out; float* H_out;
  const int8_t* Ec_in; const int8_t* Hc_in; int8_t* Ec_out; int8_t* Hc_out;
};

constexpr int kCompX = 128, kCompY = 2;

__global__ void __launch_bounds__(kCompX * kCompY)
k_h_comp(FitParams<double> p, CompState st) {
  const int i = 2 + blockIdx.x * kCompX + threadIdx.x;
  const int j = 2 + blockIdx.y * kCompY + threadIdx.y;
  const int k = 2 + blockIdx.z;
  if (i > p.Nx - 3 || j > p.Ny - 3) return;
  const long long N = p.N;
  const int sy = p.Nx, sz = (int)p.NxNy;
  const long long n = i + (long long)j * sy + (long long)k * sz;
  const float* ex = st.E_in + n;
  const float* ey = st.E_in + N + n;
  const float* ez = st.E_in + 2 * N + n;
  const float e0x = ex[0], e0y = ey[0], e0z = ez[0];
  const float ey1 = ey[1], ez1 = ez[1], ex2 = ex[sy], ez2 = ez[sy], ex3 = ex[sz], ey3 = ey[sz];
  const float h[3] = {st.H_in[n], st.H_in[N + n], st.H_in[2 * N + n]};
  const int8_t hq[3] = {st.Hc_in[n], st.Hc_in[N + n], st.Hc_in[2 * N + n]};
  const double* m0 = p.mat + 9 * load_id(p.mat_id, p.id_bytes, n);
  const double dt = p.dt;
  const double Lx = p.Lx[i], Ly = p.Ly[j], Lz = p.Lz[k];
  const double R0 = p.iAx[j + k * p.Ny] * m0[3];
  const double R1 = p.iAy[i + k * sy] * m0[4];
  const double R2 = p.iAz[i + j * sy] * m0[5];
  const bool desc = p.h_desc != 0;
  float S[3];
  S[0] = hsum_x(desc, (float)(dt * (R0 * Ly)), (float)(dt * (R0 * Lz)), e0y, ey3, e0z, ez2);
  S[1] = hsum_y(desc, (float)(dt * (R1 * Lx)), (float)(dt * (R1 * Lz)), e0x, ex3, e0z, ez1);
  S[2] = hsum_z(desc, (float)(dt * (R2 * Lx)), (float)(dt * (R2 * Ly)), e0x, ex2, e0y, ey1);
#pragma unroll
  for (int d = 0; d < 3; d++) {
    float t;
    int8_t q;
    comp_add(h[d], hq[d], -S[d], t, q);
    st.H_out[d * N + n] = t;
    st.Hc_out[d * N + n] = q;
  }
}

__global__ void __launch_bounds__(kCompX * kCompY)
k_e_comp(FitParams<double> p, CompState st, long long step) {
  const int i = 2 + blockIdx.x * kCompX + threadIdx.x;
  const int j = 2 + blockIdx.y * kCompY + threadIdx.y;
  const int k = 2 + blockIdx.z;
  if (i > p.Nx - 3 || j > p.Ny - 3) return;
  const long long N = p.N;
  const int sy = p.Nx, sz = (int)p.NxNy;
  const long long n = i + (long long)j * sy + (long long)k * sz;
  const float* hx = st.H_out + n;
  const float* hy = st.H_out + N + n;
  const float* hz = st.H_out + 2 * N + n;
  const float h0x = hx[0], h0y = hy[0], h0z = hz[0];
  const float hy1 = hy[-1], hz1 = hz[-1], hx2 = hx[-sy], hz2 = hz[-sy], hx3 = hx[-sz],
              hy3 = hy[-sz];
  const float e[3] = {st.E_in[n], st.E_in[N + n], st.E_in[2 * N + n]};
  const int8_t eq[3] = {st.Ec_in[n], st.Ec_in[N + n], st.Ec_in[2 * N + n]};
  const double* m0 = p.mat + 9 * load_id(p.mat_id, p.id_bytes, n);
  const double dt = p.dt;
  const double tLx = p.tLx[i], tLy = p.tLy[j], tLz = p.tLz[k];
  const double R0 = m0[0] * p.itAx[j + k * p.Ny];
  const double R1 = m0[1] * p.itAy[i + k * sy];
  const double R2 = m0[2] * p.itAz[i + j * sy];
  float cu[3];
  cu[0] = ecurl_x((float)(dt * (R0 * tLy)), (float)(dt * (R0 * tLz)), h0y, hz2, hy3, h0z);
  cu[1] = ecurl_y((float)(dt * (R1 * tLx)), (float)(dt * (R1 * tLz)), h0x, hz1, hx3, h0z);
  cu[2] = ecurl_z((float)(dt * (R2 * tLx)), (float)(dt * (R2 * tLy)), h0x, hy1, hx2, h0y);
  Cell c;
  c.i = i; c.j = j; c.k = k;
  const double ez_old = comp_value(e[2], eq[2]);
  if (p.cap_on) capture(p, c, n, step, ez_old);
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double eold = d == 2 ? ez_old : comp_value(e[d], eq[d]);
    const double jv = j_in(p, d, c, n, step, eold, m0[6 + d]);
    const float delta = __fsub_rn(cu[d], (float)(dt * m0[d] * jv));
    float t;
    int8_t q;
    comp_add(e[d], eq[d], delta, t, q);
    st.E_out[d * N + n] = t;
    st.Ec_out[d * N + n] = q;
  }
}

__global__ void __launch_bounds__(256) k_h_comp_shell(FitParams<double> p, CompState st,
                                                       long long count) {
  const long long idx = blockIdx.x * 256LL + threadIdx.x;
  if (idx >= count) return;
  const Cell c = shell_cell(idx, p.Nx, p.Ny, p.Nz);
  const long long n = c.i + (long long)c.j * p.Nx + (long long)c.k * p.NxNy;
  const long long N = p.N;
  const long long off[4] = {0, 1, (long long)p.Nx, p.NxNy};
  auto ev = [&](int e, int kind) -> double {
    const long long m = e * N + n + off[kind];
    return comp_value(st.E_in[m], st.Ec_in[m]);
  };
  const int id = load_id(p.mat_id, p.id_bytes, n);
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double hold = comp_value(st.H_in[d * N + n], st.Hc_in[d * N + n]);
    const double h = h_row_acc(p, hold, d, c, n, id, ev);
    float t;
    int8_t q;
    comp_split(h, t, q);
    st.H_out[d * N + n] = t;
    st.Hc_out[d * N + n] = q;
  }
}

__global__ void __launch_bounds__(256) k_e_comp_shell(FitParams<double> p, CompState st,
                                                       long long step, long long count) {
  const long long idx = blockIdx.x * 256LL + threadIdx.x;
  if (idx >= count) return;
  const Cell c = shell_cell(idx, p.Nx, p.Ny, p.Nz);
  const long long n = c.i + (long long)c.j * p.Nx + (long long)c.k * p.NxNy;
  const long long N = p.N;
  const long long off[4] = {0, 1, (long long)p.Nx, p.NxNy};
  auto hv = [&](int e, int kind) -> double {
    return (double)st.H_out[e * N + n - off[kind]];
  };
  const int id = load_id(p.mat_id, p.id_bytes, n);
  const double ez_old = comp_value(st.E_in[2 * N + n], st.Ec_in[2 * N + n]);
  if (p.cap_on) capture(p, c, n, step, ez_old);
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double ieps = p.mat[9 * id + d], sigma = p.mat[9 * id + 6 + d];
    const double eold = comp_value(st.E_in[d * N + n], st.Ec_in[d * N + n]);
    const double jv = j_in(p, d, c, n, step, eold, sigma);
    const double curl = e_curl_acc(p, d, c, n, ieps, hv);
    const double enew = eold + p.dt * (curl - ieps * jv);
    float t;
    int8_t q;
    comp_split(enew, t, q);
    st.E_out[d * N + n] = t;
    st.Ec_out[d * N + n] = q;
  }
}

__global__ void k_comp_zero_ghosts(FitParams<double> p, float* E, float* H, int8_t* Ec,
                                   int8_t* Hc) {
  const long long n = blockIdx.x * 256LL + threadIdx.x;
  if (n >= p.N) return;
  const Cell c = cell_of(n, p.Nx, p.Ny);
  const long long N = p.N;
  auto zh = [&](int d) { H[d * N + n] = 0.0f; Hc[d * N + n] = 0; };
  auto ze = [&](int d) { E[d * N + n] = 0.0f; Ec[d * N + n] = 0; };
  if (c.i == p.Nx - 1) { zh(1); zh(2); ze(0); }
  if (c.j == p.Ny - 1) { zh(0); zh(2); ze(1); }
  if (c.k == p.Nz - 1) { zh(0); zh(1); ze(2); }
}

__global__ void k_comp_sigma_e(FitParams<double> p, const float* E, const int8_t* Ec, float* J) {
  const long long n = blockIdx.x * 256LL + threadIdx.x;
  if (n >= p.N) return;
  const int id = load_id(p.mat_id, p.id_bytes, n);
#pragma unroll
  for (int d = 0; d < 3; d++)
    J[d * p.N + n] = (float)(p.mat[9 * id + 6 + d] * comp_value(E[d * p.N + n], Ec[d * p.N + n]));
}

}  // namespace wk

using namespace wk;

static int comp_desc_check(const wk_fit_desc* d, const char* where) {
  if (d->dtype != WK_F32C) return wk_fail(WK_E_DTYPE, "%s: dtype must be WK_F32C", where);
  if (!d->Ec[0] || !d->Ec[1] || !d->Hc[0] || !d->Hc[1])
    return wk_fail(WK_E_NULL, "%s: compensation buffers missing", where);
  if (d->j_mode == WK_J_ARRAY)
    return wk_fail(WK_E_MODE, "%s: WK_J_ARRAY is not available with WK_F32C", where);
  if (d->Nx < 5 || d->Ny < 5 || d->Nz < 5 || d->Nz - 4 > 65535 || (d->Ny - 4 + 1) / 2 > 65535)
    return wk_fail(WK_E_SHAPE, "%s: WK_F32C needs every dimension >= 5", where);
  return WK_OK;
}

static CompState comp_state(const wk_fit_desc* d, int par) {
  CompState s;
  s.E_in = (const float*)d->E[par];
  s.H_in = (const float*)d->H[par];
  s.E_out = (float*)d->E[par ^ 1];
  s.H_out = (float*)d->H[par ^ 1];
  s.Ec_in = (const int8_t*)d->Ec[par];
  s.Hc_in = (const int8_t*)d->Hc[par];
  s.Ec_out = (int8_t*)d->Ec[par ^ 1];
  s.Hc_out = (int8_t*)d->Hc[par ^ 1];
  return s;
}

int wk_comp_step(const wk_fit_desc* d, int n_steps, long long step0, cudaStream_t st) {
  int rc = comp_desc_check(d, "wk_fit_step");
  if (rc) return rc;
  int par = d->par;
  const long long count = (long long)d->Nx * d->Ny * d->Nz -
                          (long long)(d->Nx - 4) * (d->Ny - 4) * (d->Nz - 4);
  const unsigned sb = (unsigned)((count + 255) / 256);
  dim3 blk(kCompX, kCompY);
  dim3 grid((d->Nx - 4 + kCompX - 1) / kCompX, (d->Ny - 4 + kCompY - 1) / kCompY, d->Nz - 4);
  for (int s = 0; s < n_steps; s++) {
    FitParams<double> p = make_params<double>(d, par);
    CompState cs = comp_state(d, par);
    timer_begin(st);
    k_h_comp<<<grid, blk, 0, st>>>(p, cs);
    timer_end(st);
    k_h_comp_shell<<<sb, 256, 0, st>>>(p, cs, count);
    timer_begin(st);
    k_e_comp<<<grid, blk, 0, st>>>(p, cs, step0 + s);
    timer_end(st);
    k_e_comp_shell<<<sb, 256, 0, st>>>(p, cs, step0 + s, count);
    par ^= 1;
  }
  return wk_check_launch("wk_fit_step");
}

int wk_comp_zero_ghosts(const wk_fit_desc* d, cudaStream_t st) {
  int rc = comp_desc_check(d, "wk_zero_ghosts");
  if (rc) return rc;
  FitParams<double> p = make_params<double>(d, d->par);
  const long long N = p.N;
  k_comp_zero_ghosts<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(
      p, (float*)d->E[d->par], (float*)d->H[d->par], (int8_t*)d->Ec[d->par],
      (int8_t*)d->Hc[d->par]);
  return wk_check_launch("wk_zero_ghosts");
}

int wk_comp_sigma_e(const wk_fit_desc* d, void* J, cudaStream_t st) {
  int rc = comp_desc_check(d, "wk_sigma_e");
  if (rc) return rc;
  FitParams<double> p = make_params<double>(d, d->par);
  k_comp_sigma_e<<<(unsigned)((p.N + 255) / 256), 256, 0, st>>>(
      p, (const float*)d->E[d->par], (const int8_t*)d->Ec[d->par], (float*)J);
  return wk_check_launch("wk_sigma_e");
}
