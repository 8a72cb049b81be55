// FP32-compensated FIT step (sm_100a).
//
// State: every E and H component is a float v plus a bf16 compensation c
// holding the rounding error of the last update (v + c carries ~32
// significant bits; a bf16 word decodes with one shift).  The
// update coefficients are formed in FP64 from the FP64 tables (one rounding
// to float per coefficient, dt folded in), the row sums run in float, and
// the increment is added with a Kahan step (y = delta + c, TwoSum(v, y)).
// The Ez capture stores v + c in FP64, so the wake integration and the
// impedance DFT stay FP64.  Two passes (H, then E) over interior tiles and
// the two-cell shell; shell cells decode the state to FP64 and use the
// general FP64 row code.
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/wakis_b200.h"
#include "abi_internal.h"
#include "fit_common.cuh"
#include "fit_kernels.cuh"
#include "fit_comp.cuh"

namespace wk {

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
  const comp_t hq[3] = {st.Hc_in[n], st.Hc_in[N + n], st.Hc_in[2 * N + n]};
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
    comp_t q;
    comp_add(h[d], hq[d], -S[d], t, q);
    st.H_out[d * N + n] = t;
    st.Hc_out[d * N + n] = q;
  }
}

__global__ void __launch_bounds__(kCompX * kCompY)
k_e_comp(FitParams<double> p, CompState st, long long step) {
  step = step_index(p, step);
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
  const comp_t eq[3] = {st.Ec_in[n], st.Ec_in[N + n], st.Ec_in[2 * N + n]};
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
    comp_t q;
    comp_add(e[d], eq[d], delta, t, q);
    st.E_out[d * N + n] = t;
    st.Ec_out[d * N + n] = q;
  }
}

// Interior rows with the compensated stencil (comp_stencil = 1): every E
// (H) value a row reads is the pair v + c of the state, the update factors
// are split into two floats, and the increment is formed with the pair
// operations of fit_comp.cuh before the compensated add; the J = sigma E term
// uses the pair of E_old as well.
__global__ void __launch_bounds__(kCompX * kCompY)
k_h_comp_cs(FitParams<double> p, CompState st) {
  const int i = 2 + blockIdx.x * kCompX + threadIdx.x;
  const int j = 2 + blockIdx.y * kCompY + threadIdx.y;
  const int k = 2 + blockIdx.z;
  if (i > p.Nx - 3 || j > p.Ny - 3) return;
  const long long N = p.N;
  const int sy = p.Nx, sz = (int)p.NxNy;
  const long long n = i + (long long)j * sy + (long long)k * sz;
  // E pair of component d at n + off
  auto ev = [&](int d, long long off) { return st.E_in[d * N + n + off]; };
  auto ec = [&](int d, long long off) { return comp_dec(st.Ec_in[d * N + n + off]); };
  auto diff = [&](int d, long long oa, long long ob) {
    return pair_diff(ev(d, oa), ec(d, oa), ev(d, ob), ec(d, ob));
  };
  const double* m0 = p.mat + 9 * load_id(p.mat_id, p.id_bytes, n);
  const double dt = p.dt;
  const double Lx = p.Lx[i], Ly = p.Ly[j], Lz = p.Lz[k];
  const double R0 = p.iAx[j + k * p.Ny] * m0[3];
  const double R1 = p.iAy[i + k * sy] * m0[4];
  const double R2 = p.iAz[i + j * sy] * m0[5];
  FPair S[3];
  // S_x = a (Ey(n) - Ey(n+NxNy)) + b (Ez(n+Nx) - Ez(n)), a = dt iAx imu Ly, b = .. Lz
  S[0] = pair_add(pair_mul(pair_of(dt * (R0 * Ly)), diff(1, 0, sz)),
                  pair_mul(pair_of(dt * (R0 * Lz)), diff(2, sy, 0)));
  // S_y = a (Ex(n+NxNy) - Ex(n)) + b (Ez(n) - Ez(n+1))
  S[1] = pair_add(pair_mul(pair_of(dt * (R1 * Lx)), diff(0, sz, 0)),
                  pair_mul(pair_of(dt * (R1 * Lz)), diff(2, 0, 1)));
  // S_z = a (Ex(n) - Ex(n+Nx)) + b (Ey(n+1) - Ey(n))
  S[2] = pair_add(pair_mul(pair_of(dt * (R2 * Lx)), diff(0, 0, sy)),
                  pair_mul(pair_of(dt * (R2 * Ly)), diff(1, 1, 0)));
#pragma unroll
  for (int d = 0; d < 3; d++) {
    float t;
    comp_t q;
    comp_add_pair(st.H_in[d * N + n], st.Hc_in[d * N + n], FPair{-S[d].hi, -S[d].lo}, t, q);
    st.H_out[d * N + n] = t;
    st.Hc_out[d * N + n] = q;
  }
}

__global__ void __launch_bounds__(kCompX * kCompY)
k_e_comp_cs(FitParams<double> p, CompState st, long long step) {
  step = step_index(p, step);
  const int i = 2 + blockIdx.x * kCompX + threadIdx.x;
  const int j = 2 + blockIdx.y * kCompY + threadIdx.y;
  const int k = 2 + blockIdx.z;
  if (i > p.Nx - 3 || j > p.Ny - 3) return;
  const long long N = p.N;
  const int sy = p.Nx, sz = (int)p.NxNy;
  const long long n = i + (long long)j * sy + (long long)k * sz;
  // new-H pair of component d at n - off
  auto hv = [&](int d, long long off) { return st.H_out[d * N + n - off]; };
  auto hc = [&](int d, long long off) { return comp_dec(st.Hc_out[d * N + n - off]); };
  auto diff = [&](int d, long long oa, long long ob) {
    return pair_diff(hv(d, oa), hc(d, oa), hv(d, ob), hc(d, ob));
  };
  const float e[3] = {st.E_in[n], st.E_in[N + n], st.E_in[2 * N + n]};
  const comp_t eq[3] = {st.Ec_in[n], st.Ec_in[N + n], st.Ec_in[2 * N + n]};
  const double* m0 = p.mat + 9 * load_id(p.mat_id, p.id_bytes, n);
  const double dt = p.dt;
  const double tLx = p.tLx[i], tLy = p.tLy[j], tLz = p.tLz[k];
  const double R0 = m0[0] * p.itAx[j + k * p.Ny];
  const double R1 = m0[1] * p.itAy[i + k * sy];
  const double R2 = m0[2] * p.itAz[i + j * sy];
  FPair cu[3];
  // curl_x = c1 (Hy(n-NxNy) - Hy(n)) + c2 (Hz(n) - Hz(n-Nx)), c1 = dt ieps itAx tLy, c2 = .. tLz
  cu[0] = pair_add(pair_mul(pair_of(dt * (R0 * tLy)), diff(1, sz, 0)),
                   pair_mul(pair_of(dt * (R0 * tLz)), diff(2, 0, sy)));
  // curl_y = c1 (Hx(n) - Hx(n-NxNy)) + c2 (Hz(n-1) - Hz(n))
  cu[1] = pair_add(pair_mul(pair_of(dt * (R1 * tLx)), diff(0, 0, sz)),
                   pair_mul(pair_of(dt * (R1 * tLz)), diff(2, 1, 0)));
  // curl_z = c1 (Hx(n-Nx) - Hx(n)) + c2 (Hy(n) - Hy(n-1))
  cu[2] = pair_add(pair_mul(pair_of(dt * (R2 * tLx)), diff(0, sy, 0)),
                   pair_mul(pair_of(dt * (R2 * tLy)), diff(1, 0, 1)));
  Cell c;
  c.i = i; c.j = j; c.k = k;
  if (p.cap_on) capture(p, c, n, step, comp_value(e[2], eq[2]));
#pragma unroll
  for (int d = 0; d < 3; d++) {
    FPair jt{0.f, 0.f};   // dt ieps J of the row
    if (d == 2 && i == p.ixs && j == p.iys && (p.line_on || p.beam_on)) {
      const double jv = j_in(p, d, c, n, step, 0.0, 0.0);
      jt = pair_of(dt * m0[d] * jv);
    } else if (p.j_mode == WK_J_SIGMA_E) {
      jt = pair_mul(pair_of(dt * m0[d] * m0[6 + d]), FPair{e[d], comp_dec(eq[d])});
    }
    float t;
    comp_t q;
    comp_add_pair(e[d], eq[d], pair_sub(cu[d], jt), t, q);
    st.E_out[d * N + n] = t;
    st.Ec_out[d * N + n] = q;
  }
}

// Shell of the compensated step (block-uniform decode, ShellGrid): one
// cell per thread (comp_shell_h / comp_shell_e, fit_comp.cuh).
__global__ void __launch_bounds__(kShellBlock) k_h_comp_shell(FitParams<double> p, CompState st,
                                                               ShellGrid g) {
  Cell c;
  if (!shell_cell_of(g, blockIdx.x, threadIdx.x, p.Nx, p.Ny, p.Nz, c)) return;
  comp_shell_h(p, st, c);
}

__global__ void __launch_bounds__(kShellBlock) k_e_comp_shell(FitParams<double> p, CompState st,
                                                               long long step, ShellGrid g) {
  step = step_index(p, step);
  Cell c;
  if (!shell_cell_of(g, blockIdx.x, threadIdx.x, p.Nx, p.Ny, p.Nz, c)) return;
  comp_shell_e(p, st, c, step);
}

__global__ void k_comp_zero_ghosts(FitParams<double> p, float* E, float* H, comp_t* Ec,
                                   comp_t* Hc) {
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

__global__ void k_comp_sigma_e(FitParams<double> p, const float* E, const comp_t* Ec, float* J) {
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

int wk_comp_step(const wk_fit_desc* d, int n_steps, long long step0, cudaStream_t st) {
  int rc = comp_desc_check(d, "wk_fit_step");
  if (rc) return rc;
  int par = d->par;
  const ShellGrid sg = shell_grid(d->Nx, d->Ny, d->Nz);
  const unsigned sb = (unsigned)(sg.nbA + sg.nbB + sg.nbC);
  bool tma = false;
  const bool cstencil = d->comp_stencil != 0;
  if (cstencil && d->kernel == WK_KERNEL_TMA)
    return wk_fail(WK_E_MODE, "wk_fit_step: the compensated stencil runs the two-pass kernels");
  if (!cstencil && (d->kernel == WK_KERNEL_AUTO || d->kernel == WK_KERNEL_TMA)) {
    tma = tma_comp_supported(d, make_params<double>(d, par));
    if (!tma && d->kernel == WK_KERNEL_TMA)
      return wk_fail(WK_E_SHAPE, "wk_fit_step: compensated TMA kernel needs Nx %% 4 == 0, "
                                 "dims >= 5 and at most 64 materials");
  }
  dim3 blk(kCompX, kCompY);
  dim3 grid((d->Nx - 4 + kCompX - 1) / kCompX, (d->Ny - 4 + kCompY - 1) / kCompY, d->Nz - 4);
  for (int s = 0; s < n_steps; s++) {
    FitParams<double> p = make_params<double>(d, par);
    CompState cs = comp_state(d, par);
    if (tma) {
      // fused step (whole grid when every face is PEC-masked, else the
      // interior, then the shell: H from the old state, E from the new H)
      cudaError_t e = launch_tma_comp(d, p, par, step0 + s, st, d->tile_planes);
      if (e != cudaSuccess) return wk_fail(-(int)e, "wk_fit_step: %s", cudaGetErrorString(e));
      const int mode = tma_comp_mode(p);
      if (mode != 1) {
        const ShellGrid g2 = shell_grid(d->Nx, d->Ny, d->Nz, mode == 2);
        const unsigned sb2 = (unsigned)(g2.nbA + g2.nbB + g2.nbC);
        k_h_comp_shell<<<sb2, kShellBlock, 0, st>>>(p, cs, g2);
        k_e_comp_shell<<<sb2, kShellBlock, 0, st>>>(p, cs, step0 + s, g2);
      }
    } else {
      timer_begin(st);
      if (cstencil) k_h_comp_cs<<<grid, blk, 0, st>>>(p, cs);
      else k_h_comp<<<grid, blk, 0, st>>>(p, cs);
      timer_end(st);
      k_h_comp_shell<<<sb, kShellBlock, 0, st>>>(p, cs, sg);
      timer_begin(st);
      if (cstencil) k_e_comp_cs<<<grid, blk, 0, st>>>(p, cs, step0 + s);
      else k_e_comp<<<grid, blk, 0, st>>>(p, cs, step0 + s);
      timer_end(st);
      k_e_comp_shell<<<sb, kShellBlock, 0, st>>>(p, cs, step0 + s, sg);
    }
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
      p, (float*)d->E[d->par], (float*)d->H[d->par], (comp_t*)d->Ec[d->par],
      (comp_t*)d->Hc[d->par]);
  return wk_check_launch("wk_zero_ghosts");
}

int wk_comp_sigma_e(const wk_fit_desc* d, void* J, cudaStream_t st) {
  int rc = comp_desc_check(d, "wk_sigma_e");
  if (rc) return rc;
  FitParams<double> p = make_params<double>(d, d->par);
  k_comp_sigma_e<<<(unsigned)((p.N + 255) / 256), 256, 0, st>>>(
      p, (const float*)d->E[d->par], (const comp_t*)d->Ec[d->par], (float*)J);
  return wk_check_launch("wk_sigma_e");
}
