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

// Shell of the compensated step (block-uniform decode, ShellGrid): the state
// is decoded to FP64, lean rows where they apply, general rows elsewhere,
// and the FP64 result is split back into (float, bf16).
__global__ void __launch_bounds__(kShellBlock) k_h_comp_shell(FitParams<double> p, CompState st,
                                                               ShellGrid g) {
  Cell c;
  if (!shell_cell_of(g, blockIdx.x, threadIdx.x, p.Nx, p.Ny, p.Nz, c)) return;
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

__global__ void __launch_bounds__(kShellBlock) k_e_comp_shell(FitParams<double> p, CompState st,
                                                               long long step, ShellGrid g) {
  step = step_index(p, step);
  Cell c;
  if (!shell_cell_of(g, blockIdx.x, threadIdx.x, p.Nx, p.Ny, p.Nz, c)) return;
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
  if (d->kernel == WK_KERNEL_AUTO || d->kernel == WK_KERNEL_TMA) {
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
      k_h_comp<<<grid, blk, 0, st>>>(p, cs);
      timer_end(st);
      k_h_comp_shell<<<sb, kShellBlock, 0, st>>>(p, cs, sg);
      timer_begin(st);
      k_e_comp<<<grid, blk, 0, st>>>(p, cs, step0 + s);
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
