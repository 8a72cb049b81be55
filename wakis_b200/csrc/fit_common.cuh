// Shared device code of the FIT leap-frog kernels.
//
// The update reproduces upstream's sparse products term by term
// (wakis/solverFIT3D.py:312-322,482-503):
//   H_r -= sum_c fl(fl(dt * fl(fl(iA_r*imu_r) * L_c)) * E_c) * s_rc
//   E_r += dt * (sum_c fl(fl(fl(ieps_r*itA_r) * tL_c) * H_c) * s_rc - ieps_r*J_r)
// with s_rc = +-1 the curl signs, the same rounding of every product and
// the same summation order as scipy's CSR mat-vec over the assembled rows
// (ascending column order, or descending for the H rows when exactly one
// of the PEC/PMC masks was folded in).  All arithmetic uses explicit
// round-to-nearest intrinsics so that no multiply-add is contracted.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace wk {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }

template <typename T>
struct FitParams {
  int Nx, Ny, Nz;
  long long N, NxNy;
  T* E_in; T* H_in; T* E_out; T* H_out;
  T* J;
  int j_mode, use_cond;
  const void* mat_id; int id_bytes;
  const T* mat;
  int n_mat;
  const T *Lx, *Ly, *Lz, *tLx, *tLy, *tLz;
  const T *iAx, *iAy, *iAz, *itAx, *itAy, *itAz;
  int pec_face[6], pmc_face[6];
  int has_pec, has_pmc, h_desc;
  T dt;
  // beam
  int beam_on, ixs, iys, dt_is_f32;
  double dt64, b_qv, b_v, b_s0, b_c0, b_two_sig2, b_dx, b_dy;
  float b_v32, dt32;
  const double* zc;
  int line_on;
  long long line_step0, line_nsteps;
  const T* line;
  // capture
  int cap_on, cap_i0, cap_j0, cap_ni, cap_nj;
  long long cap_nt, cap_step0;
  T* cap;
  int* status;
  const long long* step_dev;   // optional device step counter
  int faces_clean;             // tangential E on PEC faces is +0 (wk_fit_desc)
  long long wait_ns;           // bound of the TMA step-loop waits (wk_fit_desc)
  int steps_per_launch;        // wk_fit_desc.steps_per_launch
  unsigned nx_mul;   // fast division by Nx: q = umulhi(n, nx_mul) >> nx_shift
  int nx_shift;
};

// Magic numbers for q = n / d (2 <= d, 0 <= n < 2^31): p = 31 + ceil(log2 d),
// m = ceil(2^p / d), q = umulhi(n, m) >> (p - 32).
inline void fast_div_magic(unsigned d, unsigned* m, int* shift) {
  int l = 0;
  while ((1ull << l) < d) l++;
  const int p = 31 + l;
  *m = (unsigned)(((1ull << p) + d - 1) / d);
  *shift = p - 32;
}
__device__ __forceinline__ int fast_div(int n, unsigned m, int shift) {
  return (int)(__umulhi((unsigned)n, m) >> shift);
}

__device__ __forceinline__ int load_id(const void* p, int bytes, long long n) {
  if (bytes == 1) return ((const uint8_t*)p)[n];
  if (bytes == 2) return ((const uint16_t*)p)[n];
  return (int)((const uint32_t*)p)[n];
}

// Face masks: later faces overwrite earlier ones in the order x-lo, x-hi,
// y-lo, y-hi, z-lo, z-hi (wakis/boundaries.py:92-101); component d is never
// masked on the faces normal to it.
__device__ __forceinline__ int face_val(const int* f, int d, int i, int j, int k,
                                        int Nx, int Ny, int Nz) {
  int v = 1;
  if (d != 0) { if (i == 0) v = f[0]; if (i == Nx - 1) v = f[1]; }
  if (d != 1) { if (j == 0) v = f[2]; if (j == Ny - 1) v = f[3]; }
  if (d != 2) { if (k == 0) v = f[4]; if (k == Nz - 1) v = f[5]; }
  return v;
}

// Cell coordinates of flat index n (0 <= n < N).
struct Cell { int i, j, k; };
__device__ __forceinline__ Cell cell_of(long long n, int Nx, int Ny) {
  Cell c;
  long long q = n / Nx;
  c.i = (int)(n - q * Nx);
  c.k = (int)(q / Ny);
  c.j = (int)(q - (long long)c.k * Ny);
  return c;
}

// Sum of four terms in ascending or descending order, starting from +0 as
// scipy's csr_matvec does.
template <typename T>
__device__ __forceinline__ T sum4(T a, T b, T c, T d, bool desc) {
  T z = T(0);
  if (!desc) return add(add(add(add(z, a), b), c), d);
  return add(add(add(add(z, d), c), b), a);
}

// Column factor of the H operator: primal length of the column component
// at the column cell, 0 where the PEC mask removes that column.
template <typename T>
__device__ __forceinline__ T colL(const FitParams<T>& p, int d, int i, int j, int k) {
  if (p.has_pec && !face_val(p.pec_face, d, i, j, k, p.Nx, p.Ny, p.Nz)) return T(0);
  return d == 0 ? p.Lx[i] : (d == 1 ? p.Ly[j] : p.Lz[k]);
}
// Column factor of the E operator: dual length, 0 where the PMC mask
// removes that H column.
template <typename T>
__device__ __forceinline__ T coltL(const FitParams<T>& p, int d, int i, int j, int k) {
  if (p.has_pmc && !face_val(p.pmc_face, d, i, j, k, p.Nx, p.Ny, p.Nz)) return T(0);
  return d == 0 ? p.tLx[i] : (d == 1 ? p.tLy[j] : p.tLz[k]);
}

// Neighbour cells in the flat-offset sense of upstream's difference
// operators (P shifts by +1, +Nx, +Nx*Ny on the flat index and only stops at
// the end of the block, wakis/solverFIT3D.py:207-209): stepping past i=Nx-1
// lands on (0, j+1, k), past j=Ny-1 on (i, 0, k+1).
__device__ __forceinline__ Cell plus_x(Cell c, int Nx, int Ny) {
  Cell r = c; r.i++;
  if (r.i == Nx) { r.i = 0; r.j++; if (r.j == Ny) { r.j = 0; r.k++; } }
  return r;
}
__device__ __forceinline__ Cell plus_y(Cell c, int Ny) {
  Cell r = c; r.j++;
  if (r.j == Ny) { r.j = 0; r.k++; }
  return r;
}
__device__ __forceinline__ Cell minus_x(Cell c, int Nx, int Ny) {
  Cell r = c; r.i--;
  if (r.i < 0) { r.i = Nx - 1; r.j--; if (r.j < 0) { r.j = Ny - 1; r.k--; } }
  return r;
}
__device__ __forceinline__ Cell minus_y(Cell c, int Ny) {
  Cell r = c; r.j--;
  if (r.j < 0) { r.j = Ny - 1; r.k--; }
  return r;
}

// H row update for component d at cell c (flat n).  `ev(e, kind)` returns
// the old E component e at n (kind 0), n+1 (1), n+Nx (2) or n+Nx*Ny (3); it
// is only called for terms whose flat index lies inside the grid.
template <typename T, typename EV>
__device__ __forceinline__ T h_row_acc(const FitParams<T>& p, T hold, int d, Cell c,
                                       long long n, int id, EV ev) {
  const long long N = p.N, NxNy = p.NxNy;
  const int Nx = p.Nx, Ny = p.Ny, Nz = p.Nz;
  T iA = d == 0 ? p.iAx[c.j + (long long)c.k * Ny]
                : (d == 1 ? p.iAy[c.i + (long long)c.k * Nx] : p.iAz[c.i + (long long)c.j * Nx]);
  T R = mul(iA, p.mat[9 * id + 3 + d]);
  if (p.has_pmc && !face_val(p.pmc_face, d, c.i, c.j, c.k, Nx, Ny, Nz)) R = T(0);
  const T dt = p.dt;
  auto term = [&](int e, int kind, Cell cc, bool valid, bool pos) -> T {
    if (!valid) return T(0);
    T coef = mul(dt, mul(R, colL(p, e, cc.i, cc.j, cc.k)));
    T v = mul(coef, ev(e, kind));
    return pos ? v : -v;
  };
  Cell kz = c; kz.k++;
  const bool vz = (n + NxNy) < N, vy = (n + Nx) < N, vx = (n + 1) < N;
  T t0, t1, t2, t3;
  if (d == 0) {        // (C e)_x = +ey[n] - ey[n+NxNy] - ez[n] + ez[n+Nx]
    Cell cy = plus_y(c, Ny);
    t0 = term(1, 0, c, true, true);
    t1 = term(1, 3, kz, vz, false);
    t2 = term(2, 0, c, true, false);
    t3 = term(2, 2, cy, vy, true);
  } else if (d == 1) { // (C e)_y = -ex[n] + ex[n+NxNy] + ez[n] - ez[n+1]
    Cell cx = plus_x(c, Nx, Ny);
    t0 = term(0, 0, c, true, false);
    t1 = term(0, 3, kz, vz, true);
    t2 = term(2, 0, c, true, true);
    t3 = term(2, 1, cx, vx, false);
  } else {             // (C e)_z = +ex[n] - ex[n+Nx] - ey[n] + ey[n+1]
    Cell cy = plus_y(c, Ny);
    Cell cx = plus_x(c, Nx, Ny);
    t0 = term(0, 0, c, true, true);
    t1 = term(0, 2, cy, vy, false);
    t2 = term(1, 0, c, true, false);
    t3 = term(1, 1, cx, vx, true);
  }
  return sub(hold, sum4(t0, t1, t2, t3, p.h_desc != 0));
}

// H row reading E from a flat global array.
template <typename T>
__device__ __forceinline__ T h_row(const FitParams<T>& p, const T* __restrict__ Ein,
                                   T hold, int d, Cell c, long long n, int id) {
  const long long N = p.N;
  const long long off[4] = {0, 1, (long long)p.Nx, p.NxNy};
  auto ev = [&](int e, int kind) -> T { return Ein[(long long)e * N + n + off[kind]]; };
  return h_row_acc(p, hold, d, c, n, id, ev);
}

// Curl part of the E row for component d at cell c: sum_c B_rc * H_c, with
// `hv(e, kind)` the new H component e at n (0), n-1 (1), n-Nx (2) or
// n-Nx*Ny (3), only called for in-grid indices.
template <typename T, typename HV>
__device__ __forceinline__ T e_curl_acc(const FitParams<T>& p, int d, Cell c, long long n,
                                        T ieps, HV hv) {
  const long long NxNy = p.NxNy;
  const int Nx = p.Nx, Ny = p.Ny, Nz = p.Nz;
  T itA = d == 0 ? p.itAx[c.j + (long long)c.k * Ny]
                 : (d == 1 ? p.itAy[c.i + (long long)c.k * Nx] : p.itAz[c.i + (long long)c.j * Nx]);
  T R = mul(ieps, itA);
  if (p.has_pec && !face_val(p.pec_face, d, c.i, c.j, c.k, Nx, Ny, Nz)) R = T(0);
  auto term = [&](int e, int kind, Cell cc, bool valid, bool pos) -> T {
    if (!valid) return T(0);
    T coef = mul(R, coltL(p, e, cc.i, cc.j, cc.k));
    T v = mul(coef, hv(e, kind));
    return pos ? v : -v;
  };
  Cell km = c; km.k--;
  const bool vz = n >= NxNy, vy = n >= Nx, vx = n >= 1;
  T t0, t1, t2, t3;
  if (d == 0) {        // +hy[n-NxNy] - hy[n] - hz[n-Nx] + hz[n]
    Cell cy = minus_y(c, Ny);
    t0 = term(1, 3, km, vz, true);
    t1 = term(1, 0, c, true, false);
    t2 = term(2, 2, cy, vy, false);
    t3 = term(2, 0, c, true, true);
  } else if (d == 1) { // -hx[n-NxNy] + hx[n] + hz[n-1] - hz[n]
    Cell cx = minus_x(c, Nx, Ny);
    t0 = term(0, 3, km, vz, false);
    t1 = term(0, 0, c, true, true);
    t2 = term(2, 1, cx, vx, true);
    t3 = term(2, 0, c, true, false);
  } else {             // +hx[n-Nx] - hx[n] - hy[n-1] + hy[n]
    Cell cy = minus_y(c, Ny);
    Cell cx = minus_x(c, Nx, Ny);
    t0 = term(0, 2, cy, vy, true);
    t1 = term(0, 0, c, true, false);
    t2 = term(1, 1, cx, vx, false);
    t3 = term(1, 0, c, true, true);
  }
  return sum4(t0, t1, t2, t3, false);
}

// E-row curl with H values supplied by `hval(comp, flat)`.
template <typename T, typename HV>
__device__ __forceinline__ T e_curl(const FitParams<T>& p, int d, Cell c, long long n,
                                    T ieps, HV hval) {
  const long long off[4] = {0, 1, (long long)p.Nx, p.NxNy};
  auto hv = [&](int e, int kind) -> T { return hval(e, n - off[kind]); };
  return e_curl_acc(p, d, c, n, ieps, hv);
}

// Interior cells: no flat-offset wrap and no face mask touches the cell or
// the neighbours its rows read, so every column length of a row is the
// cell's own per-axis length and each coefficient appears twice.  Same
// products, same order as h_row_acc / e_curl_acc; the leading "+0" of the
// CSR sum is dropped (it can only change the sign of a zero).
// H-row lean condition: 1 <= i <= Nx-3, 1 <= j <= Ny-3, 1 <= k <= Nz-3.
// E-row lean condition: 2 <= i <= Nx-2, 2 <= j <= Ny-2, 2 <= k <= Nz-2.
template <typename T>
__device__ __forceinline__ bool lean_h(int i, int j, int k, int Nx, int Ny, int Nz) {
  return i >= 1 && i <= Nx - 3 && j >= 1 && j <= Ny - 3 && k >= 1 && k <= Nz - 3;
}
template <typename T>
__device__ __forceinline__ bool lean_e(int i, int j, int k, int Nx, int Ny, int Nz) {
  return i >= 2 && i <= Nx - 2 && j >= 2 && j <= Ny - 2 && k >= 2 && k <= Nz - 2;
}

// Single interior H rows.  For a row at cell c: x reads ey(c), ey(c+z),
// ez(c), ez(c+y) with lengths Ly, Lz of c; y reads ex(c), ex(c+z), ez(c),
// ez(c+x) with Lx, Lz; z reads ex(c), ex(c+y), ey(c), ey(c+x) with Lx, Ly.
// R = iA*imu of the row.  Terms t0..t3 in column order, signs + - - +
// (x, z) and - + + - (y).
// Row sums S (H_new = H_old - S) from the two row coefficients a, b.
template <typename T>
__device__ __forceinline__ T hsum_x(bool desc, T a, T b, T ey0, T ey3, T ez0, T ez2) {
  const T t0 = mul(a, ey0), t1 = mul(a, ey3), t2 = mul(b, ez0), t3 = mul(b, ez2);
  return desc ? add(sub(sub(t3, t2), t1), t0) : add(sub(sub(t0, t1), t2), t3);
}
template <typename T>
__device__ __forceinline__ T hsum_y(bool desc, T a, T b, T ex0, T ex3, T ez0, T ez1) {
  const T t0 = mul(a, ex0), t1 = mul(a, ex3), t2 = mul(b, ez0), t3 = mul(b, ez1);
  return desc ? sub(add(sub(t2, t3), t1), t0) : sub(add(sub(t1, t0), t2), t3);
}
template <typename T>
__device__ __forceinline__ T hsum_z(bool desc, T a, T b, T ex0, T ex2, T ey0, T ey1) {
  const T t0 = mul(a, ex0), t1 = mul(a, ex2), t2 = mul(b, ey0), t3 = mul(b, ey1);
  return desc ? add(sub(sub(t3, t2), t1), t0) : add(sub(sub(t0, t1), t2), t3);
}

template <typename T>
__device__ __forceinline__ T h_lean_x(T dt, bool desc, T R, T Ly, T Lz, T ey0, T ey3, T ez0,
                                      T ez2, T hold) {
  return sub(hold, hsum_x(desc, mul(dt, mul(R, Ly)), mul(dt, mul(R, Lz)), ey0, ey3, ez0, ez2));
}
template <typename T>
__device__ __forceinline__ T h_lean_y(T dt, bool desc, T R, T Lx, T Lz, T ex0, T ex3, T ez0,
                                      T ez1, T hold) {
  return sub(hold, hsum_y(desc, mul(dt, mul(R, Lx)), mul(dt, mul(R, Lz)), ex0, ex3, ez0, ez1));
}
template <typename T>
__device__ __forceinline__ T h_lean_z(T dt, bool desc, T R, T Lx, T Ly, T ex0, T ex2, T ey0,
                                      T ey1, T hold) {
  return sub(hold, hsum_z(desc, mul(dt, mul(R, Lx)), mul(dt, mul(R, Ly)), ex0, ex2, ey0, ey1));
}

// All three rows of one interior cell.  E values: *0 at n, y1/z1 at n+1,
// x2/z2 at n+Nx, x3/y3 at n+Nx*Ny.
template <typename T>
__device__ __forceinline__ void h_lean(T dt, bool desc, T R0, T R1, T R2, T Lx, T Ly, T Lz,
                                       T ex0, T ey0, T ez0, T ey1, T ez1, T ex2, T ez2,
                                       T ex3, T ey3, T& hx, T& hy, T& hz) {
  hx = h_lean_x(dt, desc, R0, Ly, Lz, ey0, ey3, ez0, ez2, hx);
  hy = h_lean_y(dt, desc, R1, Lx, Lz, ex0, ex3, ez0, ez1, hy);
  hz = h_lean_z(dt, desc, R2, Lx, Ly, ex0, ex2, ey0, ey1, hz);
}

// Curl of one E row from its two coefficients c1, c2 (signs per component
// as in e_lean below).
template <typename T>
__device__ __forceinline__ T ecurl_x(T c1, T c2, T hy0, T hz2, T hy3, T hz0) {
  return add(sub(sub(mul(c1, hy3), mul(c1, hy0)), mul(c2, hz2)), mul(c2, hz0));
}
template <typename T>
__device__ __forceinline__ T ecurl_y(T c1, T c2, T hx0, T hz1, T hx3, T hz0) {
  return sub(add(sub(mul(c1, hx0), mul(c1, hx3)), mul(c2, hz1)), mul(c2, hz0));
}
template <typename T>
__device__ __forceinline__ T ecurl_z(T c1, T c2, T hx0, T hy1, T hx2, T hy0) {
  return add(sub(sub(mul(c1, hx2), mul(c1, hx0)), mul(c2, hy1)), mul(c2, hy0));
}

// Curl parts of the three E rows.  H values: *0 at n, y1/z1 at n-1,
// x2/z2 at n-Nx, x3/y3 at n-Nx*Ny; R* = ieps*itA of each row.
template <typename T>
__device__ __forceinline__ void e_lean(T R0, T R1, T R2, T tLx, T tLy, T tLz, T hx0, T hy0,
                                       T hz0, T hy1, T hz1, T hx2, T hz2, T hx3, T hy3,
                                       T& cx, T& cy, T& cz) {
  {  // x: +c1*hy3 - c1*hy0 - c2*hz2 + c2*hz0
    const T c1 = mul(R0, tLy), c2 = mul(R0, tLz);
    cx = add(sub(sub(mul(c1, hy3), mul(c1, hy0)), mul(c2, hz2)), mul(c2, hz0));
  }
  {  // y: -c1*hx3 + c1*hx0 + c2*hz1 - c2*hz0
    const T c1 = mul(R1, tLx), c2 = mul(R1, tLz);
    cy = sub(add(sub(mul(c1, hx0), mul(c1, hx3)), mul(c2, hz1)), mul(c2, hz0));
  }
  {  // z: +c1*hx2 - c1*hx0 - c2*hy1 + c2*hy0
    const T c1 = mul(R2, tLx), c2 = mul(R2, tLy);
    cz = add(sub(sub(mul(c1, hx2), mul(c1, hx0)), mul(c2, hy1)), mul(c2, hy0));
  }
}

// Step index of a kernel launched for step `step`: offset by the device
// counter when one is attached (replayed step graphs).
template <typename T>
__device__ __forceinline__ long long step_index(const FitParams<T>& p, long long step) {
  return p.step_dev ? step + *p.step_dev : step;
}

// Gaussian beam current on the line (ixs, iys) at step `step`
// (wakis/sources.py:98-110).  With a float32 time step upstream evaluates
// t = n*dt and v*t in float32 before the float64 profile; the value is
// then stored into the dtype J array.
template <typename T>
__device__ __forceinline__ T beam_j(const FitParams<T>& p, long long step, int k) {
  double vt;
  if (p.dt_is_f32) {
    float t32 = __fmul_rn((float)step, p.dt32);
    vt = (double)__fmul_rn(p.b_v32, t32);
  } else {
    double t = __dmul_rn((double)step, p.dt64);
    vt = __dmul_rn(p.b_v, t);
  }
  double s = __dsub_rn(p.zc[k], vt);
  double u = __dsub_rn(s, p.b_s0);
  double arg = __ddiv_rn(-__dmul_rn(u, u), p.b_two_sig2);
  double prof = __dmul_rn(p.b_c0, exp(arg));
  double jz = __ddiv_rn(__ddiv_rn(__dmul_rn(p.b_qv, prof), p.b_dx), p.b_dy);
  return (T)jz;
}

}  // namespace wk
