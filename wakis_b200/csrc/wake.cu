// Wake potential and impedance kernels (sm_100a) and their C-ABI launchers.
//
// wk_wake_potential  calc_long_WP_3d / calc_long_WP (wakis/wakeSolver.py:
//                    310-554): one thread per s sample, the transverse
//                    positions in upstream order with the running-sum
//                    carry-over, and the z sum in upstream's sequential
//                    order, so WP matches upstream value for value.
// wk_trans_wake      calc_trans_WP (556-612): per s sample the prefix sum
//                    of WP_3d in numpy's pairwise summation order.
// wk_dft_bins        the kept bins 0 <= f < fmax of np.fft.fft(x, n=N)
//                    (calc_long_Z / calc_trans_Z, 679-766) as a direct DFT.
#include <stdint.h>

#include <mutex>

#include "../../include/wakis_b200.h"
#include "abi_internal.h"

namespace {

template <typename H>
__global__ void k_wake_potential(const H* __restrict__ hist, long long hist_nt, int Nzh,
                                 const int* __restrict__ win_map, int n_win, int carry,
                                 const double* __restrict__ z, const double* __restrict__ dz,
                                 int nz, int k_off, const double* __restrict__ s, int ns,
                                 const long long* __restrict__ key_order, long long nt,
                                 double v, double zmin, double zmax, double t0, double ti,
                                 double dt, double qnorm, int counter_moving,
                                 double* __restrict__ WP3d) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= ns) return;
  const double sn = s[n];
  const double zmin_v = __ddiv_rn(zmin, v);
  const double zmax_v = __ddiv_rn(zmax, -v);
  double prev = 0.0;
  for (int w = 0; w < n_win; w++) {
    double acc = carry ? prev : 0.0;
    const H* hw = hist + (long long)win_map[w] * Nzh * hist_nt;
    for (int k = 0; k < nz; k++) {
      double ts;
      int kz;
      double coef;
      if (!counter_moving) {
        ts = __dadd_rn(__dsub_rn(__dsub_rn(__ddiv_rn(__dadd_rn(z[k], sn), v), zmin_v), t0), ti);
        kz = k + k_off;
        coef = dz[k];
      } else {
        int kr = nz - 1 - k;
        ts = __dadd_rn(__dsub_rn(__dsub_rn(__ddiv_rn(__dsub_rn(z[kr], sn), -v), zmax_v), t0), ti);
        kz = kr + k_off;
        coef = -dz[k];
      }
      double q = __ddiv_rn(ts, dt);
      long long it = (long long)q;   // truncation toward zero, as int()
      if (it < nt) {
        if (it < 0) it += nt;          // negative index wraps as in numpy
        if (it < 0) continue;
        long long t = key_order[it];
        if (t < 0 || t >= hist_nt) continue;   // no such history column
        double e = (double)hw[(long long)kz * hist_nt + t];
        acc = __dadd_rn(acc, __dmul_rn(e, coef));
      }
    }
    acc = __ddiv_rn(acc, qnorm);
    WP3d[(long long)w * ns + n] = acc;
    prev = acc;
  }
}

// numpy's pairwise summation (blocks of <= 128 with 8 accumulators, halves
// rounded down to a multiple of 8), evaluated with an explicit stack.
__device__ double pw_leaf(const double* a, long long n) {
  if (n < 8) {
    double r = -0.0;
    for (long long i = 0; i < n; i++) r = __dadd_rn(r, a[i]);
    return r;
  }
  double r[8];
  for (int j = 0; j < 8; j++) r[j] = a[j];
  long long i = 8;
  for (; i < n - (n % 8); i += 8)
    for (int j = 0; j < 8; j++) r[j] = __dadd_rn(r[j], a[i + j]);
  double res = __dadd_rn(__dadd_rn(__dadd_rn(r[0], r[1]), __dadd_rn(r[2], r[3])),
                         __dadd_rn(__dadd_rn(r[4], r[5]), __dadd_rn(r[6], r[7])));
  for (; i < n; i++) res = __dadd_rn(res, a[i]);
  return res;
}

__device__ __forceinline__ long long pw_half(long long n) {
  long long n2 = n / 2;
  return n2 - n2 % 8;
}

__device__ double pw_sum(const double* a, long long n) {
  long long lo_s[48], n_s[48];
  double left_s[48];
  int stage[48];
  int sp = 0;
  lo_s[0] = 0; n_s[0] = n; stage[0] = 0;
  while (true) {
    long long m = n_s[sp];
    if (m <= 128) {
      double result = pw_leaf(a + lo_s[sp], m);
      while (true) {
        if (sp == 0) return result;
        sp--;
        if (stage[sp] == 1) {
          left_s[sp] = result;
          stage[sp] = 2;
          long long n2 = pw_half(n_s[sp]);
          lo_s[sp + 1] = lo_s[sp] + n2;
          n_s[sp + 1] = n_s[sp] - n2;
          stage[sp + 1] = 0;
          sp++;
          break;
        }
        result = __dadd_rn(left_s[sp], result);
      }
    } else {
      stage[sp] = 1;
      lo_s[sp + 1] = lo_s[sp];
      n_s[sp + 1] = pw_half(m);
      stage[sp + 1] = 0;
      sp++;
    }
  }
}

// Positions (+1,0) (-1,0) (0,+1) (0,-1) are w = 7, 1, 5, 3 of the 3x3 block;
// each thread forms the four prefix integrals of its s sample directly.
__global__ void k_trans_wake(const double* __restrict__ WP3d, int ns, double ds, double dxsum,
                             double dysum, double* __restrict__ WPx, double* __restrict__ WPy) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= ns) return;
  double ixp = __dmul_rn(pw_sum(WP3d + 7LL * ns, n), ds);
  double ixm = __dmul_rn(pw_sum(WP3d + 1LL * ns, n), ds);
  double iyp = __dmul_rn(pw_sum(WP3d + 5LL * ns, n), ds);
  double iym = __dmul_rn(pw_sum(WP3d + 3LL * ns, n), ds);
  WPx[n] = __ddiv_rn(-__dsub_rn(ixp, ixm), dxsum);
  WPy[n] = __ddiv_rn(-__dsub_rn(iyp, iym), dysum);
}

// ------------------------------------------------------------- streaming --
// The s sample index n and z index k of the sum for WP(s_n) read step
// it(n, k) = (long)(ts/dt) (same rounded expression as k_wake_potential).
__device__ __forceinline__ long long wp_it(double zk, double sn, double v, double zmin_v,
                                           double zmax_v, double t0, double ti, double dt,
                                           int counter_moving) {
  double ts;
  if (!counter_moving)
    ts = __dadd_rn(__dsub_rn(__dsub_rn(__ddiv_rn(__dadd_rn(zk, sn), v), zmin_v), t0), ti);
  else
    ts = __dadd_rn(__dsub_rn(__dsub_rn(__ddiv_rn(__dsub_rn(zk, sn), -v), zmax_v), t0), ti);
  return (long long)__ddiv_rn(ts, dt);
}

// One thread per (window w, z index k, step r of the chunk): the steps
// step0 .. step0+n_steps-1 of the Ez window history are in ring columns
// 0 .. n_steps-1.  Step m sits at position p = pos[m] of upstream's sorted
// key list (pos = NULL: p = m); it adds Ez(w, k, m) * coef_k to acc[w][n]
// for every s sample n whose sum reads position p, i.e. it(n, k) == p.
// it(n, k) = it(0, k) + n within one (the s axis steps by v*dt), so the
// candidates are n = p - it(0, k) + [-4, 4], each tested with the exact
// expression.
template <typename H>
__global__ void k_wake_accumulate(const H* __restrict__ ring, long long ring_nt, int Nzh,
                                  long long step0, int n_steps, const int* __restrict__ win_map,
                                  int n_win, const double* __restrict__ z,
                                  const double* __restrict__ dz, int nz, int k_off,
                                  const double* __restrict__ s, int ns,
                                  const long long* __restrict__ pos, long long nt, double v,
                                  double zmin, double zmax, double t0, double ti, double dt,
                                  int counter_moving, double* __restrict__ acc) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per_w = (long long)nz * n_steps;
  if (g >= per_w * n_win) return;
  const int w = (int)(g / per_w);
  const long long rem = g - w * per_w;
  const int k = (int)(rem / n_steps);
  const int r = (int)(rem - (long long)k * n_steps);
  const long long m = step0 + r;
  const long long p = pos ? pos[m] : m;
  if (p < 0 || p >= nt) return;
  const double zmin_v = __ddiv_rn(zmin, v);
  const double zmax_v = __ddiv_rn(zmax, -v);
  int kz;
  double zk, coef;
  if (!counter_moving) {
    zk = z[k]; kz = k + k_off; coef = dz[k];
  } else {
    const int kr = nz - 1 - k;
    zk = z[kr]; kz = kr + k_off; coef = -dz[k];
  }
  const double e = (double)ring[((long long)win_map[w] * Nzh + kz) * ring_nt + r];
  const long long it0 = wp_it(zk, s[0], v, zmin_v, zmax_v, t0, ti, dt, counter_moving);
  const long long n_est = p - it0;
  for (long long n = n_est - 4; n <= n_est + 4; n++) {
    if (n < 0 || n >= ns) continue;
    if (wp_it(zk, s[n], v, zmin_v, zmax_v, t0, ti, dt, counter_moving) == p)
      atomicAdd(acc + (long long)w * ns + n, __dmul_rn(e, coef));
  }
}

// WP_3d[w][n] = ((carry ? WP_3d[w-1][n] : 0) + acc[w][n]) / qnorm, the
// windows in order (upstream's carry-over, wakeSolver.py:485,536).
__global__ void k_wake_finalize(const double* __restrict__ acc, int n_win, int ns, int carry,
                                double qnorm, double* __restrict__ WP3d) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= ns) return;
  double prev = 0.0;
  for (int w = 0; w < n_win; w++) {
    const double a = __ddiv_rn(__dadd_rn(carry ? prev : 0.0, acc[(long long)w * ns + n]), qnorm);
    WP3d[(long long)w * ns + n] = a;
    prev = a;
  }
}

// -------------------------------------------------- transverse, by scans --
// Double-double running sums (TwoSum, Knuth): the prefix integrals of the
// Panofsky-Wenzel transverse wake to ~106 bits, rounded once, for long s
// axes where the per-sample pairwise sums of k_trans_wake (O(ns^2)) do not
// scale.  Positions w = 7, 1, 5, 3 of the 3x3 block.
struct DD { double hi, lo; };
__device__ __forceinline__ DD dd_add(DD a, double b) {
  const double s = __dadd_rn(a.hi, b);
  const double bb = __dsub_rn(s, a.hi);
  const double err = __dadd_rn(__dsub_rn(a.hi, __dsub_rn(s, bb)), __dsub_rn(b, bb));
  const double lo = __dadd_rn(a.lo, err);
  const double hi = __dadd_rn(s, lo);
  return {hi, __dsub_rn(lo, __dsub_rn(hi, s))};
}
__device__ __forceinline__ DD dd_add(DD a, DD b) {
  DD r = dd_add(a, b.hi);
  return dd_add(r, b.lo);
}

constexpr int kScanThreads = 256;
__device__ __forceinline__ int trans_win(int q) { return q == 0 ? 7 : (q == 1 ? 1 : (q == 2 ? 5 : 3)); }

// Segment g of `seg` samples: its four window sums (double-double) into
// part[g][4] (scratch).  Deterministic: each thread sums a fixed stride,
// then a fixed-shape tree.
__global__ void k_trans_part(const double* __restrict__ WP3d, int ns, int seg,
                             DD* __restrict__ part) {
  __shared__ DD red[4][kScanThreads];
  const int g = blockIdx.x;
  const long long a = (long long)g * seg, b = min((long long)ns, a + seg);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    DD acc = {0.0, 0.0};
    const double* x = WP3d + (long long)trans_win(q) * ns;
    for (long long n = a + threadIdx.x; n < b; n += kScanThreads) acc = dd_add(acc, x[n]);
    red[q][threadIdx.x] = acc;
  }
  __syncthreads();
  for (int h = kScanThreads / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h)
#pragma unroll
      for (int q = 0; q < 4; q++) red[q][threadIdx.x] = dd_add(red[q][threadIdx.x], red[q][threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x < 4) part[(long long)g * 4 + threadIdx.x] = red[threadIdx.x][0];
}

// Exclusive scan of the segment sums, in place (one thread per window).
__global__ void k_trans_part_scan(DD* __restrict__ part, int nseg) {
  const int q = threadIdx.x;
  if (q >= 4) return;
  DD run = {0.0, 0.0};
  for (int g = 0; g < nseg; g++) {
    const DD v = part[(long long)g * 4 + q];
    part[(long long)g * 4 + q] = run;
    run = dd_add(run, v);
  }
}

// Segment g: from the segment offsets, thread 0 walks windows 7 and 1
// (WPx), thread 1 windows 5 and 3 (WPy): the exclusive prefix of each
// sample, rounded once and times ds, then the difference quotient.
__global__ void k_trans_final(const double* __restrict__ WP3d, int ns, int seg,
                              const DD* __restrict__ part, double ds, double dxsum,
                              double dysum, double* __restrict__ WPx, double* __restrict__ WPy) {
  const int g = blockIdx.x;
  const int t = threadIdx.x;
  if (t >= 2) return;
  const long long a = (long long)g * seg, b = min((long long)ns, a + seg);
  const int qp = 2 * t, qm = 2 * t + 1;             // (7, 1) or (5, 3)
  const double* xp = WP3d + (long long)trans_win(qp) * ns;
  const double* xm = WP3d + (long long)trans_win(qm) * ns;
  double* out = t == 0 ? WPx : WPy;
  const double den = t == 0 ? dxsum : dysum;
  DD rp = part[(long long)g * 4 + qp], rm = part[(long long)g * 4 + qm];
  for (long long n = a; n < b; n++) {
    const double ip = __dmul_rn(__dadd_rn(rp.hi, rp.lo), ds);
    const double im = __dmul_rn(__dadd_rn(rm.hi, rm.lo), ds);
    out[n] = __ddiv_rn(-__dsub_rn(ip, im), den);
    rp = dd_add(rp, xp[n]);
    rm = dd_add(rm, xm[n]);
  }
}

// One block per (signal, bin); fixed-shape tree reduction (deterministic).
constexpr int kDftThreads = 256;
__global__ void k_dft_bins(const double* __restrict__ x, long long len, long long N,
                           int nbins, double* __restrict__ out) {
  int m = blockIdx.x;
  int sig = blockIdx.y;
  const double* xs = x + (long long)sig * len;
  double re = 0.0, im = 0.0;
  for (long long n = threadIdx.x; n < len; n += kDftThreads) {
    long long r = ((long long)m * n) % N;
    double sn, cs;
    sincospi(__ddiv_rn(2.0 * (double)r, (double)N), &sn, &cs);
    double v = xs[n];
    re = __dadd_rn(re, __dmul_rn(v, cs));
    im = __dsub_rn(im, __dmul_rn(v, sn));
  }
  __shared__ double sre[kDftThreads], sim[kDftThreads];
  sre[threadIdx.x] = re;
  sim[threadIdx.x] = im;
  __syncthreads();
  for (int w = kDftThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sre[threadIdx.x] = __dadd_rn(sre[threadIdx.x], sre[threadIdx.x + w]);
      sim[threadIdx.x] = __dadd_rn(sim[threadIdx.x], sim[threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[((long long)sig * nbins + m) * 2] = sre[0];
    out[((long long)sig * nbins + m) * 2 + 1] = sim[0];
  }
}

}  // namespace

extern "C" int wk_wake_potential(const void* hist, int hist_dtype, long long hist_nt, int Nzh,
                                 const int* win_map, int n_win, int carry, const double* z,
                                 const double* dz, int nz, int k_off, const double* s, int ns,
                                 const long long* key_order, long long nt, double v,
                                 double zmin, double zmax, double t0, double ti, double dt,
                                 double qnorm, int counter_moving, double* WP3d, void* stream) {
  if (!hist || !win_map || !z || !dz || !s || !key_order || !WP3d)
    return wk_fail(WK_E_NULL, "wk_wake_potential: NULL pointer");
  if (hist_dtype != WK_F64 && hist_dtype != WK_F32)
    return wk_fail(WK_E_DTYPE, "wk_wake_potential: hist dtype %d", hist_dtype);
  if (ns < 0 || nz < 0 || n_win < 1 || hist_nt < 1 || Nzh < 1 || k_off < 0 ||
      k_off + nz > Nzh || nt > hist_nt)
    return wk_fail(WK_E_RANGE, "wk_wake_potential: sizes (ns %d nz %d nwin %d nt %lld)",
                   ns, nz, n_win, nt);
  if (ns == 0) return WK_OK;
  cudaStream_t st = (cudaStream_t)stream;
  int threads = 128, blocks = (ns + threads - 1) / threads;
  if (hist_dtype == WK_F64)
    k_wake_potential<double><<<blocks, threads, 0, st>>>(
        (const double*)hist, hist_nt, Nzh, win_map, n_win, carry, z, dz, nz, k_off, s, ns,
        key_order, nt, v, zmin, zmax, t0, ti, dt, qnorm, counter_moving, WP3d);
  else
    k_wake_potential<float><<<blocks, threads, 0, st>>>(
        (const float*)hist, hist_nt, Nzh, win_map, n_win, carry, z, dz, nz, k_off, s, ns,
        key_order, nt, v, zmin, zmax, t0, ti, dt, qnorm, counter_moving, WP3d);
  return wk_check_launch("wk_wake_potential");
}

extern "C" int wk_trans_wake(const double* WP3d, int ns, double ds, double dxsum, double dysum,
                             double* WPx, double* WPy, void* stream) {
  if (!WP3d || !WPx || !WPy) return wk_fail(WK_E_NULL, "wk_trans_wake: NULL pointer");
  if (ns < 0) return wk_fail(WK_E_RANGE, "wk_trans_wake: ns %d", ns);
  if (ns == 0) return WK_OK;
  cudaStream_t st = (cudaStream_t)stream;
  int threads = 128, blocks = (ns + threads - 1) / threads;
  k_trans_wake<<<blocks, threads, 0, st>>>(WP3d, ns, ds, dxsum, dysum, WPx, WPy);
  return wk_check_launch("wk_trans_wake");
}

extern "C" int wk_dft_bins(const double* x, int nsig, long long len, long long N, int nbins,
                           double* out, void* stream) {
  if (!x || !out) return wk_fail(WK_E_NULL, "wk_dft_bins: NULL pointer");
  if (nsig < 1 || len < 0 || nbins < 0 || N < 1 || len > N || nbins > N || nsig > 65535)
    return wk_fail(WK_E_RANGE, "wk_dft_bins: nsig %d len %lld N %lld nbins %d", nsig, len, N,
                   nbins);
  if (nbins == 0) return WK_OK;
  if ((double)N * (double)nbins > 9.0e18)
    return wk_fail(WK_E_RANGE, "wk_dft_bins: N*nbins overflows the index product");
  cudaStream_t st = (cudaStream_t)stream;
  dim3 grid(nbins, nsig);
  k_dft_bins<<<grid, kDftThreads, 0, st>>>(x, len, N, nbins, out);
  return wk_check_launch("wk_dft_bins");
}

extern "C" int wk_wake_accumulate(const void* ring, int ring_dtype, long long ring_nt, int Nzh,
                                  long long step0, int n_steps, const int* win_map, int n_win,
                                  const double* z, const double* dz, int nz, int k_off,
                                  const double* s, int ns, const long long* pos, long long nt,
                                  double v, double zmin, double zmax, double t0, double ti,
                                  double dt, int counter_moving, double* acc, void* stream) {
  if (!ring || !win_map || !z || !dz || !s || !acc)
    return wk_fail(WK_E_NULL, "wk_wake_accumulate: NULL pointer");
  if (ring_dtype != WK_F64 && ring_dtype != WK_F32)
    return wk_fail(WK_E_DTYPE, "wk_wake_accumulate: ring dtype %d", ring_dtype);
  if (ns < 0 || nz < 0 || n_win < 1 || n_steps < 0 || n_steps > ring_nt || Nzh < 1 ||
      k_off < 0 || k_off + nz > Nzh || step0 < 0 || nt < 0)
    return wk_fail(WK_E_RANGE, "wk_wake_accumulate: sizes (ns %d nz %d nwin %d steps %d)", ns,
                   nz, n_win, n_steps);
  if (ns == 0 || nz == 0 || n_steps == 0) return WK_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const long long total = (long long)n_win * nz * n_steps;
  const int threads = 256;
  const long long blocks = (total + threads - 1) / threads;
  if (blocks > 0x7fffffffLL) return wk_fail(WK_E_RANGE, "wk_wake_accumulate: too many steps");
  if (ring_dtype == WK_F64)
    k_wake_accumulate<double><<<(unsigned)blocks, threads, 0, st>>>(
        (const double*)ring, ring_nt, Nzh, step0, n_steps, win_map, n_win, z, dz, nz, k_off, s,
        ns, pos, nt, v, zmin, zmax, t0, ti, dt, counter_moving, acc);
  else
    k_wake_accumulate<float><<<(unsigned)blocks, threads, 0, st>>>(
        (const float*)ring, ring_nt, Nzh, step0, n_steps, win_map, n_win, z, dz, nz, k_off, s,
        ns, pos, nt, v, zmin, zmax, t0, ti, dt, counter_moving, acc);
  return wk_check_launch("wk_wake_accumulate");
}

extern "C" int wk_wake_finalize(const double* acc, int n_win, int ns, int carry, double qnorm,
                                double* WP3d, void* stream) {
  if (!acc || !WP3d) return wk_fail(WK_E_NULL, "wk_wake_finalize: NULL pointer");
  if (ns < 0 || n_win < 1) return wk_fail(WK_E_RANGE, "wk_wake_finalize: ns %d nwin %d", ns, n_win);
  if (ns == 0) return WK_OK;
  cudaStream_t st = (cudaStream_t)stream;
  k_wake_finalize<<<(ns + 127) / 128, 128, 0, st>>>(acc, n_win, ns, carry, qnorm, WP3d);
  return wk_check_launch("wk_wake_finalize");
}

// Segments of the scan: at most max_seg of them, each at least 1024 samples.
static int trans_seg_len(int ns, int max_seg) {
  long long seg = (ns + (long long)max_seg - 1) / max_seg;
  if (seg < 1024) seg = 1024;
  return (int)seg;
}

static int trans_scan_launch(const double* WP3d, int ns, double ds, double dxsum, double dysum,
                             double* WPx, double* WPy, DD* part, int max_seg, cudaStream_t st,
                             const char* where) {
  const int seg = trans_seg_len(ns, max_seg);
  const int nseg = (int)(((long long)ns + seg - 1) / seg);
  k_trans_part<<<nseg, kScanThreads, 0, st>>>(WP3d, ns, seg, part);
  k_trans_part_scan<<<1, 32, 0, st>>>(part, nseg);
  k_trans_final<<<nseg, 32, 0, st>>>(WP3d, ns, seg, part, ds, dxsum, dysum, WPx, WPy);
  return wk_check_launch(where);
}

extern "C" long long wk_trans_wake_scan_scratch_bytes(int ns) {
  if (ns <= 0) return 0;
  const int seg = trans_seg_len(ns, 1 << 20);
  const long long nseg = ((long long)ns + seg - 1) / seg;
  return nseg * 4 * (long long)sizeof(DD);
}

extern "C" int wk_trans_wake_scan(const double* WP3d, int ns, double ds, double dxsum,
                                  double dysum, double* WPx, double* WPy, void* scratch,
                                  long long scratch_bytes, void* stream) {
  if (!WP3d || !WPx || !WPy) return wk_fail(WK_E_NULL, "wk_trans_wake_scan: NULL pointer");
  if (ns < 0) return wk_fail(WK_E_RANGE, "wk_trans_wake_scan: ns %d", ns);
  if (ns == 0) return WK_OK;
  if (!scratch) return wk_fail(WK_E_NULL, "wk_trans_wake_scan: scratch is NULL");
  if (((uintptr_t)scratch % 16) != 0)
    return wk_fail(WK_E_ALIGN, "wk_trans_wake_scan: scratch not 16-byte aligned");
  const long long need = wk_trans_wake_scan_scratch_bytes(ns);
  if (scratch_bytes < need)
    return wk_fail(WK_E_RANGE, "wk_trans_wake_scan: scratch of %lld bytes, %lld needed",
                   scratch_bytes, need);
  return trans_scan_launch(WP3d, ns, ds, dxsum, dysum, WPx, WPy, (DD*)scratch, 1 << 20,
                           (cudaStream_t)stream, "wk_trans_wake_scan");
}

// ------------------------------------------------- without allocation ----
// wk_trans_wake_scan_noalloc keeps its segment sums in this file-scope
// device array instead of caller memory.  Every GPU that loads the library
// holds it (kNoAllocSegments x 4 double-double sums = 256 KiB) until the
// process exits; all calls share it.
constexpr int kNoAllocSegments = 4096;
constexpr long long kNoAllocMaxSamples = (long long)kNoAllocSegments * 65536;
static __device__ __align__(256) DD g_trans_scratch[kNoAllocSegments * 4];

// Device address of g_trans_scratch, looked up once per device (in host
// code the symbol names a host-side stand-in, not device memory).
static constexpr int kMaxDevices = 64;
static DD* g_trans_scratch_dev[kMaxDevices];
static cudaError_t g_trans_scratch_err[kMaxDevices];
static std::once_flag g_trans_scratch_once[kMaxDevices];

extern "C" int wk_trans_wake_scan_noalloc(const double* WP3d, int ns, double ds, double dxsum,
                                          double dysum, double* WPx, double* WPy,
                                          void* stream) {
  if (!WP3d || !WPx || !WPy)
    return wk_fail(WK_E_NULL, "wk_trans_wake_scan_noalloc: NULL pointer");
  if (ns < 0) return wk_fail(WK_E_RANGE, "wk_trans_wake_scan_noalloc: ns %d", ns);
  if ((long long)ns > kNoAllocMaxSamples)
    return wk_fail(WK_E_RANGE,
                   "wk_trans_wake_scan_noalloc: %d samples is above this entry point's "
                   "maximum of %lld (its built-in scratch holds %d segment sums of at most "
                   "65536 samples each); use wk_trans_wake_scan with caller scratch",
                   ns, kNoAllocMaxSamples, kNoAllocSegments);
  if (ns == 0) return WK_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return wk_fail(-(int)e, "wk_trans_wake_scan_noalloc: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return wk_fail(WK_E_RANGE, "wk_trans_wake_scan_noalloc: device %d", dev);
  std::call_once(g_trans_scratch_once[dev], [dev] {
    void* ptr = nullptr;
    g_trans_scratch_err[dev] = cudaGetSymbolAddress(&ptr, g_trans_scratch);
    g_trans_scratch_dev[dev] = static_cast<DD*>(ptr);
  });
  if (g_trans_scratch_err[dev] != cudaSuccess || !g_trans_scratch_dev[dev])
    return wk_fail(-(int)(g_trans_scratch_err[dev] != cudaSuccess ? g_trans_scratch_err[dev]
                                                                  : cudaErrorInvalidSymbol),
                   "wk_trans_wake_scan_noalloc: device address of the scratch array: %s",
                   cudaGetErrorString(g_trans_scratch_err[dev]));
  return trans_scan_launch(WP3d, ns, ds, dxsum, dysum, WPx, WPy, g_trans_scratch_dev[dev],
                           kNoAllocSegments, (cudaStream_t)stream,
                           "wk_trans_wake_scan_noalloc");
}
