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
