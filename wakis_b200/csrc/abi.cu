// C-ABI bookkeeping: version, thread-local error message, argument checks.
#include <cstdarg>
#include <cstdint>
#include <cstdio>

#include "abi_internal.h"

static thread_local char g_msg[512] = "";

extern "C" int wk_version(void) { return WK_ABI_VERSION; }

extern "C" const char* wk_last_error(void) { return g_msg; }

int wk_fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
  va_end(ap);
  return code;
}

int wk_check_launch(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return wk_fail(-(int)e, "%s: %s", where, cudaGetErrorString(e));
  return WK_OK;
}

static bool aligned(const void* p, int bytes) {
  return ((uintptr_t)p % (uintptr_t)bytes) == 0;
}

int wk_validate_fit(const wk_fit_desc* d, const char* where) {
  if (!d) return wk_fail(WK_E_NULL, "%s: descriptor is NULL", where);
  if (d->Nx < 2 || d->Ny < 2 || d->Nz < 2)
    return wk_fail(WK_E_SHAPE, "%s: grid %dx%dx%d (each dimension must be >= 2)", where,
                   d->Nx, d->Ny, d->Nz);
  if ((long long)d->Nx * d->Ny * d->Nz > (1LL << 40))
    return wk_fail(WK_E_SHAPE, "%s: grid too large", where);
  if (d->dtype != WK_F64 && d->dtype != WK_F32 && d->dtype != WK_F32C)
    return wk_fail(WK_E_DTYPE, "%s: dtype %d", where, d->dtype);
  if (d->id_bytes != 1 && d->id_bytes != 2 && d->id_bytes != 4)
    return wk_fail(WK_E_DTYPE, "%s: id_bytes %d", where, d->id_bytes);
  const int es = d->dtype == WK_F64 ? 8 : 4;          // state elements
  const int ts = d->dtype == WK_F32 ? 4 : 8;          // table elements
  const void* req[] = {d->E[0], d->E[1], d->H[0], d->H[1], d->mat_id, d->mat_table,
                       d->Lx, d->Ly, d->Lz, d->tLx, d->tLy, d->tLz,
                       d->iAx, d->iAy, d->iAz, d->itAx, d->itAy, d->itAz};
  const char* names[] = {"E[0]", "E[1]", "H[0]", "H[1]", "mat_id", "mat_table",
                         "Lx", "Ly", "Lz", "tLx", "tLy", "tLz",
                         "iAx", "iAy", "iAz", "itAx", "itAy", "itAz"};
  for (int i = 0; i < 18; i++) {
    if (!req[i]) return wk_fail(WK_E_NULL, "%s: %s is NULL", where, names[i]);
    int a = (i == 4) ? d->id_bytes : (i < 4 ? es : ts);
    if (!aligned(req[i], a)) return wk_fail(WK_E_ALIGN, "%s: %s misaligned", where, names[i]);
  }
  if (d->par != 0 && d->par != 1) return wk_fail(WK_E_MODE, "%s: par %d", where, d->par);
  if (d->n_mat <= 0) return wk_fail(WK_E_RANGE, "%s: n_mat %d", where, d->n_mat);
  if (d->j_mode < WK_J_ZERO || d->j_mode > WK_J_ARRAY)
    return wk_fail(WK_E_MODE, "%s: j_mode %d", where, d->j_mode);
  if (d->j_mode == WK_J_ARRAY && (!d->J || !aligned(d->J, es)))
    return wk_fail(WK_E_NULL, "%s: J missing or misaligned for WK_J_ARRAY", where);
  if (d->beam_on) {
    if (d->ixs < 0 || d->ixs >= d->Nx || d->iys < 0 || d->iys >= d->Ny)
      return wk_fail(WK_E_RANGE, "%s: beam line (%d,%d) off grid", where, d->ixs, d->iys);
    if (!d->zc) return wk_fail(WK_E_NULL, "%s: zc is NULL", where);
  }
  if (d->line_on) {
    if (!d->line || !aligned(d->line, es)) return wk_fail(WK_E_NULL, "%s: line buffer", where);
    if (d->ixs < 0 || d->ixs >= d->Nx || d->iys < 0 || d->iys >= d->Ny || d->line_nsteps < 1)
      return wk_fail(WK_E_RANGE, "%s: line source (%d,%d) off grid", where, d->ixs, d->iys);
  }
  if (d->cap_on) {
    if (!d->cap || !aligned(d->cap, ts)) return wk_fail(WK_E_NULL, "%s: cap buffer", where);
    if (d->cap_i0 < 0 || d->cap_j0 < 0 || d->cap_ni < 1 || d->cap_nj < 1 ||
        d->cap_i0 + d->cap_ni > d->Nx || d->cap_j0 + d->cap_nj > d->Ny || d->cap_nt < 1)
      return wk_fail(WK_E_RANGE, "%s: capture window off grid", where);
  }
  return WK_OK;
}

extern "C" int wk_read_status(int* status, int reset, void* stream) {
  if (!status) return wk_fail(WK_E_NULL, "wk_read_status: status is NULL");
  cudaStream_t st = (cudaStream_t)stream;
  int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess && h != 0 && reset) {
    e = cudaMemsetAsync(status, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  if (e != cudaSuccess)
    return wk_fail(-(int)e, "wk_read_status: %s", cudaGetErrorString(e));
  if (h != 0)
    return wk_fail(WK_E_TIMEOUT,
                   "wk_read_status: a step kernel gave up waiting for a tile load (status %d); "
                   "the fields of the steps since the last check are incomplete", h);
  return WK_OK;
}
