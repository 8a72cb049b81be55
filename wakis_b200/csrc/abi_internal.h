// Internal helpers shared by the C-ABI translation units: error reporting
// into a thread-local message and host-side validation of descriptors.
#pragma once
#include <cuda_runtime.h>
#include "../../include/wakis_b200.h"

int wk_fail(int code, const char* fmt, ...);
int wk_check_launch(const char* where);
int wk_validate_fit(const wk_fit_desc* d, const char* where);

// FP32-compensated step and ghost zeroing (fit_comp.cu).
int wk_comp_step(const wk_fit_desc* d, int n_steps, long long step0, cudaStream_t st);
int wk_comp_zero_ghosts(const wk_fit_desc* d, cudaStream_t st);
int wk_comp_sigma_e(const wk_fit_desc* d, void* J, cudaStream_t st);

// Optional CUDA-event timing of the interior kernels of each step (the
// kernels that carry the bulk of the cells), armed by wk_fit_step_timed on
// the calling thread.  Launchers bracket each interior launch with
// timer_begin / timer_end; event pairs beyond the capacity are not timed.
struct KernelTimer {
  cudaEvent_t* ev = nullptr;   // 2 * cap events: begin, end of each launch
  int cap = 0;
  int n = 0;                   // launches recorded
  cudaError_t err = cudaSuccess;
};
extern thread_local KernelTimer* g_kernel_timer;

inline void timer_begin(cudaStream_t st) {
  KernelTimer* t = g_kernel_timer;
  if (!t || t->n >= t->cap) return;
  cudaError_t e = cudaEventRecord(t->ev[2 * t->n], st);
  if (e != cudaSuccess) t->err = e;
}
inline void timer_end(cudaStream_t st) {
  KernelTimer* t = g_kernel_timer;
  if (!t || t->n >= t->cap) return;
  cudaError_t e = cudaEventRecord(t->ev[2 * t->n + 1], st);
  if (e != cudaSuccess) t->err = e;
  t->n++;
}
