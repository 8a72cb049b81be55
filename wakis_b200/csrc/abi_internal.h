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
