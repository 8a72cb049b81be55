// Internal helpers shared by the C-ABI translation units: error reporting
// into a thread-local message and host-side validation of descriptors.
#pragma once
#include <cuda_runtime.h>
#include "../../include/wakis_b200.h"

int wk_fail(int code, const char* fmt, ...);
int wk_check_launch(const char* where);
int wk_validate_fit(const wk_fit_desc* d, const char* where);
