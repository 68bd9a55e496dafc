// lcs_internal.h -- error recording shared by the C-ABI entry points.
#pragma once
#include "../../include/lcs_gpu.h"

// Records `msg` as this thread's last error and returns `code`.
int lcs_fail(int code, const char* msg);
