// lcs_internal.h -- error recording shared by the C-ABI entry points.
#pragma once
#include "../../include/lcs_gpu.h"

// Counts one kernel launch of this library (lcs_launch_count).
void lcs_count_launch();

// Records `msg` as this thread's last error and returns `code`.
int lcs_fail(int code, const char* msg);

// construct_tree with the reference's host sort (Morton codes downloaded, sorted on the CPU,
// uploaded; lbvh.cpp:983-993) -- used by the plain one-scene comparator loop only.
int lcs_bvh_construct_host_sort(lcs_bvh* h, lcs_stream stream);
