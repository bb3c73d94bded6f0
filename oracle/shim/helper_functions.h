/* Stand-in for the CUDA-samples header the reference includes at
 * src/gpu/cudaGridSearch.cuh:42 (absent from this toolkit).  The reference uses only
 * <cstdio> through it, and std::all_of (cudaImageFunctions.cuh:123) needs <algorithm>.
 * Test infrastructure: used only to build oracle/_ref. */
#pragma once
#include <cstdio>
#include <algorithm>
