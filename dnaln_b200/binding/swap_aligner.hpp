// swap_aligner.hpp — puts GpuAligner where dnaln's sources name SimdAligner.
//
// Force-included (g++ -include) ahead of an unmodified dnaln source file, it declares the
// real aligner classes first (align.hpp, guarded by #pragma once, is not read again) and
// then renames the token SimdAligner to GpuAligner for the rest of the file. Compiled this
// way, src/mapper.cpp:10 constructs a GpuAligner where it constructed a SimdAligner — the
// one-line swap a maintainer would make there — and tests/test_main.cpp runs its
// SIMD-versus-scalar checks (simd_kernel_bit_identical_to_scalar and the others) on the GPU.
#pragma once
#include "align.hpp"
#include "gpu_aligner.hpp"
#define SimdAligner GpuAligner
