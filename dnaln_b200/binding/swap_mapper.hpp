// swap_mapper.hpp — puts GpuMapper where dnaln's sources name Mapper.
//
// Force-included (g++ -include) ahead of an unmodified src/main.cpp, it declares Mapper and
// GpuMapper first (mapper.hpp, guarded by #pragma once, is not read again) and then
// renames the token Mapper to GpuMapper for the rest of the file, so that cmd_map
// (src/main.cpp:46-61) maps every batch through the whole device path and still writes its
// SAM through the reference's own append_sam.
#pragma once
#include "mapper.hpp"
#include "gpu_mapper.hpp"
#define Mapper GpuMapper
