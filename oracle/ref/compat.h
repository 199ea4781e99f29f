// TEST INFRASTRUCTURE ONLY.  Pre-included (-include) when compiling the reference rasterizer with
// this image's toolchain (GCC 13 headers, nvcc 12.9):
//  * glibc defines M_1_PIf32 / M_2_PIf32 (used by cuda_rasterizer/auxiliary.h:230-245) as
//    std::float32_t literals, which nvcc cannot generate code for; they are redefined as the plain
//    float literals of the same value;
//  * cuda_rasterizer/rasterizer_impl.h uses uint32_t / uint64_t / std::uintptr_t without including
//    <cstdint>, which older libstdc++ headers pulled in transitively.
#pragma once
#include <cstdint>
#include <math.h>
#undef M_1_PIf32
#undef M_2_PIf32
#define M_1_PIf32 0.318309886183790671537767526745028724f
#define M_2_PIf32 0.636619772367581343075535053490057448f
