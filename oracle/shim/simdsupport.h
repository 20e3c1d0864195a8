// Stand-in for the reference's CMake-generated simdsupport.h
// (src/liblightmetrica/simdsupport.h.in:24-89). The flags match what the
// reference's CMakeLists.txt:300-309 sets for GCC: SSE..SSE4.2 on, AVX off.
#pragma once
#ifndef LIB_LIGHTMETRICA_SIMD_SUPPORT_H
#define LIB_LIGHTMETRICA_SIMD_SUPPORT_H
#define LM_SSE 1
#define LM_SSE2 1
#define LM_SSE3 1
#define LM_SSSE3 1
#define LM_SSE4_1 1
#define LM_SSE4_2 1
#define LM_SSE4A 0
#define LM_AVX 0
#define LM_AVX2 0
#endif
