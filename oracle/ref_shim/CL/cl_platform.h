/* TEST INFRASTRUCTURE ONLY — stand-in for the Khronos OpenCL-Headers cl_platform.h (the
 * reference's CMakeLists.txt:22-26 fetches tag v2026.05.29), which is not installed here.  It
 * declares only the host scalar and vector types the reference's shared headers
 * (include/common/typedefs.h:6-16) use: each vector type is a union of an s[] array and named
 * x/y/z/w members, float2 8-byte and float4 16-byte aligned, as in the Khronos layout.  Used by
 * oracle/build_ref_sppm.py to compile the reference's own host sources for the CPU. */
#ifndef PHX_REF_SHIM_CL_PLATFORM_H
#define PHX_REF_SHIM_CL_PLATFORM_H

#include <stdint.h>

typedef float cl_float;
typedef uint8_t cl_uchar;
typedef int32_t cl_int;
typedef uint32_t cl_uint;
typedef uint64_t cl_ulong;

typedef union {
    cl_float s[2];
    struct {
        cl_float x, y;
    };
} __attribute__((aligned(8))) cl_float2;

typedef union {
    cl_float s[4];
    struct {
        cl_float x, y, z, w;
    };
} __attribute__((aligned(16))) cl_float4;

#endif
