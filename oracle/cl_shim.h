// ORACLE TEST INFRASTRUCTURE -- not part of the product.
//
// A minimal OpenCL-C -> C++ shim that lets the reference's own kernel sources
//   src/Helmholtz_OpenCL/BoundaryOperatorKernel.cl
//   src/Helmholtz_OpenCL/FarFieldOperatorKernel.cl
//   src/Helmholtz_OpenCL/HerglotzWaveKernel.cl
//   src/Helmholtz_OpenCL/NearFieldOperatorKernel.cl
// compile as host C++ with block_size == 1 (one work item per work group).
// With block_size == 1 every work item accumulates its row C_i over the
// sources j strictly in increasing j order, exactly as the reference does for
// any block size (BoundaryOperatorKernel.cl:69-224), and the local-memory
// barriers become no-ops.  The kernel source is streamed into the compiler by
// build_ref.sh straight from the reference tree; nothing of it is copied into
// this repository.
//
// The specialisation flags that the reference prepends as #defines
// (StringManipulation.hpp:7-17) become run-time globals here, set by the
// driver (cl_shim_driver.h) with the same rule as LoadParameters.hpp:47-80.
#pragma once
#include <cmath>
#include <cstdint>

#define __kernel
#define __global
#define __local
#define __private
#define __constant const
#define CLK_LOCAL_MEM_FENCE 0
#define barrier(x) ((void)0)
#define block_size 1

struct float3 { float x, y, z; };

static inline float3 operator-(const float3 &a, const float3 &b)
{
    float3 r; r.x = a.x - b.x; r.y = a.y - b.y; r.z = a.z - b.z; return r;
}

struct float2
{
    float x, y;
    float2() : x(0.f), y(0.f) {}
    float2(float v) : x(v), y(v) {}
    float2(float a, float b) : x(a), y(b) {}
};

struct float4
{
    union
    {
        struct { float x, y, z, w; };
        float3 xyz;
    };
};

static_assert(sizeof(float2) == 8,  "float2 layout");
static_assert(sizeof(float4) == 16, "float4 layout");

// Work-item ids: one host thread runs one work item at a time.
extern thread_local int cl_shim_global_id;
static inline int get_global_id(int) { return cl_shim_global_id; }
static inline int get_local_id(int)  { return 0; }

static inline float sincos(float x, float *c) { *c = std::cos(x); return std::sin(x); }
static inline float sqrt(float x) { return std::sqrt(x); }

// Run-time replacements for the #define flags of StringManipulation.hpp:10-17.
extern int Re_single_layer, Im_single_layer;
extern int Re_double_layer, Im_double_layer;
extern int Re_adjdbl_layer, Im_adjdbl_layer;
