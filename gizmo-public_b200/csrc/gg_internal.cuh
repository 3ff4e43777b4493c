// gg_internal.cuh -- device data layout and helpers shared by the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gizmo_gravity_b200.h"

#define GG_MAX_LEVEL 21          // key levels: 21 bits per dimension, 63-bit keys
#define GG_CHUNK_LEVEL 22        // leaf chunks below a full-depth cell
#define GG_MAX_DEPTH 28          // tree depth bound: root + 21 key levels + chunk levels; the last depth is all leaves
#define GG_WARP 32

// error bits of the device error word
#define GG_EBIT_SORT_TIMEOUT 1
#define GG_EBIT_NODE_OVERFLOW 2
#define GG_EBIT_STACK_OVERFLOW 4
#define GG_EBIT_BAD_INPUT 8
#define GG_EBIT_LIST 16
#define GG_EBIT_WALK_TIMEOUT 32

// One particle, 32 bytes: FP64 position, FP32 mass and kernel radius h.
struct __align__(32) GGPart {
    double x, y, z;
    float m, h;
};

// One tree node, 64 bytes.  The first 32 bytes carry what a used node
// contributes (FP64 centre of mass s, mass, cell side); the rest drives the
// opening tests and the descent.
//   leaf:      a = first particle (sorted order), b = -count
//   internal:  a = first child node, b = number of children (children contiguous)
struct __align__(32) GGNode {
    double cx, cy, cz;     // centre of mass (GIZMO's Nodes[].u.d.s)
    float mass, len;       // total mass, cell side (Nodes[].len)
    float maxsoft;         // max kernel radius of the members (Nodes[].maxsoft)
    float gx, gy, gz;      // geometric cell centre minus centre of mass
    int a, b;
    int level, parent;
};

struct GGDomainDev {
    double center[3];
    double corner[3];
    double len;
    double pad;
};

// walk group: `count` consecutive targets starting at `first` in the target list
struct GGGroup {
    int first, count, root, sys;
};

#define GG_CUDA_TRY(x)                                   \
    do {                                                 \
        cudaError_t e_ = (x);                            \
        if (e_ != cudaSuccess) return gg_cuda_fail(e_);  \
    } while (0)

gg_status gg_cuda_fail(cudaError_t e);

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ unsigned long long gg_dbl_to_ordered(double d)
{
    unsigned long long u = (unsigned long long)__double_as_longlong(d);
    return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double gg_ordered_to_dbl(unsigned long long u)
{
    u = (u & 0x8000000000000000ull) ? (u & 0x7FFFFFFFFFFFFFFFull) : ~u;
    return __longlong_as_double((long long)u);
}

// domain_double_to_int (domain.c:2504-2513) at `bits` bits: top mantissa bits
// of ((x - corner)/len + 1), with the division and addition rounded exactly
// as the reference's FP64 expression.
__device__ __forceinline__ unsigned gg_quantize(double x, double corner, double len)
{
    double d = __dadd_rn(__ddiv_rn(__dsub_rn(x, corner), len), 1.0);
    unsigned long long u = (unsigned long long)__double_as_longlong(d);
    return (unsigned)((u & 0xFFFFFFFFFFFFFull) >> (52 - GG_MAX_LEVEL));
}

// host-side launch helpers (defined in gg_api.cu)
int gg_num_sms();
void gg_note_launches(int k);   // count kernels launched by this library
