// common.cuh -- shared device helpers and host plumbing of libdgc (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include <atomic>
#include <cfloat>
#include <cstring>
#include <algorithm>
#include <string>

#include "dgc.h"
#include "trace.cuh"

namespace dgc {

// ---------------------------------------------------------------------------
// Host-side status plumbing
// ---------------------------------------------------------------------------

void set_error(const std::string& msg);
void clear_error();

struct Fail {
    int code;
};

#define DGC_REQUIRE(cond, msg)                                          \
    do {                                                                \
        if (!(cond)) {                                                  \
            ::dgc::set_error(std::string(msg));                         \
            return DGC_ERR_INVALID_ARGUMENT;                            \
        }                                                               \
    } while (0)

#define DGC_CUDA(call)                                                          \
    do {                                                                        \
        cudaError_t e__ = (call);                                               \
        if (e__ != cudaSuccess) {                                               \
            ::dgc::set_error(std::string(#call) + ": " + cudaGetErrorString(e__)); \
            return DGC_ERR_CUDA;                                                \
        }                                                                       \
    } while (0)

#define DGC_LAUNCH_CHECK(what)                                                   \
    do {                                                                        \
        cudaError_t e__ = cudaGetLastError();                                   \
        if (e__ != cudaSuccess) {                                               \
            ::dgc::set_error(std::string(what) + " launch failed: " +            \
                             cudaGetErrorString(e__));                          \
            return DGC_ERR_CUDA;                                                \
        }                                                                       \
    } while (0)

// Runs set() (returning a DGC status) once per device: kernel attributes such
// as the dynamic shared-memory limit belong to a device's context, so a
// process that drives several GPUs must set them on each.
template <typename F>
int once_per_device(std::atomic<unsigned long long>& done, F set) {
    int dev = 0;
    DGC_CUDA(cudaGetDevice(&dev));
    const unsigned long long bit = dev < 64 ? (1ull << dev) : 0ull;
    if (bit && (done.load() & bit)) return DGC_OK;
    const int rc = set();
    if (rc == DGC_OK && bit) done.fetch_or(bit);
    return rc;
}

// Bump allocator over a caller-owned workspace (256-byte aligned slices).
struct Workspace {
    char* base;
    size_t size;
    size_t used;
    Workspace(void* p, size_t n) : base(static_cast<char*>(p)), size(n), used(0) {}
    static size_t align(size_t n) { return (n + 255) & ~size_t(255); }
    template <typename T>
    T* take(size_t count) {
        size_t bytes = align(count * sizeof(T));
        if (base == nullptr || used + bytes > size) return nullptr;
        T* p = reinterpret_cast<T*>(base + used);
        used += bytes;
        return p;
    }
};

inline int ceil_div(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }

// Power-of-two test of a positive finite float: for such a value x/v and
// x*(1/v) are bitwise identical, so the reference's divisions by
// voxel_size / pixel_size may be executed as multiplications.
inline bool is_pow2_float(float v) {
    if (!(v > 0.0f)) return false;
    uint32_t bits;
    memcpy(&bits, &v, sizeof(bits));
    uint32_t exp = (bits >> 23) & 0xffu;
    return (bits & 0x7fffffu) == 0 && exp > 0 && exp < 254;
}

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------

// floor() of |x| < 2^22 with full-rate FP32 adds: adding 1.5*2^23 with
// round-toward-minus-infinity leaves floor(x) in the low mantissa bits.
constexpr float kFloorMagic = 12582912.0f;        // 1.5 * 2^23
constexpr uint32_t kFloorMagicBits = 0x4B400000u;  // bit pattern of kFloorMagic

struct FloorSplit {
    uint32_t biased;  // kFloorMagicBits + floor(x) (modular arithmetic)
    float frac;       // x - floor(x), exact
};

__device__ __forceinline__ FloorSplit floor_split(float x) {
    const float f = __fadd_rd(x, kFloorMagic);
    FloorSplit r;
    r.biased = __float_as_uint(f);
    r.frac = __fsub_rn(x, __fsub_rn(f, kFloorMagic));
    return r;
}

__device__ __forceinline__ float lerpf(float a, float b, float w) {
    return fmaf(w, b - a, a);
}

// Packed FP32 pairs (sm_100 f32x2 arithmetic): each lane is an IEEE FP32 op with
// the same rounding as the scalar instruction.
typedef unsigned long long f32x2;

__device__ __forceinline__ f32x2 pack2(float lo, float hi) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}

__device__ __forceinline__ float2 unpack2(f32x2 v) {
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
    return r;
}

__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}

__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

// Per-lane a + b rounded toward minus infinity (the packed __fadd_rd).
__device__ __forceinline__ f32x2 add2_rd(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("add.rm.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

__device__ __forceinline__ uint2 unpack2_bits(f32x2 v) {
    uint2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=r"(r.x), "=r"(r.y) : "l"(v));
    return r;
}

// Per-lane lerp of two packed pairs with one weight: a + w*(b-a).
__device__ __forceinline__ f32x2 lerp2(f32x2 a, f32x2 b, f32x2 w) { return fma2(w, sub2(b, a), a); }

// Float add to global memory whose result is not used (red.global.add.f32,
// round-to-nearest like atomicAdd).  The asm has no memory clobber, so the
// compiler need not assume that the add changed other memory: values staged
// in shared memory (view geometry, batched instance arguments) stay in
// registers across a scatter loop instead of being re-read after every add.
// p must point to global memory.
__device__ __forceinline__ void red_add_global(float* p, float v) {
    asm volatile("red.global.add.f32 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "f"(v));
}

// Four float adds to 16-byte-aligned global memory as one vector reduction
// (red.global.add.v4.f32; each element is added atomically), without a
// memory clobber like red_add_global.
__device__ __forceinline__ void red_add4_global(float* p, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(__cvta_generic_to_global(p)),
                 "f"(a), "f"(b), "f"(c), "f"(d));
}

// red_add4_global under a predicate inside the asm (a predicated
// instruction, not a branch around it).
__device__ __forceinline__ void red_add4_global_if(bool on, float* p, float a, float b, float c,
                                                   float d) {
    asm volatile(
        "{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %5, 0;\n\t"
        "@q red.global.add.v4.f32 [%0], {%1, %2, %3, %4};\n\t}"
        ::"l"(__cvta_generic_to_global(p)), "f"(a), "f"(b), "f"(c), "f"(d), "r"((int)on));
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Per-view geometry pointers, in the reference's argument order.
struct Geometry {
    const float* angles;
    const float* sid;
    const float* sod;
    const float* det_u0;
    const float* det_v0;
    const float* src_x;
    const float* src_y;
    const float* src_z;
};

// The eight per-view geometry-gradient outputs.
struct GeometryGrad {
    float* g[8];
};

}  // namespace dgc
