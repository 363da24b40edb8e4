// Shared definitions of libpppm_b200: status handling, small vector helpers, constants.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include "pppm_b200.h"

namespace pb
{

// TDBEM history length (taps) and ring size: STEP_NUM = 16 with a 32-slot ring
// (reference CMakeLists.txt:30, bem.h:55).
constexpr int kTaps = 16;
constexpr int kRing = 32;
// The step's own history copies keep the 16 times the taps reach (kHist slots), Neumann and
// Dirichlet interleaved by 4-tap chunks in one row of kHistRow values per triangle (step.cu).
constexpr int kHist = 16;
constexpr int kHistRow = 2 * kHist;
// Reference capacities that define parity-mode limits (particle_grid.h:9-11,
// pppm_cache.h:79); the B200 lists are CSR and only the face cache keeps a per-face bound.
constexpr int kFaceCacheSlots = 1024;

void set_error(const char *fmt, ...);
const char *last_error();

struct Status
{
    int code = PPPM_OK;
    Status() = default;
    Status(int c) : code(c) {}
    explicit operator bool() const { return code != PPPM_OK; }
};

#define PB_CUDA(call)                                                                                          \
    do                                                                                                         \
    {                                                                                                          \
        cudaError_t pb_err_ = (call);                                                                          \
        if (pb_err_ != cudaSuccess)                                                                            \
        {                                                                                                      \
            ::pb::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(pb_err_), __FILE__, __LINE__); \
            return pb_err_ == cudaErrorMemoryAllocation ? PPPM_ERR_NOMEM : PPPM_ERR_CUDA;                      \
        }                                                                                                      \
    } while (0)

#define PB_CHECK_LAUNCH()                                                                                    \
    do                                                                                                       \
    {                                                                                                        \
        cudaError_t pb_err_ = cudaGetLastError();                                                            \
        if (pb_err_ != cudaSuccess)                                                                          \
        {                                                                                                    \
            ::pb::set_error("kernel launch failed: %s (%s:%d)", cudaGetErrorString(pb_err_), __FILE__, __LINE__); \
            return PPPM_ERR_CUDA;                                                                            \
        }                                                                                                    \
    } while (0)

#define PB_TRY(expr)              \
    do                            \
    {                             \
        int pb_rc_ = (expr);      \
        if (pb_rc_ != PPPM_OK)    \
            return pb_rc_;        \
    } while (0)

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

struct f3
{
    float x, y, z;
};

__host__ __device__ inline f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__host__ __device__ inline f3 operator+(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline f3 operator-(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline f3 operator*(float s, f3 a) { return f3{s * a.x, s * a.y, s * a.z}; }
__host__ __device__ inline f3 operator*(f3 a, float s) { return f3{a.x * s, a.y * s, a.z * s}; }
__host__ __device__ inline f3 operator/(f3 a, float s) { return f3{a.x / s, a.y / s, a.z / s}; }
__host__ __device__ inline float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline f3 cross3(f3 a, f3 b)
{
    return f3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ inline float len3(f3 a) { return sqrtf(dot3(a, a)); }
__device__ inline f3 normalize3(f3 a) { return a * rsqrtf(dot3(a, a)); }

__device__ inline f3 load3(const float *p, int i) { return f3{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ inline void store3(float *p, int i, f3 v)
{
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}

// Centre of cell (i, j, k) in world coordinates: ((i + 0.5) * h, ...) + min_pos
// (particle_grid.h:172-175).
__device__ inline f3 cell_center(int i, int j, int k, float h, f3 mn)
{
    return f3{(i + 0.5f) * h, (j + 0.5f) * h, (k + 0.5f) * h} + mn;
}

}  // namespace pb
