// Shared definitions of the B200 lattice-Boltzmann library: D3Q27 constants, link encoding, error reporting.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>

#include "cerebrosim.h"

namespace cs {

constexpr int Q = 27;

// D3Q27 velocities in the reference's order (lbm.py:34-40): rest; +x -x +y -y +z -z (links 1..6 feed the
// finite-difference gradient, lbm.py:48); 12 edges and 8 corners, each followed by its opposite.
constexpr int CX[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
constexpr int CY[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
constexpr int CZ[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
constexpr int OPP[Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 20, 19, 22, 21, 24, 23, 26, 25};

// The same tables for device code: constexpr functions fold to immediates once a link loop is unrolled.
struct Lat {
    static __host__ __device__ constexpr int cx(int i) {
        constexpr int v[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
        return v[i];
    }
    static __host__ __device__ constexpr int cy(int i) {
        constexpr int v[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
        return v[i];
    }
    static __host__ __device__ constexpr int cz(int i) {
        constexpr int v[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
        return v[i];
    }
    static __host__ __device__ constexpr int opp(int i) { return i == 0 ? 0 : (i % 2 ? i + 1 : i - 1); }
};

// Lattice weights (lbm.py:40) in float32, as the reference's kernels use them.
__host__ __device__ constexpr float wgt(int i) {
    return i == 0 ? 8.0f / 27.0f : (i < 7 ? 2.0f / 27.0f : (i < 19 ? 1.0f / 54.0f : 1.0f / 216.0f));
}

// Encoded step links (cs_links_encode): >= 0 pull source; -2 inlet; -3 - k outlet k; a wall link is
// 0x80000000 | float bits of its q (q in [0, 2): bits < 0x40000000), i.e. every value below -2^30.
constexpr int32_t WALL_TAG_LIMIT = -(1 << 30);
__host__ __device__ inline bool is_wall(int32_t code) { return code < WALL_TAG_LIMIT; }
__device__ inline float wall_q(int32_t code) { return __int_as_float(code & 0x7fffffff); }

// ---- error reporting (per host thread) ------------------------------------------------------------------------
void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);
const char* last_error();

#define CS_CUDA(call)                                                                                          \
    do {                                                                                                       \
        cudaError_t e_ = (call);                                                                               \
        if (e_ != cudaSuccess) return ::cs::fail(CS_ERR_CUDA, "%s failed: %s (%s:%d)", #call,                  \
                                                 cudaGetErrorString(e_), __FILE__, __LINE__);                 \
    } while (0)

#define CS_CHECK_LAUNCH(what)                                                                                  \
    do {                                                                                                       \
        cudaError_t e_ = cudaGetLastError();                                                                   \
        if (e_ != cudaSuccess) return ::cs::fail(CS_ERR_CUDA, "launch of %s failed: %s", what,                 \
                                                 cudaGetErrorString(e_));                                     \
    } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace cs
