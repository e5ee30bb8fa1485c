// Heartbeat-loop measurements on the device: pressure probes (simulate.k_gather, simulate.py:85-90) and the
// coarse-map snapshots of the stored fields (simulate.coarse_map + the frame averaging, simulate.py:236-242,
// 346-353).
//
// Both are segmented reductions over static cell lists sorted by segment (a probe's cells, a coarse bin's cells),
// summed in FP64 in a fixed order, so a sample does not depend on thread timing (the reference adds with float
// atomics in arbitrary order).
#include "cs_common.cuh"

namespace cs {
namespace {

constexpr int G_THREADS = 256;

// One block per probe: mean density / 3 over its cells (FP64 sum by a fixed tree) and the largest speed there.
__global__ void k_probe_gather(const float* __restrict__ rho, const float* __restrict__ vel, int64_t n,
                               const int32_t* __restrict__ cells, const int32_t* __restrict__ start,
                               double* __restrict__ psum, float* __restrict__ umax) {
    __shared__ double s_sum[G_THREADS];
    __shared__ float s_max[G_THREADS];
    const int k = blockIdx.x;
    const int32_t c0 = start[k], c1 = start[k + 1];
    double acc = 0.0;
    float mx = 0.0f;
    for (int32_t j = c0 + threadIdx.x; j < c1; j += G_THREADS) {
        const int32_t c = cells[j];
        acc += double(rho[c]) / 3.0;
        const float ux = vel[c], uy = vel[n + c], uz = vel[2 * n + c];
        mx = fmaxf(mx, sqrtf(ux * ux + uy * uy + uz * uz));
    }
    s_sum[threadIdx.x] = acc;
    s_max[threadIdx.x] = mx;
    __syncthreads();
    for (int h = G_THREADS / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            s_sum[threadIdx.x] += s_sum[threadIdx.x + h];
            s_max[threadIdx.x] = fmaxf(s_max[threadIdx.x], s_max[threadIdx.x + h]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        psum[k] = s_sum[0];
        umax[k] = s_max[0];
    }
}

// One thread per coarse bin: the mean of p = rho / 3 and of u over its cells (FP64 sums).
__global__ void k_bin_fields(const float* __restrict__ rho, const float* __restrict__ vel, int64_t n,
                             const int32_t* __restrict__ cells, const int32_t* __restrict__ start, int64_t n_bins,
                             float* __restrict__ p_out, float* __restrict__ u_out) {
    const int64_t b = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (b >= n_bins) return;
    const int32_t c0 = start[b], c1 = start[b + 1];
    double sp = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
    for (int32_t j = c0; j < c1; ++j) {
        const int32_t c = cells[j];
        sp += double(rho[c]) / 3.0;
        sx += vel[c];
        sy += vel[n + c];
        sz += vel[2 * n + c];
    }
    const double inv = c1 > c0 ? 1.0 / double(c1 - c0) : 0.0;
    p_out[b] = float(sp * inv);
    u_out[3 * b] = float(sx * inv);
    u_out[3 * b + 1] = float(sy * inv);
    u_out[3 * b + 2] = float(sz * inv);
}

}  // namespace
}  // namespace cs

using namespace cs;

extern "C" int cs_probe_gather(const float* rho, const float* vel, int64_t n, const int32_t* cells,
                               const int32_t* start, int32_t n_probes, double* psum, float* umax, void* stream) {
    if (n < 0 || n_probes < 0) return fail(CS_ERR_ARG, "cs_probe_gather: n %lld probes %d", (long long)n, n_probes);
    if (n_probes == 0) return CS_OK;
    if (!rho || !vel || !cells || !start || !psum || !umax) return fail(CS_ERR_ARG, "cs_probe_gather: null buffer");
    k_probe_gather<<<unsigned(n_probes), G_THREADS, 0, as_stream(stream)>>>(rho, vel, n, cells, start, psum, umax);
    CS_CHECK_LAUNCH("k_probe_gather");
    return CS_OK;
}

extern "C" int cs_bin_fields(const float* rho, const float* vel, int64_t n, const int32_t* cells, const int32_t* start,
                             int64_t n_bins, float* p_out, float* u_out, void* stream) {
    if (n < 0 || n_bins < 0) return fail(CS_ERR_ARG, "cs_bin_fields: n %lld bins %lld", (long long)n, (long long)n_bins);
    if (n_bins == 0) return CS_OK;
    if (!rho || !vel || !cells || !start || !p_out || !u_out) return fail(CS_ERR_ARG, "cs_bin_fields: null buffer");
    k_bin_fields<<<unsigned(ceil_div(n_bins, 256)), 256, 0, as_stream(stream)>>>(rho, vel, n, cells, start, n_bins,
                                                                             p_out, u_out);
    CS_CHECK_LAUNCH("k_bin_fields");
    return CS_OK;
}
