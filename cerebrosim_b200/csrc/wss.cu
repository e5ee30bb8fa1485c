// Wall shear stress from a velocity field: the per-vertex weighted fit of wss.shear (wss.py:50-57) on the GPU.
//
// For vertex v with inward unit normal n_v and its K fit coefficients c_vj over lumen cells idx_vj (from the
// host-side fit, wss.weights), tau_v = scale * sum_j c_vj (u_j - (u_j . n_v) n_v): the tangential velocity of the
// nearby cells, weighted so that the sum is the slope a of u_t(d) = a d + b d^2 at the wall. scale = mu * 1e3
// turns (m/s)/mm into Pa. One thread per vertex; FP64 accumulation as the reference's NumPy sum.
#include "cs_common.cuh"

namespace cs {
namespace {

__global__ void k_wss_shear(const float* __restrict__ U, const int32_t* __restrict__ idx, const float* __restrict__ c,
                            const float* __restrict__ nrm, int64_t n_vert, int K, int64_t n_cells, double scale,
                            float* __restrict__ tau) {
    const int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (v >= n_vert) return;
    const double nx = nrm[3 * v], ny = nrm[3 * v + 1], nz = nrm[3 * v + 2];
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int j = 0; j < K; ++j) {
        const int64_t k = v * K + j;
        const double w = double(__ldg(c + k));
        const int32_t cell = __ldg(idx + k);
        if (w == 0.0 || cell < 0 || cell >= n_cells) continue;
        const double ux = __ldg(U + 3 * int64_t(cell)), uy = __ldg(U + 3 * int64_t(cell) + 1),
                     uz = __ldg(U + 3 * int64_t(cell) + 2);
        const double un = ux * nx + uy * ny + uz * nz;
        sx += w * (ux - un * nx);
        sy += w * (uy - un * ny);
        sz += w * (uz - un * nz);
    }
    tau[3 * v] = float(scale * sx);
    tau[3 * v + 1] = float(scale * sy);
    tau[3 * v + 2] = float(scale * sz);
}

}  // namespace
}  // namespace cs

using namespace cs;

extern "C" int cs_wss_shear(const float* U, int64_t n_cells, const int32_t* idx, const float* c, const float* normals,
                            int64_t n_vert, int32_t K, double scale, float* tau, void* stream) {
    if (n_vert < 0 || n_cells < 0 || K < 1 || K > 1024)
        return fail(CS_ERR_ARG, "cs_wss_shear: %lld vertices, %lld cells, K %d", (long long)n_vert,
                    (long long)n_cells, K);
    if (n_vert == 0) return CS_OK;
    if (!U || !idx || !c || !normals || !tau) return fail(CS_ERR_ARG, "cs_wss_shear: null buffer");
    k_wss_shear<<<unsigned(ceil_div(n_vert, 256)), 256, 0, as_stream(stream)>>>(U, idx, c, normals, n_vert, K, n_cells,
                                                                            scale, tau);
    CS_CHECK_LAUNCH("k_wss_shear");
    return CS_OK;
}
