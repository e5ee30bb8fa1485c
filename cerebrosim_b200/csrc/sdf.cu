// Signed distance of a branched vessel on a voxel grid: the field of vessel.k_sdf (vessel.py:178-207), evaluated on
// the GPU in float32 in the same order of operations, so that build_lattice sees the reference's field.
//
// Per voxel p = origin + (i, j, k) dx: for each branch, the minimum over its segments of the round-cone distance
// |p - (a + t ab)| - r(t) (t = the clamped projection of p on the segment, r interpolated linearly), cut by the flat
// caps near its open ends (a half-space max within 2.5 cap radii); branches are joined by the polynomial smooth
// minimum with blend radius `blend`. Negative inside the lumen. One thread per voxel, C order (k fastest).
#include "cs_common.cuh"

namespace cs {
namespace {

struct SdfArgs {
    float origin[3];
    float dx;
    const float* pts;        // (n_pts, 3) centreline points, branches back to back
    const float* rad;        // (n_pts,) radius at each point
    const int32_t* br_start; // (nbranch,) first point of each branch
    const int32_t* br_count; // (nbranch,) points of each branch
    const float* cap_p;      // (2 nbranch, 3) cap centres (start, end of each branch)
    const float* cap_n;      // (2 nbranch, 3) outward cap normals
    const float* cap_r;      // (2 nbranch,) cap radius, 0 = no cap
    float blend;
    int nbranch;
    int64_t nx, ny, nz;
    float* out;
};

__device__ __forceinline__ float smin(float a, float b, float k) {
    // vessel.py:178-181
    const float h = fminf(fmaxf(0.5f + 0.5f * (b - a) / k, 0.0f), 1.0f);
    return b + (a - b) * h - k * h * (1.0f - h);
}

__global__ void k_sdf(const SdfArgs s) {
    const int64_t total = s.nx * s.ny * s.nz;
    for (int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; c < total; c += int64_t(gridDim.x) * blockDim.x) {
        const int64_t l = c % s.nz, j = (c / s.nz) % s.ny, i = c / (s.ny * s.nz);
        const float px = s.origin[0] + float(i) * s.dx;
        const float py = s.origin[1] + float(j) * s.dx;
        const float pz = s.origin[2] + float(l) * s.dx;
        float d = 1.0e9f;
        for (int b = 0; b < s.nbranch; ++b) {
            float db = 1.0e9f;
            const int s0 = __ldg(s.br_start + b), cnt = __ldg(s.br_count + b);
            for (int k = s0; k < s0 + cnt - 1; ++k) {
                const float ax = __ldg(s.pts + 3 * k), ay = __ldg(s.pts + 3 * k + 1), az = __ldg(s.pts + 3 * k + 2);
                const float bx = __ldg(s.pts + 3 * k + 3) - ax, by = __ldg(s.pts + 3 * k + 4) - ay,
                            bz = __ldg(s.pts + 3 * k + 5) - az;
                const float qx = px - ax, qy = py - ay, qz = pz - az;
                const float t = fminf(fmaxf((qx * bx + qy * by + qz * bz) / fmaxf(bx * bx + by * by + bz * bz, 1.0e-12f),
                                            0.0f), 1.0f);
                const float r0 = __ldg(s.rad + k);
                const float r = r0 + (__ldg(s.rad + k + 1) - r0) * t;
                const float ex = px - (ax + bx * t), ey = py - (ay + by * t), ez = pz - (az + bz * t);
                db = fminf(db, sqrtf(ex * ex + ey * ey + ez * ez) - r);
            }
            for (int e = 0; e < 2; ++e) {
                const int cc = b * 2 + e;
                const float cr = __ldg(s.cap_r + cc);
                if (cr > 0.0f) {
                    const float qx = px - __ldg(s.cap_p + 3 * cc), qy = py - __ldg(s.cap_p + 3 * cc + 1),
                                qz = pz - __ldg(s.cap_p + 3 * cc + 2);
                    if (sqrtf(qx * qx + qy * qy + qz * qz) < 2.5f * cr)
                        db = fmaxf(db, qx * __ldg(s.cap_n + 3 * cc) + qy * __ldg(s.cap_n + 3 * cc + 1) +
                                           qz * __ldg(s.cap_n + 3 * cc + 2));
                }
            }
            d = smin(d, db, s.blend);
        }
        s.out[c] = d;
    }
}

}  // namespace
}  // namespace cs

using namespace cs;

extern "C" int cs_sdf_vessel(const float* pts, const float* rad, const int32_t* br_start, const int32_t* br_count,
                             int32_t nbranch, const float* cap_p, const float* cap_n, const float* cap_r, float blend,
                             const float* origin, float dx, int64_t nx, int64_t ny, int64_t nz, float* out,
                             void* stream) {
    if (nx < 0 || ny < 0 || nz < 0 || nbranch < 0 || !origin || !(dx > 0.0f) || !(blend > 0.0f))
        return fail(CS_ERR_ARG, "cs_sdf_vessel: grid %lld x %lld x %lld, %d branches, dx %g, blend %g", (long long)nx,
                    (long long)ny, (long long)nz, nbranch, double(dx), double(blend));
    const int64_t total = nx * ny * nz;
    if (total == 0) return CS_OK;
    if (!out || (nbranch > 0 && (!pts || !rad || !br_start || !br_count || !cap_p || !cap_n || !cap_r)))
        return fail(CS_ERR_ARG, "cs_sdf_vessel: null buffer");
    SdfArgs a{{origin[0], origin[1], origin[2]}, dx, pts, rad, br_start, br_count, cap_p, cap_n, cap_r, blend,
              nbranch, nx, ny, nz, out};
    const unsigned grid = unsigned(std::min<int64_t>(ceil_div(total, 256), 148 * 64));
    k_sdf<<<grid, 256, 0, as_stream(stream)>>>(a);
    CS_CHECK_LAUNCH("k_sdf");
    return CS_OK;
}
