// Sparse D3Q27 step on the GPU: lbm.k_clock + lbm.k_step (lbm.py:90-257) and, for the artery solver,
// simulate.k_flux + simulate.k_bc (simulate.py:65-82).
//
// One step = two or three kernels on one stream:
//  1. k_boundary — the wall / inlet / outlet link list (lbm.py:163-181) and the clock (lbm.py:94-102). One thread
//     per ghost slot (a boundary link of one direction); it evaluates what the reference's pull produces for that
//     link — Bouzidi interpolation (q < 0.5 with the second node, q >= 0.5 with the node's own population),
//     half-way bounce-back, the velocity inlet with the drive, the pressure outlet with p_out and the previous
//     velocity — and stores it in the ghost slot f_in[i * npad + n + g] of the step's input buffer. Its first
//     thread evaluates drive(tick[a]) into *drive and advances tick[1 - a] = tick[a] + 1; nothing else in the step
//     reads tick[1 - a], and the bulk kernel reads the drive from memory instead of recomputing it.
//  2. k_bulk (k_bulk_dense: the regularised step without body force in blocks of <= 128 threads, 9 per SM) — one
//     thread per fluid node, C-ordered nodes, link-major populations (the reference's SoA layout).
//     Every link is a plain pull f_in[i * npad + links[i * n + node]] (a fluid source or a ghost slot), so the 27
//     loads carry no branch and issue back to back; for each link the warp's 32 sources are mostly consecutive,
//     so each load and store moves whole 128-byte lines. Links come in pairs (i, opp(i)) with c_opp = -c_i: the
//     pull accumulates dr, j and Pi = sum c c^T f from each pair's sum and difference, and the collision output is
//     w_i (A + E_i +- O_i) with E even and O odd in c, so each pair's terms are evaluated once. By the D3Q27
//     isotropy sum_i w_i c c^T feq2_i = dr/3 I + u u^T, the regularised projection P = sum c c^T (f - feq2)
//     (lbm.py:219-223) is Pi - dr/3 I - u u^T; no population is kept in registers. Galilean correction
//     (lbm.py:192-204) from the six axis neighbours' previous velocity (a ghost slot gives the wall's q or marks an
//     opening); cells with an inlet link (om < 0) get the inlet equilibrium (lbm.py:205-216); TRT (lbm.py:241-255)
//     keeps the populations.
//  3. k_bc (only with the resistance coupling) — one block: p_out[0] = drive, p_out[k] relaxed towards R_k Q_k -
//     pref in FP64, Qlast = Q, Q = 0 (simulate.py:76-82). The slab flux Q_k = sum u . w itself is reduced in the
//     bulk kernel in FP64 by the blocks that hold flux cells (simulate.py:65-69).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "cs_common.cuh"

#include <vector>

namespace cs {
namespace {

constexpr int MAX_BLOCK = 256;
constexpr int MIN_BLOCKS = 4;   // 4 x 256 threads per SM (64 registers): occupancy hides the pulls' latency
constexpr int MAX_OPEN = 8;
constexpr int B_THREADS = 256;
constexpr float PI_F = 3.14159265358979323846f;

__constant__ int k_cx[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
__constant__ int k_cy[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
__constant__ int k_cz[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};

// ---- population storage -----------------------------------------------------------------------------------------
// 32-bit element offsets: 27 * npad < 2^31 is checked on the host.
template <int ST> struct Pop;

template <> struct Pop<CS_STORE_F32> {
    static __device__ __forceinline__ float ld(const void* b, uint32_t idx, float) {
        return __ldg(static_cast<const float*>(b) + idx);
    }
    static __device__ __forceinline__ void st(void* b, uint32_t idx, float, float v) { static_cast<float*>(b)[idx] = v; }
};

// 16-bit formats store (f - w_i) * 1024 / w_i: all links share one range, well inside FP16's normal numbers, so the
// relative rounding error is the format's 2^-11 (FP16) or 2^-8 (BF16) on every link. w is the link's weight.
template <> struct Pop<CS_STORE_F16> {
    static __device__ __forceinline__ float ld(const void* b, uint32_t idx, float w) {
        return __half2float(__ldg(static_cast<const __half*>(b) + idx)) * (w * (1.0f / 1024.0f));
    }
    static __device__ __forceinline__ void st(void* b, uint32_t idx, float w, float v) {
        static_cast<__half*>(b)[idx] = __float2half_rn(v * (1024.0f / w));
    }
    // a value already in the stored scale, (f - w) 1024 / w
    static __device__ __forceinline__ void st_scaled(void* b, uint32_t idx, float g) {
        static_cast<__half*>(b)[idx] = __float2half_rn(g);
    }
};

template <> struct Pop<CS_STORE_BF16> {
    static __device__ __forceinline__ float ld(const void* b, uint32_t idx, float w) {
        return __bfloat162float(__ldg(static_cast<const __nv_bfloat16*>(b) + idx)) * (w * (1.0f / 1024.0f));
    }
    static __device__ __forceinline__ void st(void* b, uint32_t idx, float w, float v) {
        static_cast<__nv_bfloat16*>(b)[idx] = __float2bfloat16_rn(v * (1024.0f / w));
    }
    static __device__ __forceinline__ void st_scaled(void* b, uint32_t idx, float g) {
        static_cast<__nv_bfloat16*>(b)[idx] = __float2bfloat16_rn(g);
    }
};

// ---- helpers ------------------------------------------------------------------------------------------------------
__device__ __forceinline__ float drive_value(const cs_step_desc& d, int t) {
    // lbm.py:95-100, float32
    float ph = 2.0f * PI_F * float(t % d.period) / float(d.period);
    float v = d.coef[0];
    for (int k = 1; k <= d.nh; ++k)
        v += d.coef[2 * k - 1] * cosf(float(k) * ph) + d.coef[2 * k] * sinf(float(k) * ph);
    if (t < d.ramp) v *= 0.5f - 0.5f * cosf(PI_F * float(t) / float(d.ramp));
    return v;
}

// Programmatic dependent launch (sm_90+): a kernel launched with the programmatic-serialization attribute may start
// while the previous kernel of the stream is still running; it reads only static tables until
// grid_dependency_wait(), which returns once that kernel has completed and its writes are visible. A kernel calls
// launch_dependents() once the next kernel may be scheduled beside it. Both are no-ops for an ordinary launch.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" :::); }

__device__ __forceinline__ float weight_rt(int i) {
    return i == 0 ? 8.0f / 27.0f : (i < 7 ? 2.0f / 27.0f : (i < 19 ? 1.0f / 54.0f : 1.0f / 216.0f));
}

// Non-uniform central difference (lbm.py:105-126) of one velocity component: gm / gp are the values loaded through
// the links that pull from x - e_a (sm) and x + e_a (sp) — the neighbour's previous velocity component for a fluid
// source, the ghost slot's gq for a boundary link (q >= 0: wall at distance max(q, 0.1) with u = 0; -1: an opening,
// u = u0 at distance 1). Two fluid neighbours (the common case) give the central difference (v2 - v1) / 2.
__device__ __forceinline__ float ddx_g(int32_t sm, int32_t sp, float gm, float gp, float u0, int32_t n_nodes) {
    if (sm < n_nodes && sp < n_nodes) return 0.5f * (gp - gm);
    float h1 = 1.0f, v1 = u0, h2 = 1.0f, v2 = u0;
    if (sm < n_nodes) {
        v1 = gm;
    } else if (gm >= 0.0f) {
        h1 = fmaxf(gm, 0.1f);
        v1 = 0.0f;
    }
    if (sp < n_nodes) {
        v2 = gp;
    } else if (gp >= 0.0f) {
        h2 = fmaxf(gp, 0.1f);
        v2 = 0.0f;
    }
    return (h1 * h1 * (v2 - u0) + h2 * h2 * (u0 - v1)) / (h1 * h2 * (h1 + h2));
}

// Address of what the difference along link k (1..6) reads for velocity component c: the neighbour's component, or
// the ghost slot's q.
__device__ __forceinline__ const float* grad_src(const cs_step_desc& d, const float* vin, int k, int c, int32_t s) {
    return s < d.n ? vin + int64_t(c) * d.n + s : d.gq + int64_t(k) * d.gmax + (s - d.n);
}

// Third-order equilibrium term of link I (lbm.py:129-137) from the velocity monomials; odd in c.
struct Cubic {
    float xxy, xxz, xyy, yyz, xzz, yzz, xyz;
    __device__ __forceinline__ explicit Cubic(float x, float y, float z)
        : xxy(x * x * y), xxz(x * x * z), xyy(x * y * y), yyz(y * y * z), xzz(x * z * z), yzz(y * z * z),
          xyz(x * y * z) {}
    template <int I>
    __device__ __forceinline__ float h3() const {
        constexpr float t = 1.0f / 3.0f;
        constexpr int x = Lat::cx(I), y = Lat::cy(I), z = Lat::cz(I);
        constexpr float ax = float(x * x) - t, ay = float(y * y) - t, az = float(z * z) - t;
        float s = 0.0f;
        if (y) s += ax * float(y) * xxy;
        if (z) s += ax * float(z) * xxz;
        if (x) s += ay * float(x) * xyy;
        if (z) s += ay * float(z) * yyz;
        if (x) s += az * float(x) * xzz;
        if (y) s += az * float(y) * yzz;
        if (x && y && z) s += float(2 * x * y * z) * xyz;   // 27 x y z u_x u_y u_z = 13.5 * (2 x y z) u_x u_y u_z
        return 13.5f * s;
    }
};

template <int I, int N_>
struct Unroll {
    template <class F>
    static __device__ __forceinline__ void run(F&& f) {
        f(std::integral_constant<int, I>{});
        Unroll<I + 1, N_>::run(f);
    }
};
template <int N_>
struct Unroll<N_, N_> {
    template <class F>
    static __device__ __forceinline__ void run(F&&) {}
};

// Moment sums from pulled values; a pair (I, opp(I)) enters through its sum s and difference dd.
struct Moments {
    float dr = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
    float pxx = 0.f, pyy = 0.f, pzz = 0.f, pxy = 0.f, pxz = 0.f, pyz = 0.f;
    template <int I>
    __device__ __forceinline__ void add_pair(float v, float vo) {
        constexpr int x = Lat::cx(I), y = Lat::cy(I), z = Lat::cz(I);
        const float s = v + vo, dd = v - vo;
        dr += s;
        if (x) jx += x * dd;
        if (y) jy += y * dd;
        if (z) jz += z * dd;
        if (x) pxx += s;
        if (y) pyy += s;
        if (z) pzz += s;
        if (x && y) pxy += (x * y) * s;
        if (x && z) pxz += (x * z) * s;
        if (y && z) pyz += (y * z) * s;
    }
};

// c^T M c for link I with M given by its diagonal and twice its off-diagonal entries.
template <int I>
__device__ __forceinline__ float quad(float mxx, float myy, float mzz, float mxy2, float mxz2, float myz2) {
    constexpr int x = Lat::cx(I), y = Lat::cy(I), z = Lat::cz(I);
    float s = 0.0f;
    if (x) s += mxx;
    if (y) s += myy;
    if (z) s += mzz;
    if (x && y) s += float(x * y) * mxy2;
    if (x && z) s += float(x * z) * mxz2;
    if (y && z) s += float(y * z) * myz2;
    return s;
}

template <int I>
__device__ __forceinline__ float cdot(float ax, float ay, float az) {
    constexpr int x = Lat::cx(I), y = Lat::cy(I), z = Lat::cz(I);
    float s = 0.0f;
    if (x) s += float(x) * ax;
    if (y) s += float(y) * ay;
    if (z) s += float(z) * az;
    return s;
}

// The links the grouped sums below name by index: axis 1, 3, 5 (+x, +y, +z); edges 7 (1,1,0), 9 (1,-1,0), 11 (1,0,1),
// 13 (1,0,-1), 15 (0,1,1), 17 (0,1,-1); corners 19 (1,1,1), 21 (1,1,-1), 23 (1,-1,1), 25 (-1,1,1); each with its
// opposite at index + 1.
constexpr bool pair_is(int i, int x, int y, int z) {
    return Lat::cx(i) == x && Lat::cy(i) == y && Lat::cz(i) == z && Lat::opp(i) == i + 1;
}
static_assert(pair_is(1, 1, 0, 0) && pair_is(3, 0, 1, 0) && pair_is(5, 0, 0, 1), "axis links");
static_assert(pair_is(7, 1, 1, 0) && pair_is(9, 1, -1, 0) && pair_is(11, 1, 0, 1) && pair_is(13, 1, 0, -1) &&
                  pair_is(15, 0, 1, 1) && pair_is(17, 0, 1, -1), "edge links");
static_assert(pair_is(19, 1, 1, 1) && pair_is(21, 1, 1, -1) && pair_is(23, 1, -1, 1) && pair_is(25, -1, 1, 1),
              "corner links");

// Moments of the 27 pulled values (dr = sum f, j = sum c f, Pi = sum c c^T f): each pair (I, opp I) enters through
// its sum s and difference d, and the terms several moments share are added once — the three edge planes, and the
// four corner pairs through a butterfly (their sums give the trace and the three off-diagonals of Pi, their
// differences the corner parts of j). 81 additions instead of 111 for the link-by-link sums.
__device__ __forceinline__ void moments27(const float (&f)[Q], Moments& m) {
    float sp[Q / 2 + 1], dp[Q / 2 + 1];
#pragma unroll
    for (int k = 0; k < 13; ++k) {
        sp[k] = f[1 + 2 * k] + f[2 + 2 * k];
        dp[k] = f[1 + 2 * k] - f[2 + 2 * k];
    }
    // pair k holds links 1 + 2k and 2 + 2k: k = 0, 1, 2 axis; 3 .. 8 edges; 9 .. 12 corners
    const float exy = sp[3] + sp[4], exz = sp[5] + sp[6], eyz = sp[7] + sp[8];
    const float ca = sp[9] + sp[10], cb = sp[9] - sp[10], cc = sp[11] + sp[12], ce = sp[11] - sp[12];
    const float sc = ca + cc;
    m.dr = f[0] + sp[0] + sp[1] + sp[2] + exy + exz + eyz + sc;
    m.pxx = sp[0] + exy + exz + sc;
    m.pyy = sp[1] + exy + eyz + sc;
    m.pzz = sp[2] + exz + eyz + sc;
    m.pxy = (sp[3] - sp[4]) + (ca - cc);
    m.pxz = (sp[5] - sp[6]) + (cb + ce);
    m.pyz = (sp[7] - sp[8]) + (cb - ce);
    const float dpp = dp[9] + dp[10], dpr = dp[9] - dp[10], dpt = dp[11] + dp[12], dpv = dp[11] - dp[12];
    m.jx = dp[0] + dp[3] + dp[4] + dp[5] + dp[6] + (dpp + dpv);
    m.jy = dp[1] + dp[3] - dp[4] + dp[7] + dp[8] + (dpp - dpv);
    m.jz = dp[2] + dp[5] - dp[6] + dp[7] - dp[8] + (dpr + dpt);
}

// One pair's outputs: FP32 stores w (A + e +- o); the 16-bit formats store (f - w) 1024 / w = 1024 (A + e +- o),
// for which A, e and o arrive already multiplied by 1024 (no per-link weight or scale left to apply).
template <int ST, int I>
__device__ __forceinline__ void store_pair(void* fout, uint32_t NP, int32_t n, float A, float e, float o) {
    constexpr int O = Lat::opp(I);
    if constexpr (ST == CS_STORE_F32) {
        constexpr float w = wgt(I);
        const float wb = w * (A + e);
        Pop<ST>::st(fout, uint32_t(I) * NP + uint32_t(n), w, fmaf(w, o, wb));
        Pop<ST>::st(fout, uint32_t(O) * NP + uint32_t(n), w, fmaf(-w, o, wb));
    } else {
        const float b = A + e;
        Pop<ST>::st_scaled(fout, uint32_t(I) * NP + uint32_t(n), b + o);
        Pop<ST>::st_scaled(fout, uint32_t(O) * NP + uint32_t(n), b - o);
    }
}

// Regularised collision output without a body force (lbm.py:129-137, 230-240): f_I = w_I (A + e_I + o_I) and
// f_opp = w_I (A + e_I - o_I), with e_I = c_I^T M c_I for M = 4.5 u u^T + 4.5 (1 - om) P' (given as its diagonal
// and twice its off-diagonal: m*) and o_I = 3 c_I . u + h3_I (the third-order term, with the Galilean model). Axis,
// edge and corner links differ only in signs, so the 13 pairs' e and o come from shared partial sums.
template <int ST, bool GAL>
__device__ __forceinline__ void store_regularised(void* fout, uint32_t NP, int32_t n, float A, float ux, float uy,
                                                  float uz, float mxx, float myy, float mzz, float mxy2,
                                                  float mxz2, float myz2) {
    // SC: the stored scale (1024 for the 16-bit formats, applied to A, M and the constants; exact in binary)
    constexpr float SC = ST == CS_STORE_F32 ? 1.0f : 1024.0f;
    if constexpr (ST == CS_STORE_F32) {
        Pop<ST>::st(fout, uint32_t(n), wgt(0), wgt(0) * A);
    } else {
        A *= SC;
        mxx *= SC;
        myy *= SC;
        mzz *= SC;
        mxy2 *= SC;
        mxz2 *= SC;
        myz2 *= SC;
        Pop<ST>::st_scaled(fout, uint32_t(n), A);
    }
    // third-order terms from the velocity monomials: axis links -4.5 (sum of two), edges 9 (..) - 4.5 (..),
    // corners 9 (+-A1 +-A2 +-A3) +- 27 xyz
    float h1 = 0.f, h3 = 0.f, h5 = 0.f, h7 = 0.f, h9 = 0.f, h11 = 0.f, h13 = 0.f, h15 = 0.f, h17 = 0.f;
    float h19 = 0.f, h21 = 0.f, h23 = 0.f, h25 = 0.f;
    if (GAL) {
        const float x2 = ux * ux, y2 = uy * uy, z2 = uz * uz;
        const float xxy = x2 * uy, xxz = x2 * uz, xyy = ux * y2, yyz = y2 * uz, xzz = ux * z2, yzz = uy * z2;
        const float xyz = ux * uy * uz;
        const float a1 = xxy + yzz, a2 = xxz + yyz, a3 = xyy + xzz;
        h1 = (-4.5f * SC) * a3;
        h3 = (-4.5f * SC) * a1;
        h5 = (-4.5f * SC) * a2;
        h7 = (9.0f * SC) * (xyy + xxy) - (4.5f * SC) * (xzz + yzz);
        h9 = (9.0f * SC) * (xyy - xxy) - (4.5f * SC) * (xzz - yzz);
        h11 = (9.0f * SC) * (xzz + xxz) - (4.5f * SC) * (xyy + yyz);
        h13 = (9.0f * SC) * (xzz - xxz) - (4.5f * SC) * (xyy - yyz);
        h15 = (9.0f * SC) * (yzz + yyz) - (4.5f * SC) * (xxy + xxz);
        h17 = (9.0f * SC) * (yzz - yyz) - (4.5f * SC) * (xxy - xxz);
        const float b1 = (9.0f * SC) * a1, b2 = (9.0f * SC) * a2, b3 = (9.0f * SC) * a3, bx = (27.0f * SC) * xyz;
        const float p_ = b1 + b3, q_ = b2 + bx, m_ = b3 - b1, n_ = b2 - bx;
        h19 = p_ + q_;
        h21 = p_ - q_;
        h23 = m_ + n_;
        h25 = n_ - m_;
    }
    // axis
    store_pair<ST, 1>(fout, NP, n, A, mxx, (3.0f * SC) * ux + h1);
    store_pair<ST, 3>(fout, NP, n, A, myy, (3.0f * SC) * uy + h3);
    store_pair<ST, 5>(fout, NP, n, A, mzz, (3.0f * SC) * uz + h5);
    // edges, plane by plane
    const float sxy = mxx + myy, sxz = mxx + mzz, syz = myy + mzz;
    const float u7 = ux + uy, u9 = ux - uy;
    store_pair<ST, 7>(fout, NP, n, A, sxy + mxy2, (3.0f * SC) * u7 + h7);
    store_pair<ST, 9>(fout, NP, n, A, sxy - mxy2, (3.0f * SC) * u9 + h9);
    store_pair<ST, 11>(fout, NP, n, A, sxz + mxz2, (3.0f * SC) * (ux + uz) + h11);
    store_pair<ST, 13>(fout, NP, n, A, sxz - mxz2, (3.0f * SC) * (ux - uz) + h13);
    store_pair<ST, 15>(fout, NP, n, A, syz + myz2, (3.0f * SC) * (uy + uz) + h15);
    store_pair<ST, 17>(fout, NP, n, A, syz - myz2, (3.0f * SC) * (uy - uz) + h17);
    // corners
    const float tr = sxy + mzz, ca = tr + mxy2, cb = tr - mxy2, cg = mxz2 + myz2, cd = mxz2 - myz2;
    store_pair<ST, 19>(fout, NP, n, A, ca + cg, (3.0f * SC) * (u7 + uz) + h19);
    store_pair<ST, 21>(fout, NP, n, A, ca - cg, (3.0f * SC) * (u7 - uz) + h21);
    store_pair<ST, 23>(fout, NP, n, A, cb + cd, (3.0f * SC) * (u9 + uz) + h23);
    store_pair<ST, 25>(fout, NP, n, A, cb - cd, (3.0f * SC) * (uz - u9) + h25);
}

// ---- 1. boundary-link kernel and clock ----------------------------------------------------------------------------
// Block (bx, by) of a lattice's boundary-link grid: by = direction, bx = chunk of its ghost slots.
template <int ST>
__device__ __forceinline__ void boundary_body(const cs_step_desc& d, const int a, const int bx, const int by,
                                              const bool clock) {
    // the ghost table is static: read it before waiting for the previous kernel of the stream
    const int i = by;
    const int64_t g = int64_t(bx) * B_THREADS + threadIdx.x;
    const int64_t slot = int64_t(i) * d.gmax + g;
    const bool live = g < d.gmax;
    const int32_t node = live ? __ldg(d.gnode + slot) : -1;
    const int32_t info = live ? __ldg(d.ginfo + slot) : 0;
    const float qslot = live ? __ldg(d.gq + slot) : 0.0f;
    grid_dependency_wait();
    // issue the slot's loads first: the clock below (one thread, then a barrier) overlaps their latency
    const int io = Lat::opp(i);
    const float w = weight_rt(i), wo = weight_rt(io);
    const uint32_t NP = uint32_t(d.npad);
    const void* fin = d.f[a];
    const bool live_node = node >= 0;
    const uint32_t nn = live_node ? uint32_t(node) : 0u;
    const bool is_wall = info >= CS_WALL, is_inlet = info == CS_INLET;
    float fo = 0.0f, f2 = 0.0f, e0 = 0.0f, e1 = 0.0f, e2 = 0.0f, pk = 0.0f;
    if (live_node) {
        fo = Pop<ST>::ld(fin, uint32_t(io) * NP + nn, wo);
        if (is_wall) {
            if (d.bouzidi) {
                if (qslot < 0.5f) {
                    if (info >= 0) f2 = Pop<ST>::ld(fin, uint32_t(io) * NP + uint32_t(info), wo);
                } else {
                    f2 = Pop<ST>::ld(fin, uint32_t(i) * NP + nn, w);
                }
            }
        } else if (is_inlet) {
            const float* u = d.uin + 3 * int64_t(node);
            e0 = __ldg(u);
            e1 = __ldg(u + 1);
            e2 = __ldg(u + 2);
        } else {
            const float* vin = d.vel[a];
            e0 = __ldg(vin + node);
            e1 = __ldg(vin + d.n + node);
            e2 = __ldg(vin + 2 * d.n + node);
            pk = __ldg(d.p_out + (CS_OUTLET0 - info));
        }
    }
    // the clock: the first thread of the grid publishes this step's drive and advances the tick; an inlet link
    // evaluates the drive itself (no block waits for one thread's evaluation)
    if (threadIdx.x == 0 && clock) {
        const int t = d.tick[a];
        *d.drive = drive_value(d, t);
        d.tick[1 - a] = t + 1;
    }
    launch_dependents();                                    // the bulk kernel may start its static loads
    if (!live_node) return;                                 // padding slot of a direction with fewer links
    const float cx = float(k_cx[i]), cy = float(k_cy[i]), cz = float(k_cz[i]);
    float v;
    if (is_wall) {
        // lbm.py:163-173: interpolated bounce-back, or half-way bounce-back without Bouzidi
        v = fo;
        if (d.bouzidi) {
            const float q = qslot;
            if (q < 0.5f) {
                if (info >= 0) v = 2.0f * q * fo + (1.0f - 2.0f * q) * f2;
            } else {
                v = fo / (2.0f * q) + (2.0f * q - 1.0f) / (2.0f * q) * f2;
            }
        }
    } else if (is_inlet) {
        // lbm.py:174-177: bounce-back with the prescribed velocity
        const float dv = drive_value(d, d.tick[a]);
        const float cu = cx * (e0 * dv) + cy * (e1 * dv) + cz * (e2 * dv);
        v = fo + 6.0f * w * cu;
    } else {
        // lbm.py:178-181: anti-bounce-back with the outlet's pressure and the previous velocity
        const float cu = cx * e0 + cy * e1 + cz * e2;
        const float usq = e0 * e0 + e1 * e1 + e2 * e2;
        v = -fo + 2.0f * w * (3.0f * pk + 4.5f * cu * cu - 1.5f * usq);
    }
    Pop<ST>::st(d.f[a], uint32_t(i) * NP + uint32_t(d.n + g), w, v);
}

// Direction of block b of the unpadded boundary grid: the largest i with gblock[i] <= b.
__device__ __forceinline__ int grid_direction(const int32_t* gblock, int b) {
    int lo = 0, hi = Q - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (gblock[mid] <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Work item `item` of a lattice's boundary-link grid: a 256-slot chunk of one direction (unpadded grid when gblock
// is set, else ceil(gmax / 256) chunks per direction); item 0 advances the clock.
template <int ST>
__device__ __forceinline__ void boundary_item(const cs_step_desc& d, const int a, const int item) {
    if (d.gblock[Q] > 0) {
        const int i = grid_direction(d.gblock, item);
        boundary_body<ST>(d, a, item - d.gblock[i], i, item == 0);
    } else {
        const int nbx = int(max(int64_t(1), ceil_div(d.gmax, B_THREADS)));
        boundary_body<ST>(d, a, item % nbx, item / nbx, item == 0);
    }
}

__host__ __device__ __forceinline__ int boundary_items(const cs_step_desc& d) {
    if (d.gblock[Q] > 0) return d.gblock[Q];
    const int64_t nbx = d.gmax > 0 ? (d.gmax + B_THREADS - 1) / B_THREADS : 1;
    return int(Q * nbx);
}

template <int ST>
__global__ void __launch_bounds__(B_THREADS) k_boundary(const cs_step_desc d, const int a) {
    boundary_item<ST>(d, a, blockIdx.x);
}

// ---- 2. bulk kernel -----------------------------------------------------------------------------------------------
// Writes the 27 outputs w_i (A + E_i + O_i) of a pair-symmetric collision: E(I) even and O(I) odd in c, so link I
// and its opposite share both (the rest link is w_0 A).
template <int ST, class EvenOdd>
__device__ __forceinline__ void store_pairs(void* fout, uint32_t NP, int32_t n, float A, EvenOdd&& eo) {
    Pop<ST>::st(fout, uint32_t(n), wgt(0), wgt(0) * A);
    Unroll<0, 13>::run([&](auto pc) {
        constexpr int I = 1 + 2 * decltype(pc)::value;
        constexpr int O = Lat::opp(I);
        float e, o;
        eo(std::integral_constant<int, I>{}, e, o);
        const float base = A + e;
        Pop<ST>::st(fout, uint32_t(I) * NP + uint32_t(n), wgt(I), wgt(I) * (base + o));
        Pop<ST>::st(fout, uint32_t(O) * NP + uint32_t(n), wgt(O), wgt(O) * (base - o));
    });
}

template <int ST, int MODEL, bool GAL, bool FORCE>
__device__ __forceinline__ void node_update(const cs_step_desc& d, int a, int32_t n, float& ux_o, float& uy_o,
                                            float& uz_o) {
    const int32_t N = int32_t(d.n);
    const uint32_t NP = uint32_t(d.npad);
    const void* fin = d.f[a];
    void* fout = d.f[1 - a];
    const float* vin = d.vel[a];
    float* vout = d.vel[1 - a];
    // connectivity and omega are static: load them while the boundary kernel may still be running
    int32_t lk[Q];
    const int32_t code = __ldg(d.lcode + n);
    if (code >= 0) {
        // one 112-byte row, shared by the warp's nodes of a segment: seven 128-bit loads
        const int4* sd = reinterpret_cast<const int4*>(d.segdelta + int64_t(code) * CS_SEG_STRIDE);
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            const int4 v = __ldg(sd + k);
            lk[4 * k] = n + v.x;
            if (4 * k + 1 < Q) lk[4 * k + 1] = n + v.y;
            if (4 * k + 2 < Q) lk[4 * k + 2] = n + v.z;
            if (4 * k + 3 < Q) lk[4 * k + 3] = n + v.w;
        }
    } else {
        const int32_t* ir = d.irr + (-1 - code);
#pragma unroll
        for (int i = 0; i < Q; ++i) lk[i] = __ldg(ir + int64_t(i) * d.n_irr);
    }
    const float om_signed = __ldg(d.om + n);
    grid_dependency_wait();
    const float dv = __ldg(d.drive);
    const float upx = __ldg(vin + n), upy = __ldg(vin + N + n), upz = __ldg(vin + 2 * N + n);

    // six loads for the Galilean differences, issued with the pull
    float g[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (GAL) {
#pragma unroll
        for (int k = 0; k < 6; ++k) g[k] = __ldg(grad_src(d, vin, 1 + k, k / 2, lk[1 + k]));
    }

    // the 27 pulls (TRT and the body-force path use the populations themselves after the moments)
    Moments m;
    float fk[Q];
    Unroll<0, Q>::run([&](auto ic) {
        constexpr int I = decltype(ic)::value;
        fk[I] = Pop<ST>::ld(fin, uint32_t(I) * NP + uint32_t(lk[I]), wgt(I));
    });
    moments27(fk, m);

    const bool inlet_cell = om_signed < 0.0f;
    const float om = fabsf(om_signed);
    // without a body force (FORCE false) every force term folds away at compile time
    const float Fx = FORCE ? d.force[0] * dv : 0.0f, Fy = FORCE ? d.force[1] * dv : 0.0f;
    const float Fz = FORCE ? d.force[2] * dv : 0.0f;
    const float ux = m.jx + Fx * 0.5f, uy = m.jy + Fy * 0.5f, uz = m.jz + Fz * 0.5f;
    const float usq = ux * ux + uy * uy + uz * uz;
    const float uF = ux * Fx + uy * Fy + uz * Fz;
    float t3 = 0.0f, edx = 0.0f, edy = 0.0f, edz = 0.0f;
    if (GAL) {
        t3 = 1.0f;
        const float tp3 = 3.0f * __frcp_rn(om);
        edx = tp3 * ux * ux * ddx_g(lk[1], lk[2], g[0], g[1], upx, N);
        edy = tp3 * uy * uy * ddx_g(lk[3], lk[4], g[2], g[3], upy, N);
        edz = tp3 * uz * uz * ddx_g(lk[5], lk[6], g[4], g[5], upz, N);
    }
    const float dr = m.dr;

    if (inlet_cell) {
        // lbm.py:205-216: equilibrium at the prescribed velocity
        const float* u = d.uin + 3 * int64_t(n);
        const float tx = __ldg(u) * dv, ty = __ldg(u + 1) * dv, tz = __ldg(u + 2) * dv;
        const float tsq = tx * tx + ty * ty + tz * tz;
        const Cubic cu3(tx, ty, tz);
        store_pairs<ST>(fout, NP, n, dr - 1.5f * tsq, [&](auto ic, float& e, float& o) {
            constexpr int I = decltype(ic)::value;
            const float cu = cdot<I>(tx, ty, tz);
            e = 4.5f * cu * cu;
            o = 3.0f * cu + t3 * cu3.template h3<I>();
        });
        vout[n] = tx;
        vout[N + n] = ty;
        vout[2 * N + n] = tz;
        d.rho[n] = dr;
        ux_o = tx;
        uy_o = ty;
        uz_o = tz;
        return;
    }

    const Cubic cu3(ux, uy, uz);
    if constexpr (MODEL == CS_MODEL_REGULARISED) {
        float pxx, pyy, pzz, pxy, pxz, pyz;
        if constexpr (FORCE) {
            // with a body force, P link by link as the reference sums it (lbm.py:220-223): a slowly forced steady
            // state (Poiseuille at tau ~ 0.505, forces ~1e-7) keeps the FP32 rounding of this order
            pxx = pyy = pzz = pxy = pxz = pyz = 0.0f;
            Unroll<0, Q>::run([&](auto ic) {
                constexpr int I = decltype(ic)::value;
                constexpr int x = Lat::cx(I), y = Lat::cy(I), z = Lat::cz(I);
                const float cu = cdot<I>(ux, uy, uz);
                const float sv = fk[I] - wgt(I) * (dr + 3.0f * cu + 4.5f * cu * cu - 1.5f * usq);
                if (x) pxx += sv;
                if (y) pyy += sv;
                if (z) pzz += sv;
                if (x && y) pxy += float(x * y) * sv;
                if (x && z) pxz += float(x * z) * sv;
                if (y && z) pyz += float(y * z) * sv;
            });
        } else {
            const float d3 = dr * (1.0f / 3.0f);
            pxx = m.pxx - d3 - ux * ux, pyy = m.pyy - d3 - uy * uy, pzz = m.pzz - d3 - uz * uz;
            pxy = m.pxy - ux * uy, pxz = m.pxz - ux * uz, pyz = m.pyz - uy * uz;
        }
        if (d.sigma < 1.0f) {
            // hybrid regularisation (lbm.py:224-229): G[a][b] = du_b/dx_a from the previous step's velocity
            float gr[3][3];
            const float u0[3] = {upx, upy, upz};
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) {
                const int km = 1 + 2 * ax, kp = 2 + 2 * ax;
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    gr[ax][c] = ddx_g(lk[km], lk[kp], __ldg(grad_src(d, vin, km, c, lk[km])),
                                      __ldg(grad_src(d, vin, kp, c, lk[kp])), u0[c], N);
            }
            const float sg = d.sigma, k = (1.0f - sg) / (3.0f * om);
            pxx = sg * pxx - k * (2.0f * gr[0][0]);
            pyy = sg * pyy - k * (2.0f * gr[1][1]);
            pzz = sg * pzz - k * (2.0f * gr[2][2]);
            pxy = sg * pxy - k * (gr[0][1] + gr[1][0]);
            pxz = sg * pxz - k * (gr[0][2] + gr[2][0]);
            pyz = sg * pyz - k * (gr[1][2] + gr[2][1]);
        }
        pxx -= edx;
        pyy -= edy;
        pzz -= edz;
        const float trp = (pxx + pyy + pzz) * (1.0f / 3.0f);
        const float k_ne = 1.0f - om, k_src = 1.0f - 0.5f * om;
        if constexpr (FORCE) {
            // f_out = feq + (1 - om) fneq + (1 - om/2) src per link in the reference's order (lbm.py:232-240)
            const float w0 = wgt(0);
            Pop<ST>::st(fout, uint32_t(n), w0, w0 * (dr - 1.5f * usq) + k_ne * (w0 * (4.5f * (0.0f - trp))) +
                                                   k_src * (w0 * (-3.0f * uF)));
            Unroll<0, 13>::run([&](auto pc) {
                constexpr int I = 1 + 2 * decltype(pc)::value;
                constexpr int O = Lat::opp(I);
                const float cu = cdot<I>(ux, uy, uz), cF = cdot<I>(Fx, Fy, Fz);
                const float cpc = quad<I>(pxx, pyy, pzz, 2.0f * pxy, 2.0f * pxz, 2.0f * pyz);
                const float h = t3 * cu3.template h3<I>();
                const float w = wgt(I);
                const float feq_i = w * (dr + 3.0f * cu + 4.5f * cu * cu - 1.5f * usq + h);
                const float feq_o = w * (dr - 3.0f * cu + 4.5f * cu * cu - 1.5f * usq - h);
                const float fneq_i = w * (4.5f * (cpc - trp) - 1.5f * cF);
                const float fneq_o = w * (4.5f * (cpc - trp) + 1.5f * cF);
                const float src_i = w * (3.0f * cF + 9.0f * cu * cF - 3.0f * uF);
                const float src_o = w * (-3.0f * cF + 9.0f * cu * cF - 3.0f * uF);
                Pop<ST>::st(fout, uint32_t(I) * NP + uint32_t(n), w, feq_i + k_ne * fneq_i + k_src * src_i);
                Pop<ST>::st(fout, uint32_t(O) * NP + uint32_t(n), w, feq_o + k_ne * fneq_o + k_src * src_o);
            });
            vout[n] = ux;
            vout[N + n] = uy;
            vout[2 * N + n] = uz;
            d.rho[n] = dr;
            ux_o = ux;
            uy_o = uy;
            uz_o = uz;
            return;
        }
        // without a force: f_out = feq + (1 - om) fneq + (1 - om/2) src (lbm.py:236-240) regrouped as
        // w (A + E +- O), each pair's terms evaluated once
        const float A = dr - 1.5f * usq - 4.5f * k_ne * trp;
        const float s = 4.5f * k_ne;
        const float hx = 4.5f * ux, hy = 4.5f * uy;
        store_regularised<ST, GAL>(fout, NP, n, A, ux, uy, uz, fmaf(hx, ux, s * pxx), fmaf(hy, uy, s * pyy),
                                   fmaf(4.5f * uz, uz, s * pzz), fmaf(2.0f * hx, uy, 2.0f * s * pxy),
                                   fmaf(2.0f * hx, uz, 2.0f * s * pxz), fmaf(2.0f * hy, uz, 2.0f * s * pyz));
    } else {
        // TRT + Guo forcing (lbm.py:241-255)
        const float om_m = 1.0f / (0.5f + d.magic / (1.0f / om - 0.5f));
        const float ddx_ = -(1.0f - om) * edx, ddy_ = -(1.0f - om) * edy, ddz_ = -(1.0f - om) * edz;
        const float trd = (ddx_ + ddy_ + ddz_) / 3.0f;
        Unroll<0, Q>::run([&](auto ic) {
            constexpr int I = decltype(ic)::value;
            constexpr int jo = Lat::opp(I);
            constexpr int x = Lat::cx(I), y = Lat::cy(I), z = Lat::cz(I);
            const float cv = float(x) * ux + float(y) * uy + float(z) * uz;
            const float cF = float(x) * Fx + float(y) * Fy + float(z) * Fz;
            const float eqp = wgt(I) * (dr + 4.5f * cv * cv - 1.5f * usq);
            const float eqm = wgt(I) * (3.0f * cv + t3 * cu3.template h3<I>());
            const float psi = wgt(I) * 4.5f * (float(x * x) * ddx_ + float(y * y) * ddy_ + float(z * z) * ddz_ - trd);
            const float fp = 0.5f * (fk[I] + fk[jo]);
            const float fm = 0.5f * (fk[I] - fk[jo]);
            const float sp = wgt(I) * (9.0f * cv * cF - 3.0f * uF);
            const float smv = wgt(I) * 3.0f * cF;
            Pop<ST>::st(fout, uint32_t(I) * NP + uint32_t(n), wgt(I),
                        fk[I] - om * (fp - eqp) - om_m * (fm - eqm) + (1.0f - 0.5f * om) * sp +
                            (1.0f - 0.5f * om_m) * smv + psi);
        });
    }
    vout[n] = ux;
    vout[N + n] = uy;
    vout[2 * N + n] = uz;
    d.rho[n] = dr;
    ux_o = ux;
    uy_o = uy;
    uz_o = uz;
}

// Block bx of a lattice's bulk grid (nodes bx * blockDim .. + blockDim - 1). Called by every thread of the block.
template <int ST, int MODEL, bool GAL, bool FORCE>
__device__ __forceinline__ void bulk_body(const cs_step_desc& d, const int a, const int bx) {
    __shared__ float s_u[3][MAX_BLOCK];
    const int32_t n0 = int32_t(bx) * int32_t(blockDim.x);
    const int32_t n = n0 + int32_t(threadIdx.x);
    float ux = 0.f, uy = 0.f, uz = 0.f;
    if (n < d.n) node_update<ST, MODEL, GAL, FORCE>(d, a, n, ux, uy, uz);
    grid_dependency_wait();      // (threads without a node) the flux accumulators were reset by the last step
    launch_dependents();

    if (d.n_open > 0) {
        // slab flux Q_k = sum u . w over this block's flux entries (simulate.py:65-69), FP64, in a fixed order: each
        // thread sums its entries, warps reduce by shuffles, warp 0 adds the warps in order; the block's partial
        // sums go to its own row of q_part, which k_bc adds up in a fixed order too (no atomics: bit-reproducible)
        const int e0 = __ldg(d.flux_block + bx), e1 = __ldg(d.flux_block + bx + 1);
        if (e1 > e0) {
            s_u[0][threadIdx.x] = ux;
            s_u[1][threadIdx.x] = uy;
            s_u[2][threadIdx.x] = uz;
            __syncthreads();
            double acc[MAX_OPEN];
#pragma unroll
            for (int k = 0; k < MAX_OPEN; ++k) acc[k] = 0.0;
            for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
                const int loc = __ldg(d.flux_idx + e) - n0;
                if (loc < 0 || loc >= int(blockDim.x)) continue;  // partition built for another block size
                const float* w = d.flux_w + 3 * int64_t(e);
                const double v = double(s_u[0][loc]) * double(__ldg(w)) + double(s_u[1][loc]) * double(__ldg(w + 1)) +
                                 double(s_u[2][loc]) * double(__ldg(w + 2));
                const int slot = __ldg(d.flux_slot + e);
#pragma unroll
                for (int k = 0; k < MAX_OPEN; ++k) acc[k] += slot == k ? v : 0.0;
            }
            __shared__ double s_w[MAX_BLOCK / 32][MAX_OPEN];
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
            for (int k = 0; k < MAX_OPEN; ++k) {
                double x = acc[k];
                for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
                if (lane == 0) s_w[warp][k] = x;
            }
            __syncthreads();
            if (threadIdx.x < d.n_open) {
                double t = 0.0;
                for (int w = 0; w < int(blockDim.x) / 32; ++w) t += s_w[w][threadIdx.x];
                d.q_part[int64_t(bx) * MAX_OPEN + threadIdx.x] = t;
            }
        }
    }
}

template <int ST, int MODEL, bool GAL, bool FORCE>
__global__ void __launch_bounds__(MAX_BLOCK, MIN_BLOCKS) k_bulk(const cs_step_desc d, const int a) {
    bulk_body<ST, MODEL, GAL, FORCE>(d, a, blockIdx.x);
}

// The regularised step without a body force (every open vessel) in blocks of at most 128 threads: compiled for 9
// such blocks per SM (56 registers, 8 bytes of spill) instead of 8 at 64 registers. The extra warps hide more of the
// pulls' latency: 3-4 % faster steps from a cold L2 (the batched kernel, whose descriptor handling needs the
// registers, keeps 64).
constexpr int DENSE_BLOCK = 128;
constexpr int DENSE_MIN_BLOCKS = 9;

template <int ST, bool GAL>
__global__ void __launch_bounds__(DENSE_BLOCK, DENSE_MIN_BLOCKS) k_bulk_dense(const cs_step_desc d, const int a) {
    bulk_body<ST, CS_MODEL_REGULARISED, GAL, false>(d, a, blockIdx.x);
}

// ---- 3. outlet resistances ----------------------------------------------------------------------------------------
constexpr int BC_THREADS = 256;

// simulate.py:76-82 in FP64 (one block of BC_THREADS threads); the drive of this step was stored by the boundary
// kernel. Q_k = the flux blocks' partial sums, added by a fixed-shape tree (the same order at every step and run).
__device__ __forceinline__ void bc_body(const cs_step_desc& d) {
    __shared__ double s_red[BC_THREADS];
    __shared__ double s_q[MAX_OPEN];
    for (int k = 0; k < d.n_open; ++k) {
        double t = 0.0;
        for (int j = threadIdx.x; j < d.n_fb; j += BC_THREADS) t += d.q_part[int64_t(__ldg(d.fb_list + j)) * MAX_OPEN + k];
        s_red[threadIdx.x] = t;
        __syncthreads();
        for (int h = BC_THREADS / 2; h > 0; h >>= 1) {
            if (threadIdx.x < h) s_red[threadIdx.x] += s_red[threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x == 0) s_q[k] = s_red[0];
        __syncthreads();
    }
    const int k = threadIdx.x;
    if (k >= d.n_open) return;
    const double qk = s_q[k];
    d.q_last[k] = qk;
    double pk;
    if (k == 0) {
        const float dv = *d.drive;
        d.p_out[0] = dv;
        pk = double(dv);
    } else {
        pk = d.p_out64[k] + d.alpha * (double(d.r_out[k]) * qk - d.pref - d.p_out64[k]);
        d.p_out[k] = float(pk);
    }
    d.p_out64[k] = pk;
    if (d.beat_acc) {
        // running sums for the beat means of the open ends' pressure and flow (one thread per open end)
        d.beat_acc[k] += pk;
        d.beat_acc[d.n_open + k] += qk;
        if (k == 0) d.beat_acc[2 * d.n_open] += 1.0;
    }
}

__global__ void k_bc(const cs_step_desc d) { bc_body(d); }

using StepFn = void (*)(const cs_step_desc, const int);

template <int ST>
StepFn pick_force(int model, int gal, bool force, int block) {
    if (model == CS_MODEL_REGULARISED && !force && block <= DENSE_BLOCK)
        return gal ? k_bulk_dense<ST, true> : k_bulk_dense<ST, false>;
    if (model == CS_MODEL_REGULARISED) {
        if (gal) return force ? k_bulk<ST, CS_MODEL_REGULARISED, true, true> : k_bulk<ST, CS_MODEL_REGULARISED, true, false>;
        return force ? k_bulk<ST, CS_MODEL_REGULARISED, false, true> : k_bulk<ST, CS_MODEL_REGULARISED, false, false>;
    }
    if (gal) return force ? k_bulk<ST, CS_MODEL_TRT, true, true> : k_bulk<ST, CS_MODEL_TRT, true, false>;
    return force ? k_bulk<ST, CS_MODEL_TRT, false, true> : k_bulk<ST, CS_MODEL_TRT, false, false>;
}

template <int ST>
StepFn pick_model(const cs_step_desc& d) {
    const bool force = d.force[0] != 0.0f || d.force[1] != 0.0f || d.force[2] != 0.0f;
    return pick_force<ST>(d.model, d.gal, force, d.block ? d.block : MAX_BLOCK);
}

StepFn pick_bulk(const cs_step_desc& d) {
    switch (d.storage) {
        case CS_STORE_F16: return pick_model<CS_STORE_F16>(d);
        case CS_STORE_BF16: return pick_model<CS_STORE_BF16>(d);
        default: return pick_model<CS_STORE_F32>(d);
    }
}

StepFn pick_boundary(const cs_step_desc& d) {
    switch (d.storage) {
        case CS_STORE_F16: return k_boundary<CS_STORE_F16>;
        case CS_STORE_BF16: return k_boundary<CS_STORE_BF16>;
        default: return k_boundary<CS_STORE_F32>;
    }
}

int validate(const cs_step_desc* d) {
    if (!d) return fail(CS_ERR_ARG, "cs_step: null descriptor");
    if (d->n < 0 || d->n >= (int64_t(1) << 30)) return fail(CS_ERR_SIZE, "cs_step: n = %lld", (long long)d->n);
    if (d->gmax < 0 || d->npad != d->n + d->gmax || int64_t(Q) * d->npad >= (int64_t(1) << 31))
        return fail(CS_ERR_SIZE, "cs_step: npad %lld must be n + gmax with 27 * npad < 2^31", (long long)d->npad);
    if (d->gblock[0] != 0) return fail(CS_ERR_ARG, "cs_step: gblock[0] = %d", d->gblock[0]);
    for (int i = 0; i < Q; ++i) {
        const int64_t w = int64_t(d->gblock[i + 1]) - d->gblock[i];
        if (w < 0 || w * B_THREADS > std::max<int64_t>(d->gmax, 0) + B_THREADS - 1)
            return fail(CS_ERR_ARG, "cs_step: gblock[%d..%d] = %d..%d for gmax %lld", i, i + 1, d->gblock[i],
                        d->gblock[i + 1], (long long)d->gmax);
    }
    if (d->storage < 0 || d->storage > 2) return fail(CS_ERR_ARG, "cs_step: storage %d", d->storage);
    if (d->model != CS_MODEL_TRT && d->model != CS_MODEL_REGULARISED) return fail(CS_ERR_ARG, "cs_step: model %d", d->model);
    if (d->block != 0 && (d->block < 32 || d->block > MAX_BLOCK || d->block % 32))
        return fail(CS_ERR_ARG, "cs_step: block %d (32..%d, multiple of 32)", d->block, MAX_BLOCK);
    if (d->period < 1 || d->nh < 0 || d->ramp < 0) return fail(CS_ERR_ARG, "cs_step: period %d nh %d ramp %d", d->period, d->nh, d->ramp);
    if (!d->tick || !d->drive || !d->coef || !d->p_out || d->n_out < 1)
        return fail(CS_ERR_ARG, "cs_step: null clock / outlet state");
    if (d->n > 0 && (!d->f[0] || !d->f[1] || !d->vel[0] || !d->vel[1] || !d->rho || !d->lcode || !d->uin || !d->om))
        return fail(CS_ERR_ARG, "cs_step: null lattice buffer");
    if (d->gmax > 0 && (!d->gnode || !d->ginfo || !d->gq)) return fail(CS_ERR_ARG, "cs_step: null ghost table");
    if (d->n_open < 0 || d->n_open > MAX_OPEN || d->n_open > d->n_out)
        return fail(CS_ERR_ARG, "cs_step: n_open %d (at most %d and at most n_out %d)", d->n_open, MAX_OPEN, d->n_out);
    if (d->n_open > 0 && (!d->flux_block || !d->q_part || !d->q_last || !d->p_out64 || !d->r_out ||
                          d->n_fb < 0 || (d->n_fb > 0 && !d->fb_list) ||
                          (d->n_flux > 0 && (!d->flux_idx || !d->flux_w || !d->flux_slot))))
        return fail(CS_ERR_ARG, "cs_step: null flux buffer");
    return CS_OK;
}

// Launch with programmatic stream serialization, so the kernel's static prologue overlaps the previous kernel.
int launch_pdl(StepFn fn, dim3 grid, dim3 block, cudaStream_t st, const cs_step_desc& d, int a) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, fn, d, a);
    if (e != cudaSuccess) return fail(CS_ERR_CUDA, "launch of a step kernel failed: %s", cudaGetErrorString(e));
    return CS_OK;
}

int launch_steps(const cs_step_desc* d, int a, int steps, cudaStream_t st) {
    const int block = d->block ? d->block : MAX_BLOCK;
    const unsigned grid = unsigned(d->n > 0 ? ceil_div(d->n, block) : 0);
    const dim3 bgrid(unsigned(boundary_items(*d)));
    StepFn bulk = pick_bulk(*d);
    StepFn bound = pick_boundary(*d);
    for (int s = 0; s < steps; ++s) {
        // always launched: it also advances the clock
        int rc = launch_pdl(bound, bgrid, dim3(B_THREADS), st, *d, a);
        if (rc != CS_OK) return rc;
        if (grid > 0) {
            rc = launch_pdl(bulk, dim3(grid), dim3(block), st, *d, a);
            if (rc != CS_OK) return rc;
        }
        if (d->n_open > 0) {
            k_bc<<<1, BC_THREADS, 0, st>>>(*d);
            CS_CHECK_LAUNCH("k_bc");
        }
        a = 1 - a;
    }
    return CS_OK;
}

__global__ void k_flux_blocks(const int32_t* __restrict__ idx, int64_t n_flux, int block, int32_t* __restrict__ out,
                              int64_t n_blocks) {
    const int64_t b = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (b > n_blocks) return;
    const int64_t key = b * block;
    int64_t lo = 0, hi = n_flux;  // first entry with idx >= key
    while (lo < hi) {
        const int64_t mid = (lo + hi) / 2;
        if (int64_t(idx[mid]) < key) lo = mid + 1; else hi = mid;
    }
    out[b] = int32_t(lo);
}

}  // namespace
}  // namespace cs

using namespace cs;

extern "C" int cs_flux_blocks(const int32_t* flux_idx, int64_t n_flux, int64_t n, int32_t block, int32_t* out,
                              void* stream) {
    if (n < 0 || n_flux < 0 || block < 32 || block > MAX_BLOCK || !out || (n_flux > 0 && !flux_idx))
        return fail(CS_ERR_ARG, "cs_flux_blocks: bad arguments");
    const int64_t nb = n > 0 ? ceil_div(n, block) : 1;
    k_flux_blocks<<<unsigned(ceil_div(nb + 1, 256)), 256, 0, as_stream(stream)>>>(flux_idx, n_flux, block, out, nb);
    CS_CHECK_LAUNCH("k_flux_blocks");
    return CS_OK;
}

extern "C" int cs_step(const cs_step_desc* d, int32_t a, int32_t steps, void* stream) {
    int rc = validate(d);
    if (rc != CS_OK) return rc;
    if ((a != 0 && a != 1) || steps < 0) return fail(CS_ERR_ARG, "cs_step: a %d steps %d", a, steps);
    return launch_steps(d, a, steps, as_stream(stream));
}

namespace {
struct Graph {
    cudaGraphExec_t exec;
};
}  // namespace

extern "C" int cs_graph_capture(const cs_step_desc* d, int32_t a, int32_t steps, void* stream, void** graph) {
    int rc = validate(d);
    if (rc != CS_OK) return rc;
    if ((a != 0 && a != 1) || steps < 1 || !graph) return fail(CS_ERR_ARG, "cs_graph_capture: a %d steps %d", a, steps);
    cudaStream_t st = as_stream(stream);
    if (st == nullptr) return fail(CS_ERR_ARG, "cs_graph_capture: the legacy default stream cannot be captured");
    CS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    rc = launch_steps(d, a, steps, st);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != CS_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return fail(CS_ERR_CUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(e));
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(CS_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
    *graph = new Graph{ex};
    return CS_OK;
}

extern "C" int cs_graph_launch(void* graph, void* stream) {
    if (!graph) return fail(CS_ERR_ARG, "cs_graph_launch: null graph");
    CS_CUDA(cudaGraphLaunch(static_cast<Graph*>(graph)->exec, as_stream(stream)));
    return CS_OK;
}

extern "C" int cs_graph_destroy(void* graph) {
    if (!graph) return CS_OK;
    Graph* g = static_cast<Graph*>(graph);
    cudaError_t e = cudaGraphExecDestroy(g->exec);
    delete g;
    if (e != cudaSuccess) return fail(CS_ERR_CUDA, "cudaGraphExecDestroy: %s", cudaGetErrorString(e));
    return CS_OK;
}

extern "C" int cs_step_check(const cs_step_desc* d) { return validate(d); }

// ---- batched step -------------------------------------------------------------------------------------------------
// The instances' descriptors travel in the kernels' parameter space (constant bank), CS_BATCH_GROUP instances per
// launch: every block reads the descriptor of the instance it works on there, as the single-lattice kernels read
// theirs, instead of staging it in shared memory (which costs registers and spills in the collision).
namespace cs {
namespace {

struct BatchGroup {
    int32_t n_inst, bulk_items, bnd_items, pad_;
    int32_t* counter;
    int32_t bulk_prefix[CS_BATCH_GROUP + 1];
    int32_t bnd_prefix[CS_BATCH_GROUP + 1];
    int32_t parity[CS_BATCH_GROUP];
    cs_step_desc d[CS_BATCH_GROUP];
};
static_assert(sizeof(BatchGroup) < 32000, "batched kernel parameters exceed the 32 KB limit");

// Largest i in [0, n) with prefix[i] <= item.
__device__ __forceinline__ int find_instance(const int32_t* prefix, int n, int item) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= item) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// A persistent block's share of the boundary work list: a contiguous range of items.
struct ItemRange {
    int lo, hi;
    __device__ ItemRange(int items) {
        const int per = items / int(gridDim.x), rem = items % int(gridDim.x), bx = int(blockIdx.x);
        lo = bx * per + min(bx, rem);
        hi = lo + per + (bx < rem ? 1 : 0);
    }
};

// Instance of each item for a block walking its items in increasing order.
struct InstanceCursor {
    const int32_t* prefix;
    int n, inst = -1, first = 0, end = 0;
    __device__ InstanceCursor(const int32_t* prefix_, int n_) : prefix(prefix_), n(n_) {}
    __device__ __forceinline__ int next(int item) {
        if (item >= end) {
            inst = inst < 0 ? find_instance(prefix, n, item) : inst + 1;
            while (prefix[inst + 1] <= item) ++inst;
            first = prefix[inst];
            end = prefix[inst + 1];
        }
        return item - first;
    }
};

template <int ST>
__global__ void __launch_bounds__(B_THREADS) k_boundary_batch(const __grid_constant__ BatchGroup g, const int a) {
    const ItemRange r(g.bnd_items);
    InstanceCursor cur(g.bnd_prefix, g.n_inst);
    for (int item = r.lo; item < r.hi; ++item) {
        const int local = cur.next(item);
        boundary_item<ST>(g.d[cur.inst], a ^ g.parity[cur.inst], local);
    }
    // the previous bulk kernel has finished (boundary_body waited for it) and the next one takes no item before
    // this kernel ends: reset its work counter
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        grid_dependency_wait();
        *g.counter = 0;
    }
}

// Bulk items are handed out dynamically: block x starts with item x, then takes the next unclaimed item from a
// counter (reset by the boundary kernel each step), so that blocks finishing cheap items (few boundary rows) take
// more of them. The claim for the following item is issued at the start of the current one and lands while it
// runs. Which block updates which item does not change any result (each item writes its own nodes and its own row
// of flux partial sums).
template <int ST, int MODEL, bool GAL, bool FORCE>
__global__ void __launch_bounds__(MAX_BLOCK, MIN_BLOCKS) k_bulk_batch(const __grid_constant__ BatchGroup g,
                                                                      const int a) {
    __shared__ int s_item[2];
    InstanceCursor cur(g.bulk_prefix, g.n_inst);
    int item = blockIdx.x, buf = 0;
    bool first = true;
    while (item < g.bulk_items) {
        const int local = cur.next(item);
        int claim = 0;
        if (!first && threadIdx.x == 0) claim = atomicAdd(g.counter, 1);
        bulk_body<ST, MODEL, GAL, FORCE>(g.d[cur.inst], a ^ g.parity[cur.inst], local);
        if (first && threadIdx.x == 0) claim = atomicAdd(g.counter, 1);   // after the wait inside bulk_body
        first = false;
        if (threadIdx.x == 0) s_item[buf] = int(gridDim.x) + claim;
        __syncthreads();                        // also: the flux partial sums reuse shared memory
        item = s_item[buf];
        buf ^= 1;
    }
}

// One block per bulk item, no loop and no claims (grid_bulk = 0): the regularised step without body force in blocks
// of at most 128 threads, compiled like k_bulk_dense for 9 blocks per SM, which the persistent loop's state does not
// leave registers for. The block finds its instance by a binary search over the item prefix in the parameters.
template <int ST, bool GAL>
__global__ void __launch_bounds__(DENSE_BLOCK, DENSE_MIN_BLOCKS) k_bulk_batch_dense(const __grid_constant__ BatchGroup g,
                                                                                  const int a) {
    const int item = int(blockIdx.x);
    const int inst = find_instance(g.bulk_prefix, g.n_inst, item);
    bulk_body<ST, CS_MODEL_REGULARISED, GAL, false>(g.d[inst], a ^ g.parity[inst], item - g.bulk_prefix[inst]);
}

__global__ void k_bc_batch(const __grid_constant__ BatchGroup g) {
    const cs_step_desc& d = g.d[blockIdx.x];
    if (d.n_open > 0) bc_body(d);
}

using BatchFn = void (*)(const BatchGroup, const int);

template <int ST>
BatchFn pick_batch_model(int model, int gal, bool force, bool dense) {
    if (dense && model == CS_MODEL_REGULARISED && !force)
        return gal ? k_bulk_batch_dense<ST, true> : k_bulk_batch_dense<ST, false>;
    if (model == CS_MODEL_REGULARISED) {
        if (gal) return force ? k_bulk_batch<ST, CS_MODEL_REGULARISED, true, true> : k_bulk_batch<ST, CS_MODEL_REGULARISED, true, false>;
        return force ? k_bulk_batch<ST, CS_MODEL_REGULARISED, false, true> : k_bulk_batch<ST, CS_MODEL_REGULARISED, false, false>;
    }
    if (gal) return force ? k_bulk_batch<ST, CS_MODEL_TRT, true, true> : k_bulk_batch<ST, CS_MODEL_TRT, true, false>;
    return force ? k_bulk_batch<ST, CS_MODEL_TRT, false, true> : k_bulk_batch<ST, CS_MODEL_TRT, false, false>;
}

int validate_batch(const cs_batch_desc* b) {
    if (!b) return fail(CS_ERR_ARG, "cs_batch_step: null descriptor");
    if (b->n_inst < 1 || !b->descs || !b->parity || !b->counter)
        return fail(CS_ERR_ARG, "cs_batch_step: %d instances or null tables", b->n_inst);
    if (b->storage < 0 || b->storage > 2 || (b->model != CS_MODEL_TRT && b->model != CS_MODEL_REGULARISED))
        return fail(CS_ERR_ARG, "cs_batch_step: storage %d model %d", b->storage, b->model);
    if (b->block < 32 || b->block > MAX_BLOCK || b->block % 32)
        return fail(CS_ERR_ARG, "cs_batch_step: block %d (32..%d, multiple of 32)", b->block, MAX_BLOCK);
    if (b->grid_bulk < 0 || b->grid_bnd < 0)
        return fail(CS_ERR_ARG, "cs_batch_step: grid sizes %d / %d", b->grid_bulk, b->grid_bnd);
    int64_t items = 0;
    for (int i = 0; i < b->n_inst; ++i) {
        const cs_step_desc& d = b->descs[i];
        const int rc = validate(&d);
        if (rc != CS_OK) return rc;
        if (d.storage != b->storage || d.model != b->model || d.gal != b->gal || d.block != b->block)
            return fail(CS_ERR_ARG, "cs_batch_step: instance %d differs from the batch in storage, model, Galilean "
                                    "setting or block size", i);
        if ((d.force[0] != 0.f || d.force[1] != 0.f || d.force[2] != 0.f) && !b->force)
            return fail(CS_ERR_ARG, "cs_batch_step: instance %d has a body force but the batch has force = 0", i);
        if (d.n_open > 0 && !b->any_open)
            return fail(CS_ERR_ARG, "cs_batch_step: instance %d has open ends but the batch has any_open = 0", i);
        if (b->parity[i] != 0 && b->parity[i] != 1)
            return fail(CS_ERR_ARG, "cs_batch_step: parity[%d] = %d", i, b->parity[i]);
        items += ceil_div(d.n, int64_t(b->block)) + boundary_items(d);
    }
    if (items > INT32_MAX - int64_t(MAX_BLOCK) * 2048)
        return fail(CS_ERR_SIZE, "cs_batch_step: %lld work items", (long long)items);
    return CS_OK;
}

// The launch groups of a batch: CS_BATCH_GROUP instances each, work items counted per instance.
std::vector<BatchGroup> make_groups(const cs_batch_desc* b) {
    std::vector<BatchGroup> gs;
    for (int i0 = 0; i0 < b->n_inst; i0 += CS_BATCH_GROUP) {
        BatchGroup g;
        std::memset(&g, 0, sizeof(g));
        g.n_inst = std::min(CS_BATCH_GROUP, b->n_inst - i0);
        g.counter = b->counter + i0 / CS_BATCH_GROUP;
        int64_t bulk = 0, bnd = 0;
        for (int k = 0; k < g.n_inst; ++k) {
            const cs_step_desc& d = b->descs[i0 + k];
            g.d[k] = d;
            g.parity[k] = b->parity[i0 + k];
            g.bulk_prefix[k] = int32_t(bulk);
            g.bnd_prefix[k] = int32_t(bnd);
            bulk += ceil_div(d.n, int64_t(b->block));
            bnd += boundary_items(d);
        }
        g.bulk_prefix[g.n_inst] = int32_t(bulk);
        g.bnd_prefix[g.n_inst] = int32_t(bnd);
        g.bulk_items = int32_t(bulk);
        g.bnd_items = int32_t(bnd);
        gs.push_back(g);
    }
    return gs;
}

int launch_batch_pdl(BatchFn fn, unsigned grid, unsigned block, cudaStream_t st, const BatchGroup& g, int a) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, fn, g, a);
    if (e != cudaSuccess) return fail(CS_ERR_CUDA, "launch of a batched step kernel failed: %s", cudaGetErrorString(e));
    return CS_OK;
}

int launch_batch(const cs_batch_desc* b, int a, int steps, cudaStream_t st) {
    const std::vector<BatchGroup> gs = make_groups(b);
    const bool force = b->force != 0;
    const bool dense = b->grid_bulk == 0 && b->block <= DENSE_BLOCK;     // one block per item: k_bulk_batch_dense
    BatchFn bulk = b->storage == CS_STORE_F16    ? pick_batch_model<CS_STORE_F16>(b->model, b->gal, force, dense)
                   : b->storage == CS_STORE_BF16 ? pick_batch_model<CS_STORE_BF16>(b->model, b->gal, force, dense)
                                                 : pick_batch_model<CS_STORE_F32>(b->model, b->gal, force, dense);
    BatchFn bound = b->storage == CS_STORE_F16    ? k_boundary_batch<CS_STORE_F16>
                    : b->storage == CS_STORE_BF16 ? k_boundary_batch<CS_STORE_BF16>
                                                  : k_boundary_batch<CS_STORE_F32>;
    for (int s = 0; s < steps; ++s) {
        for (const BatchGroup& g : gs) {
            const unsigned gb = unsigned(b->grid_bnd > 0 ? std::min(b->grid_bnd, g.bnd_items) : g.bnd_items);
            const int rc = launch_batch_pdl(bound, gb, B_THREADS, st, g, a);
            if (rc != CS_OK) return rc;
        }
        for (const BatchGroup& g : gs) {
            const unsigned gk = unsigned(b->grid_bulk > 0 ? std::min(b->grid_bulk, g.bulk_items) : g.bulk_items);
            if (gk == 0) continue;
            const int rc = launch_batch_pdl(bulk, gk, unsigned(b->block), st, g, a);
            if (rc != CS_OK) return rc;
        }
        if (b->any_open) {
            for (const BatchGroup& g : gs) {
                k_bc_batch<<<unsigned(g.n_inst), BC_THREADS, 0, st>>>(g);
                CS_CHECK_LAUNCH("k_bc_batch");
            }
        }
        a = 1 - a;
    }
    return CS_OK;
}

}  // namespace
}  // namespace cs

extern "C" int cs_batch_step(const cs_batch_desc* b, int32_t a, int32_t steps, void* stream) {
    int rc = validate_batch(b);
    if (rc != CS_OK) return rc;
    if ((a != 0 && a != 1) || steps < 0) return fail(CS_ERR_ARG, "cs_batch_step: a %d steps %d", a, steps);
    return launch_batch(b, a, steps, as_stream(stream));
}

extern "C" int cs_batch_graph_capture(const cs_batch_desc* b, int32_t a, int32_t steps, void* stream, void** graph) {
    int rc = validate_batch(b);
    if (rc != CS_OK) return rc;
    if ((a != 0 && a != 1) || steps < 1 || !graph)
        return fail(CS_ERR_ARG, "cs_batch_graph_capture: a %d steps %d", a, steps);
    cudaStream_t st = as_stream(stream);
    if (st == nullptr) return fail(CS_ERR_ARG, "cs_batch_graph_capture: the legacy default stream cannot be captured");
    CS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    rc = launch_batch(b, a, steps, st);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != CS_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return fail(CS_ERR_CUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(e));
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(CS_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
    *graph = new Graph{ex};
    return CS_OK;
}
