// Fused sparse D3Q27 step on the GPU: the work of lbm.k_clock + lbm.k_step (lbm.py:90-257) and, for the artery
// solver, simulate.k_flux + simulate.k_bc (simulate.py:65-82) in ONE kernel per step.
//
// One thread per fluid node, C-ordered nodes, link-major populations f[i * N + n] (the reference's SoA layout):
// for every link the warp's 32 pull sources are mostly consecutive, so each gathered load and each store is a
// coalesced 128-byte line. Per node the kernel reads 27 link codes, 27 populations, omega and the previous
// velocity (plus six neighbour velocity components for the Galilean correction, mostly L2 hits) and writes 27
// populations, the velocity and the density: the 356 B/update of an FP32 step.
//
//  - clock (lbm.py:94-101): every block evaluates drive(tick) itself; the last block to finish advances tick and
//    stores the drive value, so no separate launch is needed.
//  - boundary links (lbm.py:156-182): wall links carry their q in the link code, so no q table is read; inlet and
//    outlet links use uin / p_out; a cell with an inlet link is an equilibrium inlet cell (lbm.py:205-216, 370).
//  - regularised collision (lbm.py:217-240): instead of holding 27 populations and summing c c^T (f - feq) link
//    by link, the pull loop accumulates dr, j and Pi = sum c c^T f on the fly; by the D3Q27 isotropy
//    sum_i w_i c c^T feq2_i = dr/3 I + u u^T, so P = Pi - dr/3 I - u u^T, which is the reference's P up to
//    rounding. Populations are therefore streamed, not kept in registers.
//  - TRT (lbm.py:241-255) keeps the 27 populations (it needs f_i and f_opp(i)); it is off the validated path.
//  - slab flux + outlet resistances (simulate.py:65-82): blocks holding flux cells reduce u . w in FP64 from
//    shared memory and add to q_acc; the last block applies k_bc in FP64 (p_out64 holds the state) and resets
//    q_acc.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "cs_common.cuh"

namespace cs {
namespace {

constexpr int MAX_BLOCK = 256;
constexpr int MAX_OPEN = 8;
constexpr float PI_F = 3.14159265358979323846f;

// ---- population storage -----------------------------------------------------------------------------------------
template <int ST> struct Pop;

template <> struct Pop<CS_STORE_F32> {
    static __device__ __forceinline__ float ld(const void* b, int64_t idx, int) {
        return __ldg(static_cast<const float*>(b) + idx);
    }
    static __device__ __forceinline__ void st(void* b, int64_t idx, int, float v) { static_cast<float*>(b)[idx] = v; }
};

// 16-bit formats store (f - w_i) * 1024 / w_i: every link's values share one range, well inside FP16's normal
// numbers, so the relative rounding error is the format's 2^-11 (FP16) or 2^-8 (BF16) at every link.
template <> struct Pop<CS_STORE_F16> {
    static __device__ __forceinline__ float ld(const void* b, int64_t idx, int i) {
        return __half2float(__ldg(static_cast<const __half*>(b) + idx)) * (wgt(i) * (1.0f / 1024.0f));
    }
    static __device__ __forceinline__ void st(void* b, int64_t idx, int i, float v) {
        static_cast<__half*>(b)[idx] = __float2half_rn(v * (1024.0f / wgt(i)));
    }
};

template <> struct Pop<CS_STORE_BF16> {
    static __device__ __forceinline__ float ld(const void* b, int64_t idx, int i) {
        return __bfloat162float(__ldg(static_cast<const __nv_bfloat16*>(b) + idx)) * (wgt(i) * (1.0f / 1024.0f));
    }
    static __device__ __forceinline__ void st(void* b, int64_t idx, int i, float v) {
        static_cast<__nv_bfloat16*>(b)[idx] = __float2bfloat16_rn(v * (1024.0f / wgt(i)));
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

// One component of the non-uniform central difference (lbm.py:105-126): du_c/dx_a from the links that pull from
// x - e_a (sm) and x + e_a (sp); a wall is u = 0 at distance max(q, 0.1), an opening u = u0 at distance 1.
__device__ __forceinline__ float ddx(int32_t sm, int32_t sp, const float* __restrict__ comp, float u0) {
    float h1 = 1.0f, v1 = u0, h2 = 1.0f, v2 = u0;
    if (sm >= 0) {
        v1 = __ldg(comp + sm);
    } else if (is_wall(sm)) {
        h1 = fmaxf(wall_q(sm), 0.1f);
        v1 = 0.0f;
    }
    if (sp >= 0) {
        v2 = __ldg(comp + sp);
    } else if (is_wall(sp)) {
        h2 = fmaxf(wall_q(sp), 0.1f);
        v2 = 0.0f;
    }
    return (h1 * h1 * (v2 - u0) + h2 * h2 * (u0 - v1)) / (h1 * h2 * (h1 + h2));
}

// Third-order equilibrium term of link i (lbm.py:129-137) from the velocity monomials m.
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
        return 13.5f * (ax * (float(y) * xxy + float(z) * xxz) + ay * (float(x) * xyy + float(z) * yyz) +
                        az * (float(x) * xzz + float(y) * yzz)) +
               float(27 * x * y * z) * xyz;
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

struct NodeCtx {
    const cs_step_desc* d;
    const void* fin;
    int64_t N, n;
    float dv;
    float upx, upy, upz, upsq;
};

// Pull of link I when its code is not a fluid source (lbm.py:163-181).
template <int ST, int I>
__device__ __forceinline__ float boundary_pull(const NodeCtx& c, int32_t s, int32_t s_opp, bool& inlet_cell) {
    constexpr int io = Lat::opp(I);
    constexpr float w = wgt(I);
    constexpr float cx = float(Lat::cx(I)), cy = float(Lat::cy(I)), cz = float(Lat::cz(I));
    const float fo = Pop<ST>::ld(c.fin, int64_t(io) * c.N + c.n, io);
    if (is_wall(s)) {
        float v = fo;
        if (c.d->bouzidi) {
            const float q = wall_q(s);
            if (q < 0.5f) {
                if (s_opp >= 0)
                    v = 2.0f * q * fo + (1.0f - 2.0f * q) * Pop<ST>::ld(c.fin, int64_t(io) * c.N + s_opp, io);
            } else {
                v = fo / (2.0f * q) + (2.0f * q - 1.0f) / (2.0f * q) * Pop<ST>::ld(c.fin, int64_t(I) * c.N + c.n, I);
            }
        }
        return v;
    }
    if (s == CS_INLET) {
        inlet_cell = true;
        const float* u = c.d->uin + 3 * c.n;
        const float cu = cx * (__ldg(u) * c.dv) + cy * (__ldg(u + 1) * c.dv) + cz * (__ldg(u + 2) * c.dv);
        return fo + 6.0f * w * cu;
    }
    const int k = CS_OUTLET0 - s;
    const float cu = cx * c.upx + cy * c.upy + cz * c.upz;
    return -fo + 2.0f * w * (3.0f * __ldg(c.d->p_out + k) + 4.5f * cu * cu - 1.5f * c.upsq);
}

// Moment sums accumulated during the pull.
struct Moments {
    float dr = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
    float pxx = 0.f, pyy = 0.f, pzz = 0.f, pxy = 0.f, pxz = 0.f, pyz = 0.f;
    template <int I>
    __device__ __forceinline__ void add(float v) {
        constexpr int x = Lat::cx(I), y = Lat::cy(I), z = Lat::cz(I);
        dr += v;
        if (x) jx += x * v;
        if (y) jy += y * v;
        if (z) jz += z * v;
        if (x) pxx += v;
        if (y) pyy += v;
        if (z) pzz += v;
        if (x && y) pxy += (x * y) * v;
        if (x && z) pxz += (x * z) * v;
        if (y && z) pyz += (y * z) * v;
    }
};

template <int ST, int MODEL, bool GAL>
__device__ __forceinline__ void node_update(const cs_step_desc& d, int a, float dv, int64_t n, float& ux_o,
                                            float& uy_o, float& uz_o) {
    const int64_t N = d.n;
    const void* fin = d.f[a];
    void* fout = d.f[1 - a];
    const float* vin = d.vel[a];
    float* vout = d.vel[1 - a];

    int32_t lk[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) lk[i] = __ldg(d.links + int64_t(i) * N + n);
    const float om = __ldg(d.om + n);
    NodeCtx c;
    c.d = &d;
    c.fin = fin;
    c.N = N;
    c.n = n;
    c.dv = dv;
    c.upx = __ldg(vin + n);
    c.upy = __ldg(vin + N + n);
    c.upz = __ldg(vin + 2 * N + n);
    c.upsq = c.upx * c.upx + c.upy * c.upy + c.upz * c.upz;
    const float Fx = d.force[0] * dv, Fy = d.force[1] * dv, Fz = d.force[2] * dv;

    Moments m;
    bool inlet_cell = false;
    float fk[MODEL == CS_MODEL_TRT ? Q : 1];
    Unroll<0, Q>::run([&](auto ic) {
        constexpr int I = decltype(ic)::value;
        const int32_t s = lk[I];
        float v;
        if (s >= 0)
            v = Pop<ST>::ld(fin, int64_t(I) * N + s, I);
        else
            v = boundary_pull<ST, I>(c, s, lk[Lat::opp(I)], inlet_cell);
        m.add<I>(v);
        if constexpr (MODEL == CS_MODEL_TRT) fk[I] = v;
    });

    const float ux = m.jx + Fx * 0.5f, uy = m.jy + Fy * 0.5f, uz = m.jz + Fz * 0.5f;
    const float usq = ux * ux + uy * uy + uz * uz;
    const float uF = ux * Fx + uy * Fy + uz * Fz;
    float t3 = 0.0f, edx = 0.0f, edy = 0.0f, edz = 0.0f;
    if (GAL) {
        t3 = 1.0f;
        const float tp = 1.0f / om;
        edx = 3.0f * tp * ux * ux * ddx(lk[1], lk[2], vin, c.upx);
        edy = 3.0f * tp * uy * uy * ddx(lk[3], lk[4], vin + N, c.upy);
        edz = 3.0f * tp * uz * uz * ddx(lk[5], lk[6], vin + 2 * N, c.upz);
    }
    const float dr = m.dr;

    if (inlet_cell) {
        // lbm.py:205-216: equilibrium at the prescribed velocity
        const float* u = d.uin + 3 * n;
        const float tx = __ldg(u) * dv, ty = __ldg(u + 1) * dv, tz = __ldg(u + 2) * dv;
        const float tsq = tx * tx + ty * ty + tz * tz;
        const Cubic cu3(tx, ty, tz);
        Unroll<0, Q>::run([&](auto ic) {
            constexpr int I = decltype(ic)::value;
            constexpr float x = Lat::cx(I), y = Lat::cy(I), z = Lat::cz(I);
            const float cu = x * tx + y * ty + z * tz;
            const float feq = wgt(I) * (dr + 3.0f * cu + 4.5f * cu * cu - 1.5f * tsq + t3 * cu3.template h3<I>());
            Pop<ST>::st(fout, int64_t(I) * N + n, I, feq);
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
        // P = Pi - dr/3 I - u u^T  (= sum c c^T (f - feq2), lbm.py:219-223)
        const float d3 = dr * (1.0f / 3.0f);
        float pxx = m.pxx - d3 - ux * ux, pyy = m.pyy - d3 - uy * uy, pzz = m.pzz - d3 - uz * uz;
        float pxy = m.pxy - ux * uy, pxz = m.pxz - ux * uz, pyz = m.pyz - uy * uz;
        if (d.sigma < 1.0f) {
            // hybrid regularisation (lbm.py:224-229): G[a][b] = du_b/dx_a from the previous step's velocity
            const float* vy = vin + N;
            const float* vz = vin + 2 * N;
            float g[3][3];
            const int32_t sm[3] = {lk[1], lk[3], lk[5]}, sp[3] = {lk[2], lk[4], lk[6]};
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) {
                g[ax][0] = ddx(sm[ax], sp[ax], vin, c.upx);
                g[ax][1] = ddx(sm[ax], sp[ax], vy, c.upy);
                g[ax][2] = ddx(sm[ax], sp[ax], vz, c.upz);
            }
            const float sg = d.sigma, k = (1.0f - sg) / (3.0f * om);
            pxx = sg * pxx - k * (2.0f * g[0][0]);
            pyy = sg * pyy - k * (2.0f * g[1][1]);
            pzz = sg * pzz - k * (2.0f * g[2][2]);
            pxy = sg * pxy - k * (g[0][1] + g[1][0]);
            pxz = sg * pxz - k * (g[0][2] + g[2][0]);
            pyz = sg * pyz - k * (g[1][2] + g[2][1]);
        }
        pxx -= edx;
        pyy -= edy;
        pzz -= edz;
        const float trp = (pxx + pyy + pzz) * (1.0f / 3.0f);
        const float k_ne = 1.0f - om, k_src = 1.0f - 0.5f * om;
        Unroll<0, Q>::run([&](auto ic) {
            constexpr int I = decltype(ic)::value;
            constexpr int x = Lat::cx(I), y = Lat::cy(I), z = Lat::cz(I);
            const float cu = float(x) * ux + float(y) * uy + float(z) * uz;
            const float cF = float(x) * Fx + float(y) * Fy + float(z) * Fz;
            const float feq = wgt(I) * (dr + 3.0f * cu + 4.5f * cu * cu - 1.5f * usq + t3 * cu3.template h3<I>());
            const float cpc = float(x * x) * pxx + float(y * y) * pyy + float(z * z) * pzz +
                              2.0f * (float(x * y) * pxy + float(x * z) * pxz + float(y * z) * pyz);
            const float fneq = wgt(I) * (4.5f * (cpc - trp) - 1.5f * cF);
            const float src = wgt(I) * (3.0f * cF + 9.0f * cu * cF - 3.0f * uF);
            Pop<ST>::st(fout, int64_t(I) * N + n, I, feq + k_ne * fneq + k_src * src);
        });
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
            Pop<ST>::st(fout, int64_t(I) * N + n, I,
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

template <int ST, int MODEL, bool GAL>
__global__ void __launch_bounds__(MAX_BLOCK) k_step(const cs_step_desc d, const int a) {
    __shared__ float s_drive;
    __shared__ int s_tick;
    __shared__ int s_last;
    __shared__ float s_u[3][MAX_BLOCK];
    __shared__ double s_q[MAX_OPEN];
    if (threadIdx.x == 0) {
        s_tick = *d.tick;
        s_drive = drive_value(d, s_tick);
    }
    __syncthreads();
    const float dv = s_drive;
    const int64_t n0 = int64_t(blockIdx.x) * blockDim.x;
    const int64_t n = n0 + threadIdx.x;
    float ux = 0.f, uy = 0.f, uz = 0.f;
    if (n < d.n) node_update<ST, MODEL, GAL>(d, a, dv, n, ux, uy, uz);

    if (d.n_open > 0) {
        // slab flux Q_k += u . w over this block's flux entries (simulate.py:65-69), FP64
        const int e0 = __ldg(d.flux_block + blockIdx.x), e1 = __ldg(d.flux_block + blockIdx.x + 1);
        if (e1 > e0) {
            s_u[0][threadIdx.x] = ux;
            s_u[1][threadIdx.x] = uy;
            s_u[2][threadIdx.x] = uz;
            if (threadIdx.x < MAX_OPEN) s_q[threadIdx.x] = 0.0;
            __syncthreads();
            for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
                const int loc = int(__ldg(d.flux_idx + e) - n0);
                if (loc < 0 || loc >= int(blockDim.x)) continue;  // partition built for another block size
                const float* w = d.flux_w + 3 * int64_t(e);
                const double v = double(s_u[0][loc]) * double(__ldg(w)) + double(s_u[1][loc]) * double(__ldg(w + 1)) +
                                 double(s_u[2][loc]) * double(__ldg(w + 2));
                atomicAdd(&s_q[__ldg(d.flux_slot + e)], v);
            }
            __syncthreads();
            if (threadIdx.x < d.n_open && s_q[threadIdx.x] != 0.0) atomicAdd(d.q_acc + threadIdx.x, s_q[threadIdx.x]);
        }
    }

    // completion: the last block advances the clock (lbm.py:101-102) and applies k_bc (simulate.py:76-82)
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(d.done, 1u);
        s_last = prev == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last && threadIdx.x == 0) {
        __threadfence();
        *d.tick = s_tick + 1;
        *d.drive = dv;
        if (d.n_open > 0) {
            d.p_out[0] = dv;
            d.p_out64[0] = double(dv);
            for (int k = 0; k < d.n_open; ++k) {
                const double qk = __ldcg(d.q_acc + k);
                d.q_last[k] = qk;
                if (k > 0) {
                    const double p = d.p_out64[k] + d.alpha * (double(d.r_out[k]) * qk - d.pref - d.p_out64[k]);
                    d.p_out64[k] = p;
                    d.p_out[k] = float(p);
                }
                d.q_acc[k] = 0.0;
            }
        }
        __threadfence();
        *d.done = 0u;
    }
}

using StepFn = void (*)(const cs_step_desc, const int);

template <int ST>
StepFn pick_model(int model, int gal) {
    if (model == CS_MODEL_REGULARISED) return gal ? k_step<ST, CS_MODEL_REGULARISED, true> : k_step<ST, CS_MODEL_REGULARISED, false>;
    return gal ? k_step<ST, CS_MODEL_TRT, true> : k_step<ST, CS_MODEL_TRT, false>;
}

StepFn pick(const cs_step_desc& d) {
    switch (d.storage) {
        case CS_STORE_F16: return pick_model<CS_STORE_F16>(d.model, d.gal);
        case CS_STORE_BF16: return pick_model<CS_STORE_BF16>(d.model, d.gal);
        default: return pick_model<CS_STORE_F32>(d.model, d.gal);
    }
}

int validate(const cs_step_desc* d) {
    if (!d) return fail(CS_ERR_ARG, "cs_step: null descriptor");
    if (d->n < 0 || d->n >= (int64_t(1) << 30)) return fail(CS_ERR_SIZE, "cs_step: n = %lld", (long long)d->n);
    if (d->storage < 0 || d->storage > 2) return fail(CS_ERR_ARG, "cs_step: storage %d", d->storage);
    if (d->model != CS_MODEL_TRT && d->model != CS_MODEL_REGULARISED) return fail(CS_ERR_ARG, "cs_step: model %d", d->model);
    if (d->block != 0 && (d->block < 32 || d->block > MAX_BLOCK || d->block % 32))
        return fail(CS_ERR_ARG, "cs_step: block %d (32..%d, multiple of 32)", d->block, MAX_BLOCK);
    if (d->period < 1 || d->nh < 0 || d->ramp < 0) return fail(CS_ERR_ARG, "cs_step: period %d nh %d ramp %d", d->period, d->nh, d->ramp);
    if (!d->tick || !d->drive || !d->coef || !d->done || !d->p_out || d->n_out < 1)
        return fail(CS_ERR_ARG, "cs_step: null clock / outlet state");
    if (d->n > 0 && (!d->f[0] || !d->f[1] || !d->vel[0] || !d->vel[1] || !d->rho || !d->links || !d->uin || !d->om))
        return fail(CS_ERR_ARG, "cs_step: null lattice buffer");
    if (d->n_open < 0 || d->n_open > MAX_OPEN || d->n_open > d->n_out)
        return fail(CS_ERR_ARG, "cs_step: n_open %d (at most %d and at most n_out %d)", d->n_open, MAX_OPEN, d->n_out);
    if (d->n_open > 0 && (!d->flux_block || !d->q_acc || !d->q_last || !d->p_out64 || !d->r_out ||
                          (d->n_flux > 0 && (!d->flux_idx || !d->flux_w || !d->flux_slot))))
        return fail(CS_ERR_ARG, "cs_step: null flux buffer");
    return CS_OK;
}

int launch_steps(const cs_step_desc* d, int a, int steps, cudaStream_t st) {
    const int block = d->block ? d->block : 256;
    const unsigned grid = unsigned(d->n > 0 ? ceil_div(d->n, block) : 1);
    StepFn fn = pick(*d);
    for (int s = 0; s < steps; ++s) {
        fn<<<grid, block, 0, st>>>(*d, a);
        CS_CHECK_LAUNCH("k_step");
        a = 1 - a;
    }
    return CS_OK;
}

// ---- link table packing -------------------------------------------------------------------------------------------
__global__ void k_links_encode(const int32_t* __restrict__ nbr, const float* __restrict__ q, int64_t n, int n_out,
                               int32_t* __restrict__ links, unsigned long long* __restrict__ status) {
    const int64_t total = n * Q;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
        const int32_t s = nbr[t];
        int32_t out = s;
        bool bad = false;
        if (s >= 0) {
            bad = s >= n;
        } else if (s == CS_WALL) {
            const float qq = q[t];
            const int32_t bits = __float_as_int(qq);
            bad = !(qq >= 0.0f && qq < 2.0f);      // -0.0 passes and is stored as +0.0
            out = int32_t(0x80000000u | uint32_t(bits & 0x3fffffff));
        } else if (s != CS_INLET) {
            bad = (CS_OUTLET0 - s) >= n_out;
        }
        if (bad) {
            out = CS_WALL;
            atomicAdd(status, 1ull);
            atomicMin(status + 1, (unsigned long long)t);
        }
        links[t] = out;
    }
}

__global__ void k_links_decode(const int32_t* __restrict__ links, int64_t n, int32_t* __restrict__ nbr,
                               float* __restrict__ q) {
    const int64_t total = n * Q;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
        const int32_t s = links[t];
        if (is_wall(s)) {
            nbr[t] = CS_WALL;
            q[t] = wall_q(s);
        } else {
            nbr[t] = s;
            q[t] = 0.5f;
        }
    }
}

__global__ void k_flux_blocks(const int32_t* __restrict__ idx, int64_t n_flux, int64_t n, int block,
                              int32_t* __restrict__ out, int64_t n_blocks) {
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

extern "C" int cs_links_encode(const int32_t* nbr, const float* q, int64_t n, int32_t n_out, int32_t* links,
                               int64_t* status, void* stream) {
    if (n < 0 || n >= (int64_t(1) << 30)) return fail(CS_ERR_SIZE, "cs_links_encode: n = %lld", (long long)n);
    if (n_out < 1) return fail(CS_ERR_ARG, "cs_links_encode: n_out %d", n_out);
    if (n == 0) return CS_OK;
    if (!nbr || !q || !links || !status) return fail(CS_ERR_ARG, "cs_links_encode: null buffer");
    cudaStream_t st = as_stream(stream);
    unsigned long long init[2] = {0ull, ~0ull};
    CS_CUDA(cudaMemcpyAsync(status, init, sizeof(init), cudaMemcpyHostToDevice, st));
    const unsigned grid = unsigned(std::min<int64_t>(ceil_div(n * Q, 256), 148 * 32));
    k_links_encode<<<grid, 256, 0, st>>>(nbr, q, n, n_out, links, reinterpret_cast<unsigned long long*>(status));
    CS_CHECK_LAUNCH("k_links_encode");
    unsigned long long res[2];
    CS_CUDA(cudaMemcpyAsync(res, status, sizeof(res), cudaMemcpyDeviceToHost, st));
    CS_CUDA(cudaStreamSynchronize(st));
    if (res[0]) {
        const long long t = (long long)res[1];
        return fail(CS_ERR_ARG, "cs_links_encode: %llu invalid entries; first at link %lld node %lld "
                    "(sources must be < N, outlet codes < n_out = %d, wall q finite in [0, 2))",
                    res[0], t / n, t % n, n_out);
    }
    return CS_OK;
}

extern "C" int cs_links_decode(const int32_t* links, int64_t n, int32_t* nbr, float* q, void* stream) {
    if (n < 0) return fail(CS_ERR_ARG, "cs_links_decode: n = %lld", (long long)n);
    if (n == 0) return CS_OK;
    if (!links || !nbr || !q) return fail(CS_ERR_ARG, "cs_links_decode: null buffer");
    const unsigned grid = unsigned(std::min<int64_t>(ceil_div(n * Q, 256), 148 * 32));
    k_links_decode<<<grid, 256, 0, as_stream(stream)>>>(links, n, nbr, q);
    CS_CHECK_LAUNCH("k_links_decode");
    return CS_OK;
}

extern "C" int cs_flux_blocks(const int32_t* flux_idx, int64_t n_flux, int64_t n, int32_t block, int32_t* out,
                              void* stream) {
    if (n < 0 || n_flux < 0 || block < 32 || block > MAX_BLOCK || !out || (n_flux > 0 && !flux_idx))
        return fail(CS_ERR_ARG, "cs_flux_blocks: bad arguments");
    const int64_t nb = n > 0 ? ceil_div(n, block) : 1;
    k_flux_blocks<<<unsigned(ceil_div(nb + 1, 256)), 256, 0, as_stream(stream)>>>(flux_idx, n_flux, n, block, out, nb);
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
