// CPU restatement of CerebroSim's lattice-Boltzmann step — TEST INFRASTRUCTURE (the oracle), never the product.
//
// Follows, in the reference's order of operations (left-to-right evaluation, summation over links i = 0..26):
//   k_clock   lbm.py:90-102    drive = Fourier series x start-up ramp; tick++
//   _ddx      lbm.py:105-126   non-uniform central difference of the previous step's velocity
//   _h3       lbm.py:129-137   third-order equilibrium term
//   k_step    lbm.py:140-257   pull streaming with wall / inlet / outlet links, moments + Guo force, Galilean
//                              correction, equilibrium inlet cells, regularised BGK (model 1) or TRT (model 0)
//   k_flux    simulate.py:65-69  slab flux Q[slot] += u . w   (summed in double here, sequentially)
//   k_bc      simulate.py:72-82  p_out[0] = drive; p_out[k] relaxed towards R_k Q_k - pref; Q reset
// Templated on the arithmetic type: float restates the reference's FP32 path, double is the FP64 oracle of the
// same scheme. Built with multiply-add contraction on (-ffp-contract=fast), as the reference's GPU compiler
// contracts by default; at tau ~ 0.505 the FP32 steady state depends on rounding at the 1e-4 level.
// OpenMP over nodes; each node is written by exactly one thread, so results do not depend on the thread count.
#include <cmath>
#include <cstdint>
#include <cstring>

namespace {

constexpr int Q = 27;
constexpr int WALL = -1, INLET = -2, OUTLET0 = -3;
// lbm.py:34-40: rest, +x -x +y -y +z -z, 12 edges, 8 corners (opposites adjacent)
constexpr int CX[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
constexpr int CY[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
constexpr int CZ[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
constexpr int OP[Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 20, 19, 22, 21, 24, 23, 26, 25};
constexpr double WD[Q] = {8.0 / 27, 2.0 / 27, 2.0 / 27, 2.0 / 27, 2.0 / 27, 2.0 / 27, 2.0 / 27,
                          1.0 / 54, 1.0 / 54, 1.0 / 54, 1.0 / 54, 1.0 / 54, 1.0 / 54, 1.0 / 54, 1.0 / 54,
                          1.0 / 54, 1.0 / 54, 1.0 / 54, 1.0 / 54,
                          1.0 / 216, 1.0 / 216, 1.0 / 216, 1.0 / 216, 1.0 / 216, 1.0 / 216, 1.0 / 216, 1.0 / 216};

template <class T> struct V3 { T x, y, z; };
template <class T> inline V3<T> vadd(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> vsub(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> vmul(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> smul(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline V3<T> cvec(int i) { return {T(CX[i]), T(CY[i]), T(CZ[i])}; }

}  // namespace

extern "C" {

// One layout for both precisions: `T` buffers are float for the FP32 oracle and double for the FP64 oracle.
typedef struct {
    int64_t N;
    int n_out;                 // outlet pressures stored
    void* f[2];                // populations (Q, N) T, stored as f - w (lbm.py:23)
    void* vel[2];              // velocity (N, 3) T
    void* rho;                 // density deviation (N,) T
    const int32_t* nbr;        // (Q, N) pull source or boundary code
    const float* q;            // (Q, N) wall fraction
    const float* uin;          // (N, 3) inlet profile
    const int32_t* inl;        // (N,) 1 for cells with an inlet link
    const void* om;            // (N,) T relaxation rate per cell
    void* p_out;               // (n_out,) T
    int32_t* tick;             // step counter
    void* drive;               // (1,) T drive value of the last step
    const void* coef;          // (2 nh + 1,) T Fourier coefficients
    int nh, period, ramp;
    double force[3];
    double magic, sigma;
    int bouzidi, model, gal;
    // simulate.ArterySolver coupling (n_open == 0: none)
    int64_t n_flux;
    const int32_t* flux_idx;
    const float* flux_w;       // (n_flux, 3)
    const int32_t* flux_slot;
    int n_open;
    double* q_acc;             // (n_open,)
    double* q_last;            // (n_open,)
    const float* r_out;        // (n_open,)
    double pref, alpha;
} oracle_args;

}  // extern "C"

namespace {

template <class T>
T clock_step(const oracle_args& a) {
    // lbm.py:94-102
    const T* coef = static_cast<const T*>(a.coef);
    int t = *a.tick;
    T ph = T(2.0) * T(M_PI) * T(t % a.period) / T(a.period);
    T d = coef[0];
    for (int k = 1; k <= a.nh; ++k)
        d += coef[2 * k - 1] * std::cos(T(k) * ph) + coef[2 * k] * std::sin(T(k) * ph);
    if (t < a.ramp) d *= T(0.5) - T(0.5) * std::cos(T(M_PI) * T(t) / T(a.ramp));
    static_cast<T*>(a.drive)[0] = d;
    *a.tick = t + 1;
    return d;
}

template <class T>
V3<T> ddx(const oracle_args& a, const V3<T>* vel, int64_t n, int im, int ip, V3<T> u0) {
    // lbm.py:105-126
    const int64_t N = a.N;
    T h1 = T(1.0);
    V3<T> v1 = u0;
    int s1 = a.nbr[im * N + n];
    if (s1 >= 0) {
        v1 = vel[s1];
    } else if (s1 == WALL) {
        h1 = std::max(T(a.q[im * N + n]), T(0.1));
        v1 = {T(0), T(0), T(0)};
    }
    T h2 = T(1.0);
    V3<T> v2 = u0;
    int s2 = a.nbr[ip * N + n];
    if (s2 >= 0) {
        v2 = vel[s2];
    } else if (s2 == WALL) {
        h2 = std::max(T(a.q[ip * N + n]), T(0.1));
        v2 = {T(0), T(0), T(0)};
    }
    V3<T> num = vadd(smul(h1 * h1, vsub(v2, u0)), smul(h2 * h2, vsub(u0, v1)));
    T den = h1 * h2 * (h1 + h2);
    return {num.x / den, num.y / den, num.z / den};
}

template <class T>
T h3(V3<T> c, V3<T> u) {
    // lbm.py:129-137
    T t = T(1.0) / T(3.0);
    return T(13.5) * ((c.x * c.x - t) * (c.y * u.x * u.x * u.y + c.z * u.x * u.x * u.z)
                      + (c.y * c.y - t) * (c.x * u.x * u.y * u.y + c.z * u.y * u.y * u.z)
                      + (c.z * c.z - t) * (c.x * u.x * u.z * u.z + c.y * u.y * u.z * u.z))
           + T(27.0) * c.x * c.y * c.z * u.x * u.y * u.z;
}

template <class T>
void node_step(const oracle_args& a, int src_buf, T d, int64_t n) {
    // lbm.py:146-257 for one node
    const int64_t N = a.N;
    const T* f_in = static_cast<const T*>(a.f[src_buf]);
    T* f_out = static_cast<T*>(a.f[1 - src_buf]);
    const V3<T>* vel_old = static_cast<const V3<T>*>(a.vel[src_buf]);
    V3<T>* vel = static_cast<V3<T>*>(a.vel[1 - src_buf]);
    T* rho = static_cast<T*>(a.rho);
    const T* p_out = static_cast<const T*>(a.p_out);
    T wq[Q];
    for (int i = 0; i < Q; ++i) wq[i] = T(WD[i]);

    T om_p = static_cast<const T*>(a.om)[n];
    T magic = T(a.magic);
    T om_m = T(1.0) / (T(0.5) + magic / (T(1.0) / om_p - T(0.5)));
    V3<T> force = {T(a.force[0]), T(a.force[1]), T(a.force[2])};
    V3<T> F = vmul(force, d);
    V3<T> up = vel_old[n];
    T upsq = dot(up, up);
    T f[Q];
    for (int i = 0; i < Q; ++i) {
        int src = a.nbr[i * N + n];
        int io = OP[i];
        T v = T(0.0);
        if (src >= 0) {
            v = f_in[i * N + src];
        } else if (src == WALL) {
            T fo = f_in[io * N + n];
            v = fo;
            if (a.bouzidi != 0) {
                T q = T(a.q[i * N + n]);
                if (q < T(0.5)) {
                    int m = a.nbr[io * N + n];
                    if (m >= 0) v = T(2.0) * q * fo + (T(1.0) - T(2.0) * q) * f_in[io * N + m];
                } else {
                    v = fo / (T(2.0) * q) + (T(2.0) * q - T(1.0)) / (T(2.0) * q) * f_in[i * N + n];
                }
            }
        } else if (src == INLET) {
            V3<T> uin = {T(a.uin[3 * n]), T(a.uin[3 * n + 1]), T(a.uin[3 * n + 2])};
            V3<T> uw = vmul(uin, d);
            T cu = T(CX[i]) * uw.x + T(CY[i]) * uw.y + T(CZ[i]) * uw.z;
            v = f_in[io * N + n] + T(6.0) * wq[i] * cu;
        } else {
            int k = OUTLET0 - src;
            T cu = T(CX[i]) * up.x + T(CY[i]) * up.y + T(CZ[i]) * up.z;
            v = -f_in[io * N + n] + T(2.0) * wq[i] * (T(3.0) * p_out[k] + T(4.5) * cu * cu - T(1.5) * upsq);
        }
        f[i] = v;
    }
    T dr = T(0.0);
    V3<T> j = {T(0), T(0), T(0)};
    for (int i = 0; i < Q; ++i) {
        dr += f[i];
        j = vadd(j, vmul(cvec<T>(i), f[i]));
    }
    V3<T> u = vadd(j, vmul(F, T(0.5)));
    T usq = dot(u, u);
    T uF = dot(u, F);
    T t3 = T(0.0);
    V3<T> Ed = {T(0), T(0), T(0)};
    if (a.gal != 0) {
        t3 = T(1.0);
        V3<T> gx = ddx<T>(a, vel_old, n, 1, 2, up);
        V3<T> gy = ddx<T>(a, vel_old, n, 3, 4, up);
        V3<T> gz = ddx<T>(a, vel_old, n, 5, 6, up);
        T tp = T(1.0) / om_p;
        Ed = {T(3.0) * tp * u.x * u.x * gx.x, T(3.0) * tp * u.y * u.y * gy.y, T(3.0) * tp * u.z * u.z * gz.z};
    }
    T mneg = -(T(1.0) - om_p);
    V3<T> Dd = smul(mneg, Ed);
    T trD = (Dd.x + Dd.y + Dd.z) / T(3.0);
    if (a.inl[n] != 0) {
        V3<T> uin = {T(a.uin[3 * n]), T(a.uin[3 * n + 1]), T(a.uin[3 * n + 2])};
        V3<T> ut = vmul(uin, d);
        T utsq = dot(ut, ut);
        for (int i = 0; i < Q; ++i) {
            V3<T> c0 = cvec<T>(i);
            T c0u = dot(c0, ut);
            f_out[i * N + n] = wq[i] * (dr + T(3.0) * c0u + T(4.5) * c0u * c0u - T(1.5) * utsq + t3 * h3(c0, ut));
        }
        vel[n] = ut;
        rho[n] = dr;
        return;
    }
    if (a.model == 1) {
        T P[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int i = 0; i < Q; ++i) {
            V3<T> c1 = cvec<T>(i);
            T c1u = dot(c1, u);
            T s = f[i] - wq[i] * (dr + T(3.0) * c1u + T(4.5) * c1u * c1u - T(1.5) * usq);
            T cc[3] = {c1.x, c1.y, c1.z};
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) P[r][c] += cc[r] * cc[c] * s;
        }
        T sigma = T(a.sigma);
        if (sigma < T(1.0)) {
            V3<T> g[3] = {ddx<T>(a, vel_old, n, 1, 2, up), ddx<T>(a, vel_old, n, 3, 4, up),
                          ddx<T>(a, vel_old, n, 5, 6, up)};
            T G[3][3] = {{g[0].x, g[0].y, g[0].z}, {g[1].x, g[1].y, g[1].z}, {g[2].x, g[2].y, g[2].z}};
            T s1 = (T(1.0) - sigma) / (T(3.0) * om_p);
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) P[r][c] = sigma * P[r][c] - s1 * (G[r][c] + G[c][r]);
        }
        P[0][0] -= Ed.x;
        P[1][1] -= Ed.y;
        P[2][2] -= Ed.z;
        T trP = (P[0][0] + P[1][1] + P[2][2]) / T(3.0);
        for (int i = 0; i < Q; ++i) {
            V3<T> c2 = cvec<T>(i);
            T c2u = dot(c2, u);
            T c2F = dot(c2, F);
            T feq = wq[i] * (dr + T(3.0) * c2u + T(4.5) * c2u * c2u - T(1.5) * usq + t3 * h3(c2, u));
            V3<T> Pc = {P[0][0] * c2.x + P[0][1] * c2.y + P[0][2] * c2.z,
                        P[1][0] * c2.x + P[1][1] * c2.y + P[1][2] * c2.z,
                        P[2][0] * c2.x + P[2][1] * c2.y + P[2][2] * c2.z};
            T fneq = wq[i] * (T(4.5) * (dot(c2, Pc) - trP) - T(1.5) * c2F);
            T src2 = wq[i] * (T(3.0) * c2F + T(9.0) * c2u * c2F - T(3.0) * uF);
            f_out[i * N + n] = feq + (T(1.0) - om_p) * fneq + (T(1.0) - T(0.5) * om_p) * src2;
        }
    } else {
        for (int i = 0; i < Q; ++i) {
            int jo = OP[i];
            V3<T> ci = cvec<T>(i);
            T cv = dot(ci, u);
            T cF = dot(ci, F);
            T eqp = wq[i] * (dr + T(4.5) * cv * cv - T(1.5) * usq);
            T eqm = wq[i] * (T(3.0) * cv + t3 * h3(ci, u));
            T psi = wq[i] * T(4.5) * (ci.x * ci.x * Dd.x + ci.y * ci.y * Dd.y + ci.z * ci.z * Dd.z - trD);
            T fp = T(0.5) * (f[i] + f[jo]);
            T fm = T(0.5) * (f[i] - f[jo]);
            T sp = wq[i] * (T(9.0) * cv * cF - T(3.0) * uF);
            T sm = wq[i] * T(3.0) * cF;
            f_out[i * N + n] = f[i] - om_p * (fp - eqp) - om_m * (fm - eqm) + (T(1.0) - T(0.5) * om_p) * sp
                               + (T(1.0) - T(0.5) * om_m) * sm + psi;
        }
    }
    vel[n] = u;
    rho[n] = dr;
}

template <class T>
void flux_bc(const oracle_args& a, int dst_buf, T d) {
    // simulate.py:65-82: flux over the slab cells of the velocity just written, then the outlet pressures
    const V3<T>* vel = static_cast<const V3<T>*>(a.vel[dst_buf]);
    for (int64_t t = 0; t < a.n_flux; ++t) {
        V3<T> w = {T(a.flux_w[3 * t]), T(a.flux_w[3 * t + 1]), T(a.flux_w[3 * t + 2])};
        a.q_acc[a.flux_slot[t]] += double(dot(vel[a.flux_idx[t]], w));
    }
    T* p_out = static_cast<T*>(a.p_out);
    p_out[0] = d;
    for (int k = 0; k < a.n_open; ++k) {
        a.q_last[k] = a.q_acc[k];
        if (k > 0) {
            T qk = T(a.q_acc[k]);
            p_out[k] = p_out[k] + T(a.alpha) * (T(a.r_out[k]) * qk - T(a.pref) - p_out[k]);
        }
        a.q_acc[k] = 0.0;
    }
}

template <class T>
int run(const oracle_args* ap, int a0, int steps) {
    const oracle_args& a = *ap;
    if (a.period <= 0) return 1;
    int buf = a0;
    for (int s = 0; s < steps; ++s) {
        T d = clock_step<T>(a);
#pragma omp parallel for schedule(static)
        for (int64_t n = 0; n < a.N; ++n) node_step<T>(a, buf, d, n);
        if (a.n_open > 0) flux_bc<T>(a, 1 - buf, d);
        buf = 1 - buf;
    }
    return 0;
}

}  // namespace

extern "C" {

int oracle_run_f32(const oracle_args* a, int a0, int steps) { return run<float>(a, a0, steps); }
int oracle_run_f64(const oracle_args* a, int a0, int steps) { return run<double>(a, a0, steps); }
int oracle_args_size(void) { return (int)sizeof(oracle_args); }

}  // extern "C"
