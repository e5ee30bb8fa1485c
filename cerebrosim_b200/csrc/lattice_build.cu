// Sparse lattice / neighbour-table builder on the GPU: the tables of lbm.build_lattice (lbm.py:264-330), bit-exact.
//
// Phase 1 (cs_lattice_count): tiles of 4096 grid cells count phi < 0, one block scans the tile counts, and each
// tile ranks its fluid cells in C order (warp ballots) into a dense rank grid (scratch), so node ids equal the
// reference's np.argwhere order (lbm.py:274-278).
// Phase 2 (cs_lattice_fill): coords from the rank grid; for every (link i, node n) the pull source x - c_i with
// periodic wrap (lbm.py:288-293); missing links are matched against the openings (inlets first, then outlets, first
// hit wins: lbm.py:294-306) and wall links get q = -phi_x / (phi_s - phi_x), clipped to [1e-3, 1], non-finite -> 0.5
// (lbm.py:307-316); the inlet profile of every cell with an inlet link comes from the LAST inlet (lbm.py:322-328).
// Floating-point steps use explicitly rounded intrinsics in the order NumPy evaluates them on the host that wrote
// the reference's tables: products and sums are separate roundings, and a row dot product `rel @ nrm` is
// fma(z, n2, fma(x, n0, y * n1)) (the BLAS gemv kernel) except when the batch holds a single row, where NumPy's
// plain dot gives fma(z, n2, fma(y, n1, x * n0)).
#include "cs_common.cuh"

namespace cs {
namespace {

constexpr int TILE_THREADS = 256;
constexpr int TILE_ROUNDS = 16;
constexpr int64_t TILE = TILE_THREADS * TILE_ROUNDS;
constexpr int MAX_OPENINGS = 32;

struct ScratchLayout {
    int64_t n_tiles;
    size_t off_rank, off_tile, off_misc, total;
};

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

ScratchLayout layout(int64_t nx, int64_t ny, int64_t nz) {
    ScratchLayout s;
    int64_t m = nx * ny * nz;
    s.n_tiles = ceil_div(m, TILE);
    s.off_rank = 0;
    s.off_tile = align256(size_t(m) * sizeof(int32_t));
    s.off_misc = s.off_tile + align256(size_t(s.n_tiles + 1) * sizeof(int64_t));
    s.total = s.off_misc + align256(64 * sizeof(int64_t));  // misc: [0] n_fluid, [1..27] misses, [28] inlet cells
    return s;
}

__global__ void k_tile_count(const float* __restrict__ phi, int64_t m, int64_t* __restrict__ tile_cnt) {
    __shared__ int warp_sum[TILE_THREADS / 32];
    int64_t base = int64_t(blockIdx.x) * TILE;
    int cnt = 0;
    for (int r = 0; r < TILE_ROUNDS; ++r) {
        int64_t c = base + int64_t(r) * TILE_THREADS + threadIdx.x;
        if (c < m && phi[c] < 0.0f) ++cnt;
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t t = 0;
        for (int w = 0; w < TILE_THREADS / 32; ++w) t += warp_sum[w];
        tile_cnt[blockIdx.x] = t;
    }
}

// Exclusive scan of the tile counts by one block (tile_cnt[n_tiles] receives the total).
__global__ void k_tile_scan(int64_t* __restrict__ tile_cnt, int64_t n_tiles, int64_t* __restrict__ n_fluid) {
    __shared__ int64_t part[1024];
    int64_t per = ceil_div(n_tiles, blockDim.x);
    int64_t lo = threadIdx.x * per, hi = min(lo + per, n_tiles);
    int64_t s = 0;
    for (int64_t t = lo; t < hi; ++t) s += tile_cnt[t];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t run = 0;
        for (int k = 0; k < (int)blockDim.x; ++k) {
            int64_t v = part[k];
            part[k] = run;
            run += v;
        }
        *n_fluid = run;
        tile_cnt[n_tiles] = run;
    }
    __syncthreads();
    int64_t run = part[threadIdx.x];
    for (int64_t t = lo; t < hi; ++t) {
        int64_t v = tile_cnt[t];
        tile_cnt[t] = run;
        run += v;
    }
}

__global__ void k_tile_rank(const float* __restrict__ phi, int64_t m, const int64_t* __restrict__ tile_off,
                            int32_t* __restrict__ rank) {
    __shared__ int warp_cnt[TILE_THREADS / 32];
    __shared__ int64_t run;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) run = tile_off[blockIdx.x];
    int64_t base = int64_t(blockIdx.x) * TILE;
    for (int r = 0; r < TILE_ROUNDS; ++r) {
        int64_t c = base + int64_t(r) * TILE_THREADS + threadIdx.x;
        bool fl = c < m && phi[c] < 0.0f;
        unsigned mask = __ballot_sync(0xffffffffu, fl);
        if (lane == 0) warp_cnt[warp] = __popc(mask);
        __syncthreads();
        int64_t before = run;
        for (int w = 0; w < warp; ++w) before += warp_cnt[w];
        if (c < m) rank[c] = fl ? int32_t(before + __popc(mask & ((1u << lane) - 1u))) : -1;
        __syncthreads();
        if (threadIdx.x == 0) {
            int64_t t = 0;
            for (int w = 0; w < TILE_THREADS / 32; ++w) t += warp_cnt[w];
            run += t;
        }
        __syncthreads();
    }
}

__global__ void k_coords(const int32_t* __restrict__ rank, int64_t nx, int64_t ny, int64_t nz,
                         int32_t* __restrict__ coords) {
    int64_t m = nx * ny * nz;
    for (int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; c < m; c += int64_t(gridDim.x) * blockDim.x) {
        int32_t r = rank[c];
        if (r >= 0) {
            int64_t k = c % nz, j = (c / nz) % ny, i = c / (ny * nz);
            coords[3 * int64_t(r)] = int32_t(i);
            coords[3 * int64_t(r) + 1] = int32_t(j);
            coords[3 * int64_t(r) + 2] = int32_t(k);
        }
    }
}

struct OpeningSet {
    int n;                       // openings in claim order (inlets, then outlets)
    int last_inlet;              // index of the last inlet, -1 if none
    int code[MAX_OPENINGS];      // INLET or OUTLET0 - k
    double c[MAX_OPENINGS][3];
    double nrm[MAX_OPENINGS][3];
    double lim[MAX_OPENINGS];    // radius + slack * dx
    double radius[MAX_OPENINGS];
};

struct Grid {
    int64_t dims[3];
    int periodic;
    double origin[3];
    double dx;
};

__device__ inline int64_t wrap(int64_t x, int64_t s) { return ((x % s) + s) % s; }

// Source cell of link i at node n: fills xyz, returns true when inside the grid.
__device__ inline bool source_cell(const Grid& g, const int32_t* coords, int64_t n, int i, int64_t xyz[3]) {
    const int cc[3] = {Lat::cx(i), Lat::cy(i), Lat::cz(i)};
    bool inside = true;
    for (int a = 0; a < 3; ++a) {
        int64_t v = int64_t(coords[3 * n + a]) - cc[a];
        if ((g.periodic >> a) & 1) v = wrap(v, g.dims[a]);
        xyz[a] = v;
        inside = inside && v >= 0 && v < g.dims[a];
    }
    return inside;
}

// Pass A: pull sources; count missing links per direction (len(miss) at lbm.py:294).
__global__ void k_links_src(Grid g, const int32_t* __restrict__ coords, const int32_t* __restrict__ rank,
                            int64_t n_fl, int32_t* __restrict__ nbr, float* __restrict__ q,
                            int64_t* __restrict__ misses) {
    __shared__ int miss_blk[Q];
    if (threadIdx.x < Q) miss_blk[threadIdx.x] = 0;
    __syncthreads();
    int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (t < n_fl * Q) {
        int i = int(t / n_fl);
        int64_t n = t - int64_t(i) * n_fl;
        int64_t xyz[3];
        int32_t src = CS_WALL;
        if (source_cell(g, coords, n, i, xyz)) src = rank[(xyz[0] * g.dims[1] + xyz[1]) * g.dims[2] + xyz[2]];
        if (src < 0) {
            src = CS_WALL;
            atomicAdd(&miss_blk[i], 1);
        }
        nbr[t] = src;
        q[t] = 0.5f;
    }
    __syncthreads();
    if (threadIdx.x < Q && miss_blk[threadIdx.x]) atomicAdd((unsigned long long*)&misses[threadIdx.x],
                                                            (unsigned long long)miss_blk[threadIdx.x]);
}

__device__ inline double row_dot(double x, double y, double z, const double* nv, bool single_row) {
    if (single_row) return __fma_rn(z, nv[2], __fma_rn(y, nv[1], __dmul_rn(x, nv[0])));
    return __fma_rn(z, nv[2], __fma_rn(x, nv[0], __dmul_rn(y, nv[1])));
}

// Axial coordinate and distance from the opening's axis of point p (lbm.py:301-303).
__device__ inline void axial_lateral(const double p[3], const double* c, const double* nv, bool single_row,
                                     double* ax, double* lat) {
    double r0 = __dsub_rn(p[0], c[0]), r1 = __dsub_rn(p[1], c[1]), r2 = __dsub_rn(p[2], c[2]);
    double a = row_dot(r0, r1, r2, nv, single_row);
    double v0 = __dsub_rn(r0, __dmul_rn(a, nv[0]));
    double v1 = __dsub_rn(r1, __dmul_rn(a, nv[1]));
    double v2 = __dsub_rn(r2, __dmul_rn(a, nv[2]));
    *ax = a;
    *lat = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(v0, v0), __dmul_rn(v1, v1)), __dmul_rn(v2, v2)));
}

// Pass B: classify missing links, wall q, link counts.
__global__ void k_links_classify(Grid g, OpeningSet os, const float* __restrict__ phi,
                                 const int32_t* __restrict__ coords, int64_t n_fl, const int64_t* __restrict__ misses,
                                 int32_t* __restrict__ nbr, float* __restrict__ q, int64_t* __restrict__ counts,
                                 int n_outlets) {
    __shared__ unsigned long long cnt_blk[2 + MAX_OPENINGS];
    for (int k = threadIdx.x; k < 2 + MAX_OPENINGS; k += blockDim.x) cnt_blk[k] = 0;
    __syncthreads();
    int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (t < n_fl * Q && nbr[t] < 0) {
        int i = int(t / n_fl);
        int64_t n = t - int64_t(i) * n_fl;
        int64_t xyz[3];
        bool inside = source_cell(g, coords, n, i, xyz);
        bool single = misses[i] == 1;
        double p[3];
        for (int a = 0; a < 3; ++a) p[a] = __dadd_rn(g.origin[a], __dmul_rn(double(xyz[a]), g.dx));
        int32_t code = CS_WALL;
        for (int o = 0; o < os.n; ++o) {
            double ax, lat;
            axial_lateral(p, os.c[o], os.nrm[o], single, &ax, &lat);
            if (ax >= -1e-6 && lat < os.lim[o]) {
                code = os.code[o];
                break;
            }
        }
        nbr[t] = code;
        if (code == CS_WALL) {
            int64_t m_here = (int64_t(coords[3 * n]) * g.dims[1] + coords[3 * n + 1]) * g.dims[2] + coords[3 * n + 2];
            float px = phi[m_here];
            float ps = __int_as_float(0x7fc00000);  // NaN outside the grid
            if (inside) ps = phi[(xyz[0] * g.dims[1] + xyz[1]) * g.dims[2] + xyz[2]];
            float qq = __fdiv_rn(-px, __fsub_rn(ps, px));
            q[t] = isfinite(qq) ? fminf(fmaxf(qq, 0.001f), 1.0f) : 0.5f;
            atomicAdd(&cnt_blk[0], 1ull);
        } else if (code == CS_INLET) {
            atomicAdd(&cnt_blk[1], 1ull);
        } else {
            atomicAdd(&cnt_blk[2 + (CS_OUTLET0 - code)], 1ull);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < 2 + n_outlets; k += blockDim.x)
        if (cnt_blk[k]) atomicAdd((unsigned long long*)&counts[k], cnt_blk[k]);
}

__global__ void k_inlet_cells(const int32_t* __restrict__ nbr, int64_t n_fl, int64_t* __restrict__ n_inlet_cells,
                              float* __restrict__ uin) {
    int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (n >= n_fl) return;
    bool any = false;
    for (int i = 0; i < Q; ++i) any = any || nbr[int64_t(i) * n_fl + n] == CS_INLET;
    uin[3 * n] = 0.0f;
    uin[3 * n + 1] = 0.0f;
    uin[3 * n + 2] = 0.0f;
    if (any) atomicAdd((unsigned long long*)n_inlet_cells, 1ull);
}

__global__ void k_inlet_profile(Grid g, OpeningSet os, const int32_t* __restrict__ nbr,
                                const int32_t* __restrict__ coords, int64_t n_fl,
                                const int64_t* __restrict__ n_inlet_cells, float* __restrict__ uin) {
    int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (n >= n_fl || os.last_inlet < 0) return;
    bool any = false;
    for (int i = 0; i < Q; ++i) any = any || nbr[int64_t(i) * n_fl + n] == CS_INLET;
    if (!any) return;
    const int o = os.last_inlet;
    double p[3];
    for (int a = 0; a < 3; ++a) p[a] = __dadd_rn(g.origin[a], __dmul_rn(double(coords[3 * n + a]), g.dx));
    double ax, lat;
    axial_lateral(p, os.c[o], os.nrm[o], *n_inlet_cells == 1, &ax, &lat);
    double r = __ddiv_rn(lat, os.radius[o]);
    double prof = __dmul_rn(2.0, __dsub_rn(1.0, __dmul_rn(r, r)));
    prof = prof < 0.0 ? 0.0 : prof;  // np.clip(., 0, None): NaN stays NaN
    for (int a = 0; a < 3; ++a) uin[3 * n + a] = __double2float_rn(__dmul_rn(-prof, os.nrm[o][a]));
}

}  // namespace
}  // namespace cs

using namespace cs;

extern "C" size_t cs_lattice_scratch_bytes(int64_t nx, int64_t ny, int64_t nz) {
    if (nx < 0 || ny < 0 || nz < 0) return 0;
    return layout(nx, ny, nz).total;
}

extern "C" int cs_lattice_count(const float* phi, int64_t nx, int64_t ny, int64_t nz, void* scratch,
                                int64_t* n_fluid, void* stream) {
    if (nx < 0 || ny < 0 || nz < 0 || !n_fluid) return fail(CS_ERR_ARG, "cs_lattice_count: bad grid or output");
    int64_t m = nx * ny * nz;
    if (m > 0 && (!phi || !scratch)) return fail(CS_ERR_ARG, "cs_lattice_count: null phi or scratch");
    if (m > (int64_t(1) << 40)) return fail(CS_ERR_SIZE, "cs_lattice_count: grid of %lld cells", (long long)m);
    ScratchLayout L = layout(nx, ny, nz);
    cudaStream_t st = as_stream(stream);
    char* s = static_cast<char*>(scratch);
    int64_t* tile = reinterpret_cast<int64_t*>(s + L.off_tile);
    int64_t* misc = reinterpret_cast<int64_t*>(s + L.off_misc);
    CS_CUDA(cudaMemsetAsync(misc, 0, 64 * sizeof(int64_t), st));
    if (m > 0) {
        k_tile_count<<<unsigned(L.n_tiles), TILE_THREADS, 0, st>>>(phi, m, tile);
        CS_CHECK_LAUNCH("k_tile_count");
        k_tile_scan<<<1, 1024, 0, st>>>(tile, L.n_tiles, misc);
        CS_CHECK_LAUNCH("k_tile_scan");
        k_tile_rank<<<unsigned(L.n_tiles), TILE_THREADS, 0, st>>>(phi, m, tile,
                                                                    reinterpret_cast<int32_t*>(s + L.off_rank));
        CS_CHECK_LAUNCH("k_tile_rank");
    }
    int64_t nf = 0;
    CS_CUDA(cudaMemcpyAsync(&nf, misc, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CS_CUDA(cudaStreamSynchronize(st));
    if (nf >= (int64_t(1) << 30))
        return fail(CS_ERR_SIZE, "cs_lattice_count: %lld fluid nodes (node ids are int32 < 2^30)", (long long)nf);
    *n_fluid = nf;
    return CS_OK;
}

extern "C" int cs_lattice_fill(const float* phi, int64_t nx, int64_t ny, int64_t nz, const double* origin,
                               double dx, const cs_opening* openings, int32_t n_openings, int32_t periodic_mask,
                               double opening_slack, void* scratch, int64_t n_fluid, int32_t* nbr, float* q,
                               float* uin, int32_t* coords, int64_t* counts, void* stream) {
    if (nx < 0 || ny < 0 || nz < 0 || n_fluid < 0 || !origin) return fail(CS_ERR_ARG, "cs_lattice_fill: bad arguments");
    if (n_openings < 0 || n_openings > MAX_OPENINGS)
        return fail(CS_ERR_SIZE, "cs_lattice_fill: %d openings (at most %d)", n_openings, MAX_OPENINGS);
    if (n_openings > 0 && !openings) return fail(CS_ERR_ARG, "cs_lattice_fill: null openings");
    if (!counts) return fail(CS_ERR_ARG, "cs_lattice_fill: null counts");
    OpeningSet os{};
    int n_out = 0;
    os.last_inlet = -1;
    for (int pass = 0; pass < 2; ++pass) {          // inlets first, then outlets (lbm.py:298)
        for (int k = 0; k < n_openings; ++k) {
            const cs_opening& o = openings[k];
            if (o.kind != 0 && o.kind != 1) return fail(CS_ERR_ARG, "cs_lattice_fill: opening %d kind %d", k, o.kind);
            if (o.kind != pass) continue;
            int idx = os.n++;
            os.code[idx] = pass == 0 ? CS_INLET : CS_OUTLET0 - n_out++;
            if (pass == 0) os.last_inlet = idx;
            for (int a = 0; a < 3; ++a) {
                os.c[idx][a] = o.centre[a];
                os.nrm[idx][a] = o.normal[a];
            }
            os.lim[idx] = o.radius + opening_slack * dx;
            os.radius[idx] = o.radius;
        }
    }
    cudaStream_t st = as_stream(stream);
    CS_CUDA(cudaMemsetAsync(counts, 0, size_t(2 + n_out) * sizeof(int64_t), st));
    if (n_fluid == 0) return CS_OK;
    if (!phi || !scratch || !nbr || !q || !uin || !coords) return fail(CS_ERR_ARG, "cs_lattice_fill: null buffer");
    ScratchLayout L = layout(nx, ny, nz);
    char* s = static_cast<char*>(scratch);
    const int32_t* rank = reinterpret_cast<const int32_t*>(s + L.off_rank);
    int64_t* misc = reinterpret_cast<int64_t*>(s + L.off_misc);
    Grid g{{nx, ny, nz}, periodic_mask & 7, {origin[0], origin[1], origin[2]}, dx};
    int64_t m = nx * ny * nz;
    k_coords<<<unsigned(std::min<int64_t>(ceil_div(m, 256), 148 * 64)), 256, 0, st>>>(rank, nx, ny, nz, coords);
    CS_CHECK_LAUNCH("k_coords");
    int64_t links = n_fluid * Q;
    unsigned nb = unsigned(ceil_div(links, 256));
    k_links_src<<<nb, 256, 0, st>>>(g, coords, rank, n_fluid, nbr, q, misc + 1);
    CS_CHECK_LAUNCH("k_links_src");
    k_links_classify<<<nb, 256, 0, st>>>(g, os, phi, coords, n_fluid, misc + 1, nbr, q, counts, n_out);
    CS_CHECK_LAUNCH("k_links_classify");
    unsigned nbn = unsigned(ceil_div(n_fluid, 256));
    k_inlet_cells<<<nbn, 256, 0, st>>>(nbr, n_fluid, misc + 28, uin);
    CS_CHECK_LAUNCH("k_inlet_cells");
    if (os.last_inlet >= 0) {
        k_inlet_profile<<<nbn, 256, 0, st>>>(g, os, nbr, coords, n_fluid, misc + 28, uin);
        CS_CHECK_LAUNCH("k_inlet_profile");
    }
    return CS_OK;
}

// ---- sponge (lbm.py:398-416) --------------------------------------------------------------------------------------
// Per-cell relaxation near the openings, in the reference's float64 order of operations and rounding: tau_cell = max
// over the chosen openings of tau + (tau_max - tau) * smoothstep(clip(1 - depth / length, 0, 1)) where the cell is
// within 1.5 radii of the opening's axis, depth = -axial / dx; om = float32(1 / tau_cell). The reference's cell
// positions come from np.argwhere, a column-major (N, 3) array, and NumPy's `rel @ nrm` on it evaluates, on the host
// that wrote the fixtures, fma(x, n0, y * n1) + z * n2 for all rows but the last N mod 4, and fma(z, n2, fma(y, n1,
// x * n0)) for those (the column-major BLAS kernel's blocks of four rows and its remainder).
namespace cs {
namespace {

struct SpongeSet {
    int n;
    double c[MAX_OPENINGS][3];
    double nrm[MAX_OPENINGS][3];
    double reach[MAX_OPENINGS];   // 1.5 radius
};

__global__ void k_sponge(const int32_t* __restrict__ coords, int64_t n, double o0, double o1, double o2, double dx,
                         SpongeSet ss, double tau, double length, double tau_max, float* __restrict__ om,
                         double* __restrict__ tau_out) {
    const int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (k >= n) return;
    const double origin[3] = {o0, o1, o2};
    double p[3];
    for (int a = 0; a < 3; ++a) p[a] = __dadd_rn(origin[a], __dmul_rn(double(coords[3 * k + a]), dx));
    const bool tail = k >= n - n % 4;
    double out = tau;
    for (int j = 0; j < ss.n; ++j) {
        const double* nv = ss.nrm[j];
        const double r0 = __dsub_rn(p[0], ss.c[j][0]), r1 = __dsub_rn(p[1], ss.c[j][1]);
        const double r2 = __dsub_rn(p[2], ss.c[j][2]);
        const double ax = tail ? __fma_rn(r2, nv[2], __fma_rn(r1, nv[1], __dmul_rn(r0, nv[0])))
                               : __dadd_rn(__fma_rn(r0, nv[0], __dmul_rn(r1, nv[1])), __dmul_rn(r2, nv[2]));
        const double v0 = __dsub_rn(r0, __dmul_rn(ax, nv[0]));
        const double v1 = __dsub_rn(r1, __dmul_rn(ax, nv[1]));
        const double v2 = __dsub_rn(r2, __dmul_rn(ax, nv[2]));
        const double lat = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(v0, v0), __dmul_rn(v1, v1)), __dmul_rn(v2, v2)));
        const double depth = __ddiv_rn(-ax, dx);
        double w = __dsub_rn(1.0, __ddiv_rn(depth, length));
        w = w < 0.0 ? 0.0 : (w > 1.0 ? 1.0 : w);
        w = __dmul_rn(__dmul_rn(w, w), __dsub_rn(3.0, __dmul_rn(2.0, w)));
        const double v = lat < ss.reach[j] ? __dadd_rn(tau, __dmul_rn(__dsub_rn(tau_max, tau), w)) : tau;
        out = v > out ? v : out;
    }
    om[k] = __double2float_rn(__ddiv_rn(1.0, out));
    if (tau_out) tau_out[k] = out;
}

}  // namespace
}  // namespace cs

extern "C" int cs_sponge_om(const int32_t* coords, int64_t n, const double* origin, double dx,
                            const cs_opening* openings, int32_t n_openings, int32_t kinds_mask, double tau,
                            double length, double tau_max, float* om, double* tau_out, void* stream) {
    if (n < 0 || !origin || !(dx > 0.0) || !(length > 0.0) || (kinds_mask & ~3))
        return fail(CS_ERR_ARG, "cs_sponge_om: bad arguments");
    if (n_openings < 0 || n_openings > MAX_OPENINGS)
        return fail(CS_ERR_SIZE, "cs_sponge_om: %d openings (at most %d)", n_openings, MAX_OPENINGS);
    if (n_openings > 0 && !openings) return fail(CS_ERR_ARG, "cs_sponge_om: null openings");
    SpongeSet ss{};
    for (int k = 0; k < n_openings; ++k) {
        const cs_opening& o = openings[k];
        if (o.kind != 0 && o.kind != 1) return fail(CS_ERR_ARG, "cs_sponge_om: opening %d kind %d", k, o.kind);
        if (!(kinds_mask & (1 << o.kind))) continue;
        const int j = ss.n++;
        for (int a = 0; a < 3; ++a) {
            ss.c[j][a] = o.centre[a];
            ss.nrm[j][a] = o.normal[a];
        }
        ss.reach[j] = 1.5 * o.radius;             // one IEEE product, as NumPy
    }
    if (n == 0) return CS_OK;
    if (!coords || !om) return fail(CS_ERR_ARG, "cs_sponge_om: null buffer");
    k_sponge<<<unsigned(ceil_div(n, 256)), 256, 0, as_stream(stream)>>>(coords, n, origin[0], origin[1], origin[2], dx,
                                                                      ss, tau, length, tau_max, om, tau_out);
    CS_CHECK_LAUNCH("k_sponge");
    return CS_OK;
}
