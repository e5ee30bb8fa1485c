// Link tables of the step: the reference's nbr / q tables (lbm.py:280-321) turned into branch-free pull sources plus
// per-direction ghost-slot lists of the boundary links (wall, inlet, outlet).
//
// Count: tiles of 4096 nodes count the boundary links of each direction (27 x tiles), one block per direction scans
// them. Fill: each tile ranks its boundary links in node order with warp ballots, so ghost slot g of direction i is
// the g-th boundary link of that direction in node order; the link code becomes n + g, and the slot records the
// node, the wall's second node (the Bouzidi interpolation partner, nbr[opp(i)][node], lbm.py:169) or the opening
// code, and q.
#include "cs_common.cuh"

namespace cs {
namespace {

constexpr int T_THREADS = 256;
constexpr int T_ROUNDS = 16;
constexpr int64_t T_NODES = T_THREADS * T_ROUNDS;

struct Layout {
    int64_t tiles;
    size_t total;
};

Layout layout(int64_t n) {
    Layout l;
    l.tiles = ceil_div(n, T_NODES);
    l.total = size_t(Q) * size_t(l.tiles + 1) * sizeof(int64_t) + 256;
    return l;
}

__global__ void k_ghost_count(const int32_t* __restrict__ nbr, int64_t n, int64_t tiles, int64_t* __restrict__ part) {
    __shared__ int wsum[T_THREADS / 32];
    const int i = blockIdx.y;
    const int64_t base = int64_t(blockIdx.x) * T_NODES;
    int cnt = 0;
    for (int r = 0; r < T_ROUNDS; ++r) {
        const int64_t v = base + int64_t(r) * T_THREADS + threadIdx.x;
        if (v < n && nbr[int64_t(i) * n + v] < 0) ++cnt;
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t t = 0;
        for (int w = 0; w < T_THREADS / 32; ++w) t += wsum[w];
        part[int64_t(i) * (tiles + 1) + blockIdx.x] = t;
    }
}

// Exclusive scan of one direction's tile counts (block i); the total lands in part[i][tiles].
__global__ void k_ghost_scan(int64_t* __restrict__ part, int64_t tiles) {
    __shared__ int64_t s[1024];
    int64_t* p = part + int64_t(blockIdx.x) * (tiles + 1);
    const int64_t per = ceil_div(tiles, blockDim.x);
    const int64_t lo = threadIdx.x * per, hi = min(lo + per, tiles);
    int64_t sum = 0;
    for (int64_t t = lo; t < hi; ++t) sum += p[t];
    s[threadIdx.x] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t run = 0;
        for (int k = 0; k < (int)blockDim.x; ++k) {
            const int64_t v = s[k];
            s[k] = run;
            run += v;
        }
        p[tiles] = run;
    }
    __syncthreads();
    int64_t run = s[threadIdx.x];
    for (int64_t t = lo; t < hi; ++t) {
        const int64_t v = p[t];
        p[t] = run;
        run += v;
    }
}

__global__ void k_ghost_fill(const int32_t* __restrict__ nbr, const float* __restrict__ q, int64_t n, int n_out,
                             int64_t gmax, int64_t tiles, const int64_t* __restrict__ part,
                             int32_t* __restrict__ links, int32_t* __restrict__ gnode, int32_t* __restrict__ ginfo,
                             float* __restrict__ gq, unsigned long long* __restrict__ status) {
    __shared__ int wcnt[T_THREADS / 32];
    __shared__ int64_t run;
    const int i = blockIdx.y;
    const int io = Lat::opp(i);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) run = part[int64_t(i) * (tiles + 1) + blockIdx.x];
    const int64_t base = int64_t(blockIdx.x) * T_NODES;
    for (int r = 0; r < T_ROUNDS; ++r) {
        const int64_t v = base + int64_t(r) * T_THREADS + threadIdx.x;
        const int64_t t = int64_t(i) * n + v;
        const int32_t s = v < n ? nbr[t] : 0;
        const bool boundary = v < n && s < 0;
        const unsigned mask = __ballot_sync(0xffffffffu, boundary);
        if (lane == 0) wcnt[warp] = __popc(mask);
        __syncthreads();
        int64_t g = run;
        for (int w = 0; w < warp; ++w) g += wcnt[w];
        g += __popc(mask & ((1u << lane) - 1u));
        if (v < n) {
            bool bad = false;
            if (!boundary) {
                bad = s >= n;
                links[t] = bad ? int32_t(v) : s;
            } else if (g >= gmax) {                 // caller's gmax below this direction's count
                bad = true;
                links[t] = int32_t(v);
            } else {
                links[t] = int32_t(n + g);
                const int64_t slot = int64_t(i) * gmax + g;
                gnode[slot] = int32_t(v);
                if (s == CS_WALL) {
                    const float qq = q[t];
                    bad = !(qq >= 0.0f) || !isfinite(qq);
                    const int32_t m = nbr[int64_t(io) * n + v];
                    ginfo[slot] = m >= 0 && m < n ? m : -1;
                    gq[slot] = qq;
                } else {
                    bad = s != CS_INLET && (CS_OUTLET0 - s) >= n_out;
                    ginfo[slot] = bad ? CS_WALL : s;
                    gq[slot] = bad ? 0.5f : -1.0f;
                }
            }
            if (bad) {
                atomicAdd(status, 1ull);
                atomicMin(status + 1, (unsigned long long)t);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int64_t a = 0;
            for (int w = 0; w < T_THREADS / 32; ++w) a += wcnt[w];
            run += a;
        }
        __syncthreads();
    }
}

__global__ void k_links_decode(const int32_t* __restrict__ links, const int32_t* __restrict__ ginfo,
                               const float* __restrict__ gq, int64_t n, int64_t gmax, int32_t* __restrict__ nbr,
                               float* __restrict__ q) {
    const int64_t total = n * Q;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
        const int i = int(t / n);
        const int32_t s = links[t];
        if (s < n) {
            nbr[t] = s;
            q[t] = 0.5f;
        } else {
            const int64_t slot = int64_t(i) * gmax + (s - n);
            const int32_t info = ginfo[slot];
            nbr[t] = info >= -1 ? CS_WALL : info;
            q[t] = info >= -1 ? gq[slot] : 0.5f;
        }
    }
}

}  // namespace
}  // namespace cs

using namespace cs;

extern "C" size_t cs_links_scratch_bytes(int64_t n) { return n < 0 ? 0 : layout(n).total; }

extern "C" int cs_links_count(const int32_t* nbr, int64_t n, void* scratch, int64_t* ghosts, void* stream) {
    if (n < 0 || n >= (int64_t(1) << 30)) return fail(CS_ERR_SIZE, "cs_links_count: n = %lld", (long long)n);
    if (!ghosts) return fail(CS_ERR_ARG, "cs_links_count: null ghosts");
    for (int i = 0; i < Q; ++i) ghosts[i] = 0;
    if (n == 0) return CS_OK;
    if (!nbr || !scratch) return fail(CS_ERR_ARG, "cs_links_count: null buffer");
    const Layout l = layout(n);
    cudaStream_t st = as_stream(stream);
    int64_t* part = static_cast<int64_t*>(scratch);
    k_ghost_count<<<dim3(unsigned(l.tiles), Q), T_THREADS, 0, st>>>(nbr, n, l.tiles, part);
    CS_CHECK_LAUNCH("k_ghost_count");
    k_ghost_scan<<<Q, 1024, 0, st>>>(part, l.tiles);
    CS_CHECK_LAUNCH("k_ghost_scan");
    for (int i = 0; i < Q; ++i)
        CS_CUDA(cudaMemcpyAsync(ghosts + i, part + int64_t(i) * (l.tiles + 1) + l.tiles, sizeof(int64_t),
                                cudaMemcpyDeviceToHost, st));
    CS_CUDA(cudaStreamSynchronize(st));
    return CS_OK;
}

extern "C" int cs_links_fill(const int32_t* nbr, const float* q, int64_t n, int32_t n_out, int64_t gmax,
                             void* scratch, int32_t* links, int32_t* gnode, int32_t* ginfo, float* gq,
                             int64_t* status, void* stream) {
    if (n < 0 || n >= (int64_t(1) << 30) || gmax < 0) return fail(CS_ERR_SIZE, "cs_links_fill: n %lld gmax %lld",
                                                                  (long long)n, (long long)gmax);
    if (int64_t(Q) * (n + gmax) >= (int64_t(1) << 31))
        return fail(CS_ERR_SIZE, "cs_links_fill: 27 * (n + gmax) = %lld exceeds 2^31", (long long)(Q * (n + gmax)));
    if (n_out < 1) return fail(CS_ERR_ARG, "cs_links_fill: n_out %d", n_out);
    if (n == 0) return CS_OK;
    if (!nbr || !q || !scratch || !links || !status || (gmax > 0 && (!gnode || !ginfo || !gq)))
        return fail(CS_ERR_ARG, "cs_links_fill: null buffer");
    const Layout l = layout(n);
    cudaStream_t st = as_stream(stream);
    unsigned long long init[2] = {0ull, ~0ull};
    CS_CUDA(cudaMemcpyAsync(status, init, sizeof(init), cudaMemcpyHostToDevice, st));
    k_ghost_fill<<<dim3(unsigned(l.tiles), Q), T_THREADS, 0, st>>>(nbr, q, n, n_out, gmax, l.tiles,
                                                                   static_cast<const int64_t*>(scratch), links, gnode,
                                                                   ginfo, gq,
                                                                   reinterpret_cast<unsigned long long*>(status));
    CS_CHECK_LAUNCH("k_ghost_fill");
    unsigned long long res[2];
    CS_CUDA(cudaMemcpyAsync(res, status, sizeof(res), cudaMemcpyDeviceToHost, st));
    CS_CUDA(cudaStreamSynchronize(st));
    if (res[0]) {
        const long long t = (long long)res[1];
        return fail(CS_ERR_ARG, "cs_links_fill: %llu invalid entries; first at link %lld node %lld (sources must be "
                    "< N, outlet codes < n_out = %d, wall q finite and >= 0)", res[0], t / n, t % n, n_out);
    }
    return CS_OK;
}

extern "C" int cs_links_decode(const int32_t* links, const int32_t* ginfo, const float* gq, int64_t n, int64_t gmax,
                               int32_t* nbr, float* q, void* stream) {
    if (n < 0 || gmax < 0) return fail(CS_ERR_ARG, "cs_links_decode: n %lld gmax %lld", (long long)n, (long long)gmax);
    if (n == 0) return CS_OK;
    if (!links || !nbr || !q || (gmax > 0 && (!ginfo || !gq))) return fail(CS_ERR_ARG, "cs_links_decode: null buffer");
    const unsigned grid = unsigned(std::min<int64_t>(ceil_div(n * Q, 256), 148 * 32));
    k_links_decode<<<grid, 256, 0, as_stream(stream)>>>(links, ginfo, gq, n, gmax, nbr, q);
    CS_CHECK_LAUNCH("k_links_decode");
    return CS_OK;
}

// ---- link-table build that allocates nothing --------------------------------------------------------------------
// The scratch of cs_links_count / cs_links_fill (per-tile ghost counts and offsets, two status words) lives here, in
// memory the library owns, instead of in a caller's buffer. Every GPU that loads the library holds this array until
// the process exits. Every call shares it: the tile sums are rewritten and the status words reset by each call
// before they are read, and two calls that overlap on the GPU race on it.
namespace cs {
namespace {

constexpr int64_t NOALLOC_MAX_NODES = int64_t(1) << 24;                    // 16,777,216 fluid nodes
constexpr int64_t NOALLOC_TILES = NOALLOC_MAX_NODES / T_NODES;              // 4,096 tiles of 4,096 nodes
constexpr int64_t NOALLOC_WORDS = int64_t(Q) * (NOALLOC_TILES + 1) + 2;    // tile sums + status: about 885 KB

static __device__ __align__(256) int64_t g_noalloc_scratch[NOALLOC_WORDS];

// Device address of the static scratch on the current device. The host-side name g_noalloc_scratch is only a
// stand-in for the symbol, never a device address, so the address is looked up with the device current. It is
// looked up on every call rather than cached: a cached address would go stale if the caller reset the device
// (cudaDeviceReset) and a new context placed the array elsewhere.
int noalloc_scratch(int64_t** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return fail(CS_ERR_CUDA, "cs_links_build_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
    *out = static_cast<int64_t*>(p);
    return CS_OK;
}

}  // namespace
}  // namespace cs

extern "C" int cs_links_build_noalloc(const int32_t* nbr, const float* q, int64_t n, int32_t n_out,
                                      int64_t gmax_cap, int32_t* links, int32_t* gnode, int32_t* ginfo, float* gq,
                                      int64_t* ghosts, void* stream) {
    if (!ghosts) return fail(CS_ERR_ARG, "cs_links_build_noalloc: null ghosts");
    for (int i = 0; i < Q; ++i) ghosts[i] = 0;
    if (n < 0 || n > NOALLOC_MAX_NODES)
        return fail(CS_ERR_SIZE, "cs_links_build_noalloc: %lld nodes exceed the static scratch limit of %lld nodes; "
                    "use cs_links_count / cs_links_fill with a caller-provided scratch buffer", (long long)n,
                    (long long)NOALLOC_MAX_NODES);
    if (gmax_cap < 0 || int64_t(Q) * (n + gmax_cap) >= (int64_t(1) << 31))
        return fail(CS_ERR_SIZE, "cs_links_build_noalloc: gmax_cap %lld (27 * (n + gmax_cap) must stay below 2^31)",
                    (long long)gmax_cap);
    if (n_out < 1) return fail(CS_ERR_ARG, "cs_links_build_noalloc: n_out %d", n_out);
    if (n == 0) return CS_OK;
    if (!nbr || !q || !links || (gmax_cap > 0 && (!gnode || !ginfo || !gq)))
        return fail(CS_ERR_ARG, "cs_links_build_noalloc: null buffer");
    int64_t* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc != CS_OK) return rc;
    const Layout l = layout(n);
    int64_t* part = scratch;
    int64_t* status = scratch + int64_t(Q) * (NOALLOC_TILES + 1);
    cudaStream_t st = as_stream(stream);
    k_ghost_count<<<dim3(unsigned(l.tiles), Q), T_THREADS, 0, st>>>(nbr, n, l.tiles, part);
    CS_CHECK_LAUNCH("k_ghost_count");
    k_ghost_scan<<<Q, 1024, 0, st>>>(part, l.tiles);
    CS_CHECK_LAUNCH("k_ghost_scan");
    for (int i = 0; i < Q; ++i)
        CS_CUDA(cudaMemcpyAsync(ghosts + i, part + int64_t(i) * (l.tiles + 1) + l.tiles, sizeof(int64_t),
                                cudaMemcpyDeviceToHost, st));
    CS_CUDA(cudaStreamSynchronize(st));
    int64_t gmax = 0;
    for (int i = 0; i < Q; ++i) gmax = std::max(gmax, ghosts[i]);
    if (gmax > gmax_cap)
        return fail(CS_ERR_SIZE, "cs_links_build_noalloc: %lld ghost slots needed in one direction, gmax_cap is "
                    "%lld (ghosts holds the counts)", (long long)gmax, (long long)gmax_cap);
    unsigned long long init[2] = {0ull, ~0ull};
    CS_CUDA(cudaMemcpyAsync(status, init, sizeof(init), cudaMemcpyHostToDevice, st));
    k_ghost_fill<<<dim3(unsigned(l.tiles), Q), T_THREADS, 0, st>>>(nbr, q, n, n_out, gmax_cap, l.tiles, part, links,
                                                                   gnode, ginfo, gq,
                                                                   reinterpret_cast<unsigned long long*>(status));
    CS_CHECK_LAUNCH("k_ghost_fill");
    unsigned long long res[2];
    CS_CUDA(cudaMemcpyAsync(res, status, sizeof(res), cudaMemcpyDeviceToHost, st));
    CS_CUDA(cudaStreamSynchronize(st));
    if (res[0]) {
        const long long t = (long long)res[1];
        return fail(CS_ERR_ARG, "cs_links_build_noalloc: %llu invalid entries; first at link %lld node %lld (sources "
                    "must be < N, outlet codes < n_out = %d, wall q finite and >= 0)", res[0], t / n, t % n, n_out);
    }
    return CS_OK;
}
