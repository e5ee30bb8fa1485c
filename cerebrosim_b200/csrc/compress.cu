// Compressed pull connectivity of the bulk kernel.
//
// The step's link table (27 x n int32, from cs_links_fill) costs 108 B per node and update, as much as the FP32
// populations it addresses. In C order, a node whose 27 pull sources are all fluid nodes usually pulls from
// n + delta_i with deltas that stay the same along its z-run (the neighbouring rows advance with it). So:
//   regular node   (no ghost link): lcode[n] = s >= 0, a segment of consecutive nodes sharing one delta vector;
//                                   segdelta[s * CS_SEG_STRIDE + i] = delta_i, and the sources are n + delta_i;
//   irregular node (some ghost link): lcode[n] = -1 - k, with its 27 codes in irr[i * n_irr + k] (link-major, so
//                                   consecutive irregular nodes read consecutive words).
// A node costs 4 bytes of connectivity instead of 108 unless it is irregular; the segment table (27 words per
// segment, one segment per row of a straight vessel) is read through L1 / L2 and broadcast within a warp.
#include "cs_common.cuh"

namespace cs {
namespace {

constexpr int T_THREADS = 256;
constexpr int T_ROUNDS = 16;
constexpr int64_t T_NODES = T_THREADS * T_ROUNDS;
constexpr uint8_t F_IRR = 1, F_SEG = 2;

struct Layout {
    int64_t tiles;
    size_t off_part, total;
};

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

Layout layout(int64_t n) {
    Layout l;
    l.tiles = ceil_div(n, T_NODES);
    l.off_part = align256(size_t(n));
    l.total = l.off_part + 2 * size_t(l.tiles + 1) * sizeof(int64_t) + 256;
    return l;
}

// Flags per node: irregular (a ghost link), and start of a segment (regular, and the previous node is irregular or
// has other deltas).
__global__ void k_cmp_flags(const int32_t* __restrict__ links, int64_t n, uint8_t* __restrict__ flags) {
    const int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (v >= n) return;
    bool irr = false, prev_irr = v == 0, same = v > 0;
    for (int i = 0; i < Q; ++i) {
        const int32_t s = links[int64_t(i) * n + v];
        irr = irr || s >= n;
        if (v > 0) {
            const int32_t p = links[int64_t(i) * n + v - 1];
            prev_irr = prev_irr || p >= n;
            same = same && (int64_t(s) - v == int64_t(p) - (v - 1));
        }
    }
    uint8_t f = irr ? F_IRR : 0;
    if (!irr && (prev_irr || !same)) f |= F_SEG;
    flags[v] = f;
}

__global__ void k_cmp_count(const uint8_t* __restrict__ flags, int64_t n, int64_t tiles, int64_t* __restrict__ part) {
    __shared__ int ws[2][T_THREADS / 32];
    const int64_t base = int64_t(blockIdx.x) * T_NODES;
    int ci = 0, cs_ = 0;
    for (int r = 0; r < T_ROUNDS; ++r) {
        const int64_t v = base + int64_t(r) * T_THREADS + threadIdx.x;
        if (v < n) {
            const uint8_t f = flags[v];
            ci += (f & F_IRR) ? 1 : 0;
            cs_ += (f & F_SEG) ? 1 : 0;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        ci += __shfl_down_sync(0xffffffffu, ci, o);
        cs_ += __shfl_down_sync(0xffffffffu, cs_, o);
    }
    if ((threadIdx.x & 31) == 0) {
        ws[0][threadIdx.x >> 5] = ci;
        ws[1][threadIdx.x >> 5] = cs_;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        int64_t t = 0;
        for (int w = 0; w < T_THREADS / 32; ++w) t += ws[threadIdx.x][w];
        part[int64_t(threadIdx.x) * (tiles + 1) + blockIdx.x] = t;
    }
}

// Exclusive scan of one flag's tile counts (block b: 0 irregular, 1 segment starts); totals at part[b][tiles].
__global__ void k_cmp_scan(int64_t* __restrict__ part, int64_t tiles) {
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
            const int64_t x = s[k];
            s[k] = run;
            run += x;
        }
        p[tiles] = run;
    }
    __syncthreads();
    int64_t run = s[threadIdx.x];
    for (int64_t t = lo; t < hi; ++t) {
        const int64_t x = p[t];
        p[t] = run;
        run += x;
    }
}

__global__ void k_cmp_fill(const int32_t* __restrict__ links, const uint8_t* __restrict__ flags, int64_t n,
                           int64_t n_irr, int64_t tiles, const int64_t* __restrict__ part, int32_t* __restrict__ lcode,
                           int32_t* __restrict__ segdelta, int32_t* __restrict__ irr) {
    __shared__ int wc[2][T_THREADS / 32];
    __shared__ int64_t run[2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < 2) run[threadIdx.x] = part[int64_t(threadIdx.x) * (tiles + 1) + blockIdx.x];
    const int64_t base = int64_t(blockIdx.x) * T_NODES;
    for (int r = 0; r < T_ROUNDS; ++r) {
        const int64_t v = base + int64_t(r) * T_THREADS + threadIdx.x;
        const uint8_t f = v < n ? flags[v] : 0;
        const unsigned mi = __ballot_sync(0xffffffffu, (f & F_IRR) != 0);
        const unsigned ms = __ballot_sync(0xffffffffu, (f & F_SEG) != 0);
        if (lane == 0) {
            wc[0][warp] = __popc(mi);
            wc[1][warp] = __popc(ms);
        }
        __syncthreads();
        int64_t ki = run[0], ks = run[1];
        for (int w = 0; w < warp; ++w) {
            ki += wc[0][w];
            ks += wc[1][w];
        }
        const unsigned below = (1u << lane) - 1u;
        ki += __popc(mi & below);
        ks += __popc(ms & below);           // segment starts before this node, this warp
        if (v < n) {
            if (f & F_IRR) {
                lcode[v] = int32_t(-1 - ki);
                for (int i = 0; i < Q; ++i) irr[int64_t(i) * n_irr + ki] = links[int64_t(i) * n + v];
            } else {
                // a regular node belongs to the last segment started at or before it
                const int64_t seg = (f & F_SEG) ? ks : ks - 1;
                lcode[v] = int32_t(seg);
                if (f & F_SEG) {
                    for (int i = 0; i < Q; ++i)
                        segdelta[seg * CS_SEG_STRIDE + i] = int32_t(int64_t(links[int64_t(i) * n + v]) - v);
                    segdelta[seg * CS_SEG_STRIDE + Q] = 0;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x < 2) {
            int64_t t = 0;
            for (int w = 0; w < T_THREADS / 32; ++w) t += wc[threadIdx.x][w];
            run[threadIdx.x] += t;
        }
        __syncthreads();
    }
}

__global__ void k_cmp_expand(const int32_t* __restrict__ lcode, const int32_t* __restrict__ segdelta,
                             const int32_t* __restrict__ irr, int64_t n, int64_t n_irr, int32_t* __restrict__ links) {
    const int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (v >= n) return;
    const int32_t c = lcode[v];
    for (int i = 0; i < Q; ++i)
        links[int64_t(i) * n + v] = c >= 0 ? int32_t(v + segdelta[int64_t(c) * CS_SEG_STRIDE + i])
                                           : irr[int64_t(i) * n_irr + (-1 - c)];
}

}  // namespace
}  // namespace cs

using namespace cs;

extern "C" size_t cs_compress_scratch_bytes(int64_t n) { return n < 0 ? 0 : layout(n).total; }

extern "C" int cs_compress_count(const int32_t* links, int64_t n, void* scratch, int64_t* n_seg, int64_t* n_irr,
                                 void* stream) {
    if (n < 0 || n >= (int64_t(1) << 30)) return fail(CS_ERR_SIZE, "cs_compress_count: n = %lld", (long long)n);
    if (!n_seg || !n_irr) return fail(CS_ERR_ARG, "cs_compress_count: null outputs");
    *n_seg = *n_irr = 0;
    if (n == 0) return CS_OK;
    if (!links || !scratch) return fail(CS_ERR_ARG, "cs_compress_count: null buffer");
    const Layout l = layout(n);
    cudaStream_t st = as_stream(stream);
    char* s = static_cast<char*>(scratch);
    uint8_t* flags = reinterpret_cast<uint8_t*>(s);
    int64_t* part = reinterpret_cast<int64_t*>(s + l.off_part);
    k_cmp_flags<<<unsigned(ceil_div(n, 256)), 256, 0, st>>>(links, n, flags);
    CS_CHECK_LAUNCH("k_cmp_flags");
    k_cmp_count<<<unsigned(l.tiles), T_THREADS, 0, st>>>(flags, n, l.tiles, part);
    CS_CHECK_LAUNCH("k_cmp_count");
    k_cmp_scan<<<2, 1024, 0, st>>>(part, l.tiles);
    CS_CHECK_LAUNCH("k_cmp_scan");
    CS_CUDA(cudaMemcpyAsync(n_irr, part + l.tiles, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CS_CUDA(cudaMemcpyAsync(n_seg, part + (l.tiles + 1) + l.tiles, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CS_CUDA(cudaStreamSynchronize(st));
    return CS_OK;
}

extern "C" int cs_compress_fill(const int32_t* links, int64_t n, int64_t n_seg, int64_t n_irr, void* scratch,
                                int32_t* lcode, int32_t* segdelta, int32_t* irr, void* stream) {
    if (n < 0 || n >= (int64_t(1) << 30) || n_seg < 0 || n_irr < 0 || n_seg + n_irr > n)
        return fail(CS_ERR_SIZE, "cs_compress_fill: n %lld segments %lld irregular %lld", (long long)n,
                    (long long)n_seg, (long long)n_irr);
    if (n == 0) return CS_OK;
    if (!links || !scratch || !lcode || (n_seg > 0 && !segdelta) || (n_irr > 0 && !irr))
        return fail(CS_ERR_ARG, "cs_compress_fill: null buffer");
    const Layout l = layout(n);
    cudaStream_t st = as_stream(stream);
    char* s = static_cast<char*>(scratch);
    k_cmp_fill<<<unsigned(l.tiles), T_THREADS, 0, st>>>(links, reinterpret_cast<const uint8_t*>(s), n, n_irr, l.tiles,
                                                        reinterpret_cast<const int64_t*>(s + l.off_part), lcode,
                                                        segdelta, irr);
    CS_CHECK_LAUNCH("k_cmp_fill");
    return CS_OK;
}

extern "C" int cs_compress_expand(const int32_t* lcode, const int32_t* segdelta, const int32_t* irr, int64_t n,
                                  int64_t n_irr, int32_t* links, void* stream) {
    if (n < 0 || n_irr < 0) return fail(CS_ERR_ARG, "cs_compress_expand: n %lld", (long long)n);
    if (n == 0) return CS_OK;
    if (!lcode || !links) return fail(CS_ERR_ARG, "cs_compress_expand: null buffer");
    k_cmp_expand<<<unsigned(ceil_div(n, 256)), 256, 0, as_stream(stream)>>>(lcode, segdelta, irr, n, n_irr, links);
    CS_CHECK_LAUNCH("k_cmp_expand");
    return CS_OK;
}
