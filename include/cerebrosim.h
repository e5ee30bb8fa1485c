/* cerebrosim.h — C ABI of the B200 sparse D3Q27 lattice-Boltzmann library (libcerebrosim_b200.so).
 *
 * The reference (CerebroSim) is pure Python: its solver interface is `lbm.py` (module functions + class Solver)
 * and `simulate.py`'s `ArterySolver`; it has no FFI of its own. Each entry point below names the reference
 * function or kernel whose behaviour it provides; the Python package `cerebrosim_b200` binds them with ctypes
 * (cerebrosim_b200/_lib.py) behind the same `lbm` / `Solver` interface.
 *
 * Conventions
 *  - Every function returns an int status: CS_OK (0) or a CS_ERR_* code; cs_last_error() gives the message of the
 *    last failure on the calling host thread. Nothing aborts, traps or exits.
 *  - All array pointers are DEVICE pointers (cudaMalloc'd or from a tensor) unless the comment says host.
 *    The library allocates no device memory: callers pass scratch buffers sized by the *_scratch_bytes queries.
 *  - `stream` is a cudaStream_t passed as void*; NULL means the legacy default stream. Work is enqueued
 *    asynchronously unless the comment says the call synchronises the stream.
 *  - Lattice layout (identical to the reference's tables, lbm.py:264-330): N fluid nodes numbered in C order of
 *    the SDF grid; link-major tables nbr[i * N + n] (int32: pull source, or WALL -1, INLET -2, OUTLET k -3-k) and
 *    q[i * N + n] (float32 wall fraction); uin[n * 3 + c]; coords[n * 3 + c].
 */
#ifndef CEREBROSIM_H
#define CEREBROSIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CS_OK 0
#define CS_ERR_ARG 1     /* invalid argument (size, pointer, code out of range) */
#define CS_ERR_CUDA 2    /* a CUDA runtime call failed */
#define CS_ERR_SIZE 3    /* a size exceeds what the entry point supports */
#define CS_ERR_DEVICE 4  /* a kernel reported a failure through its status word */

/* D3Q27 link codes in the neighbour table (lbm.py:50). */
#define CS_WALL (-1)
#define CS_INLET (-2)
#define CS_OUTLET0 (-3)

/* Population storage formats (the arithmetic is FP32 in every format). */
#define CS_STORE_F32 0   /* f - w_i as float32: the reference's layout (lbm.py:23) */
#define CS_STORE_F16 1   /* (f - w_i) * 1024 / w_i as IEEE half, round to nearest */
#define CS_STORE_BF16 2  /* (f - w_i) * 1024 / w_i as bfloat16, round to nearest */

/* Words per row of the segment delta table (27 deltas + 1 padding word). */
#define CS_SEG_STRIDE 28

#define CS_MODEL_TRT 0
#define CS_MODEL_REGULARISED 1

/* One opening of the vessel (lbm.build_lattice `openings` entry, lbm.py:267-270). */
typedef struct cs_opening {
    int32_t kind;       /* 0 = inlet, 1 = outlet */
    int32_t pad_;
    double centre[3];   /* same units as origin / dx */
    double normal[3];   /* outward unit normal */
    double radius;
} cs_opening;

/* ---------------------------------------------------------------------------------------------------------------
 * Vessel signed distance — replaces vessel.k_sdf + vessel.sdf_grid (vessel.py:178-207, 230-245).
 * ------------------------------------------------------------------------------------------------------------- */

/* Signed distance (negative inside) of a branched vessel on the voxel centres origin + (i, j, k) dx, float32, C
 * order (k fastest), written to out (nx * ny * nz floats), evaluated in float32 like vessel.k_sdf: per branch the
 * minimum over its segments of the round-cone distance, cut by the flat caps within 2.5 cap radii of each open end,
 * branches joined by the polynomial smooth minimum of radius blend. Centrelines are packed as vessel._packed
 * (vessel.py:210-221) packs them: pts (n_pts * 3) and rad (n_pts) with the branches back to back, br_start /
 * br_count (nbranch) per branch, cap_p / cap_n (2 nbranch * 3) and cap_r (2 nbranch, 0 = closed end) for the start
 * and end of each branch. origin is a HOST pointer (3 floats); every other array is on the device. */
int cs_sdf_vessel(const float* pts, const float* rad, const int32_t* br_start, const int32_t* br_count,
                  int32_t nbranch, const float* cap_p, const float* cap_n, const float* cap_r, float blend,
                  const float* origin, float dx, int64_t nx, int64_t ny, int64_t nz, float* out, void* stream);

/* ---------------------------------------------------------------------------------------------------------------
 * Lattice / neighbour-table builder — replaces lbm.build_lattice (lbm.py:264-330), bit-exact tables.
 * Two phases because N is only known after the fluid count: cs_lattice_count, then cs_lattice_fill.
 * ------------------------------------------------------------------------------------------------------------- */

/* Bytes of device scratch that cs_lattice_count / cs_lattice_fill need for an nx x ny x nz grid. */
size_t cs_lattice_scratch_bytes(int64_t nx, int64_t ny, int64_t nz);

/* Count the fluid nodes (phi < 0) of the float32 grid phi (C order) and number them in C order (lbm.py:274-278).
 * Writes the count to *n_fluid (HOST pointer); synchronises `stream`. scratch must stay untouched until
 * cs_lattice_fill. */
int cs_lattice_count(const float* phi, int64_t nx, int64_t ny, int64_t nz, void* scratch, int64_t* n_fluid,
                     void* stream);

/* Fill the tables for the n_fluid nodes counted above (lbm.py:280-330).
 * openings: HOST array of n_openings entries; inlets are matched before outlets, each in list order; outlet k is
 *   the k-th outlet of the list. periodic_mask: bit a set = axis a wraps around.
 * Outputs (device): nbr (27*N int32), q (27*N float32), uin (N*3 float32), coords (N*3 int32),
 *   counts (int64: [wall, inlet, outlet_0, ..., outlet_{n_out-1}]). */
int cs_lattice_fill(const float* phi, int64_t nx, int64_t ny, int64_t nz, const double* origin, double dx,
                    const cs_opening* openings, int32_t n_openings, int32_t periodic_mask, double opening_slack,
                    void* scratch, int64_t n_fluid, int32_t* nbr, float* q, float* uin, int32_t* coords,
                    int64_t* counts, void* stream);

/* Sponge (replaces Solver.set_sponge's host computation, lbm.py:398-416) for the n nodes of `coords` (device, N*3
 * int32): per node tau_cell = max over the openings whose kind bit is set in kinds_mask (bit 0 inlets, bit 1
 * outlets) of tau + (tau_max - tau) * smoothstep(clip(1 - depth / length, 0, 1)) within 1.5 radii of the opening's
 * axis (depth = inward distance from the opening plane in cells), in the reference's float64 operations and
 * rounding. Outputs (device): om[n] = float32(1 / tau_cell); tau_out[n] = tau_cell (float64), or null.
 * openings: HOST array. */
int cs_sponge_om(const int32_t* coords, int64_t n, const double* origin, double dx, const cs_opening* openings,
                 int32_t n_openings, int32_t kinds_mask, double tau, double length, double tau_max, float* om,
                 double* tau_out, void* stream);

/* ---------------------------------------------------------------------------------------------------------------
 * Step — replaces lbm.k_clock + lbm.k_step (lbm.py:90-257) and, when n_open > 0, simulate.k_flux + simulate.k_bc
 * (simulate.py:65-82).
 *
 * Link tables of the step. Every boundary link (wall, inlet or outlet code in nbr) of direction i is given a ghost
 * slot g in 0 .. ghosts[i]-1, numbered in node order. The population rows are npad = n + gmax long (gmax = the
 * largest ghosts[i]); slot g of direction i lives at f[i * npad + n + g]. Each step, the boundary-link kernel writes
 * into every ghost slot the value the reference's k_step pulls for that link (Bouzidi wall, velocity inlet,
 * pressure outlet: lbm.py:163-181), so the bulk kernel pulls every link from links[i * n + node] (a node < n or
 * n + g) without a branch.
 *   gnode[i * gmax + g]  node of the slot
 *   ginfo[i * gmax + g]  wall: the node behind it along -c_i (nbr[opp(i)][node], the Bouzidi second node) or -1;
 *                        inlet: -2; outlet k: -3 - k
 *   gq[i * gmax + g]     wall: q; inlet / outlet: -1
 * ------------------------------------------------------------------------------------------------------------- */

/* Bytes of device scratch cs_links_count / cs_links_fill need for n nodes. */
size_t cs_links_scratch_bytes(int64_t n);

/* Count the boundary links of each direction: ghosts (HOST, 27 int64). Synchronises `stream`; scratch must stay
 * untouched until cs_links_fill. */
int cs_links_count(const int32_t* nbr, int64_t n, void* scratch, int64_t* ghosts, void* stream);

/* Build links (27 * n) and the ghost tables (27 * gmax each) from the reference's nbr / q tables. Checks every
 * entry: pull sources < n, outlet codes < n_out, wall q finite and >= 0; status (device, 2 x int64) receives the
 * number of bad entries and the first bad (link * n + node). Synchronises `stream`; CS_ERR_ARG if any is bad. */
int cs_links_fill(const int32_t* nbr, const float* q, int64_t n, int32_t n_out, int64_t gmax, void* scratch,
                  int32_t* links, int32_t* gnode, int32_t* ginfo, float* gq, int64_t* status, void* stream);

/* The link-table build of cs_links_count + cs_links_fill in one call that allocates nothing. This entry point has
 * no counterpart in the reference. It is for callers that cannot allocate device memory themselves — a plugin whose
 * host application owns all device memory and hands it only the input and output buffers, or a process whose
 * fixed device-memory budget is already committed — and so cannot provide the scratch buffer cs_links_count /
 * cs_links_fill need.
 * The scratch (per-tile ghost counts and two status words, about 885 KB) is a static array inside the library:
 * every GPU that loads the library holds it until the process exits. n is limited to 16,777,216 nodes (2^24);
 * larger lattices get CS_ERR_SIZE and must use cs_links_count / cs_links_fill. The caller passes the outputs sized
 * for gmax_cap ghost slots per direction (tables 27 * gmax_cap, gnode pre-filled with -1 so that unused slots are
 * marked); ghosts (HOST, 27 int64) receives the counts, and CS_ERR_SIZE comes back (with the counts) when a
 * direction needs more than gmax_cap. The ghost tables then have stride gmax_cap: use it as gmax in the step.
 * Each call looks up the array's device address on the current device. Every call shares the one array and resets
 * what it reads before reading it, but calls that overlap on the GPU (other streams, other host threads) race on
 * it. Synchronises `stream` (twice: to read the counts, then the status); makes no cudaMalloc, cudaFree or other
 * allocating call. */
int cs_links_build_noalloc(const int32_t* nbr, const float* q, int64_t n, int32_t n_out, int64_t gmax_cap,
                           int32_t* links, int32_t* gnode, int32_t* ginfo, float* gq, int64_t* ghosts, void* stream);

/* Inverse of cs_links_fill for checking: the reference's nbr codes and q (0.5 on non-wall links, lbm.py:281). */
int cs_links_decode(const int32_t* links, const int32_t* ginfo, const float* gq, int64_t n, int64_t gmax,
                    int32_t* nbr, float* q, void* stream);

/* Compressed pull connectivity of the bulk kernel, built from the links table of cs_links_fill. A node whose 27 codes
 * are all fluid sources and whose deltas (code - node) equal those of the previous node shares its segment:
 *   lcode[node] = s >= 0: sources node + segdelta[s * CS_SEG_STRIDE + i] (rows padded to 28 words, 16-byte
 *                         aligned, so the bulk kernel reads a row with seven 128-bit loads);
 *   lcode[node] = -1 - k: irregular node (some ghost link), codes irr[i * n_irr + k].
 * count (synchronises `stream`; n_seg / n_irr are HOST outputs), then fill with the same scratch. */
size_t cs_compress_scratch_bytes(int64_t n);
int cs_compress_count(const int32_t* links, int64_t n, void* scratch, int64_t* n_seg, int64_t* n_irr, void* stream);
int cs_compress_fill(const int32_t* links, int64_t n, int64_t n_seg, int64_t n_irr, void* scratch, int32_t* lcode,
                     int32_t* segdelta, int32_t* irr, void* stream);
/* Inverse, for checking: the 27 x n links table from the compressed form. */
int cs_compress_expand(const int32_t* lcode, const int32_t* segdelta, const int32_t* irr, int64_t n, int64_t n_irr,
                       int32_t* links, void* stream);

typedef struct cs_step_desc {
    int64_t n;               /* fluid nodes */
    int64_t npad;            /* population row length, n + gmax; 27 * npad < 2^31 */
    int64_t gmax;            /* ghost slots per direction */
    int32_t storage;         /* CS_STORE_* */
    int32_t model;           /* CS_MODEL_* (lbm.py:359) */
    int32_t bouzidi;         /* interpolated walls on / half-way bounce-back */
    int32_t gal;             /* Galilean correction (lbm.py:362) */
    float sigma;             /* hybrid regularisation blend (1 = off) */
    float magic;             /* TRT magic parameter */
    float force[3];          /* body force, scaled by the drive */
    int32_t block;           /* threads per block of the bulk kernel; 0 = default */
    void* f[2];              /* populations (27 * npad) in `storage` format, link-major */
    float* vel[2];           /* velocity, SoA: vel[b][c * n + node] */
    float* rho;              /* density deviation (n) */
    const int32_t* lcode;    /* compressed connectivity (n) from cs_compress_fill */
    const int32_t* segdelta; /* (CS_SEG_STRIDE * n_seg), 16-byte aligned */
    const int32_t* irr;      /* (27 * n_irr) */
    int64_t n_irr;
    const int32_t* gnode;    /* ghost tables (27 * gmax) from cs_links_fill */
    const int32_t* ginfo;
    const float* gq;
    const float* uin;        /* inlet profile (n * 3) */
    const float* om;         /* relaxation rate 1 / tau per node (n), negated on cells with an inlet link */
    float* p_out;            /* pressure per outlet (n_out), read by outlet links */
    int32_t n_out;
    int32_t* tick;           /* step counters (2): tick[a] is the count of a step that reads buffer a */
    float* drive;            /* drive value of the last step (1) */
    const float* coef;       /* Fourier coefficients a0, a1, b1, ... (2 nh + 1) */
    int32_t nh, period, ramp;
    /* ArterySolver coupling (n_open = 0: none) */
    int32_t n_open;          /* open ends; p_out[0] follows the drive, p_out[k >= 1] the resistances */
    int64_t n_flux;          /* entries of the slab-flux list, sorted by node */
    const int32_t* flux_idx; /* node of each entry */
    const float* flux_w;     /* weight vector of each entry (n_flux * 3) */
    const int32_t* flux_slot;/* open end of each entry */
    const int32_t* flux_block; /* first flux entry of each bulk block (n_blocks + 1) from cs_flux_blocks */
    double* q_part;          /* per bulk block partial fluxes (n_blocks * 8), written by the blocks in fb_list */
    const int32_t* fb_list;  /* the bulk blocks that hold flux entries, ascending (n_fb) */
    int32_t n_fb;
    double* q_last;          /* flux of the last step (n_open) */
    double* p_out64;         /* FP64 state of the outlet pressures (n_open) */
    const float* r_out;      /* resistance per open end (n_open) */
    double pref, alpha;
    /* Boundary-link grid without padding: gblock[i] = sum over directions j < i of ceil(ghosts[j] / 256) (gblock[0] = 0,
     * gblock[27] = the number of 256-slot blocks over all directions). All zero: the padded grid, ceil(gmax / 256)
     * blocks for every direction. */
    int32_t gblock[28];
    /* Beat means of the resistance coupling (n_open > 0; null: none): k_bc adds, every step, p_out64[k] to
     * beat_acc[k] and q_last[k] to beat_acc[n_open + k] (FP64) and 1 to beat_acc[2 * n_open]; the caller zeroes
     * it at a beat's start and divides by the count at its end (the beat means of simulate.py:325-333). */
    double* beat_acc;
} cs_step_desc;

/* Block partition of a sorted flux list for `block` threads per block: out[b] = first entry with
 * flux_idx >= b * block, b = 0 .. ceil(n / block). */
int cs_flux_blocks(const int32_t* flux_idx, int64_t n_flux, int64_t n, int32_t block, int32_t* out, void* stream);

/* Enqueue `steps` steps, the first reading buffer a (0/1) and writing 1 - a, alternating (lbm.py:422-428). A step
 * is the boundary-link kernel (one block per 256 boundary links of a direction, or a single block without any: it
 * also advances the clock), the bulk kernel and, when n_open > 0, the one-block k_bc kernel. */
int cs_step(const cs_step_desc* d, int32_t a, int32_t steps, void* stream);

/* Check a descriptor (HOST struct) as cs_step does, without launching anything. */
int cs_step_check(const cs_step_desc* d);

/* Capture `steps` steps starting from buffer a into a CUDA graph (lbm.py:436-442); *graph receives an opaque
 * handle for cs_graph_launch / cs_graph_destroy. The stream must not be the legacy default stream. */
int cs_graph_capture(const cs_step_desc* d, int32_t a, int32_t steps, void* stream, void** graph);

/* ---------------------------------------------------------------------------------------------------------------
 * Batched step — many independent lattices (vessels of different sizes, clots and drives) advanced together. The
 * reference runs one simulation per GPU process (a Slurm job array); here the instances' node lists are
 * concatenated into one work list, and one launch per kernel and step covers up to CS_BATCH_GROUP of them (larger
 * batches launch one kernel per group): the blocks take work items (a bulk block of some instance, or a boundary
 * block) from the list and read that instance's descriptor from the kernel's parameters. Each instance keeps its
 * own buffers, clock, drive, outlet pressures and coupling.
 * ------------------------------------------------------------------------------------------------------------- */
#define CS_BATCH_GROUP 64

typedef struct cs_batch_desc {
    int32_t n_inst;
    int32_t storage, model, gal, force; /* shared by all instances; force = some instance has a body force */
    int32_t any_open;                   /* some instance has the resistance coupling (runs k_bc per instance) */
    int32_t block;                      /* threads per bulk block, every instance (its flux_block must match) */
    int32_t grid_bulk, grid_bnd;        /* persistent grid sizes; 0 = one block per work item */
    int32_t pad_;
    const cs_step_desc* descs;          /* HOST array (n_inst); each is checked as cs_step_check does and copied
                                           into the kernels' parameters at launch (a captured graph keeps its copy) */
    const int32_t* parity;              /* HOST (n_inst): instance i reads buffer a ^ parity[i] */
    int32_t* counter;                   /* DEVICE, ceil(n_inst / CS_BATCH_GROUP) ints, zero before the first step:
                                           the bulk kernels' work counters (the boundary kernels reset them) */
} cs_batch_desc;

/* Enqueue `steps` batched steps; the first reads buffer a ^ parity[i] of instance i. */
int cs_batch_step(const cs_batch_desc* b, int32_t a, int32_t steps, void* stream);
int cs_batch_graph_capture(const cs_batch_desc* b, int32_t a, int32_t steps, void* stream, void** graph);
int cs_graph_launch(void* graph, void* stream);
int cs_graph_destroy(void* graph);

/* ---------------------------------------------------------------------------------------------------------------
 * Wall shear stress — replaces wss.shear (wss.py:50-57); the fit coefficients come from the host (wss.weights).
 * ------------------------------------------------------------------------------------------------------------- */

/* tau[v] = scale * sum_j c[v * K + j] (u_j - (u_j . n_v) n_v), u_j = U[idx[v * K + j]] (n_cells * 3 float, m/s),
 * n_v = normals[v] (unit, into the lumen), accumulated in FP64; scale = mu * 1e3 for mm distances and Pa. Entries
 * with c = 0 or an index outside 0 .. n_cells - 1 are skipped. Outputs tau (n_vert * 3 float). */
int cs_wss_shear(const float* U, int64_t n_cells, const int32_t* idx, const float* c, const float* normals,
                 int64_t n_vert, int32_t K, double scale, float* tau, void* stream);

/* ---------------------------------------------------------------------------------------------------------------
 * Heartbeat-loop measurements — replace simulate.k_gather (simulate.py:85-90) and the coarse-map averaging of the
 * stored frames (simulate.py:236-242, 346-353). rho (n) and vel (SoA, 3 * n) are a solver's state buffers; `cells`
 * lists cell indices (each < n, checked by the caller) grouped by segment, `start` (segments + 1) delimits them.
 * Sums are FP64 in a fixed order.
 * ------------------------------------------------------------------------------------------------------------- */

/* Per probe k: psum[k] = sum of rho / 3 over its cells, umax[k] = the largest |u| among them. */
int cs_probe_gather(const float* rho, const float* vel, int64_t n, const int32_t* cells, const int32_t* start,
                    int32_t n_probes, double* psum, float* umax, void* stream);

/* Per coarse bin b: p_out[b] = mean of rho / 3 over its cells, u_out[3 b + c] = mean of u_c (0 for an empty bin). */
int cs_bin_fields(const float* rho, const float* vel, int64_t n, const int32_t* cells, const int32_t* start,
                  int64_t n_bins, float* p_out, float* u_out, void* stream);

/* ---------------------------------------------------------------------------------------------------------------
 * Misc
 * ------------------------------------------------------------------------------------------------------------- */

/* Copy the message of the calling thread's last failure into buf (NUL-terminated); returns its length. */
int cs_last_error(char* buf, int32_t len);

/* Library version string (static). */
const char* cs_version(void);

/* sizeof of the ABI structs, so that bindings can check their layout: which = 0 cs_opening, 1 cs_step_desc;
 * which = 2 returns CS_SEG_STRIDE, 3 sizeof(cs_batch_desc). */
size_t cs_abi_sizeof(int32_t which);

#ifdef __cplusplus
}
#endif

#endif /* CEREBROSIM_H */
