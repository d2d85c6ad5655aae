// C ABI of the SPH step (include/gfsph.h): handle, device memory, the
// per-step launch sequence, CUDA-graph replay and capacity growth.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <new>
#include <type_traits>
#include <vector>

#include "../../include/gfsph.h"
#include "gfsph_kernels.cuh"
#include "gfsph_couple.cuh"
#include "gfsph_adjoint.cuh"

using namespace gfsph;

namespace {

enum KernelId {
    K_PREP, K_BOUNDS, K_HIST, K_SCAN_TILES, K_SCAN_ADD, K_SCATTER, K_CELL_SORT,
    K_REORDER, K_DENSITY, K_DENSITY_BIG, K_IFORCE, K_FORCE_BIG, K_FORCE_RK, K_XSPH, K_XSPH_BIG, K_DEM_ERODE,
    K_STEP_END, K_COPY, K_UNSORT, K_RASTER, K_HAZARD, K_EXPORT, K_MARK, K_BSCAN_TILES, K_BSCAN_ADD,
    K_DENSITY_SPARSE, K_COUPLE, K_ADJOINT, K_NORM, K_NORM_BIG, K_STAGE, K_WIR,
    K_STEPS,  // not a kernel: device time of whole gfsph_step batches (profile level 2)
    K_COUNT
};
const char* kKernelNames[K_COUNT] = {
    "k_prep", "k_bounds", "k_hist", "k_scan_tiles", "k_scan_add",
    "k_scatter", "k_cell_sort", "k_reorder", "k_density", "k_density_big", "k_iforce", "k_force_big",
    "k_force_rk", "k_xsph", "k_xsph_big", "k_dem_erode", "k_step_end", "k_copy_state", "k_unsort",
    "k_raster_idw", "k_hazard", "k_export_big", "k_mark", "k_scan_tiles(blocks)",
    "k_scan_add(blocks)", "k_density(sparse)", "k_couple", "k_adjoint", "k_norm", "k_norm_big", "k_stage", "k_wir", "step_batches"};

constexpr int kThreads = 128;
static_assert(kThreads <= 32 * kScatterWarps, "erosion_scatter keeps shared terms for kScatterWarps warps");
constexpr int kGraphSteps = 8;       // steps captured per multi-step graph
constexpr int kChunkSteps = 256;     // steps between host checks of the error word
constexpr int kMaxCells = kScanTile * 8192;
constexpr int kMaxNeighbours = 65536;  // largest initial neighbour-table capacity a handle accepts

__global__ void k_copy_state(PState A, PState B, int n) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        B.pos[s] = A.pos[s]; B.vel[s] = A.vel[s]; B.rho[s] = A.rho[s]; B.mass[s] = A.mass[s];
        B.hsml[s] = A.hsml[s]; B.flag[s] = A.flag[s]; B.id[s] = A.id[s]; B.pwp[s] = A.pwp[s];
    }
}

// Scatters the sorted state back to the original particle order.
__global__ void k_unsort(PState B, int n, PState U) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        int o = B.id[s];
        U.pos[o] = B.pos[s]; U.vel[o] = B.vel[s]; U.rho[o] = B.rho[s]; U.mass[o] = B.mass[s];
        U.hsml[o] = B.hsml[s]; U.flag[o] = B.flag[s]; U.pwp[o] = B.pwp[s];
    }
}

// Uaux(1,:) = pwp0rel * rho * alphas at input (Input_SW, SPH_SW_2019.f90:1829-1852).
__global__ void k_pwp_init(float* pwp, const float* rho, int n, float pwp0rel, float alfs) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
        pwp[s] = pwp0rel * (rho[s] * alfs);
}

// dst[s] = src[id[s]]: a caller array in the original order into slot order.
__global__ void k_gather_by_id(const float* src, const int* id, int n, float* dst) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) dst[s] = src[id[s]];
}

__global__ void k_unsort_f2(const float2* src, const int* id, int n, float2* dst) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) dst[id[s]] = src[s];
}

__global__ void k_iota(int* id, int n) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) id[s] = s;
}

__global__ void k_hazard_finish(const unsigned int* mo, float* out, int np) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
        unsigned int o = mo[k];
        out[k] = (o == 0u) ? 0.f : o2f(o);
    }
}

__global__ void k_d2f(const double* src, float* out, int np) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) out[k] = (float)src[k];
}

__global__ void k_i2f(const int* src, float* out, int np) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) out[k] = (float)src[k];
}

template <class T>
int dalloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    if (cudaMalloc((void**)p, count * sizeof(T)) == cudaSuccess) return 0;
    *p = nullptr;
    cudaGetLastError();  // a failed allocation is not sticky: later checks see only new errors
    return GFSPH_ERR_CUDA;
}
template <class T>
void dfree(T*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
}

// Launch of a step kernel with programmatic stream serialisation: the
// kernel may start (and wait in PDL_ENTRY) while the one before it in the
// stream finishes.  The stream capture records the dependency as a
// programmatic edge.
template <typename... KArgs, typename... Args>
void pdl_launch(void (*kernel)(KArgs...), int grid, int block, cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

int blocks_for(long long work, int threads = kThreads) {
    long long b = (work + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148LL * 64) b = 148LL * 64;
    return (int)b;
}

}  // namespace

struct gfsph_handle {
    int dev = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream2 = nullptr;       // side stream used only inside graph captures
    cudaEvent_t ev_fork[3]{}, ev_join[3]{};
    bool capturing = false;
    gfsph_params P;
    Rheo rheo;
    // DEM
    int nx = 0, ny = 0;
    DemView dem;
    bool dem_shared = false;    // the slope and curvature rows belong to another handle (ensembles)
    float2* d_grad = nullptr;
    float4* d_curvA = nullptr;
    float2* d_curvB = nullptr;
    float* d_z = nullptr;
    float* d_eroded = nullptr;
    float* d_avail = nullptr;
    double2* d_auxv = nullptr;
    // particles
    int n = 0;
    PState A{}, B{}, U{};
    int* cellA = nullptr;
    float2* velfin = nullptr;
    float* pterm = nullptr;
    float4* pr = nullptr;    // (pterm, h, m, 0) per slot
    int2* keyrank = nullptr;
    int* perm = nullptr;
    float2* f2tmp = nullptr;
    float4* xhm = nullptr;
    int4* nbr = nullptr;     // neighbour table: {j, W, dW/dx, dW/dy} per entry
    int* ncount = nullptr;
    int kcap = 0;
    float2* indv = nullptr;  // internal acceleration of every active particle
    float* rho0 = nullptr;   // start-of-step depth (pore-water pressure update, normalised density)
    // staged RK45 (nor_density or ic_cosTheta = 1)
    StageCarry carry{};
    float* rhoS = nullptr;   // the five depths of a step, k-major (nor_density)
    int2* rcell = nullptr;   // cell of the reference's grid per slot (skf 2, 3)
    float4* xsv = nullptr;   // (vx, vy, h, m) per slot after the RK update, for av_vel
    // soil and water (ic_ws_Interact = 1): material per caller index and per
    // slot; Z + hs and its gradient at the water particles; the soil-water
    // pair sums; Z + hs per DEM node and its FP64 accumulators
    unsigned char* spec_u = nullptr;
    unsigned char* spec_a = nullptr;
    float* zpw = nullptr;
    float2* gzw = nullptr;
    float2* bxy = nullptr;
    float* wir_hsz = nullptr;
    double2* wir_acc = nullptr;
    float* mass0_u = nullptr;  // mass per caller index at upload (nfric 3's m0)
    // cells
    int* count = nullptr;
    int* start = nullptr;
    int* tile_sum = nullptr;
    int cap_cells = 0;
    int* bmark = nullptr;   // block map: 1 where a block holds particles (cleared by k_hist)
    int* bstart = nullptr;  // its exclusive scan: slot of each occupied block
    int cap_blocks = 0;
    BoundsPart* bparts = nullptr;  // k_bounds block partials
    float level_factor = kBigFactor;  // search tunables (gfsph_set_search / gfsph_autotune)
    int reg_levels = kRegLevels;
    float cell_div = kCellDiv;
    // scalars
    StepScalars* S = nullptr;
    StepScalars* hS = nullptr;  // pinned mirror
    // graphs
    cudaGraphExec_t g1 = nullptr, gK = nullptr;
    // profiling: level 1 = per-kernel events (no graphs), 2 = events around
    // each gfsph_step's device work (graphs kept)
    bool profile = false;
    int profile_level = 0;
    cudaEvent_t ev0[K_COUNT]{}, ev1[K_COUNT]{};
    bool pending[K_COUNT]{};
    double prof_ms[K_COUNT]{};
    long long prof_cnt[K_COUNT]{};
    long long launches = 0;
    bool has_state = false, searched = false;
    // outputs
    double2* d_racc = nullptr;
    float* d_rout = nullptr;
    double* d_lam = nullptr;    // raster misfit: dL/dR per node
    double* d_lpart = nullptr;  // raster misfit: block sums of the loss
    double *haz_sum_h = nullptr, *haz_sum_v = nullptr;
    unsigned int *haz_max_h = nullptr, *haz_max_v = nullptr;
    int* haz_cnt = nullptr;
    // coupling pass (get_gradhs_w) buffers, sized for the largest window so far
    int cw_nodes = 0;
    double *cw_a1 = nullptr, *cw_a2 = nullptr;
    float *cw_hs = nullptr, *cw_ml = nullptr;
    float2 *cw_rhs = nullptr, *cw_g0 = nullptr, *cw_g1 = nullptr;
    gfsph_cg* cw_cg = nullptr;  // mass-matrix CG of the last window (niter = 0)
    int cw_key[4] = {-1, -1, -1, -1};
};

namespace {

int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return GFSPH_OK;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return GFSPH_ERR_NO_DEVICE;
    return GFSPH_ERR_CUDA;
}

#define CK(x)                                   \
    do {                                        \
        cudaError_t e_ = (x);                   \
        if (e_ != cudaSuccess) return cuda_status(e_); \
    } while (0)

void drop_graphs(gfsph_handle* h) {
    if (h->g1) cudaGraphExecDestroy(h->g1);
    if (h->gK) cudaGraphExecDestroy(h->gK);
    h->g1 = h->gK = nullptr;
}

// Adds the time of the last launch of kernel k to its profile.
void collect_one(gfsph_handle* h, int k) {
    float ms = 0.f;
    cudaEventSynchronize(h->ev1[k]);
    cudaEventElapsedTime(&ms, h->ev0[k], h->ev1[k]);
    h->prof_ms[k] += ms;
    h->prof_cnt[k] += 1;
    h->pending[k] = false;
}

template <class F>
void launch(gfsph_handle* h, int kid, F&& f) {
    if (h->profile && h->pending[kid]) collect_one(h, kid);  // launched again before the step's collection
    if (h->profile) cudaEventRecord(h->ev0[kid], h->stream);
    f();
    if (h->profile) {
        cudaEventRecord(h->ev1[kid], h->stream);
        h->pending[kid] = true;
    }
    h->launches++;
}

int profile_collect(gfsph_handle* h) {
    if (!h->profile) return 0;
    CK(cudaStreamSynchronize(h->stream));
    for (int k = 0; k < K_COUNT; k++)
        if (h->pending[k]) collect_one(h, k);
    return 0;
}

// Side stream for the coarse-level kernels while a graph is captured.
cudaStream_t side_stream(gfsph_handle* h) { return h->capturing ? h->stream2 : h->stream; }

// Calls f with std::integral_constant<int, skf>: the neighbour kernels are
// compiled per SPH kernel function (skf 1 to 4).
template <class F>
void with_skf(const gfsph_handle* h, F&& f) {
    switch (h->rheo.skf) {
    case 1: f(std::integral_constant<int, 1>{}); break;
    case 2: f(std::integral_constant<int, 2>{}); break;
    case 3: f(std::integral_constant<int, 3>{}); break;
    default: f(std::integral_constant<int, 4>{}); break;
    }
}

// Stage-dependent pressure: the step runs the staged RK45 kernels.
bool staged(const gfsph_handle* h) { return h->rheo.nor_density || h->rheo.cos_theta || h->rheo.ws; }

void fork(gfsph_handle* h, int k) {
    if (!h->capturing) return;
    cudaEventRecord(h->ev_fork[k], h->stream);
    cudaStreamWaitEvent(h->stream2, h->ev_fork[k], 0);
}

void join(gfsph_handle* h, int k) {
    if (!h->capturing) return;
    cudaEventRecord(h->ev_join[k], h->stream2);
    cudaStreamWaitEvent(h->stream, h->ev_join[k], 0);
}

Search make_search(gfsph_handle* h) {
    Search q;
    q.bstart = h->bstart;
    q.start = h->start;
    q.cellA = h->cellA;
    q.xhm = h->xhm;
    q.nbr = h->nbr;
    q.ncount = h->ncount;
    q.pterm = h->pterm;
    q.pr = h->pr;
    q.indv = h->indv;
    q.rho0 = h->rho0;
    q.rcell = h->rcell;
    q.xsv = h->xsv;
    q.spec = h->spec_a;
    q.zpw = h->zpw;
    q.gzw = h->gzw;
    q.bxy = h->bxy;
    q.mass0 = h->mass0_u;
    q.kcap = h->kcap;
    return q;
}

int big_blocks(const gfsph_handle*) { return 148 * 16; }  // 128 threads: one warp per coarse-level particle

// The cell search: bounds, grid, counting sort, reorder, neighbours+density.
// Returns the number of kernels enqueued.
int enqueue_search(gfsph_handle* h, int advance) {
    const int n = h->n;
    cudaStream_t st = h->stream;
    StepScalars* S = h->S;
    Search q = make_search(h);
    int nk = 0;
    int pb = blocks_for(n);
    int nscan = (h->cap_cells + kScanTile - 1) / kScanTile;
    int nbscan = (h->cap_blocks + kScanTile - 1) / kScanTile;
    const int* nblk = reinterpret_cast<const int*>(reinterpret_cast<const char*>(S) + offsetof(StepScalars, nblocks));
    const int* ncel = reinterpret_cast<const int*>(reinterpret_cast<const char*>(S) + offsetof(StepScalars, ncells));
    if (!advance) { launch(h, K_PREP, [&] { pdl_launch(k_prep, 1, 32, st, S, advance); }); nk++; }
    const GridArgs ga{h->cap_blocks, h->cap_cells, kMaxCells, h->level_factor, h->cell_div, h->reg_levels};
    launch(h, K_BOUNDS, [&] {
        pdl_launch(k_bounds, kBoundsBlocks, kThreadsBounds, st, h->B, n, h->rheo, h->dem, S, h->bparts, ga);
    }); nk++;
    launch(h, K_MARK, [&] { pdl_launch(k_mark, pb, kThreads, st, h->B, n, h->dem, S, h->bmark); }); nk++;
    launch(h, K_BSCAN_TILES, [&] {
        pdl_launch(k_scan_tiles, nbscan, kScanThreads, st, h->bmark, h->bstart, h->tile_sum, nblk, S, 1);
    }); nk++;
    launch(h, K_BSCAN_ADD, [&] { pdl_launch(k_scan_add, nbscan, kScanThreads, st, h->bstart, h->tile_sum, nblk, S, 1); }); nk++;
    launch(h, K_HIST, [&] {
        pdl_launch(k_hist, pb, kThreads, st, h->B, n, h->dem, S, h->bmark, h->bstart, h->count, h->keyrank, h->cap_cells);
    }); nk++;
    launch(h, K_SCAN_TILES, [&] {
        pdl_launch(k_scan_tiles, nscan, kScanThreads, st, h->count, h->start, h->tile_sum, ncel, S, 0);
    }); nk++;
    launch(h, K_SCAN_ADD, [&] { pdl_launch(k_scan_add, nscan, kScanThreads, st, h->start, h->tile_sum, ncel, S, 0); }); nk++;
    launch(h, K_SCATTER, [&] { pdl_launch(k_scatter, pb, kThreads, st, h->keyrank, n, h->start, h->bstart, S, h->perm); }); nk++;
    launch(h, K_CELL_SORT, [&] { pdl_launch(k_cell_sort, 148 * 4, 128, st, h->perm, h->B.id, h->start, h->count, S); }); nk++;
    launch(h, K_REORDER, [&] {
        pdl_launch(k_reorder, pb, kThreads, st, h->B, n, h->perm, h->keyrank, h->A, h->cellA, h->xhm, S, h->rheo, h->rho0,
                                           h->rcell, h->spec_u, h->spec_a);
    }); nk++;
    // the coarse-level kernels run beside the regular ones when graphs are
    // captured (side stream); serially otherwise
    cudaStream_t sb = side_stream(h);
    fork(h, 0);
    with_skf(h, [&](auto sk) {
        constexpr int SKF = decltype(sk)::value;
        launch(h, K_DENSITY_BIG, [&] { pdl_launch(k_density_big<SKF>, big_blocks(h), 128, sb, h->A, q, S, h->rheo); });
        // the two materials' pair types compiled in only when there are two
        if (h->rheo.ws) {
            launch(h, K_DENSITY, [&] { pdl_launch(k_density<false, SKF, true>, pb, kThreads, st, h->A, q, S, h->rheo, n); });
            launch(h, K_DENSITY_SPARSE,
                   [&] { pdl_launch(k_density<true, SKF, true>, pb, kThreads, st, h->A, q, S, h->rheo, n); });
        } else {
            launch(h, K_DENSITY, [&] { pdl_launch(k_density<false, SKF, false>, pb, kThreads, st, h->A, q, S, h->rheo, n); });
            launch(h, K_DENSITY_SPARSE,
                   [&] { pdl_launch(k_density<true, SKF, false>, pb, kThreads, st, h->A, q, S, h->rheo, n); });
        }
    });
    nk += 3;
    join(h, 0);
    return nk;
}

// The five depths of a step with nor_density: call k of sum_density_Tools
// reads the depths of call k-1 (rho0 for the first), clamped to h_inf after
// the first (IntForces_SW ran in between).  Without nor_density every stage
// uses the plain sum in A.rho.  Returns the number of kernels enqueued.
int enqueue_norms(gfsph_handle* h, PState As[5]) {
    const int n = h->n;
    cudaStream_t st = h->stream;
    const Rheo& c = h->rheo;
    Search q = make_search(h);
    int nk = 0;
    for (int k = 0; k < 5; k++) {
        As[k] = h->A;
        if (c.nor_density) As[k].rho = h->rhoS + (size_t)k * n;
    }
    if (!c.nor_density) return 0;
    for (int k = 0; k < 5; k++) {
        const float* hp = k ? As[k - 1].rho : h->rho0;
        const int clamp = k ? 1 : 0;
        launch(h, K_NORM, [&] {
            with_skf(h, [&](auto sk) {
                pdl_launch(k_norm<decltype(sk)::value>, blocks_for(n), kThreads, st, h->A, q, h->S, c, n, hp, clamp, As[k].rho);
            });
        });
        launch(h, K_NORM_BIG, [&] {
            with_skf(h, [&](auto sk) {
                pdl_launch(k_norm_big<decltype(sk)::value>, big_blocks(h), 128, st, h->A, q, h->S, c, hp, clamp, As[k].rho);
            });
        });
        nk += 2;
    }
    return nk;
}

// Pressure term of the first stage; with nor_density it takes the first
// normalised depth.
int enqueue_stage_begin(gfsph_handle* h, const PState As[5]) {
    const Rheo& c = h->rheo;
    Search q = make_search(h);
    launch(h, K_STAGE, [&] {
        if (c.cos_theta)
            pdl_launch(k_stage_begin<true>, blocks_for(h->n), kThreads, h->stream, h->A, q, h->S, c, h->dem, As[0].rho);
        else
            pdl_launch(k_stage_begin<false>, blocks_for(h->n), kThreads, h->stream, h->A, q, h->S, c, h->dem, As[0].rho);
    });
    return 1;
}

// The soil surface under the water in stage s (ic_ws_Interact = 1): the
// soil depths spread over the DEM nodes at the stage positions, Z + hs per
// node, then Zp at the water particles and every particle's pressure term.
int enqueue_wir_stage(gfsph_handle* h, const PState As[5], int s) {
    const int n = h->n;
    cudaStream_t st = h->stream;
    StepScalars* S = h->S;
    const Rheo& c = h->rheo;
    Search q = make_search(h);
    const int np = h->nx * h->ny;
    launch(h, K_WIR, [&] {
        pdl_launch(k_wir_scatter, blocks_for(n), kThreads, st, h->A, q, S, c, h->dem, h->carry, s, As[s].rho, h->wir_acc);
    });
    launch(h, K_WIR, [&] {
        pdl_launch(k_wir_nodes, blocks_for((long long)np, 256), 256, st, h->wir_acc, h->d_z, h->wir_hsz, np, S);
    });
    launch(h, K_WIR, [&] {
        pdl_launch(k_wir_press, blocks_for(n), kThreads, st, h->A, q, S, c, h->dem, h->carry, s, As[s].rho, h->wir_hsz);
    });
    return 3;
}

// The staged RK45 body (nor_density or ic_cosTheta = 1): per stage the
// internal force with that stage's pressure, then the stage of every
// particle; the last stage finishes the step.  Everything on one stream.
int enqueue_stages(gfsph_handle* h, PState As[5]) {
    const int n = h->n;
    cudaStream_t st = h->stream;
    StepScalars* S = h->S;
    const Rheo& c = h->rheo;
    Search q = make_search(h);
    const int pb = blocks_for(n);
    int nk = enqueue_norms(h, As);
    if (c.ws) {
        with_skf(h, [&](auto sk) {
            launch(h, K_WIR, [&] {
                pdl_launch(k_wir_pairs_big<decltype(sk)::value>, big_blocks(h), 128, st, h->A, q, S, c);
            });
        });
        nk += 1 + enqueue_wir_stage(h, As, 0);
    } else {
        nk += enqueue_stage_begin(h, As);
    }
    for (int s = 0; s < 4; s++) {
        launch(h, K_FORCE_BIG, [&] {
            with_skf(h, [&](auto sk) { pdl_launch(k_force_big<decltype(sk)::value>, big_blocks(h), 128, st, As[s], q, S, c); });
        });
        nk++;
        launch(h, K_IFORCE, [&] {
            with_skf(h, [&](auto sk) {
                if (c.ws)
                    pdl_launch(k_iforce<decltype(sk)::value, true>, pb, kThreads, st, As[s], q, S, c, n);
                else
                    pdl_launch(k_iforce<decltype(sk)::value, false>, pb, kThreads, st, As[s], q, S, c, n);
            });
        });
        nk++;
        launch(h, K_STAGE, [&] {
            // hprev: the depth the previous stage left (icpwp 1's bound)
            const float* hprev = (s > 0) ? As[s - 1].rho : As[0].rho;
            if (s < 3) {
                if (c.cos_theta)
                    pdl_launch(k_stage<true>, pb, kThreads, st, h->A, q, S, c, h->dem, h->carry, s, As[s].rho,
                               As[s + 1].rho, hprev);
                else
                    pdl_launch(k_stage<false>, pb, kThreads, st, h->A, q, S, c, h->dem, h->carry, s, As[s].rho,
                               As[s + 1].rho, hprev);
            } else if (c.cos_theta) {
                pdl_launch(k_stage_final<true>, pb, kThreads, st, h->A, q, S, c, h->dem, n, h->B, h->velfin, h->d_auxv,
                           h->carry, As[3].rho, As[4].rho, hprev);
            } else {
                pdl_launch(k_stage_final<false>, pb, kThreads, st, h->A, q, S, c, h->dem, n, h->B, h->velfin, h->d_auxv,
                           h->carry, As[3].rho, As[4].rho, hprev);
            }
        });
        nk++;
        if (c.ws && s < 3) nk += enqueue_wir_stage(h, As, s + 1);
    }
    return nk;
}

// The DEM update of the erosion (its last block ends the step), or the step
// end alone.  Returns the number of kernels enqueued.
int enqueue_step_end(gfsph_handle* h) {
    StepScalars* S = h->S;
    if (h->rheo.erosion)
        launch(h, K_DEM_ERODE, [&] {
            pdl_launch(k_dem_erode, 148 * 2, 256, h->stream, h->d_auxv, h->d_z, h->d_eroded, h->d_avail, h->nx, S);
        });
    else
        launch(h, K_STEP_END, [&] { pdl_launch(k_step_end, 1, 32, h->stream, S); });
    return 1;
}

// Enqueues one step; returns the number of kernels it enqueued (not a
// status: a failed launch surfaces through cudaGetLastError, which every
// caller checks after the enqueue or the capture).
int enqueue_step(gfsph_handle* h) {
    const int n = h->n;
    cudaStream_t st = h->stream;
    StepScalars* S = h->S;
    Search q = make_search(h);
    int pb = blocks_for(n);
    int nk = enqueue_search(h, 1);
    if (staged(h)) {
        PState As[5];
        nk += enqueue_stages(h, As);
        if (h->rheo.av_vel) {  // av_vel with the final depth
            launch(h, K_XSPH_BIG, [&] {
                with_skf(h, [&](auto sk) {
                    pdl_launch(k_xsph_big<decltype(sk)::value>, big_blocks(h), 128, st, As[4], q, S, h->rheo, h->B);
                });
            });
            launch(h, K_XSPH, [&] {
                with_skf(h, [&](auto sk) {
                    if (h->rheo.ws)
                        pdl_launch(k_xsph<decltype(sk)::value, true>, pb, kThreads, st, As[4], q, S, h->rheo, n, h->B);
                    else
                        pdl_launch(k_xsph<decltype(sk)::value, false>, pb, kThreads, st, As[4], q, S, h->rheo, n, h->B);
                });
            });
            nk += 2;
        }
        nk += enqueue_step_end(h);
        return nk;
    }
    cudaStream_t sb = side_stream(h);
    fork(h, 1);
    launch(h, K_FORCE_BIG, [&] {
        with_skf(h, [&](auto sk) { pdl_launch(k_force_big<decltype(sk)::value>, big_blocks(h), 128, sb, h->A, q, S, h->rheo); });
    });
    nk++;
    launch(h, K_IFORCE, [&] {
        with_skf(h, [&](auto sk) { pdl_launch(k_iforce<decltype(sk)::value, false>, pb, kThreads, st, h->A, q, S, h->rheo, n); });
    });
    nk++;
    join(h, 1);
    launch(h, K_FORCE_RK, [&] {
        const Rheo& c = h->rheo;
        const bool gen = !(c.nfric == 4 || (c.nfric >= 5 && c.nfric <= 8) || c.nfric == 26 || c.nfric == 27) ||
                         (c.erosion && c.eros_law != 1);
        auto kf = (c.icpwp == 1) ? (gen ? k_force_rk<true, true> : k_force_rk<true, false>)
                                 : (gen ? k_force_rk<false, true> : k_force_rk<false, false>);
        pdl_launch(kf, pb, kThreads, st, h->A, q, S, h->rheo, h->dem, n, h->B, h->velfin, h->d_auxv, 0, nullptr);
    }); nk++;
    if (h->rheo.av_vel) {
        fork(h, 2);
        launch(h, K_XSPH_BIG, [&] {
            with_skf(h, [&](auto sk) {
                pdl_launch(k_xsph_big<decltype(sk)::value>, big_blocks(h), 128, sb, h->A, q, S, h->rheo, h->B);
            });
        });
        nk++;
        launch(h, K_XSPH, [&] {
            with_skf(h, [&](auto sk) {
                pdl_launch(k_xsph<decltype(sk)::value, false>, pb, kThreads, st, h->A, q, S, h->rheo, n, h->B);
            });
        });
        nk++;
        join(h, 2);
    }
    nk += enqueue_step_end(h);
    return nk;
}

int build_graph(gfsph_handle* h, int steps, cudaGraphExec_t* out) {
    cudaGraph_t g = nullptr;
    long long before = h->launches;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    h->capturing = true;
    for (int s = 0; s < steps; s++) enqueue_step(h);
    h->capturing = false;
    // a launch that failed during the capture (bad configuration) is reported
    // after the capture has been ended, so the stream leaves capture mode
    const cudaError_t le = cudaGetLastError();
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    h->launches = before;  // capture launches nothing
    if (le != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return cuda_status(le);
    }
    if (e != cudaSuccess) return cuda_status(e);
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    return cuda_status(e);
}

int kernels_per_step(const gfsph_handle* h) {
    // staged: 10 k_norm launches with nor_density, k_stage_begin (with soil
    // and water: k_wir_pairs_big and per stage k_wir_scatter, k_wir_nodes,
    // k_wir_press), four stages of (k_force_big, k_iforce, k_stage)
    const int body = staged(h) ? (h->rheo.nor_density ? 10 : 0) + (h->rheo.ws ? 13 : 1) + 12 : 3;
    return 13 + body + (h->rheo.av_vel ? 2 : 0) + 1;
}

// The three buffer (re)allocations below drop the graphs (which hold the old
// buffers) and zero the capacity before freeing; on failure they leave the
// buffers freed and the capacity 0.
int alloc_blocks(gfsph_handle* h, int cap) {
    if (cap > kMaxCells) return GFSPH_ERR_CAPACITY;
    drop_graphs(h);
    h->cap_blocks = 0;
    dfree(h->bmark); dfree(h->bstart);
    int st = 0;
    st |= dalloc(&h->bmark, (size_t)cap + 1);
    st |= dalloc(&h->bstart, (size_t)cap + 1);
    if (st) { dfree(h->bmark); dfree(h->bstart); return GFSPH_ERR_CUDA; }
    CK(cudaMemsetAsync(h->bmark, 0, ((size_t)cap + 1) * sizeof(int), h->stream));
    h->cap_blocks = cap;
    return 0;
}

int alloc_cells(gfsph_handle* h, int cap) {
    if (cap > kMaxCells) return GFSPH_ERR_CAPACITY;
    drop_graphs(h);
    h->cap_cells = 0;
    dfree(h->count); dfree(h->start); dfree(h->tile_sum);
    int st = 0;
    st |= dalloc(&h->count, (size_t)cap + 1);
    st |= dalloc(&h->start, (size_t)cap + 1);
    st |= dalloc(&h->tile_sum, 8192);
    if (st) { dfree(h->count); dfree(h->start); dfree(h->tile_sum); return GFSPH_ERR_CUDA; }
    CK(cudaMemsetAsync(h->count, 0, ((size_t)cap + 1) * sizeof(int), h->stream));
    h->cap_cells = cap;
    return 0;
}

int alloc_nbr(gfsph_handle* h, int kcap) {
    drop_graphs(h);
    h->kcap = 0;
    dfree(h->nbr);
    const size_t rows = ((size_t)std::max(h->n, 1) + 31) / 32 * 32;  // whole warps (tab_base)
    if (dalloc(&h->nbr, (size_t)kcap * rows)) return GFSPH_ERR_CUDA;
    h->kcap = kcap;
    return 0;
}

void free_pstate(PState* p) {
    dfree(p->pos); dfree(p->vel); dfree(p->rho); dfree(p->mass); dfree(p->hsml); dfree(p->flag); dfree(p->id);
    dfree(p->pwp);
}

void free_particles(gfsph_handle* h) {
    PState* sets[3] = {&h->A, &h->B, &h->U};
    for (PState* p : sets) {
        dfree(p->pos); dfree(p->vel); dfree(p->rho); dfree(p->mass); dfree(p->hsml); dfree(p->flag); dfree(p->id);
        dfree(p->pwp);
    }
    dfree(h->cellA); dfree(h->velfin); dfree(h->pterm); dfree(h->keyrank); dfree(h->perm); dfree(h->ncount);
    dfree(h->nbr); dfree(h->f2tmp); dfree(h->xhm); dfree(h->indv); dfree(h->rho0);
    dfree(h->carry.v); dfree(h->carry.acc); dfree(h->carry.dx); dfree(h->carry.dv); dfree(h->carry.xo);
    dfree(h->carry.out); dfree(h->carry.u); dfree(h->carry.du); dfree(h->carry.Du); dfree(h->rhoS); dfree(h->rcell); dfree(h->xsv); dfree(h->pr);
    dfree(h->spec_u); dfree(h->spec_a); dfree(h->zpw); dfree(h->gzw); dfree(h->bxy);
    dfree(h->mass0_u);
    h->kcap = 0;
}

// After a failed device allocation: the handle keeps no particle state, no
// graphs and no buffers (every call but gfsph_upload then returns
// GFSPH_ERR_STATE); the next gfsph_upload allocates afresh.  Returns err.
int drop_state(gfsph_handle* h, int err) {
    drop_graphs(h);
    free_particles(h);
    dfree(h->count); dfree(h->start); dfree(h->tile_sum); dfree(h->bmark); dfree(h->bstart);
    h->cap_cells = 0;
    h->cap_blocks = 0;
    h->n = 0;
    h->has_state = false;
    h->searched = false;
    return err;
}

int alloc_pstate(PState* p, int n) {
    int st = 0;
    st |= dalloc(&p->pos, n); st |= dalloc(&p->vel, n); st |= dalloc(&p->rho, n); st |= dalloc(&p->mass, n);
    st |= dalloc(&p->hsml, n); st |= dalloc(&p->flag, n); st |= dalloc(&p->id, n); st |= dalloc(&p->pwp, n);
    return st;
}

// Reads the scalars back (synchronises the stream).
int read_scalars(gfsph_handle* h) {
    CK(cudaMemcpyAsync(h->hS, h->S, sizeof(StepScalars), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return 0;
}

template <class T>
int set_field(gfsph_handle* h, size_t off, T value) {
    T* host = reinterpret_cast<T*>(reinterpret_cast<char*>(h->hS) + off);
    *host = value;
    CK(cudaMemcpyAsync(reinterpret_cast<char*>(h->S) + off, host, sizeof(T), cudaMemcpyHostToDevice, h->stream));
    return 0;
}

// After a step batch stopped on a capacity error: grow and clear the error.
int grow_after_error(gfsph_handle* h) {
    StepScalars* s = h->hS;
    int e = s->err;
    if (e & kErrNonFinite) return GFSPH_ERR_NONFINITE;
    if (e & kErrEmpty) return GFSPH_ERR_DOMAIN;
    if (e & kErrCells) {
        long long want = std::max<long long>((long long)s->need_cells * 2, (long long)h->cap_cells * 2);
        if (want > kMaxCells) want = kMaxCells;
        if (want < s->need_cells) return GFSPH_ERR_CAPACITY;
        int st = alloc_cells(h, (int)want);
        if (st) return st == GFSPH_ERR_CUDA ? drop_state(h, st) : st;
        set_field<int>(h, offsetof(StepScalars, ncells), 0);
    }
    if (e & kErrBlocks) {
        long long want = std::max<long long>((long long)s->need_blocks * 2, (long long)h->cap_blocks * 2);
        if (want > kMaxCells) want = kMaxCells;
        if (want < s->need_blocks) return GFSPH_ERR_CAPACITY;
        int st = alloc_blocks(h, (int)want);
        if (st) return st == GFSPH_ERR_CUDA ? drop_state(h, st) : st;
    }
    if (e & kErrNbr) {
        int want = std::max(s->need_nbr + 16, h->kcap * 3 / 2);
        int st = alloc_nbr(h, want);
        if (st) return st == GFSPH_ERR_CUDA ? drop_state(h, st) : st;
    }
    set_field<int>(h, offsetof(StepScalars, err), 0);
    set_field<int>(h, offsetof(StepScalars, need_nbr), 0);
    set_field<int>(h, offsetof(StepScalars, need_big), 0);
    return 0;
}

// The tanfi density factor and the pore-water-pressure bounds:
// DFs_FSs_dens_and_pwp_factors (SPH_SW_2019.f90:8959-9060) for the friction,
// mini_DFs_dens_and_pwp_factors (:11502-11580) for Get_Pwp_SW's lower bound;
// ic_hrelSat = 0.
void pwp_factors(const gfsph_params* p, Rheo& c) {
    const float* k = p->cst;  // k[i-1] = const(i)
    const int fct = (int)(k[19] + 0.1f);
    const float dens = k[1], denss = k[16], densw = k[17], sr = k[18], alphas = k[13];
    c.icpwp = p->icpwp;
    c.fact_dens = 1.f; c.fact_pwp_max = 1.f; c.fact_pwp_min = 0.f; c.fpwp_max = 1.f; c.fpwp_min = 0.f;
    c.fpwp_min_g = 0.f;
    c.dens_bar = dens;  // ic_fct_dens = 0 (:8999-9008)
    c.dens_bar_eff = dens - ((densw < 1.e-3f) ? 1000.f : densw);
    if (fct == 1) {
        float porosity = (denss - dens) / (denss - densw);
        float dens2 = (1.f - porosity) * denss;
        float dens1 = (1.f - porosity) * denss + porosity * densw;
        float dens_bar = (1.f - alphas) * dens2 + alphas * dens1;
        float dens_bar_eff = dens_bar - densw * alphas;
        c.fact_dens = dens_bar_eff / dens_bar;
        c.dens_bar = dens_bar;
        c.dens_bar_eff = dens_bar_eff;
        if (p->icpwp > 0) {
            c.fact_pwp_max = 1.f + (alphas * densw) / dens_bar_eff;
            c.fpwp_min = -(alphas * densw) / dens_bar_eff;
            float g2 = (1.f - porosity) * denss + (porosity * densw) * sr;
            float gbar = (1.f - alphas) * g2 + alphas * dens1;
            float geff = gbar - densw * alphas;
            c.fpwp_min_g = -(alphas * densw) / geff;
        }
    }
    c.bfact = k[12];
    c.alphas = alphas;
    c.alphas2 = k[13] * k[13];
}

// Which quadratic nfric 23 solves for m = const(8) (SPH_SW_2019.f90:9578-9598):
// 0 for m = 1, 1 for m = 2, 2 for m within 1e-3 of 1/3 or m = 1/2, -1 for
// any other m (the reference stops there).
int hb_case(float m) {
    if (m == 1.f) return 0;
    if (m == 2.f) return 1;
    if (std::fabs(m - 0.333333f) <= 1.e-3f || m == 0.5f) return 2;
    return -1;
}

// The per-run constants of the Herschel-Bulkley laws, in the FP32 operations
// of SPH_SW_2019.f90:9541-9545 and :9609-9612 (real powers in FP64, rounded
// once).
void hb_constants(const float* k, Rheo& c) {
    const float m = k[7];
    c.m_vexp = m;
    c.hb_m = hb_case(m);
    const float cm = m / ((m + 1.f) * (2.f * m + 1.f));
    c.hb_a0 = (1.f / cm) * (float)std::pow((double)(k[6] / k[5]), (double)(1.f / m));
    c.hb_cm = 1.f;
    if (c.nfric == 25) c.hb_cm = (float)std::pow((double)((2.f * m + 1.f) / m), (double)m);
}

int validate(const gfsph_params* p) {
    int nfric = (int)(p->cst[4] + 0.01f);
    bool erosion = p->cst[20] > 1.e-9f;
    if (!(nfric == 1 || nfric == 2 || nfric == 3 || nfric == 4 || (nfric >= 5 && nfric <= 8) || nfric == 11 ||
          (nfric >= 23 && nfric <= 27)))
        return GFSPH_ERR_UNSUPPORTED;
    // Bingham and Herschel-Bulkley need a yield stress above 1e-32 (SPH_SW_2019.f90:9547-9550)
    if ((nfric == 4 || (nfric >= 23 && nfric <= 25)) && !(p->cst[5] >= 1.e-32f)) return GFSPH_ERR_ARG;
    if (nfric == 23 && hb_case(p->cst[7]) < 0) return GFSPH_ERR_UNSUPPORTED;
    // nfric 24/25 with m <= 0: (v/h)**m is infinite for a particle at rest
    if ((nfric == 24 || nfric == 25) && !(p->cst[7] > 0.f)) return GFSPH_ERR_ARG;
    const int eros_law = erosion ? (int)(p->cst[20] + 0.1f) : 0;
    if (erosion && (eros_law < 1 || eros_law > 3)) return GFSPH_ERR_UNSUPPORTED;
    if (eros_law == 3) {  // denss, densw (SPH_SW_2019.f90:10363-10367); constant dens_bar (ic_hrelSat 0)
        if (p->cst[16] <= 1.e-3f || p->cst[17] <= 1.e-3f) return GFSPH_ERR_ARG;
        if ((int)(p->cst[33] + 0.01f) != 0) return GFSPH_ERR_UNSUPPORTED;
    }
    if (eros_law == 2) {  // tanfi is a local of the frictional laws; denss, densw (SPH_SW_2019.f90:10337-10340)
        if (!((nfric >= 5 && nfric <= 8) || nfric == 26 || nfric == 27)) return GFSPH_ERR_UNSUPPORTED;
        if (p->cst[16] <= 1.e-3f || p->cst[17] <= 1.e-3f) return GFSPH_ERR_ARG;
    }
    if (p->skf < 1 || p->skf > 4) return GFSPH_ERR_UNSUPPORTED;
    // skf 2, 3 (support 3 h): the pair set depends on the reference's own
    // grid, reproduced for nnps 2; nnps 4 grids the principal-axes rotation
    // of FP32 running sums, which is order-dependent
    if ((p->skf == 2 || p->skf == 3) && p->nnps != 2) return GFSPH_ERR_UNSUPPORTED;
    if (p->pa_sph != 1 && p->pa_sph != 2) return GFSPH_ERR_UNSUPPORTED;
    if (p->nnps != 2 && p->nnps != 4) return GFSPH_ERR_UNSUPPORTED;
    if (p->max_neighbours < 0 || p->max_neighbours > kMaxNeighbours) return GFSPH_ERR_ARG;
    if (p->sle != 0 && p->sle != 1) return GFSPH_ERR_UNSUPPORTED;
    if (p->summation_density != 1 || (p->nor_density != 0 && p->nor_density != 1)) return GFSPH_ERR_UNSUPPORTED;
    if (p->ic_adapt != 0 && p->ic_adapt != 1 && p->ic_adapt != 2 && p->ic_adapt != 4 && p->ic_adapt != 10)
        return GFSPH_ERR_UNSUPPORTED;
    const int cos_theta = (int)(p->cst[15] + 0.01f);  // ic_cosTheta = const(16) (SPH_SW_2019.f90:6734)
    if (cos_theta != 0 && cos_theta != 1) return GFSPH_ERR_UNSUPPORTED;
    const int fct = (int)(p->cst[19] + 0.1f);                          // ic_fct_dens
    if (fct != 0 && fct != 1) return GFSPH_ERR_UNSUPPORTED;
    if (p->icpwp != 0 && p->icpwp != 1 && p->icpwp != 3) return GFSPH_ERR_UNSUPPORTED;
    if ((fct != 0 || p->icpwp != 0) && (int)(p->cst[33] + 0.01f) != 0) return GFSPH_ERR_UNSUPPORTED;  // ic_hrelSat
    if (p->icpwp == 3 && p->cst[25] > 0.f) return GFSPH_ERR_UNSUPPORTED;  // drag laws rescale Bfact
    if (fct == 1 && (p->cst[16] < 1.e-3f || p->cst[17] < 1.e-3f)) return GFSPH_ERR_ARG;  // denss, densw
    if (fct == 1 && p->icpwp != 0 && !(p->cst[13] > 0.01f)) return GFSPH_ERR_UNSUPPORTED;
    if (p->cst[0] < 0.f) return GFSPH_ERR_UNSUPPORTED;                 // inclined-plane gravity input
    if (p->cst[14] <= 1.e-8f || p->cst[9] <= 1.e-8f) return GFSPH_ERR_ARG;  // comp, hfrict0 (:1357-1365)
    if (!(p->dt > 0.f)) return GFSPH_ERR_ARG;
    if (p->ws_interact != 0 && p->ws_interact != 1) return GFSPH_ERR_UNSUPPORTED;
    if (p->sw_alg != 0 && p->sw_alg != 1) return GFSPH_ERR_UNSUPPORTED;
    if (p->ws_interact == 0 && p->sw_alg != 0) return GFSPH_ERR_UNSUPPORTED;  // ic_SWalg 1 of one material: not built
    // soil and water: no erosion, pore pressure, normalised density or
    // terrain-normal gravity with them here
    if (p->ws_interact == 1 && (erosion || p->icpwp != 0 || p->nor_density != 0 || cos_theta != 0))
        return GFSPH_ERR_UNSUPPORTED;
    // soil-water interface erosion (const(50) > 0) and friction (const(55) > 0), Input_SW
    // SPH_SW_2019.f90:1328-1345: not built
    if (p->ws_interact == 1 && (p->cst[49] > 0.f || p->cst[54] > 0.f)) return GFSPH_ERR_UNSUPPORTED;
    // grain crushing (const(36) > 0.01, :1312-1317), the solid-end laws (const(43) > 0, :1319-1325)
    // and the late Voellmy xi const(41) of ExtForces_SW (:8424-8434): not built
    if (p->cst[35] > 0.01f || p->cst[42] > 0.f || p->cst[40] > 1.e-6f) return GFSPH_ERR_UNSUPPORTED;
    return 0;
}

}  // namespace

extern "C" int gfsph_dem_topol(int mode, int nx, int ny, float dx, float dy, float* topol);

extern "C" {

int gfsph_version(void) { return 1; }

int gfsph_binary_version(int* version) try {
    if (!version) return GFSPH_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return GFSPH_ERR_NO_DEVICE;
    cudaFuncAttributes a{};
    CK(cudaFuncGetAttributes(&a, reinterpret_cast<const void*>(&k_prep)));
    *version = a.binaryVersion;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

const char* gfsph_strerror(int s) {
    switch (s) {
    case GFSPH_OK: return "ok";
    case GFSPH_T_END_REACHED: return "t_end reached";
    case GFSPH_ERR_ARG: return "invalid argument";
    case GFSPH_ERR_CUDA: return "CUDA runtime error";
    case GFSPH_ERR_CAPACITY: return "capacity exceeded";
    case GFSPH_ERR_UNSUPPORTED: return "unsupported option";
    case GFSPH_ERR_STATE: return "call out of order";
    case GFSPH_ERR_NO_DEVICE: return "no usable CUDA device";
    case GFSPH_ERR_NONFINITE: return "non-finite value in the particle state";
    case GFSPH_ERR_DOMAIN: return "no particle inside the DEM box";
    case GFSPH_ERR_HOST: return "host memory allocation failed";
    default: return "unknown status";
    }
}

int gfsph_num_kernels(void) { return K_COUNT; }
const char* gfsph_kernel_name(int k) { return (k >= 0 && k < K_COUNT) ? kKernelNames[k] : nullptr; }

}  // extern "C"

namespace {

__global__ void k_fill(float* a, size_t n, float v) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) a[k] = v;
}

// gfsph_create; with `share` the new handle uses share's device copy of the
// DEM slope and curvature rows (which erosion never changes) instead of its
// own, and takes its own copies of Z and the eroded depth from share (which
// must not have stepped yet) and its erodible depth from its parameters
// (Input_SW SPH_SW_2019.f90:1288-1307) or from share when the DEM was given
// as topol rows.  share must outlive the new handle.
int create_handle(const gfsph_params* p, const gfsph_dem* dem, gfsph_handle* share, gfsph_handle** out);

}  // namespace

extern "C" {

int gfsph_create(const gfsph_params* p, const gfsph_dem* dem, gfsph_handle** out) try {
    return create_handle(p, dem, nullptr, out);
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

}  // extern "C"

namespace {

int create_handle(const gfsph_params* p, const gfsph_dem* dem, gfsph_handle* share, gfsph_handle** out) {
    if (!p || !dem || !out) return GFSPH_ERR_ARG;
    *out = nullptr;
    int st = validate(p);
    if (st) return st;
    if (dem->nx < 3 || dem->ny < 3 || !(dem->dx > 0.f) || !(dem->dy > 0.f)) return GFSPH_ERR_ARG;
    if (!dem->topol && !dem->z) return GFSPH_ERR_ARG;
    if (dem->topol && dem->ntopo < 15) return GFSPH_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return GFSPH_ERR_NO_DEVICE;

    gfsph_handle* h = new (std::nothrow) gfsph_handle();
    if (!h) return GFSPH_ERR_HOST;
    cudaGetDevice(&h->dev);
    if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return GFSPH_ERR_CUDA;
    }
    h->stream = h->own_stream;
    if (cudaStreamCreateWithFlags(&h->stream2, cudaStreamNonBlocking) != cudaSuccess) {
        cudaStreamDestroy(h->own_stream);
        delete h;
        return GFSPH_ERR_CUDA;
    }
    for (int k = 0; k < 3; k++) {
        cudaEventCreateWithFlags(&h->ev_fork[k], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&h->ev_join[k], cudaEventDisableTiming);
    }
    h->P = *p;
    Rheo& c = h->rheo;
    const float* k = p->cst;  // k[i-1] = const(i)
    c.g = k[0]; c.dens = k[1]; c.xi = k[2]; c.tauy0 = k[5]; c.constK = k[6]; c.tanfi = k[8];
    c.hfrict0 = k[9]; c.comp = k[14]; c.keros = k[21];
    c.slip = (k[46] > 1.e-6f) ? (2.f * k[46]) / (1.f + k[46]) : 1.f;
    c.h_inf = p->h_inf;
    c.cgra05 = k[0] * 0.5f;
    c.nfric = (int)(k[4] + 0.01f);
    c.erosion = (k[20] > 1.e-9f) ? 1 : 0;
    c.eros_law = c.erosion ? (int)(k[20] + 0.1f) : 0;
    {  // erosion law 2, SPH_SW_2019.f90:10341-10350
        const float denss = k[16], densw = k[17];
        const float vol_conc = (k[1] - densw) / (denss - densw);
        c.er_xnum = (denss - densw) * vol_conc;
        c.er_xden = c.er_xnum + densw;
        c.er_kc = k[21] * k[22];
    }
    c.skf = p->skf; c.pa_sph = p->pa_sph; c.sle = p->sle; c.av_vel = p->average_velocity ? 1 : 0;
    c.ic_adapt = p->ic_adapt;
    c.nor_density = p->nor_density ? 1 : 0;
    c.cos_theta = ((int)(k[15] + 0.01f) == 1) ? 1 : 0;
    pwp_factors(p, c);
    // erosion law 3 with pwp_factors' dens_bar_eff, SPH_SW_2019.f90:10357-10376
    c.er_cb = k[22];
    c.er_c1 = c.dens_bar_eff * k[0];
    c.er_c2 = 1.f - k[24];
    c.er_tb = k[23];
    c.muI = (c.nfric == 8 || c.nfric == 26) ? 1 : (c.nfric == 27 ? 2 : 0);
    c.mu_a = k[2]; c.mu_r = k[5]; c.mu_b = k[6];
    if (c.muI) c.xi = 0.f;  // const(3) is a mu(I) parameter, not xi (:9653)
    hb_constants(k, c);
    c.ws = p->ws_interact;
    c.swalg = p->sw_alg;
    {
        const float densw = (k[17] < 1.e-3f) ? 1000.f : k[17];  // :9001
        c.dens_ws = densw / c.dens;
    }

    int nx = dem->nx, ny = dem->ny;
    size_t np = (size_t)nx * ny;
    if (share) {
        if (share->nx != nx || share->ny != ny) { gfsph_destroy(h); return GFSPH_ERR_ARG; }
        h->nx = nx; h->ny = ny;
        h->dem_shared = true;
        h->d_grad = share->d_grad; h->d_curvA = share->d_curvA; h->d_curvB = share->d_curvB;
        st = 0;
        st |= dalloc(&h->d_z, np); st |= dalloc(&h->d_eroded, np); st |= dalloc(&h->d_avail, np);
        st |= dalloc(&h->d_auxv, np);
        st |= dalloc(&h->S, 1);
        st |= dalloc(&h->bparts, kBoundsBlocks);
        if (st) { gfsph_destroy(h); return GFSPH_ERR_CUDA; }
        if (cudaMallocHost((void**)&h->hS, sizeof(StepScalars)) != cudaSuccess) { gfsph_destroy(h); return GFSPH_ERR_CUDA; }
        cudaMemcpy(h->d_z, share->d_z, np * sizeof(float), cudaMemcpyDeviceToDevice);
        cudaMemcpy(h->d_eroded, share->d_eroded, np * sizeof(float), cudaMemcpyDeviceToDevice);
        if (dem->topol) {
            cudaMemcpy(h->d_avail, share->d_avail, np * sizeof(float), cudaMemcpyDeviceToDevice);
        } else {
            float avail = 0.f;
            if (k[20] > 1.e-9f) avail = (k[47] > 1.e-6f) ? k[47] : 999.f;
            k_fill<<<blocks_for((long long)np, 256), 256>>>(h->d_avail, np, avail);
        }
        cudaMemset(h->d_auxv, 0, np * sizeof(double2));
        h->dem = share->dem;  // (the synchronous copy of the scalars below orders the fill before any step)
    } else {
    // DEM rows on the host, as Topo_main leaves them before the time loop
    std::vector<float> topol, z, er, av;
    std::vector<float2> grad, curvB;
    std::vector<float4> curvA;
    try {
        topol.assign(np * GFSPH_NTOPO, 0.f);
        grad.resize(np); curvB.resize(np); curvA.resize(np); z.resize(np); er.resize(np); av.resize(np);
    } catch (...) {
        gfsph_destroy(h);
        return GFSPH_ERR_HOST;
    }
    if (dem->topol) {
        for (size_t ip = 0; ip < np; ip++)
            for (int r = 0; r < 15; r++) topol[ip * GFSPH_NTOPO + r] = dem->topol[ip * (size_t)dem->ntopo + r];
    } else {
        for (size_t ip = 0; ip < np; ip++) topol[ip * GFSPH_NTOPO] = dem->z[ip];
        st = gfsph_dem_topol(p->dem_deriv, nx, ny, dem->dx, dem->dy, topol.data());
        if (st) { gfsph_destroy(h); return st; }
        // erodible depth, Input_SW SPH_SW_2019.f90:1288-1307
        float avail = 0.f;
        if (k[20] > 1.e-9f) avail = (k[47] > 1.e-6f) ? k[47] : 999.f;
        for (size_t ip = 0; ip < np; ip++) topol[ip * GFSPH_NTOPO + 14] = avail;
    }
    for (size_t ip = 0; ip < np; ip++) {
        const float* t = &topol[ip * GFSPH_NTOPO];
        z[ip] = t[0];
        grad[ip] = make_float2(t[1], t[2]);
        curvA[ip] = make_float4(t[3], t[4], t[5], t[6]);
        curvB[ip] = make_float2(t[7], t[8]);
        er[ip] = t[13];
        av[ip] = t[14];
    }
    h->nx = nx; h->ny = ny;
    st = 0;
    st |= dalloc(&h->d_grad, np); st |= dalloc(&h->d_curvA, np); st |= dalloc(&h->d_curvB, np);
    st |= dalloc(&h->d_z, np); st |= dalloc(&h->d_eroded, np); st |= dalloc(&h->d_avail, np);
    st |= dalloc(&h->d_auxv, np);
    st |= dalloc(&h->S, 1);
    st |= dalloc(&h->bparts, kBoundsBlocks);
    if (st) { gfsph_destroy(h); return GFSPH_ERR_CUDA; }
    if (cudaMallocHost((void**)&h->hS, sizeof(StepScalars)) != cudaSuccess) { gfsph_destroy(h); return GFSPH_ERR_CUDA; }
    cudaMemcpy(h->d_grad, grad.data(), np * sizeof(float2), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_curvA, curvA.data(), np * sizeof(float4), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_curvB, curvB.data(), np * sizeof(float2), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_z, z.data(), np * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_eroded, er.data(), np * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_avail, av.data(), np * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemset(h->d_auxv, 0, np * sizeof(double2));
    DemView& d = h->dem;
    d.nx = nx; d.ny = ny; d.xmin = dem->xmin; d.ymin = dem->ymin; d.dx = dem->dx; d.dy = dem->dy;
    d.xmax = d.xmin + (float)(nx - 1) * d.dx;
    d.ymax = d.ymin + (float)(ny - 1) * d.dy;
    d.grad = h->d_grad; d.curvA = h->d_curvA; d.curvB = h->d_curvB;
    }
    if (c.ws) {
        st = dalloc(&h->wir_hsz, np) | dalloc(&h->wir_acc, np);
        if (st) { gfsph_destroy(h); return GFSPH_ERR_CUDA; }
        cudaMemset(h->wir_acc, 0, np * sizeof(double2));
    }
    std::memset(h->hS, 0, sizeof(StepScalars));
    h->hS->dt = p->dt;
    h->hS->time = 0.0;
    h->hS->t_end = 1e300;
    cudaMemcpy(h->S, h->hS, sizeof(StepScalars), cudaMemcpyHostToDevice);
    for (int kk = 0; kk < K_COUNT; kk++) {
        cudaEventCreate(&h->ev0[kk]);
        cudaEventCreate(&h->ev1[kk]);
    }
    if (cudaGetLastError() != cudaSuccess) { gfsph_destroy(h); return GFSPH_ERR_CUDA; }
    *out = h;
    return GFSPH_OK;
}

}  // namespace

extern "C" {

int gfsph_destroy(gfsph_handle* h) try {
    if (!h) return GFSPH_ERR_ARG;
    if (h->stream) cudaStreamSynchronize(h->stream);
    drop_graphs(h);
    free_particles(h);
    dfree(h->count); dfree(h->start); dfree(h->tile_sum); dfree(h->bmark); dfree(h->bstart);
    if (!h->dem_shared) { dfree(h->d_grad); dfree(h->d_curvA); dfree(h->d_curvB); }
    dfree(h->d_z); dfree(h->d_eroded); dfree(h->d_avail);
    dfree(h->d_auxv); dfree(h->S); dfree(h->bparts); dfree(h->d_racc); dfree(h->d_rout); dfree(h->d_lam);
    dfree(h->d_lpart); dfree(h->wir_hsz); dfree(h->wir_acc);
    dfree(h->haz_sum_h); dfree(h->haz_sum_v); dfree(h->haz_max_h); dfree(h->haz_max_v); dfree(h->haz_cnt);
    dfree(h->cw_a1); dfree(h->cw_a2); dfree(h->cw_hs); dfree(h->cw_ml); dfree(h->cw_rhs); dfree(h->cw_g0);
    dfree(h->cw_g1);
    if (h->cw_cg) gfsph_cg_destroy(h->cw_cg);
    if (h->hS) cudaFreeHost(h->hS);
    for (int k = 0; k < K_COUNT; k++) {
        if (h->ev0[k]) cudaEventDestroy(h->ev0[k]);
        if (h->ev1[k]) cudaEventDestroy(h->ev1[k]);
    }
    for (int k = 0; k < 3; k++) {
        if (h->ev_fork[k]) cudaEventDestroy(h->ev_fork[k]);
        if (h->ev_join[k]) cudaEventDestroy(h->ev_join[k]);
    }
    if (h->stream2) cudaStreamDestroy(h->stream2);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    delete h;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_set_stream(gfsph_handle* h, void* stream) try {
    if (!h) return GFSPH_ERR_ARG;
    CK(cudaStreamSynchronize(h->stream));
    h->stream = stream ? (cudaStream_t)stream : h->own_stream;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_upload(gfsph_handle* h, int n, const float* x, const float* v, const float* rho, const float* mass,
                 const float* hsml, const int* itype, const int* out_flag) try {
    if (!h || n < 1 || !x || !v || !rho || !mass || !hsml) return GFSPH_ERR_ARG;
    if (itype)
        for (int i = 0; i < n; i++) {
            if (itype[i] == 1) continue;
            // water particles only with ic_ws_Interact = 1; no other types
            if (itype[i] != 2 || !h->rheo.ws) return GFSPH_ERR_UNSUPPORTED;
        }
    if (h->rheo.nfric == 3)  // nsoilB = (m - m0)/m; the reference stops for m <= 1e-6 (SPH_SW_2019.f90:9450-9453)
        for (int i = 0; i < n; i++)
            if (!(mass[i] > 1.e-6f)) return GFSPH_ERR_ARG;
    if (n != h->n) {
        CK(cudaStreamSynchronize(h->stream));
        drop_graphs(h);
        free_particles(h);
        h->has_state = false;
        h->n = n;
        int st = 0;
        st |= alloc_pstate(&h->A, n); st |= alloc_pstate(&h->B, n); st |= alloc_pstate(&h->U, n);
        st |= dalloc(&h->cellA, n); st |= dalloc(&h->velfin, n); st |= dalloc(&h->pterm, n);
        st |= dalloc(&h->keyrank, n); st |= dalloc(&h->perm, n); st |= dalloc(&h->ncount, n);
        st |= dalloc(&h->f2tmp, n); st |= dalloc(&h->xhm, n); st |= dalloc(&h->indv, n); st |= dalloc(&h->rho0, n);
        st |= dalloc(&h->xsv, n); st |= dalloc(&h->pr, n);
        if (staged(h)) {
            StageCarry& C = h->carry;
            st |= dalloc(&C.v, n); st |= dalloc(&C.acc, n); st |= dalloc(&C.dx, n); st |= dalloc(&C.dv, n);
            st |= dalloc(&C.xo, n); st |= dalloc(&C.out, n);
            if (h->rheo.icpwp == 1) { st |= dalloc(&C.u, n); st |= dalloc(&C.du, n); st |= dalloc(&C.Du, n); }
            if (h->rheo.nor_density) st |= dalloc(&h->rhoS, 5 * (size_t)n);
        }
        if (h->rheo.skf == 2 || h->rheo.skf == 3) st |= dalloc(&h->rcell, n);
        if (h->rheo.ws) {
            st |= dalloc(&h->spec_u, n); st |= dalloc(&h->spec_a, n); st |= dalloc(&h->zpw, n);
            st |= dalloc(&h->gzw, n); st |= dalloc(&h->bxy, n);
        }
        if (h->rheo.nfric == 3) st |= dalloc(&h->mass0_u, n);
        if (st) return drop_state(h, GFSPH_ERR_CUDA);
        st = alloc_nbr(h, h->P.max_neighbours > 0 ? h->P.max_neighbours : 96);
        if (st) return drop_state(h, st);
    }
    if (h->cap_cells == 0) {
        int st = alloc_cells(h, 1 << 18);
        if (st) return drop_state(h, st);
        set_field<int>(h, offsetof(StepScalars, ncells), 0);
    }
    if (h->cap_blocks == 0) {
        int st = alloc_blocks(h, 1 << 16);
        if (st) return drop_state(h, st);
    }
    cudaStream_t st = h->stream;
    CK(cudaMemcpyAsync(h->B.pos, x, (size_t)n * sizeof(float2), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(h->B.vel, v, (size_t)n * sizeof(float2), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(h->B.rho, rho, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(h->B.mass, mass, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, st));
    // mass0 = mass at the start of the run (Input_SW SPH_SW_2019.f90:1995)
    if (h->rheo.nfric == 3) CK(cudaMemcpyAsync(h->mass0_u, mass, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(h->B.hsml, hsml, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, st));
    if (out_flag) CK(cudaMemcpyAsync(h->B.flag, out_flag, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, st));
    else CK(cudaMemsetAsync(h->B.flag, 0, (size_t)n * sizeof(int), st));
    launch(h, K_UNSORT, [&] { k_iota<<<blocks_for(n), kThreads, 0, st>>>(h->B.id, n); });
    if (h->rheo.ws) {  // the material of each particle, in caller order
        std::vector<unsigned char> sp((size_t)n, 1);
        if (itype)
            for (int i = 0; i < n; i++) sp[i] = (unsigned char)itype[i];
        CK(cudaMemcpyAsync(h->spec_u, sp.data(), (size_t)n, cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));  // sp is a local
    }
    if (h->rheo.icpwp != 0)  // u (icpwp 1) or Uaux(1) (icpwp 3): the same start, :1724-1737, 1829-1852
        launch(h, K_UNSORT, [&] {
            k_pwp_init<<<blocks_for(n), kThreads, 0, st>>>(h->B.pwp, h->B.rho, n, h->P.pwp0rel, h->P.cst[13]);
        });
    else
        CK(cudaMemsetAsync(h->B.pwp, 0, (size_t)n * sizeof(float), st));
    CK(cudaGetLastError());
    h->has_state = true;
    h->searched = false;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_download(gfsph_handle* h, float* x, float* v, float* rho, float* mass, float* hsml, int* out_flag) try {
    if (!h) return GFSPH_ERR_ARG;
    if (!h->has_state) return GFSPH_ERR_STATE;
    int n = h->n;
    cudaStream_t st = h->stream;
    launch(h, K_UNSORT, [&] { k_unsort<<<blocks_for(n), kThreads, 0, st>>>(h->B, n, h->U); });
    if (x) CK(cudaMemcpyAsync(x, h->U.pos, (size_t)n * sizeof(float2), cudaMemcpyDeviceToHost, st));
    if (v) CK(cudaMemcpyAsync(v, h->U.vel, (size_t)n * sizeof(float2), cudaMemcpyDeviceToHost, st));
    if (rho) CK(cudaMemcpyAsync(rho, h->U.rho, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (mass) CK(cudaMemcpyAsync(mass, h->U.mass, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (hsml) CK(cudaMemcpyAsync(hsml, h->U.hsml, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (out_flag) CK(cudaMemcpyAsync(out_flag, h->U.flag, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_set_pwp(gfsph_handle* h, const float* pwp) try {
    if (!h || !pwp) return GFSPH_ERR_ARG;
    if (!h->has_state) return GFSPH_ERR_STATE;
    int n = h->n;
    cudaStream_t st = h->stream;
    CK(cudaMemcpyAsync(h->U.pwp, pwp, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, st));
    launch(h, K_UNSORT, [&] { k_gather_by_id<<<blocks_for(n), kThreads, 0, st>>>(h->U.pwp, h->B.id, n, h->B.pwp); });
    CK(cudaStreamSynchronize(st));
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_get_pwp(gfsph_handle* h, float* pwp) try {
    if (!h || !pwp) return GFSPH_ERR_ARG;
    if (!h->has_state) return GFSPH_ERR_STATE;
    int n = h->n;
    cudaStream_t st = h->stream;
    launch(h, K_UNSORT, [&] { k_unsort<<<blocks_for(n), kThreads, 0, st>>>(h->B, n, h->U); });
    CK(cudaMemcpyAsync(pwp, h->U.pwp, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_get_time(gfsph_handle* h, double* t, float* dt) try {
    if (!h) return GFSPH_ERR_ARG;
    int st = read_scalars(h);
    if (st) return st;
    if (t) *t = h->hS->time;
    if (dt) *dt = h->hS->dt;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_set_time(gfsph_handle* h, double t, float dt) try {
    if (!h || !(dt > 0.f)) return GFSPH_ERR_ARG;
    set_field<double>(h, offsetof(StepScalars, time), t);
    set_field<float>(h, offsetof(StepScalars, dt), dt);
    CK(cudaStreamSynchronize(h->stream));
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

}  // extern "C"

namespace {

// Enqueues one chunk of steps (no host synchronisation).
int enqueue_chunk(gfsph_handle* h, int chunk, double t_end) {
    set_field<double>(h, offsetof(StepScalars, t_end), t_end);
    set_field<int>(h, offsetof(StepScalars, steps_done), 0);
    launch(h, K_PREP, [&] { k_prep<<<1, 32, 0, h->stream>>>(h->S, 1); });
    if (h->profile) {
        for (int s = 0; s < chunk; s++) {
            enqueue_step(h);
            CK(cudaGetLastError());  // a launch of this step failed
            int st = profile_collect(h);
            if (st) return st;
        }
        return 0;
    }
    if (!h->g1) { int st = build_graph(h, 1, &h->g1); if (st) return st; }
    if (!h->gK) { int st = build_graph(h, kGraphSteps, &h->gK); if (st) return st; }
    int per = kernels_per_step(h);
    int s = 0;
    if (h->profile_level == 2) CK(cudaEventRecord(h->ev0[K_STEPS], h->stream));
    for (; s + kGraphSteps <= chunk; s += kGraphSteps) {
        CK(cudaGraphLaunch(h->gK, h->stream));
        h->launches += (long long)per * kGraphSteps;
    }
    for (; s < chunk; s++) {
        CK(cudaGraphLaunch(h->g1, h->stream));
        h->launches += per;
    }
    if (h->profile_level == 2) CK(cudaEventRecord(h->ev1[K_STEPS], h->stream));
    return 0;
}

// Waits for a chunk and handles its outcome: returns 1 to go on, 0 when
// t_end is reached, < 0 on error; `done` accumulates the completed steps.
int finish_chunk(gfsph_handle* h, int chunk, double t_end, int& done, int& guard) {
    if (h->profile_level == 2 && !h->profile) {
        CK(cudaEventSynchronize(h->ev1[K_STEPS]));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, h->ev0[K_STEPS], h->ev1[K_STEPS]);
        h->prof_ms[K_STEPS] += ms;
        h->prof_cnt[K_STEPS] += chunk;
    }
    CK(cudaGetLastError());
    int st = read_scalars(h);
    if (st) return st;
    done += h->hS->steps_done;
    h->searched = true;
    if (h->hS->err) {
        if (++guard > 16) return GFSPH_ERR_CAPACITY;
        st = grow_after_error(h);
        return st ? st : 1;
    }
    return (h->hS->time >= t_end) ? 0 : 1;
}

}  // namespace

extern "C" {

int gfsph_step(gfsph_handle* h, int nsteps, double t_end, double* t_out, int* steps_done) try {
    if (!h || nsteps < 0) return GFSPH_ERR_ARG;
    if (!h->has_state) return GFSPH_ERR_STATE;
    int done = 0, guard = 0, status = GFSPH_OK;
    while (done < nsteps) {
        int chunk = std::min(kChunkSteps, nsteps - done);
        int st = enqueue_chunk(h, chunk, t_end);
        if (st) return st;
        st = finish_chunk(h, chunk, t_end, done, guard);
        if (st < 0) { status = st; break; }
        if (st == 0) {
            if (done < nsteps) status = GFSPH_T_END_REACHED;
            break;
        }
    }
    if (t_out) *t_out = h->hS->time;
    if (steps_done) *steps_done = done;
    return status;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

// search + density on the current state (no advance); the state in B is
// replaced by the cell-sorted copy with the new densities.
static int search_only(gfsph_handle* h) {
    for (int tries = 0; tries < 16; tries++) {
        enqueue_search(h, 0);
        CK(cudaGetLastError());
        int st = profile_collect(h);
        if (st) return st;
        st = read_scalars(h);
        if (st) return st;
        if (h->hS->err) {
            st = grow_after_error(h);
            if (st) return st;
            continue;
        }
        h->searched = true;
        return 0;
    }
    return GFSPH_ERR_CAPACITY;
}

int gfsph_density(gfsph_handle* h, float* rho_out) try {
    if (!h) return GFSPH_ERR_ARG;
    if (!h->has_state) return GFSPH_ERR_STATE;
    int st = search_only(h);
    if (st) return st;
    int n = h->n;
    if (h->rheo.nor_density) {  // the first call of the step: normalised with the depths held
        Search q = make_search(h);
        launch(h, K_NORM, [&] {
            with_skf(h, [&](auto sk) {
                k_norm<decltype(sk)::value><<<blocks_for(n), kThreads, 0, h->stream>>>(h->A, q, h->S, h->rheo, n, h->rho0, 0,
                                                                                   h->rhoS);
            });
        });
        launch(h, K_NORM_BIG, [&] {
            with_skf(h, [&](auto sk) {
                k_norm_big<decltype(sk)::value><<<big_blocks(h), 128, 0, h->stream>>>(h->A, q, h->S, h->rheo, h->rho0, 0,
                                                                                     h->rhoS);
            });
        });
        CK(cudaMemcpyAsync(h->A.rho, h->rhoS, (size_t)n * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
    }
    launch(h, K_COPY, [&] { k_copy_state<<<blocks_for(n), kThreads, 0, h->stream>>>(h->A, h->B, n); });
    if (rho_out) return gfsph_download(h, nullptr, nullptr, rho_out, nullptr, nullptr, nullptr);
    CK(cudaStreamSynchronize(h->stream));
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_internal_forces(gfsph_handle* h, float* indvxdt) try {
    if (!h || !indvxdt) return GFSPH_ERR_ARG;
    if (!h->has_state) return GFSPH_ERR_STATE;
    int st = search_only(h);
    if (st) return st;
    int n = h->n;
    cudaStream_t s = h->stream;
    Search q = make_search(h);
    PState As[5];
    if (staged(h)) {  // the first stage's depth and pressure term
        enqueue_norms(h, As);
        enqueue_stage_begin(h, As);
    } else {
        As[0] = h->A;
    }
    launch(h, K_IFORCE, [&] {
        with_skf(h, [&](auto sk) { k_iforce<decltype(sk)::value, false><<<blocks_for(n), kThreads, 0, s>>>(As[0], q, h->S, h->rheo, n); });
    });
    launch(h, K_FORCE_BIG, [&] {
        with_skf(h, [&](auto sk) { k_force_big<decltype(sk)::value><<<big_blocks(h), 128, 0, s>>>(As[0], q, h->S, h->rheo); });
    });
    launch(h, K_FORCE_RK, [&] {
        k_force_rk<false, true><<<blocks_for(n), kThreads, 0, s>>>(h->A, q, h->S, h->rheo, h->dem, n, h->B,
                                                                  h->velfin, h->d_auxv, 1, h->velfin);
    });
    launch(h, K_UNSORT, [&] { k_unsort_f2<<<blocks_for(n), kThreads, 0, s>>>(h->velfin, h->A.id, n, h->f2tmp); });
    launch(h, K_COPY, [&] { k_copy_state<<<blocks_for(n), kThreads, 0, s>>>(h->A, h->B, n); });
    CK(cudaMemcpyAsync(indvxdt, h->f2tmp, (size_t)n * sizeof(float2), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_neighbours(gfsph_handle* h, int cap, int* offsets, int* idx) try {
    if (!h || !offsets) return GFSPH_ERR_ARG;
    if (!h->searched) return GFSPH_ERR_STATE;
    int n = h->n;
    int st = read_scalars(h);
    if (st) return st;
    int nreg = h->hS->nreg, nbig = h->hS->nbig;
    std::vector<int> cnt(n), id(n);
    std::vector<int4> tab((size_t)h->kcap * (((size_t)n + 31) / 32 * 32));
    CK(cudaMemcpy(cnt.data(), h->ncount, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(id.data(), h->A.id, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(tab.data(), h->nbr, tab.size() * sizeof(int4), cudaMemcpyDeviceToHost));
    std::vector<std::vector<int>> lists(n);
    for (int s = 0; s < nreg; s++) {
        auto& L = lists[id[s]];
        for (int k = 0; k < cnt[s] && k < h->kcap; k++)
            L.push_back(id[tab[tab_base(s, h->kcap) + (size_t)k * kTabStride].x & ~kCrossBit]);
    }
    if (nbig > 0) {  // pairs of the big particles, found on the device
        int pcap = 1 << 20;
        for (int tries = 0; tries < 8; tries++) {
            int2* dpairs = nullptr;
            int* dcount = nullptr;
            if (dalloc(&dpairs, pcap) || dalloc(&dcount, 1)) { dfree(dpairs); dfree(dcount); return GFSPH_ERR_CUDA; }
            cudaMemset(dcount, 0, sizeof(int));
            Search q = make_search(h);
            launch(h, K_EXPORT, [&] {
                with_skf(h, [&](auto sk) {
                    k_export_big<decltype(sk)::value><<<big_blocks(h), 128, 0, h->stream>>>(q, h->S, dpairs, dcount, pcap);
                });
            });
            cudaStreamSynchronize(h->stream);
            int np = 0;
            cudaMemcpy(&np, dcount, sizeof(int), cudaMemcpyDeviceToHost);
            if (np > pcap) { dfree(dpairs); dfree(dcount); pcap = np; continue; }
            std::vector<int2> pr;
            try {
                pr.resize(np);
            } catch (...) {
                dfree(dpairs); dfree(dcount);
                return GFSPH_ERR_HOST;
            }
            cudaMemcpy(pr.data(), dpairs, (size_t)np * sizeof(int2), cudaMemcpyDeviceToHost);
            dfree(dpairs); dfree(dcount);
            for (const int2& q2 : pr) lists[id[q2.x]].push_back(id[q2.y]);
            break;
        }
    }
    int tot = 0;
    for (int i = 0; i < n; i++) {
        auto& L = lists[i];
        std::sort(L.begin(), L.end());
        offsets[i] = tot;
        for (int j : L) {
            if (idx && tot < cap) idx[tot] = j;
            tot++;
        }
    }
    offsets[n] = tot;
    CK(cudaGetLastError());
    return (tot > cap) ? GFSPH_ERR_CAPACITY : GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_raster(gfsph_handle* h, int kind, float* out) try {
    if (!h || !out) return GFSPH_ERR_ARG;
    int np = h->nx * h->ny;
    cudaStream_t s = h->stream;
    int gb = blocks_for(np, 256);
    if (!h->d_rout && dalloc(&h->d_rout, np)) return GFSPH_ERR_CUDA;
    switch (kind) {
    case GFSPH_RASTER_DEPTH_IDW: {
        if (!h->has_state) return GFSPH_ERR_STATE;
        if (!h->d_racc && dalloc(&h->d_racc, np)) return GFSPH_ERR_CUDA;
        CK(cudaMemsetAsync(h->d_racc, 0, (size_t)np * sizeof(double2), s));
        launch(h, K_RASTER, [&] { k_raster_idw<<<blocks_for(h->n), kThreads, 0, s>>>(h->B, h->n, h->dem, h->d_racc); });
        launch(h, K_RASTER, [&] { k_raster_idw_finish<<<gb, 256, 0, s>>>(h->d_racc, h->d_rout, np); });
        break;
    }
    case GFSPH_RASTER_MAX_DEPTH:
    case GFSPH_RASTER_MAX_VEL:
    case GFSPH_RASTER_SUM_DEPTH:
    case GFSPH_RASTER_SUM_VEL:
    case GFSPH_RASTER_COUNT: {
        if (!h->haz_cnt) {
            CK(cudaMemsetAsync(h->d_rout, 0, (size_t)np * sizeof(float), s));
            break;
        }
        if (kind == GFSPH_RASTER_MAX_DEPTH) launch(h, K_HAZARD, [&] { k_hazard_finish<<<gb, 256, 0, s>>>(h->haz_max_h, h->d_rout, np); });
        if (kind == GFSPH_RASTER_MAX_VEL) launch(h, K_HAZARD, [&] { k_hazard_finish<<<gb, 256, 0, s>>>(h->haz_max_v, h->d_rout, np); });
        if (kind == GFSPH_RASTER_SUM_DEPTH) launch(h, K_HAZARD, [&] { k_d2f<<<gb, 256, 0, s>>>(h->haz_sum_h, h->d_rout, np); });
        if (kind == GFSPH_RASTER_SUM_VEL) launch(h, K_HAZARD, [&] { k_d2f<<<gb, 256, 0, s>>>(h->haz_sum_v, h->d_rout, np); });
        if (kind == GFSPH_RASTER_COUNT) launch(h, K_HAZARD, [&] { k_i2f<<<gb, 256, 0, s>>>(h->haz_cnt, h->d_rout, np); });
        break;
    }
    case GFSPH_RASTER_Z: CK(cudaMemcpyAsync(out, h->d_z, (size_t)np * sizeof(float), cudaMemcpyDeviceToHost, s)); break;
    case GFSPH_RASTER_ERODED: CK(cudaMemcpyAsync(out, h->d_eroded, (size_t)np * sizeof(float), cudaMemcpyDeviceToHost, s)); break;
    case GFSPH_RASTER_AVAILABLE: CK(cudaMemcpyAsync(out, h->d_avail, (size_t)np * sizeof(float), cudaMemcpyDeviceToHost, s)); break;
    default: return GFSPH_ERR_ARG;
    }
    if (kind <= GFSPH_RASTER_COUNT) CK(cudaMemcpyAsync(out, h->d_rout, (size_t)np * sizeof(float), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_raster_misfit(gfsph_handle* h, const float* target, double* loss, float* gx, float* gh) try {
    if (!h || !target || !loss) return GFSPH_ERR_ARG;
    if (!h->has_state) return GFSPH_ERR_STATE;
    const int np = h->nx * h->ny, n = h->n;
    cudaStream_t s = h->stream;
    const int gb = blocks_for(np, 256);
    if (!h->d_racc && dalloc(&h->d_racc, np)) return GFSPH_ERR_CUDA;
    if (!h->d_lam && dalloc(&h->d_lam, np)) return GFSPH_ERR_CUDA;
    if (!h->d_lpart && dalloc(&h->d_lpart, 148 * 64)) return GFSPH_ERR_CUDA;
    if (!h->d_rout && dalloc(&h->d_rout, np)) return GFSPH_ERR_CUDA;
    std::vector<double> part(gb);
    CK(cudaMemcpyAsync(h->d_rout, target, (size_t)np * sizeof(float), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(h->d_racc, 0, (size_t)np * sizeof(double2), s));
    launch(h, K_RASTER, [&] { k_raster_idw<<<blocks_for(n), kThreads, 0, s>>>(h->B, n, h->dem, h->d_racc); });
    launch(h, K_RASTER, [&] { k_misfit_nodes<<<gb, 256, 0, s>>>(h->d_racc, h->d_rout, np, h->d_lam, h->d_lpart); });
    if (gx || gh) {
        // U, the scratch of the caller-order copies, holds the gradients
        launch(h, K_RASTER, [&] {
            k_misfit_particles<<<blocks_for(n), kThreads, 0, s>>>(h->B, n, h->dem, h->d_racc, h->d_lam, h->U.pos,
                                                                  h->U.rho);
        });
        if (gx) CK(cudaMemcpyAsync(gx, h->U.pos, (size_t)n * sizeof(float2), cudaMemcpyDeviceToHost, s));
        if (gh) CK(cudaMemcpyAsync(gh, h->U.rho, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, s));
    }
    CK(cudaMemcpyAsync(part.data(), h->d_lpart, (size_t)gb * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    double l = 0.0;
    for (int b = 0; b < gb; b++) l += part[b];
    *loss = l;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_hazard_reset(gfsph_handle* h) try {
    if (!h) return GFSPH_ERR_ARG;
    int np = h->nx * h->ny;
    if (!h->haz_cnt) {
        int st = 0;
        st |= dalloc(&h->haz_sum_h, np); st |= dalloc(&h->haz_sum_v, np);
        st |= dalloc(&h->haz_max_h, np); st |= dalloc(&h->haz_max_v, np); st |= dalloc(&h->haz_cnt, np);
        if (st) {
            dfree(h->haz_sum_h); dfree(h->haz_sum_v); dfree(h->haz_max_h); dfree(h->haz_max_v); dfree(h->haz_cnt);
            return GFSPH_ERR_CUDA;
        }
    }
    cudaStream_t s = h->stream;
    CK(cudaMemsetAsync(h->haz_sum_h, 0, (size_t)np * sizeof(double), s));
    CK(cudaMemsetAsync(h->haz_sum_v, 0, (size_t)np * sizeof(double), s));
    CK(cudaMemsetAsync(h->haz_max_h, 0, (size_t)np * sizeof(unsigned int), s));
    CK(cudaMemsetAsync(h->haz_max_v, 0, (size_t)np * sizeof(unsigned int), s));
    CK(cudaMemsetAsync(h->haz_cnt, 0, (size_t)np * sizeof(int), s));
    CK(cudaStreamSynchronize(s));
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_hazard_sample(gfsph_handle* h) try {
    if (!h) return GFSPH_ERR_ARG;
    if (!h->has_state) return GFSPH_ERR_STATE;
    if (!h->haz_cnt) {
        int st = gfsph_hazard_reset(h);
        if (st) return st;
    }
    cudaStream_t s = h->stream;
    launch(h, K_HAZARD, [&] {
        k_hazard<<<blocks_for(h->n), kThreads, 0, s>>>(h->B, h->n, h->dem, h->haz_sum_h, h->haz_sum_v, h->haz_max_h,
                                                      h->haz_max_v, h->haz_cnt);
    });
    CK(cudaGetLastError());
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_profile(gfsph_handle* h, int enable) try {
    if (!h) return GFSPH_ERR_ARG;
    CK(cudaStreamSynchronize(h->stream));
    h->profile = enable == 1;
    h->profile_level = enable;
    for (int k = 0; k < K_COUNT; k++) { h->prof_ms[k] = 0; h->prof_cnt[k] = 0; h->pending[k] = false; }
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_profile_read(gfsph_handle* h, int kernel, double* total_ms, long long* launches) try {
    if (!h || kernel < 0 || kernel >= K_COUNT) return GFSPH_ERR_ARG;
    if (total_ms) *total_ms = h->prof_ms[kernel];
    if (launches) *launches = h->prof_cnt[kernel];
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

long long gfsph_launch_count(gfsph_handle* h) { return h ? h->launches : -1; }

// ---------------------------------------------------------------- ensembles

}  // extern "C"

struct gfsph_ensemble {
    std::vector<gfsph_handle*> members;
    int nx = 0, ny = 0;
    unsigned int** d_maxptr = nullptr;  // device array of the members' per-node max-depth buffers
    float* d_prob = nullptr;
};

namespace {

__global__ void k_exceedance(unsigned int* const* maxh, int nreal, int np, float threshold, float* prob) {
    unsigned int thr = f2o(threshold);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
        int c = 0;
        for (int r = 0; r < nreal; r++) c += (maxh[r][k] > thr) ? 1 : 0;  // max depth > threshold
        prob[k] = (float)c / (float)nreal;
    }
}

}  // namespace

extern "C" {

int gfsph_ensemble_create(const gfsph_params* params, const gfsph_dem* dem, int nreal, gfsph_ensemble** out) try {
    if (!params || !dem || !out || nreal < 1) return GFSPH_ERR_ARG;
    *out = nullptr;
    for (int r = 0; r < nreal; r++) {
        int st = validate(&params[r]);
        if (st) return st;
        if (params[r].dem_deriv != params[0].dem_deriv) return GFSPH_ERR_ARG;  // one set of DEM rows
    }
    // the DEM rows once on the host, shared by every member's copy
    std::vector<float> topol;
    gfsph_dem d = *dem;
    if (!dem->topol) {
        if (!dem->z || dem->nx < 3 || dem->ny < 3) return GFSPH_ERR_ARG;
        size_t np = (size_t)dem->nx * dem->ny;
        topol.assign(np * GFSPH_NTOPO, 0.f);
        for (size_t ip = 0; ip < np; ip++) topol[ip * GFSPH_NTOPO] = dem->z[ip];
        int st = gfsph_dem_topol(params[0].dem_deriv, dem->nx, dem->ny, dem->dx, dem->dy, topol.data());
        if (st) return st;
    }
    gfsph_ensemble* e = new (std::nothrow) gfsph_ensemble();
    if (!e) return GFSPH_ERR_HOST;
    try {
        e->members.reserve(nreal);  // no push_back below can throw with a handle in hand
    } catch (...) {
        delete e;
        return GFSPH_ERR_HOST;
    }
    e->nx = dem->nx; e->ny = dem->ny;
    // member 0 holds the one device copy of the DEM slope and curvature rows;
    // the others use it and keep their own Z, eroded and erodible depth
    for (int r = 0; r < nreal; r++) {
        gfsph_handle* h = nullptr;
        int st;
        if (r == 0) {
            gfsph_dem dm = d;
            if (!dem->topol) {  // erodible depth of member 0 (Input_SW SPH_SW_2019.f90:1288-1307)
                const float* k = params[0].cst;
                float avail = 0.f;
                if (k[20] > 1.e-9f) avail = (k[47] > 1.e-6f) ? k[47] : 999.f;
                size_t np = (size_t)dem->nx * dem->ny;
                for (size_t ip = 0; ip < np; ip++) topol[ip * GFSPH_NTOPO + 14] = avail;
                dm.topol = topol.data();
                dm.ntopo = GFSPH_NTOPO;
            }
            st = gfsph_create(&params[0], &dm, &h);
        } else {
            st = create_handle(&params[r], dem, e->members[0], &h);
        }
        if (st) { gfsph_ensemble_destroy(e); return st; }
        e->members.push_back(h);
    }
    *out = e;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_ensemble_destroy(gfsph_ensemble* e) try {
    if (!e) return GFSPH_ERR_ARG;
    // member 0 last: the others use its DEM rows
    for (size_t r = e->members.size(); r-- > 0;) gfsph_destroy(e->members[r]);
    dfree(e->d_maxptr);
    dfree(e->d_prob);
    delete e;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_ensemble_member(gfsph_ensemble* e, int r, gfsph_handle** out) try {
    if (!e || !out || r < 0 || r >= (int)e->members.size()) return GFSPH_ERR_ARG;
    *out = e->members[r];
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_ensemble_step(gfsph_ensemble* e, int nsteps, double t_end, int* min_steps_done) try {
    if (!e || nsteps < 0) return GFSPH_ERR_ARG;
    const int R = (int)e->members.size();
    for (gfsph_handle* h : e->members)
        if (!h->has_state) return GFSPH_ERR_STATE;
    std::vector<int> done(R, 0), guard(R, 0), active(R, 1);
    int status = GFSPH_OK, err = GFSPH_OK;
    while (err == GFSPH_OK) {
        bool any = false;
        std::vector<int> chunk(R, 0);
        for (int r = 0; r < R && err == GFSPH_OK; r++) {  // every member's chunk goes out before any wait
            if (!active[r] || done[r] >= nsteps) { active[r] = 0; continue; }
            int st = enqueue_chunk(e->members[r], std::min(kChunkSteps, nsteps - done[r]), t_end);
            if (st) { err = st; break; }
            chunk[r] = std::min(kChunkSteps, nsteps - done[r]);
            any = true;
        }
        if (!any) break;
        // every enqueued chunk is waited for, also after an error, so that no
        // member has work in flight when this returns
        for (int r = 0; r < R; r++) {
            if (!chunk[r]) continue;
            int st = finish_chunk(e->members[r], chunk[r], t_end, done[r], guard[r]);
            if (st < 0) { if (err == GFSPH_OK) err = st; active[r] = 0; continue; }
            if (st == 0) { active[r] = 0; status = GFSPH_T_END_REACHED; }
        }
    }
    if (min_steps_done) *min_steps_done = *std::min_element(done.begin(), done.end());
    return err != GFSPH_OK ? err : status;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_ensemble_sample(gfsph_ensemble* e) try {
    if (!e) return GFSPH_ERR_ARG;
    for (gfsph_handle* h : e->members) {
        int st = gfsph_hazard_sample(h);
        if (st) return st;
    }
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_ensemble_exceedance(gfsph_ensemble* e, float threshold, float* prob) try {
    if (!e || !prob) return GFSPH_ERR_ARG;
    const int R = (int)e->members.size();
    const int np = e->nx * e->ny;
    std::vector<unsigned int*> ptrs(R);
    for (int r = 0; r < R; r++) {
        gfsph_handle* h = e->members[r];
        if (!h->haz_cnt) { int st = gfsph_hazard_reset(h); if (st) return st; }
        CK(cudaStreamSynchronize(h->stream));
        ptrs[r] = h->haz_max_h;
    }
    if (!e->d_maxptr && dalloc(&e->d_maxptr, R)) return GFSPH_ERR_CUDA;
    if (!e->d_prob && dalloc(&e->d_prob, np)) return GFSPH_ERR_CUDA;
    cudaStream_t s = e->members[0]->stream;
    CK(cudaMemcpyAsync(e->d_maxptr, ptrs.data(), R * sizeof(unsigned int*), cudaMemcpyHostToDevice, s));
    k_exceedance<<<blocks_for(np, 256), 256, 0, s>>>(e->d_maxptr, R, np, threshold, e->d_prob);
    CK(cudaMemcpyAsync(prob, e->d_prob, (size_t)np * sizeof(float), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

// ---------------------------------------------------------------- adjoint

}  // extern "C"

constexpr int kAdjParams = 3;  // dL/d tanfi, dL/d xi, dL/d Bingham yield stress

struct gfsph_adjoint {
    gfsph_handle* h = nullptr;
    int n = 0, nsteps = 0, every = 1, nck = 0;
    double t0 = 0.0;
    float dt0 = 0.f;
    float2 *ckx = nullptr, *ckv = nullptr;    // checkpoints (caller order), nck * n
    float2 *segx = nullptr, *segv = nullptr;  // states of one segment, every * n
    float *rho0 = nullptr, *mass0 = nullptr, *hsml0 = nullptr;
    float* rhoN = nullptr;                    // depth of the final state
    float2 *lx = nullptr, *lv = nullptr;      // running adjoints (caller order)
    double* lm = nullptr;                     // dL/d volume, accumulated
    double* lpar = nullptr;                   // dL/d tanfi, dL/d xi, dL/d Bingham yield stress
    double par[kAdjParams] = {};              // the same on the host after a backward pass
    bool has_par = false;
    float* gh = nullptr;
    float2 *lx1 = nullptr, *lv2 = nullptr, *lvp = nullptr, *lin = nullptr, *lv0 = nullptr;
    float* lh = nullptr;
    double2* lxacc = nullptr;
    double* lms = nullptr;
    // sle 1: the smoothing lengths of every checkpoint and segment state, and
    // dL/d hsml handed from a step to the one before it (caller order)
    bool sle = false;
    float *ckh = nullptr, *segh = nullptr, *lhs = nullptr;
    double* lhsacc = nullptr;
};

namespace {

// The state of the handle (caller order) into x, v (and the constant fields).
int adj_capture(gfsph_adjoint* a, float2* x, float2* v, bool fields, float* hs = nullptr) {
    gfsph_handle* h = a->h;
    cudaStream_t st = h->stream;
    const int n = h->n;
    launch(h, K_ADJOINT, [&] { k_unsort<<<blocks_for(n), kThreads, 0, st>>>(h->B, n, h->U); });
    CK(cudaMemcpyAsync(x, h->U.pos, (size_t)n * sizeof(float2), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(v, h->U.vel, (size_t)n * sizeof(float2), cudaMemcpyDeviceToDevice, st));
    if (hs) CK(cudaMemcpyAsync(hs, h->U.hsml, (size_t)n * sizeof(float), cudaMemcpyDeviceToDevice, st));
    if (fields) {
        CK(cudaMemcpyAsync(a->rho0, h->U.rho, (size_t)n * sizeof(float), cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(a->mass0, h->U.mass, (size_t)n * sizeof(float), cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(a->hsml0, h->U.hsml, (size_t)n * sizeof(float), cudaMemcpyDeviceToDevice, st));
    }
    return 0;
}

int adj_restore(gfsph_adjoint* a, const float2* x, const float2* v, const float* rho = nullptr,
                const float* hs = nullptr, bool clear_err = true) {
    gfsph_handle* h = a->h;
    if (h->n != a->n) return GFSPH_ERR_STATE;  // the handle's buffers were dropped or resized
    launch(h, K_ADJOINT, [&] {
        k_adj_restore<<<blocks_for(a->n), kThreads, 0, h->stream>>>(h->B, a->n, x, v, rho ? rho : a->rho0, a->mass0,
                                                                    hs ? hs : a->hsml0);
    });
    CK(cudaGetLastError());
    set_field<float>(h, offsetof(StepScalars, dt), a->dt0);
    if (clear_err) set_field<int>(h, offsetof(StepScalars, err), 0);
    h->has_state = true;
    return 0;
}

// The backward sweep replays steps that the recording run has taken from
// the same states with the same deterministic kernels, so their capacity and
// their particle counts (every particle active and regular) were checked
// then: within a segment the steps are enqueued without waiting, the error
// word left set by any failed step (which also makes every later step skip),
// and checked once at the segment's end.
int adj_segment_check(gfsph_handle* h) {
    int st = read_scalars(h);
    if (st) return st;
    if (h->hS->err) return GFSPH_ERR_CAPACITY;
    if (h->hS->nactive != h->n || h->hS->nreg != h->hS->nactive) return GFSPH_ERR_UNSUPPORTED;
    return 0;
}

// One step of the handle from its current buffers; fails unless it ran.
int adj_one_step(gfsph_handle* h) {
    int done = 0, guard = 0;
    for (;;) {
        int st = enqueue_chunk(h, 1, 1e300);
        if (st) return st;
        st = finish_chunk(h, 1, 1e300, done, guard);
        if (st < 0) return st;
        if (done >= 1) break;
    }
    // every particle active and regular (nbig and nout are cleared when a step ends)
    if (h->hS->nactive != h->n || h->hS->nreg != h->hS->nactive) return GFSPH_ERR_UNSUPPORTED;
    return 0;
}

void adj_free(gfsph_adjoint* a) {
    dfree(a->ckx); dfree(a->ckv); dfree(a->segx); dfree(a->segv); dfree(a->rho0); dfree(a->mass0); dfree(a->hsml0);
    dfree(a->rhoN);
    dfree(a->lx); dfree(a->lv); dfree(a->lm); dfree(a->lpar); dfree(a->gh); dfree(a->lx1); dfree(a->lv2);
    dfree(a->lvp); dfree(a->lin); dfree(a->lv0); dfree(a->lh); dfree(a->lxacc); dfree(a->lms);
    dfree(a->ckh); dfree(a->segh); dfree(a->lhs); dfree(a->lhsacc);
}

}  // namespace

extern "C" {

int gfsph_set_search(gfsph_handle* h, float level_factor, float cell_div) try {
    if (!h || !(level_factor >= 1.f && level_factor <= 16.f) || !(cell_div >= 1.f && cell_div <= 8.f))
        return GFSPH_ERR_ARG;
    CK(cudaStreamSynchronize(h->stream));
    h->level_factor = level_factor;
    h->cell_div = cell_div;
    drop_graphs(h);
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_get_search(gfsph_handle* h, float* level_factor, float* cell_div) try {
    if (!h) return GFSPH_ERR_ARG;
    if (level_factor) *level_factor = h->level_factor;
    if (cell_div) *cell_div = h->cell_div;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_autotune(gfsph_handle* h, int steps, float* level_factor, float* cell_div, float* best_ms) try {
    if (!h || steps < 1) return GFSPH_ERR_ARG;
    if (!h->has_state) return GFSPH_ERR_STATE;
    const size_t n = (size_t)h->n, np = (size_t)h->nx * h->ny;
    cudaStream_t st = h->stream;
    // snapshot of everything a step changes: particles, scalars, DEM rows
    PState snap{};
    StepScalars* ssnap = nullptr;
    float *z = nullptr, *er = nullptr, *av = nullptr;
    int s0 = alloc_pstate(&snap, (int)n);
    s0 |= dalloc(&ssnap, 1); s0 |= dalloc(&z, np); s0 |= dalloc(&er, np); s0 |= dalloc(&av, np);
    auto cleanup = [&] {
        free_pstate(&snap);
        dfree(ssnap); dfree(z); dfree(er); dfree(av);
    };
    if (s0) { cleanup(); return GFSPH_ERR_CUDA; }
    auto copy_state = [&](PState& dst, const PState& src, StepScalars* sd, const StepScalars* ss, float* zd,
                          const float* zs, float* ed, const float* es, float* ad, const float* as) -> cudaError_t {
        cudaError_t e = cudaSuccess;
        auto cp = [&](void* d, const void* s2, size_t bytes) {
            if (e == cudaSuccess) e = cudaMemcpyAsync(d, s2, bytes, cudaMemcpyDeviceToDevice, st);
        };
        cp(dst.pos, src.pos, n * sizeof(float2)); cp(dst.vel, src.vel, n * sizeof(float2));
        cp(dst.rho, src.rho, n * sizeof(float)); cp(dst.mass, src.mass, n * sizeof(float));
        cp(dst.hsml, src.hsml, n * sizeof(float)); cp(dst.flag, src.flag, n * sizeof(int));
        cp(dst.id, src.id, n * sizeof(int)); cp(dst.pwp, src.pwp, n * sizeof(float));
        cp(sd, ss, sizeof(StepScalars));
        cp(zd, zs, np * sizeof(float)); cp(ed, es, np * sizeof(float)); cp(ad, as, np * sizeof(float));
        return e;
    };
    cudaError_t e = copy_state(snap, h->B, ssnap, h->S, z, h->d_z, er, h->d_eroded, av, h->d_avail);
    if (e != cudaSuccess) { cleanup(); return cuda_status(e); }
    const float lfs[4] = {1.5f, 2.f, 2.5f, 3.f}, cds[3] = {2.f, 3.f, 4.f};
    const float lf0 = h->level_factor, cd0 = h->cell_div;
    float best = 1e30f, blf = lf0, bcd = cd0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int status = GFSPH_OK;
    for (float lf : lfs)
        for (float cd : cds) {
            int r = gfsph_set_search(h, lf, cd);
            double t = 0.0;
            int done = 0;
            if (!r) r = cuda_status(copy_state(h->B, snap, h->S, ssnap, h->d_z, z, h->d_eroded, er, h->d_avail, av));
            if (!r) r = gfsph_step(h, 1, 1e300, &t, &done);  // graph capture, capacity growth
            if (!r) r = cuda_status(copy_state(h->B, snap, h->S, ssnap, h->d_z, z, h->d_eroded, er, h->d_avail, av));
            if (!r) r = cuda_status(cudaEventRecord(e0, st));
            if (!r) r = gfsph_step(h, steps, 1e300, &t, &done);
            if (!r) r = cuda_status(cudaEventRecord(e1, st));
            if (!r) r = cuda_status(cudaEventSynchronize(e1));
            if (r < 0) { status = r; break; }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) { best = ms; blf = lf; bcd = cd; }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int r = gfsph_set_search(h, status ? lf0 : blf, status ? cd0 : bcd);
    if (!r) r = cuda_status(copy_state(h->B, snap, h->S, ssnap, h->d_z, z, h->d_eroded, er, h->d_avail, av));
    if (!r) r = cuda_status(cudaStreamSynchronize(st));
    cleanup();
    if (status) return status;
    if (r) return r;
    if (level_factor) *level_factor = blf;
    if (cell_div) *cell_div = bcd;
    if (best_ms) *best_ms = best / (float)steps;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_adjoint_forward(gfsph_handle* h, int nsteps, int every, gfsph_adjoint** out) try {
    if (!h || !out || nsteps < 1 || every < 1) return GFSPH_ERR_ARG;
    *out = nullptr;
    if (!h->has_state) return GFSPH_ERR_STATE;
    const Rheo& c = h->rheo;
    if (!(c.nfric == 4 || c.nfric == 5 || c.nfric == 6) || (c.nfric != 4 && c.xi < 0.f) || c.erosion ||
        c.icpwp != 0 || c.pa_sph != 2 ||
        c.ic_adapt != 0 || c.muI != 0 || c.fact_dens != 1.f || c.nor_density || c.cos_theta || c.ws ||
        (c.skf != 1 && c.skf != 4))
        return GFSPH_ERR_UNSUPPORTED;
    gfsph_adjoint* a = new (std::nothrow) gfsph_adjoint();
    if (!a) return GFSPH_ERR_HOST;
    a->h = h; a->n = h->n; a->nsteps = nsteps; a->every = std::min(every, nsteps);
    a->nck = (nsteps + a->every - 1) / a->every + 1;
    const size_t n = (size_t)h->n;
    int st = 0;
    st |= dalloc(&a->ckx, n * a->nck); st |= dalloc(&a->ckv, n * a->nck);
    st |= dalloc(&a->segx, n * a->every); st |= dalloc(&a->segv, n * a->every);
    st |= dalloc(&a->rho0, n); st |= dalloc(&a->mass0, n); st |= dalloc(&a->hsml0, n); st |= dalloc(&a->rhoN, n);
    st |= dalloc(&a->lx, n); st |= dalloc(&a->lv, n); st |= dalloc(&a->lm, n); st |= dalloc(&a->lpar, kAdjParams);
    st |= dalloc(&a->gh, n); st |= dalloc(&a->lx1, n); st |= dalloc(&a->lv2, n); st |= dalloc(&a->lvp, n);
    st |= dalloc(&a->lin, n); st |= dalloc(&a->lv0, n); st |= dalloc(&a->lh, n); st |= dalloc(&a->lxacc, n);
    st |= dalloc(&a->lms, n);
    a->sle = (c.sle == 1);
    if (a->sle) {
        st |= dalloc(&a->ckh, n * a->nck); st |= dalloc(&a->segh, n * a->every);
        st |= dalloc(&a->lhs, n); st |= dalloc(&a->lhsacc, n);
    }
    if (st) { adj_free(a); delete a; return GFSPH_ERR_CUDA; }
    st = read_scalars(h);
    if (st) { adj_free(a); delete a; return st; }
    a->t0 = h->hS->time;
    a->dt0 = h->hS->dt;
    st = adj_capture(a, a->ckx, a->ckv, true, a->sle ? a->ckh : nullptr);
    for (int t = 0, k = 1; !st && t < nsteps; k++) {
        int chunk = std::min(a->every, nsteps - t);
        for (int q = 0; q < chunk && !st; q++) st = adj_one_step(h);
        t += chunk;
        if (!st) st = adj_capture(a, a->ckx + n * k, a->ckv + n * k, false, a->sle ? a->ckh + n * k : nullptr);
    }
    if (!st) {  // U holds the final state after the last capture
        std::vector<int> fl;
        try {
            fl.resize(n);
        } catch (...) {
            adj_free(a); delete a;
            return GFSPH_ERR_HOST;
        }
        cudaError_t e = cudaMemcpyAsync(a->rhoN, h->U.rho, n * sizeof(float), cudaMemcpyDeviceToDevice, h->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(fl.data(), h->U.flag, n * sizeof(int), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) st = cuda_status(e);
        for (size_t k = 0; !st && k < n; k++)
            if (fl[k]) st = GFSPH_ERR_UNSUPPORTED;  // a particle left the DEM in the last step
    }
    if (st) { adj_free(a); delete a; return st; }
    *out = a;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_adjoint_backward(gfsph_adjoint* a, const float* gx, const float* gv, const float* gh, float* gx0, float* gv0,
                           float* gm, double* gmu, double* gxi) try {
    if (!a || !gx || !gv) return GFSPH_ERR_ARG;
    gfsph_handle* h = a->h;
    // the handle must still hold a state of the recorded size (an upload of
    // another size, or a failed allocation, since the forward run voids it)
    if (!h->has_state || h->n != a->n) return GFSPH_ERR_STATE;
    cudaStream_t st = h->stream;
    const int n = a->n;
    const size_t un = (size_t)n;
    CK(cudaMemcpyAsync(a->lx, gx, un * sizeof(float2), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(a->lv, gv, un * sizeof(float2), cudaMemcpyHostToDevice, st));
    if (gh) CK(cudaMemcpyAsync(a->gh, gh, un * sizeof(float), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(a->lm, 0, un * sizeof(double), st));
    CK(cudaMemsetAsync(a->lpar, 0, kAdjParams * sizeof(double), st));
    if (a->sle) CK(cudaMemsetAsync(a->lhs, 0, un * sizeof(float), st));  // no step after the last
    const int nseg = a->nck - 1;
    for (int sg = nseg - 1; sg >= 0; sg--) {
        const int t0 = sg * a->every, len = std::min(a->every, a->nsteps - t0);
        // the segment's states: from its checkpoint, recomputed forward
        CK(cudaMemcpyAsync(a->segx, a->ckx + un * sg, un * sizeof(float2), cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(a->segv, a->ckv + un * sg, un * sizeof(float2), cudaMemcpyDeviceToDevice, st));
        if (a->sle) CK(cudaMemcpyAsync(a->segh, a->ckh + un * sg, un * sizeof(float), cudaMemcpyDeviceToDevice, st));
        auto seg_h = [&](int q) -> float* { return a->sle ? a->segh + un * q : nullptr; };
        set_field<int>(h, offsetof(StepScalars, err), 0);
        for (int q = 1; q < len; q++) {
            int r = adj_restore(a, a->segx + un * (q - 1), a->segv + un * (q - 1), nullptr, seg_h(q - 1), false);
            if (!r) r = enqueue_chunk(h, 1, 1e300);
            if (!r) r = adj_capture(a, a->segx + un * q, a->segv + un * q, false, seg_h(q));
            if (r) return r;
        }
        if (len > 1) {
            int r = adj_segment_check(h);
            if (r) return r;
        }
        for (int q = len - 1; q >= 0; q--) {
            const bool last = (t0 + q == a->nsteps - 1);
            int r = adj_restore(a, a->segx + un * q, a->segv + un * q, nullptr, seg_h(q), false);
            if (!r) r = enqueue_chunk(h, 1, 1e300);  // neighbour table, density, forces of this step
            if (r) return r;
            Search Q = make_search(h);
            const int pb = blocks_for(n);
            launch(h, K_ADJOINT, [&] {
                k_adj_seed<<<pb, kThreads, 0, st>>>(h->A, n, a->lx, a->lv, (last && gh) ? a->gh : nullptr, a->lx1,
                                                    a->lv2, a->lh, a->lxacc, a->lms, a->sle ? a->lhs : nullptr,
                                                    a->lhsacc);
            });
            if (h->rheo.av_vel) {
                launch(h, K_ADJOINT, [&] {
                    k_adj_xsph<<<pb, kThreads, 0, st>>>(h->A, Q, h->rheo, n, h->velfin, a->lv2, a->lvp, a->lh,
                                                        a->lms, a->lxacc, a->lhsacc);
                });
            } else {
                CK(cudaMemcpyAsync(a->lvp, a->lv2, un * sizeof(float2), cudaMemcpyDeviceToDevice, st));
            }
            launch(h, K_ADJOINT, [&] {
                k_adj_rk<<<pb, kThreads, 0, st>>>(h->A, Q, h->S, h->rheo, h->dem, n, a->lx1, a->lvp, a->lh, a->lin,
                                                  a->lxacc, a->lv0, a->lpar);
            });
            launch(h, K_ADJOINT, [&] {
                k_adj_gather<<<pb, kThreads, 0, st>>>(h->A, Q, h->rheo, n, a->lin, a->lh, a->lms, a->lxacc, a->lhsacc);
            });
            launch(h, K_ADJOINT, [&] {
                k_adj_scatter<<<pb, kThreads, 0, st>>>(h->A, n, a->lxacc, a->lv0, a->lms, a->lx, a->lv, a->lm,
                                                       a->lhsacc, a->lhs);
            });
            CK(cudaGetLastError());
        }
        int r = adj_segment_check(h);
        if (r) return r;
    }
    if (gx0) CK(cudaMemcpyAsync(gx0, a->lx, un * sizeof(float2), cudaMemcpyDeviceToHost, st));
    if (gv0) CK(cudaMemcpyAsync(gv0, a->lv, un * sizeof(float2), cudaMemcpyDeviceToHost, st));
    std::vector<double> lm(un);
    CK(cudaMemcpyAsync(lm.data(), a->lm, un * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(a->par, a->lpar, kAdjParams * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    a->has_par = true;
    if (gm)
        for (size_t k = 0; k < un; k++) gm[k] = (float)lm[k];
    if (gmu) *gmu = a->par[0];
    if (gxi) *gxi = a->par[1];
    // leave the handle at the final state of the recorded run
    int r = adj_restore(a, a->ckx + un * (a->nck - 1), a->ckv + un * (a->nck - 1), a->rhoN,
                        a->sle ? a->ckh + un * (a->nck - 1) : nullptr);
    if (r) return r;
    set_field<double>(h, offsetof(StepScalars, time), a->t0 + (double)a->nsteps * (double)a->dt0);
    CK(cudaStreamSynchronize(st));
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_adjoint_param(gfsph_adjoint* a, int which, double* value) try {
    if (!a || !value || which < 0 || which >= kAdjParams) return GFSPH_ERR_ARG;
    if (!a->has_par) return GFSPH_ERR_STATE;
    *value = a->par[which];
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_adjoint_destroy(gfsph_adjoint* a) try {
    if (!a) return GFSPH_ERR_ARG;
    adj_free(a);
    delete a;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_gradhs(gfsph_handle* h, int ix0, int iy0, int nwx, int nwy, int niter, float tol, float* hs_w,
                 float* gradhs_w) try {
    if (!h || nwx < 2 || nwy < 2 || ix0 < 0 || iy0 < 0 || ix0 + nwx > h->nx || iy0 + nwy > h->ny || niter < 0)
        return GFSPH_ERR_ARG;
    if (!h->has_state) return GFSPH_ERR_STATE;
    const int nn = nwx * nwy;
    if (nn > h->cw_nodes) {
        dfree(h->cw_a1); dfree(h->cw_a2); dfree(h->cw_hs); dfree(h->cw_ml); dfree(h->cw_rhs); dfree(h->cw_g0);
        dfree(h->cw_g1);
        int st = 0;
        st |= dalloc(&h->cw_a1, nn); st |= dalloc(&h->cw_a2, nn); st |= dalloc(&h->cw_hs, nn);
        st |= dalloc(&h->cw_ml, nn); st |= dalloc(&h->cw_rhs, nn); st |= dalloc(&h->cw_g0, nn);
        st |= dalloc(&h->cw_g1, nn);
        if (st) { h->cw_nodes = 0; return GFSPH_ERR_CUDA; }
        h->cw_nodes = nn;
    }
    Window w{ix0, iy0, nwx, nwy, h->dem.xmin, h->dem.ymin, h->dem.dx, h->dem.dy};
    cudaStream_t st = h->stream;
    CK(cudaMemsetAsync(h->cw_a1, 0, (size_t)nn * sizeof(double), st));
    CK(cudaMemsetAsync(h->cw_a2, 0, (size_t)nn * sizeof(double), st));
    launch(h, K_COUPLE, [&] { k_couple_idw<<<blocks_for(h->n), kThreads, 0, st>>>(h->B, h->n, w, h->cw_a1, h->cw_a2); });
    launch(h, K_COUPLE, [&] { k_couple_hs<<<blocks_for(nn), kThreads, 0, st>>>(h->cw_a1, h->cw_a2, nn, h->cw_hs); });
    launch(h, K_COUPLE, [&] {
        k_couple_rhs<<<blocks_for(nn), kThreads, 0, st>>>(w, h->cw_hs, h->cw_rhs, h->cw_ml, h->cw_g0);
    });
    CK(cudaGetLastError());
    float2* g = h->cw_g0;
    if (niter > 0) {
        float2* other = h->cw_g1;
        for (int it = 2; it <= niter; it++) {  // the first sweep leaves g = 0 (:497-501)
            launch(h, K_COUPLE, [&] {
                k_couple_jacobi<<<blocks_for(nn), kThreads, 0, st>>>(w, g, h->cw_rhs, h->cw_ml, other);
            });
            std::swap(g, other);
        }
        CK(cudaGetLastError());
        if (hs_w) CK(cudaMemcpyAsync(hs_w, h->cw_hs, (size_t)nn * sizeof(float), cudaMemcpyDeviceToHost, st));
        if (gradhs_w) CK(cudaMemcpyAsync(gradhs_w, g, (size_t)nn * sizeof(float2), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return GFSPH_OK;
    }
    // niter = 0: M g = rhs by the device CG (solvegc2 semantics), both
    // components as two dofs per node
    const int key[4] = {ix0, iy0, nwx, nwy};
    if (!h->cw_cg || std::memcmp(key, h->cw_key, sizeof(key)) != 0) {
        if (h->cw_cg) { gfsph_cg_destroy(h->cw_cg); h->cw_cg = nullptr; }
        const int nelem = 2 * (nwx - 1) * (nwy - 1);
        std::vector<int> im(3 * (size_t)nelem);
        std::vector<float> gs(36 * (size_t)nelem, 0.f);
        for (int cj = 0; cj < nwy - 1; cj++)
            for (int ci = 0; ci < nwx - 1; ci++) {
                int e = 2 * (cj * (nwx - 1) + ci), n0 = cj * nwx + ci;
                int t[2][3] = {{n0, n0 + 1, n0 + 1 + nwx}, {n0, n0 + 1 + nwx, n0 + nwx}};
                for (int q = 0; q < 2; q++) {
                    float x[3], y[3];
                    for (int k = 0; k < 3; k++) {
                        im[3 * (size_t)(e + q) + k] = t[q][k] + 1;
                        x[k] = w.xming + (float)(ix0 + t[q][k] % nwx) * w.dxg;
                        y[k] = w.yming + (float)(iy0 + t[q][k] / nwx) * w.dyg;
                    }
                    float rj = (x[1] - x[0]) * (y[2] - y[0]) - (x[2] - x[0]) * (y[1] - y[0]);
                    float coe = rj / 24.f;
                    float* ge = &gs[36 * (size_t)(e + q)];
                    for (int a = 0; a < 3; a++)
                        for (int b = 0; b < 3; b++)
                            for (int d = 0; d < 2; d++) ge[(b * 2 + d) * 6 + (a * 2 + d)] = (a == b ? 2.f : 1.f) * coe;
                }
            }
        int s2 = gfsph_cg_create(nn, nelem, 3, 2, im.data(), gs.data(), &h->cw_cg);
        if (s2) return s2;
        std::memcpy(h->cw_key, key, sizeof(key));
    }
    std::vector<float> rhs(2 * (size_t)nn), fixed(2 * (size_t)nn, 0.f), sol(2 * (size_t)nn, 0.f);
    std::vector<int> iffix(2 * (size_t)nn, 0);
    CK(cudaMemcpyAsync(rhs.data(), h->cw_rhs, (size_t)nn * sizeof(float2), cudaMemcpyDeviceToHost, st));
    if (hs_w) CK(cudaMemcpyAsync(hs_w, h->cw_hs, (size_t)nn * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    int iters = 0;
    int s3 = gfsph_cg_solve(h->cw_cg, iffix.data(), fixed.data(), rhs.data(), sol.data(), tol, &iters);
    if (s3 < 0) return s3;
    if (gradhs_w) std::memcpy(gradhs_w, sol.data(), sol.size() * sizeof(float));
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_stats(gfsph_handle* h, int* out, int nout) try {
    if (!h || !out || nout < 1) return GFSPH_ERR_ARG;
    int st = read_scalars(h);
    if (st) return st;
    const StepScalars* s = h->hS;
    // nbig and nout are cleared for the next step when a step ends; nactive
    // and nreg hold the last search's counts
    const int v[8] = {s->nactive, s->nreg, s->nactive - s->nreg, s->nlev, s->ncells, h->kcap, h->cap_cells,
                      h->n - s->nactive};
    for (int k = 0; k < nout && k < 8; k++) out[k] = v[k];
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

}  // extern "C"
