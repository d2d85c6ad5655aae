// Kernels of one SPH time step (Geoflow-SPH RK45, SPH_MAIN_2019.f90:746-1005)
// on sm_100a.  Particles live in HBM as structure-of-arrays, re-sorted by cell
// every step (counting sort); the neighbour table is built once per step and
// reused by the density, force and XSPH passes, as the reference reuses its
// pair list (w and dW frozen at the start of the step).
//
// Cell grids: while every level's grid over the bounding box fits the dense
// budget (4M cells, or 8 per particle), the cell keys are row-major over each
// level (dense mode).  Beyond it (separated releases on a large DEM with
// small smoothing lengths) the grids are block-sparse: cut into blocks of
// 32 x 8 cells, a dense block map over the box marks the blocks that hold
// particles, and only those blocks get cells (slot-major keys: slot * 256 +
// row * 32 + column), so the cell count follows the area the flow covers.
#pragma once
#include <climits>

#include "gfsph_device.cuh"

namespace gfsph {

constexpr int kScanTile = 2048;  // cells per scan tile (256 threads x 8)
constexpr int kScanThreads = 256;
constexpr float kBigFactor = 1.5f;  // default level-0 bound Hc = kBigFactor * mean(hsml)
constexpr float kCellDiv = 3.f;     // default cell size of level k: Hc * 2^k / kCellDiv
constexpr int kRegLevels = 2;       // default regular levels: their particles take a thread and the table
constexpr int kMaxLevels = 24;      // level k cell size Hc * 2^(k-1)
constexpr int kBlkX = 32;           // cells per block along x
constexpr int kBlkY = 8;            // cells per block along y
constexpr int kBlockCells = kBlkX * kBlkY;
constexpr long long kDenseCells = 1LL << 22;  // dense-mode budget (or 8 cells per particle)
constexpr int kThreadsBounds = 128;
constexpr int kBoundsBlocks = 148 * 8;

// error bits in StepScalars::err
constexpr int kErrCells = 1;
constexpr int kErrNbr = 2;
constexpr int kErrNonFinite = 4;
constexpr int kErrEmpty = 8;
constexpr int kErrBlocks = 16;

// Device-resident scalars of the step (one per handle).
struct StepScalars {
    double time;      // time_sph
    double t_end;
    double hsum;      // sum of hsml over the particles inside the DEM box
    float dt;         // dt_sph, committed at the end of a completed step
    float dt_step;    // dt of the step in flight (a step stopped by a capacity error leaves dt unchanged)
    int skip;         // this step does nothing (time >= t_end or an error)
    int err;          // sticky error bits
    int steps_done;
    unsigned int xmin_o, xmax_o, ymin_o, ymax_o, hmax_o, dtmin_o;  // reductions (ordered uint)
    int hcount;
    int bad;          // non-finite state seen by k_bounds
    float hc;         // regular-hsml bound Hc: level k holds hsml in (Hc*2^(k-1), Hc*2^k], level 0 hsml <= Hc
    int nlev;         // number of grid levels
    float lev_gx0[kMaxLevels], lev_gy0[kMaxLevels], lev_c[kMaxLevels];  // origin and cell size per level
    int lev_ndx[kMaxLevels], lev_ndy[kMaxLevels];  // cells per level along x and y
    int lev_off[kMaxLevels + 1];  // dense mode: first cell key of each level
    int lev_nbx[kMaxLevels], lev_boff[kMaxLevels + 1];  // sparse mode: blocks per level along x, first block-map entry
    int sparse;       // 1: block-sparse cell keys this step
    unsigned int lev_hmax_o[kMaxLevels];  // max hsml of the particles of each level (ordered uint, 0 = empty)
    int nblocks;      // block-map entries (all levels)
    int ncells;       // cells of the occupied blocks
    int nreg, nbig, nactive, nout;
    int need_cells, need_nbr, need_big, need_blocks;
    int ex0, ex1, ey0, ey1;  // DEM node box touched by erosion this step
    unsigned int bounds_ticket;  // blocks of k_bounds done (the last one resets it)
    unsigned int scan_ticket[2];  // tiles of k_scan_tiles done: cells, block map
    unsigned int end_ticket;      // blocks of k_dem_erode done
    int reg_levels;   // levels 0 .. reg_levels-1 are regular (thread + neighbour table)
    // the reference's own grid of grid_find_NEW_tools (skf 2, 3): origin, cell, cells
    float ref_xmin, ref_ymin, ref_delt;
    int ref_ndx, ref_ndy;
    int advance;      // 1 inside gfsph_step, 0 for search-only passes
};

// Particle state, structure of arrays, one buffer set per ordering.
struct PState {
    float2* pos;
    float2* vel;
    float* rho;
    float* mass;
    float* hsml;
    int* flag;
    int* id;
    float* pwp;  // basal pore-water pressure Uaux(1,:) (icpwp = 3)
};

// Programmatic dependent launch: every kernel of the step is launched with
// programmatic stream serialisation, so the next kernel's launch and block
// set-up overlap this one's tail.  Each kernel first waits for the kernels
// before it to finish and their writes to be visible (griddepcontrol.wait,
// a no-op for an ordinary launch), then lets its dependents launch.
#define PDL_ENTRY()                                              \
    do {                                                         \
        asm volatile("griddepcontrol.wait;" ::: "memory");       \
        asm volatile("griddepcontrol.launch_dependents;" :::);   \
    } while (0)

// Scratch of the neighbour search (sorted order).
struct Search {
    const int* bstart;   // block-map entry -> slot of its block (exclusive scan of the marks), nblocks+1
    const int* start;    // cell key -> first particle slot (exclusive scan), ncells+1
    const int* cellA;    // slot -> cell key (all levels), -1 out of the domain
    const float4* xhm;   // slot -> (x, y, hsml, mass) at the start of the step
    int4* nbr;           // neighbour table of the regular particles (layout: tab_base); entry
                         // {j, W_ij, dW_ij/dx, dW_ij/dy} (the FP32 bits of the kernel values,
                         // computed once per pair by the search, as grid_find stores w and dwdx)
    int* ncount;
    float* pterm;        // p/h^2 (pa_sph 2) or p (pa_sph 1)
    float4* pr;          // (pterm, h, m, 0): what the internal force gathers per neighbour
    float2* indv;        // internal acceleration of every active particle (slot order)
    float* rho0;         // depth at the start of the step, after Adaptive_dt's h_inf clamp (icpwp = 3)
    const int2* rcell;   // slot -> cell of the reference's own grid (skf 2, 3), else null
    float4* xsv;         // slot -> (vx, vy, h, m) after the RK update: what av_vel gathers
    // ic_ws_Interact = 1: slot -> material (1 soil, 2 water); at the water
    // particles Z + hs of the current stage and its gradient; per particle the
    // sum of its soil-water pair terms.  A soil-water pair is kept in the
    // neighbour table with the sign bit of j set (type 1 of
    // Pint_Update_SW_tools): the density, the internal force and av_vel skip it.
    const unsigned char* spec;
    float* zpw;
    float2* gzw;
    float2* bxy;
    const float* mass0;  // caller index -> mass at upload (nfric 3), else null
    int kcap;
};

// nsoilB = (m - m0)/m of basal_friction_Ext_SW (SPH_SW_2019.f90:9449-9451),
// the share of a particle's mass gained by erosion; 0 unless nfric = 3.
__device__ __forceinline__ float soil_fraction(const Rheo& c, const Search& Q, const PState& A, int i) {
    if (c.nfric != 3) return 0.f;
    const float m = A.mass[i];
    return (m - Q.mass0[A.id[i]]) / m;
}
constexpr int kCrossBit = (int)0x80000000;

__device__ __forceinline__ bool step_skipped(const StepScalars* S) { return S->skip != 0; }

// The step scalars in shared memory for the serial set-up code that one
// thread runs at the end of a kernel (grid set-up, step end): the block
// copies the struct in and out in one parallel pass each, so the set-up does
// not wait for a global round trip per field it reads.  Every thread of the
// block calls both, and nothing else writes S meanwhile.
static_assert(sizeof(StepScalars) % 4 == 0, "StepScalars is copied as 32-bit words");
__device__ __forceinline__ StepScalars* scalars_to_smem(const StepScalars* S) {
    __shared__ __align__(16) StepScalars sS;
    const int nw = (int)(sizeof(StepScalars) / 4);
    const unsigned int* src = reinterpret_cast<const unsigned int*>(S);
    unsigned int* dst = reinterpret_cast<unsigned int*>(&sS);
    for (int k = threadIdx.x; k < nw; k += blockDim.x) dst[k] = __ldcg(src + k);
    __syncthreads();
    return &sS;
}
__device__ __forceinline__ void scalars_from_smem(StepScalars* S, const StepScalars* L) {
    __syncthreads();
    const int nw = (int)(sizeof(StepScalars) / 4);
    const unsigned int* src = reinterpret_cast<const unsigned int*>(L);
    unsigned int* dst = reinterpret_cast<unsigned int*>(S);
    for (int k = threadIdx.x; k < nw; k += blockDim.x) dst[k] = src[k];
}

// Neighbour-table layout, blocked by warps of 32 particles: entry k of
// particle i is at tab_base(i, kcap) + 32 k.  The lanes of a warp read entry k
// of their particles as one 512-byte run (16-byte entries), and the entries a
// warp appends while its lanes are at different k stay within its own
// 32 kcap entries.
__host__ __device__ __forceinline__ size_t tab_base(int i, int kcap) {
    return (size_t)(i >> 5) * ((size_t)kcap << 5) + (size_t)(i & 31);
}
constexpr int kTabStride = 32;

// ---------------------------------------------------------------- prologue
// Decides whether the coming step runs and resets its reductions; run at the
// start of a batch (k_prep) and at the end of every step for the next one
// (k_step_end).
__device__ __forceinline__ void prepare_step(StepScalars* S, int advance) {
    S->advance = advance;
    S->skip = (S->err != 0) || (advance && S->time >= S->t_end);
    S->xmin_o = 0xffffffffu; S->ymin_o = 0xffffffffu;
    S->xmax_o = 0u; S->ymax_o = 0u; S->hmax_o = 0u;
    S->dtmin_o = 0xffffffffu;
    S->hsum = 0.0;
    S->hcount = 0;
    S->bad = 0;
    S->nout = 0;
    S->nbig = 0;
    S->ex0 = 0x7fffffff; S->ey0 = 0x7fffffff; S->ex1 = -1; S->ey1 = -1;
    for (int k = 0; k < kMaxLevels; k++) S->lev_hmax_o[k] = 0u;
}

__global__ void k_prep(StepScalars* S, int advance) {
    PDL_ENTRY();
    StepScalars* L = scalars_to_smem(S);
    if (threadIdx.x == 0) prepare_step(L, advance);
    scalars_from_smem(S, L);
}

__device__ __forceinline__ float warp_min(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ int warp_sum(int v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// The stability time step of Adaptive_dt_sph_SW (SPH_SW_2019.f90:6537-6567,
// min hsml/(3 max(1e-6, sqrt(g h))) [+|v|]) over the particles not yet
// flagged; then the Check_Out_Domain at the start of time_integration_sph
// (SPH_MAIN_2019.f90:232, :1764-1788) and, over the particles still inside,
// the bounds, max and mean of hsml for the cell grid.
// One launch: the per-particle part, block partials, and in the last block
// the global bounds and grid_setup.
struct BoundsPart {
    float xmn, xmx, ymn, ymx, hmx, dtm;
    double hsum;
    int hcnt, bad;
};

__device__ __forceinline__ void bounds_merge(BoundsPart& a, const BoundsPart& b) {
    a.xmn = fminf(a.xmn, b.xmn); a.xmx = fmaxf(a.xmx, b.xmx);
    a.ymn = fminf(a.ymn, b.ymn); a.ymx = fmaxf(a.ymx, b.ymx);
    a.hmx = fmaxf(a.hmx, b.hmx); a.dtm = fminf(a.dtm, b.dtm);
    a.hsum += b.hsum; a.hcnt += b.hcnt; a.bad |= b.bad;
}

// Capacities and search tunables handed to grid_setup.
struct GridArgs {
    int cap_blocks, cap_cells, max_cells;
    float level_factor, cell_div;
    int reg_levels;
};

__device__ void grid_setup(const Rheo& c, StepScalars* S, const GridArgs ga);

__global__ void __launch_bounds__(kThreadsBounds) k_bounds(PState B, int n, Rheo c, DemView dem, StepScalars* S,
                                                           BoundsPart* part, GridArgs ga) {
    PDL_ENTRY();
    if (step_skipped(S)) return;
    float xmn = 3.4e38f, xmx = -3.4e38f, ymn = 3.4e38f, ymx = -3.4e38f, hmx = 0.f, dtm = 1.e10f;
    double hs_sum = 0.0;
    int hs_cnt = 0;
    int bad = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        // every load issued before the flag test, so that they overlap
        const int fl = B.flag[i];
        float2 p = B.pos[i];
        float hs = B.hsml[i];
        float h = B.rho[i];
        float2 v = B.vel[i];
        if (fl) continue;
        if (!(isfinite(p.x) && isfinite(p.y) && isfinite(hs) && isfinite(h) && isfinite(v.x) && isfinite(v.y))) bad = 1;
        bool out = out_of_box(dem, p.x, p.y);
        if (out && S->advance) B.flag[i] = 1;
        if (!out) {
            xmn = fminf(xmn, p.x); xmx = fmaxf(xmx, p.x);
            ymn = fminf(ymn, p.y); ymx = fmaxf(ymx, p.y);
            hmx = fmaxf(hmx, hs);
            hs_sum += (double)hs;
            hs_cnt += 1;
        }
        if (c.ic_adapt != 0) {
            float vv = 0.f;
            if (c.ic_adapt != 1) vv = sqrtf(v.x * v.x + v.y * v.y);
            if (c.ic_adapt != 4) {  // modes 1, 2, 10: hsml / (3 (c [+ |v|])) with h clamped to h_inf
                float hh = (h < c.h_inf) ? c.h_inf : h;
                float cs = sqrtf(c.g * hh);
                float cc = (1.e-6f > cs) ? 1.e-6f : cs;
                if (c.ic_adapt == 2) cc = cc + vv;
                cc = hs / (3.f * cc);
                dtm = fminf(dtm, cc);
            }
            if (c.ic_adapt == 4 || c.ic_adapt == 10)  // |DEM cell diagonal| / |v|, +inf at rest
                dtm = fminf(dtm, sqrtf(dem.dx * dem.dx + dem.dy * dem.dy) / vv);
        }
    }
    // block partials, then the last block to finish reduces them in block
    // order (deterministic FP64 sum, no same-address atomics) and sets up
    // the grids
    __shared__ BoundsPart wp[kThreadsBounds / 32];
    __shared__ bool last;
    BoundsPart q{warp_min(xmn), warp_max(xmx), warp_min(ymn), warp_max(ymx), warp_max(hmx), warp_min(dtm),
                 warp_sum(hs_sum), warp_sum(hs_cnt), __any_sync(0xffffffffu, bad) ? 1 : 0};
    if ((threadIdx.x & 31) == 0) wp[threadIdx.x >> 5] = q;
    __syncthreads();
    if (threadIdx.x == 0) {
        BoundsPart b = wp[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); k++) bounds_merge(b, wp[k]);
        part[blockIdx.x] = b;
        __threadfence();
        last = (atomicAdd(&S->bounds_ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    BoundsPart b{3.4e38f, -3.4e38f, 3.4e38f, -3.4e38f, 0.f, 1.e10f, 0.0, 0, 0};
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) {
        BoundsPart o;
        const volatile BoundsPart* vp = part + k;
        o.xmn = vp->xmn; o.xmx = vp->xmx; o.ymn = vp->ymn; o.ymx = vp->ymx; o.hmx = vp->hmx; o.dtm = vp->dtm;
        o.hsum = vp->hsum; o.hcnt = vp->hcnt; o.bad = vp->bad;
        bounds_merge(b, o);
    }
    b.xmn = warp_min(b.xmn); b.xmx = warp_max(b.xmx); b.ymn = warp_min(b.ymn); b.ymx = warp_max(b.ymx);
    b.hmx = warp_max(b.hmx); b.dtm = warp_min(b.dtm); b.hsum = warp_sum(b.hsum); b.hcnt = warp_sum(b.hcnt);
    b.bad = __any_sync(0xffffffffu, b.bad) ? 1 : 0;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) wp[threadIdx.x >> 5] = b;
    __syncthreads();
    StepScalars* L = scalars_to_smem(S);
    if (threadIdx.x == 0) {
        BoundsPart t = wp[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); k++) bounds_merge(t, wp[k]);
        L->xmin_o = f2o(t.xmn); L->xmax_o = f2o(t.xmx); L->ymin_o = f2o(t.ymn); L->ymax_o = f2o(t.ymx);
        L->hmax_o = f2o(t.hmx); L->dtmin_o = f2o(t.dtm);
        L->hsum = t.hsum; L->hcount = t.hcnt; L->bad = t.bad;
        L->bounds_ticket = 0u;
        grid_setup(c, L, ga);
    }
    scalars_from_smem(S, L);
}

// dt update (Adaptive_dt_sph_SW :6658-6662) and the cell grids.  The
// reference sizes its single grid by 2*max(hsml) (grid_find :906-919), so one
// thin-front particle whose hsml keeps growing inflates every cell.  Here
// particles are split by smoothing length into levels: level 0 holds
// hsml <= Hc = min(max, level_factor*mean), level k >= 1 holds hsml in
// (Hc*2^(k-1), Hc*2^k]; level k has its own grid of cell size
// Hc*2^k/cell_div over the same box, and one cell-key space covers all
// levels.  The particles of the first reg_levels levels ("regular") take a
// thread each and the neighbour table; those of the coarser levels, few and
// with long neighbour lists, a warp each.  A particle
// searches each level within hsml_i + (that level's hsml bound), so the
// neighbour set is the reference's {j : r_ij < 2*(h_i+h_j)/2} exactly.
// level_factor and cell_div are the search's tunables (gfsph_set_search):
// Hc = min(max, level_factor * mean hsml) and level k's cell size is
// Hc * 2^k / cell_div; neither changes the neighbour sets.
__device__ void grid_setup(const Rheo& c, StepScalars* S, const GridArgs ga) {
    const int cap_blocks = ga.cap_blocks, cap_cells = ga.cap_cells, max_cells = ga.max_cells;
    const float level_factor = ga.level_factor, cell_div = ga.cell_div;
    S->reg_levels = ga.reg_levels;
    if (S->skip) return;
    if (S->bad) { S->err |= kErrNonFinite; S->skip = 1; return; }
    float xmn = o2f(S->xmin_o), xmx = o2f(S->xmax_o), ymn = o2f(S->ymin_o), ymx = o2f(S->ymax_o);
    float hmx = o2f(S->hmax_o);
    if (S->xmin_o == 0xffffffffu || !(hmx > 0.f) || S->hcount == 0) { S->err |= kErrEmpty; S->skip = 1; return; }
    float dt = S->dt;
    if (S->advance) {
        float dtmin = (c.ic_adapt != 0) ? o2f(S->dtmin_o) : 1.e10f;
        if (dtmin < dt) dt = dtmin;
        else if (c.ic_adapt != 0) dt = fminf(1.1f * dt, dtmin);
    }
    S->dt_step = dt;
    {  // the reference's grid: cells of 2*max(hsml) (grid_find_NEW_tools My_SPH_Tools_2019.f90:1168-1181)
        const float delt = hmx * 2.f;
        float len = xmx - xmn;
        int nd = (int)(len / delt + 1.f);
        S->ref_ndx = nd;
        S->ref_xmin = (xmn - ((float)nd * delt - len) / 2.f) - 0.001f * len;
        len = ymx - ymn;
        nd = (int)(len / delt + 1.f);
        S->ref_ndy = nd;
        S->ref_ymin = (ymn - ((float)nd * delt - len) / 2.f) - 0.001f * len;
        S->ref_delt = delt;
    }
    float mean = (float)(S->hsum / (double)S->hcount);
    float hc = fminf(hmx, level_factor * mean);
    int nlev = 1;
    while (nlev < kMaxLevels && ldexpf(hc, nlev - 1) < hmx) nlev++;
    if (ldexpf(hc, nlev - 1) < hmx) { S->err |= kErrCells; S->need_cells = 0x3fffffff; S->skip = 1; return; }
    float lx = xmx - xmn, ly = ymx - ymn;
    long long off = 0, doff = 0;
    for (int k = 0; k < nlev; k++) {
        float cell = ldexpf(hc, k) / cell_div;
        float fx = lx / cell + 1.f, fy = ly / cell + 1.f;
        if (!(fx < 1.0e8f) || !(fy < 1.0e8f) || !(fx * fy < 2.0e9f)) {  // far beyond any capacity
            S->err |= kErrCells;
            S->need_cells = 0x3fffffff;
            S->skip = 1;
            return;
        }
        int ndx = (int)fx, ndy = (int)fy;
        float lxn = (float)ndx * cell, lyn = (float)ndy * cell;
        S->lev_gx0[k] = (xmn - (lxn - lx) / 2.f) - 0.001f * lx;
        S->lev_gy0[k] = (ymn - (lyn - ly) / 2.f) - 0.001f * ly;
        S->lev_c[k] = cell;
        S->lev_ndx[k] = ndx;
        S->lev_ndy[k] = ndy;
        int nbx = (ndx + kBlkX - 1) / kBlkX, nby = (ndy + kBlkY - 1) / kBlkY;
        S->lev_nbx[k] = nbx;
        S->lev_boff[k] = (int)min(off, 0x7fffffffLL);
        S->lev_off[k] = (int)min(doff, 0x7fffffffLL);
        off += (long long)nbx * (long long)nby;
        doff += (long long)ndx * (long long)ndy;
    }
    S->lev_boff[nlev] = (int)min(off, 0x7fffffffLL);
    S->lev_off[nlev] = (int)min(doff, 0x7fffffffLL);
    S->hc = hc;
    S->nlev = nlev;
    const long long budget = min((long long)max_cells, max(kDenseCells, 8LL * S->hcount));
    S->sparse = (doff + 1 > budget) ? 1 : 0;
    if (!S->sparse) {
        if (doff + 1 > (long long)cap_cells) {
            S->err |= kErrCells;
            S->need_cells = (int)(doff + 1);
            S->skip = 1;
            return;
        }
        S->ncells = (int)doff;
        return;
    }
    if (off + 1 > (long long)cap_blocks) {
        S->err |= kErrBlocks;
        S->need_blocks = (off + 1 > 0x3fffffffLL) ? 0x3fffffff : (int)(off + 1);
        S->skip = 1;
        return;
    }
    S->nblocks = (int)off;
}

__device__ __forceinline__ void cell_of(float2 p, const StepScalars* S, int k, int& cx, int& cy) {
    float gd = S->lev_c[k];
    int ix = (int)((p.x - S->lev_gx0[k]) / gd + 1.f);
    int iy = (int)((p.y - S->lev_gy0[k]) / gd + 1.f);
    cx = min(max(ix, 1), S->lev_ndx[k]) - 1;
    cy = min(max(iy, 1), S->lev_ndy[k]) - 1;
}

__device__ __forceinline__ int level_of(float hs, const StepScalars* S) {
    int k = 0;
    while (k + 1 < S->nlev && hs > ldexpf(S->hc, k)) k++;
    return k;
}

// Cell coordinates are never negative: unsigned division and remainder by
// the block sides compile to shifts and masks.
__device__ __forceinline__ int block_of(const StepScalars* S, int k, int cx, int cy) {
    return S->lev_boff[k] + (int)((unsigned)cy / kBlkY) * S->lev_nbx[k] + (int)((unsigned)cx / kBlkX);
}

// Marks the blocks that hold particles (block map, all levels) and takes the
// largest smoothing length of every level, which bounds the stencils of the
// neighbour search more tightly than the level's upper limit.
__global__ void k_mark(const PState B, int n, DemView dem, StepScalars* S, int* bmark) {
    PDL_ENTRY();
    if (S->skip) return;
    // per-level largest hsml, reduced in shared memory first: every particle
    // of a level would otherwise hit the same global word
    __shared__ unsigned int lmax[kMaxLevels];
    const int nlev = S->nlev;
    for (int k = threadIdx.x; k < nlev; k += blockDim.x) lmax[k] = 0u;
    __syncthreads();
    unsigned int h0 = 0u;  // largest level-0 hsml seen by this thread
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (B.flag[i]) continue;
        float2 p = B.pos[i];
        if (out_of_box(dem, p.x, p.y)) continue;
        float hs = B.hsml[i];
        int k = level_of(hs, S);
        int cx, cy;
        cell_of(p, S, k, cx, cy);
        if (S->sparse) {
            int b = block_of(S, k, cx, cy);
            if (bmark[b] == 0) bmark[b] = 1;
        }
        if (k == 0) h0 = max(h0, f2o(hs));
        else atomicMax(&lmax[k], f2o(hs));
    }
    h0 = __reduce_max_sync(0xffffffffu, h0);
    if ((threadIdx.x & 31) == 0 && h0) atomicMax(&lmax[0], h0);
    __syncthreads();
    for (int k = threadIdx.x; k < nlev; k += blockDim.x)
        if (lmax[k]) atomicMax(&S->lev_hmax_o[k], lmax[k]);
}

// Cell key (slot of the particle's block * 256 + cell within the block) and
// within-cell arrival rank of each particle (counting sort histogram,
// grid_find :938-948); out-of-domain particles get key -1.  Clears the block
// marks for the next step.  If the occupied blocks need more cells than the
// histogram holds, nothing is counted and the step stops with kErrCells.
__global__ void k_hist(const PState B, int n, DemView dem, StepScalars* S, int* bmark, const int* bstart, int* count,
                       int2* keyrank, int cap_cells) {
    PDL_ENTRY();
    if (S->skip) return;
    const bool sparse = S->sparse != 0;
    const long long ncells = sparse ? (long long)bstart[S->nblocks] * kBlockCells : (long long)S->ncells;
    const bool over = ncells + 1 > (long long)cap_cells;
    if (over && blockIdx.x == 0 && threadIdx.x == 0) {
        atomicOr(&S->err, kErrCells);
        S->need_cells = (ncells + 1 > 0x3fffffffLL) ? 0x3fffffff : (int)(ncells + 1);
    }
    if (sparse && !over && blockIdx.x == 0 && threadIdx.x == 0) S->ncells = (int)ncells;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int2 kr = make_int2(-1, 0);
        float2 p = B.pos[i];
        if (!B.flag[i] && !out_of_box(dem, p.x, p.y)) {
            int k = level_of(B.hsml[i], S);
            int cx, cy;
            cell_of(p, S, k, cx, cy);
            int key;
            if (sparse) {
                int b = block_of(S, k, cx, cy);
                bmark[b] = 0;
                key = bstart[b] * kBlockCells + (int)((unsigned)cy % kBlkY) * kBlkX + (int)((unsigned)cx % kBlkX);
            } else {
                key = S->lev_off[k] + cy * S->lev_ndx[k] + cx;
            }
            if (!over) {
                kr.x = key;
                kr.y = atomicAdd(&count[key], 1);
            }
        }
        keyrank[i] = kr;
    }
}

// Exclusive scan of the histogram, tile pass: each block scans kScanTile
// cells and writes its tile total.
// only_sparse: the block-map scan, which dense steps skip.
// Exclusive prefix of the tile sums, by one block (1 <= ntiles <= kScanTops *
// blockDim.x): tile_sum[t] becomes the first index of tile t.
constexpr int kScanTops = 32;
__device__ void scan_tile_sums(int* tile_sum, int ntiles) {
    __shared__ int wsum[32];
    const int per = (ntiles + (int)blockDim.x - 1) / (int)blockDim.x;  // <= kScanTops
    int loc[kScanTops];
    int s = 0;
    for (int k = 0; k < kScanTops; k++) {
        if (k >= per) break;
        int g = threadIdx.x * per + k;
        int v = (g < ntiles) ? ((volatile int*)tile_sum)[g] : 0;
        loc[k] = s;
        s += v;
    }
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = s;
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int w = (lane < (int)(blockDim.x >> 5)) ? wsum[lane] : 0;
        int wi = w;
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < (int)(blockDim.x >> 5)) wsum[lane] = wi - w;
    }
    __syncthreads();
    int off = wsum[wid] + incl - s;
    for (int k = 0; k < kScanTops; k++) {
        if (k >= per) break;
        int g = threadIdx.x * per + k;
        if (g < ntiles) tile_sum[g] = off + loc[k];
    }
}

// Scan of count[0 .. *nptr] into start (exclusive), tile by tile; the last
// tile to finish also scans the tile sums (the tile offsets k_scan_add adds).
// which: 0 the cells, 1 the block map (only in the block-sparse layout).  A
// step whose earlier kernels raised an error is stopped here.
__global__ void k_scan_tiles(const int* count, int* start, int* tile_sum, const int* nptr, StepScalars* S,
                             int which) {
    PDL_ENTRY();
    if (S->skip || (which == 1 && !S->sparse)) return;
    if (S->err) {
        if (blockIdx.x == 0 && threadIdx.x == 0) S->skip = 1;
        return;
    }
    int m = *nptr + 1;
    const int ntiles = (m + kScanTile - 1) / kScanTile;
    int base = blockIdx.x * kScanTile;
    if (base >= m) return;
    __shared__ int sh[kScanTile];
    __shared__ int wsum[kScanThreads / 32];
    __shared__ bool last;
    for (int k = threadIdx.x; k < kScanTile; k += kScanThreads) {
        int g = base + k;
        sh[k] = (g < m) ? count[g] : 0;
    }
    __syncthreads();
    const int per = kScanTile / kScanThreads;
    int loc[per];
    int s = 0;
    for (int k = 0; k < per; k++) { loc[k] = s; s += sh[threadIdx.x * per + k]; }
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = s;
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int w = (lane < kScanThreads / 32) ? wsum[lane] : 0;
        int wi = w;
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < kScanThreads / 32) wsum[lane] = wi - w;
        if (lane == kScanThreads / 32 - 1) tile_sum[blockIdx.x] = wi;
    }
    __syncthreads();
    int off = wsum[wid] + incl - s;
    for (int k = 0; k < per; k++) sh[threadIdx.x * per + k] = off + loc[k];
    __syncthreads();
    for (int k = threadIdx.x; k < kScanTile; k += kScanThreads) {
        int g = base + k;
        if (g < m) start[g] = sh[k];
    }
    if (threadIdx.x == 0) {
        __threadfence();
        last = (atomicAdd(&S->scan_ticket[which], 1u) == (unsigned)ntiles - 1u);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    scan_tile_sums(tile_sum, ntiles);
    if (threadIdx.x == 0) S->scan_ticket[which] = 0u;
}

__global__ void k_scan_add(int* start, const int* tile_sum, const int* nptr, const StepScalars* S, int which) {
    PDL_ENTRY();
    if (S->skip || S->err || (which == 1 && !S->sparse)) return;
    int m = *nptr + 1;
    int base = blockIdx.x * kScanTile;
    if (base >= m) return;
    int add = tile_sum[blockIdx.x];
    for (int k = threadIdx.x; k < kScanTile; k += blockDim.x) {
        int g = base + k;
        if (g < m) start[g] += add;
    }
}

// Scatter (grid_find :952-958): particles to start[cell] + rank (level 0
// first, then the higher levels), out-of-domain particles behind them.
__global__ void k_scatter(const int2* keyrank, int n, const int* start, const int* bstart, StepScalars* S, int* perm) {
    PDL_ENTRY();
    if (S->skip) return;
    int nact = start[S->ncells];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int2 kr = keyrank[i];
        int slot = (kr.x >= 0) ? start[kr.x] + kr.y : nact + atomicAdd(&S->nout, 1);
        perm[slot] = i;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // regular particles: levels 0 .. reg_levels-1 (slots before the first
        // key of level reg_levels; lev_off[nlev] ends the key space)
        const int r = min(S->nlev, S->reg_levels);
        int first = S->sparse ? bstart[S->lev_boff[r]] * kBlockCells : S->lev_off[r];
        int nreg = start[first];
        S->nreg = nreg;
        S->nbig = nact - nreg;
        S->nactive = nact;
    }
}

// Orders each cell's particles by original index, so the within-cell order,
// hence every neighbour-sum order, is independent of atomic arrival order.
__device__ __forceinline__ void insertion_sort_by_id(int* perm, const int* id_old, int a, int b) {
    for (int k = a + 1; k < b; k++) {
        int pk = perm[k];
        int key = id_old[pk];
        int m = k - 1;
        while (m >= a && id_old[perm[m]] > key) { perm[m + 1] = perm[m]; m--; }
        perm[m + 1] = pk;
    }
}

// Also zeroes the histogram it no longer needs, so the counts start at zero
// in the next step without a clearing pass.
__global__ void k_cell_sort(int* perm, const int* id_old, const int* start, int* count, const StepScalars* S) {
    PDL_ENTRY();
    if (S->skip) return;
    int nc = S->ncells;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        insertion_sort_by_id(perm, id_old, start[c], start[c + 1]);
        count[c] = 0;
    }
}

// Gathers the state into the new (cell-sorted) order.
// With icpwp = 3 also the pore-water pressure; with icpwp = 3 or nor_density
// rho0, the depth RK45 keeps at its start (after the h_inf clamp of
// Adaptive_dt_sph_SW :6540, modes 1, 2 and 10).
__global__ void k_reorder(const PState B, int n, const int* perm, const int2* keyrank, PState A, int* cellA,
                          float4* xhm, const StepScalars* S, Rheo c, float* rho0, int2* rcell,
                          const unsigned char* spec_u, unsigned char* spec_a) {
    PDL_ENTRY();
    if (S->skip) return;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        int o = perm[s];
        float2 p = B.pos[o];
        float hs = B.hsml[o], m = B.mass[o];
        float r = B.rho[o];
        A.pos[s] = p;
        A.vel[s] = B.vel[o];
        A.rho[s] = r;
        if (c.icpwp != 0) A.pwp[s] = B.pwp[o];
        if (c.icpwp != 0 || c.nor_density)
            rho0[s] = ((c.ic_adapt == 1 || c.ic_adapt == 2 || c.ic_adapt == 10) && r < c.h_inf) ? c.h_inf : r;
        A.mass[s] = m;
        A.hsml[s] = hs;
        A.flag[s] = B.flag[o];
        A.id[s] = B.id[o];
        if (c.ws) spec_a[s] = spec_u[B.id[o]];
        cellA[s] = keyrank[o].x;
        xhm[s] = make_float4(p.x, p.y, hs, m);
        if (rcell && !B.flag[o]) {  // cell of the reference's grid (:1203-1204)
            int ix = (int)((p.x - S->ref_xmin) / S->ref_delt + 1.f);
            int iy = (int)((p.y - S->ref_ymin) / S->ref_delt + 1.f);
            rcell[s] = make_int2(min(ix, S->ref_ndx), min(iy, S->ref_ndy));
        }
    }
}

// Largest neighbour distance against a level whose hsml <= Hk:
// r < SK*(hi + hj)/2 <= SK/2 (hi + Hk).
template <int SK>
__device__ __forceinline__ float support_span(float hi, float hk) {
    return (SK == 2) ? hi + hk : 1.5f * (hi + hk);
}

// The reference's own cell test, needed for supports of 3 h (skf 2, 3):
// grid_find pairs only particles in the same or adjacent cells of its grid
// of 2*max(hsml) (My_SPH_Tools_2019.f90:1257-1264), so pairs up to 3 h apart
// are kept or dropped by where that grid falls.  (With 2 h supports every
// pair lies within one cell and the test is implied.)
template <int SK>
__device__ __forceinline__ bool ref_adjacent(const Search& Q, int2 ci, int j) {
    if (SK == 2) return true;
    const int2 cj = Q.rcell[j];
    return abs(cj.x - ci.x) <= 1 && abs(cj.y - ci.y) <= 1;
}

// Stencil of level k around particle i: every j of level k has hsml_j <= Hk
// (the level's largest smoothing length), so with r < SK/2 (hi + hj) it lies
// within floor(SK/2 (hi + Hk)/cell + 0.01) + 1 cells of i's cell in that
// level's grid, whatever the rounding of the cell coordinates.  Returns false
// for an empty level.
template <int SK = 2>
__device__ __forceinline__ bool level_stencil(const StepScalars* S, int k, float2 xi, float hi, int& x0, int& x1,
                                              int& y0, int& y1) {
    unsigned int hk = S->lev_hmax_o[k];
    if (hk == 0u) return false;
    float rr = support_span<SK>(hi, o2f(hk)) / S->lev_c[k] + 0.01f;
    int R = (rr < 1.0e8f) ? (int)rr + 1 : 100000000;
    int cx, cy;
    cell_of(xi, S, k, cx, cy);
    x0 = max(cx - R, 0); x1 = min(cx + R, S->lev_ndx[k] - 1);
    y0 = max(cy - R, 0); y1 = min(cy + R, S->lev_ndy[k] - 1);
    return true;
}

// Slot range of the cells x0..x1 of row jy inside block column bx (empty if
// the block holds no particles).
__device__ __forceinline__ void block_row_range(const Search& Q, const StepScalars* S, int k, int jy, int bx, int x0,
                                                int x1, int& ja, int& jb) {
    if (!S->sparse) {  // dense: the row is one key range (bx is 0)
        int row = S->lev_off[k] + jy * S->lev_ndx[k];
        ja = Q.start[row + x0];
        jb = Q.start[row + x1 + 1];
        return;
    }
    int b = S->lev_boff[k] + (int)((unsigned)jy / kBlkY) * S->lev_nbx[k] + bx;
    int s0 = Q.bstart[b];
    if (Q.bstart[b + 1] == s0) { ja = jb = 0; return; }
    int lo = max(x0, bx * kBlkX) - bx * kBlkX, hi = min(x1, bx * kBlkX + kBlkX - 1) - bx * kBlkX;
    int key = s0 * kBlockCells + (int)((unsigned)jy % kBlkY) * kBlkX;
    ja = Q.start[key + lo];
    jb = Q.start[key + hi + 1];
}

// Pair test of particle i (reference-grid cell ci) against the slots ja..jb-1.
template <int SK, class F>
__device__ __forceinline__ void visit_range(const Search& Q, int i, float2 xi, float hi, int2 ci, int ja, int jb,
                                            F& f) {
    for (int j = ja; j < jb; j++) {
        if (j == i) continue;
        float4 o = Q.xhm[j];
        PairGeom g;
        if (pair_search<SK>(xi, make_float2(o.x, o.y), hi, o.z, g) && ref_adjacent<SK>(Q, ci, j)) f(j, o, g);
    }
}

// Visits the particles j != i of level k that are neighbours of particle i
// (position xi, smoothing length hi), row by row of the stencil, each row in
// cell order.  Rows further than one cell from i's row are trimmed to the
// circle: a particle of row jy, d = |jy - cy| >= 2 rows away, is more than
// (d - 1) cells away in y, so with r < hi + Hk it lies within
// sqrt(rr^2 - (d - 1)^2) + 1 cells in x (rr and d - 1 carry 0.01-cell
// margins for the rounding of the cell coordinates).  A dense row is one key
// range; a sparse row is one range per block column it crosses.
template <bool SPARSE, int SK, class F>
__device__ __forceinline__ void level_neighbours(const Search& Q, const StepScalars* S, int k, int i, float2 xi, float hi,
                                                 int2 ci, F&& f) {
    const unsigned int hk = S->lev_hmax_o[k];
    if (hk == 0u) return;
    const float rr = support_span<SK>(hi, o2f(hk)) / S->lev_c[k] + 0.01f;
    const int R = (rr < 1.0e8f) ? (int)rr + 1 : 100000000;
    const float rr2 = rr * rr;
    int cx, cy;
    cell_of(xi, S, k, cx, cy);
    const int ndx = S->lev_ndx[k], nbx = S->lev_nbx[k], boff = S->lev_boff[k];
    const int y0 = max(cy - R, 0), y1 = min(cy + R, S->lev_ndy[k] - 1);
    for (int jy = y0; jy <= y1; jy++) {
        const int d = abs(jy - cy);
        int rx = R;
        if (d >= 2) {
            const float dd = (float)d - 1.01f;
            const float q = rr2 - dd * dd;
            if (!(q > 0.f)) continue;
            rx = min(R, (int)sqrtf(q) + 1);
        }
        const int x0 = max(cx - rx, 0), x1 = min(cx + rx, ndx - 1);
        if (!SPARSE) {
            const int rowoff = S->lev_off[k] + jy * ndx;
            visit_range<SK>(Q, i, xi, hi, ci, Q.start[rowoff + x0], Q.start[rowoff + x1 + 1], f);
            continue;
        }
        const int c0 = (int)((unsigned)x0 / kBlkX), c1 = (int)((unsigned)x1 / kBlkX);
        const int brow = boff + (int)((unsigned)jy / kBlkY) * nbx;
        const int row = (int)((unsigned)jy % kBlkY) * kBlkX;
        if (c1 - c0 <= 1) {
            // one or two block columns: the two slot ranges are walked as one
            // sequence, so lanes whose rows straddle a block edge and lanes
            // whose rows do not run the same loop (no divergent second pass)
            const int s0 = Q.bstart[brow + c0], s1 = Q.bstart[brow + c0 + 1];
            const int e0 = min(x1, c0 * kBlkX + kBlkX - 1);
            int ja = 0, na = 0, jb = 0, nb = 0;
            if (s1 != s0) {
                const int key = s0 * kBlockCells + row - c0 * kBlkX;
                ja = Q.start[key + x0];
                na = Q.start[key + e0 + 1] - ja;
            }
            if (c1 > c0) {
                const int s2 = Q.bstart[brow + c1 + 1];
                if (s2 != s1) {
                    const int key = s1 * kBlockCells + row - c1 * kBlkX;
                    jb = Q.start[key + c1 * kBlkX];
                    nb = Q.start[key + x1 + 1] - jb;
                }
            }
            for (int t = 0; t < na + nb; t++) {
                const int j = (t < na) ? ja + t : jb + (t - na);
                if (j == i) continue;
                float4 o = Q.xhm[j];
                PairGeom g;
                if (pair_search<SK>(xi, make_float2(o.x, o.y), hi, o.z, g) && ref_adjacent<SK>(Q, ci, j)) f(j, o, g);
            }
            continue;
        }
        int s1 = Q.bstart[brow + c0];
        for (int bx = c0; bx <= c1; bx++) {
            const int s0 = s1;
            s1 = Q.bstart[brow + bx + 1];  // end of this block = start of the next
            if (s1 == s0) continue;
            const int key = s0 * kBlockCells + row - bx * kBlkX;
            visit_range<SK>(Q, i, xi, hi, ci, Q.start[key + max(x0, bx * kBlkX)],
                        Q.start[key + min(x1, bx * kBlkX + kBlkX - 1) + 1], f);
        }
    }
}

// Neighbour search and summation density of the regular particles, fused:
// every j with r < 2*(hi+hj)/2 (the pair set of grid_find, :987-1060), on
// every level, is appended to the neighbour table (tab_base) with the pair's
// kernel value and gradient, and h_i = W(0,h_i) m_i + sum_j m_j W_ij
// (sum_density_Tools :1796-1836) is accumulated in FP64.  Also stores the
// pressure term of IntForces_SW with h clamped to h_inf (:6769, :6797): p/h^2
// (pa_sph 2) or p (pa_sph 1).
template <bool SPARSE, int SKF, bool WS>
__device__ __forceinline__ void density_regular(PState& A, const Search& Q, StepScalars* S, const Rheo& c) {
    constexpr int SK = SupportScale<SKF>::value;
    const int nreg = S->nreg, nlev = S->nlev;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nreg; i += gridDim.x * blockDim.x) {
        float4 me = Q.xhm[i];
        float2 xi = make_float2(me.x, me.y);
        float hi = me.z;
        const int2 ci = (SK == 2) ? make_int2(0, 0) : Q.rcell[i];
        double acc = (double)(sph_kernel_w<SKF>(0.f, hi) * me.w);
        int4* tab = Q.nbr + tab_base(i, Q.kcap);
        int cnt = 0;
        const unsigned char si = WS ? Q.spec[i] : 0;
        for (int k = 0; k < nlev; k++)
            level_neighbours<SPARSE, SK>(Q, S, k, i, xi, hi, ci, [&](int j, float4 o, const PairGeom& g) {
                // W and grad W of the pair, once per step: the internal force,
                // av_vel and the normalisation read them from the table
                float w, d0, d1;
                sph_kernel<SKF>(g.r, g.dx0, g.dx1, g.mh, w, d0, d1);
                const bool cross = WS && Q.spec[j] != si;
                if (cnt < Q.kcap)  // kept in L2 for the internal force (written back to front)
                    tab[(size_t)cnt * kTabStride] =
                        make_int4(cross ? (j | kCrossBit) : j, __float_as_int(w), __float_as_int(d0),
                                  __float_as_int(d1));
                cnt++;
                if (!cross) acc += (double)(o.w * w);
            });
        Q.ncount[i] = cnt;
        if (cnt > Q.kcap) {  // table too small: stop this step before any state is written
            atomicOr(&S->err, kErrNbr);
            atomicMax(&S->need_nbr, cnt);
            atomicExch(&S->skip, 1);
        }
        float h = (float)acc;
        A.rho[i] = h;
        float hc = (h < c.h_inf) ? c.h_inf : h;
        float p = (c.cgra05 * hc) * hc;
        const float pt = (c.pa_sph == 1) ? p : p / (hc * hc);
        Q.pterm[i] = pt;
        Q.pr[i] = make_float4(pt, h, me.w, 0.f);
    }
}

// Instantiated for both cell layouts; the launch whose layout this step does
// not use returns at once (one kernel with both walks would spill in the
// dense walk).  Held to 48 registers (10 blocks of 128 per SM): the gathers
// are latency-bound.
template <bool SPARSE, int SKF, bool WS>
__global__ void __launch_bounds__(128, 10) k_density(PState A, Search Q, StepScalars* S, Rheo c, int n) {
    PDL_ENTRY();
    if (S->skip || (S->sparse != 0) != SPARSE) return;
    density_regular<SPARSE, SKF, WS>(A, Q, S, c);
}

// Visits every neighbour j of particle i cooperatively over one warp: the
// lanes fetch the slot ranges of up to 32 (row, block column) segments of the
// stencil at once, then share each segment's candidates.
template <int SK, class F>
__device__ __forceinline__ void warp_neighbours(const Search& Q, const StepScalars* S, int i, int lane, F&& f) {
    const float4 me = Q.xhm[i];
    const float2 xi = make_float2(me.x, me.y);
    const float hi = me.z;
    const int2 ci = (SK == 2) ? make_int2(0, 0) : Q.rcell[i];
    for (int k = 0; k < S->nlev; k++) {
        int x0, x1, y0, y1;
        if (!level_stencil<SK>(S, k, xi, hi, x0, x1, y0, y1)) continue;
        const int bx0 = S->sparse ? (int)((unsigned)x0 / kBlkX) : 0;
        const int ncol = S->sparse ? (int)((unsigned)x1 / kBlkX) - bx0 + 1 : 1;
        const long long nseg = (long long)(y1 - y0 + 1) * ncol;
        for (long long sb = 0; sb < nseg; sb += 32) {
            long long sg = sb + lane;
            int ja = 0, jb = 0;
            if (sg < nseg) {
                int jy = y0 + (int)(sg / ncol), bx = bx0 + (int)(sg % ncol);
                block_row_range(Q, S, k, jy, bx, x0, x1, ja, jb);
            }
            int nr = (int)min(32LL, nseg - sb);
            for (int r = 0; r < nr; r++) {
                int a = __shfl_sync(0xffffffffu, ja, r), e = __shfl_sync(0xffffffffu, jb, r);
                for (int j = a + lane; j < e; j += 32) {
                    if (j == i) continue;
                    float4 o = Q.xhm[j];
                    PairGeom g;
                    if (pair_search<SK>(xi, make_float2(o.x, o.y), hi, o.z, g) && ref_adjacent<SK>(Q, ci, j))
                        f(j, o, g);
                }
            }
        }
    }
}

// Summation density of the coarse-level particles, one warp per particle.
template <int SKF>
__global__ void __launch_bounds__(128) k_density_big(PState A, Search Q, StepScalars* S, Rheo c) {
    PDL_ENTRY();
    constexpr int SK = SupportScale<SKF>::value;
    if (S->skip) return;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nreg = S->nreg, nbig = S->nbig;
    for (int b = warp; b < nbig; b += nwarps) {
        int i = nreg + b;
        double acc = 0.0;
        const unsigned char si = c.ws ? Q.spec[i] : 0;
        warp_neighbours<SK>(Q, S, i, lane, [&](int j, float4 o, const PairGeom& g) {
            if (c.ws && Q.spec[j] != si) return;  // type 1: not in the density (:1829)
            acc += (double)(o.w * sph_kernel_w<SKF>(g.r, g.mh));
        });
        acc = warp_sum(acc);
        if (lane == 0) {
            float4 me = Q.xhm[i];
            float h = (float)((double)(sph_kernel_w<SKF>(0.f, me.z) * me.w) + acc);
            A.rho[i] = h;
            float hc = (h < c.h_inf) ? c.h_inf : h;
            float p = (c.cgra05 * hc) * hc;
            const float pt = (c.pa_sph == 1) ? p : p / (hc * hc);
            Q.pterm[i] = pt;
            Q.pr[i] = make_float4(pt, h, me.w, 0.f);
        }
    }
}

// One pair term of IntForces_SW (SPH_SW_2019.f90:6905-6920) for particle i,
// from the pair's kernel gradient (d0, d1).
__device__ __forceinline__ void pressure_terms(const Rheo& c, float pi_, float rhoi, float pj, float rhoj, float mj,
                                               float d0, float d1, double& a0, double& a1) {
    float h0, h1;
    if (c.pa_sph == 1) {
        rhoi = (rhoi < c.h_inf) ? c.h_inf : rhoi;
        rhoj = (rhoj < c.h_inf) ? c.h_inf : rhoj;
        float rij = 1.f / (rhoi * rhoj);
        h0 = (-(pi_ + pj) * d0) * rij;
        h1 = (-(pi_ + pj) * d1) * rij;
    } else {
        h0 = -(pi_ + pj) * d0;
        h1 = -(pi_ + pj) * d1;
    }
    a0 += (double)(mj * h0);
    a1 += (double)(mj * h1);
}

// The same with the pair geometry: the kernel gradient evaluated here.
template <int SKF>
__device__ __forceinline__ void pressure_pair(const Rheo& c, float pi_, float rhoi, float pj, float rhoj, float mj,
                                              const PairGeom& g, double& a0, double& a1) {
    float w, d0, d1;
    sph_kernel<SKF>(g.r, g.dx0, g.dx1, g.mh, w, d0, d1);
    pressure_terms(c, pi_, rhoi, pj, rhoj, mj, d0, d1, a0, a1);
}

// Internal acceleration of the coarse-level particles, one warp per particle.
template <int SKF>
__global__ void __launch_bounds__(128) k_force_big(PState A, Search Q, StepScalars* S, Rheo c) {
    PDL_ENTRY();
    constexpr int SK = SupportScale<SKF>::value;
    if (S->skip) return;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nreg = S->nreg, nbig = S->nbig;
    for (int b = warp; b < nbig; b += nwarps) {
        int i = nreg + b;
        const float4 pri = Q.pr[i];
        double a0 = 0.0, a1 = 0.0;
        const unsigned char si = c.ws ? Q.spec[i] : 0;
        warp_neighbours<SK>(Q, S, i, lane, [&](int j, float4 o, const PairGeom& g) {
            if (c.ws && Q.spec[j] != si) return;  // type 0 only (:6899)
            const float4 prj = Q.pr[j];
            pressure_pair<SKF>(c, pri.x, pri.y, prj.x, prj.y, o.w, g, a0, a1);
        });
        a0 = warp_sum(a0);
        a1 = warp_sum(a1);
        if (lane == 0) Q.indv[i] = make_float2((float)a0, (float)a1);
    }
}

// Internal acceleration of a regular particle over its neighbour table: per
// entry the stored kernel gradient and one gather of (p-term, h, m) of the
// neighbour.  The table is read four entries at a time so that four
// independent gathers are in flight per thread; the FP64 sum keeps the table
// order.
template <bool WS>
__device__ __forceinline__ void internal_force(const Search& Q, const Rheo& c, int i, float& in0, float& in1) {
    const float4 pri = __ldg(&Q.pr[i]);
    const float pi_ = pri.x, rhoi = pri.y;
    double a0 = 0.0, a1 = 0.0;
    const int cnt = Q.ncount[i];
    const int4* tab = Q.nbr + tab_base(i, Q.kcap);
    int k = 0;
    for (; k + 4 <= cnt; k += 4) {
        int4 e[4];
        float4 prj[4];
#pragma unroll
        for (int u = 0; u < 4; u++) e[u] = __ldg(tab + (size_t)(k + u) * kTabStride);
#pragma unroll
        for (int u = 0; u < 4; u++) prj[u] = __ldg(&Q.pr[WS ? (e[u].x & ~kCrossBit) : e[u].x]);
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (!WS || e[u].x >= 0)  // type 0 only (:6899)
                pressure_terms(c, pi_, rhoi, prj[u].x, prj[u].y, prj[u].z, __int_as_float(e[u].z),
                               __int_as_float(e[u].w), a0, a1);
    }
    for (; k < cnt; k++) {
        const int4 e = __ldg(tab + (size_t)k * kTabStride);
        const float4 prj = __ldg(&Q.pr[WS ? (e.x & ~kCrossBit) : e.x]);
        if (!WS || e.x >= 0)
            pressure_terms(c, pi_, rhoi, prj.x, prj.y, prj.z, __int_as_float(e.z), __int_as_float(e.w), a0, a1);
    }
    in0 = (float)a0;
    in1 = (float)a1;
}

// DEM node box touched by the erosion scatter, kept per thread and reduced
// per block before the four atomics on the step scalars (same-address
// atomics from every warp serialise).
struct NodeBox {
    int x0, x1, y0, y1;
};
__device__ __forceinline__ NodeBox empty_node_box() { return NodeBox{INT_MAX, INT_MIN, INT_MAX, INT_MIN}; }

// Every thread of the block must call it (one __syncthreads).
__device__ __forceinline__ void flush_node_box(StepScalars* S, NodeBox b) {
    __shared__ NodeBox wb[32];
    const unsigned full = 0xffffffffu;
    b.x0 = __reduce_min_sync(full, b.x0); b.x1 = __reduce_max_sync(full, b.x1);
    b.y0 = __reduce_min_sync(full, b.y0); b.y1 = __reduce_max_sync(full, b.y1);
    if ((threadIdx.x & 31) == 0) wb[threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
        NodeBox t = wb[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
            t.x0 = min(t.x0, wb[w].x0); t.x1 = max(t.x1, wb[w].x1);
            t.y0 = min(t.y0, wb[w].y0); t.y1 = max(t.y1, wb[w].y1);
        }
        if (t.x1 >= t.x0) {
            atomicMin(&S->ex0, t.x0); atomicMax(&S->ex1, t.x1);
            atomicMin(&S->ey0, t.y0); atomicMax(&S->ey1, t.y1);
        }
    }
}

// DEM scatter of ExtForces_SW(1) (SPH_SW_2019.f90:8731-8750): the particle
// adds base/dist and 1/dist to the 4x4 DEM nodes around its DEM cell.
// Consecutive particles of the cell-sorted order mostly share a DEM cell, so
// within a warp the lanes form runs of equal DEM cell.  Each lane writes its
// 32 FP32 terms (16 nodes x {base/dist, 1/dist}) to shared memory; then lane t
// adds up term t over each run of lanes, in lane order and in FP64, and
// issues that run's atomic for it.  The run boundaries are the same for every
// lane, so the summing loop does not diverge.  Lanes with part == false take
// no part; every lane of the warp must call this, in blocks of at most
// kScatterWarps warps.
constexpr int kScatterWarps = 4;
__device__ __forceinline__ void erosion_scatter(const DemView& dem, float xx, float xy, float base, bool part,
                                                double2* auxv, NodeBox& box) {
    __shared__ float sterm[kScatterWarps][32][33];  // [term][lane], padded against bank conflicts
    __shared__ int skey[kScatterWarps][33], spx[kScatterWarps][32], spy[kScatterWarps][32];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int ipx = 0, ipy = 0, key = -1 - lane;  // non-participants: singleton runs with zero terms
    if (part) {
        ipx = (int)((xx - dem.xmin) / dem.dx + 1.f);
        ipy = (int)((xy - dem.ymin) / dem.dy + 1.f);
        key = ipy * (dem.nx + 2) + ipx;
    }
    if (!__any_sync(full, part)) return;
    float(*T)[33] = sterm[wid];
    // the 4x4 nodes (ipx-1..ipx+2) x (ipy-1..ipy+2); nodes outside the DEM add zero
    for (int o = 0; o < 16; o++) {
        const int ix = ipx + (o >> 2) - 1, iy = ipy + (o & 3) - 1;
        const bool inside = part && ix >= 1 && ix <= dem.nx && iy >= 1 && iy <= dem.ny;
        float a = 0.f, b = 0.f;
        if (inside) {
            float ddx = xx - (dem.xmin + (float)(ix - 1) * dem.dx);
            ddx = ddx * ddx;
            float ddy = xy - (dem.ymin + (float)(iy - 1) * dem.dy);
            ddy = ddy * ddy;
            float dist = sqrtf(ddx + ddy);
            dist = (1.e-6f > dist) ? 1.e-6f : dist;
            a = base / dist;
            b = 1.f / dist;
        }
        T[o][lane] = a;
        T[16 + o][lane] = b;
    }
    skey[wid][lane] = key;
    if (lane == 0) skey[wid][32] = INT_MIN;  // no key: closes the last run
    spx[wid][lane] = ipx;
    spy[wid][lane] = ipy;
    __syncwarp();
    const int o = lane & 15, ox = (o >> 2) - 1, oy = (o & 3) - 1;
    double acc = 0.0;
    int kr = skey[wid][0];
    for (int r = 0; r < 32; r++) {
        acc += (double)T[lane][r];
        const int kn = skey[wid][r + 1];
        if (kn != kr) {  // run ends at lane r (the same r for every lane)
            if (kr >= 0) {
                const int ix = spx[wid][r] + ox, iy = spy[wid][r] + oy;
                if (ix >= 1 && ix <= dem.nx && iy >= 1 && iy <= dem.ny) {
                    double* dst = &auxv[(iy - 1) * dem.nx + (ix - 1)].x;
                    atomicAdd(dst + (lane >> 4), acc);  // .x for base/dist, .y for 1/dist
                }
            }
            acc = 0.0;
            kr = kn;
        }
    }
    __syncwarp();  // the terms are rewritten by the next call
    if (part) {
        box.x0 = min(box.x0, max(1, ipx - 1)); box.x1 = max(box.x1, min(dem.nx, ipx + 2));
        box.y0 = min(box.y0, max(1, ipy - 1)); box.y1 = max(box.y1, min(dem.ny, ipy + 2));
    }
}

// A particle out of the domain at the start of the step: copied through.
__device__ __forceinline__ void rk_carry(const PState& A, const Rheo& c, const PState& B, float2* velfin, float4* xsv,
                                         int i) {
    B.pos[i] = A.pos[i]; B.vel[i] = A.vel[i]; velfin[i] = A.vel[i];
    xsv[i] = make_float4(A.vel[i].x, A.vel[i].y, A.rho[i], A.mass[i]);
    B.rho[i] = A.rho[i]; B.mass[i] = A.mass[i]; B.hsml[i] = A.hsml[i];
    B.flag[i] = A.flag[i]; B.id[i] = A.id[i];
    if (c.icpwp == 3) B.pwp[i] = 0.f;  // Get_Pwp_SW zeroes out-of-domain particles
    if (c.icpwp == 1) B.pwp[i] = A.pwp[i];  // u of a frozen particle stays
}

// The end of the RK45 body of an active particle: the final update
// (SPH_MAIN_2019.f90:908-922), Check_Out_Domain, Hungr erosion of the mass
// and the DEM scatter of ExtForces_SW(1) (SPH_SW_2019.f90:8717-8760),
// h_upgrade (:2925-2931) and the pore-pressure update, written to B.  h is
// the step's final depth; (xx, xy, vx, vy) the last stage's state, kept as
// the result when the particle left the domain in a stage (out).  Every lane
// of the warp must call it (erosion_scatter).
template <bool GEN = true>
__device__ __forceinline__ void rk_finish(const PState& A, const Search& Q, StepScalars* S, const Rheo& c,
                                          const DemView& dem, const PState& B, float2* velfin, double2* auxv, int i,
                                          float dt, float2 x0, float2 v0, float Dx0, float Dx1, float Dv0, float Dv1,
                                          float xx, float xy, float vx, float vy, bool out, float h, float pwp,
                                          float u0, float Du, float acc0, float acc1, NodeBox& box) {
    float m = A.mass[i];
    float hs = A.hsml[i];
    if (!out) {
        float dt6 = dt / 6.f;
        xx = x0.x + dt6 * Dx0;
        xy = x0.y + dt6 * Dx1;
        vx = v0.x + dt6 * Dv0;
        vy = v0.y + dt6 * Dv1;
        if (c.icpwp == 1) pwp = u0 + dt6 * Du;  // u of icpwp 1 (:921); else pwp is the stage's u
        out = out_of_box(dem, xx, xy);
    }
    float er = 0.f;
    if (!out && c.erosion)
        er = erosion_rate_final<GEN>(c, dem, xx, xy, vx, vy, h, pwp, soil_fraction(c, Q, A, i), acc0, acc1, dt);
    if (c.erosion) erosion_scatter(dem, xx, xy, dt * er, !out, auxv, box);
    if (!out) {
        if (c.erosion) m = m + ((dt * er) * m) / h;
        if (c.sle == 1) hs = 2.f * sqrtf(m / h);
    }
    B.pos[i] = make_float2(xx, xy);
    velfin[i] = make_float2(vx, vy);
    Q.xsv[i] = make_float4(vx, vy, h, m);
    B.vel[i] = make_float2(vx, vy);
    B.rho[i] = h;
    B.mass[i] = m;
    B.hsml[i] = hs;
    B.flag[i] = out ? 1 : 0;
    B.id[i] = A.id[i];
    if (c.icpwp == 3) B.pwp[i] = out ? 0.f : pwp_update(c, pwp, h, h - Q.rho0[i], dt);
    if (c.icpwp == 1) {  // bounded by the depth after ExtForces_SW(1), RK45 :974-979
        if (!out) {
            if (pwp > h) pwp = h;
            if (pwp < 0.f) pwp = 0.f;
        }
        B.pwp[i] = pwp;
    }
}

// Internal acceleration of the regular particles, one thread each.  The
// warps take the particles from the last to the first warp of the table:
// the neighbour search has just written the table front to back, so its
// last-written part (still in L2) is read first, and av_vel, which walks
// the table front to back after this pass, starts on the part this pass
// read last.
template <int SKF, bool WS>
__global__ void __launch_bounds__(128) k_iforce(PState A, Search Q, StepScalars* S, Rheo c, int n) {
    PDL_ENTRY();
    if (S->skip) return;
    const int nreg = S->nreg;
    const int nw = (nreg + 31) >> 5;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nw * 32; t += gridDim.x * blockDim.x) {
        const int i = (nw - 1 - (t >> 5)) * 32 + (t & 31);
        if (i >= nreg) continue;
        float in0, in1;
        internal_force<WS>(Q, c, i, in0, in1);
        Q.indv[i] = make_float2(in0, in1);
    }
}

// The RK45 body for each active particle, entirely in registers: the
// internal acceleration (stage-invariant, see below; from k_iforce or
// k_force_big), four stages of
// x = x0 + c_i dt v, v = v0 + c_i dt (ex + in) with ExtForces_SW(0) at each
// stage (SPH_MAIN_2019.f90:808-906), the final update (:908-922), the
// out-of-domain freeze (Check_Out_Domain), Hungr erosion of mass and the DEM
// scatter of ExtForces_SW(1) (:8717-8760), and h_upgrade (:2925-2931).
//
// Why the internal force is computed once: with summation density the stage
// density depends only on masses, hsml and the frozen W_ij, none of which
// change inside the step, so IntForces_SW returns the same value in all four
// stages.  (A particle that leaves the DEM box mid-step is frozen; the
// reference then keeps scattering its stale pressure into its neighbours for
// the remaining stages, which is not reproduced.)
// PWP1 (icpwp = 1) carries u through the stages; GEN compiles every basal
// law and erosion law (else only nfric 4-8, 26, 27 and erosion law 1).  The
// other runs are compiled without them, so their stage loop keeps its
// registers and its code small.
template <bool PWP1, bool GEN>
__global__ void __launch_bounds__(128, 6) k_force_rk(PState A, Search Q, StepScalars* S, Rheo c, DemView dem, int n,
                                                   PState B, float2* velfin, double2* auxv, int forces_only,
                                                   float2* indv_out) {
    PDL_ENTRY();
    if (S->skip) return;
    const int nact = S->nactive;
    const float dt = S->dt_step;
    if (forces_only) {
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nact; i += gridDim.x * blockDim.x)
            indv_out[i] = Q.indv[i];
        return;
    }
    // block-uniform trip count: every lane of a warp reaches erosion_scatter,
    // every thread the box flush
    NodeBox box = empty_node_box();
    for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        const int i = i0 + threadIdx.x;
        if (i >= n) {
            if (c.erosion) erosion_scatter(dem, 0.f, 0.f, 0.f, false, auxv, box);
            continue;
        }
        if (i >= nact) {  // carried particles (out of the domain at step start)
            rk_carry(A, c, B, velfin, Q.xsv, i);
            if (c.erosion) erosion_scatter(dem, 0.f, 0.f, 0.f, false, auxv, box);
            continue;
        }
        const float2 fin = Q.indv[i];
        const float in0 = fin.x, in1 = fin.y;
        const float h = A.rho[i];
        const float hc = (h < c.h_inf) ? c.h_inf : h;  // IntForces_SW clamp, seen by ExtForces_SW(0)
        const float2 x0 = A.pos[i], v0 = A.vel[i];
        // icpwp 3: Uaux(1) of the step start; icpwp 1: u0, then u of each stage
        const float u0 = (c.icpwp != 0) ? A.pwp[i] : 0.f;
        float pwp = u0, du = 0.f, Du = 0.f;
        const float nsoil = soil_fraction(c, Q, A, i);
        float xx = x0.x, xy = x0.y, vx = v0.x, vy = v0.y;
        float ex0 = 0.f, ex1 = 0.f;
        float Dx0 = 0.f, Dx1 = 0.f, Dv0 = 0.f, Dv1 = 0.f;
        bool out = false;
#pragma unroll 1  // one copy of ExtForces_SW(0): the unrolled body overflows the instruction cache
        for (int s = 0; s < 4; s++) {
            const float f1 = (s == 0) ? 0.f : (s == 3 ? 1.f : 0.5f);
            const float f2 = (s == 0 || s == 3) ? 1.f : 2.f;
            if (!out) {
                float fdt = f1 * dt;
                float nxx = x0.x + fdt * vx;
                float nxy = x0.y + fdt * vy;
                float nvx = v0.x + fdt * (ex0 + in0);
                float nvy = v0.y + fdt * (ex1 + in1);
                xx = nxx; xy = nxy; vx = nvx; vy = nvy;
                if (PWP1) {  // RK45 :823-830, bounded by the depth as the stage finds it
                    pwp = u0 + fdt * du;
                    const float rc = (s == 0) ? Q.rho0[i] : hc;
                    if (pwp > rc) pwp = rc;
                    else if (pwp < 0.f) pwp = 0.f;
                }
                if (out_of_box(dem, xx, xy)) {
                    out = true;
                } else {
                    ext_accel<false, GEN>(c, dem, dt, xx, xy, vx, vy, hc, pwp, nsoil, in0, in1, ex0, ex1);
                    if (PWP1) {
                        du = pwp1_rate(c, hc, pwp, dt);
                        Du = Du + f2 * du;
                    }
                    Dv0 = Dv0 + f2 * (ex0 + in0);
                    Dv1 = Dv1 + f2 * (ex1 + in1);
                    Dx0 = Dx0 + f2 * vx;
                    Dx1 = Dx1 + f2 * vy;
                }
            }
        }
        rk_finish<GEN>(A, Q, S, c, dem, B, velfin, auxv, i, dt, x0, v0, Dx0, Dx1, Dv0, Dv1, xx, xy, vx, vy, out, h, pwp,
                       u0, Du, GEN ? ex0 + in0 : 0.f, GEN ? ex1 + in1 : 0.f, box);
    }
    if (c.erosion) flush_node_box(S, box);
}

// ---------------------------------------------------------------- staged RK45
// With nor_density or ic_cosTheta = 1 the pressure changes from stage to
// stage: each sum_density_Tools call divides the plain sum by
// sum_j (m_j/h_j) W_ij taken with the depths of the call before it
// (My_SPH_Tools_2019.f90:1790-1846), and ic_cosTheta = 1 takes g/deng at each
// stage's position (IntForces_SW :6775-6783).  The step then runs stage by
// stage.  The five depths of the step (four stages and the sum after the
// final update) depend only on the frozen W_ij, the masses and the depths
// before them, so they are computed first (k_norm); then each stage runs the
// internal force over the neighbour table with that stage's pressure term
// and the RK stage of every particle (k_stage), whose state is carried in
// HBM between the launches; the last stage also finishes the step
// (k_stage_final).  The pressure term of stage s+1 is written by stage s,
// once the particle's stage position is known.

// RK45 state carried between the stage launches (slot order).
struct StageCarry {
    float2* v;    // velocity of the last stage
    float2* acc;  // ex + in of the last stage
    float2* dx;   // Dx_RK
    float2* dv;   // Dvx_RK
    float2* xo;   // stage position of a particle that left the DEM box
    int* out;     // 1 once it has (it is frozen for the rest of the step)
    // icpwp = 1: u of the last stage (kept by a particle that left), its
    // rate du and Du_RK
    float* u;
    float* du;
    float* Du;
};

// The stage value of icpwp 1's u (RK45 :823-830): u0 + f1 dt du of the
// previous stage, bounded by the depth that stage left (the step start's,
// after Adaptive_dt's clamp, in stage 0; else IntForces_SW's clamp to h_inf).
__device__ __forceinline__ float pwp1_stage(const Rheo& c, const PState& A, const Search& Q, const StageCarry& C,
                                            int s, int i, float fdt, const float* hprev) {
    float u = A.pwp[i] + fdt * ((s > 0) ? C.du[i] : 0.f);
    float rc = Q.rho0[i];
    if (s > 0) {
        rc = hprev[i];
        if (rc < c.h_inf) rc = c.h_inf;
    }
    if (u > rc) u = rc;
    else if (u < 0.f) u = 0.f;
    C.u[i] = u;
    return u;
}

// Its rate of this stage and the running Du_RK.
__device__ __forceinline__ void pwp1_accumulate(const Rheo& c, const StageCarry& C, int s, int i, float hc, float u,
                                                float dt, float f2) {
    const float du = pwp1_rate(c, hc, u, dt);
    C.du[i] = du;
    C.Du[i] = ((s > 0) ? C.Du[i] : 0.f) + f2 * du;
}

// Depth of the previous sum_density_Tools call as the next one reads it:
// clamped to h_inf when IntForces_SW (:6769) has run in between.
__device__ __forceinline__ float prev_depth(const Rheo& c, const float* hp, int j, int clamp_prev) {
    float h = __ldg(hp + j);
    return (clamp_prev && h < c.h_inf) ? c.h_inf : h;
}

// One normalised sum_density_Tools call for the regular particles, over the
// neighbour table: h_i = num_i / (W(0,h_i) m_i/hp_i + sum_j (m_j/hp_j) W_ij),
// num_i the plain sum of k_density (in A.rho), hp the previous call's depths.
template <int SKF>
__global__ void __launch_bounds__(128) k_norm(PState A, Search Q, StepScalars* S, Rheo c, int n, const float* hp,
                                              int clamp_prev, float* hout) {
    PDL_ENTRY();
    if (S->skip) return;
    const int nreg = S->nreg;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nreg; i += gridDim.x * blockDim.x) {
        const float4 me = Q.xhm[i];
        const float hi = me.z;
        double den = (double)((sph_kernel_w<SKF>(0.f, hi) * me.w) / prev_depth(c, hp, i, clamp_prev));
        const int cnt = Q.ncount[i];
        const int4* tab = Q.nbr + tab_base(i, Q.kcap);
        for (int k = 0; k < cnt; k++) {
            const int4 e = __ldg(tab + (size_t)k * kTabStride);  // read again by the next calls of the step
            const int j = e.x;
            den += (double)((__ldg(&A.mass[j]) / prev_depth(c, hp, j, clamp_prev)) * __int_as_float(e.y));
        }
        hout[i] = A.rho[i] / (float)den;
    }
}

// The same for the coarse-level particles, one warp each.
template <int SKF>
__global__ void __launch_bounds__(128) k_norm_big(PState A, Search Q, StepScalars* S, Rheo c, const float* hp,
                                                  int clamp_prev, float* hout) {
    PDL_ENTRY();
    constexpr int SK = SupportScale<SKF>::value;
    if (S->skip) return;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nreg = S->nreg, nbig = S->nbig;
    for (int b = warp; b < nbig; b += nwarps) {
        const int i = nreg + b;
        double den = 0.0;
        warp_neighbours<SK>(Q, S, i, lane, [&](int j, float4 o, const PairGeom& g) {
            den += (double)((o.w / prev_depth(c, hp, j, clamp_prev)) * sph_kernel_w<SKF>(g.r, g.mh));
        });
        den = warp_sum(den);
        if (lane == 0) {
            const float4 me = Q.xhm[i];
            den = (double)((sph_kernel_w<SKF>(0.f, me.z) * me.w) / prev_depth(c, hp, i, clamp_prev)) + den;
            hout[i] = A.rho[i] / (float)den;
        }
    }
}

// Pressure term of IntForces_SW for depth h at (xx, yy): h clamped to h_inf
// (:6769), p = (g_z/2) h^2 (:6797) with g_z = g/deng there when COS
// (:6775-6783); p/h^2 for pa_sph 2, p for pa_sph 1.
template <bool COS>
__device__ __forceinline__ float stage_pterm(const Rheo& c, const DemView& dem, float h, float xx, float yy) {
    const float hc = (h < c.h_inf) ? c.h_inf : h;
    float cg05 = c.cgra05;
    if (COS) {
        float zpx, zpy, top[6];
        dem_lookup(dem, xx, yy, zpx, zpy, false, top);
        cg05 = 0.5f * (c.g / terrain_deng(zpx, zpy));
    }
    const float p = (cg05 * hc) * hc;
    return (c.pa_sph == 1) ? p : p / (hc * hc);
}

// Pressure term of the first stage (positions of the step start).
template <bool COS>
__global__ void __launch_bounds__(128) k_stage_begin(PState A, Search Q, StepScalars* S, Rheo c, DemView dem,
                                                     const float* h1) {
    PDL_ENTRY();
    if (S->skip) return;
    const int nact = S->nactive;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nact; i += gridDim.x * blockDim.x) {
        const float2 p = A.pos[i];
        const float pt = stage_pterm<COS>(c, dem, h1[i], p.x, p.y);
        Q.pterm[i] = pt;
        Q.pr[i] = make_float4(pt, h1[i], A.mass[i], 0.f);
    }
}

// ---------------------------------------------------- soil and water (ic_ws_Interact = 1)
// Position of an active particle in RK45 stage s (s = 0: the step start; a
// frozen particle has none).  The same arithmetic as k_stage's.
__device__ __forceinline__ bool wir_stage_pos(const PState& A, const StageCarry& C, int s, float dt, int i,
                                              float2& p) {
    if (s == 0) {
        p = A.pos[i];
        return true;
    }
    if (C.out[i]) return false;
    const float f1 = (s == 3) ? 1.f : 0.5f;
    const float2 x0 = A.pos[i], vp = C.v[i];
    const float fdt = f1 * dt;
    p = make_float2(x0.x + fdt * vp.x, x0.y + fdt * vp.y);
    return true;
}

// Get_hs_at_w_SW (SPH_SW_2019.f90:17789-17857): each soil particle's depth
// spread over the 4 x 4 DEM nodes around it with weights 1/max(1e-6, dist),
// summed in FP64.
__global__ void __launch_bounds__(128) k_wir_scatter(PState A, Search Q, StepScalars* S, Rheo c, DemView dem,
                                                     StageCarry C, int s, const float* hdep, double2* acc) {
    PDL_ENTRY();
    if (S->skip) return;
    const int nact = S->nactive;
    const float dt = S->dt_step;
    // the same terms h/dist and 1/dist as the erosion scatter, combined over
    // runs of lanes with equal DEM cells before one FP64 atomic per run;
    // block-uniform trip count: every lane of a warp reaches the scatter
    NodeBox box = empty_node_box();
    for (int i0 = blockIdx.x * blockDim.x; i0 < nact; i0 += gridDim.x * blockDim.x) {
        const int i = i0 + threadIdx.x;
        float2 p = make_float2(0.f, 0.f);
        float h = 0.f;
        bool part = false;
        if (i < nact && Q.spec[i] == 1 && wir_stage_pos(A, C, s, dt, i, p) && !out_of_box(dem, p.x, p.y)) {
            h = hdep[i];
            part = true;
        }
        erosion_scatter(dem, p.x, p.y, h, part, acc, box);
    }
}

// Z + hs at the DEM nodes (:17861-17867); the accumulators are left zeroed
// for the next stage.
__global__ void k_wir_nodes(double2* acc, const float* z, float* hsz, int np, const StepScalars* S) {
    PDL_ENTRY();
    if (S->skip) return;
    for (int ip = blockIdx.x * blockDim.x + threadIdx.x; ip < np; ip += gridDim.x * blockDim.x) {
        const double2 a = acc[ip];
        hsz[ip] = (a.y > (double)1.e-6f) ? z[ip] + (float)(a.x / a.y) : z[ip];
        acc[ip] = make_double2(0.0, 0.0);
    }
}

// One soil-water pair term of ExtForces_SW (:8502-8521) for particle i from
// its table entry (gradient d of W_ij with x_i - x_j): a soil particle gets
// -dens_ws g m_j grad W; a water particle, with ic_SWalg = 0, +g m_j grad W
// of the pair taken from the soil side (-d here).
__device__ __forceinline__ void wir_pair_term(const Rheo& c, bool water, float mj, float d0, float d1, double& b0,
                                              double& b1) {
    if (!water) {
        b0 -= (double)(((c.dens_ws * c.g) * mj) * d0);
        b1 -= (double)(((c.dens_ws * c.g) * mj) * d1);
    } else if (c.swalg == 0) {
        b0 += (double)(-((c.g * mj) * d0));
        b1 += (double)(-((c.g * mj) * d1));
    }
}

// Per active particle in stage s: at a water particle Z + hs of the soil
// and its gradient, bilinear on its DEM cell (:17869-17933; a particle on the
// far edge of the DEM takes the last cell); then the pressure term of the
// stage (IntForces_SW :6793-6828): g/2 (h^2 - Zp^2) for the water with
// ic_SWalg = 1, g/2 h^2 otherwise, h clamped to h_inf.  In stage 0 also the
// soil-water pair sum of every regular particle, from its table.
__global__ void __launch_bounds__(128) k_wir_press(PState A, Search Q, StepScalars* S, Rheo c, DemView dem,
                                                   StageCarry C, int s, const float* hdep, const float* hsz) {
    PDL_ENTRY();
    if (S->skip) return;
    const int nact = S->nactive, nreg = S->nreg;
    const float dt = S->dt_step;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nact; i += gridDim.x * blockDim.x) {
        const bool water = Q.spec[i] == 2;
        if (s == 0 && i < nreg) {
            double b0 = 0.0, b1 = 0.0;
            const int cnt = Q.ncount[i];
            const int4* tab = Q.nbr + tab_base(i, Q.kcap);
            for (int k = 0; k < cnt; k++) {
                const int4 e = tab[(size_t)k * kTabStride];
                if (e.x >= 0) continue;
                wir_pair_term(c, water, Q.xhm[e.x & ~kCrossBit].w, __int_as_float(e.z), __int_as_float(e.w), b0, b1);
            }
            Q.bxy[i] = make_float2((float)b0, (float)b1);
        }
        float2 p;
        if (!wir_stage_pos(A, C, s, dt, i, p) || out_of_box(dem, p.x, p.y)) {  // keeps its term
            Q.pr[i] = make_float4(Q.pterm[i], hdep[i], A.mass[i], 0.f);
            continue;
        }
        float zp = 0.f;
        if (water) {
            int ipx = (int)((p.x - dem.xmin) / dem.dx + 1.f), ipy = (int)((p.y - dem.ymin) / dem.dy + 1.f);
            ipx = min(max(ipx, 1), dem.nx - 1);
            ipy = min(max(ipy, 1), dem.ny - 1);
            const int n1 = (ipy - 1) * dem.nx + (ipx - 1), n2 = n1 + 1, n3 = n1 + 1 + dem.nx, n4 = n3 - 1;
            const float xref = dem.xmin + (float)(ipx - 1) * dem.dx, yref = dem.ymin + (float)(ipy - 1) * dem.dy;
            const float xi = (p.x - xref) / dem.dx, eta = (p.y - yref) / dem.dy;
            const float sh1 = (1.f - xi) * (1.f - eta), sh2 = xi * (1.f - eta), sh3 = xi * eta, sh4 = (1.f - xi) * eta;
            const float d1x = (-1.f + eta) / dem.dx, d2x = (1.f - eta) / dem.dx, d3x = eta / dem.dx, d4x = (-eta) / dem.dx;
            const float d1y = (-1.f + xi) / dem.dy, d2y = (-xi) / dem.dy, d3y = xi / dem.dy, d4y = (1.f - xi) / dem.dy;
            const float h1 = hsz[n1], h2 = hsz[n2], h3 = hsz[n3], h4 = hsz[n4];
            zp = ((sh1 * h1 + sh2 * h2) + sh3 * h3) + sh4 * h4;
            Q.zpw[i] = zp;
            Q.gzw[i] = make_float2(((h1 * d1x + h2 * d2x) + h3 * d3x) + h4 * d4x,
                                   ((h1 * d1y + h2 * d2y) + h3 * d3y) + h4 * d4y);
        }
        const float h = hdep[i];
        const float hc = (h < c.h_inf) ? c.h_inf : h;
        const float p_ = (water && c.swalg == 1) ? c.cgra05 * (hc * hc - zp * zp) : (c.cgra05 * hc) * hc;
        const float pt = (c.pa_sph == 1) ? p_ : p_ / (hc * hc);
        Q.pterm[i] = pt;
        Q.pr[i] = make_float4(pt, h, A.mass[i], 0.f);
    }
}

// The soil-water pair sums of the coarse-level particles, one warp each.
template <int SKF>
__global__ void __launch_bounds__(128) k_wir_pairs_big(PState A, Search Q, StepScalars* S, Rheo c) {
    PDL_ENTRY();
    constexpr int SK = SupportScale<SKF>::value;
    if (S->skip) return;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nreg = S->nreg, nbig = S->nbig;
    for (int b = warp; b < nbig; b += nwarps) {
        const int i = nreg + b;
        const unsigned char si = Q.spec[i];
        double b0 = 0.0, b1 = 0.0;
        warp_neighbours<SK>(Q, S, i, lane, [&](int j, float4 o, const PairGeom& g) {
            if (Q.spec[j] == si) return;
            float w, d0, d1;
            sph_kernel<SKF>(g.r, g.dx0, g.dx1, g.mh, w, d0, d1);
            wir_pair_term(c, si == 2, o.w, d0, d1, b0, b1);
        });
        b0 = warp_sum(b0);
        b1 = warp_sum(b1);
        if (lane == 0) Q.bxy[i] = make_float2((float)b0, (float)b1);
    }
}

// RK45 stage s = 0, 1, 2 of every active particle (SPH_MAIN_2019.f90:808-906):
// x = x0 + c_s dt v, v = v0 + c_s dt (ex + in), the out-of-domain check,
// ExtForces_SW(0) with the stage depth hs_ (clamped as IntForces_SW leaves
// it) and the internal acceleration of this stage, the Dx/Dv sums; then the
// pressure term of stage s+1 at its position with depth hnext.  A particle
// that will leave the domain in stage s+1 keeps its old term, as IntForces_SW
// skips it.
template <bool COS>
__global__ void __launch_bounds__(128) k_stage(PState A, Search Q, StepScalars* S, Rheo c, DemView dem,
                                               StageCarry C, int s, const float* hs_, const float* hnext,
                                               const float* hprev) {
    PDL_ENTRY();
    if (S->skip) return;
    const int nact = S->nactive;
    const float dt = S->dt_step;
    const float f1 = (s == 0) ? 0.f : 0.5f, f2 = (s == 0) ? 1.f : 2.f;
    const float f1n = (s == 2) ? 1.f : 0.5f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nact; i += gridDim.x * blockDim.x) {
        if (s > 0 && C.out[i]) {  // frozen: its pressure term stays, its depth is the next call's
            Q.pr[i] = make_float4(Q.pterm[i], hnext[i], A.mass[i], 0.f);
            continue;
        }
        const float2 x0 = A.pos[i], v0 = A.vel[i];
        float2 vp = v0, ap = make_float2(0.f, 0.f), dx = make_float2(0.f, 0.f), dv = make_float2(0.f, 0.f);
        if (s > 0) { vp = C.v[i]; ap = C.acc[i]; dx = C.dx[i]; dv = C.dv[i]; }
        const float fdt = f1 * dt;
        const float xx = x0.x + fdt * vp.x, xy = x0.y + fdt * vp.y;
        const float vx = v0.x + fdt * ap.x, vy = v0.y + fdt * ap.y;
        const float u1 = (c.icpwp == 1) ? pwp1_stage(c, A, Q, C, s, i, fdt, hprev) : 0.f;
        if (out_of_box(dem, xx, xy)) {
            C.out[i] = 1;
            C.xo[i] = make_float2(xx, xy);
            C.v[i] = make_float2(vx, vy);
            Q.pr[i] = make_float4(Q.pterm[i], hnext[i], A.mass[i], 0.f);
            continue;
        }
        if (s == 0) C.out[i] = 0;
        const float h = hs_[i];
        const float hc = (h < c.h_inf) ? c.h_inf : h;
        const float2 fin = Q.indv[i];
        const float pwp = (c.icpwp == 3) ? A.pwp[i] : u1;
        float ex0, ex1;
        if (c.ws)
            ext_accel_wir(c, dem, dt, xx, xy, vx, vy, hc, fin.x, fin.y, Q.spec[i] == 2, Q.zpw[i], Q.gzw[i], Q.bxy[i],
                          ex0, ex1);
        else
            ext_accel<COS>(c, dem, dt, xx, xy, vx, vy, hc, pwp, soil_fraction(c, Q, A, i), fin.x, fin.y, ex0, ex1);
        if (c.icpwp == 1) pwp1_accumulate(c, C, s, i, hc, u1, dt, f2);
        const float a0 = ex0 + fin.x, a1 = ex1 + fin.y;
        dv.x = dv.x + f2 * a0;
        dv.y = dv.y + f2 * a1;
        dx.x = dx.x + f2 * vx;
        dx.y = dx.y + f2 * vy;
        C.v[i] = make_float2(vx, vy);
        C.acc[i] = make_float2(a0, a1);
        C.dx[i] = dx;
        C.dv[i] = dv;
        if (c.ws) continue;  // the next stage's pressure needs its soil surface: k_wir_press
        const float fdn = f1n * dt;
        const float nx_ = x0.x + fdn * vx, ny_ = x0.y + fdn * vy;
        float pt = Q.pterm[i];
        if (!out_of_box(dem, nx_, ny_)) {
            pt = stage_pterm<COS>(c, dem, hnext[i], nx_, ny_);
            Q.pterm[i] = pt;
        }
        Q.pr[i] = make_float4(pt, hnext[i], A.mass[i], 0.f);
    }
}

// The last stage (s = 3) and the end of the step (rk_finish) with the final
// depth hfin.
template <bool COS>
__global__ void __launch_bounds__(128) k_stage_final(PState A, Search Q, StepScalars* S, Rheo c, DemView dem, int n,
                                                     PState B, float2* velfin, double2* auxv, StageCarry C,
                                                     const float* h4, const float* hfin, const float* h3) {
    PDL_ENTRY();
    if (S->skip) return;
    const int nact = S->nactive;
    const float dt = S->dt_step;
    // block-uniform trip count: every lane of a warp reaches erosion_scatter,
    // every thread the box flush
    NodeBox box = empty_node_box();
    for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        const int i = i0 + threadIdx.x;
        if (i >= n) {
            if (c.erosion) erosion_scatter(dem, 0.f, 0.f, 0.f, false, auxv, box);
            continue;
        }
        if (i >= nact) {
            rk_carry(A, c, B, velfin, Q.xsv, i);
            if (c.erosion) erosion_scatter(dem, 0.f, 0.f, 0.f, false, auxv, box);
            continue;
        }
        const float2 x0 = A.pos[i], v0 = A.vel[i];
        float pwp = (c.icpwp == 3) ? A.pwp[i] : 0.f;
        bool out = C.out[i] != 0;
        float xx, xy, vx, vy;
        float2 dx = make_float2(0.f, 0.f), dv = make_float2(0.f, 0.f);
        float2 acc = make_float2(0.f, 0.f);  // ex + in of the last stage
        if (out) {
            const float2 xo = C.xo[i], vo = C.v[i];
            xx = xo.x; xy = xo.y; vx = vo.x; vy = vo.y;
            if (c.icpwp == 1) pwp = C.u[i];  // u of the stage it left in
        } else {
            const float2 vp = C.v[i], ap = C.acc[i];
            dx = C.dx[i];
            dv = C.dv[i];
            const float fdt = 1.f * dt;
            xx = x0.x + fdt * vp.x; xy = x0.y + fdt * vp.y;
            vx = v0.x + fdt * ap.x; vy = v0.y + fdt * ap.y;
            if (c.icpwp == 1) pwp = pwp1_stage(c, A, Q, C, 3, i, fdt, h3);
            if (out_of_box(dem, xx, xy)) {
                out = true;
            } else {
                const float h = h4[i];
                const float hc = (h < c.h_inf) ? c.h_inf : h;
                const float2 fin = Q.indv[i];
                float ex0, ex1;
                if (c.ws)
                    ext_accel_wir(c, dem, dt, xx, xy, vx, vy, hc, fin.x, fin.y, Q.spec[i] == 2, Q.zpw[i], Q.gzw[i],
                                  Q.bxy[i], ex0, ex1);
                else
                    ext_accel<COS>(c, dem, dt, xx, xy, vx, vy, hc, pwp, soil_fraction(c, Q, A, i), fin.x, fin.y,
                                   ex0, ex1);
                if (c.icpwp == 1) pwp1_accumulate(c, C, 3, i, hc, pwp, dt, 1.f);
                acc = make_float2(ex0 + fin.x, ex1 + fin.y);
                dv.x = dv.x + 1.f * acc.x;
                dv.y = dv.y + 1.f * acc.y;
                dx.x = dx.x + 1.f * vx;
                dx.y = dx.y + 1.f * vy;
            }
        }
        const float u0 = (c.icpwp == 1) ? A.pwp[i] : 0.f;
        const float Du = (c.icpwp == 1 && !out) ? C.Du[i] : 0.f;
        rk_finish(A, Q, S, c, dem, B, velfin, auxv, i, dt, x0, v0, dx.x, dx.y, dv.x, dv.y, xx, xy, vx, vy, out,
                  hfin[i], pwp, u0, Du, acc.x, acc.y, box);
    }
    if (c.erosion) flush_node_box(S, box);
}

// One pair term of av_vel (SPH_MAIN_2019.f90:3072-3080) for particle i with
// the pair's kernel value w.
__device__ __forceinline__ void xsph_terms(float2 vi, float rhoi, float2 vj, float rhoj, float mj, float w, double& a0,
                                           double& a1) {
    float den = rhoi + rhoj;
    float t0 = (((2.f * mj) * (vi.x - vj.x)) / den) * w;
    float t1 = (((2.f * mj) * (vi.y - vj.y)) / den) * w;
    a0 -= (double)t0;
    a1 -= (double)t1;
}

// The same with the pair geometry: the kernel value evaluated here.
template <int SKF>
__device__ __forceinline__ void xsph_pair(float2 vi, float rhoi, float2 vj, float rhoj, float mj, const PairGeom& g,
                                          double& a0, double& a1) {
    xsph_terms(vi, rhoi, vj, rhoj, mj, sph_kernel_w<SKF>(g.r, g.mh), a0, a1);
}

// av_vel (SPH_MAIN_2019.f90:3042-3099) with the start-of-step W_ij, then
// v += 0.3*av for particles still inside the domain (:987-993).
template <int SKF, bool WS>
__global__ void __launch_bounds__(128) k_xsph(PState A, Search Q, StepScalars* S, Rheo c, int n, PState B) {
    PDL_ENTRY();
    if (S->skip || !c.av_vel) return;
    const int nreg = S->nreg;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nreg; i += gridDim.x * blockDim.x) {
        if (B.flag[i]) continue;
        const float4 si = Q.xsv[i];
        const float2 vi = make_float2(si.x, si.y);
        const float rhoi = si.z;
        const int cnt = Q.ncount[i];
        const int4* tab = Q.nbr + tab_base(i, Q.kcap);
        double a0 = 0.0, a1 = 0.0;
        int k = 0;
        for (; k + 4 <= cnt; k += 4) {
            int4 e[4];
            float4 sj[4];
#pragma unroll
            for (int u = 0; u < 4; u++) e[u] = __ldcs(tab + (size_t)(k + u) * kTabStride);
#pragma unroll
            for (int u = 0; u < 4; u++) sj[u] = Q.xsv[WS ? (e[u].x & ~kCrossBit) : e[u].x];
#pragma unroll
            for (int u = 0; u < 4; u++)
                if (!WS || e[u].x >= 0)  // type 0 only (SPH_MAIN_2019.f90:3071)
                    xsph_terms(vi, rhoi, make_float2(sj[u].x, sj[u].y), sj[u].z, sj[u].w, __int_as_float(e[u].y), a0,
                               a1);
        }
        for (; k < cnt; k++) {
            const int4 e = __ldcs(tab + (size_t)k * kTabStride);
            const float4 sj = Q.xsv[WS ? (e.x & ~kCrossBit) : e.x];
            if (!WS || e.x >= 0) xsph_terms(vi, rhoi, make_float2(sj.x, sj.y), sj.z, sj.w, __int_as_float(e.y), a0, a1);
        }
        float av0 = 0.3f * (float)a0, av1 = 0.3f * (float)a1;
        B.vel[i] = make_float2(vi.x + av0, vi.y + av1);
    }
}

template <int SKF>
__global__ void __launch_bounds__(128) k_xsph_big(PState A, Search Q, StepScalars* S, Rheo c, PState B) {
    PDL_ENTRY();
    constexpr int SK = SupportScale<SKF>::value;
    if (S->skip || !c.av_vel) return;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nreg = S->nreg, nbig = S->nbig;
    for (int b = warp; b < nbig; b += nwarps) {
        int i = nreg + b;
        if (B.flag[i]) continue;  // uniform over the warp
        const float4 si = Q.xsv[i];
        const float2 vi = make_float2(si.x, si.y);
        const float rhoi = si.z;
        double a0 = 0.0, a1 = 0.0;
        const unsigned char si_ = c.ws ? Q.spec[i] : 0;
        warp_neighbours<SK>(Q, S, i, lane, [&](int j, float4 o, const PairGeom& g) {
            if (c.ws && Q.spec[j] != si_) return;  // type 0 only (SPH_MAIN_2019.f90:3071)
            const float4 sj = Q.xsv[j];
            xsph_pair<SKF>(vi, rhoi, make_float2(sj.x, sj.y), sj.z, sj.w, g, a0, a1);
        });
        a0 = warp_sum(a0);
        a1 = warp_sum(a1);
        if (lane == 0) {
            float av0 = 0.3f * (float)a0, av1 = 0.3f * (float)a1;
            B.vel[i] = make_float2(vi.x + av0, vi.y + av1);
        }
    }
}

// DEM update of ExtForces_SW(1) (SPH_SW_2019.f90:8795-8807) over the node box
// touched this step; resets the scatter accumulators.

// DEM update over the touched node box, grid-stride.
__device__ __forceinline__ void erode_box(double2* auxv, float* z, float* eroded, float* avail, int nx, int x0, int x1,
                                          int y0, int y1) {
    int w = x1 - x0 + 1, hgt = y1 - y0 + 1;
    long long tot = (long long)w * hgt;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < tot; k += (long long)gridDim.x * blockDim.x) {
        int ix = x0 + (int)(k % w), iy = y0 + (int)(k / w);
        int ip = (iy - 1) * nx + (ix - 1);
        double2 a = auxv[ip];
        if ((float)a.y > 1.e-6f) {
            float xnum = (float)(a.x / a.y);
            float av = avail[ip];
            if (xnum > av) xnum = av;
            if (av > 0.f) {
                eroded[ip] = eroded[ip] + xnum;
                z[ip] = z[ip] - xnum;
                avail[ip] = av - xnum;
            }
        }
        auxv[ip] = make_double2(0.0, 0.0);
    }
}

// End of a step: time, dt and the counters; then the next step's decision
// (prepare_step).  One thread.
__device__ __forceinline__ void step_end(StepScalars* S) {
    if (!S->skip && S->advance) {
        S->dt = S->dt_step;
        S->time += (double)S->dt;
        S->steps_done += 1;
    }
    prepare_step(S, 1);
}

__global__ void k_step_end(StepScalars* S) {
    PDL_ENTRY();
    StepScalars* L = scalars_to_smem(S);
    if (threadIdx.x == 0) step_end(L);
    scalars_from_smem(S, L);
}

// DEM update of ExtForces_SW(1) (:8795-8807) over the node box touched this
// step, resetting the scatter accumulators; the last block to finish also
// ends the step (k_step_end), which saves a launch.
__global__ void k_dem_erode(double2* auxv, float* z, float* eroded, float* avail, int nx, StepScalars* S) {
    PDL_ENTRY();
    __shared__ bool last;
    const int x0 = S->ex0, x1 = S->ex1, y0 = S->ey0, y1 = S->ey1;
    if (!S->skip && x1 >= x0 && y1 >= y0) erode_box(auxv, z, eroded, avail, nx, x0, x1, y0, y1);
    // the last block to finish ends the step (k_step_end)
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = (atomicAdd(&S->end_ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    StepScalars* L = scalars_to_smem(S);
    if (threadIdx.x == 0) {
        L->end_ticket = 0u;
        step_end(L);
    }
    scalars_from_smem(S, L);
}

// Neighbour pairs of the coarse-level particles, for the parity export: every
// (big i, j) pair with r < hi + hj, written as slot pairs.
template <int SKF>
__global__ void k_export_big(Search Q, StepScalars* S, int2* pairs, int* npairs, int cap) {
    constexpr int SK = SupportScale<SKF>::value;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nreg = S->nreg, nbig = S->nbig;
    for (int b = warp; b < nbig; b += nwarps) {
        int i = nreg + b;
        warp_neighbours<SK>(Q, S, i, lane, [&](int j, float4 o, const PairGeom& g) {
            int k = atomicAdd(npairs, 1);
            if (k < cap) pairs[k] = make_int2(i, j);
        });
    }
}

// ---------------------------------------------------------------- outputs

// Depth raster: IDW of h onto the 4x4 DEM nodes around each particle
// (SPH_SW_2019.f90:14310-14400, auxv(1)/auxv(5)).
__global__ void k_raster_idw(const PState B, int n, DemView dem, double2* acc) {
    float distg = sqrtf(dem.dx * dem.dx + dem.dy * dem.dy);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (B.flag[i]) continue;
        float2 p = B.pos[i];
        float h = B.rho[i];
        int ipx = (int)((p.x - dem.xmin) / dem.dx + 1.f);
        int ipy = (int)((p.y - dem.ymin) / dem.dy + 1.f);
        int ix0 = max(1, ipx - 1), iy0 = max(1, ipy - 1), ix1 = min(dem.nx, ipx + 2), iy1 = min(dem.ny, ipy + 2);
        for (int ix = ix0; ix <= ix1; ix++)
            for (int iy = iy0; iy <= iy1; iy++) {
                int ip = (iy - 1) * dem.nx + (ix - 1);
                float ddx = p.x - (dem.xmin + (float)(ix - 1) * dem.dx);
                ddx = ddx * ddx;
                float ddy = p.y - (dem.ymin + (float)(iy - 1) * dem.dy);
                ddy = ddy * ddy;
                float dist = sqrtf(ddx + ddy);
                dist = (1.e-6f > dist) ? 1.e-6f : dist;
                dist = dist / distg;
                atomicAdd(&acc[ip].x, (double)(h / dist));
                atomicAdd(&acc[ip].y, (double)(1.f / dist));
            }
    }
}

__global__ void k_raster_idw_finish(const double2* acc, float* out, int np) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
        double2 a = acc[k];
        out[k] = ((float)a.y >= 1.e-6f) ? (float)(a.x / a.y) : (float)a.x;
    }
}

// Misfit of the depth raster against a target raster, L = sum_nodes (R - T)^2
// with R the IDW raster above, for back-analysis: per node lam = dL/dR =
// 2 (R - T) and the node's share of L, summed per block (the host adds the
// block sums in block order).
__global__ void k_misfit_nodes(const double2* acc, const float* target, int np, double* lam, double* part) {
    __shared__ double sh[32];
    double l = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
        const double2 a = acc[k];
        const double R = ((float)a.y >= 1.e-6f) ? a.x / a.y : a.x;
        const double d = R - (double)target[k];
        lam[k] = 2.0 * d;
        l += d * d;
    }
    l = warp_sum(l);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w];
        part[blockIdx.x] = t;
    }
}

// dL/dh and dL/dx of every particle inside the domain, through the IDW
// weights w = 1/dhat, dhat = max(dist, 1e-6)/distg, of its 4x4 nodes: with
// S = sum w and R = sum h w / S, dR/dh_i = w_i / S and dR/dw_i = (h_i - R)/S
// (where S < 1e-6 the raster is sum h w itself: w_i and h_i);
// dw/dp = -(distg / dist^2) (p - node)/dist.  Written in caller order.
__global__ void k_misfit_particles(const PState B, int n, DemView dem, const double2* acc, const double* lam,
                                   float2* gx, float* gh) {
    const float distg = sqrtf(dem.dx * dem.dx + dem.dy * dem.dy);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int o = B.id[i];
        if (B.flag[i]) {
            gx[o] = make_float2(0.f, 0.f);
            gh[o] = 0.f;
            continue;
        }
        const float2 p = B.pos[i];
        const double h = B.rho[i];
        const int ipx = (int)((p.x - dem.xmin) / dem.dx + 1.f);
        const int ipy = (int)((p.y - dem.ymin) / dem.dy + 1.f);
        const int ix0 = max(1, ipx - 1), iy0 = max(1, ipy - 1), ix1 = min(dem.nx, ipx + 2), iy1 = min(dem.ny, ipy + 2);
        double dh = 0.0, d0 = 0.0, d1 = 0.0;
        for (int ix = ix0; ix <= ix1; ix++)
            for (int iy = iy0; iy <= iy1; iy++) {
                const int ip = (iy - 1) * dem.nx + (ix - 1);
                const double ex = (double)p.x - (double)(dem.xmin + (float)(ix - 1) * dem.dx);
                const double ey = (double)p.y - (double)(dem.ymin + (float)(iy - 1) * dem.dy);
                const double dist = sqrt(ex * ex + ey * ey);
                const double dhat = fmax(dist, 1.e-6) / (double)distg;
                const double w = 1.0 / dhat;
                const double2 a = acc[ip];
                const double L = lam[ip];
                double dRdh, dRdw;
                if ((float)a.y >= 1.e-6f) {
                    dRdh = w / a.y;
                    dRdw = (h - a.x / a.y) / a.y;
                } else {
                    dRdh = w;
                    dRdw = h;
                }
                dh += L * dRdh;
                if (dist > 1.e-6) {
                    const double c = -L * dRdw * (double)distg / (dist * dist * dist);
                    d0 += c * ex;
                    d1 += c * ey;
                }
            }
        gx[o] = make_float2((float)d0, (float)d1);
        gh[o] = (float)dh;
    }
}

// Per-node hazard statistics of Get_MC_pixel_Vars_SW (SPH_SW_2019.f90:20739-20812):
// each particle adds h and |v| to the 4 nodes of its DEM cell.
__global__ void k_hazard(const PState B, int n, DemView dem, double* sum_h, double* sum_v, unsigned int* max_h,
                         unsigned int* max_v, int* cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (B.flag[i]) continue;
        float2 p = B.pos[i];
        int ipx = (int)((p.x - dem.xmin) / dem.dx + 1.f);
        int ipy = (int)((p.y - dem.ymin) / dem.dy + 1.f);
        ipx = min(max(ipx, 1), dem.nx - 1);
        ipy = min(max(ipy, 1), dem.ny - 1);
        int ip = (ipy - 1) * dem.nx + (ipx - 1);
        int nodes[4] = {ip, ip + 1, ip + 1 + dem.nx, ip + dem.nx};
        float hh = B.rho[i];
        float2 v = B.vel[i];
        float vv = sqrtf(v.x * v.x + v.y * v.y);
        for (int k = 0; k < 4; k++) {
            int q = nodes[k];
            atomicAdd(&cnt[q], 1);
            atomicAdd(&sum_h[q], (double)hh);
            atomicAdd(&sum_v[q], (double)vv);
            atomicMax(&max_h[q], f2o(hh));
            atomicMax(&max_v[q], f2o(vv));
        }
    }
}

}  // namespace gfsph
