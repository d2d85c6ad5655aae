// Jacobi-preconditioned conjugate gradients on an element-by-element system,
// the solver of solvegc2 (SPH_GCsolver_2019.f90:16-316), on the device.
//
// The element matrices gstif(nevab, nevab, nelem) are assembled once into a
// CSR matrix (FP64).  A solve is one set-up kernel (the preconditioner and the
// -999 marks of getqmat, x = fixed, r = b - K x, the initial dot products) and
// one persistent cooperative kernel that runs every iteration: per iteration
// two phases over the dofs separated by grid barriers,
//   A: p = s + beta p_old for the block's own rows (written to the other half
//      of a double buffer) and ap = K p with the reference's mask, each term
//      forming p_j = s_j + beta p_old_j from the same two values, so the
//      product equals that of the materialised direction bit for bit; the
//      partial sums of p.ap;
//   B: alpha = prod1 / prod2, x += alpha p, r1 = r - alpha ap, s = q r1, the
//      partial sums of r1.r1 and r1.s; then beta and the convergence test
//      r.r / r0.r0 <= tol on squared norms (:112).
// Every block reduces the block partials itself in the same fixed order, so
// alpha, beta and the stop decision are identical in every block and every
// solve is bit-reproducible.  The barriers are a counter and a generation
// word; a wait gives up after a bounded number of polls and sets an error
// word that every block then sees, so a solve can end with an error but never
// hang.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "../../include/gfsph.h"

namespace {

constexpr int kCgThreads = 256;
constexpr int kIterPerGraph = 8;

struct CgScalars {
    double rnorm0;   // r0.r0 (all dofs)
    double prod1;    // r.s over free dofs of the current iterate
    double fnorm;    // fixed.fixed (rnormX of :93-103 with rnorm0)
    double tol;
    double red[2];   // results of the last barrier reduction
    int done;        // converged, or nothing to do
    int trivial;     // rnormX below tol: the solution is 0 and nothing runs
    int iters;
    int max_iters;
    int rbuf;        // half of the residual buffer that holds the returned r
    int err;         // a grid barrier gave up
    unsigned int ticket;
    unsigned int bar_count, bar_gen;
};

struct CgDev {
    int n;
    const int* rowptr;
    const int* col;
    const double* val;
    const double* diag;     // assembled diagonal
    double* q;              // 1/diag (0 where the diagonal vanishes)
    int* fix;               // iffix (device copy, -999 marks singular free dofs)
    double *x, *ap;
    double *r[2], *p[2];    // double buffers: iteration k reads [k & 1], writes [(k + 1) & 1]
    double* s;
    double* part;           // block partial sums, 3 x nblocks
    CgScalars* S;
};

__device__ __forceinline__ double block_reduce(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += sh[k];
    __syncthreads();
    return t;  // valid in thread 0
}

// Sum of nb block partials in a fixed order (a fixed assignment of partials
// to threads, then a fixed-order tree); valid in thread 0.
__device__ __forceinline__ double sum_partials(const double* part, int nb, double* sh) {
    double v = 0.0;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) v += __ldcg(part + k);
    return block_reduce(v, sh);
}

// Polls of a barrier wait before it gives up (about a second with the
// back-off below; a barrier of co-resident blocks takes microseconds).
constexpr long long kBarrierPolls = 1LL << 23;

// Grid barrier over the co-resident blocks of a cooperative launch, with a
// reduction: every block has written its partials part[r*nb + block] for
// r < nr; the last block to arrive sums each set in a fixed order into
// S->red[r], resets the counter and advances the generation; the others wait
// for the generation to change.  A wait that polls kBarrierPolls times, or
// sees the error word set, sets the error word and returns false, and every
// block then leaves the solve.  On success out[r] holds the sums in every
// thread.
__device__ bool barrier_reduce(CgScalars* S, const double* part, int nb, int nr, double* out, double* sh) {
    __shared__ int role;      // 1: this block arrived last
    __shared__ int ok;
    __shared__ unsigned int g;
    __syncthreads();          // this block's partials are written
    if (threadIdx.x == 0) {
        g = *(volatile unsigned int*)&S->bar_gen;  // before arriving
        __threadfence();
        role = (atomicAdd(&S->bar_count, 1u) == gridDim.x - 1) ? 1 : 0;
        ok = 1;
    }
    __syncthreads();
    if (role) {
        __threadfence();
        for (int r = 0; r < nr; r++) {
            const double t = sum_partials(part + (size_t)r * nb, nb, sh);
            if (threadIdx.x == 0) S->red[r] = t;
        }
        if (threadIdx.x == 0) {
            S->bar_count = 0u;
            __threadfence();
            atomicAdd(&S->bar_gen, 1u);
        }
    } else if (threadIdx.x == 0) {
        volatile unsigned int* gen = &S->bar_gen;
        volatile int* err = &S->err;
        for (long long k = 0; *gen == g; k++) {
            if (*err || k >= kBarrierPolls) {
                atomicExch(&S->err, 1);
                ok = 0;
                break;
            }
            __nanosleep(k < 64 ? 32 : 128);
        }
        __threadfence();
    }
    __syncthreads();
    if (!ok) return false;
    for (int r = 0; r < nr; r++) out[r] = __ldcg(&S->red[r]);
    return true;
}

// Set-up of a solve (getqmat :124-159 and initcg :165-205): q = 1/diag, a
// free dof with a vanishing diagonal marked -999 (q = 0); x = fixed,
// r = b - K x (unmasked), s = q r, p = s, r0.r0 over all dofs, then
// r = s = p = 0 on prescribed dofs and prod1 = r.s; fixed.fixed for rnormX.
// Two kernels: x must be complete before the product.
__global__ void k_cg_init_x(CgDev d, const float* fixed, const float* rhs_f, double* rhs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.n) {
        d.x[i] = (double)fixed[i];
        rhs[i] = (double)rhs_f[i];
        const double dg = d.diag[i];
        if (fabs(dg) <= 1.e-35) {
            if (d.fix[i] == 0) d.fix[i] = -999;
            d.q[i] = 0.0;
        } else {
            d.q[i] = 1.0 / dg;
        }
    }
}

__global__ void k_cg_init_rest(CgDev d, const double* rhs) {
    __shared__ double sh[32];
    __shared__ bool last;
    CgScalars* S = d.S;
    double rr = 0.0, rs = 0.0, ff = 0.0;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.n) {
        double sum = 0.0;
        for (int k = d.rowptr[i]; k < d.rowptr[i + 1]; k++) sum += d.val[k] * d.x[d.col[k]];
        double r = rhs[i] - sum;
        double s = d.q[i] * r;
        rr = r * r;
        ff = d.x[i] * d.x[i];
        if (d.fix[i] != 0) { r = 0.0; s = 0.0; }
        rs = r * s;
        d.r[0][i] = r;
        d.s[i] = s;
        d.p[0][i] = 0.0;  // with beta = 0 the first direction is p = s
    }
    const int nb = gridDim.x;
    double t0 = block_reduce(rr, sh);
    double t1 = block_reduce(rs, sh);
    double t2 = block_reduce(ff, sh);
    if (threadIdx.x == 0) {
        d.part[blockIdx.x] = t0;
        d.part[nb + blockIdx.x] = t1;
        d.part[2 * nb + blockIdx.x] = t2;
        __threadfence();
        last = (atomicAdd(&S->ticket, 1u) == (unsigned)nb - 1u);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    const double rn0 = sum_partials(d.part, nb, sh);
    const double p1 = sum_partials(d.part + nb, nb, sh);
    const double fn = sum_partials(d.part + 2 * nb, nb, sh);
    if (threadIdx.x == 0) {
        S->rnorm0 = rn0;
        S->prod1 = p1;
        S->fnorm = fn;
        S->ticket = 0u;
        // rnormX (:93-103): sqrt(fixed.fixed + r0.r0) below tol: the solution is 0
        if (sqrt(fn + rn0) < S->tol) { S->done = 1; S->trivial = 1; }
    }
}

// Every iteration of jcg (:208-268) in one cooperative launch.
__global__ void __launch_bounds__(kCgThreads) k_cg_iterate(CgDev d) {
    __shared__ double sh[32];
    CgScalars* S = d.S;
    if (S->done) return;  // uniform: set before the launch
    const int nb = gridDim.x;
    const int stride = gridDim.x * blockDim.x;
    double prod1 = S->prod1;
    const double rnorm0 = S->rnorm0, tol = S->tol;
    const int max_iters = S->max_iters;
    double beta = 0.0;  // first direction: p = s
    double red[2];
    for (int it = 0;; it++) {
        const int cur = it & 1;
        // selected, not indexed: a dynamic index would copy d to local memory
        const double* __restrict__ pold = cur ? d.p[1] : d.p[0];
        double* __restrict__ pnew = cur ? d.p[0] : d.p[1];
        // A: p = s + beta p_old and ap = K p, masked (kbyp :273-313)
        double acc = 0.0;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.n; i += stride) {
            const int fi = d.fix[i];
            double sum = 0.0;
            for (int k = d.rowptr[i]; k < d.rowptr[i + 1]; k++) {
                const int j = d.col[k];
                if (fi + d.fix[j] != 0) continue;
                sum += d.val[k] * (d.s[j] + beta * pold[j]);
            }
            const double pi = d.s[i] + beta * pold[i];
            pnew[i] = pi;
            d.ap[i] = sum;
            if (fi == 0) acc += pi * sum;
        }
        double t = block_reduce(acc, sh);
        if (threadIdx.x == 0) d.part[blockIdx.x] = t;
        if (!barrier_reduce(S, d.part, nb, 1, red, sh)) return;
        const double alpha = prod1 / red[0];
        // B: x += alpha p, r1 = r - alpha ap, s = q r1 (:233-241)
        const double* __restrict__ r = cur ? d.r[1] : d.r[0];
        double* __restrict__ r1 = cur ? d.r[0] : d.r[1];
        double rr = 0.0, rs = 0.0;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.n; i += stride) {
            const double pi = pnew[i];
            d.x[i] = d.x[i] + alpha * pi;
            const double v = r[i] - alpha * d.ap[i];
            r1[i] = v;
            const double si = d.q[i] * v;
            d.s[i] = si;
            rr += v * v;
            rs += v * si;
        }
        double t0 = block_reduce(rr, sh);
        double t1 = block_reduce(rs, sh);
        if (threadIdx.x == 0) {
            d.part[nb + blockIdx.x] = t0;
            d.part[2 * nb + blockIdx.x] = t1;
        }
        if (!barrier_reduce(S, d.part + nb, nb, 2, red, sh)) return;
        const double rnorm1 = red[0], prod3 = red[1];
        const int iters = it + 1;
        if (rnorm1 / rnorm0 <= tol || iters >= max_iters) {
            // converged: as jcg, the returned residual is the one before this
            // update (the copy r = r1 happens only when the loop goes on)
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                S->iters = iters;
                S->done = 1;
                S->rbuf = cur;
            }
            return;
        }
        beta = prod3 / prod1;
        prod1 = prod3;
    }
}

// Results in the caller's precision: x (0 when nothing was solved), the
// returned residual, and the -999 marks reset to 0 after a solve.
__global__ void k_cg_finish(CgDev d, float* x_f, float* r_f) {
    const CgScalars* S = d.S;
    const bool trivial = S->trivial != 0;
    const double* r = S->rbuf ? d.r[1] : d.r[0];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.n) {
        x_f[i] = trivial ? 0.f : (float)d.x[i];
        r_f[i] = (float)r[i];
        if (!trivial && d.fix[i] == -999) d.fix[i] = 0;
    }
}

}  // namespace

struct gfsph_cg {
    int npoin = 0, nelem = 0, nnode = 0, ndofn = 0, n = 0;
    cudaStream_t stream = nullptr;
    int *rowptr = nullptr, *col = nullptr, *fix = nullptr;
    double *val = nullptr, *diag = nullptr, *q = nullptr;
    double *x = nullptr, *r = nullptr, *s = nullptr, *p = nullptr, *ap = nullptr, *part = nullptr;
    double* rhs = nullptr;
    float *in_fixed = nullptr, *in_rhs = nullptr, *out_x = nullptr, *out_r = nullptr;  // caller precision
    CgScalars* S = nullptr;
    CgScalars* hS = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int nblocks = 0;      // one thread per dof (set-up and finish kernels)
    int coop_blocks = 0;  // blocks of the persistent kernel (all co-resident)
    double last_ms = 0.0; // device time of the last solve
    long long launches = 0;
};

namespace {

CgDev view(gfsph_cg* c) {
    CgDev d;
    d.n = c->n; d.rowptr = c->rowptr; d.col = c->col; d.val = c->val; d.diag = c->diag; d.q = c->q;
    d.fix = c->fix; d.x = c->x; d.ap = c->ap; d.s = c->s; d.part = c->part; d.S = c->S;
    d.r[0] = c->r; d.r[1] = c->r + c->n;
    d.p[0] = c->p; d.p[1] = c->p + c->n;
    return d;
}

template <class T>
int dal(T** p, size_t n) {
    return cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T)) == cudaSuccess ? 0 : 1;
}

void cg_free(gfsph_cg* c) {
    void* ptrs[] = {c->rowptr, c->col, c->fix, c->val, c->diag, c->q, c->x, c->r, c->s, c->p, c->ap, c->part,
                    c->rhs, c->in_fixed, c->in_rhs, c->out_x, c->out_r, c->S};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (c->hS) cudaFreeHost(c->hS);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
}

}  // namespace

extern "C" {

int gfsph_cg_create(int npoin, int nelem, int nnode, int ndofn, const int* intmat, const float* gstif,
                    gfsph_cg** out) try {
    if (!out || !intmat || !gstif || npoin < 1 || nelem < 1 || nnode < 1 || ndofn < 1) return GFSPH_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return GFSPH_ERR_NO_DEVICE;
    const int nevab = nnode * ndofn;
    const long long ntot = (long long)npoin * ndofn;
    if (ntot > 0x3fffffffLL) return GFSPH_ERR_ARG;
    const int n = (int)ntot;
    // assemble sum_e gstif_e into CSR (FP64): (row, col, value) triplets sorted by row, col
    std::vector<long long> key;
    std::vector<double> vv;
    key.reserve((size_t)nelem * nevab * nevab);
    vv.reserve((size_t)nelem * nevab * nevab);
    for (int e = 0; e < nelem; e++)
        for (int a = 0; a < nnode; a++)
            for (int ia = 0; ia < ndofn; ia++) {
                int na = intmat[(size_t)e * nnode + a];
                if (na < 1 || na > npoin) return GFSPH_ERR_ARG;
                long long row = (long long)(na - 1) * ndofn + ia;
                int ea = a * ndofn + ia;
                for (int b = 0; b < nnode; b++)
                    for (int ib = 0; ib < ndofn; ib++) {
                        int nb_ = intmat[(size_t)e * nnode + b];
                        if (nb_ < 1 || nb_ > npoin) return GFSPH_ERR_ARG;
                        long long colx = (long long)(nb_ - 1) * ndofn + ib;
                        int eb = b * ndofn + ib;
                        key.push_back(row * ntot + colx);
                        vv.push_back((double)gstif[(size_t)e * nevab * nevab + (size_t)eb * nevab + ea]);
                    }
            }
    std::vector<size_t> order(key.size());
    for (size_t k = 0; k < order.size(); k++) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return key[a] < key[b]; });
    std::vector<int> rowptr(n + 1, 0), col;
    std::vector<double> val;
    col.reserve(order.size());
    val.reserve(order.size());
    long long last = -1;
    for (size_t k : order) {
        if (key[k] != last) {
            col.push_back((int)(key[k] % ntot));
            val.push_back(vv[k]);
            rowptr[(size_t)(key[k] / ntot) + 1]++;
            last = key[k];
        } else {
            val.back() += vv[k];
        }
    }
    for (int i = 0; i < n; i++) rowptr[i + 1] += rowptr[i];
    gfsph_cg* c = new (std::nothrow) gfsph_cg();
    if (!c) return GFSPH_ERR_HOST;
    c->npoin = npoin; c->nelem = nelem; c->nnode = nnode; c->ndofn = ndofn; c->n = n;
    std::vector<double> diag(n, 0.0);
    for (int i = 0; i < n; i++)
        for (int k = rowptr[i]; k < rowptr[i + 1]; k++)
            if (col[k] == i) diag[i] = val[k];
    c->nblocks = (n + kCgThreads - 1) / kCgThreads;
    int st = 0;
    st |= dal(&c->rowptr, n + 1); st |= dal(&c->col, col.size()); st |= dal(&c->val, val.size());
    st |= dal(&c->diag, n); st |= dal(&c->fix, n); st |= dal(&c->q, n);
    st |= dal(&c->x, n); st |= dal(&c->r, 2 * (size_t)n); st |= dal(&c->s, n); st |= dal(&c->p, 2 * (size_t)n);
    st |= dal(&c->ap, n); st |= dal(&c->part, 3 * (size_t)c->nblocks); st |= dal(&c->rhs, n);
    st |= dal(&c->in_fixed, n); st |= dal(&c->in_rhs, n); st |= dal(&c->out_x, n); st |= dal(&c->out_r, n);
    st |= dal(&c->S, 1);
    if (st || cudaMallocHost((void**)&c->hS, sizeof(CgScalars)) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
        cg_free(c);
        delete c;
        return GFSPH_ERR_CUDA;
    }
    // blocks of the persistent kernel: as many as can be resident at once
    // (a cooperative launch refuses more), at most one per 256 dofs
    int dev = 0, nsm = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cg_iterate, kCgThreads, 0);
    c->coop_blocks = std::max(1, std::min(c->nblocks, nsm * std::max(per_sm, 1)));
    cudaMemcpy(c->rowptr, rowptr.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(c->col, col.data(), col.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(c->val, val.data(), val.size() * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(c->diag, diag.data(), n * sizeof(double), cudaMemcpyHostToDevice);
    if (cudaGetLastError() != cudaSuccess) { cg_free(c); delete c; return GFSPH_ERR_CUDA; }
    *out = c;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_cg_destroy(gfsph_cg* c) try {
    if (!c) return GFSPH_ERR_ARG;
    cudaStreamSynchronize(c->stream);
    cg_free(c);
    delete c;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_cg_solve(gfsph_cg* c, int* iffix, const float* fixed, float* rcg, float* ficg, float tol, int* iterations) try {
    if (!c || !iffix || !fixed || !rcg || !ficg) return GFSPH_ERR_ARG;
    const int n = c->n;
    cudaStream_t st = c->stream;
    CgScalars init{};
    init.tol = (double)tol;
    init.max_iters = (int)std::min<long long>(10LL * n, 0x7fffffffLL);  // miter = 10*ntotv
    *c->hS = init;
    if (cudaMemcpyAsync(c->fix, iffix, n * sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(c->in_fixed, fixed, n * sizeof(float), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(c->in_rhs, rcg, n * sizeof(float), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(c->S, c->hS, sizeof(CgScalars), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return GFSPH_ERR_CUDA;
    CgDev d = view(c);
    const int nb = c->nblocks;
    cudaEventRecord(c->ev0, st);
    k_cg_init_x<<<nb, kCgThreads, 0, st>>>(d, c->in_fixed, c->in_rhs, c->rhs);
    k_cg_init_rest<<<nb, kCgThreads, 0, st>>>(d, c->rhs);
    void* args[] = {&d};
    if (cudaLaunchCooperativeKernel((const void*)k_cg_iterate, dim3(c->coop_blocks), dim3(kCgThreads), args, 0, st) !=
        cudaSuccess)
        return GFSPH_ERR_CUDA;
    k_cg_finish<<<nb, kCgThreads, 0, st>>>(d, c->out_x, c->out_r);
    cudaEventRecord(c->ev1, st);
    c->launches += 4;
    if (cudaMemcpyAsync(c->hS, c->S, sizeof(CgScalars), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(ficg, c->out_x, n * sizeof(float), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(rcg, c->out_r, n * sizeof(float), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(iffix, c->fix, n * sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return GFSPH_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return GFSPH_ERR_CUDA;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->last_ms = ms;
    if (c->hS->err) return GFSPH_ERR_CUDA;  // a grid barrier gave up: the result is incomplete
    if (iterations) *iterations = c->hS->iters;
    return cudaGetLastError() == cudaSuccess ? GFSPH_OK : GFSPH_ERR_CUDA;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_cg_device_ms(gfsph_cg* c, double* ms) try {
    if (!c || !ms) return GFSPH_ERR_ARG;
    *ms = c->last_ms;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_solvegc2(int npoin, int nelem, int nnode, int ndofn, const int* intmat, int* iffix, const float* fixed,
                   const float* gstif, float* rcg, float* ficg, float tol, int* iterations) try {
    gfsph_cg* c = nullptr;
    int st = gfsph_cg_create(npoin, nelem, nnode, ndofn, intmat, gstif, &c);
    if (st) return st;
    st = gfsph_cg_solve(c, iffix, fixed, rcg, ficg, tol, iterations);
    gfsph_cg_destroy(c);
    return st;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

long long gfsph_cg_launch_count(gfsph_cg* c) { return c ? c->launches : -1; }

}  // extern "C"
