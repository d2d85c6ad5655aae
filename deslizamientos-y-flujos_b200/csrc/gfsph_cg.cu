// Jacobi-preconditioned conjugate gradients on an element-by-element system,
// the solver of solvegc2 (SPH_GCsolver_2019.f90:16-316), on the device.
//
// The element matrices gstif(nevab, nevab, nelem) are assembled once into a
// CSR matrix (FP64).  Each iteration is three kernels over the dofs: masked
// SpMV fused with the p.Ap dot product; the updates of x, r and s fused with
// the r.r and r.s dot products; the new search direction.  Dot products are
// FP64; each kernel reduces its block partial sums in the last block to
// finish (a ticket counter, no spin-waits), in a fixed order, so every solve
// is bit-reproducible.  Iterations run in CUDA graphs of kIterPerGraph and
// stop on a device-side flag once r.r / r0.r0 <= tol, the reference's test on
// squared norms (:112).
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
    double alpha, beta;
    double tol;
    int done;        // converged (or nothing to do)
    int iters;
    int max_iters;
    unsigned int ticket[3];
};

struct CgDev {
    int n;
    const int* rowptr;
    const int* col;
    const double* val;
    const double* q;        // 1/diag (0 where the dof is fixed or singular)
    const int* fix;         // iffix (device copy, -999 marks singular free dofs)
    double *x, *r, *r1, *s, *p, *ap;
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

// Last block to finish sums the partials in block order; returns true there.
__device__ __forceinline__ bool last_block(unsigned int* ticket) {
    __shared__ bool am_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) am_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    return am_last;
}

__device__ __forceinline__ double sum_partials(const double* part, int nb, double* sh) {
    double v = 0.0;
    // fixed assignment of partials to threads, then a fixed-order tree
    for (int k = threadIdx.x; k < nb; k += blockDim.x) v += part[k];
    return block_reduce(v, sh);
}

// ap = K p with the reference's mask (a term is dropped when either dof is
// prescribed, kbyp(1)), and the partial sums of p.ap over free dofs; the last
// block forms alpha = prod1 / prod2 (jcg :216-231).
__global__ void k_cg_spmv(CgDev d) {
    __shared__ double sh[32];
    CgScalars* S = d.S;
    if (S->done) return;
    double acc = 0.0;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.n) {
        double sum = 0.0;
        int fi = d.fix[i];
        for (int k = d.rowptr[i]; k < d.rowptr[i + 1]; k++) {
            int j = d.col[k];
            if (fi + d.fix[j] != 0) continue;
            sum += d.val[k] * d.p[j];
        }
        d.ap[i] = sum;
        if (fi == 0) acc = d.p[i] * sum;
    }
    double t = block_reduce(acc, sh);
    if (threadIdx.x == 0) d.part[blockIdx.x] = t;
    if (last_block(&S->ticket[0])) {
        double prod2 = sum_partials(d.part, gridDim.x, sh);
        if (threadIdx.x == 0) {
            S->alpha = S->prod1 / prod2;
            S->ticket[0] = 0;
        }
    }
}

// x += alpha p, r1 = r - alpha ap, s = q r1, and the partial sums of r1.r1
// and r1.s (jcg :233-241); the last block tests convergence and forms beta.
__global__ void k_cg_update(CgDev d) {
    __shared__ double sh[32];
    CgScalars* S = d.S;
    if (S->done) return;
    const double alpha = S->alpha;
    double rr = 0.0, rs = 0.0;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.n) {
        d.x[i] = d.x[i] + alpha * d.p[i];
        double r1 = d.r[i] - alpha * d.ap[i];
        d.r1[i] = r1;
        double s = d.q[i] * r1;
        d.s[i] = s;
        rr = r1 * r1;
        rs = r1 * s;
    }
    int nb = gridDim.x;
    double t0 = block_reduce(rr, sh);
    double t1 = block_reduce(rs, sh);
    if (threadIdx.x == 0) {
        d.part[nb + blockIdx.x] = t0;
        d.part[2 * nb + blockIdx.x] = t1;
    }
    if (last_block(&S->ticket[1])) {
        double rnorm1 = sum_partials(d.part + nb, nb, sh);
        double prod3 = sum_partials(d.part + 2 * nb, nb, sh);
        if (threadIdx.x == 0) {
            S->iters += 1;
            if (rnorm1 / S->rnorm0 <= S->tol || S->iters >= S->max_iters) {
                S->done = 1;
                S->beta = 0.0;
            } else {
                S->beta = prod3 / S->prod1;
                S->prod1 = prod3;
            }
            S->ticket[1] = 0;
        }
    }
}

// p = s + beta p, r = r1 (jcg :243-249) unless converged.
__global__ void k_cg_direction(CgDev d) {
    CgScalars* S = d.S;
    if (S->done) return;
    const double beta = S->beta;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.n) {
        d.p[i] = d.s[i] + beta * d.p[i];
        d.r[i] = d.r1[i];
    }
}

// initcg (:165-205): x = fixed, r = b - K x (unmasked), s = q r, p = s,
// rnorm0 = r.r over all dofs, then r = s = p = 0 on prescribed dofs; also
// prod1 = r.s over free dofs for the first iteration.
__global__ void k_cg_init_spmv(CgDev d, const double* fixed) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.n) d.x[i] = fixed[i];
}

__global__ void k_cg_init_rest(CgDev d, const double* rhs) {
    __shared__ double sh[32];
    CgScalars* S = d.S;
    double rr = 0.0, rs = 0.0;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.n) {
        double sum = 0.0;
        for (int k = d.rowptr[i]; k < d.rowptr[i + 1]; k++) sum += d.val[k] * d.x[d.col[k]];
        double r = rhs[i] - sum;
        double s = d.q[i] * r;
        rr = r * r;
        if (d.fix[i] != 0) { r = 0.0; s = 0.0; }
        rs = r * s;
        d.r[i] = r;
        d.s[i] = s;
        d.p[i] = s;
    }
    int nb = gridDim.x;
    double t0 = block_reduce(rr, sh);
    double t1 = block_reduce(rs, sh);
    if (threadIdx.x == 0) {
        d.part[nb + blockIdx.x] = t0;
        d.part[2 * nb + blockIdx.x] = t1;
    }
    if (last_block(&S->ticket[2])) {
        double rn0 = sum_partials(d.part + nb, nb, sh);
        double p1 = sum_partials(d.part + 2 * nb, nb, sh);
        if (threadIdx.x == 0) {
            S->rnorm0 = rn0;
            S->prod1 = p1;
            S->ticket[2] = 0;
        }
    }
}

}  // namespace

struct gfsph_cg {
    int npoin = 0, nelem = 0, nnode = 0, ndofn = 0, n = 0;
    cudaStream_t stream = nullptr;
    int *rowptr = nullptr, *col = nullptr, *fix = nullptr;
    double *val = nullptr, *q = nullptr;
    double *x = nullptr, *r = nullptr, *r1 = nullptr, *s = nullptr, *p = nullptr, *ap = nullptr, *part = nullptr;
    double *rhs = nullptr, *fixed = nullptr;
    CgScalars* S = nullptr;
    CgScalars* hS = nullptr;
    std::vector<double> diag;   // assembled diagonal (host)
    cudaGraphExec_t graph = nullptr;
    int nblocks = 0;
    long long launches = 0;
};

namespace {

CgDev view(gfsph_cg* c) {
    CgDev d;
    d.n = c->n; d.rowptr = c->rowptr; d.col = c->col; d.val = c->val; d.q = c->q; d.fix = c->fix;
    d.x = c->x; d.r = c->r; d.r1 = c->r1; d.s = c->s; d.p = c->p; d.ap = c->ap; d.part = c->part; d.S = c->S;
    return d;
}

template <class T>
int dal(T** p, size_t n) {
    return cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T)) == cudaSuccess ? 0 : 1;
}

void cg_free(gfsph_cg* c) {
    if (c->graph) cudaGraphExecDestroy(c->graph);
    void* ptrs[] = {c->rowptr, c->col, c->fix, c->val, c->q, c->x, c->r, c->r1, c->s, c->p, c->ap, c->part,
                    c->rhs, c->fixed, c->S};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (c->hS) cudaFreeHost(c->hS);
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
    if (!c) return GFSPH_ERR_ARG;
    c->npoin = npoin; c->nelem = nelem; c->nnode = nnode; c->ndofn = ndofn; c->n = n;
    c->diag.assign(n, 0.0);
    for (int i = 0; i < n; i++)
        for (int k = rowptr[i]; k < rowptr[i + 1]; k++)
            if (col[k] == i) c->diag[i] = val[k];
    c->nblocks = (n + kCgThreads - 1) / kCgThreads;
    int st = 0;
    st |= dal(&c->rowptr, n + 1); st |= dal(&c->col, col.size()); st |= dal(&c->val, val.size());
    st |= dal(&c->fix, n); st |= dal(&c->q, n);
    st |= dal(&c->x, n); st |= dal(&c->r, n); st |= dal(&c->r1, n); st |= dal(&c->s, n); st |= dal(&c->p, n);
    st |= dal(&c->ap, n); st |= dal(&c->part, 3 * (size_t)c->nblocks); st |= dal(&c->rhs, n); st |= dal(&c->fixed, n);
    st |= dal(&c->S, 1);
    if (st || cudaMallocHost((void**)&c->hS, sizeof(CgScalars)) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cg_free(c);
        delete c;
        return GFSPH_ERR_CUDA;
    }
    cudaMemcpy(c->rowptr, rowptr.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(c->col, col.data(), col.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(c->val, val.data(), val.size() * sizeof(double), cudaMemcpyHostToDevice);
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
    // getqmat (:124-159): Jacobi preconditioner; free dofs with a vanishing
    // diagonal are marked -999 for the solve and reset to 0 afterwards
    std::vector<double> q(n), fx(n), b(n);
    std::vector<int> fix(iffix, iffix + n);
    for (int i = 0; i < n; i++) {
        if (std::fabs(c->diag[i]) <= 1.e-35) {
            if (fix[i] == 0) fix[i] = -999;
            q[i] = 0.0;
        } else {
            q[i] = 1.0 / c->diag[i];
        }
        fx[i] = (double)fixed[i];
        b[i] = (double)rcg[i];
    }
    cudaStream_t st = c->stream;
    cudaMemcpyAsync(c->q, q.data(), n * sizeof(double), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(c->fix, fix.data(), n * sizeof(int), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(c->fixed, fx.data(), n * sizeof(double), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(c->rhs, b.data(), n * sizeof(double), cudaMemcpyHostToDevice, st);
    CgScalars init{};
    init.tol = (double)tol;
    init.max_iters = (int)std::min<long long>(10LL * n, 0x7fffffffLL);  // miter = 10*ntotv
    *c->hS = init;
    cudaMemcpyAsync(c->S, c->hS, sizeof(CgScalars), cudaMemcpyHostToDevice, st);
    CgDev d = view(c);
    const int nb = c->nblocks;
    k_cg_init_spmv<<<nb, kCgThreads, 0, st>>>(d, c->fixed);
    k_cg_init_rest<<<nb, kCgThreads, 0, st>>>(d, c->rhs);
    c->launches += 2;
    cudaMemcpyAsync(c->hS, c->S, sizeof(CgScalars), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return GFSPH_ERR_CUDA;
    // rnormX (:93-103): sqrt(fixed.fixed + r0.r0) below tol -> solution 0
    double rnx = c->hS->rnorm0;
    for (int i = 0; i < n; i++) rnx += fx[i] * fx[i];
    rnx = std::sqrt(rnx);
    int iters = 0;
    std::vector<double> xh(n), rh(n);
    if (rnx < (double)tol) {
        std::fill(xh.begin(), xh.end(), 0.0);
        cudaMemcpy(rh.data(), c->r, n * sizeof(double), cudaMemcpyDeviceToHost);
    } else {
        if (!c->graph) {
            cudaGraph_t g = nullptr;
            if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return GFSPH_ERR_CUDA;
            for (int k = 0; k < kIterPerGraph; k++) {
                k_cg_spmv<<<nb, kCgThreads, 0, st>>>(d);
                k_cg_update<<<nb, kCgThreads, 0, st>>>(d);
                k_cg_direction<<<nb, kCgThreads, 0, st>>>(d);
            }
            if (cudaStreamEndCapture(st, &g) != cudaSuccess) return GFSPH_ERR_CUDA;
            cudaError_t e = cudaGraphInstantiate(&c->graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return GFSPH_ERR_CUDA;
        }
        for (;;) {
            if (cudaGraphLaunch(c->graph, st) != cudaSuccess) return GFSPH_ERR_CUDA;
            c->launches += 3 * kIterPerGraph;
            cudaMemcpyAsync(c->hS, c->S, sizeof(CgScalars), cudaMemcpyDeviceToHost, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) return GFSPH_ERR_CUDA;
            if (c->hS->done) break;
        }
        iters = c->hS->iters;
        cudaMemcpy(xh.data(), c->x, n * sizeof(double), cudaMemcpyDeviceToHost);
        cudaMemcpy(rh.data(), c->r, n * sizeof(double), cudaMemcpyDeviceToHost);
        for (int i = 0; i < n; i++)
            if (fix[i] == -999) fix[i] = 0;
    }
    for (int i = 0; i < n; i++) {
        ficg[i] = (float)xh[i];
        rcg[i] = (float)rh[i];
        iffix[i] = fix[i];
    }
    if (iterations) *iterations = iters;
    return cudaGetLastError() == cudaSuccess ? GFSPH_OK : GFSPH_ERR_CUDA;
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
