// The SPH -> FEM coupling pass of get_gradhs_w
// (SPH_GFL_SW_Interactions_2019.f90:368-564) on a node window of the DEM
// background triangulation (SPH_FEM_topo_2019.f90:583-604): the depth of the
// particles is carried by inverse distance to the nodes of the triangle that
// holds each particle, differentiated per element, and projected back to the
// nodes by solving M g = sum_e (A/3) grad_e with lumped-mass Jacobi sweeps.
//
// Every node gathers from its (up to six) triangles in element order, so the
// FP32 sums run in the order of the reference's element loops and no atomics
// are needed past the particle scatter.
#pragma once
#include "gfsph_kernels.cuh"

namespace gfsph {

// Node window [ix0, ix0+nwx) x [iy0, iy0+nwy) of the DEM; cells (ci, cj) of
// the window hold triangles 2*(cj*(nwx-1)+ci) (nodes n, n+1, n+1+nwx) and
// 2*(cj*(nwx-1)+ci)+1 (n, n+1+nwx, n+nwx), n = cj*nwx + ci.
struct Window {
    int ix0, iy0, nwx, nwy;
    float xming, yming, dxg, dyg;
};

__device__ __forceinline__ float win_x(const Window& w, int i) { return w.xming + (float)(w.ix0 + i) * w.dxg; }
__device__ __forceinline__ float win_y(const Window& w, int j) { return w.yming + (float)(w.iy0 + j) * w.dyg; }

__device__ __forceinline__ void tri_nodes(const Window& w, int e, int a[3]) {
    int c = e >> 1, ci = c % (w.nwx - 1), cj = c / (w.nwx - 1), n0 = cj * w.nwx + ci;
    a[0] = n0;
    if ((e & 1) == 0) { a[1] = n0 + 1; a[2] = n0 + 1 + w.nwx; }
    else { a[1] = n0 + 1 + w.nwx; a[2] = n0 + w.nwx; }
}

__device__ __forceinline__ void node_xy(const Window& w, int node, float& x, float& y) {
    x = win_x(w, node % w.nwx);
    y = win_y(w, node / w.nwx);
}

// getgeom2D (SPH_FEM_topo_2019.f90:1675-1716): shape-function derivatives
// g[0..2] = dN/dx, g[3..5] = dN/dy and g[6] = rj (twice the area).
__device__ __forceinline__ void tri_geome(const Window& w, const int a[3], float g[7]) {
    float x[3], y[3];
    for (int k = 0; k < 3; k++) node_xy(w, a[k], x[k], y[k]);
    float x21 = x[1] - x[0], x31 = x[2] - x[0], y21 = y[1] - y[0], y31 = y[2] - y[0];
    float rj = x21 * y31 - x31 * y21;
    float rj1 = 1.f / rj;
    float xix = y31 * rj1, xiy = -(x31 * rj1), etx = -(y21 * rj1), ety = x21 * rj1;
    const float nxi[3] = {-1.f, 1.f, 0.f}, net[3] = {-1.f, 0.f, 1.f};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        g[k] = xix * nxi[k] + etx * net[k];
        g[k + 3] = xiy * nxi[k] + ety * net[k];
    }
    g[6] = rj;
}

// which_element (:309-344) and the IDW of :447-463: the barycentric test on
// the triangles of the 3 x 3 cells around the particle, the highest element
// index that passes (the reference's element loop overwrites), then
// rho/r and 1/r to the element's three nodes (FP64 accumulators).
__global__ void k_couple_idw(PState B, int n, Window w, double* a1, double* a2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (B.flag[i]) continue;
        const float2 p = B.pos[i];
        const int ci = (int)floorf((p.x - w.xming) / w.dxg) - w.ix0;
        const int cj = (int)floorf((p.y - w.yming) / w.dyg) - w.iy0;
        int which = -1;
        for (int dj = -1; dj <= 1; dj++)
            for (int di = -1; di <= 1; di++) {
                int ki = ci + di, kj = cj + dj;
                if (ki < 0 || kj < 0 || ki > w.nwx - 2 || kj > w.nwy - 2) continue;
                for (int t = 0; t < 2; t++) {
                    int e = 2 * (kj * (w.nwx - 1) + ki) + t;
                    if (e <= which) continue;
                    int a[3];
                    tri_nodes(w, e, a);
                    float x1, y1, x2, y2, x3, y3;
                    node_xy(w, a[0], x1, y1); node_xy(w, a[1], x2, y2); node_xy(w, a[2], x3, y3);
                    float x31 = x1 - x3, y31 = y1 - y3, x32 = x2 - x3, y32 = y2 - y3;
                    float detx = x31 * y32 - y31 * x32;
                    float x30 = p.x - x3, y30 = p.y - y3;
                    float sh1 = (x30 * y32 - y30 * x32) / detx;
                    float sh2 = (y30 * x31 - x30 * y31) / detx;
                    float sh3 = (1.f - sh1) - sh2;
                    if (sh1 >= 0.f && sh1 <= 1.f && sh2 >= 0.f && sh2 <= 1.f && sh3 >= 0.f && sh3 <= 1.f) which = e;
                }
            }
        if (which < 0) continue;
        int a[3];
        tri_nodes(w, which, a);
        const float h = B.rho[i];
        for (int k = 0; k < 3; k++) {
            float xn, yn;
            node_xy(w, a[k], xn, yn);
            float rdist = sqrtf((xn - p.x) * (xn - p.x) + (yn - p.y) * (yn - p.y));
            atomicAdd(&a1[a[k]], (double)(h / rdist));
            atomicAdd(&a2[a[k]], (double)(1.f / rdist));
        }
    }
}

// hs_w = sum(h/r) / sum(1/r) where sum(1/r) >= 1e-6 (:465-468).
__global__ void k_couple_hs(const double* a1, const double* a2, int nn, float* hs) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x)
        hs[k] = (a2[k] < 1.e-6) ? 0.f : (float)(a1[k] / a2[k]);
}

// The triangles of node (i, j) in element order, with the node's local index
// in each: cell (i-1, j-1) t1 (node 3), t2 (node 2); cell (i, j-1) t2 (node 3);
// cell (i-1, j) t1 (node 2); cell (i, j) t1, t2 (node 1).
__device__ __forceinline__ int node_tris(const Window& w, int i, int j, int e[6], int loc[6]) {
    int m = 0;
    const int nc = w.nwx - 1;
    if (i > 0 && j > 0) {
        int c = (j - 1) * nc + (i - 1);
        e[m] = 2 * c; loc[m++] = 2;
        e[m] = 2 * c + 1; loc[m++] = 1;
    }
    if (i < w.nwx - 1 && j > 0) { e[m] = 2 * ((j - 1) * nc + i) + 1; loc[m++] = 2; }
    if (i > 0 && j < w.nwy - 1) { e[m] = 2 * (j * nc + (i - 1)); loc[m++] = 1; }
    if (i < w.nwx - 1 && j < w.nwy - 1) {
        int c = j * nc + i;
        e[m] = 2 * c; loc[m++] = 0;
        e[m] = 2 * c + 1; loc[m++] = 0;
    }
    return m;
}

// rhs = sum_e grad_e * rj/6 (:474-490) and the lumped mass mmatl = sum_e rj/6
// (SPH_FEM_topo_2019.f90:1764-1769); g starts at 0.
__global__ void k_couple_rhs(Window w, const float* hs, float2* rhs, float* ml, float2* g) {
    const int nn = w.nwx * w.nwy;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nn; p += gridDim.x * blockDim.x) {
        int e[6], loc[6];
        int m = node_tris(w, p % w.nwx, p / w.nwx, e, loc);
        float rx = 0.f, ry = 0.f, l = 0.f;
        for (int k = 0; k < m; k++) {
            int a[3];
            float ge[7];
            tri_nodes(w, e[k], a);
            tri_geome(w, a, ge);
            float dxe = 0.f, dye = 0.f;
            for (int q = 0; q < 3; q++) {
                dxe = dxe + hs[a[q]] * ge[q];
                dye = dye + hs[a[q]] * ge[q + 3];
            }
            float coe = ge[6] / 6.f;
            rx = rx + dxe * coe;
            ry = ry + dye * coe;
            l = l + coe;
        }
        rhs[p] = make_float2(rx, ry);
        ml[p] = l;
        g[p] = make_float2(0.f, 0.f);
    }
}

// One sweep g += (rhs - M g) / mmatl with the consistent P1 mass matrix
// (rj/24) * [2 1 1; 1 2 1; 1 1 2] (:503-529).
__global__ void k_couple_jacobi(Window w, const float2* g, const float2* rhs, const float* ml, float2* gout) {
    const int nn = w.nwx * w.nwy;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nn; p += gridDim.x * blockDim.x) {
        int e[6], loc[6];
        int m = node_tris(w, p % w.nwx, p / w.nwx, e, loc);
        float hx = 0.f, hy = 0.f;
        for (int k = 0; k < m; k++) {
            int a[3];
            float ge[7];
            tri_nodes(w, e[k], a);
            tri_geome(w, a, ge);
            float coe = ge[6] / 24.f;
            for (int q = 0; q < 3; q++) {
                float cm = (q == loc[k]) ? 2.f : 1.f;
                float2 gq = g[a[q]];
                hx = hx + (cm * coe) * gq.x;
                hy = hy + (cm * coe) * gq.y;
            }
        }
        float2 gp = g[p], r = rhs[p];
        float l = ml[p];
        gout[p] = make_float2(gp.x + (r.x - hx) / l, gp.y + (r.y - hy) / l);
    }
}

}  // namespace gfsph
