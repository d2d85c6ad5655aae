// The Taylor-Galerkin shallow-water step of the GFL module
// (Time_Integration_GFL, GFL_MAIN_2019.f90:216-284) on the device, for the
// SPH <-> FEM coupling loop of the reference (SPH_FEM_Driver_2019.f90:1630-1650:
// get_gradhs_w, then time_integration_gfl on the mesh).
//
// Set-up on the host, once, in single precision and in the reference's
// order: getgeom2D (:1275-1345), getmmatl (:2794-2816), Get_Topol (:1346-1552,
// nodal slopes and curvatures by lumped-mass projection on this mesh),
// get_boun_nodes_2D (:1553-1653: boundary nodes and their tangents, the
// element means of the nodal topography rows) and bounel (:1655-1762:
// boundary sides), the last two with adjacency lists in element order where
// the reference searches every element (the same sums in the same order).
//
// One step, five kernels (niter + 3 launches):
//   k_gfl_nodes   fluxes and sources at the nodes (first_step :1890-1958);
//   k_gfl_elems   per element: the half-step values at the Gauss points
//                 (first_step :1964-2048), at each of them the fluxes and
//                 sources of second_step (:2157-2300), and the term each
//                 Gauss point adds to each of the element's nodes (:2300-2312),
//                 one float4 per (element, node, Gauss point);
//   k_gfl_rhs     per node, those terms gathered over its elements in element
//                 order (Gauss points in order), then its boundary sides in side
//                 order, as second_step adds them (:2300-2355): the right-hand
//                 side; the wall projection of solve (:2629-2656) and its first
//                 sweep;
//   k_gfl_mass    the further sweeps u += (rhs - M u)/ML with the wall
//                 filter (:2660-2785), M u gathered in element order;
//   k_gfl_update  addthem (:3199-3215) and check (:3306-3345).
// Every sum runs in the Fortran's order with IEEE FP32 operations (the
// library is built without FMA contraction), so the device step equals the
// single-precision restatement bit for bit; real powers (Manning's 7/3,
// Coussot's) and the exp of the tanfi decay are taken in FP64 and rounded once.
//
// Scope: nsour 1, itens 0, icpwpF 0, no prescribed, absorbing or loaded
// boundary nodes (every boundary node is a wall), no atmospheric pressure or
// wind, no shock smoothing, ic_adapt_dt_elem_gfl 0 (a fixed dt per call),
// nfric 0-8 (frictlaws :3801-3990).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <unordered_map>
#include <vector>

#include "../../include/gfsph.h"

namespace gfsph {
namespace gfl {

constexpr int kGflThreads = 128;

struct GflConst {
    float cgra, dens, cmanning, cori, tauy0, constK, tanfi8, hfrict0, tanfi0, bfact;
    int nfric, ntype, ngaus;
    float swl, comp;
};

struct GflDev {
    int npoin, nelem;
    const int* elem;       // (3, nelem) 0-based
    const float* geome;    // (7, nelem): dN/dx (3), dN/dy (3), 2 * area
    const float* topel;    // (9, nelem)
    const float* topol;    // (9, npoin)
    const float* mmatl;    // lumped mass
    const int* adj_ptr;    // node -> (element, local node) entries, element order
    const int2* adj;
    const int* bside_ptr;  // node -> (boundary side, position in it), side order
    const int2* bside;
    const int2* side_nodes;   // boundary side -> its two nodes
    const float4* side_geom;  // cosx, cosy, length
    const int* bnode;         // node -> boundary-node index or -1
    const float2* rtang;      // boundary-node tangents (normalised where |t| >= 1e-6)
    const float* hs_w;        // WIR: soil depth at the nodes (or null)
    const float2* gradhs_w;   // WIR: its nodal gradient
    float* unkno;             // (3, npoin) h, hu, hv
    float* fnode;             // (9, npoin): fluxp(3), fluyp(3), gpoin(3)
    float4* gt;               // per element, local node and Gauss point (3 x 3 float4): the rhs terms of
                              // second_step for h, hu, hv (w unused)
    float* rhs1;              // (3, npoin)
    float* rhs0[2];           // (3, npoin), double buffer of the sweeps
};

// frictlaws (GFL_MAIN_2019.f90:3801-3990) with pwp = 0 and no wind or
// atmospheric pressure; mt = mini_topo(1..9).
__device__ __forceinline__ void frictlaws(const GflConst& c, float tanfi, const float* mt, float h, float hu, float hv,
                                          float HH, float& frictx, float& fricty, float& slopx, float& slopy,
                                          float& correx, float& correy) {
    const float gtanfi = c.cgra * tanfi, gtanfi8 = c.cgra * c.tanfi8;
    const double c73 = (double)(7.f / 3.f);
    float hinv = 0.f;
    if (h > 0.f) hinv = 1.f / h;
    const float hfrict = fmaxf(h, c.hfrict0);
    const float hvmod = sqrtf(hu * hu + hv * hv);
    const float vmod = hvmod * hinv;
    float hvmodinv = 0.f;
    if (hvmod >= 1.e-5f) hvmodinv = 1.f / hvmod;
    const float pwp = 0.f;
    frictx = 0.f;
    fricty = 0.f;
    if (c.nfric == 1) {
        const float cf1 = (c.cgra * c.cmanning) * c.cmanning;
        const float p = (float)pow((double)hfrict, c73);
        frictx = ((cf1 * hu) * hvmod) / p;
        fricty = ((cf1 * hv) * hvmod) / p;
    } else if (c.nfric == 2) {
        const float cf2a = c.constK / (8.f * c.dens);
        frictx = (cf2a * hu) / (hfrict * hfrict);
        fricty = (cf2a * hv) / (hfrict * hfrict);
    } else if (c.nfric == 3) {
        const float cf3a = (1.93f * (float)pow((double)c.constK, (double)0.9f)) * (float)pow((double)c.tauy0, (double)0.1f);
        const float cf3b = (c.tauy0 + cf3a * (float)pow((double)(vmod / hfrict), (double)0.3f)) / c.dens;
        frictx = (cf3b * hu) * hvmodinv;
        fricty = (cf3b * hv) * hvmodinv;
    } else if (c.nfric == 4) {
        const float a_hat = ((6.f * c.constK) * hvmod) / (c.tauy0 * (hfrict * hfrict));
        const float a2 = 48.f, b2 = -(32.f * a_hat) - 114.f, c2 = 65.f;
        const float xh = (-b2 - sqrtf(b2 * b2 - (4.f * a2) * c2)) / (2.f * a2);
        const float cf4b = (c.tauy0 / xh) / c.dens;
        frictx = (cf4b * hu) * hvmodinv;
        fricty = (cf4b * hv) * hvmodinv;
    } else if (c.nfric == 5) {
        const float cf5 = gtanfi * h;
        frictx = (cf5 * hu) * hvmodinv;
        fricty = (cf5 * hv) * hvmodinv;
    } else if (c.nfric == 6) {
        float factpw = 1.f - pwp * hinv;
        if (factpw > 1.f) factpw = 1.f;
        if (factpw < 0.f) factpw = 0.f;
        const float cf5 = (gtanfi8 * factpw) * h;
        frictx = (cf5 * hu) * hvmodinv;
        fricty = (cf5 * hv) * hvmodinv;
    } else if (c.nfric == 7 || c.nfric == 8) {
        const float vx = hu * hinv, vy = hv * hinv;
        const float vm = sqrtf(vx * vx + vy * vy);
        float cv2byR = 0.f;
        if (vm >= 1e-5f) {
            const float cosa = vx / vm, sina = vy / vm;
            const float cos2 = cosa * cosa, sin2 = sina * sina, cbs = sina * cosa;
            const float xnum = (mt[6] * cos2 + mt[7] * cbs) + mt[8] * sin2;
            const float xden = (mt[3] * cos2 + mt[4] * cbs) + mt[5] * sin2;
            cv2byR = (vm * vm) * (xnum / xden);
        }
        float factaux = c.cgra + cv2byR;
        if (factaux < 0.f) factaux = 0.f;
        if (c.nfric == 7) {
            const float cf5 = (factaux * c.tanfi8) * h;
            frictx = frictx + (cf5 * hu) * hvmodinv;
            fricty = fricty + (cf5 * hv) * hvmodinv;
        } else {
            float factpw = 1.f - pwp * hinv;
            if (factpw > 1.f) factpw = 1.f;
            if (factpw < 0.f) factpw = 0.f;
            const float cf8 = ((factaux * c.tanfi8) * h) * factpw;
            frictx = (cf8 * hu) * hvmodinv;
            fricty = (cf8 * hv) * hvmodinv;
        }
    }
    if (c.cmanning != 0.f && c.nfric != 1) {
        const float cf1 = (c.cgra * c.cmanning) * c.cmanning;
        const float p = (float)pow((double)hfrict, c73);
        frictx = frictx + ((cf1 * hu) * hvmod) / p;
        fricty = fricty + ((cf1 * hv) * hvmod) / p;
    }
    slopx = -((c.cgra * (h - HH)) * mt[1]);
    slopy = -((c.cgra * (h - HH)) * mt[2]);
    correx = 0.f - (h * 0.f) / 1000.f;
    correy = 0.f - (h * 0.f) / 1000.f;
}

__device__ __forceinline__ void sources(const GflConst& c, float frx, float fry, float slx, float sly, float cx,
                                        float cy, float hu, float hv, float* g) {
    g[0] = 0.f;
    if (c.ntype == 3) {  // nsour 1: no slope term for flow over a dry bed
        g[1] = (c.cori * hv - frx) + cx;
        g[2] = (-(c.cori * hu) - fry) + cy;
    } else {
        g[1] = ((c.cori * hv - frx) + slx) + cx;
        g[2] = ((-(c.cori * hu) - fry) + sly) + cy;
    }
}

__global__ void k_gfl_nodes(GflDev d, GflConst c, float tanfi) {
    for (int ip = blockIdx.x * blockDim.x + threadIdx.x; ip < d.npoin; ip += gridDim.x * blockDim.x) {
        const float h = d.unkno[3 * ip], hu = d.unkno[3 * ip + 1], hv = d.unkno[3 * ip + 2];
        float hinv = 0.f;
        if (h >= c.comp) hinv = 1.f / h;
        float HH, pres;
        if (c.ntype == 2) {
            HH = c.swl - d.topol[9 * ip];
            if (d.hs_w) HH = HH - d.hs_w[ip];
            pres = (0.5f * c.cgra) * (h * h - HH * HH);
        } else {
            HH = 0.f;
            pres = ((0.5f * c.cgra) * h) * h;
        }
        float* f = d.fnode + 9 * (size_t)ip;
        f[0] = hu; f[1] = (hu * hu) * hinv + pres; f[2] = (hu * hv) * hinv;
        f[3] = hv; f[4] = (hu * hv) * hinv; f[5] = (hv * hv) * hinv + pres;
        float mt[9];
        for (int k = 0; k < 9; k++) mt[k] = d.topol[9 * (size_t)ip + k];
        if (d.hs_w) { mt[1] = mt[1] + d.gradhs_w[ip].x; mt[2] = mt[2] + d.gradhs_w[ip].y; }
        float frx, fry, slx, sly, cx, cy;
        frictlaws(c, tanfi, mt, h, hu, hv, HH, frx, fry, slx, sly, cx, cy);
        sources(c, frx, fry, slx, sly, cx, cy, hu, hv, f + 6);
    }
}

__device__ __forceinline__ void gauss_point(int ngaus, int ig, float sh[3]) {
    if (ngaus == 3) {
        const float p1[3] = {1.0f / 6.0f, 4.0f / 6.0f, 1.0f / 6.0f}, p2[3] = {1.0f / 6.0f, 1.0f / 6.0f, 4.0f / 6.0f};
        sh[0] = p1[ig];
        sh[1] = p2[ig];
    } else {
        sh[0] = 1.0f / 3.0f;
        sh[1] = 1.0f / 3.0f;
    }
    sh[2] = (1.0f - sh[0]) - sh[1];
}

__global__ void k_gfl_elems(GflDev d, GflConst c, float tanfi, float dt) {
    const float delt2 = 0.5f * dt;
    const float cgra05 = c.cgra * 0.5f;
    for (int ie = blockIdx.x * blockDim.x + threadIdx.x; ie < d.nelem; ie += gridDim.x * blockDim.x) {
        int nd[3];
        float gx[3], gy[3];
        for (int k = 0; k < 3; k++) {
            nd[k] = d.elem[3 * (size_t)ie + k];
            gx[k] = d.geome[7 * (size_t)ie + k];
            gy[k] = d.geome[7 * (size_t)ie + 3 + k];
        }
        float div[3] = {0.f, 0.f, 0.f};
        for (int k = 0; k < 3; k++) {
            const float* f = d.fnode + 9 * (size_t)nd[k];
            for (int ia = 0; ia < 3; ia++) div[ia] = (div[ia] + gx[k] * f[ia]) + gy[k] * f[3 + ia];
        }
        // element gradient of the WIR soil depth (get_gradhs_w :469-481)
        float gw0 = 0.f, gw1 = 0.f;
        if (d.hs_w)
            for (int k = 0; k < 3; k++) {
                gw0 = gw0 + d.hs_w[nd[k]] * gx[k];
                gw1 = gw1 + d.hs_w[nd[k]] * gy[k];
            }
        float mt[9];
        for (int k = 0; k < 9; k++) mt[k] = d.topel[9 * (size_t)ie + k];
        if (d.hs_w) { mt[1] = mt[1] + gw0; mt[2] = mt[2] + gw1; }
        for (int ig = 0; ig < c.ngaus; ig++) {
            float sh[3];
            gauss_point(c.ngaus, ig, sh);
            float src[3] = {0.f, 0.f, 0.f}, var[3] = {0.f, 0.f, 0.f};
            for (int k = 0; k < 3; k++) {
                const float* f = d.fnode + 9 * (size_t)nd[k];
                const float* u = d.unkno + 3 * (size_t)nd[k];
                for (int ia = 0; ia < 3; ia++) {
                    src[ia] = src[ia] + sh[k] * f[6 + ia];
                    var[ia] = var[ia] + sh[k] * u[ia];
                }
            }
            float ue[3];
            for (int ia = 0; ia < 3; ia++) ue[ia] = var[ia] + delt2 * (src[ia] - div[ia]);
            // second_step at this Gauss point
            const float h = ue[0], hu = ue[1], hv = ue[2];
            float hinv = 0.f;
            if (h >= c.comp) hinv = 1.f / h;
            float HH, pres;
            if (c.ntype == 2) {
                HH = 0.f;
                for (int k = 0; k < 3; k++) {
                    HH = HH + sh[k] * d.topol[9 * (size_t)nd[k]];
                    if (d.hs_w) HH = HH + sh[k] * d.hs_w[nd[k]];
                }
                HH = c.swl - HH;
                pres = cgra05 * (h * h - HH * HH);
            } else {
                HH = 0.f;
                pres = (cgra05 * h) * h;
            }
            float o[9];
            o[0] = hu; o[1] = (hu * hu) * hinv + pres; o[2] = (hu * hv) * hinv;
            o[3] = hv; o[4] = o[2]; o[5] = (hv * hv) * hinv + pres;
            float frx, fry, slx, sly, cx, cy;
            frictlaws(c, tanfi, mt, h, hu, hv, HH, frx, fry, slx, sly, cx, cy);
            sources(c, frx, fry, slx, sly, cx, cy, hu, hv, o + 6);
            // the terms this Gauss point adds to each node's rhs (:2300-2312)
            const float dvolu = d.geome[7 * (size_t)ie + 6] / (float)(2 * c.ngaus);
            for (int in = 0; in < 3; in++) {
                float t[3];
                for (int ia = 0; ia < 3; ia++)
                    t[ia] = (((gx[in] * o[ia] + gy[in] * o[3 + ia]) + sh[in] * o[6 + ia]) * dvolu) * dt;
                d.gt[3 * (3 * (size_t)ie + in) + ig] = make_float4(t[0], t[1], t[2], 0.f);
            }
        }
    }
}

// The wall projection of solve: no normal component (anx, any) = (t2, -t1).
__device__ __forceinline__ void wall(float2 t, float* r) {
    const float anx = t.y, any = -t.x;
    const float rn = r[1] * anx + r[2] * any;
    r[1] = r[1] - rn * anx;
    r[2] = r[2] - rn * any;
}

__global__ void k_gfl_rhs(GflDev d, GflConst c, float dt) {
    const float mmatb[2][2] = {{2.f, 1.f}, {1.f, 2.f}};
    for (int ip = blockIdx.x * blockDim.x + threadIdx.x; ip < d.npoin; ip += gridDim.x * blockDim.x) {
        float r[3] = {0.f, 0.f, 0.f};
        for (int q = d.adj_ptr[ip]; q < d.adj_ptr[ip + 1]; q++) {
            const int2 a = d.adj[q];  // element, local node: its terms in Gauss point order
            const float4* row = d.gt + 3 * (3 * (size_t)a.x + a.y);
            for (int ig = 0; ig < c.ngaus; ig++) {
                const float4 t = row[ig];
                r[0] = r[0] + t.x; r[1] = r[1] + t.y; r[2] = r[2] + t.z;
            }
        }
        for (int q = d.bside_ptr[ip]; q < d.bside_ptr[ip + 1]; q++) {
            const int2 b = d.bside[q];  // side, position of this node in it
            const int2 nn = d.side_nodes[b.x];
            const float4 g = d.side_geom[b.x];
            const float coe = g.z / 6.f;
            for (int j = 0; j < 2; j++) {
                const int jn = j ? nn.y : nn.x;
                const float cm = (mmatb[b.y][j] * coe) * dt;
                const float* f = d.fnode + 9 * (size_t)jn;
                for (int ia = 0; ia < 3; ia++) r[ia] = r[ia] - cm * (f[ia] * g.x + f[3 + ia] * g.y);
            }
        }
        const int bn = d.bnode[ip];
        if (bn >= 0) wall(d.rtang[bn], r);
        const float cm = d.mmatl[ip];
        float r0[3];
        for (int ia = 0; ia < 3; ia++) {
            d.rhs1[3 * (size_t)ip + ia] = r[ia];
            r0[ia] = r[ia] / cm;
        }
        if (bn >= 0) {
            const float2 t = d.rtang[bn];
            if (!(fabsf(t.x) + fabsf(t.y) < 1.e-06f)) wall(t, r0);
        }
        for (int ia = 0; ia < 3; ia++) d.rhs0[0][3 * (size_t)ip + ia] = r0[ia];
    }
}

__global__ void k_gfl_mass(GflDev d, int src) {
    const float mm[3][3] = {{2.f, 1.f, 1.f}, {1.f, 2.f, 1.f}, {1.f, 1.f, 2.f}};
    const float* __restrict__ in = src ? d.rhs0[1] : d.rhs0[0];
    float* __restrict__ out = src ? d.rhs0[0] : d.rhs0[1];
    for (int ip = blockIdx.x * blockDim.x + threadIdx.x; ip < d.npoin; ip += gridDim.x * blockDim.x) {
        float r2[3] = {0.f, 0.f, 0.f};
        for (int q = d.adj_ptr[ip]; q < d.adj_ptr[ip + 1]; q++) {
            const int2 a = d.adj[q];
            const float coe = d.geome[7 * (size_t)a.x + 6] / 24.f;
            for (int jn = 0; jn < 3; jn++) {
                const int jp = d.elem[3 * (size_t)a.x + jn];
                const float cm = mm[a.y][jn];
                for (int ia = 0; ia < 3; ia++) r2[ia] = r2[ia] + (cm * coe) * in[3 * (size_t)jp + ia];
            }
        }
        const float ml = d.mmatl[ip];
        float r0[3];
        for (int ia = 0; ia < 3; ia++) r0[ia] = in[3 * (size_t)ip + ia] + (d.rhs1[3 * (size_t)ip + ia] - r2[ia]) / ml;
        const int bn = d.bnode[ip];
        if (bn >= 0) {
            const float2 t = d.rtang[bn];
            if (!(fabsf(t.x) + fabsf(t.y) < 1.e-06f)) wall(t, r0);
        }
        for (int ia = 0; ia < 3; ia++) out[3 * (size_t)ip + ia] = r0[ia];
    }
}

__global__ void k_gfl_update(GflDev d, GflConst c, int src) {
    const float* __restrict__ du = src ? d.rhs0[1] : d.rhs0[0];
    for (int ip = blockIdx.x * blockDim.x + threadIdx.x; ip < d.npoin; ip += gridDim.x * blockDim.x) {
        float* u = d.unkno + 3 * (size_t)ip;
        for (int ia = 0; ia < 3; ia++) u[ia] = u[ia] + du[3 * (size_t)ip + ia];
        if (u[0] < c.comp) {  // check: ff = 0 without prescribed values, unkno = ff * unkno
            u[0] = 0.f * u[0]; u[1] = 0.f * u[1]; u[2] = 0.f * u[2];
        }
    }
}

template <class T>
int dal(T** p, size_t n) {
    *p = nullptr;
    return cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T)) == cudaSuccess ? 0 : 1;
}

int blocks(long long n) {
    long long b = (n + kGflThreads - 1) / kGflThreads;
    return (int)std::min<long long>(std::max<long long>(b, 1), 148LL * 32);
}

}  // namespace gfl
}  // namespace gfsph

using namespace gfsph::gfl;

struct gfsph_gfl {
    gfsph_gfl_params P{};
    GflConst c{};
    int npoin = 0, nelem = 0;
    cudaStream_t stream = nullptr;
    double time = 0.0;
    std::vector<float> topol, topel;  // host copies (gfsph_gfl_topol)
    int *elem = nullptr, *adj_ptr = nullptr, *bside_ptr = nullptr, *bnode = nullptr;
    int2 *adj = nullptr, *bside = nullptr, *side_nodes = nullptr;
    float *geome = nullptr, *d_topel = nullptr, *d_topol = nullptr, *mmatl = nullptr, *hs_w = nullptr;
    float4* side_geom = nullptr;
    float2 *rtang = nullptr, *gradhs_w = nullptr;
    float4* gt = nullptr;
    float *unkno = nullptr, *fnode = nullptr, *rhs1 = nullptr, *rhs0a = nullptr, *rhs0b = nullptr;
    bool wir = false;
    long long launches = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // around the last gfsph_gfl_step
    double last_ms = 0.0;
};

namespace {

void gfl_free(gfsph_gfl* g) {
    void* ptrs[] = {g->elem, g->adj_ptr, g->bside_ptr, g->bnode, g->adj, g->bside, g->side_nodes, g->geome,
                    g->d_topel, g->d_topol, g->mmatl, g->hs_w, g->side_geom, g->rtang, g->gradhs_w, g->unkno,
                    g->fnode, g->gt, g->rhs1, g->rhs0a, g->rhs0b};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (g->ev0) cudaEventDestroy(g->ev0);
    if (g->ev1) cudaEventDestroy(g->ev1);
    if (g->stream) cudaStreamDestroy(g->stream);
}

GflDev view(gfsph_gfl* g) {
    GflDev d;
    d.npoin = g->npoin; d.nelem = g->nelem; d.elem = g->elem; d.geome = g->geome; d.topel = g->d_topel;
    d.topol = g->d_topol; d.mmatl = g->mmatl; d.adj_ptr = g->adj_ptr; d.adj = g->adj; d.bside_ptr = g->bside_ptr;
    d.bside = g->bside; d.side_nodes = g->side_nodes; d.side_geom = g->side_geom; d.bnode = g->bnode;
    d.rtang = g->rtang; d.hs_w = g->wir ? g->hs_w : nullptr; d.gradhs_w = g->gradhs_w; d.unkno = g->unkno;
    d.fnode = g->fnode; d.gt = g->gt; d.rhs1 = g->rhs1; d.rhs0[0] = g->rhs0a; d.rhs0[1] = g->rhs0b;
    return d;
}

}  // namespace

extern "C" {

int gfsph_gfl_create(const gfsph_gfl_params* p, int npoin, int nelem, const float* coord, const int* intmat,
                     const float* z, gfsph_gfl** out) try {
    if (!p || !coord || !intmat || !z || !out || npoin < 3 || nelem < 1) return GFSPH_ERR_ARG;
    *out = nullptr;
    const float* k = p->constF;  // k[i-1] = constF(i)
    const int nfric = (int)(k[4] + 0.01f);
    if (nfric < 0 || nfric > 8) return GFSPH_ERR_UNSUPPORTED;
    if ((int)k[10] != 0) return GFSPH_ERR_UNSUPPORTED;  // itens: the viscous stresses are not built
    if (nfric == 4 && !(k[5] >= 1.e-32f)) return GFSPH_ERR_ARG;
    // Input_GFL stops on these (GFL_MAIN_2019.f90:1113-1121)
    if (!(k[9] > 1.e-32f) || (nfric == 2 && k[1] <= 0.001f)) return GFSPH_ERR_ARG;
    for (int i = 0; i < 15; i++)
        if (k[i] < 0.f) return GFSPH_ERR_ARG;  // the reader keeps absolute values (:1107-1110)
    if ((p->ntype != 2 && p->ntype != 3) || (p->ngaus != 1 && p->ngaus != 3) || p->niter < 1 || !(p->comp > 0.f))
        return GFSPH_ERR_UNSUPPORTED;
    for (long long e = 0; e < 3LL * nelem; e++)
        if (intmat[e] < 1 || intmat[e] > npoin) return GFSPH_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return GFSPH_ERR_NO_DEVICE;
    const size_t np = (size_t)npoin, ne = (size_t)nelem;
    auto IM = [&](int in, size_t ie) { return intmat[ie * 3 + in] - 1; };  // 0-based
    // getgeom2D
    std::vector<float> geome(7 * ne), mmatl(np, 0.f), topol(9 * np, 0.f), topel(9 * ne, 0.f);
    const float nxi[3] = {-1.0f, 1.0f, 0.0f}, net[3] = {-1.0f, 0.0f, 1.0f};
    for (size_t ie = 0; ie < ne; ie++) {
        float x[3], y[3];
        for (int in = 0; in < 3; in++) { x[in] = coord[2 * (size_t)IM(in, ie)]; y[in] = coord[2 * (size_t)IM(in, ie) + 1]; }
        const float x21 = x[1] - x[0], x31 = x[2] - x[0], y21 = y[1] - y[0], y31 = y[2] - y[0];
        const float rj = x21 * y31 - x31 * y21;
        if (!(rj > 0.f)) return GFSPH_ERR_ARG;  // elements must be counter-clockwise
        const float rj1 = 1.f / rj;
        const float xix = y31 * rj1, xiy = -x31 * rj1, etx = -y21 * rj1, ety = x21 * rj1;
        for (int in = 0; in < 3; in++) {
            geome[7 * ie + in] = xix * nxi[in] + etx * net[in];
            geome[7 * ie + 3 + in] = xiy * nxi[in] + ety * net[in];
        }
        geome[7 * ie + 6] = rj;
    }
    auto G = [&](int r, size_t ie) { return geome[7 * ie + r]; };
    // getmmatl
    for (size_t ie = 0; ie < ne; ie++) {
        const float area3 = G(6, ie) / 6.f;
        for (int in = 0; in < 3; in++) mmatl[IM(in, ie)] = mmatl[IM(in, ie)] + area3;
    }
    // Get_Topol: nodal Zx, Zy, then second derivatives, by lumped-mass projection (5 sweeps)
    for (size_t ip = 0; ip < np; ip++) topol[9 * ip] = z[ip];
    const float mm[3][3] = {{2.f, 1.f, 1.f}, {1.f, 2.f, 1.f}, {1.f, 1.f, 2.f}};
    std::vector<float> rhs(3 * np), rhelp(3 * np);
    auto project = [&](int nrows, const int* rows) {
        for (size_t ip = 0; ip < np; ip++)
            for (int q = 0; q < nrows; q++) topol[9 * ip + rows[q]] = rhs[3 * ip + q] / mmatl[ip];
        for (int iiter = 2; iiter <= 5; iiter++) {
            std::fill(rhelp.begin(), rhelp.end(), 0.f);
            for (size_t ie = 0; ie < ne; ie++) {
                const float coe = G(6, ie) / 24.f;
                for (int in = 0; in < 3; in++) {
                    const int ip = IM(in, ie);
                    for (int jn = 0; jn < 3; jn++) {
                        const int jp = IM(jn, ie);
                        const float cm = mm[in][jn];
                        for (int q = 0; q < nrows; q++)
                            rhelp[3 * (size_t)ip + q] = rhelp[3 * (size_t)ip + q] + cm * coe * topol[9 * (size_t)jp + rows[q]];
                    }
                }
            }
            for (size_t ip = 0; ip < np; ip++)
                for (int q = 0; q < nrows; q++)
                    topol[9 * ip + rows[q]] = topol[9 * ip + rows[q]] + (rhs[3 * ip + q] - rhelp[3 * ip + q]) / mmatl[ip];
        }
    };
    std::fill(rhs.begin(), rhs.end(), 0.f);
    for (size_t ie = 0; ie < ne; ie++) {
        float dx = 0.f, dy = 0.f;
        for (int in = 0; in < 3; in++) {
            dx = dx + topol[9 * (size_t)IM(in, ie)] * G(in, ie);
            dy = dy + topol[9 * (size_t)IM(in, ie)] * G(in + 3, ie);
        }
        topel[9 * ie + 1] = dx;
        topel[9 * ie + 2] = dy;
    }
    for (size_t ie = 0; ie < ne; ie++) {
        const float coe = G(6, ie) / 6.f;
        for (int in = 0; in < 3; in++) {
            const size_t ip = IM(in, ie);
            rhs[3 * ip] = rhs[3 * ip] + topel[9 * ie + 1] * coe;
            rhs[3 * ip + 1] = rhs[3 * ip + 1] + topel[9 * ie + 2] * coe;
        }
    }
    const int r23[2] = {1, 2};
    project(2, r23);
    std::fill(rhs.begin(), rhs.end(), 0.f);
    for (size_t ie = 0; ie < ne; ie++) {
        float dxx = 0.f, dxy = 0.f, dyx = 0.f, dyy = 0.f;
        for (int in = 0; in < 3; in++) {
            const size_t ip = IM(in, ie);
            dxx = dxx + topol[9 * ip + 1] * G(in, ie);
            dxy = dxy + topol[9 * ip + 1] * G(in + 3, ie);
            dyx = dyx + topol[9 * ip + 2] * G(in, ie);
            dyy = dyy + topol[9 * ip + 2] * G(in + 3, ie);
        }
        topel[9 * ie + 3] = dxx;
        topel[9 * ie + 4] = (dxy + dyx) / 2.f;
        topel[9 * ie + 5] = dyy;
    }
    for (size_t ie = 0; ie < ne; ie++) {
        const float coe = G(6, ie) / 6.f;
        for (int in = 0; in < 3; in++) {
            const size_t ip = IM(in, ie);
            for (int q = 0; q < 3; q++) rhs[3 * ip + q] = rhs[3 * ip + q] + topel[9 * ie + 3 + q] * coe;
        }
    }
    const int r456[3] = {3, 4, 5};
    project(3, r456);
    for (size_t ip = 0; ip < np; ip++) {
        float* t = &topol[9 * ip];
        const float zx = t[1], zy = t[2], zxx = t[3], zxy = t[4], zyy = t[5];
        const float rt = sqrtf((1.f + zx * zx) + zy * zy);
        t[3] = 1.f + zx * zx; t[4] = zx * zy; t[5] = 1.f + zy * zy;
        t[6] = zxx / rt; t[7] = zxy / rt; t[8] = zyy / rt;
    }
    // get_boun_nodes_2D: element means of the nodal rows, boundary nodes, tangents
    std::fill(topel.begin(), topel.end(), 0.f);
    std::vector<long long> ltang(np, 0);
    const float c13 = 1.f / 3.f;
    std::vector<int> deg(np + 1, 0);
    for (size_t ie = 0; ie < ne; ie++)
        for (int in = 0; in < 3; in++) {
            const int in1 = (in + 1) % 3, in2 = (in + 2) % 3;
            const size_t ip = IM(in, ie);
            ltang[ip] += (long long)IM(in2, ie) - IM(in1, ie);
            for (int it = 0; it < 9; it++) topel[9 * ie + it] = topel[9 * ie + it] + c13 * topol[9 * ip + it];
            deg[ip + 1]++;
        }
    for (size_t ip = 0; ip < np; ip++) deg[ip + 1] += deg[ip];
    std::vector<int2> adj(3 * ne);
    {
        std::vector<int> fill(deg.begin(), deg.end() - 1);
        for (size_t ie = 0; ie < ne; ie++)  // element order: the reference's order of every sum over elements
            for (int in = 0; in < 3; in++) adj[fill[IM(in, ie)]++] = make_int2((int)ie, in);
    }
    std::vector<int> bnode(np, -1);
    std::vector<float2> rtang;
    for (size_t ip = 0; ip < np; ip++) {
        if (ltang[ip] == 0) continue;
        bnode[ip] = (int)rtang.size();
        float t1 = 0.f, t2 = 0.f;
        for (int q = deg[ip]; q < deg[ip + 1]; q++) {
            const int2 a = adj[q];
            t1 = t1 - G(a.y + 3, a.x) * G(6, a.x);
            t2 = t2 + G(a.y, a.x) * G(6, a.x);
        }
        rtang.push_back(make_float2(t1, t2));
    }
    for (float2& t : rtang) {
        const float amodl = sqrtf(t.x * t.x + t.y * t.y);
        if (amodl < 1.0e-06f) continue;
        t.x = t.x / amodl;
        t.y = t.y / amodl;
    }
    // bounel: sides (ip -> ip1) of no other element in reverse, element order
    std::unordered_map<long long, int> dir;
    dir.reserve(3 * ne * 2);
    auto key = [&](long long a, long long b) { return a * (long long)np + b; };
    for (size_t ie = 0; ie < ne; ie++)
        for (int in = 0; in < 3; in++) dir[key(IM(in, ie), IM((in + 1) % 3, ie))] = 1;
    std::vector<int2> side_nodes;
    std::vector<float4> side_geom;
    for (size_t ie = 0; ie < ne; ie++)
        for (int in = 0; in < 3; in++) {
            const int ip = IM(in, ie), ip1 = IM((in + 1) % 3, ie);
            if (dir.count(key(ip1, ip))) continue;
            const float x1 = coord[2 * (size_t)ip], y1 = coord[2 * (size_t)ip + 1];
            const float x2 = coord[2 * (size_t)ip1], y2 = coord[2 * (size_t)ip1 + 1];
            const float aleng = sqrtf((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
            side_nodes.push_back(make_int2(ip, ip1));
            side_geom.push_back(make_float4((y2 - y1) / aleng, -(x2 - x1) / aleng, aleng, 0.f));
        }
    std::vector<int> bptr(np + 1, 0);
    for (const int2& s : side_nodes) { bptr[s.x + 1]++; bptr[s.y + 1]++; }
    for (size_t ip = 0; ip < np; ip++) bptr[ip + 1] += bptr[ip];
    std::vector<int2> bside(std::max<size_t>(2 * side_nodes.size(), 1));
    {
        std::vector<int> fill(bptr.begin(), bptr.end() - 1);
        for (size_t b = 0; b < side_nodes.size(); b++) {  // side order
            bside[fill[side_nodes[b].x]++] = make_int2((int)b, 0);
            bside[fill[side_nodes[b].y]++] = make_int2((int)b, 1);
        }
    }
    std::vector<int> elem(3 * ne);
    for (size_t ie = 0; ie < ne; ie++)
        for (int in = 0; in < 3; in++) elem[3 * ie + in] = IM(in, ie);

    gfsph_gfl* g = new (std::nothrow) gfsph_gfl();
    if (!g) return GFSPH_ERR_HOST;
    g->P = *p;
    g->npoin = npoin; g->nelem = nelem;
    GflConst& c = g->c;
    c.cgra = k[0]; c.dens = k[1]; c.cmanning = k[2]; c.cori = k[3]; c.nfric = nfric; c.tauy0 = k[5];
    c.constK = k[6]; c.tanfi8 = k[8]; c.hfrict0 = k[9]; c.tanfi0 = k[11]; c.bfact = k[12];
    c.ntype = p->ntype; c.ngaus = p->ngaus; c.swl = p->swl; c.comp = p->comp;
    g->topol = topol;
    g->topel = topel;
    const size_t nb = std::max<size_t>(rtang.size(), 1), ns = std::max<size_t>(side_nodes.size(), 1);
    int st = 0;
    st |= dal(&g->elem, 3 * ne); st |= dal(&g->adj_ptr, np + 1); st |= dal(&g->adj, 3 * ne);
    st |= dal(&g->bside_ptr, np + 1); st |= dal(&g->bside, bside.size()); st |= dal(&g->side_nodes, ns);
    st |= dal(&g->side_geom, ns); st |= dal(&g->bnode, np); st |= dal(&g->rtang, nb);
    st |= dal(&g->geome, 7 * ne); st |= dal(&g->d_topel, 9 * ne); st |= dal(&g->d_topol, 9 * np);
    st |= dal(&g->mmatl, np); st |= dal(&g->hs_w, np); st |= dal(&g->gradhs_w, np);
    st |= dal(&g->unkno, 3 * np); st |= dal(&g->fnode, 9 * np); st |= dal(&g->gt, 9 * ne);
    st |= dal(&g->rhs1, 3 * np); st |= dal(&g->rhs0a, 3 * np); st |= dal(&g->rhs0b, 3 * np);
    if (st || cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&g->ev0) != cudaSuccess || cudaEventCreate(&g->ev1) != cudaSuccess) {
        gfl_free(g);
        delete g;
        return GFSPH_ERR_CUDA;
    }
    cudaMemcpy(g->elem, elem.data(), elem.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(g->adj_ptr, deg.data(), deg.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(g->adj, adj.data(), adj.size() * sizeof(int2), cudaMemcpyHostToDevice);
    cudaMemcpy(g->bside_ptr, bptr.data(), bptr.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(g->bside, bside.data(), bside.size() * sizeof(int2), cudaMemcpyHostToDevice);
    if (!side_nodes.empty()) {
        cudaMemcpy(g->side_nodes, side_nodes.data(), side_nodes.size() * sizeof(int2), cudaMemcpyHostToDevice);
        cudaMemcpy(g->side_geom, side_geom.data(), side_geom.size() * sizeof(float4), cudaMemcpyHostToDevice);
    }
    cudaMemcpy(g->bnode, bnode.data(), np * sizeof(int), cudaMemcpyHostToDevice);
    if (!rtang.empty()) cudaMemcpy(g->rtang, rtang.data(), rtang.size() * sizeof(float2), cudaMemcpyHostToDevice);
    cudaMemcpy(g->geome, geome.data(), geome.size() * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(g->d_topel, topel.data(), topel.size() * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(g->d_topol, topol.data(), topol.size() * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(g->mmatl, mmatl.data(), np * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemset(g->unkno, 0, 3 * np * sizeof(float));
    if (cudaGetLastError() != cudaSuccess) { gfl_free(g); delete g; return GFSPH_ERR_CUDA; }
    *out = g;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_gfl_destroy(gfsph_gfl* g) try {
    if (!g) return GFSPH_ERR_ARG;
    cudaStreamSynchronize(g->stream);
    gfl_free(g);
    delete g;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_gfl_set_state(gfsph_gfl* g, const float* unkno, double time) try {
    if (!g || !unkno) return GFSPH_ERR_ARG;
    if (cudaMemcpyAsync(g->unkno, unkno, 3 * (size_t)g->npoin * sizeof(float), cudaMemcpyHostToDevice, g->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(g->stream) != cudaSuccess)
        return GFSPH_ERR_CUDA;
    g->time = time;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_gfl_get_state(gfsph_gfl* g, float* unkno, double* time) try {
    if (!g) return GFSPH_ERR_ARG;
    if (unkno && (cudaMemcpyAsync(unkno, g->unkno, 3 * (size_t)g->npoin * sizeof(float), cudaMemcpyDeviceToHost,
                                  g->stream) != cudaSuccess ||
                  cudaStreamSynchronize(g->stream) != cudaSuccess))
        return GFSPH_ERR_CUDA;
    if (time) *time = g->time;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_gfl_set_wir(gfsph_gfl* g, const float* hs_w, const float* gradhs_w) try {
    if (!g) return GFSPH_ERR_ARG;
    if (!hs_w || !gradhs_w) { g->wir = false; return GFSPH_OK; }
    if (g->c.ntype != 2) return GFSPH_ERR_UNSUPPORTED;  // the soil raises the bed under a free surface
    const size_t np = (size_t)g->npoin;
    if (cudaMemcpyAsync(g->hs_w, hs_w, np * sizeof(float), cudaMemcpyHostToDevice, g->stream) != cudaSuccess ||
        cudaMemcpyAsync(g->gradhs_w, gradhs_w, np * sizeof(float2), cudaMemcpyHostToDevice, g->stream) != cudaSuccess ||
        cudaStreamSynchronize(g->stream) != cudaSuccess)
        return GFSPH_ERR_CUDA;
    g->wir = true;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_gfl_step(gfsph_gfl* g, int nsteps, float dt) try {
    if (!g || nsteps < 0 || !(dt > 0.f)) return GFSPH_ERR_ARG;
    GflDev d = view(g);
    const GflConst& c = g->c;
    cudaStream_t s = g->stream;
    cudaEventRecord(g->ev0, s);
    for (int k = 0; k < nsteps; k++) {
        // tanfi of frictlaws: tanfi8 + (tanfi0 - tanfi8) exp(-time/Bfact) (:3856-3860)
        float tanfi = c.tanfi8;
        if (c.bfact >= 1.e-6f)
            tanfi = c.tanfi8 + (c.tanfi0 - c.tanfi8) * (float)exp((double)(-((float)g->time / c.bfact)));
        k_gfl_nodes<<<blocks(g->npoin), kGflThreads, 0, s>>>(d, c, tanfi);
        k_gfl_elems<<<blocks(g->nelem), kGflThreads, 0, s>>>(d, c, tanfi, dt);
        k_gfl_rhs<<<blocks(g->npoin), kGflThreads, 0, s>>>(d, c, dt);
        int src = 0;
        for (int it = 2; it <= g->P.niter; it++) {
            k_gfl_mass<<<blocks(g->npoin), kGflThreads, 0, s>>>(d, src);
            src ^= 1;
        }
        k_gfl_update<<<blocks(g->npoin), kGflThreads, 0, s>>>(d, c, src);
        g->launches += 3 + (g->P.niter - 1) + 1;
        g->time = g->time + (double)dt;
    }
    cudaEventRecord(g->ev1, s);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) return GFSPH_ERR_CUDA;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, g->ev0, g->ev1) == cudaSuccess) g->last_ms = ms;
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

int gfsph_gfl_topol(gfsph_gfl* g, float* topol, float* topel) try {
    if (!g) return GFSPH_ERR_ARG;
    if (topol) std::copy(g->topol.begin(), g->topol.end(), topol);
    if (topel) std::copy(g->topel.begin(), g->topel.end(), topel);
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}

long long gfsph_gfl_launch_count(gfsph_gfl* g) { return g ? g->launches : -1; }

int gfsph_gfl_device_ms(gfsph_gfl* g, double* ms) {
    if (!g || !ms) return GFSPH_ERR_ARG;
    *ms = g->last_ms;
    return GFSPH_OK;
}

}  // extern "C"
