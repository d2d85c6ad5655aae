// Device-side arithmetic of the SPH step: the SPH kernel, the bilinear DEM
// lookup and the basal rheology.  Every expression keeps the evaluation order
// of the Fortran source it restates (cited per function) and the library is
// compiled with --fmad=false, so each FP32 operation rounds exactly as the
// reference's FP32 build does; only the neighbour sums differ (FP64 here).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace gfsph {

constexpr float kPi = 3.14159274101257324f;  // pi = 4.*atan(1.0) in default real
constexpr float kTwoThirds = (float)(2.0 / 3.0);

// x**5 as the Fortran compiler expands an integer power: x2 = x*x,
// x3 = x2*x, x5 = x3*x2.
__device__ __forceinline__ float ipow5(float x) {
    const float x2 = x * x;
    return (x2 * x) * x2;
}

// kernel_TOOLS, My_SPH_Tools_2019.f90:2062-2180 (2-D; skf 1 cubic spline,
// skf 2 Gaussian, skf 3 quintic, skf 4 Wendland C2).  Returns w and dW/dx
// for the offset (dx0, dx1) at distance r with smoothing length hs.  The
// Gaussian's exp is evaluated in FP64 and rounded once.  The quintic's
// gradient for q <= 1 is the reference's (-120 + 120 q - 50 q^2)/h^2 dx
// (:2141), which is not the derivative of its w.
template <int SKF>
__device__ __forceinline__ void sph_kernel(float r, float dx0, float dx1, float hs, float& w, float& d0, float& d1) {
    float q = r / hs;
    w = 0.f; d0 = 0.f; d1 = 0.f;
    if (SKF == 1) {
        float factor = 15.f / (((7.f * kPi) * hs) * hs);
        if (q >= 0.f && q <= 1.f) {
            w = factor * ((kTwoThirds - q * q) + ((q * q) * q) / 2.f);
            float t = (factor * (-2.f + 1.5f * q)) / (hs * hs);
            d0 = t * dx0;
            d1 = t * dx1;
        } else if (q > 1.f && q <= 2.f) {
            float u = 2.f - q;
            w = ((factor * 1.f) / 6.f) * ((u * u) * u);
            float t = ((((factor * 1.f) / 6.f) * 3.f) * (u * u)) / hs;
            d0 = -(t * (dx0 / r));
            d1 = -(t * (dx1 / r));
        }
    } else if (SKF == 2) {
        float factor = 1.f / ((hs * hs) * kPi);  // hsml**ndimn * pi**(ndimn/2.)
        if (q >= 0.f && q <= 3.f) {
            w = factor * (float)exp((double)(-(q * q)));
            d0 = w * (-(((2.f * dx0) / hs) / hs));
            d1 = w * (-(((2.f * dx1) / hs) / hs));
        }
    } else if (SKF == 3) {
        float factor = 7.f / (((478.f * kPi) * hs) * hs);
        if (q >= 0.f && q <= 1.f) {
            w = factor * ((ipow5(3.f - q) - 6.f * ipow5(2.f - q)) + 15.f * ipow5(1.f - q));
            float t = ((-120.f + 120.f * q) - 50.f * (q * q)) / (hs * hs);
            d0 = factor * (t * dx0);
            d1 = factor * (t * dx1);
        } else if (q > 1.f && q <= 2.f) {
            w = factor * (ipow5(3.f - q) - 6.f * ipow5(2.f - q));
            float a = 3.f - q, b = 2.f - q;
            float t = (factor * (-(5.f * ((a * a) * (a * a))) + 30.f * ((b * b) * (b * b)))) / hs;
            d0 = t * (dx0 / r);
            d1 = t * (dx1 / r);
        } else if (q > 2.f && q <= 3.f) {
            w = factor * ipow5(3.f - q);
            float a = 3.f - q;
            float t = (factor * (-(5.f * ((a * a) * (a * a))))) / hs;
            d0 = t * (dx0 / r);
            d1 = t * (dx1 / r);
        }
    } else {  // skf == 4
        float factor = 7.f / (((4.f * kPi) * hs) * hs);
        if (q >= 0.f && q <= 2.f) {
            float a = 1.f - q / 2.f;
            w = factor * (((a * a) * (a * a)) * (2.f * q + 1.f));
            float t = factor * (-(5.f * ((a * a) * a)));
            float s = (1.f / hs) / hs;
            d0 = t * (s * dx0);
            d1 = t * (s * dx1);
        }
    }
}

template <int SKF>
__device__ __forceinline__ float sph_kernel_w(float r, float hs) {
    float w, a, b;
    sph_kernel<SKF>(r, 0.f, 0.f, hs, w, a, b);
    return w;
}

// The same with skf known only at run time.
__device__ __forceinline__ void sph_kernel(int skf, float r, float dx0, float dx1, float hs, float& w, float& d0,
                                           float& d1) {
    switch (skf) {
    case 1: sph_kernel<1>(r, dx0, dx1, hs, w, d0, d1); break;
    case 2: sph_kernel<2>(r, dx0, dx1, hs, w, d0, d1); break;
    case 3: sph_kernel<3>(r, dx0, dx1, hs, w, d0, d1); break;
    default: sph_kernel<4>(r, dx0, dx1, hs, w, d0, d1); break;
    }
}

__device__ __forceinline__ float sph_kernel_w(int skf, float r, float hs) {
    float w, a, b;
    sph_kernel(skf, r, 0.f, 0.f, hs, w, a, b);
    return w;
}

// scale_k of grid_find (My_SPH_Tools_2019.f90:1155-1161): the support in
// units of the mean smoothing length.
template <int SKF> struct SupportScale { static constexpr int value = (SKF == 2 || SKF == 3) ? 3 : 2; };

// Neighbour test of grid_find (My_SPH_Tools_2019.f90:1010-1019):
// dr = dx*dx + dy*dy, mh = (hi+hj)/2, r = sqrt(dr), neighbour iff r < 2*mh.
struct PairGeom {
    float dx0, dx1, r, mh;
};

__device__ __forceinline__ bool pair_test(float2 xi, float2 xj, float hi, float hj, PairGeom& g) {
    g.dx0 = xi.x - xj.x;
    float dr = g.dx0 * g.dx0;
    g.dx1 = xi.y - xj.y;
    dr = dr + g.dx1 * g.dx1;
    g.mh = (hi + hj) / 2.f;
    g.r = sqrtf(dr);
    return g.r < 2.f * g.mh;
}

// The same test for a search over candidates, r < SK*mh with SK = scale_k
// (2 for skf 1 and 4, 3 for skf 2 and 3, My_SPH_Tools_2019.f90:1155-1161),
// with a cheap early reject: sqrt_rn(dr) < t implies dr < t*t in exact
// arithmetic, and dr > fl(fl(t*t) * (1 + 1e-5)) implies dr >= t*t (the two
// roundings move t*t by at most 2^-23 relative), so the reject never drops a
// pair that the exact test keeps.
template <int SK = 2>
__device__ __forceinline__ bool pair_search(float2 xi, float2 xj, float hi, float hj, PairGeom& g) {
    float d0 = xi.x - xj.x;
    float d1 = xi.y - xj.y;
    float dr = d0 * d0;
    dr = dr + d1 * d1;
    // SK*((hi+hj)/2): for SK = 2 exactly hi+hj (scaling by 2 and 1/2 is exact)
    float t = (SK == 2) ? hi + hj : (float)SK * ((hi + hj) / 2.f);
    if (dr > (t * t) * 1.00001f) return false;
    g.dx0 = d0;
    g.dx1 = d1;
    g.mh = (hi + hj) / 2.f;
    g.r = sqrtf(dr);
    return g.r < (float)SK * g.mh;
}

// Float <-> order-preserving uint, for atomicMin/atomicMax reductions.
__device__ __forceinline__ unsigned int f2o(float f) {
    unsigned int b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__host__ __device__ __forceinline__ float o2f(unsigned int o) {
#ifdef __CUDA_ARCH__
    unsigned int b = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
    return __uint_as_float(b);
#else
    unsigned int b = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
    float f;
    memcpy(&f, &b, 4);
    return f;
#endif
}

// DEM on the device: node (ix, iy) at (xmin + ix*dx, ymin + iy*dy), x fastest.
struct DemView {
    int nx, ny;
    float xmin, ymin, dx, dy, xmax, ymax;
    const float2* __restrict__ grad;  // topol(2:3,:)
    const float4* __restrict__ curvA; // topol(4:7,:)  (nfric 7 only)
    const float2* __restrict__ curvB; // topol(8:9,:)
};

// Get_Z_Topo, SPH_FEM_topo_2019.f90:2395-2491: bilinear shape functions on
// the DEM cell containing (xx, yy).  Returns Zx, Zy and, when want_curv, the
// six curvature terms topol(4..9).
__device__ __forceinline__ void dem_lookup(const DemView& d, float xx, float yy, float& zpx, float& zpy,
                                           bool want_curv, float top[6]) {
    int ipx = (int)((xx - d.xmin) / d.dx + 1.f);
    int ipy = (int)((yy - d.ymin) / d.dy + 1.f);
    ipx = min(max(ipx, 1), d.nx - 1);
    ipy = min(max(ipy, 1), d.ny - 1);
    int ip = (ipy - 1) * d.nx + (ipx - 1);
    int n1 = ip, n2 = ip + 1, n3 = ip + 1 + d.nx, n4 = n3 - 1;
    float xref = d.xmin + (float)(ipx - 1) * d.dx;
    float yref = d.ymin + (float)(ipy - 1) * d.dy;
    float xi = (xx - xref) / d.dx;
    float eta = (yy - yref) / d.dy;
    float sh1 = (1.f - xi) * (1.f - eta);
    float sh2 = xi * (1.f - eta);
    float sh3 = xi * eta;
    float sh4 = (1.f - xi) * eta;
    float2 g1 = __ldg(&d.grad[n1]), g2 = __ldg(&d.grad[n2]), g3 = __ldg(&d.grad[n3]), g4 = __ldg(&d.grad[n4]);
    zpx = ((sh1 * g1.x + sh2 * g2.x) + sh3 * g3.x) + sh4 * g4.x;
    zpy = ((sh1 * g1.y + sh2 * g2.y) + sh3 * g3.y) + sh4 * g4.y;
    if (want_curv) {
        float4 a1 = __ldg(&d.curvA[n1]), a2 = __ldg(&d.curvA[n2]), a3 = __ldg(&d.curvA[n3]), a4 = __ldg(&d.curvA[n4]);
        float2 b1 = __ldg(&d.curvB[n1]), b2 = __ldg(&d.curvB[n2]), b3 = __ldg(&d.curvB[n3]), b4 = __ldg(&d.curvB[n4]);
        top[0] = ((sh1 * a1.x + sh2 * a2.x) + sh3 * a3.x) + sh4 * a4.x;
        top[1] = ((sh1 * a1.y + sh2 * a2.y) + sh3 * a3.y) + sh4 * a4.y;
        top[2] = ((sh1 * a1.z + sh2 * a2.z) + sh3 * a3.z) + sh4 * a4.z;
        top[3] = ((sh1 * a1.w + sh2 * a2.w) + sh3 * a3.w) + sh4 * a4.w;
        top[4] = ((sh1 * b1.x + sh2 * b2.x) + sh3 * b3.x) + sh4 * b4.x;
        top[5] = ((sh1 * b1.y + sh2 * b2.y) + sh3 * b3.y) + sh4 * b4.y;
    }
}

// Constants of the basal rheology, read from const(1..110).
struct Rheo {
    float g, dens, xi, tauy0, constK, tanfi, hfrict0, comp, keros, slip, h_inf, cgra05;
    int nfric, erosion, skf, pa_sph, sle, av_vel, ic_adapt;
    // stage-dependent pressure: normalised density (nor_density) and the
    // terrain-normal gravity (ic_cosTheta = 1); either runs the staged RK45
    int nor_density, cos_theta;
    // basal pore-water pressure (icpwp = 3) and the density factor of tanfi:
    // DFs_FSs_dens_and_pwp_factors (SPH_SW_2019.f90:8959-9060) for the
    // friction, mini_DFs_dens_and_pwp_factors (:11502-11580) for the update
    int icpwp;
    float fact_dens, fact_pwp_max, fact_pwp_min, fpwp_max, fpwp_min, fpwp_min_g, bfact, alphas, alphas2;
    // mu(I) rheologies (nfric 8 and 26: b, r, n = const(3), (6), (7); nfric 27:
    // Mu2, r, I0 = const(3), (6), (7)), basal_friction_Ext_SW :9651-9668
    int muI;
    float mu_a, mu_r, mu_b;
    // Herschel-Bulkley laws (nfric 23-25, :9538-9618) with m = const(8):
    // hb_m selects nfric 23's quadratic (0: m = 1, 1: m = 2, 2: m ~ 1/3 or
    // 1/2); hb_a0 = (1/Cm) (K/tauy0)**(1/m); hb_cm = nfric 25's
    // ((2m+1)/m)**m (1 for nfric 24)
    int hb_m;
    float m_vexp, hb_a0, hb_cm;  // m_vexp = const(8) is also nfric 3's Manning n
    // erosion law const(21) (1 Hungr, 2 bed angle, 3 basal shear) and the
    // constants of laws 2 and 3; dens_bar, dens_bar_eff of
    // DFs_FSs_dens_and_pwp_factors (SPH_SW_2019.f90:8959-9060)
    int eros_law;
    float er_kc, er_xnum, er_xden;
    float dens_bar, dens_bar_eff, er_cb, er_c1, er_c2, er_tb;
    // soil and water particles (ic_ws_Interact = 1, ic_SWalg sw_alg): pairs of
    // one material only in the density, forces and av_vel; the soil-water
    // pairs push the soil by -dens_ws g m_j grad W (SPH_SW_2019.f90:8502-8521,
    // dens_ws = densw/dens :8999-9002); the water is a Manning fluid
    int ws, swalg;
    float dens_ws;
};

// x**y for a real exponent, evaluated in FP64 and rounded once.
__device__ __forceinline__ float powr(float x, float y) { return (float)pow((double)x, (double)y); }

// Locals of ExtForces_SW shared with its contained routines.
struct ExtLocal {
    float h, hu, hv, hinv, vmod, hvmod, hvmodinv, frictx, fricty, totfrict, cf5, gravx, gravy;
    float hrho;  // rho(ipoin) as ExtForces_SW reads it, before the comp clamp
    // read by erosion law 2: vxx, vyy and tanfi as the friction leaves them,
    // the slopes of Get_Z_Topo
    float vxx, vyy, tanfi, zpx, zpy;
};

// Start of the ExtForces_SW particle loop, SPH_SW_2019.f90:8564-8596.
__device__ __forceinline__ void ext_locals(const Rheo& c, float hdepth, float vx, float vy, ExtLocal& L) {
    L.hrho = hdepth;
    L.vxx = vx;  // :8566-8569
    L.vyy = vy;
    L.tanfi = 0.f;
    L.h = hdepth;
    L.hu = L.h * vx;
    L.hv = L.h * vy;
    if (L.h < c.comp) {
        L.h = c.comp;
        L.hu = 0.f; L.hv = 0.f; L.hinv = 0.f; L.vmod = 0.f; L.hvmod = 0.f; L.hvmodinv = 0.f;
    } else {
        L.hinv = 1.f / L.h;
        L.hvmod = sqrtf(L.hu * L.hu + L.hv * L.hv);
        L.vmod = L.hvmod * L.hinv;
        L.hvmodinv = (L.hvmod >= 1.e-5f) ? 1.f / L.hvmod : 0.f;
    }
}

// g / sqrt(1 + |grad Z|^2), the gravity normal to the terrain of
// ic_cosTheta = 1 (Get_Grav_Ext_SW :9264-9270, IntForces_SW :6775-6783).
// deng = (1 + Zx^2 + Zy^2)**0.5 is taken as a correctly rounded square root.
__device__ __forceinline__ float terrain_deng(float zpx, float zpy) { return sqrtf((1.f + zpx * zpx) + zpy * zpy); }

// Get_Grav_Ext_SW (SPH_SW_2019.f90:9241-9349; ic_cosTheta = 0, or 1 when
// COS) and basal_friction_Ext_SW (:9355-9828) before its reversal filter.
// With ic_cosTheta = 1 the friction's gravz (gtanfi :9706, the mu(I) Froude
// number :9658-9665) is g/deng; the Voellmy term keeps cgra = g (:9749).
// GEN = false compiles only the Bingham, frictional and mu(I) laws (nfric 4-8,
// 26, 27), the common ones, so the kernels that inline them for those runs
// stay small; GEN = true has every law.
template <bool COS = false, bool GEN = true>
__device__ __forceinline__ void grav_and_friction(const Rheo& c, const DemView& d, float xx, float yy, float vx,
                                                  float vy, float pwp, float nsoil, ExtLocal& L) {
    const bool frictional = (c.nfric >= 5 && c.nfric <= 8) || c.nfric == 26 || c.nfric == 27;
    const bool v2byr = (c.nfric == 7 || c.nfric == 8 || c.nfric == 26 || c.nfric == 27);
    float zpx, zpy, top[6];
    dem_lookup(d, xx, yy, zpx, zpy, v2byr, top);
    L.zpx = zpx;
    L.zpy = zpy;
    float gz = c.g;
    if (COS) {
        const float deng = terrain_deng(zpx, zpy);
        gz = c.g / deng;
        L.gravx = -((c.g * zpx) / deng);
        L.gravy = -((c.g * zpy) / deng);
    } else {
        L.gravx = -(c.g * zpx);
        L.gravy = -(c.g * zpy);
    }
    float hfrict = (L.h > c.hfrict0) ? L.h : c.hfrict0;
    L.frictx = 0.f; L.fricty = 0.f; L.totfrict = 0.f; L.cf5 = 0.f;
    if (c.nfric == 4) {  // Bingham regimes, :9552-9572
        float a_hat = ((6.f * c.constK) * L.hvmod) / (c.tauy0 * (hfrict * hfrict));
        if (a_hat > 50.f) {
            float cf4b = (3.f * c.constK) / c.dens;
            L.frictx = (cf4b * L.hu) / (hfrict * hfrict);
            L.fricty = (cf4b * L.hv) / (hfrict * hfrict);
        } else if (a_hat < 0.01f) {
            float cf4b = c.tauy0 / c.dens;
            L.frictx = (cf4b * L.hu) * L.hvmodinv;
            L.fricty = (cf4b * L.hv) * L.hvmodinv;
        } else {
            float a2 = 48.f, b2 = -(32.f * a_hat) - 114.f, c2 = 65.f;
            float xh = (-b2 - sqrtf(b2 * b2 - (4.f * a2) * c2)) / (2.f * a2);
            float tau0 = c.tauy0 / xh;
            float cf4b = tau0 / c.dens;
            L.frictx = (cf4b * L.hu) * L.hvmodinv;
            L.fricty = (cf4b * L.hv) * L.hvmodinv;
        }
        L.totfrict = sqrtf(L.frictx * L.frictx + L.fricty * L.fricty);
    } else if (GEN && c.nfric == 3) {  // Bingham of the eroded soil fraction nsoil, :9443-9489
        const float fsoil = 1.f - (float)exp((double)(-(c.xi * nsoil)));  // C3 = const(3)
        const float constKB = c.constK * fsoil, tauy0B = c.tauy0 * fsoil;
        const float densB = 1000.f + (c.dens - 1000.f) * nsoil;
        if (nsoil > 0.01f) {
            const float a_hat = ((6.f * constKB) * L.hvmod) / (tauy0B * (hfrict * hfrict));
            if (a_hat > 50.f) {
                const float cf4b = (3.f * constKB) / densB;
                L.frictx = (cf4b * L.hu) / (hfrict * hfrict);
                L.fricty = (cf4b * L.hv) / (hfrict * hfrict);
            } else if (a_hat < 0.01f) {
                const float cf4b = tauy0B / densB;
                L.frictx = (cf4b * L.hu) * L.hvmodinv;
                L.fricty = (cf4b * L.hv) * L.hvmodinv;
            } else {
                const float a2 = 48.f, b2 = -(32.f * a_hat) - 114.f, c2 = 65.f;
                const float xh = (-b2 - sqrtf(b2 * b2 - (4.f * a2) * c2)) / (2.f * a2);
                const float cf4b = (tauy0B / xh) / densB;
                L.frictx = (cf4b * L.hu) * L.hvmodinv;
                L.fricty = (cf4b * L.hv) * L.hvmodinv;
            }
        }
        // the Manning friction (n = const(8)) where it is larger, per component
        const float cf1 = (c.g * c.m_vexp) * c.m_vexp;
        const float p73 = powr(hfrict, 7.f / 3.f);
        const float fxx = ((cf1 * L.hu) * L.hvmod) / p73, fyy = ((cf1 * L.hv) * L.hvmod) / p73;
        if (fabsf(fxx) > fabsf(L.frictx)) L.frictx = fxx;
        if (fabsf(fyy) > fabsf(L.fricty)) L.fricty = fyy;
        L.totfrict = sqrtf(L.frictx * L.frictx + L.fricty * L.fricty);
    } else if (GEN && c.nfric == 1) {  // Newtonian turbulent (Manning n = const(3)), :9426-9430
        const float cf1 = (c.g * c.xi) * c.xi;
        const float p73 = powr(hfrict, 7.f / 3.f);
        L.frictx = ((cf1 * L.hu) * L.hvmod) / p73;
        L.fricty = ((cf1 * L.hv) * L.hvmod) / p73;
        L.totfrict = sqrtf(L.frictx * L.frictx + L.fricty * L.fricty);
    } else if (GEN && c.nfric == 2) {  // Newtonian laminar, :9431-9437
        const float cf2a = c.constK / (8.f * c.dens);
        L.frictx = (cf2a * L.hu) / (hfrict * hfrict);
        L.fricty = (cf2a * L.hv) / (hfrict * hfrict);
        L.totfrict = sqrtf(L.frictx * L.frictx + L.fricty * L.fricty);
    } else if (GEN && c.nfric == 11) {  // Bagnold, K = const(3), :9791-9796
        L.vxx = L.hu * L.hinv;
        L.vyy = L.hv * L.hinv;
        L.frictx = ((c.xi * L.vxx) * L.vmod) / (hfrict * hfrict);
        L.fricty = ((c.xi * L.vyy) * L.vmod) / (hfrict * hfrict);
        L.totfrict = sqrtf(L.frictx * L.frictx + L.fricty * L.fricty);
    } else if (GEN && c.nfric >= 23 && c.nfric <= 25) {  // Herschel-Bulkley, :9538-9618
        float tau0;
        if (c.nfric == 23) {  // exact solution, :9576-9603
            float a_hat, a2 = 48.f, b2, c2 = 65.f;
            if (c.hb_m == 2) {
                a_hat = ((4.5f * c.constK) * L.hvmod) / (c.tauy0 * (hfrict * hfrict));
            } else {
                a_hat = c.hb_a0 * (L.hvmod / (hfrict * hfrict));
            }
            if (c.hb_m == 1) {
                a2 = 10.f;
                b2 = -a_hat - 19.2188f;
                c2 = 9.1875f;
            } else {
                b2 = -(32.f * a_hat) - 114.f;
            }
            const float xh = (-b2 - sqrtf(b2 * b2 - (4.f * a2) * c2)) / (2.f * a2);
            tau0 = c.tauy0 / xh;
        } else {  // approximations, :9606-9613
            tau0 = c.constK * powr(L.vmod / hfrict, c.m_vexp);
            tau0 = c.tauy0 + tau0 * c.hb_cm;
        }
        const float cf4b = tau0 / c.dens;
        L.frictx = (cf4b * L.hu) * L.hvmodinv;
        L.fricty = (cf4b * L.hv) * L.hvmodinv;
        L.totfrict = sqrtf(L.frictx * L.frictx + L.fricty * L.fricty);
    } else if (frictional) {  // :9660-9750
        float cv2byr = 0.f;
        if (v2byr) {
            float vxx = L.hu * L.hinv, vyy = L.hv * L.hinv;
            L.vxx = vxx;
            L.vyy = vyy;
            L.vmod = sqrtf(vxx * vxx + vyy * vyy);
            if (L.vmod >= 1e-5f) {
                float cosa = vxx / L.vmod, sina = vyy / L.vmod;
                float cos2 = cosa * cosa, sin2 = sina * sina, cbs = sina * cosa;
                float xnum = (top[3] * cos2 + top[4] * cbs) + top[5] * sin2;
                float xden = (top[0] * cos2 + top[1] * cbs) + top[2] * sin2;
                float rinv = xnum / xden;
                cv2byr = (L.vmod * L.vmod) * rinv;
            }
        }
        float tanfi = c.tanfi;
        if (c.muI == 1) {  // nfric 8, 26
            float froude = L.vmod / sqrtf(gz * L.h);
            float ff = 1.f + c.mu_a * powr((froude * c.mu_r) / L.h, c.mu_b);
            tanfi = tanfi * ff;
        } else if (c.muI == 2) {  // nfric 27
            float froude = L.vmod / sqrtf(gz * L.h);
            float inert = (froude * c.mu_r) / L.h;
            tanfi = tanfi + (c.mu_a - tanfi) / (1.f + c.mu_b / inert);
        }
        if (c.icpwp != 0) {  // :9670-9688: pwp = u(ipoin) (icpwp 1) or Uaux(1,ipoin) (3), filtered, then tanfi*factpw
            float hhh = L.hrho;
            if (pwp > c.fpwp_max * hhh) pwp = c.fpwp_max * hhh;
            if (pwp < c.fpwp_min * hhh) pwp = c.fpwp_min * hhh;
            float factpw = 1.f - pwp * L.hinv;
            if (factpw < c.fact_pwp_min) factpw = c.fact_pwp_min;
            if (factpw > c.fact_pwp_max) factpw = c.fact_pwp_max;
            tanfi = tanfi * factpw;
        }
        L.tanfi = tanfi;
        float gtanfi = ((gz + cv2byr) * tanfi) * c.fact_dens;  // :9706
        if (gtanfi < 0.f) gtanfi = 0.f;
        L.cf5 = gtanfi;
        L.frictx = ((L.cf5 * L.hu) * L.hvmodinv) * L.h;
        L.fricty = ((L.cf5 * L.hv) * L.hvmodinv) * L.h;
        if (c.xi != 0.f) {
            L.vxx = vx;  // :9720-9723, 9752-9755
            L.vyy = vy;
            float vm = vx * vx + vy * vy;
            vm = (vm > 0.f) ? sqrtf(vm) : 0.f;
            L.vmod = vm;
            if (c.xi > 0.f) {
                L.frictx = L.frictx + ((c.g * L.vmod) * vx) / c.xi;
                L.fricty = L.fricty + ((c.g * L.vmod) * vy) / c.xi;
            } else {
                float constMu = -((25.f * c.xi) / 4.f);
                L.frictx = L.frictx + ((constMu * L.vmod) * vx) / (hfrict * hfrict);
                L.fricty = L.fricty + ((constMu * L.vmod) * vy) / (hfrict * hfrict);
            }
        }
        L.totfrict = sqrtf(L.frictx * L.frictx + L.fricty * L.fricty);
    }
}

// Reversal filter of basal_friction_Ext_SW, SPH_SW_2019.f90:9829-9895.
__device__ __forceinline__ void reversal_filter(const Rheo& c, float dt, float vx, float vy, float acc0, float acc1,
                                                ExtLocal& L) {
    const bool frictional = (c.nfric >= 5 && c.nfric <= 8) || c.nfric == 26 || c.nfric == 27;
    float dc0 = -(L.frictx * L.hinv), dc1 = -(L.fricty * L.hinv);
    if (L.vmod > 1.e-5f) {
        float vs0 = vx + dt * (acc0 + dc0), vs1 = vy + dt * (acc1 + dc1);
        float vdot = vs0 * vx + vs1 * vy;
        if (vdot < 0.f) {
            float vt0 = vx / L.vmod, vt1 = vy / L.vmod;
            float accT = acc0 * vt0 + acc1 * vt1;
            float decT = dc0 * vt0 + dc1 * vt1;
            if (accT * decT < 0.f) {
                dc0 = -vx / dt - acc0;
                dc1 = -vy / dt - acc1;
                L.frictx = -dc0 * L.h;
                L.fricty = -dc1 * L.h;
            }
        }
    } else {
        float accT = sqrtf(acc0 * acc0 + acc1 * acc1);
        if (accT > 1.e-5f) {
            float ctf = frictional ? L.cf5 : L.totfrict;
            L.frictx = (ctf * acc0) / accT;
            L.fricty = (ctf * acc1) / accT;
            float fricT = sqrtf(L.frictx * L.frictx + L.fricty * L.fricty);
            if (accT <= fricT) { L.frictx = acc0; L.fricty = acc1; }
        } else {
            L.frictx = 0.f; L.fricty = 0.f;
        }
        L.frictx = L.frictx * L.h;
        L.fricty = L.fricty * L.h;
    }
}

// Get_Erosion_Rate_SW, SPH_SW_2019.f90:10329-10356, with the ExtForces_SW
// locals after the basal friction: law 1 (Hungr) E = C22 h |v|; law 2
// E = C22 C23 |v| tan(theta - theta_e) where the bed slope along the flow,
// theta = atan2(-grad Z . v/|v|, 1), exceeds the equilibrium angle
// tan(theta_e) = (denss - densw) c tanfi / ((denss - densw) c + densw),
// c = (dens - densw)/(denss - densw) (er_xnum = (denss - densw) c, er_xden =
// er_xnum + densw, er_kc = C22 C23); atan2, atan and tan in FP64, rounded once.
// Law 2 is kept out of line: its FP64 atan2/atan/tan would otherwise raise the
// register count of every kernel that inlines the friction.
static __device__ __noinline__ float erosion_rate_bed_angle(float er_kc, float er_xnum, float er_xden, float vmod,
                                                            float vxx, float vyy, float zpx, float zpy, float tanfi) {
    float er = 0.f;
    if (vmod > 1.e-5f) {
        const float cosa = vxx / vmod, sina = vyy / vmod;
        const float gradzv = zpx * cosa + zpy * sina;
        const float theta = (float)atan2((double)(-gradzv), 1.0);
        const float tanthetae = (er_xnum * tanfi) / er_xden;
        const float thetae = (float)atan((double)tanthetae);
        if (theta > thetae) er = (er_kc * vmod) * (float)tan((double)(theta - thetae));
    }
    return er;
}

template <bool GEN = true>
__device__ __forceinline__ float erosion_rate(const Rheo& c, const ExtLocal& L) {
    if (!GEN || c.eros_law == 1) return (c.keros * L.h) * L.vmod;
    return erosion_rate_bed_angle(c.er_kc, c.er_xnum, c.er_xden, L.vmod, L.vxx, L.vyy, L.zpx, L.zpy, L.tanfi);
}

// Erosion law 3 (SPH_SW_2019.f90:10357-10376) with the friction after the
// reversal filter: E = C22 (Taub - Tauf) / dens_bar_eff where the basal
// shear Taub = dens_bar |frict| exceeds the bed strength Tauf = C23 +
// dens_bar_eff g h (1 - C25) C24 (er_c1 = dens_bar_eff g, er_c2 = 1 - C25).
__device__ __forceinline__ float erosion_rate_shear(const Rheo& c, const ExtLocal& L) {
    float er = 0.f;
    if (L.vmod > 1.e-5f) {
        const float taub = c.dens_bar * sqrtf(L.frictx * L.frictx + L.fricty * L.fricty);
        const float tauf = c.er_cb + ((c.er_c1 * L.h) * c.er_c2) * c.er_tb;
        if (taub > tauf && L.vmod > 1.e-3f) er = (c.keros * (taub - tauf)) / c.dens_bar_eff;
    }
    return er;
}

// External acceleration of one particle in one RK stage: ExtForces_SW(0)
// particle loop, SPH_SW_2019.f90:8532-8716 (gravity, basal friction with the
// reversal filter, Hungr erosion momentum :8664-8697).
template <bool COS = false, bool GEN = true>
__device__ __forceinline__ void ext_accel(const Rheo& c, const DemView& d, float dt, float xx, float yy, float vx,
                                          float vy, float hdepth, float pwp, float nsoil, float in0, float in1,
                                          float& ex0, float& ex1) {
    ExtLocal L;
    ext_locals(c, hdepth, vx, vy, L);
    grav_and_friction<COS, GEN>(c, d, xx, yy, vx, vy, pwp, nsoil, L);
    // erosion laws 1 and 2 read nothing that the reversal filter changes, so
    // their rate is taken here and the locals it reads need not outlive the
    // filter; law 3 reads the filtered friction
    float er = (c.erosion && !(GEN && c.eros_law == 3)) ? erosion_rate<GEN>(c, L) : 0.f;
    ex0 = 0.f + L.gravx;
    ex1 = 0.f + L.gravy;
    reversal_filter(c, dt, vx, vy, ex0 + in0, ex1 + in1, L);
    ex0 = ex0 - L.frictx / L.h;
    ex1 = ex1 - L.fricty / L.h;
    if (c.erosion) {
        if (GEN && c.eros_law == 3) er = erosion_rate_shear(c, L);
        ex0 = ex0 - ((er * vx) * L.hinv) * c.slip;
        ex1 = ex1 - ((er * vy) * L.hinv) * c.slip;
    }
}

// The same for ic_ws_Interact = 1 (no erosion, pore pressure or terrain-
// normal gravity in its scope).  ex starts from the particle's soil-water pair
// sum b (ExtForces_SW :8502-8521).  A water particle (:8600-8606) is a
// Manning fluid, nfric 1 with n = const(3) (basal_friction_Ext_SW
// :9426-9430), not frictional in the reversal filter; with ic_SWalg = 1 its
// gravity is -g (h + Zp) grad Zp / h over the soil surface Zp = Z + hs
// (Get_Grav_Ext_SW :9322-9331).
__device__ __forceinline__ void ext_accel_wir(const Rheo& c, const DemView& d, float dt, float xx, float yy, float vx,
                                              float vy, float hdepth, float in0, float in1, bool water, float zp,
                                              float2 gzp, float2 b, float& ex0, float& ex1) {
    ExtLocal L;
    ext_locals(c, hdepth, vx, vy, L);
    Rheo cw = c;
    if (water) {
        cw.nfric = 1;
        cw.muI = 0;
        cw.icpwp = 0;
    }
    float gz = c.g;
    if (water) {
        float zpx, zpy, top[6];
        dem_lookup(d, xx, yy, zpx, zpy, false, top);
        L.gravx = -(c.g * zpx);
        L.gravy = -(c.g * zpy);
        const float hfrict = (L.h > c.hfrict0) ? L.h : c.hfrict0;
        const float cf1 = (c.g * c.xi) * c.xi;  // cmanning = const(3)
        const float p73 = powr(hfrict, 7.f / 3.f);
        L.frictx = ((cf1 * L.hu) * L.hvmod) / p73;
        L.fricty = ((cf1 * L.hv) * L.hvmod) / p73;
        L.totfrict = sqrtf(L.frictx * L.frictx + L.fricty * L.fricty);
        L.cf5 = 0.f;
    } else {
        grav_and_friction<false>(c, d, xx, yy, vx, vy, 0.f, 0.f, L);
    }
    if (water && c.swalg == 1) {
        const float hhsz = hdepth + zp;
        ex0 = b.x - (gz * (hhsz * gzp.x)) / hdepth;
        ex1 = b.y - (gz * (hhsz * gzp.y)) / hdepth;
    } else {
        ex0 = b.x + L.gravx;
        ex1 = b.y + L.gravy;
    }
    reversal_filter(cw, dt, vx, vy, ex0 + in0, ex1 + in1, L);
    ex0 = ex0 - L.frictx / L.h;
    ex1 = ex1 - L.fricty / L.h;
}

// The erosion rate after the RK update (ExtForces_SW(1), :8717-8760) with
// the ExtForces locals after basal friction.  Law 3 applies the reversal
// filter first, with the last stage's total acceleration (exdvxdt + indvxdt
// as ExtForces_SW(1) finds them).
template <bool GEN = true>
__device__ __forceinline__ float erosion_rate_final(const Rheo& c, const DemView& d, float xx, float yy, float vx,
                                                    float vy, float hdepth, float pwp, float nsoil, float acc0,
                                                    float acc1, float dt) {
    ExtLocal L;
    ext_locals(c, hdepth, vx, vy, L);
    grav_and_friction<false, GEN>(c, d, xx, yy, vx, vy, pwp, nsoil, L);
    if (!GEN || c.eros_law != 3) return erosion_rate<GEN>(c, L);
    reversal_filter(c, dt, vx, vy, acc0, acc1, L);
    return erosion_rate_shear(c, L);
}

// Get_Pwp_SW with one pwp point (icpwp = 3), SPH_SW_2019.f90:11176-11371 (no
// basal flux, no DF terms): the basal pressure head relaxes exponentially
// towards the depth change of the step, dhh = Drho_RK (RK45 :918-919), then
// is bounded by the depth and by hh * alphas * fpwp_min.
__device__ __forceinline__ float pwp_update(const Rheo& c, float u, float hh, float dhh, float dt) {
    float hinv;
    if (hh < c.comp) {
        hh = c.comp;
        hinv = 1.f / c.comp;
    } else {
        hinv = 1.f / hh;
    }
    float betaw = ((c.bfact * hinv) * hinv) / c.alphas2;
    // exp in FP64 rounded once to FP32 (a correctly rounded FP32 exp in all
    // but vanishing cases): (1 - e) below cancels to a few bits when
    // betaw*dt is small, so an FP32 exp that is off by an ulp would change the
    // update by ~1e-3 relative
    float e = (float)exp((double)(-(betaw * dt)));
    u = u * e + ((dhh / dt) * (1.f - e)) / betaw;
    if (u > hh) u = hh;
    if (u < (hh * c.alphas) * c.fpwp_min_g) u = (hh * c.alphas) * c.fpwp_min_g;
    return u;
}

// The basal pore pressure of icpwp = 1, u(ipoin), integrated by the RK45
// itself: ExtForces_SW(0) (SPH_SW_2019.f90:8648-8652) gives du = -(u/dt)
// (1 - exp(-beta dt)), beta = Bfact hinv^2 / const(14)^2, with hinv of the
// ExtForces locals (0 below comp); exp in FP64, rounded once.
__device__ __forceinline__ float pwp1_rate(const Rheo& c, float hc, float u, float dt) {
    const float hinv = (hc < c.comp) ? 0.f : 1.f / hc;
    const float betaw = ((c.bfact * hinv) * hinv) / c.alphas2;
    const float e = (float)exp((double)(-(betaw * dt)));
    return -((u / dt) * (1.f - e));
}

__device__ __forceinline__ bool out_of_box(const DemView& d, float xx, float yy) {
    float a = (xx - d.xmin) * (xx - d.xmax);
    float b = (yy - d.ymin) * (yy - d.ymax);
    return (a > 0.f) || (b > 0.f);
}

}  // namespace gfsph
