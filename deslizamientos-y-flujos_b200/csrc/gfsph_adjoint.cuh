// Reverse-mode (adjoint) kernels of one SPH step, for gradients of a loss on
// the final state with respect to the rheology (tanfi = const(9), xi =
// const(3), the Bingham yield stress const(6)), the particle volumes and the
// initial positions and velocities.
//
// Scope: frictional basal friction (nfric 5/6) with Voellmy xi >= 0 or the
// Bingham law (nfric 4), no curvature, erosion or pore pressure, pa_sph 2,
// fixed hsml (sle 0) or its update hsml' = 2 sqrt(m/h) after every step
// (sle 1, h_upgrade SPH_MAIN_2019.f90:2925-2931), fixed dt, all particles
// regular (no coarse level) and inside the DEM.  The step is differentiated
// with its neighbour list held fixed (the reference freezes its pair list per
// step too); branches (reversal filter, h_inf/comp clamps) take the forward's
// decisions.  With pa_sph 2 the pressure term p/h^2 = g/2 does not depend on
// h, so the internal force depends on positions and volumes only.
//
// Every kernel is a gather over the step's neighbour table in the step's
// cell-sorted order and writes only its own particle, so no atomics are
// needed except for the two parameter sums.
#pragma once
#include "gfsph_kernels.cuh"

namespace gfsph {

// Hessian of the kernel at separation d (r = |d|, smoothing length mh):
// d(grad W)/dd = ca * dhat dhat^T + cb * I.
__device__ __forceinline__ void sph_kernel_hess(int skf, float r, float mh, float& ca, float& cb) {
    float q = r / mh;
    ca = 0.f; cb = 0.f;
    if (skf == 1) {
        float s = (15.f / (((7.f * kPi) * mh) * mh)) / (mh * mh);
        if (q <= 1.f) {
            ca = s * (1.5f * q);
            cb = s * (-2.f + 1.5f * q);
        } else if (q <= 2.f) {
            float u = 2.f - q;
            ca = s * (u + (u * u) / (2.f * q));
            cb = s * (-(u * u) / (2.f * q));
        }
    } else {
        float s = (7.f / (((4.f * kPi) * mh) * mh)) / (mh * mh);
        if (q <= 2.f) {
            float a = 1.f - q / 2.f;
            ca = s * ((7.5f * q) * (a * a));
            cb = s * (-(5.f * ((a * a) * a)));
        }
    }
}

// Derivatives of the kernel with respect to its smoothing length mh at
// separation r, with W = f(h) g(q), q = r/h, f = C/h^2 in 2-D and
// grad W = G d (d the separation vector, G = f g'(q) / (h r)):
// dW/dh = -(2 W + f q g'(q)) / h and dG/dh = -(f / (r h^2)) (q g''(q) + 3 g'(q)),
// written with g'(q)/q where r -> 0 would divide 0 by 0.
__device__ __forceinline__ void sph_kernel_dh(int skf, float r, float mh, double& dwdh, double& dgdh) {
    const double h = mh, q = (double)r / h;
    dwdh = 0.0; dgdh = 0.0;
    if (skf == 1) {
        const double f = 15.0 / (7.0 * 3.14159265358979323846 * h * h);
        if (q <= 1.0) {
            const double g = 2.0 / 3.0 - q * q + 0.5 * q * q * q, gp = -2.0 * q + 1.5 * q * q;
            dwdh = -(f / h) * (2.0 * g + q * gp);
            dgdh = -(f / (h * h * h)) * (-8.0 + 7.5 * q);
        } else if (q <= 2.0) {
            const double u = 2.0 - q, g = u * u * u / 6.0, gp = -0.5 * u * u, gpp = u;
            dwdh = -(f / h) * (2.0 * g + q * gp);
            dgdh = -(f / ((double)r * h * h)) * (q * gpp + 3.0 * gp);
        }
    } else {  // skf 4, Wendland C2
        const double f = 7.0 / (4.0 * 3.14159265358979323846 * h * h);
        if (q <= 2.0) {
            const double a = 1.0 - 0.5 * q, g = a * a * a * a * (2.0 * q + 1.0), gp = -5.0 * q * a * a * a;
            dwdh = -(f / h) * (2.0 * g + q * gp);
            dgdh = -(f / (h * h * h)) * (-20.0 * a * a * a + 7.5 * q * a * a);
        }
    }
}

// Jacobian of the bilinear slope lookup of dem_lookup: j[0] = dZx/dx,
// j[1] = dZx/dy, j[2] = dZy/dx, j[3] = dZy/dy.
__device__ __forceinline__ void dem_slope_jac(const DemView& d, float xx, float yy, float j[4]) {
    int ipx = (int)((xx - d.xmin) / d.dx + 1.f);
    int ipy = (int)((yy - d.ymin) / d.dy + 1.f);
    ipx = min(max(ipx, 1), d.nx - 1);
    ipy = min(max(ipy, 1), d.ny - 1);
    int ip = (ipy - 1) * d.nx + (ipx - 1);
    int n1 = ip, n2 = ip + 1, n3 = ip + 1 + d.nx, n4 = n3 - 1;
    float xref = d.xmin + (float)(ipx - 1) * d.dx;
    float yref = d.ymin + (float)(ipy - 1) * d.dy;
    float xi = (xx - xref) / d.dx, eta = (yy - yref) / d.dy;
    float2 g1 = d.grad[n1], g2 = d.grad[n2], g3 = d.grad[n3], g4 = d.grad[n4];
    float ax = ((1.f - eta) * (g2.x - g1.x) + eta * (g3.x - g4.x)) / d.dx;
    float ay = ((1.f - xi) * (g4.x - g1.x) + xi * (g3.x - g2.x)) / d.dy;
    float bx = ((1.f - eta) * (g2.y - g1.y) + eta * (g3.y - g4.y)) / d.dx;
    float by = ((1.f - xi) * (g4.y - g1.y) + xi * (g3.y - g2.y)) / d.dy;
    j[0] = ax; j[1] = ay; j[2] = bx; j[3] = by;
}

// Vector-Jacobian product of ext_accel (one RK stage, frictional + Voellmy):
// given lex = dL/d(ex), adds dL/d(x, y, vx, vy, hc, in, tanfi, xi).  The
// forward quantities and the reversal filter's branch are recomputed with the
// same FP32 code as the forward kernel.
struct ExtGrad {
    float x, y, vx, vy, hc, in0, in1;
    double mu, xi, tauy;
};

// Vector-Jacobian product of the Bingham friction f = frict / h of
// basal_friction_Ext_SW (nfric 4, SPH_SW_2019.f90:9552-9572) in its regime at
// (v, h), for a sliding particle (|h v| >= 1e-5, h >= comp): given lf = dL/df,
// adds dL/d(vx, vy, hc, tauy).  Regimes: a_hat = 6 K |h v| / (tauy hf^2) with
// hf = max(h, hfrict0); a_hat > 50: f = (3K/dens) v / hf^2 (viscous);
// a_hat < 0.01: f = (tauy/dens) vhat / h (plastic); otherwise
// f = tauy / (dens xh h) vhat, xh the smaller root of
// 48 x^2 - (32 a_hat + 114) x + 65 = 0.
__device__ __forceinline__ void bingham_vjp(const Rheo& c, const ExtLocal& L, float vx, float vy, float lf0, float lf1,
                                            ExtGrad& g) {
    const float h = L.h;
    const bool hf_is_h = h > c.hfrict0;
    // the regime as the forward decides it, in FP32
    const float hfr = hf_is_h ? h : c.hfrict0;
    const float a_hat = ((6.f * c.constK) * L.hvmod) / (c.tauy0 * (hfr * hfr));
    if (a_hat <= 50.f && L.hvmodinv == 0.f) return;  // the forward's friction is 0 here
    const double hd = h, vm = sqrt((double)vx * vx + (double)vy * vy);
    const double vh0 = vx / vm, vh1 = vy / vm;
    const double hf = hfr;
    const double K = c.constK, ty = c.tauy0, dens = c.dens;
    const double a = (6.0 * K * hd * vm) / (ty * hf * hf);
    const double pv = vh0 * lf0 + vh1 * lf1;  // lf . vhat
    if (a_hat > 50.f) {
        const double k = (3.0 * K / dens) / (hf * hf);
        g.vx += (float)(k * lf0);
        g.vy += (float)(k * lf1);
        if (hf_is_h) g.hc += (float)(-2.0 * k * ((double)vx * lf0 + (double)vy * lf1) / hd);
        return;
    }
    double F, dF_dv, dF_dh, dF_dty;  // f = F vhat
    if (a_hat < 0.01f) {
        F = ty / (dens * hd);
        dF_dv = 0.0;
        dF_dh = -F / hd;
        dF_dty = F / ty;
    } else {
        const double B = 32.0 * a + 114.0, sq = sqrt(B * B - 4.0 * 48.0 * 65.0);
        const double xh = (B - sq) / 96.0;
        const double dxh_da = (32.0 / 96.0) * (1.0 - B / sq);
        F = ty / (dens * xh * hd);
        const double dF_da = -F / xh * dxh_da;
        const double da_dh = hf_is_h ? -a / hd : a / hd;  // a ~ h/hf^2
        dF_dv = dF_da * (a / vm);
        dF_dh = -F / hd + dF_da * da_dh;
        dF_dty = F / ty + dF_da * (-a / ty);
    }
    // d(F vhat)/dv = (F/|v|)(I - vhat vhat^T) + vhat dF/d|v| vhat^T
    g.vx += (float)((F / vm) * (lf0 - vh0 * pv) + vh0 * dF_dv * pv);
    g.vy += (float)((F / vm) * (lf1 - vh1 * pv) + vh1 * dF_dv * pv);
    g.hc += (float)(dF_dh * pv);
    g.tauy += dF_dty * pv;
}

__device__ __forceinline__ void ext_vjp(const Rheo& c, const DemView& dem, float dt, float xx, float yy, float vx,
                                        float vy, float hc, float in0, float in1, float lex0, float lex1,
                                        ExtGrad& g) {
    ExtLocal L;
    ext_locals(c, hc, vx, vy, L);
    grav_and_friction<false, false>(c, dem, xx, yy, vx, vy, 0.f, 0.f, L);  // nfric 4-6 only here
    const float acc0 = L.gravx + in0, acc1 = L.gravy + in1;
    // branch of reversal_filter
    float dc0 = -(L.frictx * L.hinv), dc1 = -(L.fricty * L.hinv);
    int branch = 0;  // 0 sliding (friction law), 1 reversal, 2 static, 3 from rest, 4 no force
    if (L.vmod > 1.e-5f) {
        float vs0 = vx + dt * (acc0 + dc0), vs1 = vy + dt * (acc1 + dc1);
        if (vs0 * vx + vs1 * vy < 0.f) {
            float vt0 = vx / L.vmod, vt1 = vy / L.vmod;
            float accT = acc0 * vt0 + acc1 * vt1;
            float decT = dc0 * vt0 + dc1 * vt1;
            if (accT * decT < 0.f) branch = 1;
        }
    } else {
        float accT = sqrtf(acc0 * acc0 + acc1 * acc1);
        if (accT > 1.e-5f) {
            float f0 = (L.cf5 * acc0) / accT, f1 = (L.cf5 * acc1) / accT;
            branch = (accT <= sqrtf(f0 * f0 + f1 * f1)) ? 2 : 3;
        } else {
            branch = 4;
        }
    }
    float lg0 = 0.f, lg1 = 0.f;  // dL/d(gravity acceleration)
    if (branch == 1) {
        g.vx -= lex0 / dt; g.vy -= lex1 / dt;
        g.in0 -= lex0; g.in1 -= lex1;
    } else if (branch == 2) {
        g.in0 -= lex0; g.in1 -= lex1;
    } else if (branch == 3) {
        float an = sqrtf(acc0 * acc0 + acc1 * acc1);
        float ah0 = acc0 / an, ah1 = acc1 / an;
        float pd = ah0 * lex0 + ah1 * lex1;
        float t0 = (L.cf5 * (lex0 - ah0 * pd)) / an, t1 = (L.cf5 * (lex1 - ah1 * pd)) / an;
        lg0 = lex0 - t0; lg1 = lex1 - t1;
        g.in0 -= t0; g.in1 -= t1;
        if (c.nfric != 4) g.mu -= (double)(c.g * pd);  // a Bingham particle at rest has no friction (cf5 = 0)
    } else if (branch == 4) {
        lg0 = lex0; lg1 = lex1;
    } else if (c.nfric == 4) {  // sliding under the Bingham law: ex = grav - f
        lg0 = lex0; lg1 = lex1;
        bingham_vjp(c, L, vx, vy, -lex0, -lex1, g);
    } else {
        lg0 = lex0; lg1 = lex1;
        const float vm = sqrtf(vx * vx + vy * vy);
        const float vh0 = vx / vm, vh1 = vy / vm;
        const float pd = vh0 * lex0 + vh1 * lex1;
        if (L.hvmodinv != 0.f) {  // Coulomb part cf5 * v/|v|
            g.vx -= (L.cf5 * (lex0 - vh0 * pd)) / vm;
            g.vy -= (L.cf5 * (lex1 - vh1 * pd)) / vm;
            g.mu -= (double)(c.g * pd);
        }
        if (c.xi > 0.f) {  // Voellmy part g |v| v / (xi h)
            const float k = c.g / (c.xi * L.h);
            const float vd = vx * lex0 + vy * lex1;
            g.vx -= k * (vm * lex0 + vh0 * vd);
            g.vy -= k * (vm * lex1 + vh1 * vd);
            const float e = (c.g * vm * vd) / (c.xi * L.h);
            if (hc >= c.comp) g.hc += e / L.h;
            g.xi += (double)(e / c.xi);
        }
    }
    if (lg0 != 0.f || lg1 != 0.f) {
        float j[4];
        dem_slope_jac(dem, xx, yy, j);
        g.x -= c.g * (lg0 * j[0] + lg1 * j[2]);
        g.y -= c.g * (lg0 * j[1] + lg1 * j[3]);
    }
}

// Seeds the step's adjoints in sorted order from the caller-order ones:
// lx1 = dL/dx', lv2 = dL/dv'' (after XSPH), lh = dL/dh (final depth, last
// step only); clears the accumulators.
// With sle 1, lhs_o = dL/d hsml' of the next step (caller order, zero after
// the last) goes back through h_upgrade, hsml' = 2 sqrt(m/h):
// d hsml'/dh = -hsml'/(2h), d hsml'/dm = hsml'/(2m).
__global__ void k_adj_seed(const PState A, int n, const float2* lx_o, const float2* lv_o, const float* gh_o,
                           float2* lx1, float2* lv2, float* lh, double2* lxacc, double* lm, const float* lhs_o,
                           double* lhsacc) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        int o = A.id[s];
        lx1[s] = lx_o[o];
        lv2[s] = lv_o[o];
        float lhv = gh_o ? gh_o[o] : 0.f;
        double lmv = 0.0;
        if (lhs_o) {
            const double ls = lhs_o[o], hh = A.rho[s], mm = A.mass[s];
            const double hs1 = 2.0 * sqrt(mm / hh);
            lhv += (float)(-ls * hs1 / (2.0 * hh));
            lmv = ls * hs1 / (2.0 * mm);
            lhsacc[s] = 0.0;
        }
        lh[s] = lhv;
        lxacc[s] = make_double2(0.0, 0.0);
        lm[s] = lmv;
    }
}

// Adjoint of av_vel: v''_k = v'_k + eps sum_j c_kj (v'_j - v'_k),
// c_kj = 2 m_j W_kj / (h_k + h_j), W at the start-of-step geometry.
__global__ void __launch_bounds__(128) k_adj_xsph(PState A, Search Q, Rheo c, int n, const float2* velfin,
                                                  const float2* lv2, float2* lvp, float* lh, double* lm,
                                                  double2* lxacc, double* lhsacc) {
    const float eps = 0.3f;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float4 me = Q.xhm[k];
        const float2 xk = make_float2(me.x, me.y), vk = velfin[k], lk = lv2[k];
        const float hk = A.rho[k], mk = me.w;
        const int cnt = Q.ncount[k];
        double s = 0.0, a0 = 0.0, a1 = 0.0, dm = 0.0, dh = 0.0, dx0 = 0.0, dx1 = 0.0, dhs = 0.0;
        for (int q = 0; q < cnt; q++) {
            // the pair's W and grad W as the replayed step's search stored them
            const int4 e = Q.nbr[tab_base(k, Q.kcap) + (size_t)q * kTabStride];
            const int j = e.x & ~kCrossBit;
            const float w = __int_as_float(e.y), d0 = __int_as_float(e.z), d1 = __int_as_float(e.w);
            const float4 o = Q.xhm[j];
            // the pair terms in FP64: their sums over the neighbours cancel
            // strongly (antisymmetric in k, j)
            const float2 vj = velfin[j], lj = lv2[j];
            const double den = (double)hk + (double)A.rho[j], mj = o.w, wd = w;
            const double rden = 1.0 / den;
            const double ckj = (2.0 * mj * wd) * rden, cjk = (2.0 * (double)mk * wd) * rden;
            const double D0 = (double)vj.x - vk.x, D1 = (double)vj.y - vk.y;
            const double pk = lk.x * D0 + lk.y * D1;     // lambda_k . (v_j - v_k)
            const double pj = -(lj.x * D0 + lj.y * D1);  // lambda_j . (v_k - v_j)
            s += ckj;
            a0 += cjk * lj.x;
            a1 += cjk * lj.y;
            dm += (2.0 * wd * rden) * pj;
            dh -= (ckj * pk + cjk * pj) * rden;
            const double lw = (2.0 * mj * rden) * pk + (2.0 * (double)mk * rden) * pj;
            dx0 += lw * d0;
            dx1 += lw * d1;
            if (lhsacc) {  // W_kj through mh = (hs_k + hs_j)/2
                PairGeom g;
                pair_test(xk, make_float2(o.x, o.y), me.z, o.z, g);
                double dwdh, dgdh;
                sph_kernel_dh(c.skf, g.r, g.mh, dwdh, dgdh);
                dhs += 0.5 * lw * dwdh;
            }
        }
        if (lhsacc) lhsacc[k] += eps * dhs;
        lvp[k] = make_float2((float)(lk.x * (1.0 - eps * s) + eps * a0), (float)(lk.y * (1.0 - eps * s) + eps * a1));
        lh[k] += (float)(eps * dh);
        lm[k] += eps * dm;
        double2 ax = lxacc[k];
        lxacc[k] = make_double2(ax.x + eps * dx0, ax.y + eps * dx1);
    }
}

// Adjoint of the fused RK4 of k_force_rk (stages recomputed in registers):
// from dL/dx', dL/dv' to dL/dx0, dL/dv0, dL/d(internal acceleration), dL/dh
// and the parameter sums.
__global__ void __launch_bounds__(128) k_adj_rk(PState A, Search Q, const StepScalars* S, Rheo c, DemView dem, int n,
                                                const float2* lx1, const float2* lvp, float* lh, float2* lin,
                                                double2* lxacc, float2* lv0, double* lpar) {
    const float dt = S->dt_step;
    double smu = 0.0, sxi = 0.0, sty = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float2 fin = Q.indv[i];
        const float in0 = fin.x, in1 = fin.y;
        const float h = A.rho[i];
        const float hc = (h < c.h_inf) ? c.h_inf : h;
        const float2 x0 = A.pos[i], v0 = A.vel[i];
        float xs[4], ys[4], us[4], ws[4];
        float vx = v0.x, vy = v0.y, ex0 = 0.f, ex1 = 0.f;
#pragma unroll
        for (int s = 0; s < 4; s++) {
            const float f1 = (s == 0) ? 0.f : (s == 3 ? 1.f : 0.5f);
            float fdt = f1 * dt;
            float nxx = x0.x + fdt * vx, nxy = x0.y + fdt * vy;
            float nvx = v0.x + fdt * (ex0 + in0), nvy = v0.y + fdt * (ex1 + in1);
            xs[s] = nxx; ys[s] = nxy; us[s] = nvx; ws[s] = nvy;
            vx = nvx; vy = nvy;
            // the adjoint's scope (nfric 4-6, no erosion) needs only the common laws
            ext_accel<false, false>(c, dem, dt, nxx, nxy, nvx, nvy, hc, 0.f, 0.f, in0, in1, ex0, ex1);
        }
        const float2 lx = lx1[i], lv = lvp[i];
        const float dt6 = dt / 6.f;
        ExtGrad g{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.0, 0.0, 0.0};
        float lxs0[4], lxs1[4], lvs0[4], lvs1[4], lex0[4], lex1[4];
#pragma unroll
        for (int s = 0; s < 4; s++) {
            const float f2 = (s == 0 || s == 3) ? 1.f : 2.f;
            lxs0[s] = 0.f; lxs1[s] = 0.f;
            lvs0[s] = dt6 * f2 * lx.x; lvs1[s] = dt6 * f2 * lx.y;
            lex0[s] = dt6 * f2 * lv.x; lex1[s] = dt6 * f2 * lv.y;
        }
        float lx00 = lx.x, lx01 = lx.y, lv00 = lv.x, lv01 = lv.y;
        float li0 = dt * lv.x, li1 = dt * lv.y;
#pragma unroll
        for (int s = 3; s >= 0; s--) {
            g.x = 0.f; g.y = 0.f; g.vx = 0.f; g.vy = 0.f; g.in0 = 0.f; g.in1 = 0.f;
            ext_vjp(c, dem, dt, xs[s], ys[s], us[s], ws[s], hc, in0, in1, lex0[s], lex1[s], g);
            lxs0[s] += g.x; lxs1[s] += g.y;
            lvs0[s] += g.vx; lvs1[s] += g.vy;
            li0 += g.in0; li1 += g.in1;
            if (s > 0) {
                const float f1 = (s == 3) ? 1.f : 0.5f;
                lx00 += lxs0[s]; lx01 += lxs1[s];
                lvs0[s - 1] += f1 * dt * lxs0[s]; lvs1[s - 1] += f1 * dt * lxs1[s];
                lv00 += lvs0[s]; lv01 += lvs1[s];
                lex0[s - 1] += f1 * dt * lvs0[s]; lex1[s - 1] += f1 * dt * lvs1[s];
                li0 += f1 * dt * lvs0[s]; li1 += f1 * dt * lvs1[s];
            } else {
                lx00 += lxs0[0]; lx01 += lxs1[0];
                lv00 += lvs0[0]; lv01 += lvs1[0];
            }
        }
        double2 ax = lxacc[i];
        lxacc[i] = make_double2(ax.x + lx00, ax.y + lx01);
        lv0[i] = make_float2(lv00, lv01);
        lin[i] = make_float2(li0, li1);
        if (h >= c.h_inf) lh[i] += g.hc;
        smu += g.mu;
        sxi += g.xi;
        sty += g.tauy;
    }
    smu = warp_sum(smu);
    sxi = warp_sum(sxi);
    sty = warp_sum(sty);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&lpar[0], smu);
        atomicAdd(&lpar[1], sxi);
        atomicAdd(&lpar[2], sty);
    }
}

// Adjoint of the summation density h_k = W0 m_k + sum_j m_j W_kj and of the
// internal force a_k = -sum_j m_j (P_k + P_j) grad W_kj, gathered at k.
__global__ void __launch_bounds__(128) k_adj_gather(PState A, Search Q, Rheo c, int n, const float2* lin,
                                                    const float* lh, double* lm, double2* lxacc, double* lhsacc) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float4 me = Q.xhm[k];
        const float2 xk = make_float2(me.x, me.y);
        const float mk = me.w, pk = Q.pterm[k], lhk = lh[k];
        const float2 lak = lin[k];
        const int cnt = Q.ncount[k];
        const float w0 = sph_kernel_w(c.skf, 0.f, me.z);
        double dm = (double)(lhk * w0);
        double dx0 = 0.0, dx1 = 0.0;
        // the self term W(0, hs_k) m_k: dW/dh = -2 W/h
        double dhs = lhsacc ? (double)lhk * (double)mk * (-2.0 * (double)w0 / (double)me.z) : 0.0;
        for (int q = 0; q < cnt; q++) {
            // the pair's W and grad W as the replayed step's search stored them
            const int4 e = Q.nbr[tab_base(k, Q.kcap) + (size_t)q * kTabStride];
            const int j = e.x & ~kCrossBit;
            const float w = __int_as_float(e.y), d0 = __int_as_float(e.z), d1 = __int_as_float(e.w);
            const float4 o = Q.xhm[j];
            PairGeom g;
            pair_test(xk, make_float2(o.x, o.y), me.z, o.z, g);
            float ca, cb;
            sph_kernel_hess(c.skf, g.r, g.mh, ca, cb);
            // the pair terms in FP64: their sums over the neighbours cancel
            // strongly (the kernel gradient is antisymmetric in k, j)
            const double mj = o.w, pj = Q.pterm[j], lhj = lh[j];
            const float2 laj = lin[j];
            const double cp = (double)pk + pj;
            dm += lhj * (double)w + cp * ((double)laj.x * d0 + (double)laj.y * d1);
            const double fd = (double)lhk * mj + lhj * (double)mk;
            dx0 += fd * d0;
            dx1 += fd * d1;
            // (P_k + P_j) H(d_kj) (m_k lambda_j - m_j lambda_k), H = ca dhat dhat^T + cb I
            const double u0 = (double)mk * laj.x - mj * lak.x, u1 = (double)mk * laj.y - mj * lak.y;
            const double ir = 1.0 / (double)g.r;
            const double dh0 = (double)g.dx0 * ir, dh1 = (double)g.dx1 * ir;
            const double du = dh0 * u0 + dh1 * u1;
            dx0 += cp * ((double)ca * dh0 * du + (double)cb * u0);
            dx1 += cp * ((double)ca * dh1 * du + (double)cb * u1);
            if (lhsacc) {  // W_kj and grad W_kj through mh = (hs_k + hs_j)/2
                double dwdh, dgdh;
                sph_kernel_dh(c.skf, g.r, g.mh, dwdh, dgdh);
                dhs += 0.5 * dwdh * fd;
                dhs += 0.5 * cp * dgdh * ((double)g.dx0 * u0 + (double)g.dx1 * u1);
            }
        }
        if (lhsacc) lhsacc[k] += dhs;
        lm[k] += dm;
        double2 ax = lxacc[k];
        lxacc[k] = make_double2(ax.x + dx0, ax.y + dx1);
    }
}

// The step's input adjoints back to the caller's order; volumes accumulate
// over the steps.
__global__ void k_adj_scatter(const PState A, int n, const double2* lxacc, const float2* lv0, const double* lm,
                              float2* lx_o, float2* lv_o, double* lm_o, const double* lhsacc, float* lhs_o) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        int o = A.id[s];
        double2 a = lxacc[s];
        lx_o[o] = make_float2((float)a.x, (float)a.y);
        lv_o[o] = lv0[s];
        lm_o[o] += lm[s];
        if (lhsacc) lhs_o[o] = (float)lhsacc[s];
    }
}

// Puts a stored state (caller order) back into the step buffers.
__global__ void k_adj_restore(PState B, int n, const float2* x, const float2* v, const float* rho, const float* mass,
                              const float* hsml) {  // hsml: the state's own (sle 1) or the run's constant ones
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        B.pos[s] = x[s]; B.vel[s] = v[s]; B.rho[s] = rho[s]; B.mass[s] = mass[s]; B.hsml[s] = hsml[s];
        B.flag[s] = 0; B.id[s] = s; B.pwp[s] = 0.f;
    }
}

}  // namespace gfsph
