/*
 * TEST INFRASTRUCTURE ONLY — CPU oracle for the gfsph GPU step.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py (its CPU-baseline leg and
 * its reference arm) may load this library, and only as the checker or as the
 * timed CPU baseline.  The product (libgfsph.so) never links or calls it.
 *
 * What it is: a literal restatement, in C++, of the per-time-step path of
 * Geoflow-SPH (EL-BID/Deslizamientos-y-flujos, Fortran, "Codes Geoflow_SPH"),
 * following the reference's own control flow: the pair list is built once per
 * step (grid_find_NEW_tools / _tools3), then RK45 re-evaluates summation
 * density, IntForces_SW and ExtForces_SW(0) in each of its four stages,
 * recomputes the density after the final update, applies ExtForces_SW(1)
 * erosion, the basal pore-water pressure of Get_Pwp_SW (icpwp = 3),
 * h_upgrade and av_vel.  With icpwp = 1 the pore pressure u is a fifth
 * RK45 variable whose rate ExtForces_SW(0) sets.  Every floating-point
 * expression keeps the Fortran left-to-right evaluation order, without FMA
 * contraction (build with -ffp-contract=off).
 *
 * Soil and water particles (ic_ws_Interact = 1, ic_SWalg 0 or 1): the
 * material of each particle travels in bit 1 of the flag array of this
 * interface (value 2: water, itype 2), bit 0 being If_Out_Domain.  The pair
 * types of Pint_Update_SW_tools, the soil surface of Get_hs_at_w_SW at every
 * stage, the water's pressure, Manning friction and gravity, and the
 * soil-water pair terms of ExtForces_SW are restated; the sums of the soil
 * surface are A-typed like the pair sums.  A water particle on the far edge
 * of the DEM takes the last DEM cell (the reference reads past the row).
 *
 * Precision modes (template <R, A>: R = state and arithmetic, A = accumulators
 * of the pair sums and of the erosion scatter):
 *   mode 0  R=float,  A=float  : the reference as shipped (irk = k_real,
 *                                SPH_FEM_variable_types_2019.f90:14), pair sums
 *                                in pair-list order.
 *   mode 1  R=float,  A=double : the precision scheme of the GPU path
 *                                (FP32 state and per-pair terms, FP64 sums).
 *   mode 2  R=double, A=double : the reference rebuilt with irk = k_double
 *                                (:13).  Fortran literals without a kind
 *                                suffix stay default-real (single precision)
 *                                in such a build, so every such literal is
 *                                taken as its float value here (lit()).
 *
 * Parity status: UNPINNED.  The reference ships no tests, no golden vectors
 * and no expected outputs, and it cannot be compiled here (Fortran; no
 * gfortran/ifort/flang in the image).  This oracle is pinned instead by
 * known-answer tests derived from the mathematics (kernel normalisation and
 * gradient consistency, still layer on flat ground, infinite-slope Voellmy
 * terminal velocity, mass conservation, brute-force neighbour sets) in
 * tests/test_oracle_kat.py.
 *
 * Threads: built without OpenMP (the checker) every loop runs serially in
 * the order above.  The same source built with -fopenmp is a timing-only
 * variant of the CPU baseline: per-particle loops split over threads; the
 * pair list generated by ranges of cells holding equal numbers of particles
 * and concatenated in cell order (the serial list); the erosion terms of
 * each particle computed in parallel and added to the DEM nodes in particle
 * order (the serial sums); the pair sums accumulated per thread and added in
 * thread order, so those round differently from the checker's.
 *
 * Deviations from the literal Fortran, each one a place where the literal
 * code reads undefined or out-of-range data:
 *   - Bingham (nfric = 4): SPH_SW_2019.f90:9616-9618 overwrite the regime
 *     friction of :9552-9572 with Tau0/dens*hu/|hu|, where Tau0 is only set
 *     in the intermediate regime and is otherwise stale from a previous
 *     particle (or undefined).  The regime value of :9552-9572 is kept.
 *   - Get_Z_Topo (SPH_FEM_topo_2019.f90:2420-2432) only warns when a point
 *     maps to the last node column/row and then reads the next row; the cell
 *     index is clamped to the last cell instead.
 *   - hsml = 2*(m/h)**(1./2) and deng = (1 + Zx^2 + Zy^2)**0.5 of
 *     ic_cosTheta = 1 are evaluated with a correctly rounded sqrt.
 *   - Pair traversal order: generation order of grid_find (the linked list's
 *     order depends on the node-reuse history of earlier steps).
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/gfsph.h"

/* Forward-mode (tangent) numbers: the oracle instantiated on DualT gives the
 * exact derivative of its step along one seeded direction (the reference
 * gradient for the device adjoint).  The value is carried in T (double for
 * the FP64 step; float for the single-precision step, rounded as the FP32
 * arithmetic rounds it), the derivative always in double.  Branches follow
 * the values. */
template <class T>
struct DualT {
    T v;
    double d;
    DualT() : v(0), d(0) {}
    DualT(double a) : v((T)a), d(0) {}
    DualT(double a, double b) : v((T)a), d(b) {}
    template <class U>
    DualT(const DualT<U>& o) : v((T)o.v), d(o.d) {}
    explicit operator double() const { return (double)v; }
    explicit operator float() const { return (float)v; }
    explicit operator int() const { return (int)v; }
    explicit operator long() const { return (long)v; }
    DualT operator-() const { return DualT(-v, -d); }
    DualT& operator+=(const DualT& b) { v = v + b.v; d += b.d; return *this; }
    DualT& operator-=(const DualT& b) { v = v - b.v; d -= b.d; return *this; }
    static DualT make(T a, double b) { DualT r; r.v = a; r.d = b; return r; }
    friend DualT operator+(const DualT& a, const DualT& b) { return make(a.v + b.v, a.d + b.d); }
    friend DualT operator-(const DualT& a, const DualT& b) { return make(a.v - b.v, a.d - b.d); }
    friend DualT operator*(const DualT& a, const DualT& b) {
        return make(a.v * b.v, a.d * (double)b.v + (double)a.v * b.d);
    }
    friend DualT operator/(const DualT& a, const DualT& b) {
        T q = a.v / b.v;
        return make(q, (a.d - (double)q * b.d) / (double)b.v);
    }
    friend bool operator<(const DualT& a, const DualT& b) { return a.v < b.v; }
    friend bool operator>(const DualT& a, const DualT& b) { return a.v > b.v; }
    friend bool operator<=(const DualT& a, const DualT& b) { return a.v <= b.v; }
    friend bool operator>=(const DualT& a, const DualT& b) { return a.v >= b.v; }
    friend bool operator==(const DualT& a, const DualT& b) { return a.v == b.v; }
    friend bool operator!=(const DualT& a, const DualT& b) { return a.v != b.v; }
    /* scalars: an int or float operand joins the arithmetic in T (as in
     * float op int), a double one promotes to double (as float op double) */
#define GF_SCALAR(op)                                                                                             \
    friend DualT operator op(const DualT& a, int b) { return a op make((T)b, 0.0); }                              \
    friend DualT operator op(int b, const DualT& a) { return make((T)b, 0.0) op a; }                              \
    friend DualT operator op(const DualT& a, float b) { return a op make((T)b, 0.0); }                            \
    friend DualT operator op(float b, const DualT& a) { return make((T)b, 0.0) op a; }                            \
    friend DualT<double> operator op(const DualT& a, double b) { return DualT<double>(a) op DualT<double>(b); }     \
    friend DualT<double> operator op(double b, const DualT& a) { return DualT<double>(b) op DualT<double>(a); }
    GF_SCALAR(+) GF_SCALAR(-) GF_SCALAR(*) GF_SCALAR(/)
#undef GF_SCALAR
#define GF_SCALAR_CMP(op)                                                                   \
    friend bool operator op(const DualT& a, double b) { return (double)a.v op b; }          \
    friend bool operator op(double b, const DualT& a) { return b op (double)a.v; }
    GF_SCALAR_CMP(<) GF_SCALAR_CMP(>) GF_SCALAR_CMP(<=) GF_SCALAR_CMP(>=) GF_SCALAR_CMP(==) GF_SCALAR_CMP(!=)
#undef GF_SCALAR_CMP
};
using Dual = DualT<double>;
using DualF = DualT<float>;
/* mixed single/double operands promote to double, as float op double does */
#define GF_MIXED(op)                                                                          \
    inline Dual operator op(const DualF& a, const Dual& b) { return Dual(a) op b; }           \
    inline Dual operator op(const Dual& a, const DualF& b) { return a op Dual(b); }
GF_MIXED(+) GF_MIXED(-) GF_MIXED(*) GF_MIXED(/)
#undef GF_MIXED
#define GF_MIXED_CMP(op)                                                                      \
    inline bool operator op(const DualF& a, const Dual& b) { return (double)a.v op b.v; }     \
    inline bool operator op(const Dual& a, const DualF& b) { return a.v op (double)b.v; }
GF_MIXED_CMP(<) GF_MIXED_CMP(>) GF_MIXED_CMP(<=) GF_MIXED_CMP(>=) GF_MIXED_CMP(==) GF_MIXED_CMP(!=)
#undef GF_MIXED_CMP
namespace std {
template <class T>
inline DualT<T> sqrt(const DualT<T>& x) {
    T r = std::sqrt(x.v);
    return DualT<T>::make(r, r > 0 ? x.d / (2.0 * (double)r) : 0.0);
}
inline Dual exp(const Dual& x) {
    double e = std::exp(x.v);
    return Dual(e, e * x.d);
}
template <class T>
inline DualT<T> atan2(const DualT<T>& y, const DualT<T>& x) {
    double xv = x.v, yv = y.v, q = xv * xv + yv * yv;
    return DualT<T>::make(std::atan2(y.v, x.v), q > 0 ? (xv * y.d - yv * x.d) / q : 0.0);
}
template <class T>
inline DualT<T> cos(const DualT<T>& x) { return DualT<T>::make(std::cos(x.v), -std::sin((double)x.v) * x.d); }
template <class T>
inline DualT<T> sin(const DualT<T>& x) { return DualT<T>::make(std::sin(x.v), std::cos((double)x.v) * x.d); }
template <class T>
inline DualT<T> fabs(const DualT<T>& x) { return x.v < 0 ? -x : x; }
}  // namespace std

namespace {

/* default-real literal: the value a Fortran constant like 0.3 or 2./3. has */
template <class R> inline R lit(double v) { return (R)(float)v; }

template <class R> inline R fpi() { return (R)(4.0f * atanf(1.0f)); } /* pi = 4.*atan(1.0) */

template <class R> inline R rmax(R a, R b) { return (a > b) ? a : b; } /* MAX(a,b) */
template <class R> inline R rmin(R a, R b) { return (a < b) ? a : b; }

/* exp of a default real, evaluated in FP64 and rounded once */
inline float rexp(float x) { return (float)std::exp((double)x); }
inline double rexp(double x) { return std::exp(x); }
inline Dual rexp(const Dual& x) { return std::exp(x); }
inline DualF rexp(const DualF& x) {
    double e = std::exp((double)x.v);
    return DualF::make((float)e, e * x.d);
}

/* x**5 with an integer exponent as the Fortran compiler expands it:
 * x2 = x*x, x3 = x2*x, x5 = x3*x2 */
template <class R> inline R ipow5(R x) { R x2 = x * x; return (x2 * x) * x2; }

/* kernel_TOOLS, My_SPH_Tools_2019.f90:2062-2180, 2-D, skf 1 to 4.  The
 * quintic's gradient for q <= 1 is the reference's (-120 + 120 q - 50 q**2)
 * / h**2 dx (:2141) as written (not the derivative of its w). */
template <class R>
inline void kernel_tools(int skf, R r, R dx0, R dx1, R hs, R& w, R& d0, R& d1) {
    const R pi = fpi<R>();
    R q = r / hs;
    w = 0; d0 = 0; d1 = 0;
    if (skf == 1) {
        R factor = (R)15 / ((((R)7 * pi) * hs) * hs);                 /* :2089 */
        if (q >= 0 && q <= 1) {                                           /* :2095-2099 */
            w = factor * (((lit<R>(2.0 / 3.0) - q * q) + ((q * q) * q) / (R)2));
            R t = (factor * ((R)-2 + (R)1.5 * q)) / (hs * hs);
            d0 = t * dx0;
            d1 = t * dx1;
        } else if (q > 1 && q <= 2) {                                     /* :2100-2104 */
            R u = (R)2 - q;
            w = ((factor * (R)1) / (R)6) * ((u * u) * u);
            R t = ((((factor * (R)1) / (R)6) * (R)3) * (u * u)) / hs;
            d0 = -(t * (dx0 / r));
            d1 = -(t * (dx1 / r));
        }
    } else if (skf == 2) {
        R factor = (R)1 / ((hs * hs) * pi);                              /* :2116, pi**(2/2.) = pi */
        if (q >= 0 && q <= 3) {                                           /* :2117-2122 */
            w = factor * rexp(-(q * q));
            d0 = w * (-((((R)2 * dx0) / hs) / hs));
            d1 = w * (-((((R)2 * dx1) / hs) / hs));
        }
    } else if (skf == 3) {
        R factor = (R)7 / ((((R)478 * pi) * hs) * hs);                  /* :2131 */
        if (q >= 0 && q <= 1) {                                           /* :2138-2142 */
            w = factor * ((ipow5((R)3 - q) - (R)6 * ipow5((R)2 - q)) + (R)15 * ipow5((R)1 - q));
            R t = (((R)-120 + (R)120 * q) - (R)50 * (q * q)) / (hs * hs);
            d0 = factor * (t * dx0);
            d1 = factor * (t * dx1);
        } else if (q > 1 && q <= 2) {                                     /* :2143-2147 */
            w = factor * (ipow5((R)3 - q) - (R)6 * ipow5((R)2 - q));
            R a = (R)3 - q, b = (R)2 - q;
            R t = (factor * (-((R)5 * ((a * a) * (a * a))) + (R)30 * ((b * b) * (b * b)))) / hs;
            d0 = t * (dx0 / r);
            d1 = t * (dx1 / r);
        } else if (q > 2 && q <= 3) {                                     /* :2148-2152 */
            w = factor * ipow5((R)3 - q);
            R a = (R)3 - q;
            R t = (factor * (-((R)5 * ((a * a) * (a * a))))) / hs;
            d0 = t * (dx0 / r);
            d1 = t * (dx1 / r);
        }
    } else if (skf == 4) {
        R factor = (R)7 / ((((R)4 * pi) * hs) * hs);                    /* :2164 */
        if (q >= 0 && q <= 2) {                                           /* :2169-2174 */
            R a = (R)1 - q / (R)2;
            w = factor * (((a * a) * (a * a)) * ((R)2 * q + (R)1));
            R t = factor * (-((R)5 * ((a * a) * a)));
            R s = ((R)1 / hs) / hs;
            d0 = t * (s * dx0);
            d1 = t * (s * dx1);
        }
    }
}

template <class R> inline R self_density_w(int skf, R hs) {
    R w, a, b;
    kernel_tools<R>(skf, (R)0, (R)0, (R)0, hs, w, a, b);
    return w;
}

struct Pair { int i, j; };

template <class R, class A>
struct Oracle {
    /* options */
    const gfsph_params* P;
    R cst[GFSPH_NCONST + 1]; /* 1-based like const(k) */
    int nfric = 0, ic_erosion = 0, eros_law = 0, ic_costheta = 0;
    /* DEM */
    int nx, ny, npoig;
    R xming, yming, dxg, dyg, xmaxg, ymaxg;
    std::vector<R> topol; /* (16, npoig) column-major, like topol(16,npoig) */
    /* particles */
    int n;
    std::vector<R> x, v, rho, mass, hsml, x0, v0, p;
    std::vector<R> mass0; /* mass at the start of the run (Input_SW SPH_SW_2019.f90:1995), nfric 3 */
    /* mode 3 (a precision experiment, not the reference): the RK45 position
     * updates carried in FP64 (xd), everything else as in mode 1; x holds
     * the single-precision positions that every other term reads */
    bool pos64 = false;
    std::vector<double> xd, x0d;
    std::vector<R> uaux, rho0; /* basal pore-water pressure u (icpwp 1) or Uaux(1,:) (3); rho at the RK45 start */
    std::vector<R> u0, du1, Du; /* icpwp 1: u at the RK45 start, du of the last stage, Du_RK */
    /* pore-water-pressure and density factors: DFs_FSs_dens_and_pwp_factors
     * (ExtForces_SW, SPH_SW_2019.f90:8959-9109) for the friction, and
     * mini_DFs_dens_and_pwp_factors (Get_Pwp_SW, :11502-11632) for the update */
    int icpwp;
    R fact_dens, fact_pwp_max, fact_pwp_min, fpwp_max, fpwp_min, fpwp_min_g, bfact, alphas, alphas2;
    R dens_bar, dens_bar_eff; /* of DFs_FSs_dens_and_pwp_factors, read by erosion law 3 */
    std::vector<R> ex, in, Dx, Dv, av;
    std::vector<int> flag;
    /* pairs */
    std::vector<Pair> pairs;
    std::vector<R> pw, pd0, pd1;
    /* OpenMP build only: per-range pair lists and per-thread partial sums,
     * kept between steps so that their storage is reused */
    std::vector<std::vector<Pair>> rp;
    std::vector<std::vector<R>> rw, r0, r1;
    std::vector<A> part;
    R dt;
    double time;
    std::vector<A> auxv1, auxv2; /* erosion scatter, ExtForces_SW(1) */
    /* soil and water particles (ic_ws_Interact = 1): itype 1 soil, 2 water;
     * the pair types of Pint_Update_SW_tools (0 same material, 1 soil-water);
     * Z + hs at the DEM nodes and, at the water particles, its value and
     * gradient (Get_hs_at_w_SW) */
    int ws = 0, swalg = 0;
    std::vector<int> itype;
    std::vector<char> ptype;
    std::vector<R> hsz, zpw, gzw;

    /* the flag array of the interface: bit 0 out of the domain, bit 1 water */
    void set_flags(const int* f) {
        flag.resize(n);
        itype.resize(n);
        for (int i = 0; i < n; i++) {
            flag[i] = f[i] & 1;
            itype[i] = (f[i] & 2) ? 2 : 1;
        }
    }
    int out_flag(int i) const { return flag[i] | (itype[i] == 2 ? 2 : 0); }
    bool cross(size_t k) const { return ws && ptype[k]; }

    R& T(int k, int ip) { return topol[(size_t)ip * GFSPH_NTOPO + (k - 1)]; }
    R coorgx(int ix) { return xming + (R)ix * dxg; } /* 0-based ix */
    R coorgy(int iy) { return yming + (R)iy * dyg; }

    /* Check_Out_Domain, SPH_MAIN_2019.f90:1764-1788 */
    void check_out_domain() {
        for (int i = 0; i < n; i++) {
            R d0 = (x[2 * i] - xming) * (x[2 * i] - xmaxg);
            if (d0 > 0) flag[i] = 1;
            R d1 = (x[2 * i + 1] - yming) * (x[2 * i + 1] - ymaxg);
            if (d1 > 0) flag[i] = 1;
        }
    }

    /* Adaptive_dt_sph_SW, SPH_SW_2019.f90:6521-6664 (modes 0, 1, 2, 4, 10).
     * Modes 1, 2 and 10 clamp the depth to h_inf in place; mode 4 does not.
     * dxg_mod = (dx^2 + dy^2)**0.5 is taken as a square root. */
    void adaptive_dt() {
        R dtmin = lit<R>(1.e10);
        R cgra = cst[1];
        const int mode = P->ic_adapt;
        const R dxg_mod = std::sqrt(dxg * dxg + dyg * dyg);
        if (mode == 1 || mode == 2 || mode == 4 || mode == 10) {
            for (int i = 0; i < n; i++) {
                if (flag[i]) continue;
                R vv = 0;
                if (mode != 1) vv = std::sqrt(v[2 * i] * v[2 * i] + v[2 * i + 1] * v[2 * i + 1]);
                if (mode != 4) {
                    if (rho[i] < (R)P->h_inf) rho[i] = (R)P->h_inf;
                    R c = std::sqrt(cgra * rho[i]);
                    R cc = rmax<R>(lit<R>(1.e-6), c);
                    if (mode == 2) cc = cc + vv;
                    cc = hsml[i] / ((R)3 * cc);
                    dtmin = rmin<R>(cc, dtmin);
                }
                if (mode == 4 || mode == 10) {
                    R cc = dxg_mod / vv;  /* +inf for a particle at rest */
                    dtmin = rmin<R>(cc, dtmin);
                }
            }
        }
        if (dtmin < dt) dt = dtmin;
        else if (P->ic_adapt != 0) dt = rmin<R>(lit<R>(1.1) * dt, dtmin);
    }

    /* grid_find_NEW_tools (nnps=2, My_SPH_Tools_2019.f90:1109-1370) and
     * grid_find_NEW_tools3 (nnps=4, :802-1104): counting sort into cells of
     * size 2*max(hsml), half-stencil pair enumeration, r < scale_k*(hi+hj)/2. */
    void grid_find() {
        pairs.clear(); pw.clear(); pd0.clear(); pd1.clear();
        if (!any_active()) return;  /* no pairs (and no cell size) without a particle in the box */
        std::vector<R> xr(2 * (size_t)n);
        if (P->nnps == 4) {
            R xg0 = 0, xg1 = 0; int cnt = 0;
            for (int i = 0; i < n; i++) {
                if (flag[i]) continue;
                cnt++; xg0 = xg0 + x[2 * i]; xg1 = xg1 + x[2 * i + 1];
            }
            if (cnt == 0) return;
            xg0 = xg0 / (R)cnt; xg1 = xg1 / (R)cnt;
            R ixx = 0, ixy = 0, iyy = 0;
            for (int i = 0; i < n; i++) {
                if (flag[i]) continue;
                R a = x[2 * i] - xg0, b = x[2 * i + 1] - xg1;
                ixx = ixx + b * b; ixy = ixy + a * b; iyy = iyy + a * a;
            }
            R th = -(lit<R>(0.5) * std::atan2((R)2 * ixy, iyy - ixx));
            R c = std::cos(th), s = std::sin(th);
            for (int i = 0; i < n; i++) {
                if (flag[i]) continue;
                R a = x[2 * i] - xg0, b = x[2 * i + 1] - xg1;
                xr[2 * i] = c * a + s * b;
                xr[2 * i + 1] = -s * a + c * b;
            }
        } else {
            xr = x;
        }
        R xmin[2] = {lit<R>(1.e10), lit<R>(1.e10)}, xmax[2] = {-lit<R>(1.e10), -lit<R>(1.e10)};
        R deltx[2] = {0, 0};
        int ndiv[2] = {1, 1};
        for (int d = 0; d < 2; d++) {
            for (int i = 0; i < n; i++) {
                if (flag[i]) continue;
                if (xr[2 * i + d] < xmin[d]) xmin[d] = xr[2 * i + d];
                if (xr[2 * i + d] > xmax[d]) xmax[d] = xr[2 * i + d];
                if (deltx[d] < hsml[i]) deltx[d] = hsml[i];
            }
            deltx[d] = deltx[d] * (R)2;
            R length = xmax[d] - xmin[d];
            ndiv[d] = (int)(length / deltx[d] + (R)1);
            R length_new = (R)ndiv[d] * deltx[d];
            xmin[d] = (xmin[d] - (length_new - length) / (R)2) - lit<R>(0.001) * length;
        }
        long ndivt = (long)ndiv[0] * ndiv[1];
        std::vector<int> cell(n, -1), cnt(ndivt + 1, 0), start(ndivt + 1, 0), list(n);
        for (int i = 0; i < n; i++) {
            if (flag[i]) continue;
            int id[2];
            for (int d = 0; d < 2; d++) {
                id[d] = (int)((xr[2 * i + d] - xmin[d]) / deltx[d] + (R)1);
                if (id[d] > ndiv[d]) id[d] = ndiv[d];
            }
            long c = (long)ndiv[0] * (id[1] - 1) + (id[0] - 1);
            cell[i] = (int)c;
            cnt[c]++;
        }
        for (long c = 0, s = 0; c < ndivt; c++) { start[c] = (int)s; s += cnt[c]; }
        std::vector<int> fill(ndivt, 0);
        for (int i = 0; i < n; i++) {
            if (flag[i]) continue;
            list[start[cell[i]] + fill[cell[i]]++] = i;
        }
        const int scale_k = (P->skf == 2 || P->skf == 3) ? 3 : 2; /* :1155-1161 */
        /* the pairs of the particles of cell ic (row idy, column idx, 1-based)
         * with the same and the following cells of the half stencil */
        auto cell_pairs = [&](long ic, std::vector<Pair>& pp, std::vector<R>& ww, std::vector<R>& g0s,
                              std::vector<R>& g1s) {
            const int idx = (int)(ic % ndiv[0]) + 1, idy = (int)(ic / ndiv[0]) + 1;
            for (int a = 0; a < cnt[ic]; a++) {
                int it = list[start[ic] + a];
                int jx0 = std::max(1, idx - 1), jx1 = std::min(ndiv[0], idx + 1);
                int jy1 = std::min(ndiv[1], idy + 1);
                for (int jdy = idy; jdy <= jy1; jdy++)
                    for (int jdx = jx0; jdx <= jx1; jdx++) {
                        long jc = (long)ndiv[0] * (jdy - 1) + (jdx - 1);
                        if (jc < ic) continue;
                        int b0 = (jc == ic) ? a + 1 : 0;
                        for (int b = b0; b < cnt[jc]; b++) {
                            int jt = list[start[jc] + b];
                            R d0 = x[2 * it] - x[2 * jt];
                            R dr = d0 * d0;
                            R d1 = x[2 * it + 1] - x[2 * jt + 1];
                            dr = dr + d1 * d1;
                            R mh = (hsml[it] + hsml[jt]) / (R)2;
                            R r = std::sqrt(dr);
                            if (r < (R)scale_k * mh) {
                                R w, g0, g1;
                                kernel_tools<R>(P->skf, r, d0, d1, mh, w, g0, g1);
                                pp.push_back({it, jt});
                                ww.push_back(w); g0s.push_back(g0); g1s.push_back(g1);
                            }
                        }
                    }
            }
        };
        /* cells in row-major order (idy outer, idx inner), as grid_find walks them */
#ifdef _OPENMP
        const int T = omp_get_max_threads();
        if (T > 1) {
            /* contiguous cell ranges holding about the same number of
             * particles, taken by the threads in any order and concatenated
             * in range order: the same pair list as the serial walk */
            const int nch = 16 * T;
            std::vector<long> cut(nch + 1, ndivt);
            cut[0] = 0;
            const long per = ((long)start[ndivt - 1] + cnt[ndivt - 1] + nch - 1) / nch;
            for (long c = 0, k = 1; c < ndivt && k < nch; c++)
                if (start[c] + cnt[c] >= per * k) cut[k++] = c + 1;
            for (int k = 1; k <= nch; k++) cut[k] = std::max(cut[k], cut[k - 1]);
            rp.resize(nch); rw.resize(nch); r0.resize(nch); r1.resize(nch);
#pragma omp parallel for schedule(dynamic, 1)
            for (int k = 0; k < nch; k++) {
                /* filled through vectors on this thread's stack: the
                 * neighbouring ranges' vector headers share cache lines */
                std::vector<Pair> lp; std::vector<R> lw, l0, l1;
                lp.swap(rp[k]); lw.swap(rw[k]); l0.swap(r0[k]); l1.swap(r1[k]);
                lp.clear(); lw.clear(); l0.clear(); l1.clear();
                for (long ic = cut[k]; ic < cut[k + 1]; ic++) cell_pairs(ic, lp, lw, l0, l1);
                lp.swap(rp[k]); lw.swap(rw[k]); l0.swap(r0[k]); l1.swap(r1[k]);
            }
            std::vector<size_t> off(nch + 1, 0);
            for (int k = 0; k < nch; k++) off[k + 1] = off[k] + rp[k].size();
            pairs.resize(off[nch]); pw.resize(off[nch]); pd0.resize(off[nch]); pd1.resize(off[nch]);
#pragma omp parallel for schedule(dynamic, 1)
            for (int k = 0; k < nch; k++) {
                std::copy(rp[k].begin(), rp[k].end(), pairs.begin() + off[k]);
                std::copy(rw[k].begin(), rw[k].end(), pw.begin() + off[k]);
                std::copy(r0[k].begin(), r0[k].end(), pd0.begin() + off[k]);
                std::copy(r1[k].begin(), r1[k].end(), pd1.begin() + off[k]);
            }
            return;
        }
#endif
        for (long ic = 0; ic < ndivt; ic++) cell_pairs(ic, pairs, pw, pd0, pd1);
        /* Pint_Update_SW_tools (My_SPH_Tools_2019.f90:1652-1758) follows in
         * pint_update: with one material every pair is type 0 and keeps its
         * order. */
    }

    /* Accumulator view handed to a pair body: a(c, i) is the c-th sum of
     * particle i. */
    struct ArrayAcc {
        A** a;
        A& operator()(int c, int i) const { return a[c][i]; }
    };

    /* A loop over the pairs that adds pair k's terms into nc (<= 4)
     * accumulator arrays of n entries: f(k, a) adds into a(c, i) and
     * a(c, j).  Serially in pair order (the checker).  The OpenMP build
     * splits the pairs into one contiguous block per thread, each adding
     * into its own zeroed copy of the arrays, and adds the copies to the
     * arrays in thread order: the same terms, summed in another order. */
    template <class F>
    void pair_loop(int nc, A** acc, F&& f) {
#ifdef _OPENMP
        const int T = omp_get_max_threads();
        if (T > 1 && pairs.size() > 4096) {
            part.resize((size_t)T * nc * n);
#pragma omp parallel
            {
                const int t = omp_get_thread_num();
                A* mine[4];
                for (int c = 0; c < nc; c++) {
                    mine[c] = part.data() + ((size_t)t * nc + c) * n;
                    std::fill(mine[c], mine[c] + n, (A)0);
                }
                ArrayAcc own{mine};
#pragma omp barrier
#pragma omp for schedule(static)
                for (long k = 0; k < (long)pairs.size(); k++) f((size_t)k, own);
#pragma omp for schedule(static)
                for (int i = 0; i < n; i++)
                    for (int c = 0; c < nc; c++) {
                        A sacc = acc[c][i];
                        for (int u = 0; u < T; u++) sacc = sacc + part[((size_t)u * nc + c) * n + i];
                        acc[c][i] = sacc;
                    }
            }
            return;
        }
#endif
        ArrayAcc all{acc};
        for (size_t k = 0; k < pairs.size(); k++) f(k, all);
    }

    /* Pint_Update_SW_tools, My_SPH_Tools_2019.f90:1652-1710, soil (1) and
     * water (2): a pair of one material is type 0, a soil-water pair type 1,
     * ordered soil first (the gradient changes sign with the order). */
    void pint_update() {
        if (!ws) return;
        ptype.assign(pairs.size(), 0);
        for (size_t k = 0; k < pairs.size(); k++) {
            int i = pairs[k].i, j = pairs[k].j;
            if (itype[j] < itype[i]) {
                pairs[k].i = j;
                pairs[k].j = i;
                pd0[k] = -pd0[k];
                pd1[k] = -pd1[k];
            }
            ptype[k] = (itype[i] != itype[j]) ? 1 : 0;
        }
    }

    /* Get_hs_at_w_SW, SPH_SW_2019.f90:17789-17938: the soil depth spread
     * over the DEM nodes (inverse distance over the 4 x 4 nodes around each
     * soil particle; the sums in A), Z + hs per node, and at each water
     * particle its bilinear value and gradient on the particle's DEM cell.
     * A water particle on the far edge of the DEM takes the last cell. */
    void hs_at_w() {
        std::vector<A> a1((size_t)npoig, (A)0), a2((size_t)npoig, (A)0);
        for (int i = 0; i < n; i++) {
            if (flag[i] || itype[i] != 1) continue;
            R xx = x[2 * i], yy = x[2 * i + 1];
            int ipx = (int)((xx - xming) / dxg + (R)1), ipy = (int)((yy - yming) / dyg + (R)1);
            int inx0 = std::max(1, ipx - 1), iny0 = std::max(1, ipy - 1);
            int inx1 = std::min(nx, ipx + 2), iny1 = std::min(ny, ipy + 2);
            for (int inx = inx0; inx <= inx1; inx++)
                for (int iny = iny0; iny <= iny1; iny++) {
                    size_t ip = (size_t)(iny - 1) * nx + (inx - 1);
                    R dx2 = xx - coorgx(inx - 1);
                    dx2 = dx2 * dx2;
                    R dy2 = yy - coorgy(iny - 1);
                    dy2 = dy2 * dy2;
                    R dist = rmax<R>(lit<R>(1.e-6), std::sqrt(dx2 + dy2));
                    a1[ip] = a1[ip] + (A)(rho[i] / dist);
                    a2[ip] = a2[ip] + (A)((R)1 / dist);
                }
        }
        hsz.resize(npoig);
        for (int ip = 0; ip < npoig; ip++)
            hsz[ip] = (a2[ip] > (A)lit<R>(1.e-6)) ? T(1, ip) + (R)(a1[ip] / a2[ip]) : T(1, ip);
        zpw.assign(n, (R)0);
        gzw.assign(2 * (size_t)n, (R)0);
        for (int i = 0; i < n; i++) {
            if (flag[i] || itype[i] != 2) continue;
            R xx = x[2 * i], yy = x[2 * i + 1];
            int ipx = (int)((xx - xming) / dxg + (R)1), ipy = (int)((yy - yming) / dyg + (R)1);
            ipx = std::min(std::max(ipx, 1), nx - 1);
            ipy = std::min(std::max(ipy, 1), ny - 1);
            size_t n1 = (size_t)(ipy - 1) * nx + (ipx - 1), n2 = n1 + 1, n3 = n1 + 1 + nx, n4 = n3 - 1;
            R xref = xming + (R)(ipx - 1) * dxg, yref = yming + (R)(ipy - 1) * dyg;
            R xi = (xx - xref) / dxg, eta = (yy - yref) / dyg;
            R sh1 = ((R)1 - xi) * ((R)1 - eta), sh2 = xi * ((R)1 - eta), sh3 = xi * eta, sh4 = ((R)1 - xi) * eta;
            R d1x = ((R)-1 + eta) / dxg, d2x = ((R)1 - eta) / dxg, d3x = eta / dxg, d4x = (-eta) / dxg;
            R d1y = ((R)-1 + xi) / dyg, d2y = (-xi) / dyg, d3y = xi / dyg, d4y = ((R)1 - xi) / dyg;
            zpw[i] = ((sh1 * hsz[n1] + sh2 * hsz[n2]) + sh3 * hsz[n3]) + sh4 * hsz[n4];
            gzw[2 * i] = ((hsz[n1] * d1x + hsz[n2] * d2x) + hsz[n3] * d3x) + hsz[n4] * d4x;
            gzw[2 * i + 1] = ((hsz[n1] * d1y + hsz[n2] * d2y) + hsz[n3] * d3y) + hsz[n4] * d4y;
        }
    }

    /* sum_density_Tools, My_SPH_Tools_2019.f90:1763-1859.  With nor_density
     * (:1841-1846) the sum is divided by wi = W(0,h_i) m_i/rho_i +
     * sum_j (m_j/rho_j) W_ij (:1793-1810), taken with the depths of the
     * previous call (after IntForces_SW's in-place h_inf clamp). */
    void sum_density() {
        std::vector<A> acc(n), wi;
        const bool nor = P->nor_density != 0;
        if (nor) wi.assign(n, (A)0);
        for (int i = 0; i < n; i++) {
            if (flag[i]) { acc[i] = (A)rho[i]; continue; }
            R sd = self_density_w<R>(P->skf, hsml[i]);
            if (nor) wi[i] = (A)((sd * mass[i]) / rho[i]);
            acc[i] = (A)(sd * mass[i]);
        }
        if (nor) {
            A* arr[1] = {wi.data()};
            pair_loop(1, arr, [&](size_t k, auto& a) {
                int i = pairs[k].i, j = pairs[k].j;
                a(0, i) = a(0, i) + (A)((mass[j] / rho[j]) * pw[k]);
                a(0, j) = a(0, j) + (A)((mass[i] / rho[i]) * pw[k]);
            });
        }
        {
            A* arr[1] = {acc.data()};
            pair_loop(1, arr, [&](size_t k, auto& a) {
                if (cross(k)) return; /* type 0 only, :1829 */
                int i = pairs[k].i, j = pairs[k].j;
                a(0, i) = a(0, i) + (A)(mass[j] * pw[k]);
                a(0, j) = a(0, j) + (A)(mass[i] * pw[k]);
            });
        }
        for (int i = 0; i < n; i++) rho[i] = (R)acc[i];
        if (nor)
            for (int i = 0; i < n; i++) {
                if (flag[i]) continue;
                rho[i] = rho[i] / (R)wi[i];
            }
    }

    /* deng = (1 + Zx^2 + Zy^2)**0.5 of ic_cosTheta = 1 (taken as a square root) */
    R terrain_deng(R zpx, R zpy) { return std::sqrt(((R)1 + zpx * zpx) + zpy * zpy); }

    /* IntForces_SW, SPH_SW_2019.f90:6669-6941 (ic_ws_Interact = 0, ic_SWalg = 0,
     * no K0, no end-solid law).  ic_cosTheta = 1 (:6775-6783): the pressure
     * of each particle takes g/deng at its current position. */
    void int_forces() {
        R cgra05 = cst[1] * lit<R>(0.5); /* gravz*0.5, gravz = const(1) */
        if (ws) hs_at_w(); /* :6763-6764, before the clamp */
        for (int i = 0; i < n; i++)
            if (rho[i] < (R)P->h_inf) rho[i] = (R)P->h_inf; /* :6769 */
        for (int i = 0; i < n; i++) {
            if (flag[i]) continue;
            if (ic_costheta == 1) {
                R zp, zpx, zpy, top[6];
                get_z_topo(x[2 * i], x[2 * i + 1], zp, zpx, zpy, top, false);
                R gravz = cst[1] / terrain_deng(zpx, zpy);
                cgra05 = lit<R>(0.5) * gravz;
            }
            if (ws && swalg == 1 && itype[i] == 2) { /* water over the soil surface, :6819-6826 */
                R zp = zpw[i];
                p[i] = cgra05 * (rho[i] * rho[i] - zp * zp);
            } else {
                p[i] = (cgra05 * rho[i]) * rho[i]; /* :6797 */
            }
        }
        std::vector<A> a0(n, (A)0), a1(n, (A)0);
        A* arr[2] = {a0.data(), a1.data()};
        pair_loop(2, arr, [&](size_t k, auto& a) {
            if (cross(k)) return; /* type 0 only, :6899 */
            int i = pairs[k].i, j = pairs[k].j;
            R mi = mass[i], mj = mass[j];
            R g[2] = {pd0[k], pd1[k]};
            for (int d = 0; d < 2; d++) {
                R h;
                if (P->pa_sph == 1) { /* :6905-6912 */
                    R rij = (R)1 / (rho[i] * rho[j]);
                    h = -(p[i] + p[j]) * g[d];
                    h = h * rij;
                } else { /* :6914-6920 */
                    h = -(p[i] / (rho[i] * rho[i]) + p[j] / (rho[j] * rho[j])) * g[d];
                }
                a(d, i) = a(d, i) + (A)(mj * h);
                a(d, j) = a(d, j) - (A)(mi * h);
            }
        });
        for (int i = 0; i < n; i++) { in[2 * i] = (R)a0[i]; in[2 * i + 1] = (R)a1[i]; }
    }

    /* Get_Z_Topo, SPH_FEM_topo_2019.f90:2395-2491: bilinear shape functions
     * on the DEM cell; all nodes inside the model (kpoin = 4). */
    void get_z_topo(R xx, R yy, R& zp, R& zpx, R& zpy, R top[6], bool want_top) {
        int ipx = (int)((xx - xming) / dxg + (R)1);
        int ipy = (int)((yy - yming) / dyg + (R)1);
        if (ipx >= nx) ipx = nx - 1;
        if (ipy >= ny) ipy = ny - 1;
        if (ipx < 1) ipx = 1;
        if (ipy < 1) ipy = 1;
        int ip = (ipy - 1) * nx + (ipx - 1);
        int n1 = ip, n2 = ip + 1, n3 = ip + 1 + nx, n4 = n3 - 1;
        R xref = xming + (R)(ipx - 1) * dxg;
        R yref = yming + (R)(ipy - 1) * dyg;
        R xi = (xx - xref) / dxg;
        R eta = (yy - yref) / dyg;
        R sh1 = ((R)1 - xi) * ((R)1 - eta);
        R sh2 = xi * ((R)1 - eta);
        R sh3 = xi * eta;
        R sh4 = ((R)1 - xi) * eta;
        auto interp = [&](int k) {
            return ((sh1 * T(k, n1) + sh2 * T(k, n2)) + sh3 * T(k, n3)) + sh4 * T(k, n4);
        };
        zp = interp(1);
        zpx = interp(2);
        zpy = interp(3);
        if (want_top)
            for (int k = 0; k < 6; k++) top[k] = interp(4 + k);
    }

    struct Local { /* ExtForces_SW locals shared with its contained routines */
        R h, hu, hv, hinv, vmod, hvmod, hvmodinv, frictx, fricty, totfrict, cf5, gravx, gravy, gravz;
        R hrho; /* rho(ipoin) as ExtForces_SW reads it, before the comp clamp */
        /* read by erosion law 2: vxx, vyy and tanfi as the friction leaves
           them, the slopes of Get_Z_Topo */
        R vxx, vyy, tanfi, zpx, zpy;
    };

    /* the start of the ExtForces_SW particle loop, SPH_SW_2019.f90:8564-8596 */
    void ext_locals(int i, R hdepth, Local& L) {
        L.hrho = hdepth;
        L.vxx = v[2 * i]; /* :8566-8569 */
        L.vyy = v[2 * i + 1];
        L.tanfi = 0;
        L.h = hdepth;
        L.hu = L.h * v[2 * i];
        L.hv = L.h * v[2 * i + 1];
        if (L.h < cst[15]) {
            L.h = cst[15];
            L.hu = 0; L.hv = 0; L.hinv = 0; L.vmod = 0; L.hvmod = 0; L.hvmodinv = 0;
        } else {
            L.hinv = (R)1 / L.h;
            L.hvmod = std::sqrt(L.hu * L.hu + L.hv * L.hv);
            L.vmod = L.hvmod * L.hinv;
            L.hvmodinv = (L.hvmod >= lit<R>(1.e-5)) ? (R)1 / L.hvmod : (R)0;
        }
    }

    /* Get_Grav_Ext_SW (SPH_SW_2019.f90:9241-9349, ic_cosTheta = 0) followed by
     * basal_friction_Ext_SW (:9355-9901) up to, not including, its reversal
     * filter.  Returns via L the friction and the (possibly recomputed) vmod. */
    void grav_and_friction(int i, Local& L, R top[6], int nfric) {
        R cgra = cst[1];
        bool frictional = (nfric >= 5 && nfric <= 8) || nfric == 26 || nfric == 27;
        bool v2byr = (nfric == 7 || nfric == 8 || nfric == 26 || nfric == 27);
        R zp, zpx, zpy;
        get_z_topo(x[2 * i], x[2 * i + 1], zp, zpx, zpy, top, v2byr);
        L.zpx = zpx;
        L.zpy = zpy;
        if (ic_costheta == 1) { /* :9264-9270 */
            R deng = terrain_deng(zpx, zpy);
            L.gravz = cgra / deng;
            L.gravx = -((cgra * zpx) / deng);
            L.gravy = -((cgra * zpy) / deng);
        } else {
            L.gravz = cgra;
            L.gravx = -(cgra * zpx);
            L.gravy = -(cgra * zpy);
        }
        R hfrict = rmax<R>(L.h, cst[10]);
        L.frictx = 0; L.fricty = 0; L.totfrict = 0; L.cf5 = 0;
        R dens = cst[2];
        if (nfric == 1) { /* Manning, :9426-9430 (also the water of ic_ws_Interact 1) */
            R cmanning = cst[3];
            R cf1 = (cgra * cmanning) * cmanning;
            R p73 = (R)std::pow((double)hfrict, (double)lit<R>(7.0 / 3.0));
            L.frictx = ((cf1 * L.hu) * L.hvmod) / p73;
            L.fricty = ((cf1 * L.hv) * L.hvmod) / p73;
            L.totfrict = std::sqrt(L.frictx * L.frictx + L.fricty * L.fricty);
        } else if (nfric == 4) { /* Bingham, :9538-9572 (regime value kept, see header) */
            R tauy0 = cst[6], constK = cst[7];
            R a_hat = (((R)6 * constK) * L.hvmod) / (tauy0 * (hfrict * hfrict));
            if (a_hat > (R)50) {
                R cf4b = ((R)3 * constK) / dens;
                L.frictx = (cf4b * L.hu) / (hfrict * hfrict);
                L.fricty = (cf4b * L.hv) / (hfrict * hfrict);
            } else if (a_hat < lit<R>(0.01)) {
                R cf4b = tauy0 / dens;
                L.frictx = (cf4b * L.hu) * L.hvmodinv;
                L.fricty = (cf4b * L.hv) * L.hvmodinv;
            } else {
                R a2 = (R)48, b2 = -((R)32 * a_hat) - (R)114, c2 = (R)65;
                R xh = (-b2 - std::sqrt(b2 * b2 - ((R)4 * a2) * c2)) / ((R)2 * a2);
                R tau0 = tauy0 / xh;
                R cf4b = tau0 / dens;
                L.frictx = (cf4b * L.hu) * L.hvmodinv;
                L.fricty = (cf4b * L.hv) * L.hvmodinv;
            }
            L.totfrict = std::sqrt(L.frictx * L.frictx + L.fricty * L.fricty);
        } else if (nfric == 3) { /* Bingham of the eroded soil fraction, :9443-9489 */
            /* nsoilB = (m - m0)/m, the share of the mass gained by erosion
               (setup refuses masses <= 1e-6, where the reference stops) */
            R nsoil = (mass[i] - mass0[i]) / mass[i];
            R fsoil = (R)1 - rexp(-(cst[3] * nsoil));
            R constKB = cst[7] * fsoil, tauy0B = cst[6] * fsoil;
            R densB = (R)1000 + (dens - (R)1000) * nsoil;
            if (nsoil > lit<R>(0.01)) {
                R a_hat = (((R)6 * constKB) * L.hvmod) / (tauy0B * (hfrict * hfrict));
                if (a_hat > (R)50) {
                    R cf4b = ((R)3 * constKB) / densB;
                    L.frictx = (cf4b * L.hu) / (hfrict * hfrict);
                    L.fricty = (cf4b * L.hv) / (hfrict * hfrict);
                } else if (a_hat < lit<R>(0.01)) {
                    R cf4b = tauy0B / densB;
                    L.frictx = (cf4b * L.hu) * L.hvmodinv;
                    L.fricty = (cf4b * L.hv) * L.hvmodinv;
                } else {
                    R a2 = (R)48, b2 = -((R)32 * a_hat) - (R)114, c2 = (R)65;
                    R xh = (-b2 - std::sqrt(b2 * b2 - ((R)4 * a2) * c2)) / ((R)2 * a2);
                    R cf4b = (tauy0B / xh) / densB;
                    L.frictx = (cf4b * L.hu) * L.hvmodinv;
                    L.fricty = (cf4b * L.hv) * L.hvmodinv;
                }
            }
            /* the Manning friction with n = const(8) where it is larger, per component */
            R cf1 = (cgra * cst[8]) * cst[8];
            R p73 = (R)std::pow((double)hfrict, (double)lit<R>(7.0 / 3.0));
            R fxx = ((cf1 * L.hu) * L.hvmod) / p73;
            R fyy = ((cf1 * L.hv) * L.hvmod) / p73;
            if (std::fabs(fxx) > std::fabs(L.frictx)) L.frictx = fxx;
            if (std::fabs(fyy) > std::fabs(L.fricty)) L.fricty = fyy;
            L.totfrict = std::sqrt(L.frictx * L.frictx + L.fricty * L.fricty);
        } else if (nfric == 2) { /* Newtonian laminar, :9431-9437; hfrict**2. = hfrict*hfrict */
            R cf2a = cst[7] / ((R)8 * dens);
            L.frictx = (cf2a * L.hu) / (hfrict * hfrict);
            L.fricty = (cf2a * L.hv) / (hfrict * hfrict);
            L.totfrict = std::sqrt(L.frictx * L.frictx + L.fricty * L.fricty);
        } else if (nfric == 11) { /* Bagnold with K_Bagnold = const(3), :9791-9796 */
            L.vxx = L.hu * L.hinv;
            L.vyy = L.hv * L.hinv;
            L.frictx = ((cst[3] * L.vxx) * L.vmod) / (hfrict * hfrict);
            L.fricty = ((cst[3] * L.vyy) * L.vmod) / (hfrict * hfrict);
            L.totfrict = std::sqrt(L.frictx * L.frictx + L.fricty * L.fricty);
        } else if (nfric >= 23 && nfric <= 25) { /* Herschel-Bulkley, :9538-9618 */
            R tauy0 = cst[6], constK = cst[7], m = cst[8];
            R tau0;
            if (nfric == 23) { /* :9541-9545 then :9576-9603 */
                R cm = m / ((m + (R)1) * ((R)2 * m + (R)1));
                R a_hat = ((R)1 / cm) * (R)std::pow((double)(constK / tauy0), (double)((R)1 / m));
                a_hat = a_hat * (L.hvmod / (hfrict * hfrict));
                R a2, b2, c2;
                if (m == (R)1) {
                    a2 = (R)48; b2 = -((R)32 * a_hat) - (R)114; c2 = (R)65;
                } else if (m == (R)2) {
                    a2 = (R)10; b2 = -a_hat - lit<R>(19.2188); c2 = lit<R>(9.1875);
                } else { /* m ~ 1/3 or m = 1/2 (setup refuses any other m) */
                    a_hat = ((lit<R>(4.5) * constK) * L.hvmod) / (tauy0 * (hfrict * hfrict));
                    a2 = (R)48; b2 = -((R)32 * a_hat) - (R)114; c2 = (R)65;
                }
                R xh = (-b2 - std::sqrt(b2 * b2 - ((R)4 * a2) * c2)) / ((R)2 * a2);
                tau0 = tauy0 / xh;
            } else { /* :9606-9613, constMu_CF = const(7) */
                tau0 = constK * (R)std::pow((double)(L.vmod / hfrict), (double)m);
                R cmf = (R)1;
                if (nfric == 25) cmf = (R)std::pow((double)(((R)2 * m + (R)1) / m), (double)m);
                tau0 = tauy0 + tau0 * cmf;
            }
            R cf4b = tau0 / dens; /* :9615-9618 */
            L.frictx = (cf4b * L.hu) * L.hvmodinv;
            L.fricty = (cf4b * L.hv) * L.hvmodinv;
            L.totfrict = std::sqrt(L.frictx * L.frictx + L.fricty * L.fricty);
        } else if (frictional) { /* :9660-9750 */
            R cv2byr = 0;
            if (v2byr) {
                R vxx = L.hu * L.hinv, vyy = L.hv * L.hinv;
                L.vxx = vxx;
                L.vyy = vyy;
                L.vmod = std::sqrt(vxx * vxx + vyy * vyy);
                if (L.vmod >= lit<R>(1e-5)) {
                    R cosa = vxx / L.vmod, sina = vyy / L.vmod;
                    R cos2 = cosa * cosa, sin2 = sina * sina, cbs = sina * cosa;
                    R xnum = (top[3] * cos2 + top[4] * cbs) + top[5] * sin2;
                    R xden = (top[0] * cos2 + top[1] * cbs) + top[2] * sin2;
                    R rinv = xnum / xden;
                    cv2byr = (L.vmod * L.vmod) * rinv;
                }
            }
            R tanfi = cst[9];
            R xi = cst[3];
            if (nfric == 8 || nfric == 26 || nfric == 27) { /* mu(I), :9651-9668 */
                xi = 0; /* const(3) is a mu(I) parameter here */
                R froude = L.vmod / std::sqrt(L.gravz * L.h);
                if (nfric == 27) {
                    R inert = (froude * cst[6]) / L.h;
                    tanfi = tanfi + (cst[3] - tanfi) / ((R)1 + cst[7] / inert);
                } else {
                    R ff = (R)1 + cst[3] * (R)std::pow((double)((froude * cst[6]) / L.h), (double)cst[7]);
                    tanfi = tanfi * ff;
                }
            }
            if (icpwp != 0) { /* :9670-9688: pwp = u(ipoin) (1) or Uaux(1,ipoin) (3), filtered, then tanfi*factpw */
                R pwp = uaux[i];
                R hhh = L.hrho;
                if (pwp > fpwp_max * hhh) pwp = fpwp_max * hhh;
                if (pwp < fpwp_min * hhh) pwp = fpwp_min * hhh;
                R factpw = (R)1 - pwp * L.hinv;
                if (factpw < fact_pwp_min) factpw = fact_pwp_min;
                if (factpw > fact_pwp_max) factpw = fact_pwp_max;
                tanfi = tanfi * factpw;
            }
            L.tanfi = tanfi;
            R gtanfi = ((L.gravz + cv2byr) * tanfi) * fact_dens; /* :9706 */
            if (gtanfi < 0) gtanfi = 0;
            L.cf5 = gtanfi;
            L.frictx = ((L.cf5 * L.hu) * L.hvmodinv) * L.h;
            L.fricty = ((L.cf5 * L.hv) * L.hvmodinv) * L.h;
            if (xi != 0) {
                R vxx = v[2 * i], vyy = v[2 * i + 1];
                L.vxx = vxx; /* :9720-9723, 9752-9755 */
                L.vyy = vyy;
                R vm = vxx * vxx + vyy * vyy;
                vm = (vm > 0) ? std::sqrt(vm) : (R)0;
                L.vmod = vm;
                if (xi > 0) {
                    L.frictx = L.frictx + ((cgra * L.vmod) * vxx) / xi;
                    L.fricty = L.fricty + ((cgra * L.vmod) * vyy) / xi;
                } else {
                    R constMu = -(((R)25 * cst[3]) / (R)4);
                    L.frictx = L.frictx + ((constMu * L.vmod) * vxx) / (hfrict * hfrict);
                    L.fricty = L.fricty + ((constMu * L.vmod) * vyy) / (hfrict * hfrict);
                }
            }
            L.totfrict = std::sqrt(L.frictx * L.frictx + L.fricty * L.fricty);
        }
    }

    /* the reversal filter of basal_friction_Ext_SW, SPH_SW_2019.f90:9829-9895 */
    void reversal_filter(int i, Local& L, R acc0, R acc1, int nfric) {
        bool frictional = (nfric >= 5 && nfric <= 8) || nfric == 26 || nfric == 27;
        R dc0 = -(L.frictx * L.hinv), dc1 = -(L.fricty * L.hinv);
        if (L.vmod > lit<R>(1.e-5)) {
            R vc0 = v[2 * i], vc1 = v[2 * i + 1];
            R vs0 = vc0 + dt * (acc0 + dc0), vs1 = vc1 + dt * (acc1 + dc1);
            R vdot = vs0 * vc0 + vs1 * vc1;
            if (vdot < 0) {
                R vt0 = vc0 / L.vmod, vt1 = vc1 / L.vmod;
                R accT = acc0 * vt0 + acc1 * vt1;
                R decT = dc0 * vt0 + dc1 * vt1;
                if (accT * decT < 0) {
                    dc0 = -vc0 / dt - acc0;
                    dc1 = -vc1 / dt - acc1;
                    L.frictx = -dc0 * L.h;
                    L.fricty = -dc1 * L.h;
                }
            }
        } else {
            R accT = std::sqrt(acc0 * acc0 + acc1 * acc1);
            if (accT > lit<R>(1.e-5)) {
                R ctf = frictional ? L.cf5 : L.totfrict;
                L.frictx = (ctf * acc0) / accT;
                L.fricty = (ctf * acc1) / accT;
                R fricT = std::sqrt(L.frictx * L.frictx + L.fricty * L.fricty);
                if (accT <= fricT) { L.frictx = acc0; L.fricty = acc1; }
            } else {
                L.frictx = 0; L.fricty = 0;
            }
            L.frictx = L.frictx * L.h;
            L.fricty = L.fricty * L.h;
        }
    }

    R slip_fact() {
        R s = 1;
        if (cst[47] > lit<R>(1.e-6)) s = ((R)2 * cst[47]) / ((R)1 + cst[47]);
        return s;
    }

    /* ExtForces_SW(0): SPH_SW_2019.f90:8483 and the particle loop :8532-8716 */
    void ext_forces0() {
        std::fill(ex.begin(), ex.end(), (R)0);
        if (ws) { /* soil-water pairs, :8502-8521 (dens_ws = densw/dens, :8999-9002) */
            R densw = (cst[18] < lit<R>(1.e-3)) ? (R)1000 : cst[18];
            R dens_ws = densw / cst[2];
            R cgra = cst[1];
            std::vector<A> b0(n, (A)0), b1(n, (A)0);
            for (size_t k = 0; k < pairs.size(); k++) {
                if (!ptype[k]) continue;
                int i = pairs[k].i, j = pairs[k].j; /* i soil, j water */
                R g[2] = {pd0[k], pd1[k]};
                A* b[2] = {b0.data(), b1.data()};
                for (int d = 0; d < 2; d++) {
                    b[d][i] = b[d][i] - (A)(((dens_ws * cgra) * mass[j]) * g[d]);
                    if (swalg == 0) b[d][j] = b[d][j] + (A)((cgra * mass[i]) * g[d]);
                }
            }
            for (int i = 0; i < n; i++) { ex[2 * i] = (R)b0[i]; ex[2 * i + 1] = (R)b1[i]; }
        }
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) {
            if (flag[i]) continue;
            R top[6];
            Local L;
            ext_locals(i, rho[i], L);
            const bool water = ws && itype[i] == 2;
            const int nf = water ? 1 : nfric; /* :8600-8606: the water is a Manning fluid */
            grav_and_friction(i, L, top, nf);
            if (water && swalg == 1) { /* Get_Grav_Ext_SW :9322-9331 */
                R hhsz = rho[i] + zpw[i];
                ex[2 * i] = ex[2 * i] - (L.gravz * (hhsz * gzw[2 * i])) / rho[i];
                ex[2 * i + 1] = ex[2 * i + 1] - (L.gravz * (hhsz * gzw[2 * i + 1])) / rho[i];
            } else {
                ex[2 * i] = ex[2 * i] + L.gravx;
                ex[2 * i + 1] = ex[2 * i + 1] + L.gravy;
            }
            reversal_filter(i, L, ex[2 * i] + in[2 * i], ex[2 * i + 1] + in[2 * i + 1], nf);
            ex[2 * i] = ex[2 * i] - L.frictx / L.h;
            ex[2 * i + 1] = ex[2 * i + 1] - L.fricty / L.h;
            if (icpwp == 1) { /* du, :8648-8652 */
                R betaw = ((cst[13] * L.hinv) * L.hinv) / (cst[14] * cst[14]);
                R e = rexp(-(betaw * dt));
                du1[i] = -((uaux[i] / dt) * ((R)1 - e));
            }
            if (ic_erosion) { /* Get_Erosion_Rate_SW; momentum :8664-8697 */
                R er = erosion_rate(L);
                R sf = slip_fact();
                ex[2 * i] = ex[2 * i] - ((er * v[2 * i]) * L.hinv) * sf;
                ex[2 * i + 1] = ex[2 * i + 1] - ((er * v[2 * i + 1]) * L.hinv) * sf;
            }
        }
    }

    /* Get_Erosion_Rate_SW, SPH_SW_2019.f90:10329-10356: law 1 (Hungr) E =
     * C22 h |v|; law 2 E = C22 C23 |v| tan(theta - theta_e) where the bed
     * slope along the flow, theta = atan2(-grad Z . v/|v|, 1), exceeds the
     * equilibrium angle tan(theta_e) = (denss - densw) c tanfi /
     * ((denss - densw) c + densw), c = (dens - densw)/(denss - densw); atan2,
     * atan and tan in FP64, rounded once */
    R erosion_rate(const Local& L) {
        if (eros_law == 1) return (cst[22] * L.h) * L.vmod;
        if (eros_law == 3) { /* :10357-10376, with the friction after the reversal filter */
            R er = 0;
            if (L.vmod > lit<R>(1.e-5)) {
                R taub = dens_bar * std::sqrt(L.frictx * L.frictx + L.fricty * L.fricty);
                R tauf = cst[23] + (((dens_bar_eff * cst[1]) * L.h) * ((R)1 - cst[25])) * cst[24];
                if (taub > tauf && L.vmod > lit<R>(1.e-3)) er = (cst[22] * (taub - tauf)) / dens_bar_eff;
            }
            return er;
        }
        R er = 0;
        if (L.vmod > lit<R>(1.e-5)) {
            R denss = cst[17], densw = cst[18], dens = cst[2];
            R vol_conc = (dens - densw) / (denss - densw);
            R cosa = L.vxx / L.vmod, sina = L.vyy / L.vmod;
            R gradzv = L.zpx * cosa + L.zpy * sina;
            R theta = (R)std::atan2((double)(-gradzv), 1.0);
            R xnum = (denss - densw) * vol_conc;
            R xden = xnum + densw;
            xnum = xnum * L.tanfi;
            R tanthetae = xnum / xden;
            R thetae = (R)std::atan((double)tanthetae);
            if (theta > thetae) er = ((cst[22] * cst[23]) * L.vmod) * (R)std::tan((double)(theta - thetae));
        }
        return er;
    }

    /* ExtForces_SW(1): erosion after the RK update, SPH_SW_2019.f90:8717-8807 */
    void ext_forces1() {
        if (!ic_erosion) return;
        std::fill(auxv1.begin(), auxv1.end(), (A)0);
        std::fill(auxv2.begin(), auxv2.end(), (A)0);
        /* particle i's terms for its (up to 4 x 4) DEM nodes, in the
         * order they are added: emit(ip, base / dist, 1 / dist) */
        auto node_terms = [&](int i, auto&& emit) {
            R top[6];
            Local L;
            ext_locals(i, rho[i], L);
            grav_and_friction(i, L, top, nfric);
            /* law 3 reads the friction after the reversal filter, with the
               last stage's exdvxdt + indvxdt (ExtForces_SW(1) keeps them) */
            if (eros_law == 3) reversal_filter(i, L, ex[2 * i] + in[2 * i], ex[2 * i + 1] + in[2 * i + 1], nfric);
            R er = erosion_rate(L);
            R base = dt * er;
            R xx = x[2 * i], yy = x[2 * i + 1];
            int ipx = (int)((xx - xming) / dxg + (R)1);
            int ipy = (int)((yy - yming) / dyg + (R)1);
            int x0_ = std::max(1, ipx - 1), y0_ = std::max(1, ipy - 1);
            int x1_ = std::min(nx, ipx + 2), y1_ = std::min(ny, ipy + 2);
            for (int ix = x0_; ix <= x1_; ix++)
                for (int iy = y0_; iy <= y1_; iy++) {
                    int ip = (iy - 1) * nx + (ix - 1);
                    R dx2 = xx - coorgx(ix - 1); dx2 = dx2 * dx2;
                    R dy2 = yy - coorgy(iy - 1); dy2 = dy2 * dy2;
                    R dist = rmax<R>(lit<R>(1.e-6), std::sqrt(dx2 + dy2));
                    emit(ip, (A)(base / dist), (A)((R)1 / dist));
                }
            mass[i] = mass[i] + ((dt * er) * mass[i]) / rho[i];
        };
        bool done = false;
#ifdef _OPENMP
        if (omp_get_max_threads() > 1) {
            /* terms computed in parallel, added to the nodes in particle
             * order: the same sums as the serial loop */
            std::vector<int> tip((size_t)16 * n, -1);
            std::vector<A> tv1((size_t)16 * n), tv2((size_t)16 * n);
#pragma omp parallel for schedule(static)
            for (int i = 0; i < n; i++) {
                if (flag[i]) continue;
                int m = 0;
                node_terms(i, [&](int ip, A a1, A a2) {
                    tip[16 * (size_t)i + m] = ip; tv1[16 * (size_t)i + m] = a1; tv2[16 * (size_t)i + m] = a2; m++;
                });
            }
            for (size_t e = 0; e < tip.size(); e++) {
                if (tip[e] < 0) continue;
                auxv1[tip[e]] = auxv1[tip[e]] + tv1[e];
                auxv2[tip[e]] = auxv2[tip[e]] + tv2[e];
            }
            done = true;
        }
#endif
        for (int i = 0; i < n && !done; i++) {
            if (flag[i]) continue;
            node_terms(i, [&](int ip, A a1, A a2) {
                auxv1[ip] = auxv1[ip] + a1;
                auxv2[ip] = auxv2[ip] + a2;
            });
        }
#pragma omp parallel for schedule(static)
        for (int ip = 0; ip < npoig; ip++) {
            if ((R)auxv2[ip] > lit<R>(1.e-6)) {
                R xnum = (R)(auxv1[ip] / auxv2[ip]);
                if (xnum > T(15, ip)) xnum = T(15, ip);
                if (T(15, ip) > 0) {
                    T(14, ip) = T(14, ip) + xnum;
                    T(1, ip) = T(1, ip) - xnum;
                    T(15, ip) = T(15, ip) - xnum;
                }
            }
        }
    }

    /* Get_Pwp_SW with one pwp point (icpwp = 3), SPH_SW_2019.f90:11176-11371
     * (no basal flux, no DF terms): exponential dissipation of Uaux towards
     * the depth change of the step, Drho_RK = rho - rho0 (RK45 :918-919). */
    void get_pwp() {
        if (icpwp != 3) return;
        R comp = cst[15];
        for (int i = 0; i < n; i++) {
            if (flag[i]) { uaux[i] = 0; continue; }
            R hh = rho[i];
            R dhh = rho[i] - rho0[i];
            R hinv;
            if (hh < comp) {
                hh = comp;
                hinv = (R)1 / comp;
            } else {
                hinv = (R)1 / hh;
            }
            R betaw = ((bfact * hinv) * hinv) / alphas2;
            R e = (R)std::exp((double)(-(betaw * dt))); /* exp rounded once to R */
            uaux[i] = uaux[i] * e + ((dhh / dt) * ((R)1 - e)) / betaw;
            if (uaux[i] > hh) uaux[i] = hh;
            if (uaux[i] < (hh * alphas) * fpwp_min_g) uaux[i] = (hh * alphas) * fpwp_min_g;
        }
    }

    /* h_upgrade sle = 1, SPH_MAIN_2019.f90:2925-2931 */
    void h_upgrade() {
        if (P->sle != 1) return;
        for (int i = 0; i < n; i++) {
            if (flag[i]) continue;
            hsml[i] = (R)2 * std::sqrt(mass[i] / rho[i]);
        }
    }

    /* av_vel, SPH_MAIN_2019.f90:3042-3099, and v += av (:987-993) */
    void av_vel() {
        std::vector<A> a0(n, (A)0), a1(n, (A)0);
        A* arr[2] = {a0.data(), a1.data()};
        pair_loop(2, arr, [&](size_t k, auto& a) {
            if (cross(k)) return; /* type 0 only, SPH_MAIN_2019.f90:3071 */
            int i = pairs[k].i, j = pairs[k].j;
            for (int d = 0; d < 2; d++) {
                R dvx = v[2 * i + d] - v[2 * j + d];
                R den = rho[i] + rho[j];
                R ti = ((((R)2 * mass[j]) * dvx) / den) * pw[k];
                R tj = ((((R)2 * mass[i]) * dvx) / den) * pw[k];
                a(d, i) = a(d, i) - (A)ti;
                a(d, j) = a(d, j) + (A)tj;
            }
        });
        const R eps = lit<R>(0.3);
        for (int i = 0; i < n; i++) {
            if (flag[i]) continue;
            av[2 * i] = eps * (R)a0[i];
            av[2 * i + 1] = eps * (R)a1[i];
            v[2 * i] = v[2 * i] + av[2 * i];
            v[2 * i + 1] = v[2 * i + 1] + av[2 * i + 1];
        }
    }

    /* RK45, SPH_MAIN_2019.f90:746-1005 */
    void rk45() {
        std::fill(in.begin(), in.end(), (R)0);
        std::fill(ex.begin(), ex.end(), (R)0);
        std::fill(Dx.begin(), Dx.end(), (R)0);
        std::fill(Dv.begin(), Dv.end(), (R)0);
        grid_find();
        pint_update();
        x0 = x; v0 = v;
        if (pos64) x0d = xd;
        rho0 = rho;
        if (icpwp == 1) { /* u0 = u; du keeps the last step's values (times f1 = 0 in stage 1) */
            u0 = uaux;
            du1.resize(n, (R)0);
            Du.assign(n, (R)0);
        }
        const R f1[4] = {0, lit<R>(0.5), lit<R>(0.5), 1};
        const R f2[4] = {1, 2, 2, 1};
        for (int s = 0; s < 4; s++) {
            R fdt = f1[s] * dt;
            for (int i = 0; i < n; i++) {
                if (flag[i]) continue;
                for (int d = 0; d < 2; d++) {
                    const size_t k = 2 * i + d;
                    x[k] = pos64 ? (R)(x0d[k] + (double)fdt * (double)v[k]) : x0[k] + fdt * v[k];
                    v[k] = v0[k] + fdt * (ex[k] + in[k]);
                }
                if (icpwp == 1) { /* RK45 :823-830: bounded by the depth as this stage finds it */
                    uaux[i] = u0[i] + fdt * du1[i];
                    if (uaux[i] > rho[i]) uaux[i] = rho[i];
                    else if (uaux[i] < 0) uaux[i] = 0;
                }
            }
            check_out_domain();
            sum_density();
            int_forces();
            ext_forces0();
            for (int i = 0; i < n; i++) {
                if (flag[i]) continue;
                for (int d = 0; d < 2; d++) {
                    Dv[2 * i + d] = Dv[2 * i + d] + f2[s] * (ex[2 * i + d] + in[2 * i + d]);
                    Dx[2 * i + d] = Dx[2 * i + d] + f2[s] * v[2 * i + d];
                }
                if (icpwp == 1) Du[i] = Du[i] + f2[s] * du1[i];
            }
        }
        R dt6 = dt / (R)6;
        for (int i = 0; i < n; i++) {
            if (flag[i]) {
                if (pos64) { xd[2 * i] = (double)x[2 * i]; xd[2 * i + 1] = (double)x[2 * i + 1]; }
                continue;
            }
            for (int d = 0; d < 2; d++) {
                const size_t k = 2 * i + d;
                if (pos64) {
                    xd[k] = x0d[k] + (double)dt6 * (double)Dx[k];
                    x[k] = (R)xd[k];
                } else {
                    x[k] = x0[k] + dt6 * Dx[k];
                }
                v[k] = v0[k] + dt6 * Dv[k];
            }
            if (icpwp == 1) uaux[i] = u0[i] + dt6 * Du[i]; /* :921 */
        }
        sum_density();
        check_out_domain();
        ext_forces1();
        get_pwp();
        if (icpwp == 1) /* :974-979 */
            for (int i = 0; i < n; i++) {
                if (flag[i]) continue;
                if (uaux[i] > rho[i]) uaux[i] = rho[i];
                if (uaux[i] < 0) uaux[i] = 0;
            }
        h_upgrade();
        if (P->average_velocity) av_vel();
    }

    bool any_active() const {
        for (int i = 0; i < n; i++)
            if (!flag[i]) return true;
        return false;
    }

    /* one iteration of the DTGT loop, SPH_FEM_Driver_2019.f90:1580-1630.
     * A step that starts with every particle out of the DEM box returns
     * GFSPH_ERR_DOMAIN, as the device does: the reference's grid_find would
     * size its cells by the largest hsml of no particle (zero). */
    int step() {
        if (!any_active()) return GFSPH_ERR_DOMAIN;
        adaptive_dt();
        check_out_domain();           /* time_integration_sph :232 */
        rk45();
        check_out_domain();           /* :266 */
        time += (double)dt;
        return 0;
    }

    int setup(const gfsph_params* p_, int nx_, int ny_, double xmin, double ymin, double dx, double dy,
              const double* topol_in) {
        P = p_;
        cst[0] = 0;
        for (int k = 1; k <= GFSPH_NCONST; k++) cst[k] = (R)P->cst[k - 1];
        nfric = (int)(cst[5] + lit<R>(0.01));
        ic_costheta = (int)(cst[16] + lit<R>(0.01)); /* SPH_SW_2019.f90:6734 */
        if (ic_costheta != 0 && ic_costheta != 1) return GFSPH_ERR_UNSUPPORTED;
        ic_erosion = (cst[21] > lit<R>(1.e-9)) ? 1 : 0;
        if (!(nfric == 1 || nfric == 2 || nfric == 3 || nfric == 4 || (nfric >= 5 && nfric <= 8) || nfric == 11 ||
              (nfric >= 23 && nfric <= 27)))
            return GFSPH_ERR_UNSUPPORTED;
        if ((nfric == 4 || (nfric >= 23 && nfric <= 25)) && !(P->cst[5] >= 1.e-32f)) return GFSPH_ERR_ARG; /* :9547 */
        if (nfric == 23) { /* m = 1, 2, ~1/3 or 1/2, :9578-9598 */
            float m = P->cst[7];
            if (!(m == 1.f || m == 2.f || std::fabs(m - 0.333333f) <= 1.e-3f || m == 0.5f)) return GFSPH_ERR_UNSUPPORTED;
        }
        if ((nfric == 24 || nfric == 25) && !(P->cst[7] > 0.f)) return GFSPH_ERR_ARG;
        /* crushing (const(36)), the solid-end laws (const(43)), the late xi const(41) (:1312-1325, 8424-8434) */
        if (P->cst[35] > 0.01f || P->cst[42] > 0.f || P->cst[40] > 1.e-6f) return GFSPH_ERR_UNSUPPORTED;
        if (P->ws_interact == 1 && (P->cst[49] > 0.f || P->cst[54] > 0.f)) return GFSPH_ERR_UNSUPPORTED; /* :1328-1345 */
        eros_law = ic_erosion ? (int)(cst[21] + lit<R>(0.1)) : 0;
        if (ic_erosion && (eros_law < 1 || eros_law > 3)) return GFSPH_ERR_UNSUPPORTED;
        if (eros_law == 3) { /* denss, densw (:10363-10367); constant dens_bar (ic_hrelSat 0) */
            if (P->cst[16] <= 1.e-3f || P->cst[17] <= 1.e-3f) return GFSPH_ERR_ARG;
            if ((int)(P->cst[33] + 0.01f) != 0) return GFSPH_ERR_UNSUPPORTED;
        }
        if (eros_law == 2) { /* tanfi is a friction-law local: frictional laws only; denss, densw (:10337-10340) */
            if (!((nfric >= 5 && nfric <= 8) || nfric == 26 || nfric == 27)) return GFSPH_ERR_UNSUPPORTED;
            if (P->cst[16] <= 1.e-3f || P->cst[17] <= 1.e-3f) return GFSPH_ERR_ARG;
        }
        if (P->skf < 1 || P->skf > 4) return GFSPH_ERR_UNSUPPORTED;
        ws = P->ws_interact;
        swalg = P->sw_alg;
        if (ws < 0 || ws > 1 || swalg < 0 || swalg > 1 || (ws == 0 && swalg != 0)) return GFSPH_ERR_UNSUPPORTED;
        if (ws && (ic_erosion || P->icpwp != 0 || P->nor_density != 0 || ic_costheta != 0))
            return GFSPH_ERR_UNSUPPORTED;
        nx = nx_; ny = ny_; npoig = nx * ny;
        xming = (R)(float)xmin; yming = (R)(float)ymin; dxg = (R)(float)dx; dyg = (R)(float)dy;
        xmaxg = xming + (R)(nx - 1) * dxg;
        ymaxg = yming + (R)(ny - 1) * dyg;
        topol.assign((size_t)npoig * GFSPH_NTOPO, (R)0);
        for (size_t k = 0; k < topol.size(); k++) topol[k] = (R)topol_in[k];
        auxv1.assign(npoig, (A)0);
        auxv2.assign(npoig, (A)0);
        return pwp_factors();
    }

    /* the factors of DFs_FSs_dens_and_pwp_factors (:8959-9060) and
     * mini_DFs_dens_and_pwp_factors (:11502-11580), ic_hrelSat = 0 */
    int pwp_factors() {
        icpwp = P->icpwp;
        int ic_fct_dens = (int)(cst[20] + lit<R>(0.1));
        R dens = cst[2], denss = cst[17], densw = cst[18], sr = cst[19];
        alphas = cst[14];
        fact_pwp_max = 1; fact_pwp_min = 0; fpwp_max = 1; fpwp_min = 0; fpwp_min_g = 0;
        fact_dens = 1;
        dens_bar = dens; /* ic_fct_dens = 0, :8999-9008 */
        dens_bar_eff = dens - ((densw < lit<R>(1.e-3)) ? (R)1000 : densw);
        if (ic_fct_dens == 1) {
            if (denss < lit<R>(1.e-3) || densw < lit<R>(1.e-3)) return GFSPH_ERR_ARG;
            R porosity = (denss - dens) / (denss - densw);
            R dens2 = ((R)1 - porosity) * denss;
            R dens1 = ((R)1 - porosity) * denss + porosity * densw;
            dens_bar = ((R)1 - alphas) * dens2 + alphas * dens1;
            dens_bar_eff = dens_bar - densw * alphas;
            fact_dens = dens_bar_eff / dens_bar;
            if (icpwp > 0) {
                fact_pwp_max = (R)1 + (alphas * densw) / dens_bar_eff;
                fact_pwp_min = 0;
                fpwp_max = 1;
                fpwp_min = -(alphas * densw) / dens_bar_eff;
                /* Get_Pwp_SW's own factors keep the unsaturated-layer water (Sr) */
                R g2 = ((R)1 - porosity) * denss + (porosity * densw) * sr;
                R gbar = ((R)1 - alphas) * g2 + alphas * dens1;
                R geff = gbar - densw * alphas;
                fpwp_min_g = -(alphas * densw) / geff;
            }
        } else if (ic_fct_dens != 0) {
            return GFSPH_ERR_UNSUPPORTED;
        }
        if (icpwp != 0 && icpwp != 1 && icpwp != 3) return GFSPH_ERR_UNSUPPORTED;
        if ((ic_fct_dens != 0 || icpwp != 0) && (int)(cst[34] + lit<R>(0.01)) != 0) return GFSPH_ERR_UNSUPPORTED;
        if (icpwp == 3 && cst[26] > 0) return GFSPH_ERR_UNSUPPORTED; /* drag laws rescale Bfact */
        if (ic_fct_dens == 1 && icpwp != 0 && !(alphas > lit<R>(0.01))) return GFSPH_ERR_UNSUPPORTED;
        bfact = cst[13];
        alphas2 = cst[14] * cst[14];
        return 0;
    }

    /* Uaux(1,:) = pwp0rel * rho * alphas at input (Input_SW, SPH_SW_2019.f90:1829-1852) */
    void init_pwp(const double* pwp_in) {
        uaux.assign(n, (R)0);
        if (icpwp != 3 && icpwp != 1) return;
        for (int i = 0; i < n; i++)
            uaux[i] = pwp_in ? (R)pwp_in[i] : (R)P->pwp0rel * (rho[i] * cst[14]);
    }
};

struct OracleBase {
    virtual ~OracleBase() {}
    virtual int advance(int nsteps, double t_end) = 0;
    virtual void get(double* x, double* v, double* rho, double* mass, double* hsml, int* flag, double* dt,
                     double* t, double* topol) = 0;
    virtual void get_pwp(double* pwp) = 0;
};

template <class R, class A>
struct OracleObj : OracleBase {
    Oracle<R, A> o;
    gfsph_params params;
    int advance(int nsteps, double t_end) override {
        int done = 0;
        for (int s = 0; s < nsteps; s++) {
            if (o.time >= t_end) break;
            if (o.step()) break;
            done++;
        }
        return done;
    }
    void get(double* x, double* v, double* rho, double* mass, double* hsml, int* flag, double* dt, double* t,
             double* topol) override {
        int n = o.n;
        for (size_t k = 0; k < 2 * (size_t)n; k++) {
            if (x) x[k] = o.pos64 ? o.xd[k] : (double)o.x[k];
            if (v) v[k] = (double)o.v[k];
        }
        for (int k = 0; k < n; k++) {
            if (rho) rho[k] = (double)o.rho[k];
            if (mass) mass[k] = (double)o.mass[k];
            if (hsml) hsml[k] = (double)o.hsml[k];
            if (flag) flag[k] = o.out_flag(k);
        }
        if (topol)
            for (size_t k = 0; k < o.topol.size(); k++) topol[k] = (double)o.topol[k];
        if (dt) *dt = (double)o.dt;
        if (t) *t = o.time;
    }
    void get_pwp(double* pwp) override {
        for (int k = 0; k < o.n; k++) pwp[k] = (double)o.uaux[k];
    }
};

template <class R, class A>
OracleBase* make_obj(const gfsph_params* p, int nx, int ny, double xmin, double ymin, double dx, double dy,
                     const double* topol, int n, const double* x, const double* v, const double* rho,
                     const double* mass, const double* hsml, const int* flag, const double* pwp, double dt, double t,
                     int* status, bool pos64 = false) {
    OracleObj<R, A>* ob = new OracleObj<R, A>();
    ob->params = *p;
    Oracle<R, A>& o = ob->o;
    int st = o.setup(&ob->params, nx, ny, xmin, ymin, dx, dy, topol);
    if (st) { delete ob; *status = st; return nullptr; }
    o.n = n;
    o.pos64 = pos64;
    if (pos64) o.xd.assign(x, x + 2 * (size_t)n);
    auto cp = [&](std::vector<R>& dst, const double* src, size_t m) {
        dst.resize(m);
        for (size_t k = 0; k < m; k++) dst[k] = (R)src[k];
    };
    cp(o.x, x, 2 * (size_t)n); cp(o.v, v, 2 * (size_t)n);
    cp(o.rho, rho, n); cp(o.mass, mass, n); cp(o.hsml, hsml, n);
    cp(o.mass0, mass, n);
    if (o.nfric == 3)
        for (int k = 0; k < n; k++)
            if (!(o.mass[k] > lit<R>(1.e-6))) { delete ob; *status = GFSPH_ERR_ARG; return nullptr; } /* :9450-9453 */
    o.set_flags(flag);
    o.p.assign(n, (R)0);
    o.ex.assign(2 * (size_t)n, (R)0); o.in = o.ex; o.Dx = o.ex; o.Dv = o.ex; o.av = o.ex;
    o.dt = (R)dt;
    o.time = t;
    o.init_pwp(pwp);
    *status = 0;
    return ob;
}

template <class R, class A>
int run_mode(const gfsph_params* p, int nx, int ny, double xmin, double ymin, double dx, double dy,
             double* topol, int n, double* x, double* v, double* rho, double* mass, const double* mass0,
             double* hsml, int* flag, double* pwp, int pwp_init, int nsteps, double* dt, double* t, double t_end,
             int* steps_done) {
    Oracle<R, A> o;
    int st = o.setup(p, nx, ny, xmin, ymin, dx, dy, topol);
    if (st) return st;
    o.n = n;
    auto cp = [&](std::vector<R>& dst, const double* src, size_t m) {
        dst.resize(m);
        for (size_t k = 0; k < m; k++) dst[k] = (R)src[k];
    };
    cp(o.x, x, 2 * (size_t)n); cp(o.v, v, 2 * (size_t)n);
    cp(o.rho, rho, n); cp(o.mass, mass, n); cp(o.hsml, hsml, n);
    cp(o.mass0, mass0 ? mass0 : mass, n);
    if (o.nfric == 3)
        for (int k = 0; k < n; k++)
            if (!(o.mass[k] > lit<R>(1.e-6))) return GFSPH_ERR_ARG; /* the reference stops, :9450-9453 */
    o.set_flags(flag);
    o.p.assign(n, (R)0);
    o.ex.assign(2 * (size_t)n, (R)0); o.in = o.ex; o.Dx = o.ex; o.Dv = o.ex; o.av = o.ex;
    o.dt = (R)*dt;
    o.time = *t;
    o.init_pwp(pwp_init ? nullptr : pwp);
    int done = 0, status = 0;
    for (int s = 0; s < nsteps; s++) {
        if (o.time >= t_end) break;
        status = o.step();
        if (status) break;
        done++;
    }
    for (size_t k = 0; k < 2 * (size_t)n; k++) { x[k] = (double)o.x[k]; v[k] = (double)o.v[k]; }
    for (int k = 0; k < n; k++) {
        rho[k] = (double)o.rho[k]; mass[k] = (double)o.mass[k]; hsml[k] = (double)o.hsml[k]; flag[k] = o.out_flag(k);
    }
    for (size_t k = 0; k < o.topol.size(); k++) topol[k] = (double)o.topol[k];
    if (pwp)
        for (int k = 0; k < n; k++) pwp[k] = (double)o.uaux[k];
    *dt = (double)o.dt;
    *t = o.time;
    if (steps_done) *steps_done = done;
    return status;
}

template <class R, class A>
int pairs_mode(const gfsph_params* p, int n, const double* x, const double* hsml, const double* mass,
               const double* rho_in, const int* flag, int cap, int* offsets, int* idx, double* rho_out,
               double* indvxdt) {
    Oracle<R, A> o;
    o.P = p;
    o.n = n;
    o.ws = p->ws_interact; /* the pair types; the forces of ic_ws_Interact 1 need the DEM */
    if (o.ws && indvxdt) return GFSPH_ERR_UNSUPPORTED;
    o.x.resize(2 * (size_t)n); o.hsml.resize(n); o.mass.resize(n); o.rho.resize(n);
    for (size_t k = 0; k < 2 * (size_t)n; k++) o.x[k] = (R)x[k];
    for (int k = 0; k < n; k++) {
        o.hsml[k] = (R)hsml[k];
        o.mass[k] = mass ? (R)mass[k] : (R)0;
        o.rho[k] = rho_in ? (R)rho_in[k] : (R)0;
    }
    o.set_flags(flag);
    for (int k = 1; k <= GFSPH_NCONST; k++) o.cst[k] = (R)p->cst[k - 1];
    o.grid_find();
    o.pint_update();
    if (offsets) {
        std::vector<std::vector<int>> nb(n);
        for (auto& pr : o.pairs) { nb[pr.i].push_back(pr.j); nb[pr.j].push_back(pr.i); }
        int tot = 0;
        for (int i = 0; i < n; i++) {
            std::sort(nb[i].begin(), nb[i].end());
            offsets[i] = tot;
            for (int j : nb[i]) { if (tot < cap && idx) idx[tot] = j; tot++; }
        }
        offsets[n] = tot;
        if (tot > cap) return GFSPH_ERR_CAPACITY;
    }
    if (rho_out || indvxdt) {
        o.sum_density();
        if (rho_out) for (int k = 0; k < n; k++) rho_out[k] = (double)o.rho[k];
        if (indvxdt) {
            o.p.assign(n, (R)0);
            o.in.assign(2 * (size_t)n, (R)0);
            o.int_forces();
            for (size_t k = 0; k < 2 * (size_t)n; k++) indvxdt[k] = (double)o.in[k];
        }
    }
    return 0;
}

/* getgeom2D + Get_Topol (SPH_FEM_topo_2019.f90:1660-1939) on the regular
 * background triangulation of :583-604, and Fdiff_derivs (:2812-2877). */
template <class R>
int dem_topol_mode(int mode, int nx, int ny, double dx, double dy, double* topol_io) {
    int np = nx * ny;
    std::vector<R> t((size_t)np * GFSPH_NTOPO);
    for (size_t k = 0; k < t.size(); k++) t[k] = (R)topol_io[k];
    auto T = [&](int k, int ip) -> R& { return t[(size_t)ip * GFSPH_NTOPO + (k - 1)]; };
    R dxg = (R)(float)dx, dyg = (R)(float)dy;
    if (mode == 1) {
        R del2x = (R)2 * dxg, del2y = (R)2 * dyg, delx2 = dxg * dxg, dely2 = dyg * dyg, delxy = dxg * dyg;
        for (int iy = 1; iy < ny - 1; iy++)
            for (int ix = 1; ix < nx - 1; ix++) {
                int a = iy * nx + ix;
                int al = a - 1, ar = a + 1, at = a + nx, atl = at - 1, atr = at + 1, ab = a - nx, abl = ab - 1,
                    abr = ab + 1;
                R zx = (T(1, ar) - T(1, al)) / del2x;
                R zy = (T(1, at) - T(1, ab)) / del2y;
                R rt = std::sqrt(((R)1 + zx * zx) + zy * zy);
                R zxx = ((T(1, al) - (R)2 * T(1, a)) + T(1, ar)) / delx2;
                R zyy = ((T(1, ab) - (R)2 * T(1, a)) + T(1, at)) / dely2;
                R zxy = (((T(1, atr) - T(1, abr)) - T(1, atl)) + T(1, abl)) / ((R)4 * delxy);
                T(2, a) = zx; T(3, a) = zy;
                T(4, a) = (R)1 + zx * zx; T(5, a) = zx * zy; T(6, a) = (R)1 + zy * zy;
                T(7, a) = zxx / rt; T(8, a) = zxy / rt; T(9, a) = zyy / rt;
                T(10, a) = rt; T(11, a) = zxx; T(12, a) = zxy; T(13, a) = zyy;
            }
    } else {
        int ne = 2 * (nx - 1) * (ny - 1);
        std::vector<int> im(3 * (size_t)ne);
        for (int iy = 0; iy < ny - 1; iy++)
            for (int ix = 0; ix < nx - 1; ix++) {
                int e = iy * (nx - 1) + ix;
                int ip = iy * nx + ix;
                int e1 = 2 * e, e2 = 2 * e + 1;
                im[3 * e1 + 0] = ip; im[3 * e1 + 1] = ip + 1; im[3 * e1 + 2] = ip + 1 + nx;
                im[3 * e2 + 0] = ip; im[3 * e2 + 1] = ip + 1 + nx; im[3 * e2 + 2] = ip + nx;
            }
        std::vector<R> geo(7 * (size_t)ne);
        const R nxi[3] = {-1, 1, 0}, net[3] = {-1, 0, 1};
        for (int e = 0; e < ne; e++) {
            R xx[3], yy[3];
            for (int k = 0; k < 3; k++) {
                int ip = im[3 * e + k];
                /* node coordinates relative to the DEM origin (xming, yming) */
                xx[k] = (R)(ip % nx) * dxg;
                yy[k] = (R)(ip / nx) * dyg;
            }
            R x21 = xx[1] - xx[0], x31 = xx[2] - xx[0], y21 = yy[1] - yy[0], y31 = yy[2] - yy[0];
            R rj = x21 * y31 - x31 * y21;
            R rj1 = (R)1 / rj;
            R xix = y31 * rj1, xiy = -(x31 * rj1), etx = -(y21 * rj1), ety = x21 * rj1;
            for (int k = 0; k < 3; k++) {
                geo[7 * e + k] = xix * nxi[k] + etx * net[k];
                geo[7 * e + k + 3] = xiy * nxi[k] + ety * net[k];
            }
            geo[7 * e + 6] = rj;
        }
        std::vector<R> ml(np, (R)0);
        for (int e = 0; e < ne; e++) {
            R a3 = geo[7 * e + 6] / (R)6;
            for (int k = 0; k < 3; k++) ml[im[3 * e + k]] = ml[im[3 * e + k]] + a3;
        }
        std::vector<R> tel2(ne), tel3(ne);
        for (int e = 0; e < ne; e++) {
            R ddx = 0, ddy = 0;
            for (int k = 0; k < 3; k++) {
                int ip = im[3 * e + k];
                ddx = ddx + T(1, ip) * geo[7 * e + k];
                ddy = ddy + T(1, ip) * geo[7 * e + k + 3];
            }
            tel2[e] = ddx; tel3[e] = ddy;
        }
        const R mm[3][3] = {{2, 1, 1}, {1, 2, 1}, {1, 1, 2}};
        auto project = [&](int nf, std::vector<R>* tel, int* rows) {
            std::vector<R> rhs((size_t)np * nf, (R)0), rh((size_t)np * nf);
            for (int e = 0; e < ne; e++) {
                R coe = geo[7 * e + 6] / (R)6;
                for (int k = 0; k < 3; k++) {
                    int ip = im[3 * e + k];
                    for (int f = 0; f < nf; f++) rhs[(size_t)ip * nf + f] = rhs[(size_t)ip * nf + f] + tel[f][e] * coe;
                }
            }
            for (int ip = 0; ip < np; ip++)
                for (int f = 0; f < nf; f++) T(rows[f], ip) = rhs[(size_t)ip * nf + f] / ml[ip];
            for (int it = 2; it <= 5; it++) {
                std::fill(rh.begin(), rh.end(), (R)0);
                for (int e = 0; e < ne; e++) {
                    R coe = geo[7 * e + 6] / (R)24;
                    for (int a = 0; a < 3; a++) {
                        int ip = im[3 * e + a];
                        for (int b = 0; b < 3; b++) {
                            int jp = im[3 * e + b];
                            R cm = mm[a][b];
                            for (int f = 0; f < nf; f++)
                                rh[(size_t)ip * nf + f] = rh[(size_t)ip * nf + f] + (cm * coe) * T(rows[f], jp);
                        }
                    }
                }
                for (int ip = 0; ip < np; ip++)
                    for (int f = 0; f < nf; f++)
                        T(rows[f], ip) = T(rows[f], ip) + (rhs[(size_t)ip * nf + f] - rh[(size_t)ip * nf + f]) / ml[ip];
            }
        };
        std::vector<R> tl1[2] = {tel2, tel3};
        int rows1[2] = {2, 3};
        project(2, tl1, rows1);
        std::vector<R> t4(ne), t5(ne), t6(ne);
        for (int e = 0; e < ne; e++) {
            R dxx = 0, dxy = 0, dyx = 0, dyy = 0;
            for (int k = 0; k < 3; k++) {
                int ip = im[3 * e + k];
                dxx = dxx + T(2, ip) * geo[7 * e + k];
                dxy = dxy + T(2, ip) * geo[7 * e + k + 3];
                dyx = dyx + T(3, ip) * geo[7 * e + k];
                dyy = dyy + T(3, ip) * geo[7 * e + k + 3];
            }
            t4[e] = dxx; t5[e] = (dxy + dyx) / (R)2; t6[e] = dyy;
        }
        std::vector<R> tl2[3] = {t4, t5, t6};
        int rows2[3] = {4, 5, 6};
        project(3, tl2, rows2);
        for (int ip = 0; ip < np; ip++) {
            R zx = T(2, ip), zy = T(3, ip), zxx = T(4, ip), zxy = T(5, ip), zyy = T(6, ip);
            R rt = std::sqrt(((R)1 + zx * zx) + zy * zy);
            T(4, ip) = (R)1 + zx * zx; T(5, ip) = zx * zy; T(6, ip) = (R)1 + zy * zy;
            T(7, ip) = zxx / rt; T(8, ip) = zxy / rt; T(9, ip) = zyy / rt;
            T(10, ip) = rt; T(11, ip) = zxx; T(12, ip) = zxy; T(13, ip) = zyy;
        }
    }
    for (size_t k = 0; k < t.size(); k++) topol_io[k] = (double)t[k];
    return 0;
}

/* solvegc2, SPH_GCsolver_2019.f90:16-316, literally: element-by-element K.p,
 * Jacobi preconditioner from the assembled diagonal, prescribed dofs masked,
 * stop when r.r / r0.r0 <= tol. intmat (nnode, nelem) column-major, 1-based. */
template <class R>
int solvegc2_mode(int npoin, int nelem, int nnode, int ndofn, const int* intmat, int* iffix, const double* fixed,
                  const double* gstif, double* rcg_io, double* ficg_out, double tol_in, int* iters_out) {
    const int ntotv = npoin * ndofn, nevab = nnode * ndofn;
    const R tol = (R)tol_in;
    std::vector<R> r1(ntotv, 0), s(ntotv, 0), p(ntotv, 0), q(ntotv, 0), ap(ntotv, 0), fi(ntotv, 0), rcg(ntotv),
        fx(ntotv), gs((size_t)nevab * nevab * nelem);
    for (int i = 0; i < ntotv; i++) { rcg[i] = (R)rcg_io[i]; fx[i] = (R)fixed[i]; }
    for (size_t k = 0; k < gs.size(); k++) gs[k] = (R)gstif[k];
    auto G = [&](int a, int b, int e) { return gs[(size_t)e * nevab * nevab + (size_t)b * nevab + a]; };
    auto pos = [&](int node, int idofn) { return (node - 1) * ndofn + idofn; };
    /* getqmat */
    for (int e = 0; e < nelem; e++)
        for (int in = 0; in < nnode; in++)
            for (int id = 0; id < ndofn; id++) {
                int ie = in * ndofn + id;
                q[pos(intmat[(size_t)e * nnode + in], id)] += G(ie, ie, e);
            }
    for (int i = 0; i < ntotv; i++) {
        if (std::fabs(q[i]) <= lit<R>(1.e-35)) {
            if (iffix[i] == 0) iffix[i] = -999;
        } else {
            q[i] = (R)1 / q[i];
        }
    }
    auto kbyp = [&](int iflag) {
        std::fill(ap.begin(), ap.end(), (R)0);
        for (int e = 0; e < nelem; e++)
            for (int in = 0; in < nnode; in++)
                for (int id = 0; id < ndofn; id++) {
                    int ie = in * ndofn + id;
                    int np_ = pos(intmat[(size_t)e * nnode + in], id);
                    for (int jn = 0; jn < nnode; jn++)
                        for (int jd = 0; jd < ndofn; jd++) {
                            int je = jn * ndofn + jd;
                            int mp = pos(intmat[(size_t)e * nnode + jn], jd);
                            R sum = G(ie, je, e) * p[mp];
                            if (iflag == 1 && iffix[np_] + iffix[mp] != 0) sum = 0;
                            ap[np_] = ap[np_] + sum;
                        }
                }
    };
    /* initcg */
    for (int i = 0; i < ntotv; i++) { fi[i] = fx[i]; p[i] = fi[i]; }
    kbyp(0);
    R rnorm0 = 0;
    for (int i = 0; i < ntotv; i++) {
        rcg[i] = rcg[i] - ap[i];
        s[i] = q[i] * rcg[i];
        p[i] = s[i];
        rnorm0 = rnorm0 + rcg[i] * rcg[i];
    }
    for (int i = 0; i < ntotv; i++)
        if (iffix[i] != 0) { p[i] = 0; rcg[i] = 0; s[i] = 0; }
    R rnx = 0;
    for (int i = 0; i < ntotv; i++) rnx = rnx + fx[i] * fx[i];
    rnx = std::sqrt(rnx + rnorm0);
    int it = 0;
    if (rnx < tol) {
        std::fill(fi.begin(), fi.end(), (R)0);
    } else {
        const long miter = 10L * ntotv;
        for (long iter = 1; iter <= miter; iter++) {
            /* jcg */
            kbyp(1);
            R prod1 = 0, prod2 = 0;
            for (int i = 0; i < ntotv; i++)
                if (iffix[i] == 0) { prod1 = prod1 + rcg[i] * s[i]; prod2 = prod2 + p[i] * ap[i]; }
            R alfa = prod1 / prod2;
            R prod3 = 0, rnorm1 = 0;
            for (int i = 0; i < ntotv; i++) {
                fi[i] = fi[i] + alfa * p[i];
                r1[i] = rcg[i] - alfa * ap[i];
                rnorm1 = rnorm1 + r1[i] * r1[i];
                s[i] = q[i] * r1[i];
                prod3 = prod3 + r1[i] * s[i];
            }
            it++;
            if (rnorm1 / rnorm0 > tol) {
                R beta = prod3 / prod1;
                for (int i = 0; i < ntotv; i++) { p[i] = s[i] + beta * p[i]; rcg[i] = r1[i]; }
            } else {
                break;
            }
        }
        for (int i = 0; i < ntotv; i++)
            if (iffix[i] == -999) iffix[i] = 0;
    }
    for (int i = 0; i < ntotv; i++) { ficg_out[i] = (double)fi[i]; rcg_io[i] = (double)rcg[i]; }
    if (iters_out) *iters_out = it;
    return 0;
}

} // namespace

/* The window mesh of the DEM background triangulation
 * (SPH_FEM_topo_2019.f90:583-604): nodes [ix0, ix0+nwx) x [iy0, iy0+nwy),
 * two triangles per cell, (n, n+1, n+1+nx) and (n, n+1+nx, n+nx), numbered
 * cell by cell, x fastest; node coordinates xming + i*deltxg (:284-291). */
template <class R>
struct WindowMesh {
    int nwx, nwy, nelem;
    std::vector<R> cx, cy;     /* node coordinates */
    std::vector<int> im;       /* 3 nodes per element, 0-based window nodes */
    std::vector<R> geome;      /* 7 per element: dN/dx (3), dN/dy (3), rj = 2 area (getgeom2D :1675-1716) */
    WindowMesh(int ix0, int iy0, int nwx_, int nwy_, R xming, R yming, R dxg, R dyg)
        : nwx(nwx_), nwy(nwy_), nelem(2 * (nwx_ - 1) * (nwy_ - 1)) {
        cx.resize((size_t)nwx * nwy); cy.resize((size_t)nwx * nwy);
        for (int j = 0; j < nwy; j++)
            for (int i = 0; i < nwx; i++) {
                cx[(size_t)j * nwx + i] = xming + (R)(ix0 + i) * dxg;
                cy[(size_t)j * nwx + i] = yming + (R)(iy0 + j) * dyg;
            }
        im.resize(3 * (size_t)nelem);
        geome.resize(7 * (size_t)nelem);
        for (int j = 0; j < nwy - 1; j++)
            for (int i = 0; i < nwx - 1; i++) {
                int e = 2 * (j * (nwx - 1) + i), n0 = j * nwx + i;
                int* a = &im[3 * (size_t)e];
                a[0] = n0; a[1] = n0 + 1; a[2] = n0 + 1 + nwx;
                a[3] = n0; a[4] = n0 + 1 + nwx; a[5] = n0 + nwx;
            }
        const R nxi[3] = {-1, 1, 0}, net[3] = {-1, 0, 1};
        for (int e = 0; e < nelem; e++) {
            const int* a = &im[3 * (size_t)e];
            R x21 = cx[a[1]] - cx[a[0]], x31 = cx[a[2]] - cx[a[0]];
            R y21 = cy[a[1]] - cy[a[0]], y31 = cy[a[2]] - cy[a[0]];
            R rj = x21 * y31 - x31 * y21;
            R rj1 = (R)1 / rj;
            R xix = y31 * rj1, xiy = -x31 * rj1, etx = -y21 * rj1, ety = x21 * rj1;
            R* g = &geome[7 * (size_t)e];
            for (int k = 0; k < 3; k++) {
                g[k] = xix * nxi[k] + etx * net[k];
                g[k + 3] = xiy * nxi[k] + ety * net[k];
            }
            g[6] = rj;
        }
    }
};

/* get_gradhs_w, SPH_GFL_SW_Interactions_2019.f90:368-564, on the window
 * mesh: which_element by the barycentric test of :309-344 (elements in
 * order, the last one that contains the point wins), IDW of the particle
 * depths to the element's nodes, element gradients, rhs = sum A/3 grad, and
 * niter sweeps g += (rhs - M g)/mmatl from g = 0, the first of which leaves
 * g = 0 (it divides the zeroed gradhs_w by mmatl, :497-501).  hs_in (when n
 * is 0) replaces the IDW node depths. */
template <class R, class A>
int gradhs_mode(int ix0, int iy0, int nwx, int nwy, double xmin, double ymin, double dx, double dy, int n,
                const double* x, const double* rho, const int* flag, const double* hs_in, int niter, double* hs_out,
                double* g_out) {
    WindowMesh<R> m(ix0, iy0, nwx, nwy, (R)(float)xmin, (R)(float)ymin, (R)(float)dx, (R)(float)dy);
    const int nn = nwx * nwy;
    std::vector<R> hs(nn, (R)0);
    if (n > 0) {
        std::vector<A> a1(nn, (A)0), a2(nn, (A)0);
        for (int ip = 0; ip < n; ip++) {
            if (flag && flag[ip]) continue;
            R xx = (R)x[2 * ip], yy = (R)x[2 * ip + 1];
            int which = -1;
            for (int e = 0; e < m.nelem; e++) {
                const int* a = &m.im[3 * (size_t)e];
                R xmin_e = std::min(std::min(m.cx[a[0]], m.cx[a[1]]), m.cx[a[2]]);
                R xmax_e = std::max(std::max(m.cx[a[0]], m.cx[a[1]]), m.cx[a[2]]);
                R ymin_e = std::min(std::min(m.cy[a[0]], m.cy[a[1]]), m.cy[a[2]]);
                R ymax_e = std::max(std::max(m.cy[a[0]], m.cy[a[1]]), m.cy[a[2]]);
                if (xx < xmin_e - (R)dx || xx > xmax_e + (R)dx || yy < ymin_e - (R)dy || yy > ymax_e + (R)dy) continue;
                R x1 = m.cx[a[0]], y1 = m.cy[a[0]], x2 = m.cx[a[1]], y2 = m.cy[a[1]], x3 = m.cx[a[2]], y3 = m.cy[a[2]];
                R x31 = x1 - x3, y31 = y1 - y3, x32 = x2 - x3, y32 = y2 - y3;
                R detx = x31 * y32 - y31 * x32;
                R x30 = xx - x3, y30 = yy - y3;
                R sh1 = (x30 * y32 - y30 * x32) / detx;
                R sh2 = (y30 * x31 - x30 * y31) / detx;
                R sh3 = ((R)1 - sh1) - sh2;
                if (sh1 >= 0 && sh1 <= 1 && sh2 >= 0 && sh2 <= 1 && sh3 >= 0 && sh3 <= 1) which = e;
            }
            if (which < 0) continue;
            const int* a = &m.im[3 * (size_t)which];
            for (int k = 0; k < 3; k++) {
                R xn = m.cx[a[k]], yn = m.cy[a[k]];
                R rdist = std::sqrt((xn - xx) * (xn - xx) + (yn - yy) * (yn - yy));
                a1[a[k]] = a1[a[k]] + (A)((R)rho[ip] / rdist);
                a2[a[k]] = a2[a[k]] + (A)((R)1 / rdist);
            }
        }
        for (int k = 0; k < nn; k++)
            if (!(a2[k] < (A)1.e-6)) hs[k] = (R)(a1[k] / a2[k]);
    } else {
        for (int k = 0; k < nn; k++) hs[k] = (R)hs_in[k];
    }
    std::vector<R> rhs(2 * (size_t)nn, (R)0), ml(nn, (R)0), g(2 * (size_t)nn, (R)0), rh(2 * (size_t)nn);
    for (int e = 0; e < m.nelem; e++) {
        const int* a = &m.im[3 * (size_t)e];
        const R* ge = &m.geome[7 * (size_t)e];
        R dxe = 0, dye = 0;
        for (int k = 0; k < 3; k++) { dxe = dxe + hs[a[k]] * ge[k]; dye = dye + hs[a[k]] * ge[k + 3]; }
        R coe = ge[6] / (R)6;
        for (int k = 0; k < 3; k++) {
            rhs[2 * a[k]] = rhs[2 * a[k]] + dxe * coe;
            rhs[2 * a[k] + 1] = rhs[2 * a[k] + 1] + dye * coe;
            ml[a[k]] = ml[a[k]] + coe; /* mmatl (SPH_FEM_topo_2019.f90:1764-1769) */
        }
    }
    for (int it = 2; it <= niter; it++) {
        std::fill(rh.begin(), rh.end(), (R)0);
        for (int e = 0; e < m.nelem; e++) {
            const int* a = &m.im[3 * (size_t)e];
            R coe = m.geome[7 * (size_t)e + 6] / (R)24;
            for (int in = 0; in < 3; in++)
                for (int jn = 0; jn < 3; jn++) {
                    R cm = (in == jn) ? (R)2 : (R)1;
                    for (int d = 0; d < 2; d++) rh[2 * a[in] + d] = rh[2 * a[in] + d] + (cm * coe) * g[2 * a[jn] + d];
                }
        }
        for (int k = 0; k < nn; k++)
            for (int d = 0; d < 2; d++) g[2 * k + d] = g[2 * k + d] + (rhs[2 * k + d] - rh[2 * k + d]) / ml[k];
    }
    for (int k = 0; k < nn; k++) {
        hs_out[k] = (double)hs[k];
        g_out[2 * k] = (double)g[2 * k];
        g_out[2 * k + 1] = (double)g[2 * k + 1];
    }
    return 0;
}

extern "C" {

int oracle_solvegc2(int mode, int npoin, int nelem, int nnode, int ndofn, const int* intmat, int* iffix,
                    const double* fixed, const double* gstif, double* rcg, double* ficg, double tol, int* iters) {
    if (npoin < 1 || nelem < 1 || !intmat || !iffix || !fixed || !gstif || !rcg || !ficg) return GFSPH_ERR_ARG;
    return mode == 2 ? solvegc2_mode<double>(npoin, nelem, nnode, ndofn, intmat, iffix, fixed, gstif, rcg, ficg, tol, iters)
                     : solvegc2_mode<float>(npoin, nelem, nnode, ndofn, intmat, iffix, fixed, gstif, rcg, ficg, tol, iters);
}

/* Runs nsteps steps of the reference path on the given state (in/out).
 * topol: (16, nx*ny) in/out (erosion lowers Z).  mode: 0, 1, 2 as above.
 * pwp: u (icpwp = 1) or Uaux(1,:) (icpwp = 3) in/out (may be NULL); pwp_init = 1 starts
 * it from pwp0rel*rho*const(14) as Input_SW does instead of reading it. */
int oracle_run(int mode, const gfsph_params* p, int nx, int ny, double xmin, double ymin, double dx, double dy,
               double* topol, int n, double* x, double* v, double* rho, double* mass, const double* mass0,
               double* hsml, int* flag, double* pwp, int pwp_init, int nsteps, double* dt, double* t, double t_end,
               int* steps_done) {
    if (!p || !topol || !x || !v || !rho || !mass || !hsml || !flag || !dt || !t || n < 0 || nx < 2 || ny < 2)
        return GFSPH_ERR_ARG;
    if (p->summation_density != 1) return GFSPH_ERR_UNSUPPORTED;
    switch (mode) {
    case 0: return run_mode<float, float>(p, nx, ny, xmin, ymin, dx, dy, topol, n, x, v, rho, mass, mass0, hsml, flag, pwp, pwp_init, nsteps, dt, t, t_end, steps_done);
    case 1: return run_mode<float, double>(p, nx, ny, xmin, ymin, dx, dy, topol, n, x, v, rho, mass, mass0, hsml, flag, pwp, pwp_init, nsteps, dt, t, t_end, steps_done);
    case 2: return run_mode<double, double>(p, nx, ny, xmin, ymin, dx, dy, topol, n, x, v, rho, mass, mass0, hsml, flag, pwp, pwp_init, nsteps, dt, t, t_end, steps_done);
    default: return GFSPH_ERR_ARG;
    }
}

} /* extern "C" */

/* Forward-mode derivative of nsteps FP64 steps along one direction: the
 * tangents seed_mu of const(9) (tanfi), seed_xi of const(3) (xi), seed_ty of
 * const(6) (the Bingham yield stress), seed_m of the volumes and seed_x,
 * seed_v of the initial positions and velocities.  Returns the final
 * positions, velocities and depths and their tangents. */
template <class R>
int tangent_run(const gfsph_params* p, int nx, int ny, double xmin, double ymin, double dx, double dy,
                   const double* topol, int n, const double* x, const double* v, const double* rho,
                   const double* mass, const double* hsml, const int* flag, int nsteps, double dt, double t,
                   double seed_mu, double seed_xi, double seed_ty, const double* seed_m, const double* seed_x,
                   const double* seed_v, double* out_x, double* out_v, double* out_h, double* tan_x, double* tan_v,
                   double* tan_h) {
    if (!p || !topol || !x || !v || !rho || !mass || !hsml || !flag || n < 0 || nx < 2 || ny < 2) return GFSPH_ERR_ARG;
    if (p->summation_density != 1 || p->nor_density != 0) return GFSPH_ERR_UNSUPPORTED;
    Oracle<R, Dual> o;
    int st = o.setup(p, nx, ny, xmin, ymin, dx, dy, topol);
    if (st) return st;
    o.cst[9].d = seed_mu;
    o.cst[3].d = seed_xi;
    o.cst[6].d = seed_ty;
    o.n = n;
    o.x.resize(2 * (size_t)n); o.v.resize(2 * (size_t)n);
    o.rho.resize(n); o.mass.resize(n); o.hsml.resize(n);
    for (size_t k = 0; k < 2 * (size_t)n; k++) {
        o.x[k] = R(x[k], seed_x ? seed_x[k] : 0.0);
        o.v[k] = R(v[k], seed_v ? seed_v[k] : 0.0);
    }
    for (int k = 0; k < n; k++) {
        o.rho[k] = R(rho[k]);
        o.mass[k] = R(mass[k], seed_m ? seed_m[k] : 0.0);
        o.hsml[k] = R(hsml[k]);
    }
    o.mass0 = o.mass;
    o.set_flags(flag);
    o.p.assign(n, R(0.0));
    o.ex.assign(2 * (size_t)n, R(0.0)); o.in = o.ex; o.Dx = o.ex; o.Dv = o.ex; o.av = o.ex;
    o.dt = R(dt);
    o.time = t;
    o.init_pwp(nullptr);
    int status = 0;
    for (int s2 = 0; s2 < nsteps && !status; s2++) status = o.step();
    for (size_t k = 0; k < 2 * (size_t)n; k++) {
        out_x[k] = (double)o.x[k].v; out_v[k] = (double)o.v[k].v;
        tan_x[k] = o.x[k].d; tan_v[k] = o.v[k].d;
    }
    for (int k = 0; k < n; k++) { out_h[k] = (double)o.rho[k].v; tan_h[k] = o.rho[k].d; }
    return status;
}

extern "C" {

/* The FP64 step (values and derivatives in double). */
int oracle_tangent(const gfsph_params* p, int nx, int ny, double xmin, double ymin, double dx, double dy,
                   const double* topol, int n, const double* x, const double* v, const double* rho,
                   const double* mass, const double* hsml, const int* flag, int nsteps, double dt, double t,
                   double seed_mu, double seed_xi, double seed_ty, const double* seed_m, const double* seed_x,
                   const double* seed_v, double* out_x, double* out_v, double* out_h, double* tan_x, double* tan_v,
                   double* tan_h) {
    return tangent_run<Dual>(p, nx, ny, xmin, ymin, dx, dy, topol, n, x, v, rho, mass, hsml, flag, nsteps, dt, t, seed_mu, seed_xi, seed_ty, seed_m, seed_x, seed_v, out_x, out_v, out_h, tan_x, tan_v, tan_h);
}

/* The single-precision step of mode 1 (FP32 values, FP64 sums), rounded as
 * its FP32 arithmetic rounds, with the derivatives in double: the exact
 * derivative of the trajectory the device computes. */
int oracle_tangent32(const gfsph_params* p, int nx, int ny, double xmin, double ymin, double dx, double dy,
                   const double* topol, int n, const double* x, const double* v, const double* rho,
                   const double* mass, const double* hsml, const int* flag, int nsteps, double dt, double t,
                   double seed_mu, double seed_xi, double seed_ty, const double* seed_m, const double* seed_x,
                   const double* seed_v, double* out_x, double* out_v, double* out_h, double* tan_x, double* tan_v,
                   double* tan_h) {
    return tangent_run<DualF>(p, nx, ny, xmin, ymin, dx, dy, topol, n, x, v, rho, mass, hsml, flag, nsteps, dt, t, seed_mu, seed_xi, seed_ty, seed_m, seed_x, seed_v, out_x, out_v, out_h, tan_x, tan_v, tan_h);
}

/* Persistent oracle run: create on a state, advance, read back, free. */
void* oracle_new(int mode, const gfsph_params* p, int nx, int ny, double xmin, double ymin, double dx, double dy,
                 const double* topol, int n, const double* x, const double* v, const double* rho,
                 const double* mass, const double* hsml, const int* flag, const double* pwp, double dt, double t,
                 int* status) {
    *status = GFSPH_ERR_ARG;
    if (!p || !topol || !x || !v || !rho || !mass || !hsml || !flag || n < 0 || nx < 2 || ny < 2) return nullptr;
    if (p->summation_density != 1) { *status = GFSPH_ERR_UNSUPPORTED; return nullptr; }
    switch (mode) {
    case 0: return make_obj<float, float>(p, nx, ny, xmin, ymin, dx, dy, topol, n, x, v, rho, mass, hsml, flag, pwp, dt, t, status);
    case 1: return make_obj<float, double>(p, nx, ny, xmin, ymin, dx, dy, topol, n, x, v, rho, mass, hsml, flag, pwp, dt, t, status);
    case 2: return make_obj<double, double>(p, nx, ny, xmin, ymin, dx, dy, topol, n, x, v, rho, mass, hsml, flag, pwp, dt, t, status);
    case 3: return make_obj<float, double>(p, nx, ny, xmin, ymin, dx, dy, topol, n, x, v, rho, mass, hsml, flag, pwp, dt, t, status, true);
    default: return nullptr;
    }
}

int oracle_advance(void* h, int nsteps, double t_end) {
    return h ? static_cast<OracleBase*>(h)->advance(nsteps, t_end) : GFSPH_ERR_ARG;
}

int oracle_get(void* h, double* x, double* v, double* rho, double* mass, double* hsml, int* flag, double* dt,
               double* t, double* topol) {
    if (!h) return GFSPH_ERR_ARG;
    static_cast<OracleBase*>(h)->get(x, v, rho, mass, hsml, flag, dt, t, topol);
    return 0;
}

/* The coupling pass get_gradhs_w on a node window of the DEM background
 * triangulation (see gradhs_mode).  hs_out: nwx*nwy; g_out: 2*nwx*nwy. */
int oracle_gradhs(int mode, int ix0, int iy0, int nwx, int nwy, double xmin, double ymin, double dx, double dy, int n,
                  const double* x, const double* rho, const int* flag, const double* hs_in, int niter, double* hs_out,
                  double* g_out) {
    if (nwx < 2 || nwy < 2 || !hs_out || !g_out || (n > 0 && (!x || !rho)) || (n == 0 && !hs_in)) return GFSPH_ERR_ARG;
    switch (mode) {
    case 0: return gradhs_mode<float, float>(ix0, iy0, nwx, nwy, xmin, ymin, dx, dy, n, x, rho, flag, hs_in, niter, hs_out, g_out);
    case 1: return gradhs_mode<float, double>(ix0, iy0, nwx, nwy, xmin, ymin, dx, dy, n, x, rho, flag, hs_in, niter, hs_out, g_out);
    case 2: return gradhs_mode<double, double>(ix0, iy0, nwx, nwy, xmin, ymin, dx, dy, n, x, rho, flag, hs_in, niter, hs_out, g_out);
    default: return GFSPH_ERR_ARG;
    }
}

int oracle_get_pwp(void* h, double* pwp) {
    if (!h || !pwp) return GFSPH_ERR_ARG;
    static_cast<OracleBase*>(h)->get_pwp(pwp);
    return 0;
}

void oracle_free(void* h) { delete static_cast<OracleBase*>(h); }

/* Threads of the OpenMP build's parallel regions entered from the calling
 * thread (t > 0 sets them); returns the count in effect, 1 without OpenMP. */
int oracle_set_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
    return omp_get_max_threads();
#else
    (void)t;
    return 1;
#endif
}

/* Neighbour sets (CSR, sorted), summation density and internal forces of the
 * reference on one state. Any of offsets/rho_out/indvxdt may be NULL. */
int oracle_pairs(int mode, const gfsph_params* p, int n, const double* x, const double* hsml, const double* mass,
                 const double* rho_in, const int* flag, int cap, int* offsets, int* idx, double* rho_out,
                 double* indvxdt) {
    if (!p || !x || !hsml || !flag || n < 0) return GFSPH_ERR_ARG;
    switch (mode) {
    case 0: return pairs_mode<float, float>(p, n, x, hsml, mass, rho_in, flag, cap, offsets, idx, rho_out, indvxdt);
    case 1: return pairs_mode<float, double>(p, n, x, hsml, mass, rho_in, flag, cap, offsets, idx, rho_out, indvxdt);
    case 2: return pairs_mode<double, double>(p, n, x, hsml, mass, rho_in, flag, cap, offsets, idx, rho_out, indvxdt);
    default: return GFSPH_ERR_ARG;
    }
}

/* SPH kernel values, for known-answer tests. */
int oracle_kernel(int mode, int skf, int m, const double* r, const double* dx, const double* dy, const double* hs,
                  double* w, double* d0, double* d1) {
    for (int k = 0; k < m; k++) {
        if (mode == 2) {
            double a, b, c;
            kernel_tools<double>(skf, r[k], dx[k], dy[k], hs[k], a, b, c);
            w[k] = a; d0[k] = b; d1[k] = c;
        } else {
            float a, b, c;
            kernel_tools<float>(skf, (float)r[k], (float)dx[k], (float)dy[k], (float)hs[k], a, b, c);
            w[k] = a; d0[k] = b; d1[k] = c;
        }
    }
    return 0;
}

/* DEM slope/curvature rows from Z (row 1 of topol). */
int oracle_dem_topol(int mode, int deriv, int nx, int ny, double dx, double dy, double* topol) {
    if (!topol || nx < 3 || ny < 3) return GFSPH_ERR_ARG;
    return mode == 2 ? dem_topol_mode<double>(deriv, nx, ny, dx, dy, topol)
                     : dem_topol_mode<float>(deriv, nx, ny, dx, dy, topol);
}

/* Depth raster: IDW of h over the 4x4 node stencil (SPH_SW_2019.f90:14310-14400,
 * auxv(1)/auxv(5)); zero where no particle contributes. */
int oracle_raster_idw(int nx, int ny, double xmin, double ymin, double dx, double dy, int n, const double* x,
                      const double* rho, const int* flag, double* out) {
    float xm = (float)xmin, ym = (float)ymin, dxg = (float)dx, dyg = (float)dy;
    float distg = std::sqrt(dxg * dxg + dyg * dyg);
    std::vector<float> a1((size_t)nx * ny, 0.f), a5((size_t)nx * ny, 0.f);
    for (int i = 0; i < n; i++) {
        if (flag[i]) continue;
        float xx = (float)x[2 * i], yy = (float)x[2 * i + 1];
        int ipx = (int)((xx - xm) / dxg + 1.f), ipy = (int)((yy - ym) / dyg + 1.f);
        int x0 = std::max(1, ipx - 1), y0 = std::max(1, ipy - 1), x1 = std::min(nx, ipx + 2), y1 = std::min(ny, ipy + 2);
        for (int ix = x0; ix <= x1; ix++)
            for (int iy = y0; iy <= y1; iy++) {
                int ip = (iy - 1) * nx + (ix - 1);
                float ddx = xx - (xm + (float)(ix - 1) * dxg); ddx = ddx * ddx;
                float ddy = yy - (ym + (float)(iy - 1) * dyg); ddy = ddy * ddy;
                float dist = std::max(1.e-6f, std::sqrt(ddx + ddy));
                dist = dist / distg;
                a1[ip] = a1[ip] + (float)rho[i] / dist;
                a5[ip] = a5[ip] + 1.f / dist;
            }
    }
    for (size_t ip = 0; ip < a1.size(); ip++) out[ip] = (a5[ip] >= 1.e-6f) ? (double)(a1[ip] / a5[ip]) : (double)a1[ip];
    return 0;
}

/* Per-node hazard sample (Get_MC_pixel_Vars_SW, SPH_SW_2019.f90:20739-20812):
 * each in-domain particle visits the 4 nodes of its DEM cell and adds h and
 * |v| to the sums, the count, and the maxima.  acc: (4, nx*ny) in/out:
 * sum h, max h, sum |v|, max |v|; cnt (nx*ny) in/out. */
int oracle_hazard_sample(int nx, int ny, double xmin, double ymin, double dx, double dy, int n, const double* x,
                         const double* v, const double* rho, const int* flag, double* acc, int* cnt) {
    float xm = (float)xmin, ym = (float)ymin, dxg = (float)dx, dyg = (float)dy;
    for (int i = 0; i < n; i++) {
        if (flag[i]) continue;
        float xx = (float)x[2 * i], yy = (float)x[2 * i + 1];
        int ipx = (int)((xx - xm) / dxg + 1.f), ipy = (int)((yy - ym) / dyg + 1.f);
        if (ipx >= nx) ipx = nx - 1;
        if (ipy >= ny) ipy = ny - 1;
        int ip = (ipy - 1) * nx + (ipx - 1);
        int nodes[4] = {ip, ip + 1, ip + 1 + nx, ip + nx};
        float hh = (float)rho[i];
        float vx = (float)v[2 * i], vy = (float)v[2 * i + 1];
        float vv = std::sqrt(vx * vx + vy * vy);
        for (int k = 0; k < 4; k++) {
            int q = nodes[k];
            cnt[q]++;
            double* o = acc + 4 * (size_t)q;
            o[0] = (double)((float)o[0] + hh);
            o[2] = (double)((float)o[2] + vv);
            if (hh > (float)o[1]) o[1] = hh;
            if (vv > (float)o[3]) o[3] = vv;
        }
    }
    return 0;
}

int oracle_version(void) { return 1; }

} /* extern "C" */
