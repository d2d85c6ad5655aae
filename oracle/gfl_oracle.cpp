/* CPU restatement of the Taylor-Galerkin shallow-water step of the GFL
 * module (GFL_MAIN_2019.f90) in single precision (irk = k_real), literally:
 * the loops, their order and every expression's evaluation order follow the
 * Fortran, so the sums round as the reference's do.  Test infrastructure: it
 * checks the device step (gfsph_gfl_*), nothing loads it in the product.
 *
 * Set-up (Init_GFL :65-214): getgeom2D :1275-1345, getmmatl :2794-2816,
 * Get_Topol :1346-1552 (nodal slopes and curvatures of the mesh by lumped
 * mass projection, 5 sweeps), get_boun_nodes_2D :1553-1653 (boundary nodes,
 * their tangents, the element means of the nodal topography rows), bounel
 * :1655-1762 (boundary sides).
 * Step (Time_Integration_GFL :216-284) for nsour 1, no prescribed, absorbing
 * or loaded boundaries (every boundary node is a wall), no atmospheric
 * pressure or wind, itens 0, icpwpF 0, no shock smoothing: first_step
 * :1862-2050, second_step :2055-2357, solve :2604-2790 (niter sweeps of the
 * consistent mass system), addthem :3199-3215, check :3306-3345;
 * frictlaws :3801-3990 (nfric 0-8, Manning added when const(3) != 0).
 * With WIR interaction (hs_w given, ntype 2) the soil depth raises the bed
 * in HH and its gradient is added to the slopes (:1920-1936, :2196-2200,
 * :2269-2277), the element gradient formed as get_gradhs_w does
 * (SPH_GFL_SW_Interactions_2019.f90:469-481). */
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <set>
#include <utility>
#include <vector>

namespace {

typedef float R;

struct Gfl {
    int npoin, nelem, ntopo = 9, ntype, ngaus, niter;
    R comp, swl;
    R constF[15];  /* 1-based */
    std::vector<R> coord, topol, topel, geome, mmatl, unkno;  /* column-major like the Fortran */
    std::vector<int> intmat;                                   /* (3, nelem) 1-based */
    std::vector<int> bconl;                                    /* boundary nodes, 1-based */
    std::vector<R> rtang;                                      /* (2, nboun) */
    std::vector<int> intmab;                                   /* (3, neleb) */
    std::vector<R> geomb;                                      /* (3, neleb) */
    std::vector<R> hs_w, gradhs_w, gradhs_w_elem;
    bool wir = false;
    double time_gfl = 0.0;

    R& T(int it, int ip) { return topol[(size_t)(ip - 1) * ntopo + (it - 1)]; }
    R& TE(int it, int ie) { return topel[(size_t)(ie - 1) * ntopo + (it - 1)]; }
    R& G(int k, int ie) { return geome[(size_t)(ie - 1) * 7 + (k - 1)]; }
    int& IM(int in, int ie) { return intmat[(size_t)(ie - 1) * 3 + (in - 1)]; }
    R& U(int ia, int ip) { return unkno[(size_t)(ip - 1) * 3 + (ia - 1)]; }

    void getgeom2D() {
        geome.assign((size_t)7 * nelem, 0.f);
        const R nxi[3] = {-1.0f, 1.0f, 0.0f}, net[3] = {-1.0f, 0.0f, 1.0f};
        for (int ie = 1; ie <= nelem; ie++) {
            R x[3], y[3];
            for (int in = 1; in <= 3; in++) {
                int ip = IM(in, ie);
                x[in - 1] = coord[(size_t)(ip - 1) * 2];
                y[in - 1] = coord[(size_t)(ip - 1) * 2 + 1];
            }
            R x21 = x[1] - x[0], x31 = x[2] - x[0], y21 = y[1] - y[0], y31 = y[2] - y[0];
            R rj = x21 * y31 - x31 * y21;
            R rj1 = 1.f / rj;
            R xix = y31 * rj1, xiy = -x31 * rj1, etx = -y21 * rj1, ety = x21 * rj1;
            for (int in = 1; in <= 3; in++) {
                G(in, ie) = xix * nxi[in - 1] + etx * net[in - 1];
                G(in + 3, ie) = xiy * nxi[in - 1] + ety * net[in - 1];
            }
            G(7, ie) = rj;
        }
    }

    void getmmatl() {
        mmatl.assign(npoin, 0.f);
        for (int ie = 1; ie <= nelem; ie++) {
            R area3 = G(7, ie) / 6.f;
            for (int in = 1; in <= 3; in++) mmatl[IM(in, ie) - 1] = mmatl[IM(in, ie) - 1] + area3;
        }
    }

    /* M v (consistent P1 mass, coe = area*2/24) of rows v(idx) into out */
    void projection(int nrows, const int* rows, std::vector<R>& rhs /*(3,npoin)*/) {
        const R mm[3][3] = {{2.f, 1.f, 1.f}, {1.f, 2.f, 1.f}, {1.f, 1.f, 2.f}};
        for (int ip = 1; ip <= npoin; ip++) {
            R cm = mmatl[ip - 1];
            for (int k = 0; k < nrows; k++) T(rows[k], ip) = rhs[(size_t)(ip - 1) * 3 + k] / cm;
        }
        std::vector<R> rhelp((size_t)3 * npoin);
        for (int iiter = 2; iiter <= 5; iiter++) {
            std::fill(rhelp.begin(), rhelp.end(), 0.f);
            for (int ie = 1; ie <= nelem; ie++) {
                R coe = G(7, ie) / 24.f;
                for (int in = 1; in <= 3; in++) {
                    int ip = IM(in, ie);
                    for (int jn = 1; jn <= 3; jn++) {
                        int jp = IM(jn, ie);
                        R cm = mm[in - 1][jn - 1];
                        for (int k = 0; k < nrows; k++)
                            rhelp[(size_t)(ip - 1) * 3 + k] = rhelp[(size_t)(ip - 1) * 3 + k] + cm * coe * T(rows[k], jp);
                    }
                }
            }
            for (int ip = 1; ip <= npoin; ip++) {
                R cm = mmatl[ip - 1];
                for (int k = 0; k < nrows; k++)
                    T(rows[k], ip) = T(rows[k], ip) + (rhs[(size_t)(ip - 1) * 3 + k] - rhelp[(size_t)(ip - 1) * 3 + k]) / cm;
            }
        }
    }

    void get_topol() {
        std::vector<R> rhs((size_t)3 * npoin, 0.f);
        for (int ie = 1; ie <= nelem; ie++) {
            R dx = 0.f, dy = 0.f;
            for (int in = 1; in <= 3; in++) {
                int ip = IM(in, ie);
                dx = dx + T(1, ip) * G(in, ie);
                dy = dy + T(1, ip) * G(in + 3, ie);
            }
            TE(2, ie) = dx;
            TE(3, ie) = dy;
        }
        for (int ie = 1; ie <= nelem; ie++) {
            R coe = G(7, ie) / 6.f;
            for (int in = 1; in <= 3; in++) {
                int ip = IM(in, ie);
                rhs[(size_t)(ip - 1) * 3 + 0] = rhs[(size_t)(ip - 1) * 3 + 0] + TE(2, ie) * coe;
                rhs[(size_t)(ip - 1) * 3 + 1] = rhs[(size_t)(ip - 1) * 3 + 1] + TE(3, ie) * coe;
            }
        }
        const int r23[2] = {2, 3};
        projection(2, r23, rhs);
        std::fill(rhs.begin(), rhs.end(), 0.f);
        for (int ie = 1; ie <= nelem; ie++) {
            R dxx = 0.f, dxy = 0.f, dyx = 0.f, dyy = 0.f;
            for (int in = 1; in <= 3; in++) {
                int ip = IM(in, ie);
                dxx = dxx + T(2, ip) * G(in, ie);
                dxy = dxy + T(2, ip) * G(in + 3, ie);
                dyx = dyx + T(3, ip) * G(in, ie);
                dyy = dyy + T(3, ip) * G(in + 3, ie);
            }
            TE(4, ie) = dxx;
            TE(5, ie) = (dxy + dyx) / 2.f;
            TE(6, ie) = dyy;
        }
        for (int ie = 1; ie <= nelem; ie++) {
            R coe = G(7, ie) / 6.f;
            for (int in = 1; in <= 3; in++) {
                int ip = IM(in, ie);
                for (int k = 0; k < 3; k++)
                    rhs[(size_t)(ip - 1) * 3 + k] = rhs[(size_t)(ip - 1) * 3 + k] + TE(4 + k, ie) * coe;
            }
        }
        const int r456[3] = {4, 5, 6};
        projection(3, r456, rhs);
        for (int ip = 1; ip <= npoin; ip++) {
            R zx = T(2, ip), zy = T(3, ip), zxx = T(4, ip), zxy = T(5, ip), zyy = T(6, ip);
            R rt = std::sqrt((1.f + zx * zx) + zy * zy);
            T(4, ip) = 1.f + zx * zx;
            T(5, ip) = zx * zy;
            T(6, ip) = 1.f + zy * zy;
            T(7, ip) = zxx / rt;
            T(8, ip) = zxy / rt;
            T(9, ip) = zyy / rt;
        }
    }

    void boun_nodes() {
        std::vector<long> ltang(npoin, 0);
        std::fill(topel.begin(), topel.end(), 0.f);
        const R c13 = 1.f / 3.f;
        for (int ie = 1; ie <= nelem; ie++)
            for (int in = 1; in <= 3; in++) {
                int in1 = in + 1, in2 = in + 2;
                if (in1 > 3) in1 -= 3;
                if (in2 > 3) in2 -= 3;
                int ip = IM(in, ie), ip1 = IM(in1, ie), ip2 = IM(in2, ie);
                ltang[ip - 1] += ip2 - ip1;
                for (int it = 1; it <= ntopo; it++) TE(it, ie) = TE(it, ie) + c13 * T(it, ip);
            }
        bconl.clear();
        rtang.clear();
        /* the elements of each node in element order: the reference scans every
         * element for the node (:1611-1622); the sums run in the same order */
        std::vector<std::vector<std::pair<int, int>>> elems_of(npoin);
        for (int ie = 1; ie <= nelem; ie++)
            for (int k = 1; k <= 3; k++) elems_of[IM(k, ie) - 1].push_back({ie, k});
        for (int ip = 1; ip <= npoin; ip++) {
            if (ltang[ip - 1] == 0) continue;
            bconl.push_back(ip);
            R t1 = 0.f, t2 = 0.f;
            for (const auto& e : elems_of[ip - 1]) {
                int ie = e.first, in = e.second;
                t1 = t1 - G(in + 3, ie) * G(7, ie);
                t2 = t2 + G(in, ie) * G(7, ie);
            }
            rtang.push_back(t1);
            rtang.push_back(t2);
        }
        for (size_t b = 0; b < bconl.size(); b++) {
            R amodl = std::sqrt(rtang[2 * b] * rtang[2 * b] + rtang[2 * b + 1] * rtang[2 * b + 1]);
            if (amodl < 1.0e-06f) continue;
            rtang[2 * b] = rtang[2 * b] / amodl;
            rtang[2 * b + 1] = rtang[2 * b + 1] / amodl;
        }
    }

    void bounel() {
        intmab.clear();
        geomb.clear();
        /* a side ip -> ip1 is inner when some element has the side ip1 -> ip;
         * the reference searches every element for it (:1685-1694), a set of
         * the directed sides answers the same question */
        std::set<std::pair<int, int>> sides;
        for (int je = 1; je <= nelem; je++)
            for (int jn = 1; jn <= 3; jn++) sides.insert({IM(jn, je), IM(jn % 3 + 1, je)});
        for (int ie = 1; ie <= nelem; ie++)
            for (int in = 1; in <= 3; in++) {
                int in1 = in + 1;
                if (in1 == 4) in1 = 1;
                int ip = IM(in, ie), ip1 = IM(in1, ie);
                bool inner = sides.count({ip1, ip}) != 0;
                if (inner) continue;
                intmab.push_back(ip); intmab.push_back(ip1); intmab.push_back(ie);
                R x1 = coord[(size_t)(ip - 1) * 2], y1 = coord[(size_t)(ip - 1) * 2 + 1];
                R x2 = coord[(size_t)(ip1 - 1) * 2], y2 = coord[(size_t)(ip1 - 1) * 2 + 1];
                R aleng = std::sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
                geomb.push_back((y2 - y1) / aleng);
                geomb.push_back(-(x2 - x1) / aleng);
                geomb.push_back(aleng);
            }
    }

    R tanfi_now() const {
        R tanfi8 = constF[9], tanfi0 = constF[12], Bfact = constF[13];
        if (Bfact >= 1.e-6f) return tanfi8 + (tanfi0 - tanfi8) * (R)std::exp((double)(-((R)time_gfl / Bfact)));
        return tanfi8;
    }

    /* frictlaws :3801-3990; mt = mini_topo(1..9); pwp = 0, no wind or patm */
    void frictlaws(const R* mt, R h, R hu, R hv, R HH, R& frictx, R& fricty, R& slopx, R& slopy, R& correx,
                   R& correy) const {
        R cgra = constF[1], dens = constF[2], cmanning = constF[3];
        int nfric = (int)(constF[5] + 0.01f);
        R tauy0 = constF[6], constK = constF[7], tanfi8 = constF[9], hfrict0 = constF[10];
        const double c73 = (double)(7.f / 3.f);
        R tanfi = tanfi_now();
        R gtanfi = cgra * tanfi, gtanfi8 = cgra * tanfi8;
        R hinv = 0.f;
        if (h > 0.f) hinv = 1.f / h;
        R hfrict = std::max(h, hfrict0);
        R hvmod = std::sqrt(hu * hu + hv * hv);
        R vmod = hvmod * hinv;
        R hvmodinv = 0.f;
        if (hvmod >= 1.e-5f) hvmodinv = 1.f / hvmod;
        const R pwp = 0.f;
        frictx = 0.f; fricty = 0.f;
        auto pw73 = [&](R a) { return (R)std::pow((double)a, c73); };
        if (nfric == 1) {
            R cf1 = (cgra * cmanning) * cmanning;
            frictx = ((cf1 * hu) * hvmod) / pw73(hfrict);
            fricty = ((cf1 * hv) * hvmod) / pw73(hfrict);
        } else if (nfric == 2) {
            R cf2a = constK / (8.f * dens);
            frictx = (cf2a * hu) / (hfrict * hfrict);
            fricty = (cf2a * hv) / (hfrict * hfrict);
        } else if (nfric == 3) {
            R cf3a = (1.93f * (R)std::pow((double)constK, (double)0.9f)) * (R)std::pow((double)tauy0, (double)0.1f);
            R cf3b = (tauy0 + cf3a * (R)std::pow((double)(vmod / hfrict), (double)0.3f)) / dens;
            frictx = (cf3b * hu) * hvmodinv;
            fricty = (cf3b * hv) * hvmodinv;
        } else if (nfric == 4) {
            R a_hat = ((6.f * constK) * hvmod) / (tauy0 * (hfrict * hfrict));
            R a2 = 48.f, b2 = -(32.f * a_hat) - 114.f, c2 = 65.f;
            R xh = (-b2 - std::sqrt(b2 * b2 - (4.f * a2) * c2)) / (2.f * a2);
            R Tau0 = tauy0 / xh;
            R cf4b = Tau0 / dens;
            frictx = (cf4b * hu) * hvmodinv;
            fricty = (cf4b * hv) * hvmodinv;
        } else if (nfric == 5) {
            R cf5 = gtanfi * h;
            frictx = (cf5 * hu) * hvmodinv;
            fricty = (cf5 * hv) * hvmodinv;
        } else if (nfric == 6) {
            R factpw = 1.f - pwp * hinv;
            if (factpw > 1.f) factpw = 1.f;
            if (factpw < 0.f) factpw = 0.f;
            R cf5 = (gtanfi8 * factpw) * h;
            frictx = (cf5 * hu) * hvmodinv;
            fricty = (cf5 * hv) * hvmodinv;
        } else if (nfric == 7 || nfric == 8) {
            R vx = hu * hinv, vy = hv * hinv;
            R vm = std::sqrt(vx * vx + vy * vy);
            R cv2byR = 0.f;
            if (vm >= 1e-5f) {
                R cosa = vx / vm, sina = vy / vm;
                R cos2 = cosa * cosa, sin2 = sina * sina, cbs = sina * cosa;
                R xnum = (mt[6] * cos2 + mt[7] * cbs) + mt[8] * sin2;
                R xden = (mt[3] * cos2 + mt[4] * cbs) + mt[5] * sin2;
                R rinv = xnum / xden;
                cv2byR = (vm * vm) * rinv;
            }
            R factaux = cgra + cv2byR;
            if (factaux < 0.f) factaux = 0.f;
            if (nfric == 7) {
                R cf5 = (factaux * tanfi8) * h;
                frictx = frictx + (cf5 * hu) * hvmodinv;
                fricty = fricty + (cf5 * hv) * hvmodinv;
            } else {
                R factpw = 1.f - pwp * hinv;
                if (factpw > 1.f) factpw = 1.f;
                if (factpw < 0.f) factpw = 0.f;
                R cf8 = ((factaux * tanfi8) * h) * factpw;
                frictx = (cf8 * hu) * hvmodinv;
                fricty = (cf8 * hv) * hvmodinv;
            }
        }
        if (cmanning != 0.f && nfric != 1) {
            R cf1 = (cgra * cmanning) * cmanning;
            frictx = frictx + ((cf1 * hu) * hvmod) / pw73(hfrict);
            fricty = fricty + ((cf1 * hv) * hvmod) / pw73(hfrict);
        }
        slopx = -((cgra * (h - HH)) * mt[1]);
        slopy = -((cgra * (h - HH)) * mt[2]);
        correx = 0.f - (h * 0.f) / 1000.f;
        correy = 0.f - (h * 0.f) / 1000.f;
    }

    void setup() {
        getgeom2D();
        getmmatl();
        topel.assign((size_t)ntopo * nelem, 0.f);
        get_topol();
        boun_nodes();
        bounel();
    }

    void step(R dt) {
        const R cgra = constF[1], cori = constF[4];
        const int namat = 3;
        std::vector<R> fluxp((size_t)3 * npoin, 0.f), fluyp((size_t)3 * npoin, 0.f), gpoin((size_t)3 * npoin, 0.f);
        if (wir) {  /* element gradients of hs_w (get_gradhs_w :469-481) */
            gradhs_w_elem.assign((size_t)2 * nelem, 0.f);
            for (int ie = 1; ie <= nelem; ie++) {
                R dx = 0.f, dy = 0.f;
                for (int in = 1; in <= 3; in++) {
                    int ip = IM(in, ie);
                    dx = dx + hs_w[ip - 1] * G(in, ie);
                    dy = dy + hs_w[ip - 1] * G(in + 3, ie);
                }
                gradhs_w_elem[2 * (size_t)(ie - 1)] = dx;
                gradhs_w_elem[2 * (size_t)(ie - 1) + 1] = dy;
            }
        }
        /* first_step */
        for (int ip = 1; ip <= npoin; ip++) {
            R h = U(1, ip), hu = U(2, ip), hv = U(3, ip);
            R hinv = 0.f;
            if (h >= comp) hinv = 1.f / h;
            R HH, pres;
            if (ntype == 2) {
                HH = swl - T(1, ip);
                if (wir) HH = HH - hs_w[ip - 1];
                pres = (0.5f * cgra) * (h * h - HH * HH);
            } else {
                HH = 0.f;
                pres = (0.5f * cgra) * h * h;
            }
            R* fx = &fluxp[(size_t)(ip - 1) * 3];
            R* fy = &fluyp[(size_t)(ip - 1) * 3];
            fx[0] = hu; fx[1] = (hu * hu) * hinv + pres; fx[2] = (hu * hv) * hinv;
            fy[0] = hv; fy[1] = (hu * hv) * hinv; fy[2] = (hv * hv) * hinv + pres;
            R mt[9];
            for (int it = 0; it < 9; it++) mt[it] = T(it + 1, ip);
            if (wir) { mt[1] = mt[1] + gradhs_w[2 * (size_t)(ip - 1)]; mt[2] = mt[2] + gradhs_w[2 * (size_t)(ip - 1) + 1]; }
            R frx, fry, slx, sly, cx, cy;
            frictlaws(mt, h, hu, hv, HH, frx, fry, slx, sly, cx, cy);
            R* g = &gpoin[(size_t)(ip - 1) * 3];
            g[0] = 0.f;
            if (ntype == 3) {
                g[1] = (cori * hv - frx) + cx;
                g[2] = (-(cori * hu) - fry) + cy;
            } else {
                g[1] = ((cori * hv - frx) + slx) + cx;
                g[2] = ((-(cori * hu) - fry) + sly) + cy;
            }
        }
        const R alpha = 0.5f;
        R posgp[3][2];
        if (ngaus == 3) {
            posgp[0][0] = 1.0f / 6.0f; posgp[0][1] = 1.0f / 6.0f;
            posgp[1][0] = 4.0f / 6.0f; posgp[1][1] = 1.0f / 6.0f;
            posgp[2][0] = 1.0f / 6.0f; posgp[2][1] = 4.0f / 6.0f;
        } else {
            posgp[0][0] = 1.0f / 3.0f; posgp[0][1] = 1.0f / 3.0f;
        }
        std::vector<R> unkne((size_t)3 * nelem * ngaus, 0.f);
        for (int ie = 1; ie <= nelem; ie++) {
            R delt2 = alpha * dt;
            R divef2[3] = {0.f, 0.f, 0.f};
            for (int in = 1; in <= 3; in++) {
                R anx = G(in, ie), any = G(in + 3, ie);
                int ip = IM(in, ie);
                for (int ia = 0; ia < namat; ia++)
                    divef2[ia] = (divef2[ia] + anx * fluxp[(size_t)(ip - 1) * 3 + ia]) + any * fluyp[(size_t)(ip - 1) * 3 + ia];
            }
            for (int ig = 0; ig < ngaus; ig++) {
                R sh[3] = {posgp[ig][0], posgp[ig][1], (1.0f - posgp[ig][0]) - posgp[ig][1]};
                R source[3] = {0.f, 0.f, 0.f}, variab[3] = {0.f, 0.f, 0.f};
                for (int in = 1; in <= 3; in++) {
                    int ip = IM(in, ie);
                    for (int ia = 0; ia < namat; ia++) {
                        source[ia] = source[ia] + sh[in - 1] * gpoin[(size_t)(ip - 1) * 3 + ia];
                        variab[ia] = variab[ia] + sh[in - 1] * U(ia + 1, ip);
                    }
                }
                size_t kt = ((size_t)(ie - 1) * ngaus + ig) * 3;
                for (int ia = 0; ia < namat; ia++) unkne[kt + ia] = variab[ia] + delt2 * (source[ia] - divef2[ia]);
            }
        }
        /* second_step */
        std::vector<R> rhs1((size_t)3 * npoin, 0.f);
        const R cgra05 = cgra * 0.5f;
        for (int ie = 1; ie <= nelem; ie++) {
            for (int ig = 0; ig < ngaus; ig++) {
                R sh[3] = {posgp[ig][0], posgp[ig][1], (1.0f - posgp[ig][0]) - posgp[ig][1]};
                R dvolu = G(7, ie) / (R)(2 * ngaus);
                size_t kt = ((size_t)(ie - 1) * ngaus + ig) * 3;
                R h = unkne[kt], hu = unkne[kt + 1], hv = unkne[kt + 2];
                R hinv = 0.f;
                if (h >= comp) hinv = 1.f / h;
                R HH, pres;
                if (ntype == 2) {
                    HH = 0.f;
                    for (int in = 1; in <= 3; in++) {
                        int ip = IM(in, ie);
                        HH = HH + sh[in - 1] * T(1, ip);
                        if (wir) HH = HH + sh[in - 1] * hs_w[ip - 1];
                    }
                    HH = swl - HH;
                    pres = cgra05 * (h * h - HH * HH);
                } else {
                    HH = 0.f;
                    pres = (cgra05 * h) * h;
                }
                R fx[3] = {hu, (hu * hu) * hinv + pres, (hu * hv) * hinv};
                R fy[3] = {hv, fx[2], (hv * hv) * hinv + pres};
                R mt[9];
                for (int it = 0; it < 9; it++) mt[it] = TE(it + 1, ie);
                if (wir) {
                    mt[1] = mt[1] + gradhs_w_elem[2 * (size_t)(ie - 1)];
                    mt[2] = mt[2] + gradhs_w_elem[2 * (size_t)(ie - 1) + 1];
                }
                R frx, fry, slx, sly, cx, cy;
                frictlaws(mt, h, hu, hv, HH, frx, fry, slx, sly, cx, cy);
                R ge[3];
                ge[0] = 0.f;
                if (ntype == 3) {
                    ge[1] = (cori * hv - frx) + cx;
                    ge[2] = (-(cori * hu) - fry) + cy;
                } else {
                    ge[1] = ((cori * hv - frx) + slx) + cx;
                    ge[2] = ((-(cori * hu) - fry) + sly) + cy;
                }
                for (int in = 1; in <= 3; in++) {
                    int ip = IM(in, ie);
                    R anx = G(in, ie), any = G(in + 3, ie), xni = sh[in - 1];
                    for (int ia = 0; ia < namat; ia++)
                        rhs1[(size_t)(ip - 1) * 3 + ia] = rhs1[(size_t)(ip - 1) * 3 + ia] +
                            (((anx * fx[ia] + any * fy[ia]) + xni * ge[ia]) * dvolu) * dt;
                }
            }
        }
        const R mmatb[2][2] = {{2.f, 1.f}, {1.f, 2.f}};
        const int neleb = (int)(intmab.size() / 3);
        for (int b = 0; b < neleb; b++) {
            R cosx = geomb[3 * (size_t)b], cosy = geomb[3 * (size_t)b + 1], aleng = geomb[3 * (size_t)b + 2];
            R coe = aleng / 6.f;
            for (int i = 0; i < 2; i++) {
                int in = intmab[3 * (size_t)b + i];
                for (int j = 0; j < 2; j++) {
                    int jn = intmab[3 * (size_t)b + j];
                    R cm = (mmatb[i][j] * coe) * dt;
                    for (int ia = 0; ia < namat; ia++)
                        rhs1[(size_t)(in - 1) * 3 + ia] = rhs1[(size_t)(in - 1) * 3 + ia] -
                            cm * (fluxp[(size_t)(jn - 1) * 3 + ia] * cosx + fluyp[(size_t)(jn - 1) * 3 + ia] * cosy);
                }
            }
        }
        /* solve */
        const int nboun = (int)bconl.size();
        for (int i = 0; i < nboun; i++) {  /* wall nodes: no normal component in the rhs */
            int ip = bconl[i];
            R anx = rtang[2 * (size_t)i + 1], any = -rtang[2 * (size_t)i];
            R* r = &rhs1[(size_t)(ip - 1) * 3];
            R rn = r[1] * anx + r[2] * any;
            r[1] = r[1] - rn * anx;
            r[2] = r[2] - rn * any;
        }
        std::vector<R> rhs0((size_t)3 * npoin, 0.f), rhs2((size_t)3 * npoin, 0.f);
        const R mm[3][3] = {{2.f, 1.f, 1.f}, {1.f, 2.f, 1.f}, {1.f, 1.f, 2.f}};
        for (int iiter = 1; iiter <= niter; iiter++) {
            if (iiter == 1) {
                for (int ip = 1; ip <= npoin; ip++)
                    for (int ia = 0; ia < namat; ia++)
                        rhs0[(size_t)(ip - 1) * 3 + ia] = rhs1[(size_t)(ip - 1) * 3 + ia] / mmatl[ip - 1];
            } else {
                std::fill(rhs2.begin(), rhs2.end(), 0.f);
                for (int ie = 1; ie <= nelem; ie++) {
                    R coe = G(7, ie) / 24.f;
                    for (int in = 1; in <= 3; in++) {
                        int ip = IM(in, ie);
                        for (int jn = 1; jn <= 3; jn++) {
                            int jp = IM(jn, ie);
                            R cm = mm[in - 1][jn - 1];
                            for (int ia = 0; ia < namat; ia++)
                                rhs2[(size_t)(ip - 1) * 3 + ia] = rhs2[(size_t)(ip - 1) * 3 + ia] + (cm * coe) * rhs0[(size_t)(jp - 1) * 3 + ia];
                        }
                    }
                }
                for (int ip = 1; ip <= npoin; ip++)
                    for (int ia = 0; ia < namat; ia++)
                        rhs0[(size_t)(ip - 1) * 3 + ia] = rhs0[(size_t)(ip - 1) * 3 + ia] +
                            (rhs1[(size_t)(ip - 1) * 3 + ia] - rhs2[(size_t)(ip - 1) * 3 + ia]) / mmatl[ip - 1];
            }
            for (int i = 0; i < nboun; i++) {
                R amodl = std::fabs(rtang[2 * (size_t)i]) + std::fabs(rtang[2 * (size_t)i + 1]);
                if (amodl < 1.e-06f) continue;
                int ip = bconl[i];
                R anx = rtang[2 * (size_t)i + 1], any = -rtang[2 * (size_t)i];
                R* r = &rhs0[(size_t)(ip - 1) * 3];
                R rn = r[1] * anx + r[2] * any;
                r[1] = r[1] - rn * anx;
                r[2] = r[2] - rn * any;
            }
        }
        /* addthem, check */
        for (int ip = 1; ip <= npoin; ip++) {
            for (int ia = 1; ia <= 3; ia++) U(ia, ip) = U(ia, ip) + rhs0[(size_t)(ip - 1) * 3 + ia - 1];
            if (U(1, ip) < comp) {  /* ff = 0 without prescribed values: unkno = ff * unkno */
                U(1, ip) = 0.f * U(1, ip); U(2, ip) = 0.f * U(2, ip); U(3, ip) = 0.f * U(3, ip);
            }
        }
        time_gfl = time_gfl + (double)dt;
    }
};

}  // namespace

extern "C" {

/* nsteps GFL steps of dt on the P1 mesh coord (npoin, 2), intmat (nelem, 3)
 * 1-based, nodal Z (npoin); const15[k] = constF(k) for k = 1..14; hs_w,
 * gradhs_w (npoin, 2) may be NULL (no WIR).  unkno (npoin, 3): h, hu, hv in
 * and out; topol_out (npoin, 9) and topel_out (nelem, 9), if not NULL,
 * receive the set-up's nodal and element topography rows; *time in/out. */
int oracle_gfl_run(int npoin, int nelem, const double* coord, const int* intmat, const double* z, const double* const15,
                   int ntype, int ngaus, int niter, double swl, double comp, const double* hs_w, const double* gradhs_w,
                   double* unkno, int nsteps, double dt, double* time, double* topol_out, double* topel_out) {
    if (npoin < 3 || nelem < 1 || (ntype != 2 && ntype != 3) || (ngaus != 1 && ngaus != 3) || niter < 1) return -1;
    if (!((float)const15[10] > 1.e-32f)) return -2; /* Input_GFL stops (GFL_MAIN_2019.f90:1118-1121) */
    Gfl g;
    g.npoin = npoin; g.nelem = nelem; g.ntype = ntype; g.ngaus = ngaus; g.niter = niter;
    g.comp = (R)comp; g.swl = (R)swl;
    for (int k = 0; k < 15; k++) g.constF[k] = (R)const15[k];
    g.coord.resize((size_t)2 * npoin);
    for (size_t k = 0; k < g.coord.size(); k++) g.coord[k] = (R)coord[k];
    g.intmat.assign(intmat, intmat + (size_t)3 * nelem);
    g.topol.assign((size_t)9 * npoin, 0.f);
    for (int ip = 0; ip < npoin; ip++) g.topol[(size_t)ip * 9] = (R)z[ip];
    g.setup();
    if (hs_w && gradhs_w) {
        g.wir = true;
        g.hs_w.resize(npoin);
        g.gradhs_w.resize((size_t)2 * npoin);
        for (int ip = 0; ip < npoin; ip++) g.hs_w[ip] = (R)hs_w[ip];
        for (size_t k = 0; k < g.gradhs_w.size(); k++) g.gradhs_w[k] = (R)gradhs_w[k];
    }
    g.unkno.resize((size_t)3 * npoin);
    for (size_t k = 0; k < g.unkno.size(); k++) g.unkno[k] = (R)unkno[k];
    g.time_gfl = *time;
    for (int s = 0; s < nsteps; s++) g.step((R)dt);
    for (size_t k = 0; k < g.unkno.size(); k++) unkno[k] = (double)g.unkno[k];
    *time = g.time_gfl;
    if (topol_out)
        for (size_t k = 0; k < g.topol.size(); k++) topol_out[k] = (double)g.topol[k];
    if (topel_out)
        for (size_t k = 0; k < g.topel.size(); k++) topel_out[k] = (double)g.topel[k];
    return 0;
}

}  // extern "C"
