// Host-side DEM set-up (run once before the time loop, as Topo_main does):
// slope and curvature rows topol(2..13,:) from the elevation row topol(1,:).
//   mode 0: Get_Topol (SPH_FEM_topo_2019.f90:1723-1939) — element slopes of
//           the regular two-triangles-per-cell mesh (:583-604, geometry from
//           getgeom2D :1660-1720) projected to the nodes with the lumped mass
//           matrix and refined by 4 Jacobi corrections with the consistent
//           P1 mass matrix (5 iterations in total), then the same for the
//           second derivatives.
//   mode 1: Fdiff_derivs (:2812-2877) — central differences, boundary rows
//           left at zero.
#include <cmath>
#include <vector>

#include "../../include/gfsph.h"

namespace {

struct Mesh {
    int nx, ny, ne;
    std::vector<int> tri;     // 3 nodes per element
    std::vector<float> geo;   // 7 per element: dN/dx (3), dN/dy (3), 2*area
    std::vector<float> lumped;
};

Mesh build_mesh(int nx, int ny, float dx, float dy) {
    Mesh m;
    m.nx = nx; m.ny = ny; m.ne = 2 * (nx - 1) * (ny - 1);
    m.tri.resize(3 * (size_t)m.ne);
    m.geo.resize(7 * (size_t)m.ne);
    for (int iy = 0; iy + 1 < ny; iy++)
        for (int ix = 0; ix + 1 < nx; ix++) {
            int cell = iy * (nx - 1) + ix, node = iy * nx + ix;
            int* a = &m.tri[6 * (size_t)cell];
            a[0] = node; a[1] = node + 1; a[2] = node + 1 + nx;       // lower-right triangle
            a[3] = node; a[4] = node + 1 + nx; a[5] = node + nx;      // upper-left triangle
        }
    const float dnxi[3] = {-1.f, 1.f, 0.f}, dnet[3] = {-1.f, 0.f, 1.f};
    for (int e = 0; e < m.ne; e++) {
        float px[3], py[3];
        for (int k = 0; k < 3; k++) {
            int node = m.tri[3 * (size_t)e + k];
            px[k] = (float)(node % nx) * dx;
            py[k] = (float)(node / nx) * dy;
        }
        float x21 = px[1] - px[0], x31 = px[2] - px[0], y21 = py[1] - py[0], y31 = py[2] - py[0];
        float jac = x21 * y31 - x31 * y21;
        float ij = 1.f / jac;
        float xix = y31 * ij, xiy = -(x31 * ij), etx = -(y21 * ij), ety = x21 * ij;
        float* g = &m.geo[7 * (size_t)e];
        for (int k = 0; k < 3; k++) {
            g[k] = xix * dnxi[k] + etx * dnet[k];
            g[k + 3] = xiy * dnxi[k] + ety * dnet[k];
        }
        g[6] = jac;
    }
    m.lumped.assign((size_t)nx * ny, 0.f);
    for (int e = 0; e < m.ne; e++) {
        float third = m.geo[7 * (size_t)e + 6] / 6.f;
        for (int k = 0; k < 3; k++) m.lumped[m.tri[3 * (size_t)e + k]] += third;
    }
    return m;
}

// Projects nf element fields onto the nodes: lumped solve + 4 Jacobi
// corrections with the consistent mass matrix (coefficients (2,1,1)/24 * 2A).
void project(const Mesh& m, int nf, const std::vector<float>* elem, float* topol, const int* rows) {
    size_t np = (size_t)m.nx * m.ny;
    std::vector<float> rhs(np * nf, 0.f), help(np * nf);
    for (int e = 0; e < m.ne; e++) {
        float coe = m.geo[7 * (size_t)e + 6] / 6.f;
        for (int k = 0; k < 3; k++) {
            size_t node = m.tri[3 * (size_t)e + k];
            for (int f = 0; f < nf; f++) rhs[node * nf + f] += elem[f][e] * coe;
        }
    }
    for (size_t node = 0; node < np; node++)
        for (int f = 0; f < nf; f++) topol[node * GFSPH_NTOPO + rows[f]] = rhs[node * nf + f] / m.lumped[node];
    for (int it = 2; it <= 5; it++) {
        std::fill(help.begin(), help.end(), 0.f);
        for (int e = 0; e < m.ne; e++) {
            float coe = m.geo[7 * (size_t)e + 6] / 24.f;
            const int* t = &m.tri[3 * (size_t)e];
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    float cm = (a == b) ? 2.f : 1.f;
                    for (int f = 0; f < nf; f++)
                        help[(size_t)t[a] * nf + f] += (cm * coe) * topol[(size_t)t[b] * GFSPH_NTOPO + rows[f]];
                }
        }
        for (size_t node = 0; node < np; node++)
            for (int f = 0; f < nf; f++) {
                float& v = topol[node * GFSPH_NTOPO + rows[f]];
                v = v + (rhs[node * nf + f] - help[node * nf + f]) / m.lumped[node];
            }
    }
}

void fill_curvature(float* t) {
    float zx = t[1], zy = t[2], zxx = t[3], zxy = t[4], zyy = t[5];
    float rt = std::sqrt((1.f + zx * zx) + zy * zy);
    t[3] = 1.f + zx * zx; t[4] = zx * zy; t[5] = 1.f + zy * zy;
    t[6] = zxx / rt; t[7] = zxy / rt; t[8] = zyy / rt;
    t[9] = rt; t[10] = zxx; t[11] = zxy; t[12] = zyy;
}

}  // namespace

extern "C" int gfsph_dem_topol(int mode, int nx, int ny, float dx, float dy, float* topol) try {
    if (!topol || nx < 3 || ny < 3 || !(dx > 0.f) || !(dy > 0.f)) return GFSPH_ERR_ARG;
    size_t np = (size_t)nx * ny;
    if (mode == 1) {
        float d2x = 2.f * dx, d2y = 2.f * dy, dx2 = dx * dx, dy2 = dy * dy, dxy = dx * dy;
        auto Z = [&](size_t node) { return topol[node * GFSPH_NTOPO]; };
        for (int iy = 1; iy + 1 < ny; iy++)
            for (int ix = 1; ix + 1 < nx; ix++) {
                size_t a = (size_t)iy * nx + ix;
                float* t = &topol[a * GFSPH_NTOPO];
                t[1] = (Z(a + 1) - Z(a - 1)) / d2x;
                t[2] = (Z(a + nx) - Z(a - nx)) / d2y;
                t[3] = ((Z(a - 1) - 2.f * Z(a)) + Z(a + 1)) / dx2;
                t[5] = ((Z(a - nx) - 2.f * Z(a)) + Z(a + nx)) / dy2;
                t[4] = (((Z(a + nx + 1) - Z(a - nx + 1)) - Z(a + nx - 1)) + Z(a - nx - 1)) / (4.f * dxy);
                fill_curvature(t);
            }
        return GFSPH_OK;
    }
    if (mode != 0) return GFSPH_ERR_ARG;
    Mesh m = build_mesh(nx, ny, dx, dy);
    std::vector<float> sx(m.ne), sy(m.ne);
    for (int e = 0; e < m.ne; e++) {
        const int* t = &m.tri[3 * (size_t)e];
        const float* g = &m.geo[7 * (size_t)e];
        float ax = 0.f, ay = 0.f;
        for (int k = 0; k < 3; k++) {
            ax += topol[(size_t)t[k] * GFSPH_NTOPO] * g[k];
            ay += topol[(size_t)t[k] * GFSPH_NTOPO] * g[k + 3];
        }
        sx[e] = ax; sy[e] = ay;
    }
    std::vector<float> e1[2] = {sx, sy};
    const int r1[2] = {1, 2};
    project(m, 2, e1, topol, r1);
    std::vector<float> cxx(m.ne), cxy(m.ne), cyy(m.ne);
    for (int e = 0; e < m.ne; e++) {
        const int* t = &m.tri[3 * (size_t)e];
        const float* g = &m.geo[7 * (size_t)e];
        float xx = 0.f, xy = 0.f, yx = 0.f, yy = 0.f;
        for (int k = 0; k < 3; k++) {
            const float* tn = &topol[(size_t)t[k] * GFSPH_NTOPO];
            xx += tn[1] * g[k]; xy += tn[1] * g[k + 3];
            yx += tn[2] * g[k]; yy += tn[2] * g[k + 3];
        }
        cxx[e] = xx; cxy[e] = (xy + yx) / 2.f; cyy[e] = yy;
    }
    std::vector<float> e2[3] = {cxx, cxy, cyy};
    const int r2[3] = {3, 4, 5};
    project(m, 3, e2, topol, r2);
    for (size_t node = 0; node < np; node++) fill_curvature(&topol[node * GFSPH_NTOPO]);
    return GFSPH_OK;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}
