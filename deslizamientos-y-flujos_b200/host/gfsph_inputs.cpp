// Readers of the Geoflow-SPH input files (see gfsph_inputs.h).
#include "gfsph_inputs.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace gfsph_host {

namespace {

std::string lower(std::string s) {
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

std::vector<std::string> split_items(const std::string& line) {
    std::vector<std::string> out;
    std::string cur;
    bool quoted = false;
    for (char c : line) {
        if (c == '\'' || c == '"') { quoted = !quoted; continue; }
        if (!quoted && (c == ' ' || c == '\t' || c == ',' || c == '\r')) {
            if (!cur.empty()) out.push_back(cur);
            cur.clear();
        } else {
            cur += c;
        }
    }
    if (!cur.empty()) out.push_back(cur);
    return out;
}

float to_real(const std::string& s, const std::string& where) {
    std::string t = s;
    for (char& c : t)
        if (c == 'd' || c == 'D') c = 'e';  // Fortran double-precision exponent
    char* end = nullptr;
    double v = std::strtod(t.c_str(), &end);
    if (end == t.c_str()) throw std::runtime_error(where + ": expected a number, got '" + s + "'");
    return (float)v;
}

}  // namespace

FortranReader::FortranReader(const std::string& path) : path_(path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::string line;
    while (std::getline(f, line)) lines_.push_back(line);
}

std::string FortranReader::label() {
    if (line_ >= lines_.size()) throw std::runtime_error(path_ + ": unexpected end of file (label)");
    return lines_[line_++];
}

std::vector<std::string> FortranReader::values(int n) {
    std::vector<std::string> out;
    while ((int)out.size() < n) {
        if (line_ >= lines_.size()) throw std::runtime_error(path_ + ": unexpected end of file (values)");
        for (const std::string& it : split_items(lines_[line_++])) {
            if ((int)out.size() < n) out.push_back(it);
        }
    }
    return out;
}

int FortranReader::read_int() { return (int)std::lround(to_real(values(1)[0], path_)); }
float FortranReader::read_real() { return to_real(values(1)[0], path_); }
bool FortranReader::read_logical() {
    std::string v = lower(values(1)[0]);
    return v == "t" || v == ".true." || v == "true" || v == "1";
}

MasterDat read_master(const std::string& path) {
    FortranReader r(path);
    MasterDat m;
    int nline = r.read_int();
    for (int k = 0; k < nline; k++) m.title += r.label() + "\n";
    r.label();
    auto v = r.values(3);
    m.if_sph = (int)to_real(v[0], path); m.if_gfl = (int)to_real(v[1], path); m.ic_cases_mat = (int)to_real(v[2], path);
    if (m.if_sph == 1) {
        r.label();
        v = r.values(2);
        m.problem_type = (int)to_real(v[0], path);
        m.integ_alg = (int)to_real(v[1], path);
        r.label();
        m.sph_name = split_items(r.label()).at(0);
    }
    if (m.if_gfl == 1) throw std::runtime_error(path + ": the GFL solver (if_gfl = 1) is not part of this step");
    r.label();
    v = r.values(3);
    m.dt = to_real(v[0], path); m.time_end = to_real(v[1], path); m.maxtimesteps = (int)to_real(v[2], path);
    r.label();
    v = r.values(3);
    m.print_step = (int)to_real(v[0], path); m.save_step = (int)to_real(v[1], path); m.plot_step = (int)to_real(v[2], path);
    if (m.print_step < 0) {  // nsearch_step (SPH_FEM_Driver_2019.f90:265-270)
        r.label();
        r.values(1);
        m.print_step = -m.print_step;
    }
    if (m.if_sph == 1) {
        r.label();
        v = r.values(2);
        m.dt_sph = to_real(v[0], path);
        m.ic_adapt = (int)to_real(v[1], path);
    }
    return m;
}

// A grid of nx x ny DEM nodes that the library takes (3 x 3 nodes or more)
// and whose node count fits an int; nx, ny as read (checked before the cast).
static void check_grid(double nx, double ny, const std::string& path) {
    if (!(nx >= 3.0 && ny >= 3.0 && nx * ny <= 2147483647.0))
        throw std::runtime_error(path + ": a DEM grid of " + std::to_string(nx) + " x " + std::to_string(ny) +
                                 " nodes is outside 3 x 3 .. 2^31 - 1 nodes");
}

// Topo_main (SPH_FEM_topo_2019.f90:208-260) with Get_DTM (:1155-1445).
TopoData read_top(const std::string& path) {
    FortranReader r(path);
    TopoData t;
    r.label();
    t.ictop = r.read_int();
    if (t.ictop >= 100) { t.fdiff = true; t.ictop -= 100; }
    if (t.ictop == 0) {
        r.label();
        auto v = r.values(2);
        check_grid(to_real(v[0], path), to_real(v[1], path), path);
        t.nx = (int)to_real(v[0], path);
        t.ny = (int)to_real(v[1], path);
        r.label();
        int np = t.nx * t.ny;
        std::vector<float> cx(np), cy(np);
        t.z.assign(np, 0.f);
        float xmin = 1.e9f, ymin = 1.e9f, xmax = -1.e9f, ymax = -1.e9f;
        for (int k = 0; k < np; k++) {
            v = r.values(4);
            int ip = (int)to_real(v[0], path) - 1;
            if (ip < 0 || ip >= np) throw std::runtime_error(path + ": node number out of range");
            cx[ip] = to_real(v[1], path); cy[ip] = to_real(v[2], path); t.z[ip] = to_real(v[3], path);
            xmin = std::min(xmin, cx[ip]); xmax = std::max(xmax, cx[ip]);
            ymin = std::min(ymin, cy[ip]); ymax = std::max(ymax, cy[ip]);
        }
        t.xmin = xmin; t.ymin = ymin;
        t.dx = (xmax - xmin) / (float)(t.nx - 1);
        t.dy = (ymax - ymin) / (float)(t.ny - 1);
        t.in_model.assign(np, 1);
        return t;
    }
    if (t.ictop < 10 || t.ictop > 16 || t.ictop == 12 || t.ictop == 13 || t.ictop == 14)
        throw std::runtime_error(path + ": ictop " + std::to_string(t.ictop) + " is not supported (0, 10, 11, 15, 16 are)");
    r.label();
    auto v = r.values(2);
    const float np_read = to_real(v[0], path);
    float deltx = to_real(v[1], path);
    if (!(np_read >= 1.f && np_read <= 2147483647.f))
        throw std::runtime_error(path + ": the DTM point count " + std::to_string(np_read) + " is out of range");
    if (!(deltx > 0.f) || !std::isfinite(deltx))
        throw std::runtime_error(path + ": the DTM lattice spacing must be positive");
    int np_dtm = (int)np_read;
    float xw0 = 0.f, xw1 = 0.f, yw0 = 0.f, yw1 = 0.f;
    if (t.ictop == 15 || t.ictop == 16) {
        r.label();
        v = r.values(4);
        xw0 = to_real(v[0], path); xw1 = to_real(v[1], path); yw0 = to_real(v[2], path); yw1 = to_real(v[3], path);
    }
    r.label();
    std::vector<float> px(np_dtm), py(np_dtm), pz(np_dtm);
    float xming = 1.e9f, yming = 1.e9f, xmaxg = -1.e9f, ymaxg = -1.e9f, zmaxg = -1.e9f;
    for (int k = 0; k < np_dtm; k++) {
        v = r.values(3);
        px[k] = to_real(v[0], path); py[k] = to_real(v[1], path); pz[k] = to_real(v[2], path);
        if (px[k] <= xming) xming = px[k];
        if (px[k] >= xmaxg) xmaxg = px[k];
        if (py[k] <= yming) yming = py[k];
        if (py[k] >= ymaxg) ymaxg = py[k];
        if (pz[k] >= zmaxg) zmaxg = pz[k];
    }
    check_grid((double)((xmaxg - xming) / deltx + 1.f), (double)((ymaxg - yming) / deltx + 1.f), path);
    int nx = (int)((xmaxg - xming) / deltx + 1.f);
    int ny = (int)((ymaxg - yming) / deltx + 1.f);
    float dxg = (xmaxg - xming) / (float)(nx - 1);
    float dyg = (ymaxg - yming) / (float)(ny - 1);
    if (t.ictop == 11) {  // relative coordinates
        t.xshift = xming; t.yshift = yming;
        for (int k = 0; k < np_dtm; k++) { px[k] -= xming; py[k] -= yming; }
        xmaxg -= xming; ymaxg -= yming; xming = 0.f; yming = 0.f;
    } else if (t.ictop == 15 || t.ictop == 16) {
        t.xshift = xming; t.yshift = yming;
        if (t.ictop == 15) { xw0 -= t.xshift; xw1 -= t.xshift; yw0 -= t.yshift; yw1 -= t.yshift; }
        xming = xw0; xmaxg = xw1; yming = yw0; ymaxg = yw1;
        nx = (int)((xmaxg - xming) / deltx + 1.f);
        ny = (int)((ymaxg - yming) / deltx + 1.f);
        dxg = (xmaxg - xming) / (float)(nx - 1);
        dyg = (ymaxg - yming) / (float)(ny - 1);
        for (int k = 0; k < np_dtm; k++) { px[k] -= t.xshift; py[k] -= t.yshift; }
    }
    t.nx = nx; t.ny = ny; t.xmin = xming; t.ymin = yming; t.dx = dxg; t.dy = dyg;
    // IDW of the scattered points onto the 4x4 nodes around each (:1315-1359)
    const int np = nx * ny;
    std::vector<float> a1(np, 0.f), a2(np, 0.f);
    const float distg = std::sqrt(dxg * dxg + dyg * dyg);
    for (int k = 0; k < np_dtm; k++) {
        float xx = px[k], yy = py[k];
        if (!((xx >= xming) && (xx <= xmaxg) && (yy >= yming) && (yy <= ymaxg))) continue;
        int ipx = (int)((xx - xming) / dxg + 1.f), ipy = (int)((yy - yming) / dyg + 1.f);
        int x0 = std::max(1, ipx - 1), y0 = std::max(1, ipy - 1), x1 = std::min(nx, ipx + 2), y1 = std::min(ny, ipy + 2);
        for (int ix = x0; ix <= x1; ix++)
            for (int iy = y0; iy <= y1; iy++) {
                int ip = (iy - 1) * nx + (ix - 1);
                float ddx = xx - (xming + (float)(ix - 1) * dxg);
                ddx = ddx * ddx;
                float ddy = yy - (yming + (float)(iy - 1) * dyg);
                ddy = ddy * ddy;
                float dist = std::max(1.e-6f, std::sqrt(ddx + ddy));
                dist = dist / distg;
                a1[ip] = a1[ip] + pz[k] / dist;
                a2[ip] = a2[ip] + 1.f / dist;
            }
    }
    t.z.assign(np, 0.f);
    t.in_model.assign(np, 0);
    for (int ip = 0; ip < np; ip++) {
        if (a2[ip] >= 1.e-6f) { t.z[ip] = a1[ip] / a2[ip]; t.in_model[ip] = 1; }
        else { t.z[ip] = zmaxg; t.in_model[ip] = 0; }
    }
    return t;
}

// Input_SW (SPH_SW_2019.f90:800-1390), up to the pore-pressure switch.
SwDat read_dat(const std::string& path) {
    FortranReader r(path);
    SwDat d;
    int nline = r.read_int();
    for (int k = 0; k < nline; k++) r.label();
    r.label();
    d.ic_swalg = r.read_int();
    if (d.ic_swalg == 2) throw std::runtime_error(path + ": the rotating drum (ic_SWAlg = 2) is not part of this step");
    r.label();
    d.n_hist = r.read_int();
    r.label();
    d.ndimn = r.read_int();
    if (d.ndimn != 2)
        throw std::runtime_error(path + ": ndimn " + std::to_string(d.ndimn) + " is not supported (the depth-integrated model is 2-D)");
    r.label();
    auto v = r.values(4);
    d.ic_soil = (int)to_real(v[0], path); d.ic_water = (int)to_real(v[1], path);
    d.ic_vps = (int)to_real(v[2], path); d.ic_abs = (int)to_real(v[3], path);
    if (d.ic_soil == 1) {  // Get_soil_points (:3185-3204) and the pts name (:5058-5059)
        r.label();
        v = r.values(2);
        d.icunk_s = (int)to_real(v[0], path);
        d.h_inf = to_real(v[1], path);
        if (d.icunk_s != 7 && d.icunk_s != 8 && d.icunk_s != 200)
            throw std::runtime_error(path + ": icunk_s " + std::to_string(d.icunk_s) +
                                     " is not supported (7, 8 and the restart 200 are)");
        // the pts name (Read_Source_plus_New :5058-5059) or, for a restart,
        // the problem name (Get_Restart_Info_SW :3302-3305): a label and a name
        r.label();
        d.pts_name = split_items(r.label()).at(0);
    }
    if (d.ic_water == 1) {  // Get_water_points (:2226-2273)
        r.label();
        if (d.ic_soil == 1) {
            d.icunk_w = r.read_int();
        } else {
            v = r.values(2);
            d.icunk_w = (int)to_real(v[0], path);
            d.h_inf = to_real(v[1], path);
        }
        if (d.icunk_w != 7 && d.icunk_w != 8)
            throw std::runtime_error(path + ": icunk_w " + std::to_string(d.icunk_w) +
                                     " is not supported (7 and 8, a .pts source, are)");
        // Read_Source_plus_New_WATER (:5329-5336): a label and the problem name (a16)
        r.label();
        std::string nm = r.label();
        if (nm.size() > 16) nm = nm.substr(0, 16);
        d.water_pts_name = split_items(nm).at(0);
        if (d.ic_soil != 1) throw std::runtime_error(path + ": water without soil particles is not supported");
        if (d.ic_swalg != 0 && d.ic_swalg != 1)
            throw std::runtime_error(path + ": ic_SWAlg " + std::to_string(d.ic_swalg) +
                                     " with soil and water is the debris-flow mixture (ic_ws_Interact = 2), not built");
    } else if (d.ic_swalg != 0) {
        throw std::runtime_error(path + ": ic_SWAlg " + std::to_string(d.ic_swalg) +
                                 " is supported only with soil and water particles (ic_soil = ic_water = 1)");
    }
    r.label();
    v = r.values(4);
    d.pa_sph = (int)to_real(v[0], path); d.nnps = (int)to_real(v[1], path);
    d.sle = (int)to_real(v[2], path); d.skf = (int)to_real(v[3], path);
    r.label();
    v = r.values(4);
    auto lg = [&](const std::string& s) { std::string t = lower(s); return t == "t" || t == ".true." || t == "true"; };
    d.sum_den = lg(v[0]); d.av_vel = lg(v[1]); d.virt_part = lg(v[2]); d.nor_dens = lg(v[3]);
    r.label();
    v = r.values(15);
    for (int k = 0; k < 15; k++) d.cst[k] = to_real(v[k], path);
    if (d.cst[3] > 1.e-4f) { d.cst[20] = 1.f; d.cst[21] = d.cst[3]; }  // old erosion input (:1157-1160)
    const int blocks[3][3] = {{11, 16, 30}, {30, 31, 45}, {45, 46, 60}};
    for (auto& b : blocks) {
        if (d.cst[b[0] - 1] < 0.f) {
            r.label();
            v = r.values(15);
            for (int k = 0; k < 15; k++) d.cst[b[1] - 1 + k] = to_real(v[k], path);
        }
    }
    int nfric = (int)(d.cst[4] + 0.01f);
    if (nfric == 201 || nfric == 202 || nfric == 203)
        throw std::runtime_error(path + ": nfric " + std::to_string(nfric) + " is not supported");
    if (d.cst[0] < 0.f) throw std::runtime_error(path + ": inclined-plane gravity input (const(1) < 0) is not supported");
    bool frictional = (nfric >= 5 && nfric <= 10) || nfric == 26 || nfric == 27;
    if (frictional) {
        r.label();
        d.ic_k0 = r.read_int();
        if (d.ic_k0 == 1) { r.label(); r.values(2); }
    }
    r.label();
    d.icpwp = r.read_int();
    if (d.icpwp == 1 || d.icpwp == 3) {  // Input_SW SPH_SW_2019.f90:1724-1729, 1829-1835
        r.label();
        d.pwp0rel = r.read_real();
    }
    return d;
}

// Read_Source_plus_New (SPH_SW_2019.f90:4999-5272): the source points are
// averaged by inverse distance onto a lattice of spacing delt2D, and every
// lattice node that received weight becomes a particle.
Particles read_pts(const std::string& path, float h_inf, int icunk_s, float xshift, float yshift) {
    FortranReader r(path);
    Particles P;
    r.label();
    auto v = r.values(5);
    int np_src = (int)to_real(v[0], path);
    float dx_s = to_real(v[1], path);
    float delt2Dx = to_real(v[2], path), delt2Dy = to_real(v[3], path);
    float facthsml = to_real(v[4], path);
    float delt2D = std::max(delt2Dx, delt2Dy);
    if (np_src <= 0) throw std::runtime_error(path + ": sources from topol(15) (np_Src <= 0) are not supported");
    r.label();
    std::vector<float> sx(np_src), sy(np_src), sh(np_src);
    float xmin2 = 1.e9f, ymin2 = 1.e9f, xmax2 = -1.e9f, ymax2 = -1.e9f;
    for (int k = 0; k < np_src; k++) {
        v = r.values(3);
        sx[k] = to_real(v[0], path) - xshift;
        sy[k] = to_real(v[1], path) - yshift;
        sh[k] = to_real(v[2], path);
        if (sx[k] <= xmin2) xmin2 = sx[k];
        if (sx[k] >= xmax2) xmax2 = sx[k];
        if (sy[k] <= ymin2) ymin2 = sy[k];
        if (sy[k] >= ymax2) ymax2 = sy[k];
    }
    if (icunk_s == 8) r.values(4);  // h_expans, mass_expans, mass_shift: read, not applied
    int n2x = (int)((xmax2 - xmin2) / delt2Dx + 1.f);
    int n2y = (int)((ymax2 - ymin2) / delt2Dy + 1.f);
    if (n2x < 2 || n2y < 2) throw std::runtime_error(path + ": the source covers less than two lattice nodes");
    delt2Dx = (xmax2 - xmin2) / (float)(n2x - 1);
    delt2Dy = (ymax2 - ymin2) / (float)(n2y - 1);
    const int np2 = n2x * n2y;
    std::vector<float> gx(np2), gy(np2);
    for (int iy = 0; iy < n2y; iy++)
        for (int ix = 0; ix < n2x; ix++) {
            gx[iy * n2x + ix] = xmin2 + (float)ix * delt2Dx;
            gy[iy * n2x + ix] = ymin2 + (float)iy * delt2Dy;
        }
    const float dist2D = std::sqrt(delt2Dx * delt2Dx + delt2Dy * delt2Dy);
    const int ndivx = (int)std::max(2.f, dx_s / delt2Dx), ndivy = (int)std::max(2.f, dx_s / delt2Dy);
    std::vector<float> a2(np2, 0.f), a3(np2, 0.f), a4(np2, 0.f);
    for (int k = 0; k < np_src; k++) {
        float xx = sx[k], yy = sy[k];
        int ipx = (int)((xx - xmin2) / delt2Dx + 1.f), ipy = (int)((yy - ymin2) / delt2Dy + 1.f);
        int x0 = std::max(1, ipx - ndivx + 1), y0 = std::max(1, ipy - ndivy);
        int x1 = std::min(n2x, ipx + ndivx + 1), y1 = std::min(n2y, ipy + ndivy);
        for (int ix = x0; ix <= x1; ix++)
            for (int iy = y0; iy <= y1; iy++) {
                int ip = (iy - 1) * n2x + (ix - 1);
                float ddx = xx - gx[ip];
                ddx = ddx * ddx;
                float ddy = yy - gy[ip];
                ddy = ddy * ddy;
                float dist = std::max(1.e-6f, std::sqrt(ddx + ddy));
                dist = dist / dist2D;
                a2[ip] = a2[ip] + 1.f / dist;
                a3[ip] = a3[ip] + sh[k] / dist;
            }
    }
    for (int iy = 0; iy + 1 < n2y; iy++)
        for (int ix = 0; ix + 1 < n2x; ix++) {
            int n1 = iy * n2x + ix, n2 = n1 + 1, n3 = n1 + n2x, n4 = n3 + 1;
            if (a2[n1] >= 1.e-6f && a2[n2] >= 1.e-6f && a2[n3] >= 1.e-6f && a2[n4] >= 1.e-6f) {
                a4[n1] += 1.f; a4[n2] += 1.f; a4[n3] += 1.f; a4[n4] += 1.f;
            }
        }
    const float d_area = delt2Dx * delt2Dy / 4.f;
    for (int ip = 0; ip < np2; ip++) {
        if (!(a2[ip] >= 1.e-6f)) continue;
        float h = a3[ip] / a2[ip];
        if (h < h_inf) h = h_inf;
        float m = (d_area * h) * a4[ip];
        P.x.push_back(gx[ip]);
        P.x.push_back(gy[ip]);
        P.h.push_back(h);
        P.mass.push_back(m);
        P.hsml.push_back(delt2D * facthsml);
        P.total_volume += m;
    }
    P.delt2d = delt2D;
    P.facthsml = facthsml;
    P.np_src = np_src;
    return P;
}

RestartState read_restart(const std::string& path) {
    FortranReader r(path);
    RestartState s;
    r.label();                          // ' ----- npoin_s      time at restart ----- '
    auto v = r.values(2);               // npoin_s, time_sph_restart (:3312)
    const long long n = (long long)to_real(v[0], path);
    if (n < 1 || n > 0x7fffffffLL) throw std::runtime_error(path + ": npoin_s out of range");
    s.time = std::strtod(v[1].c_str(), nullptr);
    r.label();                          // the column header
    s.itype.resize(n); s.x.resize(2 * n); s.v.resize(2 * n);
    s.h.resize(n); s.mass.resize(n); s.hsml.resize(n); s.pwp.resize(n);
    for (long long i = 0; i < n; i++) {  // ipoin, itype, x, y, vx, vy, h, mass, hsml, u (:3318-3319)
        v = r.values(10);
        s.itype[i] = (int)to_real(v[1], path);
        s.x[2 * i] = to_real(v[2], path); s.x[2 * i + 1] = to_real(v[3], path);
        s.v[2 * i] = to_real(v[4], path); s.v[2 * i + 1] = to_real(v[5], path);
        s.h[i] = to_real(v[6], path); s.mass[i] = to_real(v[7], path);
        s.hsml[i] = to_real(v[8], path); s.pwp[i] = to_real(v[9], path);
    }
    return s;
}

TopoRestart read_topo_restart(const std::string& path, int npoig) {
    FortranReader r(path);
    TopoRestart t;
    r.label();
    auto v = r.values(2);               // npoig, time (:2904)
    if ((long long)to_real(v[0], path) != npoig)
        throw std::runtime_error(path + ": its node count differs from the DEM's");
    t.time = std::strtod(v[1].c_str(), nullptr);
    r.label();
    t.z.resize(npoig); t.eroded.resize(npoig); t.avail.resize(npoig);
    for (int i = 0; i < npoig; i++) {   // ip, Topol(1), Topol(14), Topol(15) (:2910)
        v = r.values(4);
        t.z[i] = to_real(v[1], path); t.eroded[i] = to_real(v[2], path); t.avail[i] = to_real(v[3], path);
    }
    return t;
}

void write_restart(const std::string& path, const RestartState& s) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) throw std::runtime_error("cannot write " + path);
    std::fprintf(f, " ----- npoin_s      time at restart -----  %.17G\n", s.time);
    std::fprintf(f, " %d %.17G\n", s.n(), s.time);
    std::fprintf(f, " ipoin...itype....x ............   y ..........   vx............. vy ..........   h........   "
                    "mass..........   hsml ..........   pwp   \n");
    for (int i = 0; i < s.n(); i++)
        std::fprintf(f, "%7d  %5d  %16.9E  %16.9E  %16.9E  %16.9E  %16.9E  %16.9E  %16.9E  %16.9E\n", i + 1, s.itype[i],
                     (double)s.x[2 * i], (double)s.x[2 * i + 1], (double)s.v[2 * i], (double)s.v[2 * i + 1],
                     (double)s.h[i], (double)s.mass[i], (double)s.hsml[i], (double)s.pwp[i]);
    if (std::fclose(f) != 0) throw std::runtime_error("cannot write " + path);
}

void write_topo_restart(const std::string& path, const TopoRestart& t) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) throw std::runtime_error("cannot write " + path);
    std::fprintf(f, " ----- npoig      time at restart -----  %.17G\n", t.time);
    std::fprintf(f, " %zu %.17G\n", t.z.size(), t.time);
    std::fprintf(f, " ipoig...Topol (1,:)....Topol (14,:) ..........Topol (16,:)  \n");
    for (size_t i = 0; i < t.z.size(); i++)
        std::fprintf(f, "%7zu    %16.9E  %16.9E  %16.9E\n", i + 1, (double)t.z[i], (double)t.eroded[i], (double)t.avail[i]);
    if (std::fclose(f) != 0) throw std::runtime_error("cannot write " + path);
}

}  // namespace gfsph_host
