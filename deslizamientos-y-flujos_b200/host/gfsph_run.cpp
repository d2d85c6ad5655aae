// gfsph_run — a C++ stand-in for the Geoflow-SPH Fortran driver over the
// gfsph C ABI: reads the reference's <problem>.MASTER.dat, the SW .dat, the
// .top DEM and the .pts source (or, with icunk_s = 200, the restart files
// restart.dat and restart.top, Get_Restart_Info_SW SPH_SW_2019.f90:3270-3337
// and Get_Topo_restart SPH_FEM_topo_2019.f90:2883-2920), runs the DTGT loop
// (SPH_FEM_Driver_2019.f90:1580-1697) on the GPU with the reference's output
// cadence, and writes:
//   - at every plot time (plot_step * dt): a summary line, the depth raster
//     (ESRI ASCII grid) and the GiD results <problem>.post.res (height and
//     velocity at the DEM nodes, displacement and velocity of the particles,
//     the pore pressure at the nodes with icpwp = 1, OutputRes_Classic
//     SPH_SW_2019.f90:13316-13471); the GiD mesh <problem>.post.msh
//     (the DEM quadrilaterals and the particles, OutputMesh_Classic) at the
//     start;
//   - at every save time (save_step * dt): the restart files
//     <problem>.restart.dat and, with erosion, <problem>.restart.top
//     (OutputSave_SW SPH_SW_2019.f90:12416-12485); also at the end of a run
//     stopped by --max-steps, so that it can be resumed;
//   - at the end, the per-node maximum depth and velocity.
//
//   gfsph_run <problem> [--dir D] [--topo NAME] [--out D] [--max-steps N] [--parse-only] [--dump FILE]
//
// --dump writes the parsed run (params struct, DEM grid and elevations, the
// particles) to a binary file and exits: little-endian, "GFSPHDMP", int32
// version 1, int32 sizeof(gfsph_params), the params bytes, int32 nx, ny,
// float32 xmin, ymin, dx, dy, float32 z[nx*ny], int32 n, float32 x[2n],
// v[2n], rho[n], mass[n], hsml[n].
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/gfsph.h"
#include "gfsph_inputs.h"

using namespace gfsph_host;

namespace {

std::string join(const std::string& dir, const std::string& f) { return dir.empty() ? f : dir + "/" + f; }

bool exists(const std::string& p) {
    FILE* f = std::fopen(p.c_str(), "r");
    if (f) std::fclose(f);
    return f != nullptr;
}

std::string find_file(const std::string& dir, const std::string& stem, const char* const* exts) {
    for (int k = 0; exts[k]; k++) {
        std::string p = join(dir, stem + exts[k]);
        if (exists(p)) return p;
    }
    return join(dir, stem + exts[0]);
}

void write_asc(const std::string& path, const TopoData& t, const std::vector<float>& v) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) throw std::runtime_error("cannot write " + path);
    std::fprintf(f, "ncols %d\nnrows %d\nxllcenter %.6f\nyllcenter %.6f\ncellsize %.6f\nNODATA_value -9999\n", t.nx,
                 t.ny, (double)(t.xmin + t.xshift), (double)(t.ymin + t.yshift), (double)t.dx);
    for (int iy = t.ny - 1; iy >= 0; iy--) {  // first row is the northernmost
        for (int ix = 0; ix < t.nx; ix++) std::fprintf(f, "%.5g ", (double)v[(size_t)iy * t.nx + ix]);
        std::fprintf(f, "\n");
    }
    std::fclose(f);
}

// Get_Z_Topo (SPH_FEM_topo_2019.f90:2395-2491): bilinear Z on the DEM cell
// of (xx, yy), the cell index clamped at the last row and column.
float z_at(const TopoData& t, const std::vector<float>& z, float xx, float yy) {
    int ipx = (int)((xx - t.xmin) / t.dx + 1.f), ipy = (int)((yy - t.ymin) / t.dy + 1.f);
    ipx = std::min(std::max(ipx, 1), t.nx - 1);
    ipy = std::min(std::max(ipy, 1), t.ny - 1);
    const size_t n1 = (size_t)(ipy - 1) * t.nx + (ipx - 1), n2 = n1 + 1, n3 = n1 + 1 + t.nx, n4 = n1 + t.nx;
    const float xi = (xx - (t.xmin + (float)(ipx - 1) * t.dx)) / t.dx;
    const float eta = (yy - (t.ymin + (float)(ipy - 1) * t.dy)) / t.dy;
    return (((1.f - xi) * (1.f - eta)) * z[n1] + (xi * (1.f - eta)) * z[n2]) + (xi * eta) * z[n3] +
           ((1.f - xi) * eta) * z[n4];
}

// OutputMesh_Classic: the DEM nodes (1..npoig) and quadrilaterals, then the
// particles inside the domain as nodes npoig + i and point elements.
void write_gid_mesh(const std::string& path, const TopoData& t, const std::vector<float>& z, int n,
                    const std::vector<float>& x, const std::vector<int>& flag) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) throw std::runtime_error("cannot write " + path);
    const int npoig = t.nx * t.ny;
    std::fprintf(f, " MESH SPH_quads   dimension   3    ElemType Quadrilateral  Nnode 4 \n coordinates\n");
    for (int iy = 0; iy < t.ny; iy++)
        for (int ix = 0; ix < t.nx; ix++)
            std::fprintf(f, " %d %.9G %.9G %.9G\n", iy * t.nx + ix + 1, (double)(t.xmin + (float)ix * t.dx),
                         (double)(t.ymin + (float)iy * t.dy), (double)z[(size_t)iy * t.nx + ix]);
    for (int i = 0; i < n; i++) {
        if (flag[i]) continue;
        std::fprintf(f, " %d %.9G %.9G %.9G\n", npoig + i + 1, (double)x[2 * i], (double)x[2 * i + 1],
                     (double)z_at(t, z, x[2 * i], x[2 * i + 1]));
    }
    std::fprintf(f, " End coordinates\n Elements\n");
    int e = 0;
    for (int iy = 0; iy < t.ny - 1; iy++)
        for (int ix = 0; ix < t.nx - 1; ix++) {
            const int ip = iy * t.nx + ix + 1;
            std::fprintf(f, " %d %d %d %d %d    1 \n", ++e, ip, ip + 1, ip + t.nx + 1, ip + t.nx);
        }
    std::fprintf(f, " End elements\n MESH SPH_points dimension 3   ElemType Point  Nnode 1 \n Elements\n");
    for (int i = 0; i < n; i++) std::fprintf(f, " %d %d 1\n", i + 1, npoig + i + 1);
    std::fprintf(f, " End elements\n");
    std::fclose(f);
}

// OutputRes_Classic at one plot time: IDW averages (4x4 nodes around each
// particle, weights 1/(dist/distg)) of h and v at the DEM nodes; the
// particles' displacement from their first position (z from the current
// terrain) and velocity; with icpwp = 1 (pwp given) the IDW average of the
// pore pressure u as the "Pwp" result (SPH_SW_2019.f90:13363, 13436-13443).
void write_gid_results(FILE* f, double time, const TopoData& t, const std::vector<float>& z, int n,
                       const std::vector<float>& x, const std::vector<float>& v, const std::vector<float>& h,
                       const std::vector<int>& flag, const std::vector<float>& x00, const std::vector<float>& z00,
                       const std::vector<float>* pwp) {
    const int npoig = t.nx * t.ny;
    std::vector<float> a1(npoig, 0.f), a2(npoig, 0.f), a3(npoig, 0.f), a4(npoig, 0.f), a5(npoig, 0.f);
    const float distg = std::sqrt(t.dx * t.dx + t.dy * t.dy);
    for (int i = 0; i < n; i++) {
        if (flag[i]) continue;
        const float xx = x[2 * i], yy = x[2 * i + 1];
        const int ipx = (int)((xx - t.xmin) / t.dx + 1.f), ipy = (int)((yy - t.ymin) / t.dy + 1.f);
        for (int ix = std::max(1, ipx - 1); ix <= std::min(t.nx, ipx + 2); ix++)
            for (int iy = std::max(1, ipy - 1); iy <= std::min(t.ny, ipy + 2); iy++) {
                const int ip = (iy - 1) * t.nx + (ix - 1);
                float ddx = xx - (t.xmin + (float)(ix - 1) * t.dx);
                ddx = ddx * ddx;
                float ddy = yy - (t.ymin + (float)(iy - 1) * t.dy);
                ddy = ddy * ddy;
                float dist = std::max(1.e-6f, std::sqrt(ddx + ddy));
                dist = dist / distg;
                a1[ip] = a1[ip] + h[i] / dist;
                a5[ip] = a5[ip] + 1.f / dist;
                if (pwp) a4[ip] = a4[ip] + (*pwp)[i] / dist;
                a2[ip] = a2[ip] + v[2 * i] / dist;
                a3[ip] = a3[ip] + v[2 * i + 1] / dist;
            }
    }
    for (int ip = 0; ip < npoig; ip++)
        if (a5[ip] >= 1.e-6f) {
            a1[ip] = a1[ip] / a5[ip]; a2[ip] = a2[ip] / a5[ip]; a3[ip] = a3[ip] / a5[ip]; a4[ip] = a4[ip] / a5[ip];
        }
    std::fprintf(f, " Result \"height\" \"Height\" %.9G Vector OnNodes \"where\" \n Values \n", time);
    for (int ip = 0; ip < npoig; ip++)
        if (a1[ip] > 1.e-6f) std::fprintf(f, " %d 0. 0. %.9G\n", ip + 1, (double)a1[ip]);
    std::fprintf(f, " End Values \n Result \"dis\" \"Disp\" %.9G Vector OnNodes \"where\" \n Values  \n", time);
    for (int i = 0; i < n; i++) {
        if (flag[i]) continue;
        const float zp = z_at(t, z, x[2 * i], x[2 * i + 1]);
        std::fprintf(f, " %d %.9G %.9G %.9G\n", npoig + i + 1, (double)(x[2 * i] - x00[2 * i]),
                     (double)(x[2 * i + 1] - x00[2 * i + 1]), (double)(zp - z00[i]));
    }
    std::fprintf(f, " End Values \n Result \"vel\" \"veloc\" %.9G Vector OnNodes \"where\" \n Values \n", time);
    for (int ip = 0; ip < npoig; ip++)
        if (a1[ip] > 1.e-6f) std::fprintf(f, " %d %.9G %.9G 0.0\n", ip + 1, (double)a2[ip], (double)a3[ip]);
    for (int i = 0; i < n; i++)
        if (!flag[i]) std::fprintf(f, " %d %.9G %.9G 0.0\n", npoig + i + 1, (double)v[2 * i], (double)v[2 * i + 1]);
    std::fprintf(f, " End Values \n");
    if (pwp) {
        std::fprintf(f, " Result \"Pwp\" \"pwpress\" %.9G Vector OnNodes \"where\" \n Values \n", time);
        for (int ip = 0; ip < npoig; ip++)
            if (a1[ip] > 1.e-6f) std::fprintf(f, " %d 0.0 0.0 %.9G\n", ip + 1, (double)a4[ip]);
        std::fprintf(f, " End Values \n");
    }
    std::fflush(f);
}

int check(int st, const char* what) {
    if (st < 0) {
        std::fprintf(stderr, "%s: %s\n", what, gfsph_strerror(st));
        std::exit(2);
    }
    return st;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr,
                     "usage: %s <problem> [--dir D] [--topo NAME] [--out D] [--max-steps N] [--parse-only] [--dump FILE]\n",
                     argv[0]);
        return 1;
    }
    std::string problem = argv[1], dir, topo, out = ".";
    long long max_steps = -1;
    bool parse_only = false;
    std::string dump;
    for (int k = 2; k < argc; k++) {
        std::string a = argv[k];
        if (a == "--dir" && k + 1 < argc) dir = argv[++k];
        else if (a == "--topo" && k + 1 < argc) topo = argv[++k];
        else if (a == "--out" && k + 1 < argc) out = argv[++k];
        else if (a == "--max-steps" && k + 1 < argc) max_steps = std::atoll(argv[++k]);
        else if (a == "--parse-only") parse_only = true;
        else if (a == "--dump" && k + 1 < argc) dump = argv[++k];
        else { std::fprintf(stderr, "unknown argument %s\n", a.c_str()); return 1; }
    }
    if (topo.empty()) topo = problem;  // the reference asks for it on stdin (SPH_FEM_topo_2019.f90:181)
    try {
        static const char* const mexts[] = {".MASTER.dat", ".master.dat", ".MASTER.DAT", nullptr};
        static const char* const dexts[] = {".dat", ".DAT", nullptr};
        static const char* const texts[] = {".top", ".TOP", nullptr};
        static const char* const pexts[] = {".pts", ".PTS", nullptr};
        MasterDat m = read_master(find_file(dir, problem, mexts));
        if (m.if_sph != 1 || m.problem_type != 1 || m.integ_alg != 4)
            throw std::runtime_error("only SPH_ProblemType = 1 with SPH_t_Integ_Alg = 4 (RK45) is implemented");
        SwDat d = read_dat(find_file(dir, m.sph_name, dexts));
        TopoData t = read_top(find_file(dir, topo, texts));
        const bool restart = (d.icunk_s == 200);
        int dropped = 0;
        std::vector<float> x, v0, h, mass, hsml, pwp0;
        std::vector<int> itype;  // 1 soil, 2 water (ic_ws_Interact = 1)
        const bool wir = (d.ic_soil == 1 && d.ic_water == 1);
        double time0 = 0.0;
        Particles P;
        if (restart) {  // Get_Restart_Info_SW opens restart.dat whatever the problem name (:3307)
            RestartState R = read_restart(join(dir, "restart.dat"));
            for (int k : R.itype)
                if (k != 1 && !(k == 2 && wir))
                    throw std::runtime_error("restart.dat: itype " + std::to_string(k) +
                                             " (soil 1, and water 2 with ic_water = 1, are supported)");
            x = R.x; v0 = R.v; h = R.h; mass = R.mass; hsml = R.hsml; pwp0 = R.pwp; itype = R.itype;
            time0 = R.time;
        } else {
            auto add = [&](const Particles& Q, int type) {
                for (int i = 0; i < Q.n(); i++) {
                    if (!(Q.mass[i] > 0.f)) { dropped++; continue; }  // lattice nodes with no complete cell: zero volume
                    x.push_back(Q.x[2 * i]); x.push_back(Q.x[2 * i + 1]);
                    h.push_back(Q.h[i]); mass.push_back(Q.mass[i]); hsml.push_back(Q.hsml[i]);
                    itype.push_back(type);
                }
            };
            // Read_Source_plus_New opens problem_name_Global.pts whatever name the .dat gives (:5058-5061)
            P = read_pts(find_file(dir, problem, pexts), d.h_inf, d.icunk_s, t.xshift, t.yshift);
            add(P, 1);
            if (wir) {  // the water after the soil (npoin = npoin_s + npoin_w, :997); no expansion lines
                Particles W = read_pts(find_file(dir, d.water_pts_name, pexts), d.h_inf, 7, t.xshift, t.yshift);
                add(W, 2);
                P.total_volume += W.total_volume;
            }
            v0.assign(x.size(), 0.f);
        }
        int n_water = 0;
        for (int k : itype) n_water += (k == 2);
        const int n = (int)h.size();
        double total_volume = P.total_volume;
        if (restart)
            for (float mm : mass) total_volume += mm;
        if (parse_only) {
            std::printf("{\"title\": \"%s\", \"dt\": %g, \"time_end\": %g, \"plot_step\": %d, \"dt_sph\": %g, "
                        "\"ic_adapt\": %d, \"nx\": %d, \"ny\": %d, \"xmin\": %.6f, \"ymin\": %.6f, \"dx\": %g, \"dy\": %g, "
                        "\"ictop\": %d, \"fdiff\": %d, \"n\": %d, \"dropped\": %d, \"volume\": %.6f, \"hsml\": %g, "
                        "\"pa_sph\": %d, \"nnps\": %d, \"sle\": %d, \"skf\": %d, \"nfric\": %d, \"icpwp\": %d, \"pwp0rel\": %g, \"h_inf\": %g, "
                        "\"n_water\": %d, \"ws_interact\": %d, \"sw_alg\": %d, \"const\": [",
                        "", m.dt, m.time_end, m.plot_step, m.dt_sph, m.ic_adapt, t.nx, t.ny, (double)t.xmin,
                        (double)t.ymin, t.dx, t.dy, t.ictop, t.fdiff ? 1 : 0, n, dropped, total_volume,
                        n ? hsml[0] : 0.f, d.pa_sph, d.nnps, d.sle, d.skf, (int)(d.cst[4] + 0.01f), d.icpwp, d.pwp0rel, d.h_inf,
                        n_water, wir ? 1 : 0, d.ic_swalg);
            for (int k = 0; k < 60; k++) std::printf("%s%g", k ? ", " : "", d.cst[k]);
            double zsum = 0.0;
            for (float z : t.z) zsum += z;
            std::printf("], \"z_mean\": %.6f}\n", zsum / (double)t.z.size());
            return 0;
        }
        if (d.icpwp != 0 && d.icpwp != 1 && d.icpwp != 3)
            throw std::runtime_error("icpwp = " + std::to_string(d.icpwp) + " is not implemented (0, 1 and 3 are)");
        gfsph_params p;
        std::memset(&p, 0, sizeof(p));
        for (int k = 0; k < GFSPH_NCONST; k++) p.cst[k] = d.cst[k];
        p.pa_sph = d.pa_sph; p.nnps = d.nnps; p.sle = d.sle; p.skf = d.skf;
        p.summation_density = d.sum_den ? 1 : 0; p.average_velocity = d.av_vel ? 1 : 0;
        p.nor_density = d.nor_dens ? 1 : 0; p.ic_adapt = m.ic_adapt; p.h_inf = d.h_inf; p.dt = m.dt_sph;
        p.dem_deriv = t.fdiff ? 1 : 0;
        p.icpwp = d.icpwp;
        p.pwp0rel = d.pwp0rel;
        p.ws_interact = wir ? 1 : 0;  // Input_SW :947-951
        p.sw_alg = d.ic_swalg;
        gfsph_dem dem;
        std::memset(&dem, 0, sizeof(dem));
        dem.nx = t.nx; dem.ny = t.ny; dem.xmin = t.xmin; dem.ymin = t.ymin; dem.dx = t.dx; dem.dy = t.dy;
        dem.z = t.z.data();
        const bool erosion = d.cst[20] > 1.e-9f;
        const size_t npoig = (size_t)t.nx * t.ny;
        std::vector<float> topol;
        if (restart && erosion) {
            // Input_SW (SPH_SW_2019.f90:1289-1301): the slopes of the .top DEM,
            // Z and the eroded depth of restart.top, then the erodible depth
            // set anew to const(48) (or 999) whatever restart.top holds
            topol.assign(npoig * GFSPH_NTOPO, 0.f);
            for (size_t ip = 0; ip < npoig; ip++) topol[ip * GFSPH_NTOPO] = t.z[ip];
            check(gfsph_dem_topol(p.dem_deriv, t.nx, t.ny, t.dx, t.dy, topol.data()), "gfsph_dem_topol");
            TopoRestart tr = read_topo_restart(join(dir, "restart.top"), (int)npoig);
            const float avail = (d.cst[47] > 1.e-6f) ? d.cst[47] : 999.f;
            for (size_t ip = 0; ip < npoig; ip++) {
                topol[ip * GFSPH_NTOPO] = tr.z[ip];
                topol[ip * GFSPH_NTOPO + 13] = tr.eroded[ip];
                topol[ip * GFSPH_NTOPO + 14] = avail;
            }
            dem.topol = topol.data();
            dem.ntopo = GFSPH_NTOPO;
        }
        if (!dump.empty()) {
            FILE* f = std::fopen(dump.c_str(), "wb");
            if (!f) throw std::runtime_error("cannot write " + dump);
            const int ver = 2, psz = (int)sizeof(p);
            std::fwrite("GFSPHDMP", 1, 8, f);
            std::fwrite(&ver, 4, 1, f); std::fwrite(&psz, 4, 1, f); std::fwrite(&p, sizeof(p), 1, f);
            std::fwrite(&t.nx, 4, 1, f); std::fwrite(&t.ny, 4, 1, f);
            std::fwrite(&t.xmin, 4, 1, f); std::fwrite(&t.ymin, 4, 1, f);
            std::fwrite(&t.dx, 4, 1, f); std::fwrite(&t.dy, 4, 1, f);
            std::fwrite(t.z.data(), 4, t.z.size(), f);
            std::fwrite(&n, 4, 1, f);
            std::fwrite(x.data(), 4, x.size(), f); std::fwrite(v0.data(), 4, v0.size(), f);
            std::fwrite(h.data(), 4, h.size(), f); std::fwrite(mass.data(), 4, mass.size(), f);
            std::fwrite(hsml.data(), 4, hsml.size(), f);
            std::fwrite(itype.data(), 4, itype.size(), f);  // version 2: the material per particle
            std::fclose(f);
            return 0;
        }
        gfsph_handle* hd = nullptr;
        check(gfsph_create(&p, &dem, &hd), "gfsph_create");
        check(gfsph_upload(hd, n, x.data(), v0.data(), h.data(), mass.data(), hsml.data(), itype.data(), nullptr),
              "gfsph_upload");
        if (restart) {
            if (d.icpwp != 0) check(gfsph_set_pwp(hd, pwp0.data()), "gfsph_set_pwp");
            check(gfsph_set_time(hd, time0, m.dt_sph), "gfsph_set_time");
        }
        check(gfsph_hazard_reset(hd), "gfsph_hazard_reset");
        // a zero cadence turns the output off (it would stop every step at t)
        const double never = 1e300;
        const double time_plot = (m.plot_step > 0 && m.dt > 0.f) ? (double)m.plot_step * (double)m.dt : never;
        const double time_save = (m.save_step > 0 && m.dt > 0.f) ? (double)m.save_step * (double)m.dt : never;
        const std::string logp = join(out, problem + ".gfsph.log");
        FILE* log = std::fopen(logp.c_str(), "w");
        if (!log) throw std::runtime_error("cannot write " + logp);
        std::fprintf(log, "# plot time steps volume max_depth max_speed inside\n");
        double tnow = time0;
        long long total = 0;
        int iplot = 0;
        std::vector<float> rx(2 * (size_t)n), rv(2 * (size_t)n), rh(n), rm(n), rs(n), rp(n);
        std::vector<int> rf(n);
        std::vector<float> raster(npoig), zcur(t.z);
        // the GiD mesh with the particles' first positions (OutputMesh_Classic)
        const std::vector<float> x00 = x;
        std::vector<float> z00(n);
        std::vector<int> noflag(n, 0);
        if (erosion) check(gfsph_raster(hd, GFSPH_RASTER_Z, zcur.data()), "gfsph_raster");
        for (int i = 0; i < n; i++) z00[i] = z_at(t, zcur, x[2 * i], x[2 * i + 1]);
        write_gid_mesh(join(out, problem + ".post.msh"), t, zcur, n, x, noflag);
        const std::string resp = join(out, problem + ".post.res");
        FILE* gid = std::fopen(resp.c_str(), "w");
        if (!gid) throw std::runtime_error("cannot write " + resp);
        std::fprintf(gid, "GiD Post Results File 1.0\n");
        auto save = [&]() {  // OutputSave_SW: the state in the caller's order
            check(gfsph_download(hd, rx.data(), rv.data(), rh.data(), rm.data(), rs.data(), rf.data()), "gfsph_download");
            RestartState R;
            R.time = tnow;
            R.itype = itype;
            R.x = rx; R.v = rv; R.h = rh; R.mass = rm; R.hsml = rs;
            R.pwp.assign(n, 0.f);
            if (d.icpwp != 0) check(gfsph_get_pwp(hd, R.pwp.data()), "gfsph_get_pwp");
            write_restart(join(out, problem + ".restart.dat"), R);
            if (erosion) {
                TopoRestart T;
                T.time = tnow;
                T.z.resize(npoig); T.eroded.resize(npoig); T.avail.resize(npoig);
                check(gfsph_raster(hd, GFSPH_RASTER_Z, T.z.data()), "gfsph_raster");
                check(gfsph_raster(hd, GFSPH_RASTER_ERODED, T.eroded.data()), "gfsph_raster");
                check(gfsph_raster(hd, GFSPH_RASTER_AVAILABLE, T.avail.data()), "gfsph_raster");
                write_topo_restart(join(out, problem + ".restart.top"), T);
            }
        };
        // DTGT (SPH_FEM_Driver_2019.f90:1580-1697): plot when plot_step * dt
        // has passed since the last plot, save when save_step * dt has
        // passed since the last save (t_plot_reset, t_save_reset :1583-1585)
        double next_plot = tnow + time_plot, next_save = tnow + time_save;
        bool stopped_by_steps = false;
        while (tnow < (double)m.time_end) {
            if (max_steps >= 0 && total >= max_steps) { stopped_by_steps = true; break; }
            int budget = (max_steps < 0) ? 1000000000 : (int)std::min<long long>(max_steps - total, 1000000000LL);
            int done = 0;
            const double t_stop = std::min(std::min(next_plot, next_save), (double)m.time_end);
            int st = gfsph_step(hd, budget, t_stop, &tnow, &done);
            // every particle has left the DEM: the run ends with this plot time
            const bool all_left = (st == GFSPH_ERR_DOMAIN);
            if (!all_left) check(st, "gfsph_step");
            total += done;
            if (tnow >= next_plot || all_left) {
                check(gfsph_download(hd, rx.data(), rv.data(), rh.data(), rm.data(), rs.data(), rf.data()),
                      "gfsph_download");
                check(gfsph_hazard_sample(hd), "gfsph_hazard_sample");
                double vol = 0.0, hmax = 0.0, vmax = 0.0;
                int inside = 0;
                for (int i = 0; i < n; i++) {
                    vol += rm[i];
                    if (rf[i]) continue;
                    inside++;
                    hmax = std::max(hmax, (double)rh[i]);
                    vmax = std::max(vmax, std::hypot((double)rv[2 * i], (double)rv[2 * i + 1]));
                }
                std::fprintf(log, "%d %.6f %lld %.6f %.6f %.6f %d\n", iplot, tnow, total, vol, hmax, vmax, inside);
                std::fflush(log);
                check(gfsph_raster(hd, GFSPH_RASTER_DEPTH_IDW, raster.data()), "gfsph_raster");
                char name[64];
                std::snprintf(name, sizeof(name), ".depth_%04d.asc", iplot);
                write_asc(join(out, problem + name), t, raster);
                if (erosion) check(gfsph_raster(hd, GFSPH_RASTER_Z, zcur.data()), "gfsph_raster");
                if (d.icpwp == 1) check(gfsph_get_pwp(hd, rp.data()), "gfsph_get_pwp");
                write_gid_results(gid, tnow, t, zcur, n, rx, rv, rh, rf, x00, z00, d.icpwp == 1 ? &rp : nullptr);
                iplot++;
                next_plot = tnow + time_plot;
            }
            if (tnow >= next_save || all_left) {
                save();
                next_save = tnow + time_save;
            }
            if (all_left) {
                std::printf("gfsph_run: every particle has left the DEM at t = %.4f s\n", tnow);
                break;
            }
        }
        if (stopped_by_steps) save();  // the state where --max-steps ended the run, for a restart
        std::fclose(gid);
        check(gfsph_raster(hd, GFSPH_RASTER_MAX_DEPTH, raster.data()), "gfsph_raster");
        write_asc(join(out, problem + ".max_depth.asc"), t, raster);
        check(gfsph_raster(hd, GFSPH_RASTER_MAX_VEL, raster.data()), "gfsph_raster");
        write_asc(join(out, problem + ".max_velocity.asc"), t, raster);
        std::fclose(log);
        std::printf("gfsph_run: %s, %d particles, %lld steps, t = %.4f s, %d plot times\n", problem.c_str(), n, total,
                    tnow, iplot);
        gfsph_destroy(hd);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "gfsph_run: %s\n", e.what());
        return 2;
    }
    return 0;
}
