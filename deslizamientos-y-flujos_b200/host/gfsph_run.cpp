// gfsph_run — a C++ stand-in for the Geoflow-SPH Fortran driver over the
// gfsph C ABI: reads the reference's <problem>.MASTER.dat, the SW .dat, the
// .top DEM and the .pts source, runs the DTGT loop (SPH_FEM_Driver_2019.f90:1580-1697)
// on the GPU with the reference's output cadence (plot_step * dt), and
// writes, at every plot time, a summary line and the depth raster (ESRI ASCII
// grid), and at the end the per-node maximum depth and velocity.
//
//   gfsph_run <problem> [--dir D] [--topo NAME] [--out D] [--max-steps N] [--parse-only] [--dump FILE]
//
// --dump writes the parsed run (params struct, DEM grid and elevations, the
// particles) to a binary file and exits: little-endian, "GFSPHDMP", int32
// version 1, int32 sizeof(gfsph_params), the params bytes, int32 nx, ny,
// float32 xmin, ymin, dx, dy, float32 z[nx*ny], int32 n, float32 x[2n],
// v[2n], rho[n], mass[n], hsml[n].
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
        // Read_Source_plus_New opens problem_name_Global.pts whatever name the .dat gives (:5058-5061)
        Particles P = read_pts(find_file(dir, problem, pexts), d.h_inf, d.icunk_s, t.xshift, t.yshift);
        int dropped = 0;
        std::vector<float> x, h, mass, hsml;
        for (int i = 0; i < P.n(); i++) {
            if (!(P.mass[i] > 0.f)) { dropped++; continue; }  // lattice nodes with no complete cell: zero volume
            x.push_back(P.x[2 * i]); x.push_back(P.x[2 * i + 1]);
            h.push_back(P.h[i]); mass.push_back(P.mass[i]); hsml.push_back(P.hsml[i]);
        }
        const int n = (int)h.size();
        if (parse_only) {
            std::printf("{\"title\": \"%s\", \"dt\": %g, \"time_end\": %g, \"plot_step\": %d, \"dt_sph\": %g, "
                        "\"ic_adapt\": %d, \"nx\": %d, \"ny\": %d, \"xmin\": %.6f, \"ymin\": %.6f, \"dx\": %g, \"dy\": %g, "
                        "\"ictop\": %d, \"fdiff\": %d, \"n\": %d, \"dropped\": %d, \"volume\": %.6f, \"hsml\": %g, "
                        "\"pa_sph\": %d, \"nnps\": %d, \"sle\": %d, \"skf\": %d, \"nfric\": %d, \"icpwp\": %d, \"pwp0rel\": %g, \"h_inf\": %g, "
                        "\"const\": [",
                        "", m.dt, m.time_end, m.plot_step, m.dt_sph, m.ic_adapt, t.nx, t.ny, (double)t.xmin,
                        (double)t.ymin, t.dx, t.dy, t.ictop, t.fdiff ? 1 : 0, n, dropped, P.total_volume,
                        n ? hsml[0] : 0.f, d.pa_sph, d.nnps, d.sle, d.skf, (int)(d.cst[4] + 0.01f), d.icpwp, d.pwp0rel, d.h_inf);
            for (int k = 0; k < 60; k++) std::printf("%s%g", k ? ", " : "", d.cst[k]);
            double zsum = 0.0;
            for (float z : t.z) zsum += z;
            std::printf("], \"z_mean\": %.6f}\n", zsum / (double)t.z.size());
            return 0;
        }
        if (d.icpwp != 0 && d.icpwp != 3)
            throw std::runtime_error("icpwp = " + std::to_string(d.icpwp) + " is not implemented (0 and 3 are)");
        gfsph_params p;
        std::memset(&p, 0, sizeof(p));
        for (int k = 0; k < GFSPH_NCONST; k++) p.cst[k] = d.cst[k];
        p.pa_sph = d.pa_sph; p.nnps = d.nnps; p.sle = d.sle; p.skf = d.skf;
        p.summation_density = d.sum_den ? 1 : 0; p.average_velocity = d.av_vel ? 1 : 0;
        p.nor_density = d.nor_dens ? 1 : 0; p.ic_adapt = m.ic_adapt; p.h_inf = d.h_inf; p.dt = m.dt_sph;
        p.dem_deriv = t.fdiff ? 1 : 0;
        p.icpwp = d.icpwp;
        p.pwp0rel = d.pwp0rel;
        gfsph_dem dem;
        std::memset(&dem, 0, sizeof(dem));
        dem.nx = t.nx; dem.ny = t.ny; dem.xmin = t.xmin; dem.ymin = t.ymin; dem.dx = t.dx; dem.dy = t.dy;
        dem.z = t.z.data();
        if (!dump.empty()) {
            FILE* f = std::fopen(dump.c_str(), "wb");
            if (!f) throw std::runtime_error("cannot write " + dump);
            const int ver = 1, psz = (int)sizeof(p);
            std::fwrite("GFSPHDMP", 1, 8, f);
            std::fwrite(&ver, 4, 1, f); std::fwrite(&psz, 4, 1, f); std::fwrite(&p, sizeof(p), 1, f);
            std::fwrite(&t.nx, 4, 1, f); std::fwrite(&t.ny, 4, 1, f);
            std::fwrite(&t.xmin, 4, 1, f); std::fwrite(&t.ymin, 4, 1, f);
            std::fwrite(&t.dx, 4, 1, f); std::fwrite(&t.dy, 4, 1, f);
            std::fwrite(t.z.data(), 4, t.z.size(), f);
            std::vector<float> vz(2 * (size_t)n, 0.f);
            std::fwrite(&n, 4, 1, f);
            std::fwrite(x.data(), 4, x.size(), f); std::fwrite(vz.data(), 4, vz.size(), f);
            std::fwrite(h.data(), 4, h.size(), f); std::fwrite(mass.data(), 4, mass.size(), f);
            std::fwrite(hsml.data(), 4, hsml.size(), f);
            std::fclose(f);
            return 0;
        }
        gfsph_handle* hd = nullptr;
        check(gfsph_create(&p, &dem, &hd), "gfsph_create");
        std::vector<float> v(2 * (size_t)n, 0.f);
        check(gfsph_upload(hd, n, x.data(), v.data(), h.data(), mass.data(), hsml.data(), nullptr, nullptr),
              "gfsph_upload");
        check(gfsph_hazard_reset(hd), "gfsph_hazard_reset");
        const double time_plot = (double)m.plot_step * (double)m.dt;
        const std::string logp = join(out, problem + ".gfsph.log");
        FILE* log = std::fopen(logp.c_str(), "w");
        if (!log) throw std::runtime_error("cannot write " + logp);
        std::fprintf(log, "# plot time steps volume max_depth max_speed inside\n");
        double tnow = 0.0;
        long long total = 0;
        int iplot = 0;
        std::vector<float> rx(2 * (size_t)n), rv(2 * (size_t)n), rh(n), rm(n), rs(n);
        std::vector<int> rf(n);
        std::vector<float> raster((size_t)t.nx * t.ny);
        while (tnow < (double)m.time_end && (max_steps < 0 || total < max_steps)) {
            int budget = (max_steps < 0) ? 1000000000 : (int)std::min<long long>(max_steps - total, 1000000000LL);
            int done = 0;
            int st = gfsph_step(hd, budget, tnow + time_plot, &tnow, &done);
            // every particle has left the DEM: the run ends with this plot time
            const bool all_left = (st == GFSPH_ERR_DOMAIN);
            if (!all_left) check(st, "gfsph_step");
            total += done;
            check(gfsph_download(hd, rx.data(), rv.data(), rh.data(), rm.data(), rs.data(), rf.data()), "gfsph_download");
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
            iplot++;
            if (all_left) {
                std::printf("gfsph_run: every particle has left the DEM at t = %.4f s\n", tnow);
                break;
            }
        }
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
