// Readers of the Geoflow-SPH input files, for a C++ host that stands in for
// the reference's Fortran driver: <name>.MASTER.dat (Driver_Input,
// SPH_FEM_Driver_2019.f90:218-409), <name>.dat (Input_SW, SPH_SW_2019.f90:668-1573),
// <topo>.top (Topo_main, SPH_FEM_topo_2019.f90:133-637) and <pts>.pts
// (Read_Source_plus_New, SPH_SW_2019.f90:4999-5272).  Only the subset of
// options on the implemented step is read; anything else is reported.
#pragma once
#include <string>
#include <vector>

namespace gfsph_host {

struct MasterDat {
    std::string title;
    int if_sph = 0, if_gfl = 0, ic_cases_mat = 0;
    int problem_type = 0, integ_alg = 0;
    std::string sph_name;
    float dt = 0.f, time_end = 0.f;
    int maxtimesteps = 0;
    int print_step = 0, save_step = 0, plot_step = 0;
    float dt_sph = 0.f;
    int ic_adapt = 0;
};

struct TopoData {
    int ictop = 0;
    bool fdiff = false;         // ictop >= 100: slopes by finite differences
    int nx = 0, ny = 0;
    float xmin = 0.f, ymin = 0.f, dx = 0.f, dy = 0.f;
    float xshift = 0.f, yshift = 0.f;
    std::vector<float> z;       // nx*ny, x fastest
    std::vector<int> in_model;  // poig_in_model
};

struct SwDat {
    int ic_swalg = 0, n_hist = 0, ndimn = 2;
    int ic_soil = 1, ic_water = 0, ic_vps = 0, ic_abs = 0;
    int icunk_s = 7;            // 7, 8: .pts source; 200: restart (Get_Restart_Info_SW)
    float h_inf = 0.01f;
    std::string pts_name;       // the .pts name, or the problem name of a restart
    int icunk_w = 0;            // water points (Get_water_points): 7, 8 a .pts source
    std::string water_pts_name; // the water .pts name (Read_Source_plus_New_WATER :5329-5336)
    int pa_sph = 2, nnps = 2, sle = 1, skf = 1;
    bool sum_den = true, av_vel = true, virt_part = false, nor_dens = false;
    float cst[110] = {};        // const(1..110)
    int ic_k0 = 0;
    int icpwp = 0;
    float pwp0rel = 0.f;        // icpwp = 3
};

struct Particles {
    std::vector<float> x;       // (2, n)
    std::vector<float> h, mass, hsml;
    float delt2d = 0.f, facthsml = 0.f;
    int np_src = 0;
    double total_volume = 0.0;
    int n() const { return (int)h.size(); }
};

// A restart state: OutputSave_SW writes it (SPH_SW_2019.f90:12416-12460),
// Get_Restart_Info_SW reads it (:3270-3337) when icunk_s = 200.
struct RestartState {
    double time = 0.0;
    std::vector<int> itype;
    std::vector<float> x, v;    // (2, n)
    std::vector<float> h, mass, hsml, pwp;
    int n() const { return (int)h.size(); }
};

// The eroded DEM rows of a restart: Topol(1), Topol(14), Topol(15) per node
// (OutputSave_SW :12473-12481, Get_Topo_restart SPH_FEM_topo_2019.f90:2883-2920).
struct TopoRestart {
    double time = 0.0;
    std::vector<float> z, eroded, avail;
};

// Each reader throws std::runtime_error with the file and the item on failure.
MasterDat read_master(const std::string& path);
TopoData read_top(const std::string& path);
SwDat read_dat(const std::string& path);
Particles read_pts(const std::string& path, float h_inf, int icunk_s, float xshift, float yshift);
RestartState read_restart(const std::string& path);
TopoRestart read_topo_restart(const std::string& path, int npoig);
// Writers of the same files.  The fields and their order are the
// reference's; the numbers carry 9 significant digits (17 for the time)
// instead of its g14.7, so that an FP32 state is read back bit for bit (the
// reference reads these files list-directed, whatever the width).
void write_restart(const std::string& path, const RestartState& s);
void write_topo_restart(const std::string& path, const TopoRestart& t);

// Fortran list-directed and a60-label reading over a text file.
class FortranReader {
  public:
    explicit FortranReader(const std::string& path);
    std::string label();                    // one whole line (format a60)
    std::vector<std::string> values(int n); // n list-directed items, over as many lines as needed
    int read_int();
    float read_real();
    bool read_logical();
    const std::string& path() const { return path_; }

  private:
    std::vector<std::string> lines_;
    size_t line_ = 0;
    std::string path_;
};

}  // namespace gfsph_host
