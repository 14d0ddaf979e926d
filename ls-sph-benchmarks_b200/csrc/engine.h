// engine.h -- internal declarations of the LS-SPH engine (not part of the C ABI).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/lssph.h"

namespace lssph {

constexpr double kPi = 3.14159265358979323846;  // == acos(-1.0d0)

// Thread-local message for calls without a handle.
void set_last_error(const std::string& msg);
const std::string& last_error();

// ---- host-side reference restatements used by the engine (host.cpp) ----
double kernel_norm(int kernel_type, double h);                   // 7/(4 pi h^2) etc.
double kernel_W_host(int kernel_type, double r, double h);       // cal_W
void   init_param(lssph_params* p);                              // init_param_mod.f90:92-199
int    check_param(const lssph_params* p, std::string* msg);     // check_param_mod.f90:22-284
void   default_params(lssph_params* p);                          // shipped config.h
int    parse_config(const char* path, lssph_params* p, std::string* msg);
int    closed_box_counts(const lssph_params* p, int* num_total, int* num_int);
int    setup_particles(const lssph_params* p, int num_total, int32_t* ptype, double* x, double* y,
                       double* u, double* v, double* rho, double* pre, double* tem, std::string* msg);

// Virtual markers (init_virtual_markers_mod.f90:59-137) for ghosts num_int..num_total-1.
struct VirtualMarkers {
    std::vector<int32_t> ptype;
    std::vector<double> x, y, nx, ny;
};
int build_virtual_markers(const lssph_params* p, int num_total, int num_int, const int32_t* ptype,
                          const double* x, const double* y, VirtualMarkers* vm, std::string* msg);

// Static cell-grid description built on the host (init_cell_mod.f90:36-180).
struct CellGrid {
    int nx = 0, ny = 0, ncell = 0;
    int capacity = 0;   // max particles per cell at init (all particles, division keys)
    int cap = 0;        // slot capacity per cell on the device (>= 2 * capacity)
    double inv_cw = 0.0;   // periodic domain: 1 / cell width (cells L / n >= h_eff, n even)
    std::vector<int32_t> ghost_key;    // [num_ext] 0-based cell of each ghost (division)
    std::vector<int32_t> vm_key;       // [num_ext] 0-based cell of each virtual marker
    std::vector<int32_t> gstart;       // [ncell+1] CSR of ghosts per cell
    std::vector<int32_t> glist;        // [num_ext] ghost particle indices, ascending per cell
};
int build_cell_grid(const lssph_params* p, int num_total, int num_int, const double* x,
                    const double* y, const VirtualMarkers& vm, CellGrid* g, std::string* msg);

// Formatting of Fortran edit descriptors used by write_param_mod.f90.
std::string fortran_e21_14(double v);

// results/ layout (write_data_mod.f90, write_param_mod.f90, restart_mod.f90)
int write_data_file(const std::string& path, int num_total, bool with_tem, const int32_t* ptype,
                    const double* x, const double* y, const double* u, const double* v,
                    const double* rho, const double* pre, const double* tem, std::string* msg);
int write_parameters_csv(const std::string& path, const lssph_params* p, int num_total, int num_int,
                         int num_ext, std::string* msg);
int make_dirs(const std::string& path);
int copy_file(const std::string& from, const std::string& to);

}  // namespace lssph
