// host.cpp -- host side of the LS-SPH engine: the config.h parameter surface, particle
// setup and the results/ file layout of LS-SPH-Benchmarks, behind the C ABI of lssph.h.
//
// These run once per solve (or once per snapshot) and are restated from the reference
// Fortran so that a handle built here starts from exactly the state the reference
// builds:
//   init_param         source/setup/init_param_mod.f90:92-199
//   check_param        source/check/check_param_mod.f90:22-284
//   setup_closed_box   source/setup/setup_closed_box_mod.f90:72-235
//   impose_*           source/setup/impose_initial_conditions_mod.f90
//   virtual markers    source/setup/init_virtual_markers_mod.f90:59-137
//   cell grid          source/neighbor/init_cell_mod.f90:36-180
//   write_data         source/io/write_data_mod.f90:22-55
//   write_param        source/io/write_param_mod.f90:27-162
//   restart            source/setup/restart_mod.f90:22-53

#include "engine.h"

#include <sys/stat.h>
#include <sys/types.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>

namespace lssph {

namespace {
thread_local std::string g_last_error;

// Powers as products, the convention shared by every kernel-function evaluation here.
inline double p2(double t) { return t * t; }
}  // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }
const std::string& last_error() { return g_last_error; }

double kernel_norm(int kt, double h) {
    const double hh = h * h;
    switch (kt) {
        case 1: return 5.0 / ((14.0 * kPi) * hh);
        case 2: return 7.0 / ((478.0 * kPi) * hh);
        case 3: return 7.0 / ((4.0 * kPi) * hh);
        case 4: return 9.0 / ((4.0 * kPi) * hh);
        default: return 39.0 / ((14.0 * kPi) * hh);
    }
}

// cal_W (kernel_functions_mod.f90:26-81); used for W_ave = W(dx, h).
double kernel_W_host(int kt, double r, double h) {
    const double q = r * (1.0 / h);   // a division by the loop-invariant h as a reciprocal multiply
    double W = 0.0;
    if (kt == 1) {
        const double a = 2.0 - q, b = 1.0 - q, a3 = p2(a) * a, b3 = p2(b) * b;
        if (0.0 <= q && q <= 1.0) W = a3 - 4.0 * b3;
        else if (1.0 < q && q <= 2.0) W = a3;
    } else if (kt == 2) {
        const double a = 3.0 - q, b = 2.0 - q, c = 1.0 - q;
        const double a5 = p2(p2(a)) * a, b5 = p2(p2(b)) * b, c5 = p2(p2(c)) * c;
        if (0.0 <= q && q <= 1.0) W = (a5 - 6.0 * b5) + 15.0 * c5;
        else if (1.0 < q && q <= 2.0) W = a5 - 6.0 * b5;
        else if (2.0 < q && q <= 3.0) W = a5;
    } else if (kt == 3) {
        if (0.0 <= q && q <= 2.0) {
            const double t = 1.0 - 0.5 * q, t4 = p2(p2(t));
            W = t4 * (1.0 + 2.0 * q);
        }
    } else if (kt == 4) {
        if (0.0 <= q && q <= 2.0) {
            const double t = 1.0 - 0.5 * q, t4 = p2(p2(t)), t6 = t4 * p2(t);
            W = t6 * ((1.0 + 3.0 * q) + (35.0 * (q * q)) / 12.0);
        }
    } else {
        if (0.0 <= q && q <= 2.0) {
            const double t = 1.0 - 0.5 * q, t4 = p2(p2(t)), t8 = t4 * t4;
            const double q2 = q * q, q3 = q2 * q;
            W = t8 * (((1.0 + 4.0 * q) + (25.0 * q2) / 4.0) + 4.0 * q3);
        }
    }
    return kernel_norm(kt, h) * W;
}

// Values of the config.h shipped with the reference.
void default_params(lssph_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->target_problem = 2;
    p->u_bc_top = 1; p->u_bc_bottom = 1; p->u_bc_left = 1; p->u_bc_right = 1;
    p->tem_bc_top = 1; p->tem_bc_bottom = 1; p->tem_bc_left = 2; p->tem_bc_right = 2;
    p->u_top = 1.0;
    p->tem_top = 0.0; p->tem_bottom = 1.0e-2; p->tem_left = 0.0; p->tem_right = 0.0;
    std::snprintf(p->save_name, sizeof(p->save_name), "%s", "tg_compare_100_write");
    std::snprintf(p->read_name, sizeof(p->read_name), "%s", "new");
    p->omp_threads = 8;
    p->len_x = 1.0; p->len_y = 1.0;
    p->num_x = 100; p->num_y = 100;
    p->rk = 4;
    p->start_step = 1; p->end_step = 10000; p->write_step = 100;
    p->threshold = 1.0e-10;
    p->coe_CFL = 0.5; p->coe_dif = 0.2;
    p->zeta_RSST = 1.0; p->xi_VIM = 1.0;
    p->rho_ref = 1.0; p->vis_ref = 1.0e-2; p->K_ref = 1.0e2;
    p->k_th_ref = 1.0e-2; p->cp_ref = 1.0e3; p->alpha_ref = 7.1e-3;
    p->gravity = 10.0; p->pos_pert = 0.0;
    p->tg_a = 1; p->tg_b = 1;
    p->coe_h = 1.2; p->PST_c = 1.5; p->coe_delta_sph = 0.0;
    p->kernel_type = 3; p->sph_model = 3; p->wall_model = 2;
    p->precision = LSSPH_PRECISION_FP64;
    p->lanes = 0;
    p->seed = 0;
    init_param(p);
}

// init_param_mod.f90:92-199
void init_param(lssph_params* p) {
    p->total_step = (std::strcmp(p->read_name, "new") == 0) ? p->end_step : p->end_step - p->start_step;
    p->dx = p->len_x / (double)p->num_x;
    p->SP_mass = p->rho_ref * (p->dx * p->dx);
    p->h = p->coe_h * p->dx;
    p->h_eff = (p->kernel_type == 2) ? 3.0 * p->h : 2.0 * p->h;
    p->W_ave = kernel_W_host(p->kernel_type, p->dx, p->h);
    p->num_WL = (int32_t)std::ceil(p->h_eff / p->dx);
    if (p->periodic) p->num_WL = 0;   // no wall layers in a periodic domain
    p->WL_thick = (double)p->num_WL * p->dx;
    if (p->target_problem == 4) {
        p->delta_tem = p->tem_bottom - p->tem_top;
        p->tem_ave = 0.5 * (p->tem_bottom + p->tem_top);
    } else {
        p->delta_tem = 0.0;
        p->tem_ave = 0.0;
    }
    p->sound_speed = std::sqrt(p->K_ref / p->rho_ref);
    p->kinematic_vis = (p->target_problem == 1) ? 1.0 : p->vis_ref / p->rho_ref;
    p->thermal_dif = p->k_th_ref / (p->rho_ref * p->cp_ref);
    p->Re = (p->target_problem == 2) ? (1.0 * p->len_x) / p->kinematic_vis
                                     : (p->u_top * p->len_x) / p->kinematic_vis;
    p->Ra = (((p->alpha_ref * p->delta_tem) * p->gravity) * ((p->len_y * p->len_y) * p->len_y)) /
            (p->kinematic_vis * p->thermal_dif);
    p->Pr = p->kinematic_vis / p->thermal_dif;
    p->dt_CFL = p->coe_CFL * (p->dx / p->sound_speed);
    p->dt_vis = p->coe_dif * ((p->dx * p->dx) / p->kinematic_vis);
    p->dt_th = p->coe_dif * ((p->dx * p->dx) / p->thermal_dif);
    p->dt_CFL_relax = (p->dt_CFL * p->zeta_RSST) * p->xi_VIM;
    p->dt_vis_relax = p->dt_vis * (p->xi_VIM * p->xi_VIM);
    if (p->target_problem == 1) p->dt = p->dt_vis;
    else if (p->target_problem == 4) p->dt = std::min(std::min(p->dt_CFL_relax, p->dt_vis_relax), p->dt_th);
    else p->dt = std::min(p->dt_CFL_relax, p->dt_vis_relax);
}

// check_param_mod.f90:22-284 (each `error stop` becomes LSSPH_E_BAD_PARAM + message)
int check_param(const lssph_params* p, std::string* msg) {
    auto fail = [&](const char* m) { if (msg) *msg = m; return LSSPH_E_BAD_PARAM; };
    if (p->target_problem < 1 || p->target_problem > 4) return fail("TARGET_PROBLEM must be between 1 and 4.");
    if (p->kernel_type < 1 || p->kernel_type > 5) return fail("KERNEL_TYPE must be between 1 and 5.");
    if (p->sph_model < 1 || p->sph_model > 6) return fail("SPH_MODEL must be between 1 and 6.");
    if (p->wall_model < 1 || p->wall_model > 3) return fail("WALL_MODEL must be between 1 and 3.");
    if (p->rk != 2 && p->rk != 4) return fail("RK must be 2 or 4.");
    auto in12 = [](int b) { return b == 1 || b == 2; };
    if (p->target_problem == 1 &&
        !(in12(p->u_bc_top) && in12(p->u_bc_bottom) && in12(p->u_bc_left) && in12(p->u_bc_right)))
        return fail("TARGET_PROBLEM: Diffusion Equation Test - U_BOUNDARY_* must be 1 or 2.");
    if (p->target_problem == 2 &&
        !(p->u_bc_top == 1 && p->u_bc_bottom == 1 && p->u_bc_left == 1 && p->u_bc_right == 1))
        return fail("TARGET_PROBLEM: Taylor-Green Vortex - U_BOUNDARY_* must be 1.");
    if (p->target_problem == 3 &&
        !(p->u_bc_top == 3 && p->u_bc_bottom == 2 && p->u_bc_left == 2 && p->u_bc_right == 2))
        return fail("TARGET_PROBLEM: Lid-driven Cavity Flow - U_BOUNDARY_TOP must be 3, all other U_BOUNDARY_* must be 2.");
    if (p->target_problem == 4 &&
        !(in12(p->u_bc_top) && in12(p->u_bc_bottom) && in12(p->u_bc_left) && in12(p->u_bc_right) &&
          p->tem_bc_top == 1 && p->tem_bc_bottom == 1 && p->tem_bc_left == 2 && p->tem_bc_right == 2))
        return fail("TARGET_PROBLEM: Boussinesq Convection - U_BOUNDARY_* must be 1 or 2, TEM_BOUNDARY_TOP and _BOTTOM must be 1, TEM_BOUNDARY_LEFT and _RIGHT must be 2.");
    if (p->target_problem == 1 && (p->len_x != 1.0 || p->len_y != 1.0))
        return fail("For Diffusion Equation Test, LEN_X and LEN_Y must be exactly 1.0.");
    if (p->target_problem == 2 && (p->tg_a <= 0 || p->tg_b <= 0)) return fail("TG_A and TG_B must be positive.");
    if (p->len_x <= 0.0 || p->len_y <= 0.0) return fail("LEN_X and LEN_Y must be positive.");
    if (p->num_x <= 0 || p->num_y <= 0) return fail("NUM_X and NUM_Y must be positive.");
    if (p->start_step <= 0 || p->end_step <= 0 || p->write_step <= 0)
        return fail("START_STEP, END_STEP and WRITE_STEP must be positive.");
    if (p->start_step >= p->end_step) return fail("START_STEP must be less than END_STEP.");
    if (p->coe_CFL <= 0.0 || p->coe_dif <= 0.0 || p->coe_CFL >= 1.0 || p->coe_dif >= 1.0)
        return fail("COE_CFL and COE_DIF must be between 0 and 1.");
    if (p->zeta_RSST < 1.0 || p->xi_VIM < 1.0) return fail("ZETA_RSST and XI_VIM must be 1.0 or greater.");
    if (p->rho_ref <= 0.0 || p->vis_ref <= 0.0 || p->K_ref <= 0.0 || p->k_th_ref <= 0.0 ||
        p->cp_ref <= 0.0 || p->alpha_ref <= 0.0)
        return fail("Physical properties must be positive.");
    if (p->gravity < 0.0) return fail("GRAVITY must be non-negative.");
    if (p->target_problem == 1 && (p->pos_pert < 0.0 || p->pos_pert >= 0.5))
        return fail("POS_PERT must be between 0.0 and 0.5");
    if (p->coe_h <= 0.0) return fail("COE_H must be positive.");
    if (p->PST_c < 0.0 || p->coe_delta_sph < 0.0) return fail("PST_C and COE_DELTA_SPH must be non-negative.");
    const double dx = p->len_x / (double)p->num_x, dy = p->len_y / (double)p->num_y;
    if (std::fabs(dx - dy) > 1.0e-8) return fail("Particle spacing must be isotropic (dx == dy).");
    if (p->precision != LSSPH_PRECISION_FP64 && p->precision != LSSPH_PRECISION_MIXED &&
        p->precision != LSSPH_PRECISION_MIXED_COMPENSATED)
        return fail("precision must be LSSPH_PRECISION_FP64, LSSPH_PRECISION_MIXED or "
                    "LSSPH_PRECISION_MIXED_COMPENSATED.");
    if (!(p->lanes == 0 || p->lanes == 1 || p->lanes == 2 || p->lanes == 4 || p->lanes == 8))
        return fail("lanes must be 0 (auto), 1, 2, 4 or 8.");
    if (p->periodic != 0 && p->periodic != 1) return fail("periodic must be 0 or 1.");
    if (p->periodic) {
        if (p->target_problem != 1 && p->target_problem != 2)
            return fail("A periodic domain is available for problems 1 and 2 (no walls).");
        if (p->len_x != p->len_y || p->num_x != p->num_y)
            return fail("A periodic domain must be square (LEN_X == LEN_Y, NUM_X == NUM_Y).");
        if (p->h_eff > 0.0 && p->len_x < 4.0 * p->h_eff)
            return fail("A periodic domain needs LEN_X >= 4 h_eff.");
    }
    return LSSPH_OK;
}

// ---------------------------------------------------------------------------------
// config.h parser: `#define NAME value` lines; C comments removed; Fortran double
// literals (1.0d-2) accepted; strings in double quotes.
// ---------------------------------------------------------------------------------
namespace {
std::string strip_comments(const std::string& src) {
    std::string out;
    out.reserve(src.size());
    for (size_t i = 0; i < src.size();) {
        if (src.compare(i, 2, "/*") == 0) {
            size_t e = src.find("*/", i + 2);
            i = (e == std::string::npos) ? src.size() : e + 2;
        } else if (src.compare(i, 2, "//") == 0) {
            size_t e = src.find('\n', i);
            i = (e == std::string::npos) ? src.size() : e;
        } else {
            out.push_back(src[i++]);
        }
    }
    return out;
}

bool parse_fortran_double(std::string s, double* out) {
    for (auto& c : s) if (c == 'd' || c == 'D') c = 'e';
    char* end = nullptr;
    errno = 0;
    const double v = std::strtod(s.c_str(), &end);
    if (end == s.c_str() || *end != '\0' || errno != 0) return false;
    *out = v;
    return true;
}

bool parse_int(const std::string& s, int32_t* out) {
    char* end = nullptr;
    errno = 0;
    const long v = std::strtol(s.c_str(), &end, 10);
    if (end == s.c_str() || *end != '\0' || errno != 0) return false;
    *out = (int32_t)v;
    return true;
}
}  // namespace

int parse_config(const char* path, lssph_params* p, std::string* msg) {
    std::ifstream f(path);
    if (!f) { if (msg) *msg = std::string("cannot open config file: ") + path; return LSSPH_E_IO; }
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = strip_comments(ss.str());
    std::map<std::string, std::string> defs;
    std::istringstream lines(text);
    std::string line;
    while (std::getline(lines, line)) {
        std::istringstream ls(line);
        std::string tok, name, value;
        if (!(ls >> tok) || tok != "#define") continue;
        if (!(ls >> name)) continue;
        std::getline(ls, value);
        const size_t b = value.find_first_not_of(" \t\r");
        const size_t e = value.find_last_not_of(" \t\r");
        value = (b == std::string::npos) ? "" : value.substr(b, e - b + 1);
        defs[name] = value;
    }
    default_params(p);
    struct IntField { const char* name; int32_t* dst; };
    struct DblField { const char* name; double* dst; };
    const IntField ints[] = {
        {"TARGET_PROBLEM", &p->target_problem}, {"U_BOUNDARY_TOP", &p->u_bc_top},
        {"U_BOUNDARY_BOTTOM", &p->u_bc_bottom}, {"U_BOUNDARY_LEFT", &p->u_bc_left},
        {"U_BOUNDARY_RIGHT", &p->u_bc_right}, {"TEM_BOUNDARY_TOP", &p->tem_bc_top},
        {"TEM_BOUNDARY_BOTTOM", &p->tem_bc_bottom}, {"TEM_BOUNDARY_LEFT", &p->tem_bc_left},
        {"TEM_BOUNDARY_RIGHT", &p->tem_bc_right}, {"OMP_THREADS", &p->omp_threads},
        {"NUM_X", &p->num_x}, {"NUM_Y", &p->num_y}, {"RK", &p->rk}, {"START_STEP", &p->start_step},
        {"END_STEP", &p->end_step}, {"WRITE_STEP", &p->write_step}, {"TG_A", &p->tg_a},
        {"TG_B", &p->tg_b}, {"KERNEL_TYPE", &p->kernel_type}, {"SPH_MODEL", &p->sph_model},
        {"WALL_MODEL", &p->wall_model}, {"PERIODIC", &p->periodic}};
    const DblField dbls[] = {
        {"U_TOP", &p->u_top}, {"TEM_TOP", &p->tem_top}, {"TEM_BOTTOM", &p->tem_bottom},
        {"TEM_LEFT", &p->tem_left}, {"TEM_RIGHT", &p->tem_right}, {"LEN_X", &p->len_x},
        {"LEN_Y", &p->len_y}, {"THRESHOLD", &p->threshold}, {"COE_CFL", &p->coe_CFL},
        {"COE_DIF", &p->coe_dif}, {"ZETA_RSST", &p->zeta_RSST}, {"XI_VIM", &p->xi_VIM},
        {"RHO_REF", &p->rho_ref}, {"VIS_REF", &p->vis_ref}, {"K_REF", &p->K_ref},
        {"K_TH_REF", &p->k_th_ref}, {"CP_REF", &p->cp_ref}, {"ALPHA_REF", &p->alpha_ref},
        {"GRAVITY", &p->gravity}, {"POS_PERT", &p->pos_pert}, {"COE_H", &p->coe_h},
        {"PST_C", &p->PST_c}, {"COE_DELTA_SPH", &p->coe_delta_sph}};
    for (const auto& fi : ints) {
        auto it = defs.find(fi.name);
        if (it == defs.end()) continue;
        if (!parse_int(it->second, fi.dst)) {
            if (msg) *msg = std::string("bad integer for ") + fi.name + ": " + it->second;
            return LSSPH_E_BAD_PARAM;
        }
    }
    for (const auto& fd : dbls) {
        auto it = defs.find(fd.name);
        if (it == defs.end()) continue;
        if (!parse_fortran_double(it->second, fd.dst)) {
            if (msg) *msg = std::string("bad number for ") + fd.name + ": " + it->second;
            return LSSPH_E_BAD_PARAM;
        }
    }
    auto str_field = [&](const char* name, char* dst, size_t n) {
        auto it = defs.find(name);
        if (it == defs.end()) return;
        std::string v = it->second;
        if (v.size() >= 2 && v.front() == '"' && v.back() == '"') v = v.substr(1, v.size() - 2);
        std::snprintf(dst, n, "%s", v.c_str());
    };
    str_field("SAVE_NAME", p->save_name, sizeof(p->save_name));
    str_field("READ_NAME", p->read_name, sizeof(p->read_name));
    init_param(p);
    return check_param(p, msg);
}

// ---------------------------------------------------------------------------------
// Particle setup
// ---------------------------------------------------------------------------------
int closed_box_counts(const lssph_params* p, int* num_total, int* num_int) {
    const int nxf = p->num_x + 2 * p->num_WL, nyf = p->num_y + 2 * p->num_WL;
    // Interior particles are the lattice sites strictly inside the fluid box; the site
    // coordinates are cumulative sums (setup_closed_box_mod.f90:74-85), so count them the
    // same way rather than assuming num_x * num_y.
    std::vector<double> xs(nxf), ys(nyf);
    xs[0] = p->dx / 2.0;
    for (int i = 1; i < nxf; ++i) xs[i] = xs[i - 1] + p->dx;
    ys[0] = p->dx / 2.0;
    for (int j = 1; j < nyf; ++j) ys[j] = ys[j - 1] + p->dx;
    const double x_min = 0.0 + p->WL_thick, x_max = p->len_x + p->WL_thick;
    const double y_min = 0.0 + p->WL_thick, y_max = p->len_y + p->WL_thick;
    int nix = 0, niy = 0;
    for (int i = 0; i < nxf; ++i) if (x_min < xs[i] && x_max > xs[i]) ++nix;
    for (int j = 0; j < nyf; ++j) if (y_min < ys[j] && y_max > ys[j]) ++niy;
    *num_total = nxf * nyf;
    *num_int = nix * niy;
    return LSSPH_OK;
}

namespace {
struct SplitMix64 {  // seeded stand-in for the clock-seeded Fortran RNG
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};
}  // namespace

int setup_particles(const lssph_params* p, int num_total, int32_t* ptype, double* x, double* y,
                    double* u, double* v, double* rho, double* pre, double* tem, std::string* msg) {
    const int nxf = p->num_x + 2 * p->num_WL, nyf = p->num_y + 2 * p->num_WL, nf = nxf * nyf;
    if (num_total != nf) { if (msg) *msg = "num_total does not match the closed-box lattice"; return LSSPH_E_CAPACITY; }
    if (p->target_problem == 4 && !tem) { if (msg) *msg = "tem buffer required for problem 4"; return LSSPH_E_BAD_PARAM; }
    // 1. lattice with cumulative spacing (setup_closed_box_mod.f90:74-85)
    std::vector<double> xs(nf), ys(nf);
    xs[0] = p->dx / 2.0;
    ys[0] = p->dx / 2.0;
    for (int i = 1; i < nf; ++i) {
        if (i < nxf) { xs[i] = xs[i - 1] + p->dx; ys[i] = ys[i - 1]; }
        else { xs[i] = xs[i - nxf]; ys[i] = ys[i - nxf] + p->dx; }
    }
    // 2. interior first, ghosts after, both in scan order (:120-136)
    const double x_min = 0.0 + p->WL_thick, x_max = p->len_x + p->WL_thick;
    const double y_min = 0.0 + p->WL_thick, y_max = p->len_y + p->WL_thick;
    int ni = 0;
    std::vector<int> ext;
    ext.reserve(nf);
    for (int i = 0; i < nf; ++i) {
        if (x_min < xs[i] && x_max > xs[i] && y_min < ys[i] && y_max > ys[i]) {
            x[ni] = xs[i]; y[ni] = ys[i]; ++ni;
        } else {
            ext.push_back(i);
        }
    }
    for (size_t k = 0; k < ext.size(); ++k) { x[ni + k] = xs[ext[k]]; y[ni + k] = ys[ext[k]]; }
    for (int i = 0; i < nf; ++i) { u[i] = 0.0; v[i] = 0.0; rho[i] = 0.0; pre[i] = 0.0; if (tem) tem[i] = 0.0; }
    // 3. ghost ptype 1..8 (:207-235)
    for (int i = 0; i < ni; ++i) ptype[i] = 0;
    for (int i = ni; i < nf; ++i) {
        rho[i] = p->rho_ref;
        int t;
        if (y[i] < y_min) { t = 1; if (x[i] < x_min) t = 5; if (x[i] > x_max) t = 6; }
        else if (y[i] > y_max) { t = 2; if (x[i] < x_min) t = 7; if (x[i] > x_max) t = 8; }
        else if (x[i] < x_min) t = 3;
        else if (x[i] > x_max) t = 4;
        else { if (msg) *msg = "setup_closed_box: unclassified ghost particle"; return LSSPH_E_BAD_PARAM; }
        ptype[i] = t;
    }
    // 4. initial conditions (impose_initial_conditions_mod.f90)
    if (p->target_problem == 1) {
        for (int i = 0; i < nf; ++i) { rho[i] = p->rho_ref; u[i] = 0.0; pre[i] = 0.0; v[i] = 0.0; }
        SplitMix64 rng{p->seed};
        for (int i = 0; i < ni; ++i) {
            double r = rng.uniform();
            x[i] = x[i] + (p->pos_pert * p->dx) * (2.0 * r - 1.0);
            r = rng.uniform();
            y[i] = y[i] + (p->pos_pert * p->dx) * (2.0 * r - 1.0);
        }
        if (p->periodic) {   // free decay of sin(2 pi x) sin(2 pi y), rate 8 pi^2
            for (int i = 0; i < ni; ++i)
                u[i] = std::sin(((2.0 * kPi) * x[i]) / p->len_x) * std::sin(((2.0 * kPi) * y[i]) / p->len_y);
        }
    } else if (p->target_problem == 2) {
        const double a = (double)p->tg_a, b = (double)p->tg_b, Lx = p->len_x, Ly = p->len_y;
        const double ratio = (a * Ly) / (b * Lx);
        for (int i = 0; i < ni; ++i) {
            const double xx = x[i] - p->WL_thick, yy = y[i] - p->WL_thick;
            u[i] = (1.0 * std::sin(((a * kPi) * xx) / Lx)) * std::cos(((b * kPi) * yy) / Ly);
            v[i] = ((-1.0 * ratio) * std::cos(((a * kPi) * xx) / Lx)) * std::sin(((b * kPi) * yy) / Ly);
            pre[i] = ((0.25 * p->rho_ref) * 1.0) *
                     (std::cos((((2.0 * a) * kPi) * xx) / Lx) + (ratio * ratio) * std::cos((((2.0 * b) * kPi) * yy) / Ly));
            rho[i] = p->rho_ref + pre[i] / (p->sound_speed * p->sound_speed);
        }
    } else {
        for (int i = 0; i < nf; ++i) { rho[i] = p->rho_ref; pre[i] = 0.0; u[i] = 0.0; v[i] = 0.0; }
        if (p->target_problem == 4) {
            for (int i = 0; i < ni; ++i) {
                const double xx = x[i] - p->WL_thick, yy = y[i] - p->WL_thick;
                tem[i] = -(p->delta_tem / p->len_y) * yy + p->tem_bottom;
                if (yy <= 0.1 * p->len_y) tem[i] = tem[i] + (1.0e-2 * p->delta_tem) * std::cos((kPi * xx) / p->len_x);
            }
        }
    }
    return LSSPH_OK;
}

int build_virtual_markers(const lssph_params* p, int num_total, int num_int, const int32_t* ptype,
                          const double* x, const double* y, VirtualMarkers* vm, std::string* msg) {
    const int ne = num_total - num_int;
    vm->ptype.assign(ne, 0);
    vm->x.assign(ne, 0.0); vm->y.assign(ne, 0.0); vm->nx.assign(ne, 0.0); vm->ny.assign(ne, 0.0);
    const double x_min = 0.0 + p->WL_thick, x_max = p->len_x + p->WL_thick;
    const double y_min = 0.0 + p->WL_thick, y_max = p->len_y + p->WL_thick;
    const double r2 = 1.0 / std::sqrt(2.0);
    for (int me = 0; me < ne; ++me) {
        const int you = num_int + me;
        const int t = ptype[you];
        double vx = x[you], vy = y[you], nx = 0.0, ny = 0.0;
        switch (t) {
            case 1: vy = 2.0 * y_min - y[you]; ny = -1.0; break;
            case 2: vy = 2.0 * y_max - y[you]; ny = 1.0; break;
            case 3: vx = 2.0 * x_min - x[you]; nx = -1.0; break;
            case 4: vx = 2.0 * x_max - x[you]; nx = 1.0; break;
            case 5: vx = 2.0 * x_min - x[you]; vy = 2.0 * y_min - y[you]; nx = -r2; ny = -r2; break;
            case 6: vx = 2.0 * x_max - x[you]; vy = 2.0 * y_min - y[you]; nx = r2; ny = -r2; break;
            case 7: vx = 2.0 * x_min - x[you]; vy = 2.0 * y_max - y[you]; nx = -r2; ny = r2; break;
            case 8: vx = 2.0 * x_max - x[you]; vy = 2.0 * y_max - y[you]; nx = r2; ny = r2; break;
            default:
                if (msg) *msg = "init_virtual_markers: ghost particle with ptype outside 1..8";
                return LSSPH_E_BAD_PARAM;
        }
        vm->ptype[me] = t; vm->x[me] = vx; vm->y[me] = vy; vm->nx[me] = nx; vm->ny[me] = ny;
    }
    return LSSPH_OK;
}

int build_cell_grid(const lssph_params* p, int num_total, int num_int, const double* x,
                    const double* y, const VirtualMarkers& vm, CellGrid* g, std::string* msg) {
    const double xm = p->len_x + 2.0 * p->WL_thick, ym = p->len_y + 2.0 * p->WL_thick;
    g->nx = (int)std::ceil(xm / p->h_eff);
    g->ny = (int)std::ceil(ym / p->h_eff);
    g->ncell = g->nx * g->ny;
    const int ne = num_total - num_int;
    std::vector<int> count(g->ncell, 0);
    if (p->periodic) {   // an even number of cells of width L / n >= h_eff per side
        const int n = 2 * (int)std::floor(p->len_x / (2.0 * p->h_eff));
        if (n < 4) {
            if (msg) *msg = "a periodic domain needs at least 4 cells of h_eff per side";
            return LSSPH_E_BAD_PARAM;
        }
        g->nx = g->ny = n;
        g->ncell = n * n;
        g->inv_cw = 1.0 / (p->len_x / (double)n);
    }
    auto key_div = [&](double px, double py, int* key) {
        double cxd = std::ceil(px / p->h_eff), cyd = std::ceil(py / p->h_eff);
        if (p->periodic) {   // positions in (0, L], rounding at the ends clamped
            if (!(px > 0.0 && px <= p->len_x && py > 0.0 && py <= p->len_y)) return false;
            cxd = std::min(std::max(std::ceil(px * g->inv_cw), 1.0), (double)g->nx);
            cyd = std::min(std::max(std::ceil(py * g->inv_cw), 1.0), (double)g->ny);
        }
        if (!(cxd >= 1.0 && cxd <= g->nx && cyd >= 1.0 && cyd <= g->ny)) return false;
        *key = ((int)cxd - 1) + ((int)cyd - 1) * g->nx;
        return true;
    };
    g->ghost_key.assign(ne, 0);
    g->vm_key.assign(ne, 0);
    for (int me = 0; me < num_total; ++me) {   // init_cell_mod.f90:72-88
        int key;
        if (!key_div(x[me], y[me], &key)) {
            if (msg) *msg = "init_cell: particle outside the cell grid";
            return LSSPH_E_OUT_OF_DOMAIN;
        }
        count[key] += 1;
        if (me >= num_int) g->ghost_key[me - num_int] = key;
    }
    g->capacity = *std::max_element(count.begin(), count.end());
    // Slot capacity: the reference allocates 2*capacity per cell (init_cell_mod.f90:99);
    // rounded up to a multiple of 4 for aligned slot rows.
    g->cap = ((2 * g->capacity + 3) / 4) * 4;
    if (g->cap < 8) g->cap = 8;
    if (g->cap > 64) {
        if (msg) *msg = "cell capacity above 64 particles per cell is not supported";
        return LSSPH_E_UNSUPPORTED;
    }
    g->gstart.assign(g->ncell + 1, 0);
    for (int me = 0; me < ne; ++me) g->gstart[g->ghost_key[me] + 1] += 1;
    for (int c = 0; c < g->ncell; ++c) g->gstart[c + 1] += g->gstart[c];
    g->glist.assign(ne, 0);
    std::vector<int> fill(g->gstart.begin(), g->gstart.end() - 1);
    for (int me = 0; me < ne; ++me) g->glist[fill[g->ghost_key[me]]++] = num_int + me;   // :105-109
    for (int me = 0; me < ne; ++me) {   // :166-180
        int key;
        if (!key_div(vm.x[me], vm.y[me], &key)) {
            if (msg) *msg = "init_cell: virtual marker outside the cell grid";
            return LSSPH_E_OUT_OF_DOMAIN;
        }
        g->vm_key[me] = key;
    }
    return LSSPH_OK;
}

// Fortran `e21.14`: [sign]0.ddddddddddddddE+ee right-justified in 21 columns.
std::string fortran_e21_14(double v) {
    char buf[64];
    if (std::isnan(v)) return std::string(18, ' ') + "NaN";
    if (std::isinf(v)) return std::string(v < 0 ? 17 : 18, ' ') + (v < 0 ? "-Inf" : "Inf");
    std::string digits;
    int exp10 = 0;
    if (v == 0.0) {
        digits = std::string(14, '0');
    } else {
        std::snprintf(buf, sizeof(buf), "%.13E", std::fabs(v));   // d.ddddddddddddd E+xx
        std::string s(buf);
        const size_t epos = s.find('E');
        digits = s.substr(0, 1) + s.substr(2, epos - 2);
        exp10 = std::atoi(s.c_str() + epos + 1) + 1;
    }
    std::string out = (std::signbit(v) && v != 0.0) ? "-" : "";
    out += "0." + digits;
    const int ae = std::abs(exp10);
    if (ae <= 99) {
        std::snprintf(buf, sizeof(buf), "E%c%02d", exp10 < 0 ? '-' : '+', ae);
    } else {
        std::snprintf(buf, sizeof(buf), "%c%03d", exp10 < 0 ? '-' : '+', ae);
    }
    out += buf;
    if (out.size() < 21) out = std::string(21 - out.size(), ' ') + out;
    return out;
}

int make_dirs(const std::string& path) {
    std::string cur;
    for (size_t i = 0; i <= path.size(); ++i) {
        if (i == path.size() || path[i] == '/') {
            if (!cur.empty() && cur != "/" && mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST) return LSSPH_E_IO;
        }
        if (i < path.size()) cur.push_back(path[i]);
    }
    return LSSPH_OK;
}

int copy_file(const std::string& from, const std::string& to) {
    std::ifstream in(from, std::ios::binary);
    if (!in) return LSSPH_E_IO;
    std::ofstream out(to, std::ios::binary | std::ios::trunc);
    if (!out) return LSSPH_E_IO;
    out << in.rdbuf();
    return out.good() ? LSSPH_OK : LSSPH_E_IO;
}

int write_data_file(const std::string& path, int n, bool with_tem, const int32_t* ptype,
                    const double* x, const double* y, const double* u, const double* v,
                    const double* rho, const double* pre, const double* tem, std::string* msg) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) { if (msg) *msg = "cannot open " + path; return LSSPH_E_IO; }
    bool ok = std::fwrite(ptype, sizeof(int32_t), n, f) == (size_t)n;
    for (const double* a : {x, y, u, v, rho, pre}) ok = ok && std::fwrite(a, sizeof(double), n, f) == (size_t)n;
    if (with_tem) ok = ok && std::fwrite(tem, sizeof(double), n, f) == (size_t)n;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) { if (msg) *msg = "short write to " + path; return LSSPH_E_IO; }
    return LSSPH_OK;
}

int write_parameters_csv(const std::string& path, const lssph_params* p, int num_total, int num_int,
                         int num_ext, std::string* msg) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) { if (msg) *msg = "cannot open " + path; return LSSPH_E_IO; }
    auto I = [&](const char* k, long v) { std::fprintf(f, "%s,%ld\n", k, v); };
    auto E = [&](const char* k, double v) { std::fprintf(f, "%s,%s\n", k, fortran_e21_14(v).c_str()); };
    std::fprintf(f, "Parameter, Value\n");
    I("target_problem", p->target_problem);
    E("u_top", p->u_top); E("tem_top", p->tem_top); E("tem_bottom", p->tem_bottom);
    E("tem_left", p->tem_left); E("tem_right", p->tem_right);
    E("len_x", p->len_x); E("len_y", p->len_y);
    I("num_x", p->num_x); I("num_y", p->num_y);
    I("start_step", p->start_step); I("end_step", p->end_step); I("write_step", p->write_step);
    E("threshold", p->threshold); E("coe_CFL", p->coe_CFL); E("coe_dif", p->coe_dif);
    E("zeta_RSST", p->zeta_RSST); E("xi_VIM", p->xi_VIM);
    E("rho_ref", p->rho_ref); E("vis_ref", p->vis_ref); E("K_ref", p->K_ref);
    E("k_th_ref", p->k_th_ref); E("cp_ref", p->cp_ref); E("alpha_ref", p->alpha_ref);
    E("gravity", p->gravity); E("pos_pert", p->pos_pert);
    I("tg_a", p->tg_a); I("tg_b", p->tg_b);
    E("coe_h", p->coe_h); E("PST_c", p->PST_c); E("coe_delta_sph", p->coe_delta_sph);
    I("kernel_type", p->kernel_type); I("sph_model", p->sph_model); I("wall_model", p->wall_model);
    I("total_step", p->total_step);
    E("dx", p->dx); E("SP_mass", p->SP_mass); E("h", p->h); E("h_eff", p->h_eff); E("W_ave", p->W_ave);
    I("num_WL", p->num_WL);
    E("WL_thick", p->WL_thick); E("delta_tem", p->delta_tem); E("tem_ave", p->tem_ave);
    E("sound_speed", p->sound_speed); E("kinematic_vis", p->kinematic_vis); E("thermal_dif", p->thermal_dif);
    E("Re", p->Re); E("Ra", p->Ra); E("Pr", p->Pr);
    E("dt_CFL", p->dt_CFL); E("dt_vis", p->dt_vis); E("dt_th", p->dt_th);
    E("dt_CFL_relax", p->dt_CFL_relax); E("dt_vis_relax", p->dt_vis_relax); E("dt", p->dt);
    I("num_total", num_total); I("num_int", num_int); I("num_ext", num_ext);
    const bool ok = std::fclose(f) == 0;
    if (!ok) { if (msg) *msg = "write failed: " + path; return LSSPH_E_IO; }
    return LSSPH_OK;
}

}  // namespace lssph

// =====================================================================================
// C ABI: parameters, setup and file I/O (no device work)
// =====================================================================================
using namespace lssph;

extern "C" {

int lssph_abi_version(void) { return LSSPH_ABI_VERSION; }

size_t lssph_params_sizeof(void) { return sizeof(lssph_params); }

const char* lssph_last_error(void) { return last_error().c_str(); }

const char* lssph_status_string(int s) {
    switch (s) {
        case LSSPH_OK: return "ok";
        case LSSPH_E_BAD_PARAM: return "bad parameter";
        case LSSPH_E_CUDA: return "CUDA error";
        case LSSPH_E_CELL_OVERFLOW: return "cell list overflow";
        case LSSPH_E_OUT_OF_DOMAIN: return "particle outside the cell grid";
        case LSSPH_E_NONFINITE: return "non-finite value in the state";
        case LSSPH_E_SINGULAR: return "singular moment matrix";
        case LSSPH_E_IO: return "I/O error";
        case LSSPH_E_CAPACITY: return "buffer too small";
        case LSSPH_E_TIMEOUT: return "device wait timed out";
        case LSSPH_E_UNSUPPORTED: return "unsupported option";
        default: return "unknown status";
    }
}

int lssph_params_default(lssph_params* out) {
    if (!out) { set_last_error("null params"); return LSSPH_E_BAD_PARAM; }
    default_params(out);
    return LSSPH_OK;
}

int lssph_params_from_config(const char* path, lssph_params* out) {
    if (!path || !out) { set_last_error("null argument"); return LSSPH_E_BAD_PARAM; }
    std::string msg;
    const int rc = parse_config(path, out, &msg);
    if (rc != LSSPH_OK) set_last_error(msg);
    return rc;
}

int lssph_init_param(lssph_params* p) {
    if (!p) { set_last_error("null params"); return LSSPH_E_BAD_PARAM; }
    init_param(p);
    return LSSPH_OK;
}

int lssph_check_param(const lssph_params* p) {
    if (!p) { set_last_error("null params"); return LSSPH_E_BAD_PARAM; }
    std::string msg;
    const int rc = check_param(p, &msg);
    if (rc != LSSPH_OK) set_last_error(msg);
    return rc;
}

int lssph_setup_counts(const lssph_params* p, int32_t* num_total, int32_t* num_int) {
    if (!p || !num_total || !num_int) { set_last_error("null argument"); return LSSPH_E_BAD_PARAM; }
    int nt, ni;
    closed_box_counts(p, &nt, &ni);
    *num_total = nt;
    *num_int = ni;
    return LSSPH_OK;
}

int lssph_setup_particles(const lssph_params* p, int32_t num_total, int32_t* ptype, double* x,
                          double* y, double* u, double* v, double* rho, double* pre, double* tem) {
    if (!p || !ptype || !x || !y || !u || !v || !rho || !pre) { set_last_error("null argument"); return LSSPH_E_BAD_PARAM; }
    std::string msg;
    const int rc = setup_particles(p, num_total, ptype, x, y, u, v, rho, pre, tem, &msg);
    if (rc != LSSPH_OK) set_last_error(msg);
    return rc;
}

int lssph_write_parameters(const lssph_params* p, int32_t num_total, int32_t num_int, const char* path) {
    if (!p || !path) { set_last_error("null argument"); return LSSPH_E_BAD_PARAM; }
    std::string msg;
    const int rc = write_parameters_csv(path, p, num_total, num_int, num_total - num_int, &msg);
    if (rc != LSSPH_OK) set_last_error(msg);
    return rc;
}

int lssph_read_data(const char* path, int32_t n, int32_t with_tem, int32_t* ptype, double* x,
                    double* y, double* u, double* v, double* rho, double* pre, double* tem) {
    FILE* f = path ? std::fopen(path, "rb") : nullptr;
    if (!f) { set_last_error(std::string("cannot open ") + (path ? path : "(null)")); return LSSPH_E_IO; }
    bool ok = std::fread(ptype, sizeof(int32_t), n, f) == (size_t)n;
    for (double* a : {x, y, u, v, rho, pre}) ok = ok && std::fread(a, sizeof(double), n, f) == (size_t)n;
    if (with_tem) ok = ok && tem && std::fread(tem, sizeof(double), n, f) == (size_t)n;
    std::fclose(f);
    if (!ok) { set_last_error(std::string("short read from ") + path); return LSSPH_E_IO; }
    return LSSPH_OK;
}

}  // extern "C"
